# -*- coding: utf-8 -*-
"""Loader for tabulated symmetric spherical designs.

Reads the same files frfs ships under frfs/sphericaldesign/symmetric/
(``<rule>-ss<degree>-m<npts>.txt``, one ``x y z`` point per line) and applies
the same selection rule as frfs/sphericaldesign/__init__.py:56-107: among the
files of the requested rule name and point count, the one of highest degree.

Search order for the directory: the ``paths`` argument, then the
``DGFS_SPHDESIGN_PATH`` environment variable (os.pathsep separated), then
the tables shipped with this package (``data/sphericaldesign``: the
Womersley symmetric designs of frfs/sphericaldesign/symmetric that the
workloads use), then the ``frfs`` package if it is importable.
"""

import os
import re

import numpy as np

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data',
                        'sphericaldesign')
_PAT = re.compile(r'([a-zA-Z0-9\-~+]+)-ss(\d+)(?:-m(\d+))?\.txt$')


class SphericalRule:
    def __init__(self, pts, path):
        self.pts = pts
        self.path = path


def _search_dirs(paths):
    dirs = list(paths or [])
    env = os.environ.get('DGFS_SPHDESIGN_PATH')
    if env:
        dirs += env.split(os.pathsep)
    dirs.append(DATA_DIR)
    try:
        import importlib.util
        spec = importlib.util.find_spec('frfs')
        if spec and spec.submodule_search_locations:
            for loc in spec.submodule_search_locations:
                dirs.append(os.path.join(loc, 'sphericaldesign', 'symmetric'))
    except (ImportError, ValueError):
        pass
    return [d for d in dirs if os.path.isdir(d)]


def get_sphquadrule(sstype='symmetric', rule=None, npts=None, paths=None):
    if sstype != 'symmetric':
        raise ValueError(f'unsupported spherical design type {sstype!r}')
    if not npts:
        raise ValueError('npts is required')
    best = None
    for d in _search_dirs(paths):
        for f in sorted(os.listdir(d)):
            m = _PAT.match(f)
            if not m:
                continue
            rname, rdeg, rn = m.group(1), int(m.group(2)), int(m.group(3) or -1)
            if (rule and rname != rule) or rn != npts:
                continue
            if best is None or rdeg > best[1]:
                best = (os.path.join(d, f), rdeg)
    if best is None:
        raise ValueError(f'No suitable spherical quadrature rule found '
                         f'(rule={rule}, npts={npts}); set '
                         f'DGFS_SPHDESIGN_PATH to a directory of '
                         f'<rule>-ssD-mNNNNN.txt tables')
    pts = np.loadtxt(best[0], dtype=np.float64, ndmin=2)
    if pts.shape != (npts, 3):
        raise ValueError(f'{best[0]}: expected {npts} points in 3D')
    return SphericalRule(pts, best[0])
