# -*- coding: utf-8 -*-
"""Structured quadrilateral meshes in frfs's mesh dictionary form.

frfs reads meshes as a dict of arrays (frfs/readers/base.py:19-244):
``spt_<etype>_p0`` shape (nspts, neles, ndims) with the shape points in the
element's standard order, ``con_p0`` holding the left and right sides of every
internal interface as (etype, element, face, flags) records, and
``bcon_<name>_p0`` the (etype, element, face, flags) records of boundary
region <name>.  This module generates the same dictionary for straight-sided
quadrilateral boxes and strips and for O-grids around a cylinder;
periodic directions are closed by internal interfaces, as frfs's importer
does for periodic boundary pairs.

Quadrilateral faces follow frfs/shapes.py:QuadShape.faces: 0 bottom
(eta = -1), 1 right (xi = 1), 2 top (eta = 1), 3 left (xi = -1); shape
points are ordered x fastest (frfs/shapes.py:TensorProdShape.std_ele).
"""

import numpy as np

_REC = np.dtype([('etype', 'U4'), ('eidx', 'i4'), ('fidx', 'i1'),
                 ('flags', 'i1')])


def quad_box(nx, ny, xlo, xhi, ylo, yhi, periodic_x=False, periodic_y=False,
             names=('bottom', 'right', 'top', 'left'), jitter=0.0, seed=0):
    """nx*ny straight-sided quads (element e = i + nx*j).  ``jitter`` moves
    interior nodes by up to that fraction of the cell size (seeded), giving
    non-affine elements for testing the metric terms."""
    xs = np.linspace(xlo, xhi, nx + 1)
    ys = np.linspace(ylo, yhi, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing='ij')
    if jitter:
        rng = np.random.default_rng(seed)
        hx, hy = (xhi - xlo)/nx, (yhi - ylo)/ny
        X[1:-1, 1:-1] += jitter*hx*rng.uniform(-1, 1, (nx - 1, ny - 1))
        Y[1:-1, 1:-1] += jitter*hy*rng.uniform(-1, 1, (nx - 1, ny - 1))
    neles = nx*ny
    spt = np.empty((4, neles, 2))
    for j in range(ny):
        for i in range(nx):
            e = i + nx*j
            spt[0, e] = (X[i, j], Y[i, j])
            spt[1, e] = (X[i + 1, j], Y[i + 1, j])
            spt[2, e] = (X[i, j + 1], Y[i, j + 1])
            spt[3, e] = (X[i + 1, j + 1], Y[i + 1, j + 1])

    lhs, rhs = [], []
    bcon = {n: [] for n in names}
    for j in range(ny):
        for i in range(nx):
            e = i + nx*j
            # right face (1) of (i, j) meets left face (3) of (i+1, j)
            if i + 1 < nx or periodic_x:
                lhs.append(('quad', e, 1, 0))
                rhs.append(('quad', (i + 1) % nx + nx*j, 3, 0))
            # top face (2) of (i, j) meets bottom face (0) of (i, j+1)
            if j + 1 < ny or periodic_y:
                lhs.append(('quad', e, 2, 0))
                rhs.append(('quad', i + nx*((j + 1) % ny), 0, 0))
            if j == 0 and not periodic_y:
                bcon[names[0]].append(('quad', e, 0, 0))
            if i == nx - 1 and not periodic_x:
                bcon[names[1]].append(('quad', e, 1, 0))
            if j == ny - 1 and not periodic_y:
                bcon[names[2]].append(('quad', e, 2, 0))
            if i == 0 and not periodic_x:
                bcon[names[3]].append(('quad', e, 3, 0))

    mesh = {'spt_quad_p0': spt,
            'con_p0': np.array([lhs, rhs], dtype=_REC)}
    for n, recs in bcon.items():
        if recs:
            mesh[f'bcon_{n}_p0'] = np.array(recs, dtype=_REC)
    return mesh


def quad_ogrid(ntheta, nr, r_in, r_out, stretch=1.0,
               names=('cylinder', 'inflow', 'outflow')):
    """Quadrilateral O-grid around a circle of radius r_in (the cylinder)
    out to r_out: ntheta elements around (closed by internal interfaces),
    nr across, radial sizes growing geometrically by ``stretch``.  Element
    e = i + ntheta j; i runs clockwise so that (xi, eta) = (clockwise,
    outward) is right-handed.  Straight-sided elements.  Boundary regions:
    names[0] the inner circle (face 0), and the outer circle (face 2) split
    into names[1] where the face midpoint has x < 0 (upstream of a flow
    along +x) and names[2] elsewhere."""
    if ntheta < 3 or nr < 1 or not 0 < r_in < r_out:
        raise ValueError('bad O-grid parameters')
    w = stretch**np.arange(nr)
    r = r_in + (r_out - r_in)*np.r_[0.0, np.cumsum(w)]/np.sum(w)
    th = -2*np.pi*np.arange(ntheta)/ntheta
    X = np.outer(np.cos(th), r)
    Y = np.outer(np.sin(th), r)
    neles = ntheta*nr
    spt = np.empty((4, neles, 2))
    for j in range(nr):
        for i in range(ntheta):
            e, ip = i + ntheta*j, (i + 1) % ntheta
            spt[0, e] = (X[i, j], Y[i, j])
            spt[1, e] = (X[ip, j], Y[ip, j])
            spt[2, e] = (X[i, j + 1], Y[i, j + 1])
            spt[3, e] = (X[ip, j + 1], Y[ip, j + 1])
    lhs, rhs = [], []
    bcon = {n: [] for n in names}
    for j in range(nr):
        for i in range(ntheta):
            e = i + ntheta*j
            lhs.append(('quad', e, 1, 0))
            rhs.append(('quad', (i + 1) % ntheta + ntheta*j, 3, 0))
            if j + 1 < nr:
                lhs.append(('quad', e, 2, 0))
                rhs.append(('quad', i + ntheta*(j + 1), 0, 0))
            if j == 0:
                bcon[names[0]].append(('quad', e, 0, 0))
            if j == nr - 1:
                xm = 0.5*(spt[2, e, 0] + spt[3, e, 0])
                bcon[names[1] if xm < 0 else names[2]].append(
                    ('quad', e, 2, 0))
    mesh = {'spt_quad_p0': spt,
            'con_p0': np.array([lhs, rhs], dtype=_REC)}
    for n, recs in bcon.items():
        if recs:
            mesh[f'bcon_{n}_p0'] = np.array(recs, dtype=_REC)
    return mesh


def from_config(cfg):
    """Mesh described by the ``[mesh]`` section of a workload config."""
    kind = cfg.get('mesh', 'type')
    if kind == 'quad-ogrid':
        return quad_ogrid(cfg.getint('mesh', 'ntheta'),
                          cfg.getint('mesh', 'nr'),
                          cfg.getfloat('mesh', 'r-in'),
                          cfg.getfloat('mesh', 'r-out'),
                          cfg.getfloat('mesh', 'stretch', 1.0))
    if kind not in ('quad-box', 'quad-strip'):
        raise ValueError(f'unsupported [mesh] type {kind!r}')
    g = lambda k, d=None: cfg.getfloat('mesh', k, d)
    names = ('bottom', 'right', 'top', 'left')
    if kind == 'quad-strip':
        names = ('bottom', 'right', 'top', 'left')
    return quad_box(cfg.getint('mesh', 'nx'), cfg.getint('mesh', 'ny'),
                    g('xlo'), g('xhi'), g('ylo'), g('yhi'),
                    periodic_x=cfg.getint('mesh', 'periodic-x', 0) == 1,
                    periodic_y=cfg.getint('mesh', 'periodic-y', 0) == 1,
                    names=names)
