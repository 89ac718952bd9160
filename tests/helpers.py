# -*- coding: utf-8 -*-
"""Shared setup for the tests: workload configs, oracle instances, banks."""

import glob
import os

import numpy as np

from conftest import GOLDEN, SPHDESIGN
from frfs_b200 import workloads
from frfs_b200.inifile import Inifile
from oracle import vhs as ovhs


def config(name, precision='double', **kw):
    ini = workloads.WORKLOADS[name](precision=precision, **kw)
    cfg = Inifile(ini)
    cfg.set('spherical-design-rule', 'path', SPHDESIGN)
    return cfg


def small_config(precision='double', Nv=8, Nrho=4, M=6):
    cfg = config('channel-n32', precision, Nv=Nv, Nrho=Nrho, M=M)
    return cfg


def load_sphdesign(M):
    f = glob.glob(os.path.join(SPHDESIGN, f'*-m{2*M:05d}.txt'))
    assert f, f'no spherical design with {2*M} points in {SPHDESIGN}'
    return np.loadtxt(f[0])


def oracle_for(cfg):
    """Oracle velocity mesh, precomputation and prefactor for a config."""
    g = lambda s, k: cfg.getfloat(s, k)
    M = cfg.getint('spherical-design-rule', 'M')
    vm = ovhs.velocity_mesh(
        cfg.getint('constants', 'Nv'), cfg.getint('constants', 'Nrho'), M,
        load_sphdesign(M), g('non-dim', 'H0'), g('non-dim', 'T0'),
        g('non-dim', 'rho0'), g('non-dim', 'molarMass0'),
        g('velocity-mesh', 'cmax'), g('velocity-mesh', 'Tmax'),
        g('velocity-mesh', 'dev'))
    gam, prefac = ovhs.vhs_parameters(
        g('scattering-model', 'omega'), g('scattering-model', 'dRef'),
        g('scattering-model', 'Tref'), g('non-dim', 'H0'), vm['n0'],
        g('non-dim', 'T0'))
    pre = ovhs.vhs_precompute(vm, gam)
    return vm, pre, prefac


def golden(name):
    return np.load(os.path.join(GOLDEN, f'ref_vm_{name}.npz'))


def random_states(cv, npts, seed=0, noise=0.01):
    """A batch of positive distributions: bimodal Maxwellian mixtures with
    random moments, times (1 + noise xi)."""
    rng = np.random.default_rng(seed)
    out = np.empty((npts, cv.shape[1]))
    for i in range(npts):
        rho = rng.uniform(0.5, 2.0)
        T1, T2 = rng.uniform(0.5, 1.5, size=2)
        u = rng.uniform(-1.0, 1.0, size=(2, 3))*0.7
        w = rng.uniform(0.2, 0.8)
        f = rho*(w*ovhs.maxwellian(cv, 1.0, u[0], T1) +
                 (1 - w)*ovhs.maxwellian(cv, 1.0, u[1], T2))
        out[i] = f*(1 + noise*rng.standard_normal(cv.shape[1]))
    return out


def rel_err(a, b):
    """max |a - b| / max |b| (normwise relative error)."""
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) /
                 np.max(np.abs(np.asarray(b))))


def dg_setup(cfg, mesh):
    """Product-side operators/geometry (pinned to reference fixtures by
    test_geometry.py) and an oracle DG instance on the same mesh."""
    from frfs_b200.elements import ElementGeometry
    from frfs_b200.initcond import MaxwellianSection
    from frfs_b200.shapes import QuadShape
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    from oracle.dg import DGOracle

    sh = QuadShape(cfg.getint('solver', 'order'))
    geo = ElementGeometry(sh, mesh['spt_quad_p0'])
    vm = DGFSVelocityMesh(None, cfg)
    ops = {'M0': sh.opmat('M0'), 'M132': sh.opmat('M1 - M3*M2'),
           'M3': sh.opmat('M3')}
    g = {'smats': geo.smat_at(sh.upts), 'rcpdjac': geo.rcpdjac_at(sh.upts),
         'nrm': geo.norm_pnorm_fpts, 'mag': geo.mag_pnorm_fpts,
         'srtd': geo.srtd_face_fpts}
    lhs, rhs = mesh['con_p0']
    con = ([(int(r['eidx']), int(r['fidx'])) for r in lhs],
           [(int(r['eidx']), int(r['fidx'])) for r in rhs])
    bcons, bcs = {}, {}
    for k in mesh:
        if k.startswith('bcon_'):
            name = k[5:-3]
            bcons[name] = [(int(r['eidx']), int(r['fidx'])) for r in mesh[k]]
            sect = f'soln-bcs-{name}'
            btype = cfg.get(sect, 'type')
            if btype in ('dgfs-wall-diffuse', 'dgfs-inlet',
                         'dgfs-inlet-normalshock'):
                ms = MaxwellianSection(cfg, vm, sect)
                bcs[name] = {'type': btype, 'fw': ms.values, 'uw': ms.u}
            else:
                bcs[name] = {'type': btype, 'fw': None, 'uw': np.zeros(3)}
    dg = DGOracle(ops, g, con, bcons, vm.cv(), vm.cw(), bcs)
    # cylinder walls: the config's wall expressions at the region's flux
    # points (host-side input, evaluated by the product's expression reader)
    from frfs_b200.initcond import cylinder_wall_states
    for name, bc in bcs.items():
        if bc['type'] == 'dgfs-wall-diffuse-cyl':
            xy = np.array([geo.plocfpts[j, e] for j, e in dg.bpts[name]])
            bc['w'] = cylinder_wall_states(cfg, vm, f'soln-bcs-{name}',
                                           xy[:, 0], xy[:, 1])
    return dg, sh, geo, vm
