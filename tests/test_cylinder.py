# -*- coding: utf-8 -*-
"""Cylinder-in-crossflow pieces on CPU: the O-grid mesh (interfaces close,
boundaries lie on the two circles), the boundary expressions of the
cylinder wall, and the oracle's cylinder wall against its plain diffuse
wall (frfs/solvers/dgfs/inters.py:446-492 is a diffuse wall whose state may
vary along it; with a constant state the two must agree, the wall
Maxwellian's normalisation cancelling in the flux ratio)."""

import numpy as np
import pytest

from helpers import config, dg_setup
from frfs_b200 import mesh as mgen
from frfs_b200.initcond import cylinder_wall_states, eval_point_expr
from frfs_b200.velocitymesh import DGFSVelocityMesh


@pytest.mark.parametrize('order', [1, 3])
def test_ogrid_closes_and_bounds(order):
    from frfs_b200.elements import ElementGeometry
    from frfs_b200.shapes import QuadShape
    m = mgen.quad_ogrid(10, 3, 0.5, 4.0, stretch=1.4)
    sh = QuadShape(order)
    geo = ElementGeometry(sh, m['spt_quad_p0'])
    assert geo.djac_at(sh.upts).min() > 0
    srtd, ploc, nrm = geo.srtd_face_fpts, geo.plocfpts, geo.norm_pnorm_fpts
    seen = np.zeros((sh.nfpts, geo.neles), bool)
    lhs, rhs = m['con_p0']
    for l, r in zip(lhs, rhs):
        for jl, jr in zip(srtd[l['fidx']][l['eidx']], srtd[r['fidx']][r['eidx']]):
            el, er = l['eidx'], r['eidx']
            assert np.allclose(ploc[jl, el], ploc[jr, er], atol=1e-12)
            assert np.allclose(nrm[jl, el], -nrm[jr, er], atol=1e-12)
            seen[jl, el] = seen[jr, er] = True
    radii = {'cylinder': 0.5, 'inflow': 4.0, 'outflow': 4.0}
    for name, rad in radii.items():
        for rec in m[f'bcon_{name}_p0']:
            js = srtd[rec['fidx']][rec['eidx']]
            # inflow faces: the upstream half (face centre at x <= 0)
            xc = np.mean([ploc[j, rec['eidx']][0] for j in js])
            if name == 'inflow':
                assert xc < 1e-12
            elif name == 'outflow':
                assert xc > -1e-12
            for j in js:
                p = ploc[j, rec['eidx']]
                # straight-sided faces: the face's end points lie on the circle
                assert np.linalg.norm(p) <= rad + 1e-12
                assert np.linalg.norm(p) >= rad*np.cos(np.pi/10) - 1e-12
                # outward normal of the domain: into the cylinder, out of
                # the far field
                sgn = np.dot(nrm[j, rec['eidx']], p)
                assert sgn < 0 if name == 'cylinder' else sgn > 0
                seen[j, rec['eidx']] = True
    assert seen.all()


def test_wall_expressions():
    cfg = config('relax0d-n16')
    vm = DGFSVelocityMesh(None, cfg)
    sect = 'soln-bcs-cyl'
    cfg.set(sect, 'type', 'dgfs-wall-diffuse-cyl')
    cfg.set(sect, 'ux', '-omega*y')
    cfg.set(sect, 'uy', 'omega*x')
    cfg.set(sect, 'uz', '0')
    cfg.set(sect, 'T', '273*(1 + 0.1*sqrt(x*x + y*y))')
    cfg.set('constants', 'omega', '50.0')
    x, y = np.array([0.3, -0.1]), np.array([0.4, 0.2])
    w = cylinder_wall_states(cfg, vm, sect, x, y)
    assert np.allclose(w[:, 0], -50*y/vm.u0()) and np.allclose(w[:, 1], 50*x/vm.u0())
    assert np.allclose(w[:, 3], 273*(1 + 0.1*np.hypot(x, y))/vm.T0())
    cfg.set(sect, 'uz', '__import__')
    with pytest.raises(ValueError):
        eval_point_expr(cfg, sect, 'uz', x, y)


def _cfg(kind):
    cfg = config('relax0d-n16')
    cfg.set('solver', 'order', 2)
    u0 = DGFSVelocityMesh(None, cfg).u0()
    for name in ('bottom', 'top'):
        sect = f'soln-bcs-{name}'
        cfg.set(sect, 'type', kind)
        cfg.set(sect, 'rho', 1.5e-3)
        cfg.set(sect, 'T', 300.0 if name == 'top' else 250.0)
        cfg.set(sect, 'ux', 0.2*u0)
        cfg.set(sect, 'uy', 0.0)
        cfg.set(sect, 'uz', 0.0)
    return cfg


def test_cylinder_wall_with_constant_state_is_the_diffuse_wall():
    m = mgen.quad_box(3, 2, 0.0, 1.0, 0.0, 0.5, periodic_x=True, jitter=0.2,
                      seed=5)
    rng = np.random.default_rng(1)
    out = []
    for kind in ('dgfs-wall-diffuse', 'dgfs-wall-diffuse-cyl'):
        dg, sh, geo, vm = dg_setup(_cfg(kind), m)
        if not out:
            u = rng.uniform(0.5, 1.5, (sh.nupts, vm.vsize(), geo.neles))
        uf = dg.disu(u)
        dg.update_bc(uf)
        out.append(dg.rhs(u, uf))
    assert np.max(np.abs(out[0] - out[1])) < 1e-12*np.max(np.abs(out[0]))
