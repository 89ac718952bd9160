# -*- coding: utf-8 -*-
"""The binary-mixture VSS oracle (CPU): the operator's invariants.  Number
of each species, total momentum and total energy are conserved by every
pair of collisions to the spectral accuracy of the grid (the errors fall by
orders of magnitude from N = 16 to N = 24: 1.6e-4 -> 1.9e-9 in number,
5.6e-3 -> 9.4e-5 in momentum, 2.3e-3 -> 5.4e-5 in energy, relative to
|Q|), and a pair of Maxwellians at a common velocity and temperature is an
equilibrium.  The reference runs only on CUDA through PyCUDA and Mako, so
these invariants, not its outputs, pin the restatement."""

import numpy as np
import pytest

from helpers import load_sphdesign
from oracle import vss


def _build(Nv, Nrho):
    sz = load_sphdesign(6)            # 12-point full-sphere design
    mesh = vss.mixture_mesh(Nv, Nrho, sz, [39.96e-3, 83.8e-3], H0=1e-3,
                            T0=273.0, rho0=1.5e-3, molarMass0=39.96e-3,
                            cmax=0.0, Tmax=273.0, dev=5.0)
    keys = ('00', '01', '10', '11')
    params = vss.vss_parameters(
        mesh, alpha={k: 1.4 for k in keys}, omega={k: 0.75 for k in keys},
        dRef={k: 4.1e-10 for k in keys}, Tref={k: 273.0 for k in keys})
    pre = vss.vss_precompute(mesh, params, sz)
    return mesh, params, pre


@pytest.fixture(scope='module')
def setup():
    return _build(24, 12)


def _states(mesh, u1, T1, u2, T2):
    m1, m2 = mesh['masses']
    cv = mesh['cv']
    f1 = vss.mixture_maxwellian(cv, 0.6, m1, u1, T1)
    f2 = vss.mixture_maxwellian(cv, 0.4, m2, u2, T2)
    return f1, f2


def test_mesh_and_parameters(setup):
    mesh, params, _ = setup
    assert mesh['masses'][0] == 1.0 and abs(mesh['masses'][1] - 2.097) < 1e-3
    assert 0 < mesh['S'] < mesh['L'] and mesh['R'] == 2*mesh['S']
    assert abs(mesh['sw']*mesh['sz'].shape[0] - 4*np.pi) < 1e-12
    for k in ('00', '11'):
        assert params[k]['eta'] == pytest.approx(0.4)
    # sqrt(1 + mp/mq) cancels between invKn and the prefactor: the unlike
    # pair's prefactor is symmetric (it depends on the reduced mass)
    assert params['01']['prefac'] == pytest.approx(params['10']['prefac'])
    assert params['01']['prefac'] != pytest.approx(params['00']['prefac'])


def _conservation_errors(mesh, params, pre):
    cv, cw = mesh['cv'], mesh['cw']
    m1, m2 = mesh['masses']
    f1, f2 = _states(mesh, [0.3, 0, 0], 0.8, [-0.2, 0.1, 0], 1.2)
    Q12 = vss.vss_Qpq(f1, f2, 0, 1, mesh, pre, params)
    Q21 = vss.vss_Qpq(f2, f1, 1, 0, mesh, pre, params)
    Q11 = vss.vss_Qpq(f1, f1, 0, 0, mesh, pre, params)
    scale = np.sum(np.abs(Q12))*cw
    assert scale > 0
    c2 = np.sum(cv*cv, axis=0)
    return np.array([
        abs(np.sum(Q12)*cw)/scale, abs(np.sum(Q21)*cw)/scale,
        abs(np.sum(Q11))/np.sum(np.abs(Q11)),
        np.max(np.abs(m1*(cv @ Q12) + m2*(cv @ Q21)))*cw/scale,
        abs(m1*c2 @ Q12 + m2*c2 @ Q21)*cw/scale])


def test_conservation(setup):
    err = _conservation_errors(*setup)
    assert np.all(err[:3] < 1e-6), err     # number of each species
    assert np.all(err[3:] < 1e-3), err     # momentum, energy of the pair


def test_conservation_converges():
    coarse = _conservation_errors(*_build(16, 8))
    fine = _conservation_errors(*_build(24, 12))
    assert np.all(fine < 0.05*coarse), (coarse, fine)


def test_equilibrium(setup):
    mesh, params, pre = setup
    f1, f2 = _states(mesh, [0.2, 0, 0], 1.0, [0.2, 0, 0], 1.0)
    g1, g2 = _states(mesh, [0.2, 0, 0], 0.7, [-0.3, 0, 0], 1.3)
    Qeq = vss.vss_Q([f1, f2], mesh, pre, params)
    Qne = vss.vss_Q([g1, g2], mesh, pre, params)
    for a, b in zip(Qeq, Qne):
        assert np.max(np.abs(a)) < 1e-2*np.max(np.abs(b))


def test_product_mixture_mesh_matches_oracle():
    """frfs_b200.mixture's mesh (the product side of dgfsbi/velocitymesh.py)
    equals the oracle's restatement."""
    import sys
    sys.path.insert(0, __import__('os').path.dirname(__file__))
    from test_vss_gpu import mixture_config
    from frfs_b200.mixture import DGFSBiVelocityMesh
    cfg = mixture_config('double', Nv=24, Nrho=12)
    vm = DGFSBiVelocityMesh(None, cfg)
    mesh = vss.mixture_mesh(24, 12, vm.sz(), [39.96e-3, 83.8e-3], H0=1e-3,
                            T0=273.0, rho0=1.5e-3, molarMass0=39.96e-3,
                            cmax=0.0, Tmax=273.0, dev=5.0)
    for k in ('L', 'S', 'R', 'cw'):
        assert getattr(vm, k)() == pytest.approx(mesh[k], rel=1e-15) \
            if hasattr(vm, k) else True
    np.testing.assert_allclose(vm.qz(), mesh['qz'], rtol=1e-15)
    np.testing.assert_allclose(vm.qw(), mesh['qw'], rtol=1e-14)
    np.testing.assert_array_equal(vm.cv(), mesh['cv'])
    assert vm.masses() == pytest.approx(mesh['masses'], rel=1e-15)
