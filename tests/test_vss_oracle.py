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


def test_single_species_alpha1_reduces_to_vhs():
    """With one species, alpha = 1 and the direction integrals of the gain
    and loss kernels taken analytically (the VHS kernels' sinc forms,
    vhs-gll.mako:11-14 and 84-97), the VSS operator is the VHS operator of
    the (reference-pinned) VHS oracle on the same grid: the phases
    exp(+-i a/2), the weights over the full sphere (twice the half-sphere
    sum at the same sw), the prefactor (sqrt(1 + mp/mq) cancels, mu = 1/2)
    and the loss term agree.  Only the numerical direction integrals of
    b and c (vss-gll.mako:73-91) are left out, and they are checked
    separately against their limit."""
    from oracle import vhs as ovhs
    Nv, Nrho, M = 16, 8, 6
    half = load_sphdesign(M)[:M]
    full = np.vstack([half, -half])
    mm, H0, T0, rho0 = 39.96e-3, 1e-3, 273.0, 1.5e-3
    mesh = vss.mixture_mesh(Nv, Nrho, full, [mm], H0=H0, T0=T0, rho0=rho0,
                            molarMass0=mm, cmax=0.0, Tmax=T0, dev=5.0)
    omega, dRef = 0.81, 4.17e-10
    params = vss.vss_parameters(mesh, alpha={'00': 1.0},
                                omega={'00': omega}, dRef={'00': dRef},
                                Tref={'00': T0})
    pre = vss.vss_precompute(mesh, params, full)
    vm = ovhs.velocity_mesh(Nv, Nrho, M, np.vstack([half, -half]), H0, T0,
                            rho0, mm, 0.0, T0, 5.0)
    gam, prefac = ovhs.vhs_parameters(omega, dRef, T0, H0, vm['n0'], T0)
    assert params['00']['gamma'] == gam
    assert params['00']['prefac'] == pytest.approx(prefac, rel=1e-14)
    for k in ('L', 'R'):
        assert mesh[k] == pytest.approx(vm[k], rel=1e-15)
    vpre = ovhs.vhs_precompute(vm, gam)

    # the direction integrals against their limit: the full-sphere design's
    # sum of exp(-i k s.l) approaches 4 pi sinc(k |l|) where k |l| is small
    # (below 0.5, the whole grid at the innermost radial node: 9e-8)
    L, qz, qw = mesh['L'], mesh['qz'], mesh['qw']
    lmag = np.sqrt(np.sum(vpre['l']**2, axis=0))
    small = lmag*np.pi/L*qz[0]/2 < 0.5
    b_exact = np.array([qz[x]**(gam + 2)*4*np.pi *
                        ovhs._sinc(np.pi/L*qz[x]/2*lmag)
                        for x in range(Nrho)])
    b_num = pre['00']['b']
    np.testing.assert_allclose(b_num[0][:, small].real,
                               np.broadcast_to(b_exact[0][small],
                                               b_num[0][:, small].shape),
                               rtol=1e-6)
    assert np.max(np.abs(b_num[0][:, small].imag)) < 1e-12*np.max(b_exact[0])
    # analytic kernels in place of the numerical ones
    pre['00']['b'] = np.broadcast_to(b_exact[:, None, :],
                                     b_num.shape).astype(np.complex128)
    pre['00']['c'] = np.sum([qw[x]*qz[x]**(gam + 2)*16*np.pi**2 *
                             ovhs._sinc(np.pi/L*qz[x]*lmag)
                             for x in range(Nrho)], axis=0).astype(
                                 np.complex128)
    np.testing.assert_allclose(b_exact, vpre['bb1'], rtol=1e-14)
    np.testing.assert_allclose(pre['00']['c'].real, vpre['bb2'], rtol=0,
                               atol=1e-13*np.max(np.abs(vpre['bb2'])))

    f = 0.5*(ovhs.maxwellian(vm['cv'], 1.0, [0.7, -0.2, 0.1], 0.8) +
             ovhs.maxwellian(vm['cv'], 1.0, [-0.6, 0.3, 0.0], 1.1))
    Qv = ovhs.vhs_Q(f, vm, vpre, prefac)
    Qs = vss.vss_Q([f], mesh, pre, params)[0]
    assert np.max(np.abs(Qs - Qv)) < 1e-11*np.max(np.abs(Qv))
