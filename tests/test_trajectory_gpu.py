# -*- coding: utf-8 -*-
"""Whole trajectories of the B200 solver against the FP64 oracle (GPU).

The single-call parity tests check one collision or one residual; these run
the configurations the reference is compared on for many steps, through the
product's steppers (frfs/integrators/std/steppers.py:39-225), and compare
the distribution and its moments with the oracle's own stepper
(oracle/dg.py: ssp_rk2_step, euler_step) driving the restated collision
operator (oracle/vhs.py) and DG residual (oracle/dg.py) on the same mesh.

* space-homogeneous relaxation (N=16, Nrho=8, M=6, hard spheres): the two
  Maxwellians at u = (+-1.5, 0, 0), 50 SSP-RK2 steps of dt = 0.01, and the
  same with the Euler stepper; a uniform state on a doubly periodic single
  element, where the advection residual vanishes;
* the Couette slab (N=24, Nrho=12, M=16, omega=0.81) on a 4x1 strip with its
  moving diffuse walls, 2 SSP-RK2 steps.

Tolerance: 1e-10 normwise relative in FP64 (the parity bar of the collision
and residual tests), on f and on rho, u, T.
"""

import numpy as np
import pytest
import torch

from helpers import config, dg_setup, oracle_for, rel_err
from frfs_b200 import mesh as mgen
from frfs_b200.backend import B200Backend
from frfs_b200.steppers import StdEulerDGFSStepper, StdTVDRK2DGFSStepper
from frfs_b200.system import DGFSSystem
from oracle import dg as odg
from oracle import vhs as ovhs

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _moments(f, cv, cw):
    """rho, u, T of every point of a bank (nupts, V, neles), FP64."""
    rho = np.einsum('ive->ie', f)*cw
    u = np.einsum('ive,dv->die', f, cv)*cw/rho
    c2 = np.sum((cv[:, None, :, None] - u[:, :, None, :])**2, axis=0)
    T = (2.0/3.0)*np.einsum('ive,ive->ie', f, c2)*cw/rho
    return rho, u, T


def _collision(cfg, uniform=False):
    ovm, pre, prefac = oracle_for(cfg)

    def Q(x):
        out = np.empty_like(x)
        if uniform:
            # every point holds the same state (to round-off): one
            # evaluation, broadcast, is the oracle's answer at each
            q = ovhs.vhs_Q(x[0, :, 0], ovm, pre, prefac)
            out[:] = q[None, :, None]
            return out
        for i in range(x.shape[0]):
            for e in range(x.shape[2]):
                out[i, :, e] = ovhs.vhs_Q(x[i, :, e], ovm, pre, prefac)
        return out
    return Q


def _compare(s, bankidx, ref, vm):
    got = s.bank[bankidx].get()
    assert np.all(np.isfinite(got))
    assert rel_err(got, ref) < TOL, rel_err(got, ref)
    cv, cw = vm.cv(), vm.cw()
    mg, mr = _moments(got, cv, cw), _moments(ref, cv, cw)
    for name, a, b in zip(('rho', 'u', 'T'), mg, mr):
        scale = 1.0 if name == 'u' else np.max(np.abs(b))
        err = float(np.max(np.abs(a - b)))/scale
        assert err < TOL, f'{name}: {err:.3e}'


@pytest.mark.parametrize('stepper', [StdTVDRK2DGFSStepper,
                                     StdEulerDGFSStepper])
def test_relaxation_50_steps(stepper):
    """The space-homogeneous relaxation (N = 16): 50 steps of dt = 0.01
    in FP64."""
    cfg = config('relax0d-n16', 'double')
    m = mgen.quad_box(1, 1, 0.0, 1.0, 0.0, 1.0, periodic_x=True,
                      periodic_y=True)
    be = B200Backend(cfg, device='cuda:0')
    s = DGFSSystem(be, cfg, mesh=m)
    st = stepper(s, cfg)
    st.dt = 0.01
    u0 = s.bank[0].get().astype(np.float64)
    dg, sh, geo, vm = dg_setup(cfg, m)
    Q = _collision(cfg, uniform=True)
    step = odg.ssp_rk2_step if stepper is StdTVDRK2DGFSStepper \
        else odg.euler_step
    ref = u0
    for _ in range(50):
        ref = step(dg, Q, ref, 0.01)
    st.advance(50)
    torch.cuda.synchronize()
    _compare(s, st._idxcurr, ref, vm)
    # the run did relax: the temperature anisotropy of the initial state
    # has decayed (a check that 50 steps were taken, not the parity bar)
    f0, f1 = u0[0, :, 0], ref[0, :, 0]
    cx = vm.cv()[0]
    Txx = lambda f: np.sum(f*cx*cx)/np.sum(f)
    assert Txx(f1) < Txx(f0)


def test_couette_strip_two_steps():
    """The Couette workload's discretisation on a 4x1 strip: 2 SSP-RK2
    steps in FP64 with both moving diffuse walls."""
    cfg = config('couette-n24', 'double', nele=4)
    m = mgen.from_config(cfg)
    be = B200Backend(cfg, device='cuda:0')
    s = DGFSSystem(be, cfg, mesh=m)
    st = StdTVDRK2DGFSStepper(s, cfg)
    dt = 2e-3
    st.dt = dt
    u0 = s.bank[0].get().astype(np.float64)
    dg, sh, geo, vm = dg_setup(cfg, m)
    Q = _collision(cfg)
    ref = u0
    for _ in range(2):
        ref = odg.ssp_rk2_step(dg, Q, ref, dt)
    st.advance(2)
    torch.cuda.synchronize()
    _compare(s, st._idxcurr, ref, vm)
    # the walls moved the gas: the wall-adjacent points carry momentum
    assert np.max(np.abs(ref - u0)) > 1e-6*np.max(np.abs(u0))
