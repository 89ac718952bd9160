# -*- coding: utf-8 -*-
"""The CPU oracle against the reference's own outputs and invariants.

The golden fixtures were produced by running the reference's numpy code
(tests/golden/make_golden.py).  Exact equality is expected for the pieces the
oracle restates operation by operation.
"""

import numpy as np
import pytest

from helpers import config, golden, oracle_for, rel_err
from oracle import vhs as ovhs

CASES = ['small-n8', 'relax0d-n16', 'couette-n24', 'channel-n32']


def _cfg_for(name):
    if name == 'small-n8':
        return config('channel-n32', Nv=8, Nrho=4, M=6)
    return config(name)


@pytest.mark.parametrize('name', CASES)
def test_velocity_mesh_matches_reference(name):
    g = golden(name)
    vm, pre, prefac = oracle_for(_cfg_for(name))
    assert vm['L'] == g['L']
    assert vm['cw'] == g['cw']
    np.testing.assert_array_equal(vm['c0'], g['c0'])
    np.testing.assert_array_equal(vm['qz'], g['qz'])
    np.testing.assert_array_equal(vm['qw'], g['qw'])
    np.testing.assert_array_equal(vm['sz'], g['sz'])
    assert vm['sw'] == g['sw']
    if 'cv' in g:
        np.testing.assert_array_equal(vm['cv'], g['cv'])
    assert prefac == g['prefactor']


@pytest.mark.parametrize('name', ['couette-n24', 'channel-n32'])
def test_maxwellian_matches_reference(name):
    g = golden(name)
    vm, _, _ = oracle_for(_cfg_for(name))
    f0 = ovhs.maxwellian(vm['cv'], 1.0, [0, 0, 0], 1.0)
    np.testing.assert_array_equal(f0, g['f0'])
    for key in g.files:
        if key.startswith('fw_'):
            uy = {'left': -0.5, 'right': 0.5}.get(key[3:], 0.0)
            fw = ovhs.maxwellian(vm['cv'], 1.0, [0, uy, 0], 1.0)
            assert rel_err(fw, g[key]) < 1e-13


def test_bimaxwellian_matches_reference():
    g = golden('relax0d-n16')
    vm, _, _ = oracle_for(config('relax0d-n16'))
    fp = ovhs.maxwellian(vm['cv'], 1.0, [1.5, 0, 0], 1.0)
    fm = ovhs.maxwellian(vm['cv'], 1.0, [-1.5, 0, 0], 1.0)
    assert rel_err(fp, g['f0_plus']) < 1e-13
    assert rel_err(fm, g['f0_minus']) < 1e-13


def test_fft_form_matches_direct_dft():
    """vhs_Q (FFT, reference order) vs an explicit-DFT evaluation."""
    vm, pre, prefac = oracle_for(_cfg_for('small-n8'))
    rng = np.random.default_rng(3)
    f = ovhs.maxwellian(vm['cv'], 1.0, [0.4, -0.3, 0.2], 0.9)
    f *= 1 + 0.05*rng.standard_normal(vm['V'])
    assert rel_err(ovhs.vhs_Q(f, vm, pre, prefac),
                   ovhs.vhs_direct(f, vm, pre, prefac)) < 1e-12


@pytest.mark.parametrize('name', ['relax0d-n16', 'couette-n24'])
def test_maxwellian_is_near_fixed_point(name):
    """Q(M) vanishes to the method's spectral accuracy."""
    vm, pre, prefac = oracle_for(_cfg_for(name))
    f = ovhs.maxwellian(vm['cv'], 1.0, [0.2, 0.0, -0.1], 1.0)
    Q = ovhs.vhs_Q(f, vm, pre, prefac)
    loss = ovhs.vhs_Q_gain_loss(f, vm, pre, prefac)[1]*f
    tol = {'relax0d-n16': 2e-3, 'couette-n24': 2e-5}[name]
    assert np.max(np.abs(Q))/np.max(np.abs(loss)) < tol


def test_momentum_conserved_for_symmetric_state():
    vm, pre, prefac = oracle_for(config('couette-n24'))
    f = 0.5*(ovhs.maxwellian(vm['cv'], 1, [1.0, 0, 0], 1) +
             ovhs.maxwellian(vm['cv'], 1, [-1.0, 0, 0], 1))
    Q = ovhs.vhs_Q(f, vm, pre, prefac)
    scale = np.sum(np.abs(Q))*vm['cw']
    mom = (Q*vm['cv']).sum(axis=1)*vm['cw']
    assert np.all(np.abs(mom) < 1e-12*scale)
