# -*- coding: utf-8 -*-
"""The surrogate's training-state generators (CPU): every initial state
lies inside the parameter box the training data are specified on
(rho in [0.5, 2], T in [0.5, 3], |u| <= 1), and the states near the
reference state reach down to weak mismatches."""

import numpy as np

from helpers import config
from frfs_b200.surrogate import random_near_state, random_uniform_state
from frfs_b200.velocitymesh import DGFSVelocityMesh
from oracle import vhs as ovhs


def _frame(vm, f):
    cv, cw = vm.cv(), vm.cw()
    rho = np.sum(f)*cw
    u = cv @ f*cw/rho
    T = np.sum(np.sum((cv - u[:, None])**2, axis=0)*f)*cw/(1.5*rho)
    return rho, u, T


def test_states_stay_in_the_box():
    vm = DGFSVelocityMesh(None, config('couette-n24'))
    dist = []
    for seed in range(60):
        rng = np.random.default_rng(seed)
        for f, spread in ((random_near_state(vm, rng), 0.0),
                          (random_uniform_state(vm, rng, False), 0.0),
                          (random_uniform_state(vm, rng, True), 2/3)):
            # a bimodal mixture of Maxwellians at +-u (|u| <= 1) has the
            # components' temperature plus 2|u|^2/3 from their separation
            rho, u, T = _frame(vm, f)
            assert 0.5 - 1e-6 <= rho <= 2 + 1e-6
            assert np.linalg.norm(u) <= 1 + 1e-6
            assert 0.5 - 1e-3 <= T <= 3 + spread + 1e-3
        rho, u, T = _frame(vm, random_near_state(
            vm, np.random.default_rng(seed)))
        dist.append(max(np.linalg.norm(u), abs(np.log(T)), abs(np.log(rho))))
    # log-uniform distance from (1, 1, 0): both weak and strong mismatches
    assert min(dist) < 0.05 and max(dist) > 0.3


def test_near_state_is_a_maxwellian():
    vm = DGFSVelocityMesh(None, config('couette-n24'))
    f = random_near_state(vm, np.random.default_rng(3))
    rho, u, T = _frame(vm, f)
    m = ovhs.maxwellian(vm.cv(), rho, u, T)
    assert np.max(np.abs(f - m)) < 1e-6*np.max(m)
