# -*- coding: utf-8 -*-
"""What the learned surrogate gains over the plain operator (GPU): a
shortened run of frfs_b200.surrogate_study on the Couette workload --
harvest from the plain solver, train with the project's kernels, then the
workload from its own initial state with the surrogate against the plain
FP64 solution.

Bars: relative L2 error of rho, u, T below 1e-3 against the plain FP64
solution; the surrogate-assisted collision sweep at least 2x faster than
the fastest plain kernel; training lowers the loss by 5x.  What the
network itself gains: against the same gate with the network's output
replaced by zero (gated points keep only the exact loss term), the error
in u is at least 2x lower at the default gate threshold (0.05) and 5x
lower at 0.2, where the network stays within 1e-3.  (Measured on this
shortened run: 7.8e-5 against 6.9e-4, and 1.8e-4 against 5.4e-3 at 0.2;
bench.py reports the full-length figures.)
"""

import os

import pytest

from conftest import SPHDESIGN
from frfs_b200 import workloads
from frfs_b200.surrogate_study import run_study

pytestmark = pytest.mark.gpu


def test_surrogate_gain_on_couette():
    res = run_study(workloads.couette_n24, device='cuda:0', runs=2,
                    near_runs=4, steps=50, nsteps=100, epochs=20,
                    relax_steps=50, check_every=50, reps=3,
                    extra_thresholds=(0.2,), sphdesign=SPHDESIGN)
    assert res['train_loss_last'] < 0.2*res['train_loss_first']
    for k in ('rho', 'u', 'T'):
        assert res['err_surrogate'][k] < 1e-3, res['err_surrogate']
        assert res['err_plain_fp32'][k] < 1e-4, res['err_plain_fp32']
    assert res['gate_fraction'] > 0.5
    assert res['speedup'] > 2.0, res
    # the network against the gate without it
    assert res['err_surrogate_without_checks']['u'] < \
        0.5*res['err_gate_without_network']['u'], res
    wide = res['threshold_sweep']['0.2']
    assert wide['err']['u'] < 1e-3, wide
    assert wide['err']['u'] < 0.2*wide['err_gate_without_network']['u'], wide
