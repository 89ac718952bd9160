# -*- coding: utf-8 -*-
"""On-device FP64 moments against the oracle's restatement of frfs's moment
writer (GPU)."""

import numpy as np
import pytest

from helpers import config, random_states
from frfs_b200.backend import B200Backend
from frfs_b200.system import bank_moments
from frfs_b200.velocitymesh import DGFSVelocityMesh
from oracle import vhs as ovhs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_moments_match_oracle(precision):
    cfg = config('relax0d-n16', precision)
    be = B200Backend(cfg, device='cuda:0')
    vm = DGFSVelocityMesh(be, cfg)
    nupts, neles = 3, 37
    f = random_states(vm.cv(), nupts*neles, seed=8)
    arr = np.ascontiguousarray(f.reshape(nupts, neles, -1).transpose(0, 2, 1))
    bank = be.matrix(arr.shape, arr)
    m = bank_moments(bank, vm, be)
    fused = bank.get().astype(np.float64)
    cv, cw = vm.cv(), vm.cw()
    tol = 1e-12 if precision == 'double' else 1e-12
    for u in range(nupts):
        for e in range(neles):
            fv = fused[u, :, e]
            rho, uu, T, q = ovhs.moments(fv, cv, cw)
            c = cv - uu[:, None]
            P = [2*np.sum(fv*c[i]*c[j])*cw
                 for i, j in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))]
            ref = np.concatenate([[rho], uu, [T], q, P])
            assert np.allclose(m[u, e], ref, rtol=tol, atol=tol*np.abs(ref).max())
