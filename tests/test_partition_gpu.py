# -*- coding: utf-8 -*-
"""Partitioned FR-DG residual on the GPU.

Two parts of one mesh run as two DGFSSystem instances on one device; the
face values of the shared faces go from one part's send rows
(dgfs_dg_pack) to the other's halo rows (dgfs_dg_set_halo) by a device copy,
which stands in for the NCCL exchange between ranks (the exchange itself is
tested with gloo ranks on the CPU, tests/test_partition.py).  Each part's
residual equals the whole mesh's residual on its elements.

Tolerance: FP64 1e-12 and FP32 1e-6 against the whole-mesh kernel (same
arithmetic on the same face values), FP64 1e-10 against the oracle.
"""

import numpy as np
import pytest
import torch

from helpers import config, dg_setup, random_states, rel_err
from frfs_b200 import mesh as mgen
from frfs_b200 import partition as pt
from frfs_b200.backend import B200Backend
from frfs_b200.system import DGFSSystem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('precision,tol', [('double', 1e-12),
                                           ('single', 1e-6)])
@pytest.mark.parametrize('order', [2, 3])
def test_two_parts_match_whole_mesh(precision, tol, order):
    cfg = config('channel-n32', precision, Nv=16, Nrho=4, M=6)
    cfg.set('solver', 'order', order)
    m = mgen.quad_box(6, 4, 0.0, 1.5, -0.25, 0.25, periodic_x=True,
                      jitter=0.15, seed=5)
    dg, sh, geo, vm = dg_setup(cfg, m)
    V = vm.vsize()
    u = random_states(vm.cv(), sh.nupts*geo.neles, seed=4, noise=0.05)
    u = u.reshape(sh.nupts, geo.neles, V).transpose(0, 2, 1).copy()

    be = B200Backend(cfg, device='cuda:0')
    whole = DGFSSystem(be, cfg, mesh=m, initsoln=u)
    whole.updatebc(0.0, 0, 1, 0, 0)
    whole.rhs(0.0, 0, 1, 0, 0)

    pm, glob = pt.partition_mesh(m, pt.partition_elements(m['spt_quad_p0'],
                                                          2))
    noop = lambda send, recv, nbrs, counts: None
    parts = [DGFSSystem(be, cfg, mesh=pm, prank=k, halo_exchange=noop,
                        initsoln=u[:, :, glob[k]]) for k in range(2)]
    for p in parts:
        assert p.halo is not None and p.halo[0] == [1 - p.prank]
        p.updatebc(0.0, 0, 1, 0, 0)
    # the exchange: each part's send rows are the other's halo rows
    parts[0].halo_recv.copy_(parts[1].halo_send)
    parts[1].halo_recv.copy_(parts[0].halo_send)
    for p in parts:
        p.rhs(0.0, 0, 1, 0, 0)
    torch.cuda.synchronize()

    Rw = whole.bank[1].get()
    for k, p in enumerate(parts):
        err = rel_err(p.bank[1].get(), Rw[:, :, glob[k]])
        assert err < tol, (k, err)
    if precision == 'double':
        uf = dg.disu(u)
        dg.update_bc(uf)
        assert rel_err(Rw, dg.rhs(u, uf)) < 1e-10
