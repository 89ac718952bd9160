# -*- coding: utf-8 -*-
"""Stage graphs through the C ABI (GPU).

An SSP-RK2 stage on the Couette workload's discretisation (4x1 strip,
N = 24, FP32), made of the library's own entry points (dgfs_vhs_apply,
dgfs_dg_updatebc, dgfs_dg_interp, dgfs_dg_rhs), is captured between
dgfs_graph_begin and dgfs_graph_end and replayed with dgfs_graph_launch.
The replayed stage gives bit-identical banks to the stage run call by call,
on two replays in a row, and the capture itself runs nothing.
"""

import ctypes as ct

import numpy as np
import pytest
import torch

from helpers import config
from frfs_b200 import _lib
from frfs_b200 import mesh as mgen
from frfs_b200.backend import B200Backend
from frfs_b200.system import DGFSSystem

pytestmark = pytest.mark.gpu

_lib.declare('dgfs_graph_begin', ct.c_int, [ct.c_void_p])
_lib.declare('dgfs_graph_end', ct.c_int, [ct.c_void_p, ct.c_void_p])
_lib.declare('dgfs_graph_launch', ct.c_int, [ct.c_void_p, ct.c_void_p])
_lib.declare('dgfs_graph_destroy', ct.c_int, [ct.c_void_p])


def _stage(s, dt):
    """Stage 1 of StdTVDRK2DGFSStepper: r1 = r0 + dt (L(r0) + Q(r0))."""
    s.collide(0.0, 0, 1)
    s.updatebc(0.0, 0, 1, 0, 0)
    s.rk_stage(0, 1, 1.0, 0, 0.0, None, dt, 1, interp=False)


def test_stage_graph_replays_the_stage():
    cfg = config('couette-n24', 'single', nele=4)
    m = mgen.from_config(cfg)
    be = B200Backend(cfg, device='cuda:0')
    s = DGFSSystem(be, cfg, mesh=m)
    lib = _lib.load()
    dt = 2e-3
    side = torch.cuda.Stream(device=be.device)
    side.wait_stream(torch.cuda.current_stream(be.device))
    with torch.cuda.stream(side):
        _stage(s, dt)                  # call by call (and every first call)
        side.synchronize()
        ref = s.bank[1].get().copy()
        s.bank[1].set(np.zeros_like(ref))
        g = ct.c_void_p()
        _lib.check(lib.dgfs_graph_begin(side.cuda_stream), 'dgfs_graph_begin')
        _stage(s, dt)                  # recorded, not run
        _lib.check(lib.dgfs_graph_end(side.cuda_stream, ct.byref(g)),
                   'dgfs_graph_end')
        side.synchronize()
        assert np.all(s.bank[1].get() == 0)   # capture ran nothing
        for _ in range(2):
            _lib.check(lib.dgfs_graph_launch(g, side.cuda_stream),
                       'dgfs_graph_launch')
            side.synchronize()
            assert np.array_equal(s.bank[1].get(), ref)
        _lib.check(lib.dgfs_graph_destroy(g), 'dgfs_graph_destroy')
    torch.cuda.current_stream(be.device).wait_stream(side)


def test_graph_begin_rejects_the_legacy_stream():
    with pytest.raises(_lib.DgfsError):
        _lib.check(_lib.load().dgfs_graph_begin(None), 'dgfs_graph_begin')
