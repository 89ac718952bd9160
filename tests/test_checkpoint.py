# -*- coding: utf-8 -*-
"""Checkpoint record and restart interpolation (CPU): the record round-trips
through a file, the fields check rejects a solution of another velocity
grid, and restarting at a higher order reproduces a solution that is a
polynomial of the stored order exactly (frfs/solvers/dgfs/system.py:79-112
interpolates with the stored basis)."""

import numpy as np
import pytest

from helpers import config
from frfs_b200 import checkpoint as ck
from frfs_b200 import mesh as mgen
from frfs_b200.elements import ElementGeometry
from frfs_b200.shapes import QuadShape


def _poly_solution(order, mesh, V, deg):
    sh = QuadShape(order)
    geo = ElementGeometry(sh, mesh['spt_quad_p0'])
    x, y = geo.ploc_upts[..., 0], geo.ploc_upts[..., 1]   # (nupts, neles)
    k = np.arange(V)[None, :, None]
    return (1 + 0.1*k*x[:, None, :]**deg + 0.05*y[:, None, :]**deg
            - 0.02*k*x[:, None, :]*y[:, None, :])


def test_record_round_trip_and_order_change(tmp_path):
    m = mgen.quad_box(3, 2, 0.0, 1.0, 0.0, 0.5, jitter=0.0)
    cfg = config('relax0d-n16')
    cfg.set('solver', 'order', 2)
    V = 5
    u2 = _poly_solution(2, m, V, 2)
    rec = ck.solution_record(u2, cfg, 0.25, 7, m)
    np.savez(tmp_path/'c.npz', **rec)
    back = ck.read(tmp_path/'c.npz')
    assert np.array_equal(back['soln_quad_p0'], u2)
    assert ck.restart_time(back) == (0.25, 7)
    # same order: identity
    assert np.allclose(ck.restart_bank(back, cfg, V, m), u2, rtol=0,
                       atol=1e-14)
    # p = 2 -> 3 on affine elements: quadratics are reproduced
    cfg3 = config('relax0d-n16')
    cfg3.set('solver', 'order', 3)
    u3 = ck.restart_bank(back, cfg3, V, m)
    assert np.allclose(u3, _poly_solution(3, m, V, 2), rtol=0, atol=1e-12)
    with pytest.raises(RuntimeError):
        ck.restart_bank(back, cfg, V + 1, m)
    with pytest.raises(RuntimeError):
        ck.restart_bank(back, cfg, V, mgen.quad_box(2, 2, 0.0, 1.0, 0.0, 0.5))
