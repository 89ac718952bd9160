# -*- coding: utf-8 -*-
"""Spatial partitions of the DG mesh (CPU).

The partitioned mesh keeps frfs's format (frfs/partitioners/base.py:180-235)
and every interface of the whole mesh appears exactly once, either inside a
part or as paired records of two parts.  With two gloo ranks, each rank
builds its part's residual from its own elements and the face values it
receives from the other rank through the product's halo maps and exchange
(frfs_b200.partition); the residual, computed by the oracle on the part
with the received values as the partner states (kernels/mpicflux.mako),
equals the whole-mesh residual on that part's elements.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from helpers import config, dg_setup, random_states
from frfs_b200 import mesh as mgen
from frfs_b200 import partition as pt


def _mesh():
    return mgen.quad_box(6, 4, 0.0, 1.5, -0.25, 0.25, periodic_x=True,
                         jitter=0.15, seed=5)


def _faces(recs):
    return [(int(r['eidx']), int(r['fidx'])) for r in recs]


@pytest.mark.parametrize('nparts', [2, 3, 4])
def test_partitioned_mesh_keeps_every_interface_once(nparts):
    m = _mesh()
    parts = pt.partition_elements(m['spt_quad_p0'], nparts)
    counts = np.bincount(parts, minlength=nparts)
    assert counts.max() - counts.min() <= 1
    pm, glob = pt.partition_mesh(m, parts)
    seen = set()
    for k in range(nparts):
        np.testing.assert_array_equal(pm[f'spt_quad_p{k}'],
                                      m['spt_quad_p0'][:, glob[k]])
        lhs, rhs = pm[f'con_p{k}']
        for l, r in zip(_faces(lhs), _faces(rhs)):
            seen.add(frozenset([(glob[k][l[0]], l[1]),
                                (glob[k][r[0]], r[1])]))
        for s in pt.neighbours(pm, k):
            a, b = _faces(pm[f'con_p{k}p{s}']), _faces(pm[f'con_p{s}p{k}'])
            assert len(a) == len(b)
            for l, r in zip(a, b):
                seen.add(frozenset([(glob[k][l[0]], l[1]),
                                    (glob[s][r[0]], r[1])]))
    lhs, rhs = m['con_p0']
    want = {frozenset([(int(l['eidx']), int(l['fidx'])),
                       (int(r['eidx']), int(r['fidx']))])
            for l, r in zip(lhs, rhs)}
    assert seen == want
    nb = sum(len(m[k]) for k in m if k.startswith('bcon_'))
    nbp = sum(len(pm[k]) for k in pm if k.startswith('bcon_'))
    assert nb == nbp


def _local(pm, k):
    """Part k as a whole-mesh dictionary for the oracle."""
    loc = {'spt_quad_p0': pm[f'spt_quad_p{k}'], 'con_p0': pm[f'con_p{k}']}
    sfx = f'_p{k}'
    for key in pm:
        if key.startswith('bcon_') and key.endswith(sfx):
            loc[key[:-len(sfx)] + '_p0'] = pm[key]
    return loc


def _worker(rank, world, port, out):
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    import torch.distributed as dist
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        cfg = config('channel-n32', 'double', Nv=16, Nrho=4, M=6)
        m = _mesh()
        dg, sh, geo, vm = dg_setup(cfg, m)
        V = vm.vsize()
        u = random_states(vm.cv(), sh.nupts*geo.neles, seed=9, noise=0.05)
        u = u.reshape(sh.nupts, geo.neles, V).transpose(0, 2, 1).copy()
        uf = dg.disu(u)
        dg.update_bc(uf)
        R = dg.rhs(u, uf)

        pm, glob = pt.partition_mesh(
            m, pt.partition_elements(m['spt_quad_p0'], world))
        loc = _local(pm, rank)
        dgl, shl, geol, _ = dg_setup(cfg, loc)
        ul = u[:, :, glob[rank]]
        ufl = dgl.disu(ul)
        # this part's send rows, exchanged with the neighbours (gloo)
        nbrs, counts, rows = pt.halo_rows(pm, rank, geol.srtd_face_fpts)
        send = torch.from_numpy(np.ascontiguousarray(
            np.array([ufl[j, :, e] for j, e in rows]).reshape(-1, V)))
        recv = torch.zeros_like(send)
        pt.exchange(send, recv, nbrs, counts)
        # the received rows as the partner states of an 'mpi' region per
        # neighbour, in the same order
        off = 0
        for s, n in zip(nbrs, counts):
            name = f'mpi{s}'
            recs = _faces(pm[f'con_p{rank}p{s}'])
            dgl.bpts[name] = [(j, e) for e, f in recs
                              for j in geol.srtd_face_fpts[f][e]]
            dgl.bcvals[name] = np.ones((2, n))
            dgl.bcs[name] = {'type': 'mpi',
                             'ur': recv[off:off + n].numpy()}
            off += n
        dgl.update_bc(ufl)
        Rl = dgl.rhs(ul, ufl)
        err = float(np.max(np.abs(Rl - R[:, :, glob[rank]])) /
                    np.max(np.abs(R)))
        out[rank] = err
    finally:
        dist.destroy_process_group()


def _port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


@pytest.mark.parametrize('world', [2, 3])
def test_partitioned_residual_equals_whole_mesh_residual(world):
    ctx = mp.get_context('spawn')
    out = ctx.Manager().dict()
    mp.start_processes(_worker, args=(world, _port(), out), nprocs=world,
                       join=True, start_method='spawn')
    assert sorted(out.keys()) == list(range(world))
    for r in range(world):
        assert out[r] < 1e-13, (r, out[r])


@pytest.mark.parametrize('workload,world', [('couette-n24', 2),
                                            ('couette-n24', 8),
                                            ('channel-n32', 2),
                                            ('channel-n32', 4),
                                            ('channel-n32', 8)])
def test_weak_scaled_bench_partitions(workload, world):
    """bench.py's multi-GPU set-up: the workload widened to `world` copies
    along x splits into `world` parts of exactly the single-GPU workload's
    element count, every part has the shared faces of a strip (two
    neighbours, one for the walled Couette slab's end parts) and its halo
    rows pair up with its neighbours' rows."""
    import argparse
    import importlib.util
    import os
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location(
        'bench', os.path.join(ROOT, 'bench.py'))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    args = argparse.Namespace(workload=workload, precision='single',
                              project=1, elements=None)
    cfg1 = bench._cfg(args, 1)
    cfg = bench._cfg(args, world)
    nupts, neles = bench._points_shape(cfg, world)
    assert (nupts, neles) == bench._points_shape(cfg1, 1)
    whole = mgen.from_config(cfg)
    pm, glob = pt.partition_mesh(whole, pt.partition_elements(
        whole['spt_quad_p0'], world))
    from frfs_b200.elements import ElementGeometry
    from frfs_b200.shapes import QuadShape
    sh = QuadShape(cfg.getint('solver', 'order'))
    rows = {}
    for k in range(world):
        assert len(glob[k]) == neles
        geo = ElementGeometry(sh, pm[f'spt_quad_p{k}'])
        nbrs, counts, hr = pt.halo_rows(pm, k, geo.srtd_face_fpts)
        periodic = workload == 'channel-n32'
        want = 2 if (periodic or 0 < k < world - 1) else 1
        assert len(set(nbrs)) == min(want, world - 1)
        rows[k] = dict(zip(nbrs, counts))
    for k in rows:
        for s, n in rows[k].items():
            assert rows[s][k] == n
