# -*- coding: utf-8 -*-
"""Spatial partitions of the DG mesh and the face-value halo exchange.

The collision operator is independent per solution point; the DG residual
couples elements only through the common flux at shared faces.  A partition
therefore runs the whole step on its own elements and needs, once per
residual, the face values ``uf`` of the flux points that a neighbouring
partition owns across a shared face -- frfs's MPI interfaces
(frfs/solvers/dgfs/inters.py:61-112, ``DGFSMPIInters``: pack the local face
values, persistent MPI send/recv, Riemann solve against the received values
in kernels/mpicflux.mako; frfs/backends/base/packing.py:31-39).

* ``partition_elements``: element-to-part map by recursive coordinate
  bisection of the element centroids (frfs calls METIS or SCOTCH,
  frfs/partitioners/; graph partitioners are out of scope here, and the
  meshes of the workloads are structured).
* ``partition_mesh``: the partitioned mesh dictionary in frfs's format
  (frfs/partitioners/base.py:180-235): ``spt_quad_p{k}``, ``con_p{k}``,
  ``bcon_{name}_p{k}`` and ``con_p{k}p{j}``, whose i-th record pairs with the
  i-th record of ``con_p{j}p{k}``; local element numbers follow the global
  order within each part.
* ``halo_rows``: the flux points a part sends to and receives from each
  neighbour, in the order both sides agree on (interface record order, then
  the coordinate-sorted flux points of each face, the same pairing as
  interior faces, frfs/solvers/base/inters.py:14-19).
* ``exchange``: the P2P exchange of the packed rows over torch.distributed
  (NCCL for device buffers, gloo for host buffers), one send and one receive
  per neighbour.
"""

import numpy as np

_REC = np.dtype([('etype', 'U4'), ('eidx', 'i4'), ('fidx', 'i1'),
                 ('flags', 'i1')])


def partition_elements(spt, nparts):
    """Part index of every element: recursive coordinate bisection of the
    element centroids, splitting the longest extent of each group into
    sizes proportional to the parts on either side (stable sort, so equal
    centroids keep their global order)."""
    spt = np.asarray(spt, dtype=np.float64)
    neles = spt.shape[1]
    if nparts < 1 or nparts > neles:
        raise ValueError(f'cannot split {neles} elements into {nparts} parts')
    cent = spt.mean(axis=0)
    parts = np.zeros(neles, dtype=np.int64)

    def split(idx, k, p0):
        if k == 1:
            parts[idx] = p0
            return
        k1 = k // 2
        ext = cent[idx].max(axis=0) - cent[idx].min(axis=0)
        ax = int(np.argmax(ext))
        order = idx[np.argsort(cent[idx, ax], kind='stable')]
        n1 = int(round(len(idx)*k1/k))
        split(order[:n1], k1, p0)
        split(order[n1:], k - k1, p0 + k1)

    split(np.arange(neles), nparts, 0)
    return parts


def partition_mesh(mesh, parts):
    """Split a single-part mesh dictionary (keys ``*_p0``) by the element
    part map ``parts``; returns (partitioned mesh, global element ids of
    every part in local order)."""
    parts = np.asarray(parts)
    nparts = int(parts.max()) + 1
    spt = mesh['spt_quad_p0']
    glob = [np.nonzero(parts == k)[0] for k in range(nparts)]
    local = np.empty(len(parts), dtype=np.int64)
    for k, g in enumerate(glob):
        local[g] = np.arange(len(g))
    out = {f'spt_quad_p{k}': spt[:, g] for k, g in enumerate(glob)}
    con, conxy = {}, {}
    lhs, rhs = mesh['con_p0']
    for l, r in zip(lhs, rhs):
        el, er = int(l['eidx']), int(r['eidx'])
        pl, pr = int(parts[el]), int(parts[er])
        recl = ('quad', int(local[el]), int(l['fidx']), int(l['flags']))
        recr = ('quad', int(local[er]), int(r['fidx']), int(r['flags']))
        if pl == pr:
            con.setdefault(pl, ([], []))
            con[pl][0].append(recl)
            con[pl][1].append(recr)
        else:
            conxy.setdefault((pl, pr), []).append(recl)
            conxy.setdefault((pr, pl), []).append(recr)
    for k in range(nparts):
        l_, r_ = con.get(k, ([], []))
        out[f'con_p{k}'] = np.array([l_, r_], dtype=_REC).reshape(2, -1)
    for (a, b), recs in conxy.items():
        out[f'con_p{a}p{b}'] = np.array(recs, dtype=_REC)
    for key in mesh:
        if key.startswith('bcon_') and key.endswith('_p0'):
            name = key[5:-3]
            for rec in mesh[key]:
                e = int(rec['eidx'])
                k = int(parts[e])
                out.setdefault(f'bcon_{name}_p{k}', []).append(
                    ('quad', int(local[e]), int(rec['fidx']),
                     int(rec['flags'])))
    for key in list(out):
        if key.startswith('bcon_') and isinstance(out[key], list):
            out[key] = np.array(out[key], dtype=_REC)
    return out, glob


def neighbours(mesh, prank):
    """Ranks that share a face with part ``prank``, ascending."""
    pre = f'con_p{prank}p'
    return sorted(int(k[len(pre):]) for k in mesh if k.startswith(pre))


def halo_rows(mesh, prank, srtd):
    """Send/receive rows of part ``prank``.

    Returns (nbrs, counts, rows): for every neighbour in ``nbrs`` (ascending
    rank) ``counts`` flux points, and ``rows`` the (flux point, element) of
    each of this part's flux points on the shared faces, neighbour by
    neighbour, interface record by record, each face's points in the
    coordinate-sorted order ``srtd[face][element]``.  Row h is both what
    this part sends (its own face value there) and where the neighbour's
    value at the paired flux point arrives."""
    nbrs = neighbours(mesh, prank)
    counts, rows = [], []
    for s in nbrs:
        n0 = len(rows)
        for rec in mesh[f'con_p{prank}p{s}']:
            e, f = int(rec['eidx']), int(rec['fidx'])
            rows.extend((int(j), e) for j in srtd[f][e])
        counts.append(len(rows) - n0)
    return nbrs, counts, rows


def exchange(send, recv, nbrs, counts, group=None):
    """Send rows send[off:off+n] to every neighbour and receive the same
    number of rows from it into recv[off:off+n] (torch tensors of shape
    (nrows, V) on the backend's device for NCCL, on the host for gloo).
    All sends and receives are posted before any is waited on."""
    import torch.distributed as dist
    ops, off = [], 0
    for s, n in zip(nbrs, counts):
        if n:
            ops.append(dist.P2POp(dist.isend, send[off:off + n], s, group))
            ops.append(dist.P2POp(dist.irecv, recv[off:off + n], s, group))
        off += n
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
