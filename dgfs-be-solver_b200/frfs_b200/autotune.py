# -*- coding: utf-8 -*-
"""Autotuner for the fused VHS kernel's launch shape.

The kernel is compiled for several shapes per (precision, Nv): cluster size
(CTAs sharing one solution point through distributed shared memory),
double-buffered or single exchange buffers, and the CTAs per SM the register
budget targets.  Which one is fastest depends on the point count (tail of the
last wave), Nrho*M and the GPU, so it is measured: each shape runs the
caller's bank ``reps`` times under CUDA events and the fastest is selected.
Results are cached on disk keyed by GPU name, precision, Nv, Nrho, M and the
number of points.
"""

import json
import os

import torch


def _cache_path():
    base = os.environ.get('DGFS_B200_CACHE',
                          os.path.join(os.path.expanduser('~'), '.cache',
                                       'dgfs_b200'))
    return os.path.join(base, 'vhs_tune.json')


def _load():
    try:
        with open(_cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(db):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + '.tmp'
        with open(tmp, 'w') as fh:
            json.dump(db, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def tune_vhs(sm, fin, fout, npts=None, reps=2, cache=True, verbose=False):
    nupts, nvars, neles = fin.ioshape
    total = nupts*neles
    npts = min(npts or total, total)
    vm = sm.vm
    dev = torch.cuda.get_device_name(sm.backend.device)
    key = (f'{dev}|{sm.backend.precision}|{vm.Nv()}|{vm.Nrho()}|{vm.M()}|'
           f'{npts}|{sm._project}')
    db = _load() if cache else {}
    variants = sm.variants()
    if key in db and db[key]['index'] < len(variants):
        sm.select(db[key]['index'])
        return db[key]

    stream = torch.cuda.current_stream(sm.backend.device)
    results = []
    for i, v in enumerate(variants):
        try:
            sm.select(i)
        except RuntimeError:
            continue
        sm.fs_range(fin, fout, 0, npts)          # warm-up
        best = None
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sm.fs_range(fin, fout, 0, npts)
            e1.record(stream)
            e1.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        results.append((best, i, v))
        if verbose:
            print(f'vhs variant {i} {v}: {best:.3f} ms')
    if not results:
        raise RuntimeError('no VHS launch shape could run on this device')
    best, idx, v = min(results, key=lambda r: r[0])
    sm.select(idx)
    entry = {'index': idx, 'ms': best, 'variant': v,
             'all_ms': {str(i): t for t, i, _ in results}}
    if cache:
        db[key] = entry
        _store(db)
    return entry
