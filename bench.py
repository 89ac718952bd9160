# -*- coding: utf-8 -*-
"""Benchmark of the B200 DGFS hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload couette-n24] [--precision single|double]
                    [--mode collide|step]

Workload: the 1D/3V Couette slab (64 x 1 quadrilateral strip, p = 2, 576
solution points, N = 24^3 velocities, Nrho = 12, M = 16, VHS omega = 0.81),
synthetic distributions (Maxwellians with seeded 1% noise).  One step is one
SSP-RK2 solver step (default ``--mode step``: two collision sweeps over every
solution point, two DG residuals with their boundary updates, one CUDA graph
per stage) or one collision sweep alone (``--mode collide``: a single
persistent launch of the fused VHS kernel).  The metric is Q(f) evaluations
per second, whole job; the line also carries the DG step time and, at N=1
on the Couette workload, the learned surrogate's run (``surrogate``: pairs
harvested from the solver, training, rho/u/T errors against the plain FP64
solution after 200 steps, evaluations per second plain vs surrogate).

Multi-GPU (torchrun, --mode step): the workload's domain is widened to N
copies side by side along x and split into N spatial partitions, one per
rank (weak scaling: every rank holds the single-GPU workload's elements);
the ranks exchange the face values of their shared faces once per residual
over NCCL (frfs's MPI interfaces) and the time is the max over ranks.  With
--mode collide every rank evaluates its own copy (no exchange).

``--impl reference`` times the reference's algorithm on the host cores: the
reference itself is PyCUDA/cuFFT-only (no CPU path) and cannot be imported on
this software stack, so the FP64 numpy restatement in oracle/ stands in for it.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, 'dgfs-be-solver_b200')
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

SPHDESIGN = os.path.join(PKG, 'frfs_b200', 'data', 'sphericaldesign')
METRIC = 'Q(f) evals/s'

# DRAM bytes (read + write) per launch measured by ncu, keyed by (kernel,
# workload, points, precision bits); only exact matches are reported
# dram__bytes_read.sum + dram__bytes_write.sum per launch from ncu captures:
# (kernel, workload, points, precision bits) -> (bytes, how it was taken)
TRAFFIC = {
    ('vhs_cube_kernel', 'couette-n24', 576, 32):
        (36.7e6, 'captured at this size'),
    ('vhs_pair_kernel', 'channel-n32', 10368, 32):
        (208.3e6*72, 'captured on the 4 x 4-element channel (144 points, '
                     '208.3 MB, 512-thread layout) and scaled by the point '
                     'count (x72)'),
}
# the same for one DG stage (interp + residual): (workload, points, bits)
DG_TRAFFIC = {
    ('couette-n24', 576, 32):
        (148.9e6, 'captured at this size (interp 33.5 MB + residual '
                  '115.4 MB, residual shape of 8 velocities per warp)'),
}


def _parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--workload', default='couette-n24')
    ap.add_argument('--precision', default='single',
                    choices=['single', 'double'])
    ap.add_argument('--project', type=int, default=1)
    ap.add_argument('--mode', default='step', choices=['collide', 'step'])
    ap.add_argument('--cpu-seconds', type=float, default=12.0)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--variant', type=int, default=-1,
                    help='VHS launch shape index (default: autotune)')
    ap.add_argument('--graphs', type=int, default=1,
                    help='CUDA graph per SSP-RK2 stage (--mode step)')
    ap.add_argument('--surrogate', type=int, default=-1,
                    help='train and evaluate the learned surrogate in this run '
                         '(-1: on for couette-n24 at N=1)')
    ap.add_argument('--surrogate-steps', type=int, default=200)
    ap.add_argument('--surrogate-harvest-steps', type=int, default=100,
                    help='steps of every training trajectory (random '
                         'initial states) the surrogate is harvested from')
    ap.add_argument('--initial', default='synthetic',
                    choices=['synthetic', 'workload'],
                    help='step mode: synthetic noisy Maxwellians or the '
                         "workload's own initial condition")
    ap.add_argument('--e2e', type=int, default=1,
                    help='0: skip the end-to-end measurement (banks too '
                         'large for a pinned host copy)')
    ap.add_argument('--elements', type=int, nargs=2, default=None,
                    metavar=('NX', 'NY'),
                    help='mesh size override (quad box: nx ny; O-grid: '
                         'ntheta nr), for small profiling cases')
    return ap.parse_args()


def _cfg(args, world=1):
    """The workload's config; with world > 1 (partitioned runs) the
    domain is ``world`` copies of the workload laid side by side along x,
    one per rank (weak scaling)."""
    from frfs_b200 import workloads
    from frfs_b200.inifile import Inifile
    kw = {}
    if args.elements:
        a, b = args.elements
        kw = ({'ntheta': a, 'nr': b} if args.workload.startswith('cylinder')
              else {'nx': a, 'ny': b})
    if world > 1:
        if args.workload not in ('couette-n24', 'channel-n32'):
            raise SystemExit(f'{args.workload}: partitioned runs are set up '
                             'for couette-n24 and channel-n32')
        kw['copies'] = world
    cfg = Inifile(workloads.WORKLOADS[args.workload](
        precision=args.precision, **kw))
    cfg.set('spherical-design-rule', 'path', SPHDESIGN)
    cfg.set('backend-b200', 'vhs-project', int(args.project))
    return cfg


def _workload_desc(args, cfg, npts, world=1):
    return {
        'parallelism': (f'{world} spatial partitions, NCCL face-value halo '
                        'exchange' if world > 1 and args.mode == 'step'
                        else f'{world} independent replicas' if world > 1
                        else 'single GPU'),
        'workload': f'{args.workload}: DGFS fast-spectral VHS Q(f) at every '
                    f'solution point' + (' + FR-DG SSP-RK2 step'
                                         if args.mode == 'step' else ''),
        'points': npts,
        'Nv': cfg.getint('constants', 'Nv'),
        'Nrho': cfg.getint('constants', 'Nrho'),
        'M': cfg.getint('spherical-design-rule', 'M'),
        'omega': cfg.getfloat('scattering-model', 'omega'),
        'precision': args.precision,
        'projection': bool(args.project),
        'mode': args.mode,
        'l2': 'flushed between timed steps (256 MiB write)',
    }


def _points_shape(cfg, world=1):
    """(nupts, neles) of the workload's mesh ((p+1)^2 points per quad),
    per rank when the mesh is split over ``world`` ranks."""
    order = cfg.getint('solver', 'order')
    if cfg.hasopt('mesh', 'nx'):
        neles = cfg.getint('mesh', 'nx')*cfg.getint('mesh', 'ny')
        return (order + 1)**2, neles//world
    if cfg.hasopt('mesh', 'ntheta'):
        neles = cfg.getint('mesh', 'ntheta')*cfg.getint('mesh', 'nr')
        return (order + 1)**2, neles
    return 1, 1


def _synthetic_f(cv, nupts, neles, seed=0):
    """Maxwellian (rho=1, T=1, u=0) times (1 + 0.01 xi), xi ~ N(0,1) i.i.d.
    per velocity node and point; shape (nupts, V, neles)."""
    rng = np.random.default_rng(seed)
    V = cv.shape[1]
    m = np.exp(-np.sum(cv*cv, axis=0))/np.pi**1.5
    xi = rng.standard_normal((nupts, V, neles))
    return m[None, :, None]*(1.0 + 0.01*xi)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,'
              'clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
              'clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,'
              'clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index, period_ms=200):
        self.idx = gpu_index
        self.period_ms = period_ms
        self.proc = None
        self.lines = []
        self._first = 0

    def start(self, wait_s=5.0):
        """Start sampling and wait (bounded) for the first sample, so that
        the region timed after this call is covered; samples taken before
        it are not counted."""
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.idx),
                 f'--query-gpu={self.FIELDS}', '--format=csv,noheader,nounits',
                 '-lms', str(self.period_ms)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, ValueError):
            self.proc = None
            return
        t0 = time.time()
        while (not self.lines and self.proc.poll() is None
               and time.time() - t0 < wait_s):
            time.sleep(0.005)
        self._first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        # samples of the timed region; if the region was shorter than one
        # period, the first sample after it
        n_end = len(self.lines)
        if n_end == self._first:
            t0 = time.time()
            while (len(self.lines) == n_end and self.proc.poll() is None
                   and time.time() - t0 < 1.0):
                time.sleep(0.005)
            n_end = min(len(self.lines), n_end + 1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self._t.join(timeout=2)
        self.lines = self.lines[self._first:n_end]
        sm, smax, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
                 'sw_power_cap']
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == 'active':
                    reasons.add(n)
        if not sm:
            return None
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': smax,
                'reasons': sorted(reasons), 'samples': len(sm)}


# ---------------------------------------------------------------------------
# CPU baselines (the oracle restatement of the reference algorithm)
# ---------------------------------------------------------------------------
def _cpu_setup(cfg, seed=0):
    """The FP64 oracle's velocity mesh, precomputation and prefactor for the
    workload, and 64 of its synthetic points."""
    from oracle import vhs as ovhs
    g = lambda s, k: cfg.getfloat(s, k)
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    vm = DGFSVelocityMesh(None, cfg)
    ovm = ovhs.velocity_mesh(vm.Nv(), vm.Nrho(), vm.M(),
                             np.vstack([vm.sz(), -vm.sz()]),
                             g('non-dim', 'H0'), g('non-dim', 'T0'),
                             g('non-dim', 'rho0'), g('non-dim', 'molarMass0'),
                             g('velocity-mesh', 'cmax'),
                             g('velocity-mesh', 'Tmax'),
                             g('velocity-mesh', 'dev'))
    gam, prefac = ovhs.vhs_parameters(g('scattering-model', 'omega'),
                                      g('scattering-model', 'dRef'),
                                      g('scattering-model', 'Tref'),
                                      g('non-dim', 'H0'), ovm['n0'],
                                      g('non-dim', 'T0'))
    pre = ovhs.vhs_precompute(ovm, gam)
    f = _synthetic_f(vm.cv(), 1, 64, seed)[0].T
    return dict(ovm=ovm, pre=pre, prefac=prefac, f=f, M=vm.M())


def _cpu_proc(cfg_text, seed, budgets, wid, out):
    """One process of the CPU baseline (spawned): single-threaded FFTs,
    points of the sample evaluated one after another for each budget in
    ``budgets`` (seconds); puts (step, points, seconds) per budget."""
    os.environ['DGFS_ORACLE_THREADS'] = '1'
    from frfs_b200.inifile import Inifile
    from oracle import vhs as ovhs
    s = _cpu_setup(Inifile(cfg_text), seed)
    k = wid
    for step, budget in enumerate(budgets):
        n, t0 = 0, time.perf_counter()
        while True:
            # one radial node per batch of transforms (bounded memory)
            ovhs.vhs_Q(s['f'][k % len(s['f'])], s['ovm'], s['pre'],
                       s['prefac'], batch_pm=s['M'])
            n, k = n + 1, k + 1
            dt = time.perf_counter() - t0
            if dt >= budget:
                break
        out.put((step, n, dt))


def _cpu_baseline_runs(cfg, budgets, seed=0):
    """The FP64 oracle on every host core, one single-threaded process per
    core (spawned, so it is safe after CUDA has been initialised), each
    evaluating whole points.  Per budget: (throughput, points, seconds,
    cores), the throughput being all processes' points over the slowest
    process's time."""
    import multiprocessing as mp
    cores = len(os.sched_getaffinity(0))
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    procs = [ctx.Process(target=_cpu_proc,
                         args=(cfg.tostr(), seed, list(budgets), w, out))
             for w in range(cores)]
    for p in procs:
        p.start()
    res = [out.get() for _ in range(cores*len(budgets))]
    for p in procs:
        p.join()
    runs = []
    for step in range(len(budgets)):
        r = [x for x in res if x[0] == step]
        n = sum(x[1] for x in r)
        dt = max(x[2] for x in r)
        runs.append((n/dt, n, dt, cores))
    return runs


def _cpu_baseline(cfg, budget_s, seed=0):
    value, n, dt, cores = _cpu_baseline_runs(cfg, [budget_s], seed)[0]
    return _cpu_desc(value, n, cores), n, dt


def _cpu_desc(value, n, cores):
    return {'value': value, 'unit': 'evals/s', 'cores': cores,
            'kind': 'port',
            'sample': f'{n} solution points of the workload (64 synthetic '
                      f'points, FP64 numpy/scipy.fft restatement of '
                      f'scattering.py:227-286), {cores} single-threaded '
                      f'processes, one point at a time each'}


def run_reference(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    cfg = _cfg(args)
    nupts, neles = _points_shape(cfg)
    per_step = max(5.0, 60.0/max(1, args.steps + args.warmup))
    runs = _cpu_baseline_runs(cfg, [min(per_step, 5.0)]*args.warmup +
                              [per_step]*args.steps)[args.warmup:]
    value = float(np.mean([r[0] for r in runs]))
    cb = _cpu_desc(value, sum(r[1] for r in runs), runs[0][3])
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value,
        'unit': 'evals/s', 'n_gpus': args.gpus, 'steps': args.steps,
        'warmup': args.warmup,
        'ms_per_step': 1e3*nupts*neles/value,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f64', 'data': 'synthetic',
        'config': _workload_desc(args, cfg, nupts*neles),
        'cpu_baseline': cb,
        'e2e': {'value': value, 'unit': 'evals/s',
                'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
        'note': 'reference is PyCUDA+cuFFT only; its algorithm is timed as '
                'the FP64 oracle restatement on the host cores; each step '
                'is a bounded sample of the sweep',
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def _timed(fn, steps, stream, flush):
    """Per-step CUDA-event times (ms) of fn on ``stream``; L2 is flushed
    before every step, outside the events."""
    import torch
    times = []
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


def _e2e_pipelined(step, src_bank, dst_bank, hin, hout, nsteps, stream,
                   flush):
    """Device time (ms) of nsteps end-to-end steps: step i's input goes
    host -> device staging buffer on one copy stream while step i - 1
    computes, and step i's result goes staging buffer -> host on another
    while step i + 1 computes.  The compute stream moves the staged input
    into the bank and the result out of it (device-to-device copies), runs
    the step and flushes L2 before it.  Events on the compute stream bracket
    everything from the first host-to-device copy to the last device-to-host
    copy."""
    import torch
    dev = src_bank.data.device
    h2d, d2h = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    sin = [torch.empty_like(src_bank.data) for _ in range(2)]
    sout = [torch.empty_like(dst_bank.data) for _ in range(2)]
    ev = lambda: torch.cuda.Event()
    in_ready, in_free = [ev() for _ in range(2)], [ev() for _ in range(2)]
    out_ready, out_free = [ev() for _ in range(2)], [ev() for _ in range(2)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    t0.record(stream)
    h2d.wait_event(t0)
    d2h.wait_event(t0)

    def load(i):
        b = i % 2
        with torch.cuda.stream(h2d):
            if i >= 2:
                h2d.wait_event(in_free[b])
            sin[b].copy_(hin.view_as(sin[b]), non_blocking=True)
            in_ready[b].record(h2d)
    load(0)
    for i in range(nsteps):
        b = i % 2
        if i + 1 < nsteps:
            load(i + 1)
        stream.wait_event(in_ready[b])
        flush.zero_()
        src_bank.data.copy_(sin[b], non_blocking=True)
        in_free[b].record(stream)
        step()
        if i >= 2:
            stream.wait_event(out_free[b])
        sout[b].copy_(dst_bank.data, non_blocking=True)
        out_ready[b].record(stream)
        with torch.cuda.stream(d2h):
            d2h.wait_event(out_ready[b])
            hout.view_as(sout[b]).copy_(sout[b], non_blocking=True)
            out_free[b].record(d2h)
    stream.wait_stream(d2h)
    t1.record(stream)
    t1.synchronize()
    torch.cuda.synchronize(dev)
    return t0.elapsed_time(t1)


def _max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _fp64_line(args, stream, flush, fin32):
    import torch
    from frfs_b200 import _lib
    from frfs_b200.backend import B200Backend
    from frfs_b200.scattering import DGFSVHSGLLScatteringModel
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    a = argparse.Namespace(**vars(args))
    a.precision = 'double'
    cfg = _cfg(a)
    be = B200Backend(cfg, device=fin32.backend.device)
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    f = fin32.get().astype(np.float64)
    fin = be.matrix(f.shape, f)
    fout = be.matrix(f.shape)
    npts = f.shape[0]*f.shape[2]
    # the autotuner picks the FP64 launch shape on this bank as well
    tune = sm.autotune(fin, fout, cache=False)
    sm.fs_all(fin, fout)
    sm.status()
    ms = float(np.mean(_timed(lambda: sm.fs_all(fin, fout), 3, stream,
                              flush)))
    sm.status()
    tf = _lib.c_double()
    pms = _lib.ct.c_float()
    _lib.check(_lib.load().dgfs_probe_fma_peak(
        64, 1024, _lib.ct.byref(tf), _lib.ct.byref(pms), stream.cuda_stream),
        'dgfs_probe_fma_peak')
    achieved = sm.flops_per_point()*npts/(ms*1e-3)/1e12
    kind = sm.variants()[getattr(sm, '_variant', 0)]['exchange']
    torch.cuda.synchronize()
    return {'metric': METRIC, 'value': npts/(ms*1e-3), 'unit': 'evals/s',
            'dtype': 'f64', 'sweep_ms': ms, 'points': npts,
            'kernel': {'push': 'vhs_push_kernel',
                       'pull': 'vhs_cluster_kernel'}.get(kind, kind),
            'launch': sm.variants()[getattr(sm, '_variant', 0)],
            'ms_by_variant': tune.get('all_ms', {}),
            'roofline': {'bound': 'fp64-simt', 'achieved': achieved,
                         'peak': tf.value, 'unit': 'TFLOP/s',
                         'frac': achieved/tf.value,
                         'peak_source': 'measured in this run: FP64 FMA '
                                        'loop on every SM '
                                        '(dgfs_probe_fma_peak)'}}


def run_b200(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120))

    from frfs_b200 import _lib
    from frfs_b200.backend import B200Backend
    from frfs_b200.scattering import DGFSVHSGLLScatteringModel
    from frfs_b200.velocitymesh import DGFSVelocityMesh

    part = world > 1 and args.mode == 'step'
    cfg = _cfg(args, world if part else 1)
    be = B200Backend(cfg, device=f'cuda:{local}')
    nupts, neles = _points_shape(cfg, world if part else 1)
    npts = nupts*neles
    stream = torch.cuda.current_stream()
    flush = torch.empty(256*1024*1024 // 4, dtype=torch.float32,
                        device=be.device)

    if args.mode == 'step':
        from frfs_b200.steppers import StdTVDRK2DGFSStepper
        from frfs_b200.system import DGFSSystem
        cfg.set('backend-b200', 'cuda-graphs', int(args.graphs))
        vm0 = DGFSVelocityMesh(None, cfg)
        # synthetic noisy Maxwellians, or (--initial workload) the
        # workload's own initial condition, filled on the device when it is
        # uniform in space (banks too large for a host copy)
        f0 = (_synthetic_f(vm0.cv(), nupts, neles, seed=rank)
              if args.initial == 'synthetic' else None)
        mesh, prank = None, 0
        if part:
            # spatial partitions: rank r runs part r of the widened mesh
            # and exchanges face values with its neighbours over NCCL
            from frfs_b200 import mesh as meshmod
            from frfs_b200 import partition as pt
            whole = meshmod.from_config(cfg)
            mesh, _ = pt.partition_mesh(whole, pt.partition_elements(
                whole['spt_quad_p0'], world))
            prank = rank
        system = DGFSSystem(be, cfg, mesh=mesh, prank=prank, initsoln=f0)
        if part:
            # every rank joins one collective before the first
            # point-to-point exchange (NCCL communicator set-up)
            dist.barrier()
        # residual launch shape: timed on this mesh, fastest kept (setup,
        # not timed; bank 1 is scratch before the first step)
        dg_tune = system.autotune_dg(0, 1)
        vm, sm = system.vm, system.sm
        stepper = StdTVDRK2DGFSStepper(system, cfg)
        fin, fout = system.bank[0], system.bank[1]
        evals_per_step = 2*npts
        # per stage: VHS, interp, residual, the two boundary-sum kernels
        # when the part has boundary flux points, the pack kernel when it
        # has faces shared with other parts
        launches_per_step = 2*(3 + (2 if len(system.bpts) else 0) +
                               (1 if system.halo is not None else 0))

        def step():
            stepper.advance(1)
    else:
        vm = DGFSVelocityMesh(be, cfg)
        sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
        V = vm.vsize()
        f0 = _synthetic_f(vm.cv(), nupts, neles, seed=rank)
        fin = be.matrix((nupts, V, neles), f0)
        fout = be.matrix((nupts, V, neles))
        evals_per_step = npts
        launches_per_step = 1

        def step():
            sm.fs_all(fin, fout)

    # project-written autotuner: time every compiled launch shape on this
    # bank (setup, not timed) and keep the fastest
    if args.variant >= 0:
        sm.select(args.variant)
        tune = {'variant': sm.variants()[args.variant], 'all_ms': {}}
        tune_idx = args.variant
    else:
        tune = sm.autotune(fin, fout, cache=False)
        tune_idx = getattr(sm, "_variant", 0)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    times = _timed(step, args.steps, stream, flush)
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_ms = _max_over_ranks(float(np.sum(times)), world, be.device)
    if world > 1:
        dist.barrier()
    ms_per_step = t_ms/args.steps
    value = world*evals_per_step*args.steps/(t_ms*1e-3)

    # end to end through the public API: every step's distribution comes
    # from pinned host memory and its result goes back to pinned host
    # memory, all inside the timed region
    e2e = None
    if args.e2e:
        src_bank = fin
        dst_bank = fin if args.mode == 'step' else fout
        hin = torch.empty(src_bank.data.numel(), dtype=src_bank.data.dtype,
                          pin_memory=True)
        hin.copy_(src_bank.data.cpu())
        hout = torch.empty_like(hin, pin_memory=True)
        for _ in range(2):
            src_bank.data.copy_(hin, non_blocking=True)
            step()
            hout.copy_(dst_bank.data, non_blocking=True)
        torch.cuda.synchronize()
        te = _max_over_ranks(_e2e_pipelined(step, src_bank, dst_bank, hin,
                                            hout, args.steps, stream, flush),
                             world, be.device)
        e2e = {'value': world*evals_per_step*args.steps/(te*1e-3),
               'unit': 'evals/s',
               'h2d_bytes_per_step': int(hin.numel()*hin.element_size()),
               'd2h_bytes_per_step': int(hout.numel()*hout.element_size()),
               'copies': 'host to device and device to host on their own '
                         'streams, double-buffered in device memory, '
                         'overlapping the neighbouring steps; the first '
                         'input and the last result are inside the timed '
                         'region; L2 flushed before every step'}
        del hin, hout

    # dominant kernel: the fused VHS launch, timed alone on the same bank
    prec = 64 if args.precision == 'double' else 32
    vhs_ms = float(np.mean(_timed(lambda: sm.fs_all(fin, fout),
                                  max(2, min(args.steps, 5)), stream,
                                  flush)))
    tf = _lib.c_double()
    pms = _lib.ct.c_float()
    _lib.check(_lib.load().dgfs_probe_fma_peak(
        prec, 4096, _lib.ct.byref(tf), _lib.ct.byref(pms),
        stream.cuda_stream), 'dgfs_probe_fma_peak')
    flops_pt = sm.flops_per_point()
    achieved = flops_pt*npts/(vhs_ms*1e-3)/1e12
    # DRAM traffic of the launch is not measured by this run (it needs an
    # ncu capture); it is reported only from a capture of this exact kernel,
    # workload, size and precision (TRAFFIC), else null
    kind = None
    try:
        kind = sm.variants()[tune_idx]['exchange']
    except Exception:
        pass
    kname = {'single-cta': 'vhs_cube_kernel', 'push': 'vhs_push_kernel',
             'pair': 'vhs_pair_kernel',
             'pull': 'vhs_cluster_kernel'}.get(kind, kind)
    tkey = (kname, args.workload, npts, prec)
    traffic, tsrc = TRAFFIC.get(tkey, (None, None))
    roof = {'bound': 'fp32-simt' if prec == 32 else 'fp64-simt',
            'achieved': achieved, 'peak': tf.value, 'unit': 'TFLOP/s',
            'frac': achieved/tf.value,
            'peak_source': 'measured in this run: FMA loop on every SM '
                           '(dgfs_probe_fma_peak)',
            'flops_per_point': flops_pt, 'launch_ms': vhs_ms,
            'traffic': traffic,
            'traffic_source': ('ncu dram__bytes_read.sum + '
                               'dram__bytes_write.sum of this kernel: ' +
                               tsrc) if traffic
            else 'not captured for this kernel/workload/size/precision',
            'kernel': kname}
    extra = {}
    if args.mode == 'step':
        extra['dg_step_ms'] = ms_per_step
        # DG residual + RK combination, HBM bound: time it alone, replayed
        # from a CUDA graph as the solver's stages are (--graphs 1; the
        # partitioned stage, with its collective, runs eagerly)
        def dg_stage():
            system.rk_stage(1, 0, 0.5, 0, 0.5, 1, 1e-3, 2, interp=True)
        dg_fn = dg_stage
        if args.graphs and system.halo is None:
            dg_stage()
            torch.cuda.synchronize()
            dg_graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(dg_graph):
                dg_stage()
            dg_fn = dg_graph.replay
        dg_ms = float(np.mean(_timed(dg_fn, max(2, min(args.steps, 5)),
                                     stream, flush)))
        dg_fn = dg_graph = None
        esz = 8 if prec == 64 else 4
        U, F, V = system.nupts, system.nfpts, vm.vsize()
        # interp: read u, write uf; residual: read u, A, B, C, uf of the
        # partners, write out
        dg_bytes = (U + F + 4*U + F + U)*V*neles*esz
        peaks = {}
        try:
            with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
                peaks = json.load(fh)
        except (OSError, ValueError):
            pass
        hbm = peaks.get('hbm_gbs', 6650.0)
        dg_traffic, dg_tsrc = DG_TRAFFIC.get((args.workload, npts, prec),
                                             (None, None))
        extra['dg_roofline'] = {
            'bound': 'hbm', 'achieved': dg_bytes/(dg_ms*1e-3)/1e9,
            'peak': hbm, 'unit': 'GB/s',
            'frac': dg_bytes/(dg_ms*1e-3)/1e9/hbm,
            'peak_source': 'MEASURED_PEAKS.json hbm_gbs' if peaks
            else 'fallback 6650 GB/s',
            'bytes_per_launch': dg_bytes, 'launch_ms': dg_ms,
            'traffic': dg_traffic,
            'traffic_source': ('ncu dram__bytes_read.sum + '
                               'dram__bytes_write.sum: ' + dg_tsrc)
            if dg_traffic else 'not captured for this workload/size/'
                               'precision',
            'kernels': 'dg_interp_kernel + dg_residual_kernel',
            'residual_shape': system.dg_variants()[system._dg_shape],
            'ms_by_shape': dg_tune}
    launch = sm.launch_info()

    if rank == 0 and world == 1 and args.precision == 'single' and \
            npts <= 20000:
        # the FP64 mode on the same points: one collision sweep in full
        # double precision (the parity mode), against the FP64 FMA peak
        extra['fp64'] = _fp64_line(args, stream, flush, fin)

    sur = None
    want_sur = args.surrogate if args.surrogate >= 0 else int(
        args.workload == 'couette-n24' and world == 1 and
        args.mode == 'step')
    if want_sur and world == 1:
        # learned surrogate: harvested from the solver, trained with the
        # project's kernels, measured against the plain FP64 solution
        from frfs_b200 import workloads
        from frfs_b200.surrogate_study import run_study
        sur = run_study(workloads.WORKLOADS[args.workload],
                        device=be.device, nsteps=args.surrogate_steps,
                        steps=args.surrogate_harvest_steps,
                        sphdesign=SPHDESIGN, extra_thresholds=(0.1, 0.2))

    if rank == 0:
        cb = None
        if world == 1 and not args.no_cpu_baseline:
            cb = _cpu_baseline(cfg, args.cpu_seconds)[0]
        line = {
            'metric': METRIC, 'value': value, 'unit': 'evals/s',
            'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': ms_per_step, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f32' if prec == 32 else 'f64',
            'data': 'synthetic',
            'config': _workload_desc(args, cfg, npts, world),
            'clocks': clk, 'e2e': e2e,
            'gpu_launches': args.steps*launches_per_step,
            'roofline': roof, 'cpu_baseline': cb,
            'launch': launch,
            'autotune': {'selected': tune['variant'],
                         'ms_by_variant': tune['all_ms']},
        }
        line.update(extra)
        if sur is not None:
            line['surrogate'] = sur
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_mixture(args):
    """Binary-mixture VSS operator (frfs's dgfsbi 'vss-gll'): Q_p =
    sum_q Q(f_p, f_q) for both species at every point of a 576-point bank
    (the Couette layout, 9 x 64), one persistent launch per ordered pair.
    One step is one sweep; evaluations count one Q_p per species and point."""
    import torch
    from frfs_b200 import _lib, workloads
    from frfs_b200.backend import B200Backend
    from frfs_b200.inifile import Inifile
    from frfs_b200.mixture import (DGFSBiVelocityMesh,
                                   DGFSBiVSSGLLScatteringModel)
    cfg = Inifile(workloads.MIXTURES[args.workload](precision=args.precision))
    cfg.set('spherical-design-rule', 'path', SPHDESIGN)
    torch.cuda.set_device(0)
    be = B200Backend(cfg, device='cuda:0')
    vm = DGFSBiVelocityMesh(be, cfg)
    sm = DGFSBiVSSGLLScatteringModel(be, cfg, vm)
    nupts, neles = 9, 64
    npts = nupts*neles
    V = vm.vsize()
    m1, m2 = vm.masses()
    rng = np.random.default_rng(0)
    cv = vm.cv()
    c2 = np.sum(cv*cv, axis=0)
    fs = []
    for nden, m in ((0.6, m1), (0.4, m2)):
        mx = nden*(m/np.pi)**1.5*np.exp(-m*c2)
        fs.append(mx[None, :, None] *
                  (1.0 + 0.01*rng.standard_normal((nupts, V, neles))))
    f0, f1 = (be.matrix((nupts, V, neles), f) for f in fs)
    q0, q1 = be.matrix((nupts, V, neles)), be.matrix((nupts, V, neles))
    stream = torch.cuda.current_stream()
    flush = torch.empty(256*1024*1024 // 4, dtype=torch.float32,
                        device=be.device)

    def step():
        sm.fs_all(f0, f1, q0, q1)
    for _ in range(args.warmup):
        step()
    sm.status()
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    times = _timed(step, args.steps, stream, flush)
    torch.cuda.synchronize()
    clk = clocks.stop()
    sm.status()
    t_ms = float(np.sum(times))
    evals = 2*npts
    value = evals*args.steps/(t_ms*1e-3)
    # end to end: both species' banks in from pinned host memory, both
    # results back, every step
    hin = [torch.empty(x.data.numel(), dtype=x.data.dtype, pin_memory=True)
           for x in (f0, f1)]
    for h, x in zip(hin, (f0, f1)):
        h.copy_(x.data.cpu())
    hout = [torch.empty_like(h, pin_memory=True) for h in hin]

    def e2e_step():
        for h, x in zip(hin, (f0, f1)):
            x.data.copy_(h.view_as(x.data), non_blocking=True)
        step()
        for h, x in zip(hout, (q0, q1)):
            h.view_as(x.data).copy_(x.data, non_blocking=True)
    e2e_step()
    torch.cuda.synchronize()
    te = float(np.sum(_timed(e2e_step, args.steps, stream, flush)))
    nbytes = int(sum(h.numel()*h.element_size() for h in hin))
    prec = 64 if args.precision == 'double' else 32
    tf = _lib.c_double()
    pms = _lib.ct.c_float()
    _lib.check(_lib.load().dgfs_probe_fma_peak(
        prec, 4096 if prec == 32 else 1024, _lib.ct.byref(tf),
        _lib.ct.byref(pms), stream.cuda_stream), 'dgfs_probe_fma_peak')
    achieved = sm.flops_per_point()*npts/(t_ms/args.steps*1e-3)/1e12
    line = {
        'metric': METRIC, 'value': value, 'unit': 'evals/s', 'n_gpus': 1,
        'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': t_ms/args.steps, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32' if prec == 32 else 'f64', 'data': 'synthetic',
        'config': {'workload': f'{args.workload}: binary-mixture VSS Q_p '
                               f'at every point, both species',
                   'points': npts, 'Nv': vm.Nv(), 'Nrho': vm.Nrho(),
                   'M': vm.M(), 'species': 2, 'mode': 'collide',
                   'l2': 'flushed between timed steps (256 MiB write)'},
        'clocks': clk,
        'e2e': {'value': evals*args.steps/(te*1e-3), 'unit': 'evals/s',
                'h2d_bytes_per_step': nbytes, 'd2h_bytes_per_step': nbytes},
        'gpu_launches': 4*args.steps,
        'roofline': {'bound': 'fp32-simt' if prec == 32 else 'fp64-simt',
                     'achieved': achieved, 'peak': tf.value,
                     'unit': 'TFLOP/s', 'frac': achieved/tf.value,
                     'peak_source': 'measured in this run: FMA loop on '
                                    'every SM (dgfs_probe_fma_peak)',
                     'flops_per_point': sm.flops_per_point(),
                     'launch_ms': t_ms/args.steps, 'traffic': None,
                     'traffic_source': 'not captured',
                     'kernel': ('vss_pair_kernel' if prec == 32 and
                                round(V**(1/3)) == 24 else 'vss_push_kernel') +
                               ' (4 launches, one per ordered pair)'},
        'cpu_baseline': None,
    }
    print(json.dumps(line))


def main():
    args = _parse()
    from frfs_b200 import workloads
    if args.workload in workloads.MIXTURES:
        if args.impl == 'reference':
            print(json.dumps({'impl': 'reference', 'unavailable':
                              'the reference arm times the VHS workloads'}))
            return
        run_mixture(args)
    elif args.impl == 'reference':
        run_reference(args)
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
