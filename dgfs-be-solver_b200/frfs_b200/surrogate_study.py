# -*- coding: utf-8 -*-
"""Train the collision surrogate on the solver's own trajectories and measure
its error with the plain operator (no counterpart in the reference).

``run_study`` does, on one GPU:

1. harvest (f, Q(f)) pairs from the plain FP32 solver started from random
   uniform states (Maxwellians with rho in [0.5, 2], T in [0.5, 3],
   |u| <= 1, and bimodal mixtures; and Maxwellians at a log-uniform
   distance from the reference state, whose mismatch with the walls covers
   weak to strong wall fronts), and from space-homogeneous relaxations of
   random per-point states (which cross every distance from equilibrium);
2. train the MLP with the project's kernels;
3. run the workload from its own initial state: plain FP64 (the reference
   solution; once more with the conservation projection, the solution the
   projected surrogate output tends to), plain FP32, surrogate-assisted
   FP32 (with a sampled residual
   check every ``check_every`` steps that drops the surrogate when it
   fails), the same without checks, and an ablation in which the gated
   points get Q = 0 (the gate without the network);
4. report the relative L2 errors of rho, u and T against the FP64 solution
   and the Q(f) evaluations per second of a plain and of a
   surrogate-assisted collision sweep on the final state.
"""

import time

import numpy as np
import torch

from frfs_b200.backend import B200Backend
from frfs_b200.initcond import initial_distribution
from frfs_b200.inifile import Inifile
from frfs_b200.steppers import StdTVDRK2DGFSStepper
from frfs_b200.surrogate import VHSSurrogate, harvest, harvest_relaxation
from frfs_b200.system import DGFSSystem


class ZeroSurrogate(VHSSurrogate):
    """The gate without the network: gated points get Q = 0."""

    def predict(self, X, rows=None, count=None):
        Bp = self.ws.get('Bp0', (X.shape[0], X.shape[1]))
        Bp.zero_()
        return Bp


def make_system(ini, precision, device, sphdesign=None, graphs=True,
                project=False):
    """The workload's system, with the reference operator (no conservation
    projection) unless ``project``: the projection removes the operator's
    own spectral conservation error, which changes the solution against the
    reference's by more than FP32 round-off does (Couette, 200 steps: u
    4.7e-4 with it, 5.7e-5 without)."""
    cfg = Inifile(ini(precision=precision))
    if sphdesign:
        cfg.set('spherical-design-rule', 'path', sphdesign)
    cfg.set('backend-b200', 'cuda-graphs', '1' if graphs else '0')
    cfg.set('backend-b200', 'vhs-project', '1' if project else '0')
    be = B200Backend(cfg, device=device)
    return DGFSSystem(be, cfg)


def _reset(system):
    nupts, V, neles = system.bank[0].ioshape
    system.bank[0].set(initial_distribution(system.cfg, system.vm, nupts,
                                            neles))


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b)/np.linalg.norm(b))


def run_workload(system, nsteps, sur=None, check_every=0, tol=5e-3,
                 scratch=None):
    """nsteps SSP-RK2 steps from the workload's initial state; returns the
    final (rho, u, T), the bank index and the record of the run: residual
    checks, and the device time of the steps (CUDA events around every
    stretch of steps, the residual checks between them excluded), so that
    the step time is an average over the whole trajectory.  One untimed
    step from the initial state comes first and is discarded: it captures
    the stage graphs (a one-time set-up) outside the timed steps."""
    system.surrogate = sur
    _reset(system)
    st = StdTVDRK2DGFSStepper(system, system.cfg)
    t0 = st.tcurr
    st.advance(1)
    torch.cuda.synchronize(system.backend.device)
    _reset(system)
    st._idxcurr, st.tcurr = 0, t0
    fallbacks, checks, worst = [], 0, 0.0
    done = 0
    dev = system.backend.device
    stream = torch.cuda.current_stream(dev)
    step_ms = 0.0
    while done < nsteps:
        n = min(check_every or nsteps, nsteps - done)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st.advance(n)
        e1.record(stream)
        e1.synchronize()
        step_ms += e0.elapsed_time(e1)
        done += n
        if sur is not None and check_every and system.surrogate is not None \
                and done < nsteps:
            cur = system.bank[st._idxcurr]
            sur.collide(cur, scratch[0])
            r = sur.residual_check(cur, scratch[0], scratch[1], seed=done)
            checks += 1
            worst = max(worst, r)
            if r > tol:
                fallbacks.append(done)
                system.surrogate = None
    torch.cuda.synchronize(system.backend.device)
    m = system.moments(st._idxcurr)
    system.surrogate = None
    return ((m[..., 0], m[..., 1:4], m[..., 4]), st._idxcurr,
            {'checks': checks, 'worst_residual': worst,
             'fallback_at_step': fallbacks,
             'ms_per_step': step_ms/max(nsteps, 1)})


def time_sweep(fn, reps, device):
    """Mean device time (ms) of fn() over reps calls (CUDA events)."""
    s = torch.cuda.current_stream(device)
    fn()
    torch.cuda.synchronize(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.synchronize(device)
    return e0.elapsed_time(e1)/reps


def run_study(ini, device='cuda:0', runs=5, near_runs=10, steps=100,
              nsteps=200,
              epochs=60, batch=1024, lr=1e-3, threshold=0.05, eps_max=0.2,
              check_every=50, tol=5e-3, reps=10, sphdesign=None, seed=1,
              max_pairs=200000, relax_points=576, relax_steps=100,
              relax_dt=0.005, extra_thresholds=None, log=None):
    t0 = time.time()
    say = log or (lambda *a: None)
    s32 = make_system(ini, 'single', device, sphdesign)
    npts = s32.nupts*s32.neles
    sur = VHSSurrogate(s32.sm, threshold=threshold, seed=0)

    # 1. data from the plain solver's trajectories
    th = time.time()
    X, B = harvest(s32, StdTVDRK2DGFSStepper, sur, runs, steps, seed=seed,
                   eps_max=eps_max, max_pairs=max_pairs)
    if near_runs:
        Xn, Bn = harvest(s32, StdTVDRK2DGFSStepper, sur, near_runs, steps,
                         seed=seed + 1000, eps_max=eps_max,
                         max_pairs=max_pairs, near=True)
        X, B = torch.cat([X, Xn]), torch.cat([B, Bn])
        del Xn, Bn
    npairs_solver = int(X.shape[0])
    if relax_steps:
        Xr, Br = harvest_relaxation(s32.sm, sur, relax_points, relax_steps,
                                    relax_dt, seed=seed, eps_max=eps_max,
                                    max_pairs=max_pairs)
        X, B = torch.cat([X, Xr]), torch.cat([B, Br])
        del Xr, Br
    torch.cuda.synchronize(device)
    t_harvest = time.time() - th
    npairs = int(X.shape[0])
    say(f'harvest: {npairs_solver} solver pairs, {npairs} in total, '
        f'in {t_harvest:.1f} s')

    # 2. training
    tt = time.time()
    sur.set_normalisation(X, B)
    hist = sur.train(X, B, epochs=epochs, batch=batch, lr=lr)
    torch.cuda.synchronize(device)
    t_train = time.time() - tt
    rows = (npairs//min(batch, npairs))*min(batch, npairs)*epochs
    train_tflops = sur.mlp.train_flops_per_row()*rows/t_train*1e-12
    say(f'train: loss {hist[0]:.3e} -> {hist[-1]:.3e} in {t_train:.1f} s '
        f'({train_tflops:.1f} TFLOP/s)')
    del X, B

    # 3. the workload from its own initial state
    s64 = make_system(ini, 'double', device, sphdesign)
    (r64, u64, T64), _, _ = run_workload(s64, nsteps)
    del s64
    torch.cuda.empty_cache()
    # the same with the conservation projection: the surrogate's output is
    # projected, so against this solution its error is that of the network
    # and the gate alone, without the plain operator's own conservation error
    s64 = make_system(ini, 'double', device, sphdesign, project=True)
    (p64, v64, S64), _, _ = run_workload(s64, nsteps)
    del s64
    torch.cuda.empty_cache()
    (r32, u32, T32), _, rec32 = run_workload(s32, nsteps)
    zero = ZeroSurrogate(s32.sm, threshold=threshold)
    (rz, uz, Tz), _, _ = run_workload(s32, nsteps, zero)
    (rn, un, Tn), _, recn = run_workload(s32, nsteps, sur)
    scratch = [s32.backend.matrix(s32.bank[0].ioshape) for _ in range(2)]
    (rs, us, Ts), idx, chk = run_workload(s32, nsteps, sur, check_every,
                                          tol, scratch)

    def errs(r, u, T):
        return {'rho': rel_l2(r, r64), 'u': rel_l2(u, u64),
                'T': rel_l2(T, T64)}

    def errs_proj(r, u, T):
        return {'rho': rel_l2(r, p64), 'u': rel_l2(u, v64),
                'T': rel_l2(T, S64)}

    # the gate threshold: error and speed of the surrogate run at others
    sweep = {}
    for thr in (extra_thresholds or ()):
        sur.threshold = zero.threshold = thr
        (ra, ua, Ta), _, _ = run_workload(s32, nsteps, zero)
        (rt, ut, Tt), it, rect = run_workload(s32, nsteps, sur)
        ft, ot = s32.bank[it], scratch[0]
        tp = time_sweep(lambda: s32.sm.fs_all(ft, ot), reps, device)
        ts = time_sweep(lambda: sur.collide(ft, ot), reps, device)
        sweep[str(thr)] = {'err': errs(rt, ut, Tt),
                           'err_gate_without_network': errs(ra, ua, Ta),
                           'err_vs_projected_fp64': errs_proj(rt, ut, Tt),
                           'err_gate_without_network_vs_projected_fp64':
                           errs_proj(ra, ua, Ta),
                           'speedup': tp/ts,
                           'step_ms': rect['ms_per_step'],
                           'step_speedup_over_run':
                           rec32['ms_per_step']/rect['ms_per_step'],
                           'gate_fraction':
                           float((sur._last[0] != 0).float().mean())}
    sur.threshold = zero.threshold = threshold

    # 4. throughput of one collision sweep on the surrogate run's final state
    fin = s32.bank[idx]
    out = scratch[0]
    t_plain = time_sweep(lambda: s32.sm.fs_all(fin, out), reps, device)
    t_sur = time_sweep(lambda: sur.collide(fin, out), reps, device)
    g = sur._last[0]
    gfrac = float((g != 0).float().mean())
    gzero = float((g == 2).float().mean())
    eps = sur._last[1].cpu().numpy()
    return {
        'points': npts, 'pairs': npairs, 'pairs_solver': npairs_solver,
        'train_loss_first': hist[0], 'train_loss_last': hist[-1],
        'harvest_s': t_harvest, 'train_s': t_train,
        'train_tflops': train_tflops,
        'train_products': {'tma': 'tensor cores, TMA-fed BF16 operands',
                           'staged': 'tensor cores, operands staged by the '
                                     'threads',
                           False: 'SIMT'}[sur.mlp.tc],
        'epochs': epochs, 'runs': runs, 'near_runs': near_runs,
        'steps_per_run': steps,
        'nsteps': nsteps, 'threshold': threshold,
        'step_ms_plain': rec32['ms_per_step'],
        'step_ms_surrogate': recn['ms_per_step'],
        'step_ms_surrogate_with_checks': chk['ms_per_step'],
        'step_speedup_over_run': rec32['ms_per_step']/recn['ms_per_step'],
        'err_surrogate': errs(rs, us, Ts),
        'err_surrogate_without_checks': errs(rn, un, Tn),
        'err_plain_fp32': errs(r32, u32, T32),
        'err_gate_without_network': errs(rz, uz, Tz),
        'err_vs_projected_fp64': {
            'surrogate_without_checks': errs_proj(rn, un, Tn),
            'gate_without_network': errs_proj(rz, uz, Tz),
            'plain_fp32': errs_proj(r32, u32, T32),
            'plain_fp64_unprojected': errs_proj(r64, u64, T64)},
        'residual_checks': chk,
        'gate_fraction': gfrac, 'relaxation_only_fraction': gzero,
        'eps_quantiles': [float(q) for q in
                          np.quantile(eps, [0.1, 0.5, 0.9, 0.99])],
        'plain_ms_per_sweep': t_plain, 'surrogate_ms_per_sweep': t_sur,
        'plain_evals_per_s': npts/(t_plain*1e-3),
        'surrogate_evals_per_s': npts/(t_sur*1e-3),
        'speedup': t_plain/t_sur,
        'threshold_sweep': sweep,
        'wall_s': time.time() - t0,
    }


if __name__ == '__main__':
    import argparse
    import os

    from frfs_b200 import workloads
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--workload', default='couette-n24')
    ap.add_argument('--sphdesign', default=os.path.join(
        os.path.dirname(__file__), 'data', 'sphericaldesign'))
    args = ap.parse_args()
    ini = workloads.WORKLOADS[args.workload]
    sph = os.path.abspath(args.sphdesign)
    import json
    print(json.dumps(run_study(ini, sphdesign=sph,
                               log=lambda m: print(m, flush=True))))
