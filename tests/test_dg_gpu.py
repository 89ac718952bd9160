# -*- coding: utf-8 -*-
"""Parity of the B200 FR-DG kernels with the FP64 oracle (GPU).

Tolerances (normwise relative): FP64 1e-10, FP32 2e-5.
"""

import numpy as np
import pytest
import torch

from helpers import config, dg_setup, oracle_for, random_states, rel_err
from frfs_b200 import mesh as mgen
from frfs_b200.backend import B200Backend
from frfs_b200.system import DGFSSystem
from oracle import dg as odg
from oracle import vhs as ovhs

pytestmark = pytest.mark.gpu

TOL = {'double': 1e-10, 'single': 2e-5}


def _cfg(precision, bottom='dgfs-wall-diffuse', top='dgfs-wall-diffuse',
         order=2, batch=None):
    cfg = config('relax0d-n16', precision)
    cfg.set('solver', 'order', order)
    if batch:
        cfg.set('constants', 'NvBatchSize', batch)
    u0 = np.sqrt(2*8.3144598/39.96e-3*273.0)
    for name, kind, uy in (('bottom', bottom, -0.3), ('top', top, 0.4)):
        sect = f'soln-bcs-{name}'
        cfg.set(sect, 'type', kind)
        cfg.set(sect, 'rho', 1.5e-3)
        cfg.set(sect, 'T', 273.0*(1.1 if name == 'top' else 0.9))
        cfg.set(sect, 'ux', 0.1*u0)
        cfg.set(sect, 'uy', 0.0 if kind == 'dgfs-inlet' else uy*u0)
        cfg.set(sect, 'uz', 0.0)
        if kind == 'dgfs-wall-diffuse-cyl':
            # a wall state that varies along the wall (x in [0, 1])
            cfg.set(sect, 'ux', f'{0.1*u0}*(1 + y)')
            cfg.set(sect, 'uy', f'{uy*u0}*x')
            cfg.set(sect, 'T', '273*(0.9 + 0.2*x)')
    return cfg


def _mesh(order=2):
    return mgen.quad_box(4, 3, 0.0, 1.0, 0.0, 0.75, periodic_x=True,
                         jitter=0.2, seed=order)


def _system(cfg, mesh, u):
    be = B200Backend(cfg, device='cuda:0')
    sys_ = DGFSSystem(be, cfg, mesh=mesh, initsoln=u)
    return be, sys_


def _states(vm, nupts, neles, seed=0):
    f = random_states(vm.cv(), nupts*neles, seed=seed, noise=0.02)
    return f.reshape(nupts, neles, -1).transpose(0, 2, 1).copy()


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('order', [1, 2, 3])
def test_residual_and_wall_sums(precision, order):
    cfg, m = _cfg(precision, order=order), _mesh(order)
    dg, sh, geo, vm = dg_setup(cfg, m)
    u = _states(vm, sh.nupts, geo.neles, seed=order)
    be, s = _system(cfg, m, u)
    u_used = s.bank[0].get().astype(np.float64)
    s.updatebc(0.0, 0, 1, 0, 0)
    s.rhs(0.0, 0, 1, 0, 0)
    torch.cuda.synchronize()
    # face values and diffuse-wall sums
    uf = dg.disu(u_used)
    assert rel_err(s.face_values(), uf) < TOL[precision]
    dg.update_bc(uf)
    bcg = s.bc_values()
    for b, (g, j, e) in enumerate(s.bpts):
        name = sorted(dg.bpts)[g]
        k = dg.bpts[name].index((j, e))
        ref = dg.bcvals[name][:, k]
        assert abs(bcg[b, 0] - ref[0]) <= TOL[precision]*abs(ref[0]) + 1e-14
        assert abs(bcg[b, 1] - ref[1]) <= TOL[precision]*abs(ref[1]) + 1e-14
    R = dg.rhs(u_used, uf)
    err = rel_err(s.bank[1].get(), R)
    assert err < TOL[precision], err


@pytest.mark.parametrize('kinds', [('dgfs-inlet', 'dgfs-outlet'),
                                   ('dgfs-vanish', 'dgfs-wall-specular'),
                                   ('dgfs-wall-specular', 'dgfs-wall-diffuse'),
                                   ('dgfs-wall-diffuse-cyl',
                                    'dgfs-inlet-normalshock')])
def test_boundary_kinds(kinds):
    cfg, m = _cfg('double', *kinds), _mesh()
    dg, sh, geo, vm = dg_setup(cfg, m)
    u = _states(vm, sh.nupts, geo.neles, seed=7)
    be, s = _system(cfg, m, u)
    s.updatebc(0.0, 0, 1, 0, 0)
    s.rhs(0.0, 0, 1, 0, 0)
    torch.cuda.synchronize()
    uf = dg.disu(u)
    dg.update_bc(uf)
    assert rel_err(s.bank[1].get(), dg.rhs(u, uf)) < TOL['double']


def test_velocity_batches_match_full_range():
    cfg, m = _cfg('double', batch=1024), _mesh()
    dg, sh, geo, vm = dg_setup(cfg, m)
    u = _states(vm, sh.nupts, geo.neles, seed=3)
    be, s = _system(cfg, m, u)
    for b in range(vm.NvBatches()):
        s.updatebc(0.0, 0, 1, b, b*vm.NvBatchSize())
    for b in range(vm.NvBatches()):
        s.rhs(0.0, 0, 1, b, b*vm.NvBatchSize())
    torch.cuda.synchronize()
    uf = dg.disu(u)
    dg.update_bc(uf)
    assert rel_err(s.bank[1].get(), dg.rhs(u, uf)) < TOL['double']


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('graphs', [0, 1])
def test_ssp_rk2_steps_match_oracle(precision, graphs):
    """Two SSP-RK2 steps (collision + advection) against the oracle."""
    from frfs_b200.steppers import StdTVDRK2DGFSStepper
    cfg, m = _cfg(precision), mgen.quad_box(2, 2, 0.0, 0.5, 0.0, 0.5,
                                            periodic_x=True, jitter=0.1)
    cfg.set('backend-b200', 'cuda-graphs', graphs)
    dg, sh, geo, vm = dg_setup(cfg, m)
    ovm, pre, prefac = oracle_for(cfg)
    u = _states(vm, sh.nupts, geo.neles, seed=5)
    be, s = _system(cfg, m, u)
    st = StdTVDRK2DGFSStepper(s, cfg)
    dt = 1e-3
    st.dt = dt
    st.advance(2)
    torch.cuda.synchronize()

    def Q(x):
        out = np.empty_like(x)
        for i in range(x.shape[0]):
            for e in range(x.shape[2]):
                out[i, :, e] = ovhs.vhs_Q(x[i, :, e], ovm, pre, prefac)
        return out

    # FP32 banks start from the rounded input
    u0 = u.astype(np.float32).astype(np.float64) if precision == 'single' \
        else u
    for _ in range(2):
        u0 = odg.ssp_rk2_step(dg, Q, u0, dt)
    err = rel_err(s.bank[st._idxcurr].get(), u0)
    assert err < (1e-10 if precision == 'double' else 1e-5), err


def _cylinder(precision, **kw):
    cfg = config('cylinder-n32', precision, ntheta=8, nr=2, Nv=24, Nrho=4,
                 M=6, **kw)
    return cfg, mgen.from_config(cfg)


def test_cylinder_ogrid_p3_residual():
    """The cylinder workload's discretisation at small size: p=3 on the
    O-grid, diffuse cylinder wall, Maxwellian inflow and outflow, against
    the oracle (FP64)."""
    cfg, m = _cylinder('double')
    dg, sh, geo, vm = dg_setup(cfg, m)
    assert sh.nupts == 16
    rng = np.random.default_rng(4)
    from frfs_b200.initcond import MaxwellianSection
    f0 = MaxwellianSection(cfg, vm, 'soln-ics').values
    u = f0[None, :, None]*(1 + 0.05*rng.standard_normal(
        (sh.nupts, vm.vsize(), geo.neles)))
    be, s = _system(cfg, m, u)
    s.updatebc(0.0, 0, 1, 0, 0)
    s.rhs(0.0, 0, 1, 0, 0)
    torch.cuda.synchronize()
    uf = dg.disu(u)
    dg.update_bc(uf)
    assert rel_err(s.bank[1].get(), dg.rhs(u, uf)) < TOL['double']


def test_cylinder_steps_run():
    """Two SSP-RK2 steps of the cylinder workload (FP32, collision and
    advection on the O-grid with its three boundary kinds): finite, and the
    density stays within a few per cent of the freestream's (the wall
    disturbance has had four stages of dt = 2e-4 to spread; the workload's
    own dt grows with the element size of this coarse 8 x 2 grid)."""
    from frfs_b200.steppers import StdTVDRK2DGFSStepper
    cfg, m = _cylinder('single', dt=2e-4)
    be = B200Backend(cfg, device='cuda:0')
    s = DGFSSystem(be, cfg, mesh=m)
    st = StdTVDRK2DGFSStepper(s, cfg)
    st.advance(2)
    torch.cuda.synchronize()
    f = s.bank[st._idxcurr].get()
    assert np.all(np.isfinite(f))
    rho = s.moments(st._idxcurr)[..., 0]
    assert np.all(np.isfinite(rho))
    assert np.max(np.abs(rho - 1.0)) < 0.05, np.max(np.abs(rho - 1.0))


def test_checkpoint_restart_continues_bit_for_bit(tmp_path):
    """Write a checkpoint after two SSP-RK2 steps, run two more; a new
    system restarted from the checkpoint reaches the same bank bit for
    bit (frfs's restart path, __main__.py:228-242, system.py:79-112)."""
    from frfs_b200 import checkpoint as ck
    from frfs_b200.steppers import StdTVDRK2DGFSStepper
    cfg, m = _cfg('single'), mgen.quad_box(2, 2, 0.0, 0.5, 0.0, 0.5,
                                           periodic_x=True, jitter=0.1)
    dg, sh, geo, vm = dg_setup(cfg, m)
    u = _states(vm, sh.nupts, geo.neles, seed=6)
    be, s = _system(cfg, m, u)
    st = StdTVDRK2DGFSStepper(s, cfg)
    st.dt = 1e-3
    st.advance(2)
    path = ck.write(str(tmp_path/'ck.npz'), s, st)
    st.advance(2)
    torch.cuda.synchronize()
    want = s.bank[st._idxcurr].get()

    rec = ck.read(path)
    s2 = DGFSSystem(B200Backend(cfg, device='cuda:0'), cfg, mesh=m,
                    initsoln=rec)
    st2 = StdTVDRK2DGFSStepper(s2, cfg)
    st2.dt = 1e-3
    st2.tcurr, st2.nacptsteps = ck.restart_time(rec)
    assert st2.nacptsteps == 2
    st2.advance(2)
    torch.cuda.synchronize()
    assert np.array_equal(s2.bank[st2._idxcurr].get(), want)


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('order', [1, 2, 3])
def test_invmass_matches_reference_operator(precision, order):
    """DGFSSystem.invmass (frfs/solvers/dgfs/system.py:221-231): the bank
    times M12, with M12 taken from the reference's own shapes fixture."""
    from conftest import GOLDEN
    M12 = np.load(f'{GOLDEN}/ref_shape_quad_p{order}.npz')['M12']
    cfg, m = _cfg(precision, order=order), _mesh(order)
    dg, sh, geo, vm = dg_setup(cfg, m)
    u = _states(vm, sh.nupts, geo.neles, seed=order + 10)
    be, s = _system(cfg, m, u)
    u_used = s.bank[0].get().astype(np.float64)
    s.invmass(0, 2)
    torch.cuda.synchronize()
    ref = np.einsum('ij,jve->ive', M12, u_used)
    assert rel_err(s.bank[2].get(), ref) < TOL[precision]


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('order', [2, 3])
def test_every_residual_shape_matches_oracle(precision, order):
    """Each compiled residual launch shape (velocities per warp, prefetch
    of the Runge-Kutta terms, register budget; in FP32 also the shapes
    whose element-operator contraction runs on the tensor cores) gives the
    oracle's out = a A + b B + g (L(u) + C), and autotune_dg keeps one of
    them."""
    cfg, m = _cfg(precision, order=order), _mesh(order)
    dg, sh, geo, vm = dg_setup(cfg, m)
    u = _states(vm, sh.nupts, geo.neles, seed=order + 20)
    be, s = _system(cfg, m, u)
    u_used = s.bank[0].get().astype(np.float64)
    uf = dg.disu(u_used)
    dg.update_bc(uf)
    R = dg.rhs(u_used, uf)
    ref = 0.3*u_used + 0.7*u_used + 2e-3*(R + u_used)
    s.updatebc(0.0, 0, 1, 0, 0)
    variants = s.dg_variants()
    ntc = sum(v['tensor_cores'] for v in variants)
    assert ntc == (4 if precision == 'single' else 0)
    for i in range(len(variants)):
        s.select_dg(i)
        s.updatebc(0.0, 0, 1, 0, 0)       # the shape's interp chunk too
        s.rk_stage(0, 1, 0.3, 0, 0.7, 0, 2e-3, 0, interp=False)
        torch.cuda.synchronize()
        assert rel_err(s.bank[1].get(), ref) < TOL[precision], i
    s.dg_status()
    ms = s.autotune_dg(0, 2)
    assert set(ms) == set(range(len(s.dg_variants())))
    assert s._dg_shape == min(ms, key=ms.get)
