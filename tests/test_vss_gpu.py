# -*- coding: utf-8 -*-
"""Binary-mixture VSS operator on the GPU against the FP64 oracle.

The product's mixture mesh, pair parameters and the C ABI
(dgfs_vss_create/apply) evaluate Q_p = sum_q Q(f_p, f_q) for an
argon-krypton mixture (frfs/solvers/dgfsbi/scattering.py:317-330); the
oracle (oracle/vss.py) restates the reference's operator in FP64.

Tolerances (normwise relative, as the VHS tests): FP64 1e-10, FP32 2e-4.
"""

import numpy as np
import pytest
import torch

from conftest import SPHDESIGN
from helpers import rel_err
from frfs_b200.backend import B200Backend
from frfs_b200.inifile import Inifile
from frfs_b200.mixture import DGFSBiVelocityMesh, DGFSBiVSSGLLScatteringModel
from oracle import vss

pytestmark = pytest.mark.gpu

TOL = {'double': 1e-10, 'single': 2e-4}


def mixture_config(precision, Nv=16, Nrho=6, M=12):
    keys = ('00', '01', '10', '11')
    sm = '\n'.join(f'alpha{k} = 1.4\nomega{k} = 0.75\ndRef{k} = 4.1e-10\n'
                   f'Tref{k} = 273.0' for k in keys)
    return Inifile(f"""
[backend]
precision = {precision}
[constants]
Nv = {Nv}
Nrho = {Nrho}
[non-dim]
T0 = 273.0
H0 = 1e-3
rho0 = 1.5e-3
molarMass0 = 39.96e-3
[velocity-mesh]
cmax = 0.0
Tmax = 273.0
dev = 5.0
molarMass1 = 39.96e-3
molarMass2 = 83.8e-3
[spherical-design-rule]
ssrule = womersley
M = {M}
path = {SPHDESIGN}
[scattering-model]
type = vss-gll
ssrulepre = womersley
Mpre = {M}
{sm}
""")


def _oracle(vm, cfg):
    mesh = vss.mixture_mesh(vm.Nv(), vm.Nrho(), vm.sz(),
                            [39.96e-3, 83.8e-3], H0=1e-3, T0=273.0,
                            rho0=1.5e-3, molarMass0=39.96e-3, cmax=0.0,
                            Tmax=273.0, dev=5.0)
    keys = ('00', '01', '10', '11')
    params = vss.vss_parameters(
        mesh, alpha={k: 1.4 for k in keys}, omega={k: 0.75 for k in keys},
        dRef={k: 4.1e-10 for k in keys}, Tref={k: 273.0 for k in keys})
    return mesh, params, vss.vss_precompute(mesh, params, vm.sz())


def _states(mesh, npts, seed):
    rng = np.random.default_rng(seed)
    m1, m2 = mesh['masses']
    out = []
    for _ in range(npts):
        u1, u2 = rng.uniform(-0.4, 0.4, (2, 3))
        T1, T2 = rng.uniform(0.7, 1.3, 2)
        f1 = vss.mixture_maxwellian(mesh['cv'], rng.uniform(0.4, 0.8), m1,
                                    u1, T1)
        f2 = vss.mixture_maxwellian(mesh['cv'], rng.uniform(0.2, 0.6), m2,
                                    u2, T2)
        out.append((f1*(1 + 0.01*rng.standard_normal(f1.size)),
                    f2*(1 + 0.01*rng.standard_normal(f2.size))))
    return out


@pytest.mark.parametrize('precision,Nv,pair', [
    ('double', 16, 0), ('single', 16, 0), ('single', 24, 1), ('single', 24, 0),
    ('double', 8, 0)])
def test_vss_bank_matches_oracle(precision, Nv, pair):
    """Q_p of both species on a bank of 6 points against the oracle; at
    FP32 N = 24 with the two-CTA kernel (the default there) and with the
    cluster exchange kernel."""
    cfg = mixture_config(precision, Nv=Nv, Nrho=6 if Nv > 8 else 4)
    be = B200Backend(cfg, device='cuda:0')
    vm = DGFSBiVelocityMesh(be, cfg)
    sm = DGFSBiVSSGLLScatteringModel(be, cfg, vm)
    sm.select(pair)
    mesh, params, pre = _oracle(vm, cfg)
    for pq in ('00', '01', '10', '11'):
        assert sm.prefactor(pq) == pytest.approx(params[pq]['prefac'],
                                                 rel=1e-14)
    nupts, neles = 2, 3
    st = _states(mesh, nupts*neles, seed=Nv)
    V = vm.vsize()
    banks = []
    for s in range(2):
        a = np.array([st[i][s] for i in range(nupts*neles)])
        a = a.reshape(nupts, neles, V).transpose(0, 2, 1).copy()
        banks.append(be.matrix((nupts, V, neles), a))
    outs = [be.matrix((nupts, V, neles)) for _ in range(2)]
    sm.fs_all(banks[0], banks[1], outs[0], outs[1])
    sm.status()
    got = [o.get() for o in outs]
    used = [b.get().astype(np.float64) for b in banks]
    worst = 0.0
    for u in range(nupts):
        for e in range(neles):
            fs = [used[0][u, :, e], used[1][u, :, e]]
            Qo = vss.vss_Q(fs, mesh, pre, params)
            for s in range(2):
                worst = max(worst, rel_err(got[s][u, :, e], Qo[s]))
    assert worst < TOL[precision], worst


def test_vss_single_point_leaves_the_rest():
    """fs(elem, upt, ...) writes only that point (scattering.py:317)."""
    cfg = mixture_config('double')
    be = B200Backend(cfg, device='cuda:0')
    vm = DGFSBiVelocityMesh(be, cfg)
    sm = DGFSBiVSSGLLScatteringModel(be, cfg, vm)
    mesh, params, pre = _oracle(vm, cfg)
    st = _states(mesh, 3, seed=2)
    V = vm.vsize()
    banks = [be.matrix((1, V, 3), np.array([x[s] for x in st]).T[None])
             for s in range(2)]
    outs = [be.matrix((1, V, 3)) for _ in range(2)]
    sm.fs(1, 0, banks[0], banks[1], outs[0], outs[1])
    sm.status()
    Qo = vss.vss_Q([st[1][0], st[1][1]], mesh, pre, params)
    for s in range(2):
        o = outs[s].get()
        assert rel_err(o[0, :, 1], Qo[s]) < TOL['double']
        assert not np.any(o[0, :, 0]) and not np.any(o[0, :, 2])
