# -*- coding: utf-8 -*-
"""The allocation-free collision entry point against the allocating one.

dgfs_vhs_apply_noalloc serves callers that cannot allocate device memory
while they run (a host whose allocator owns the device heap, a plugin that may
only use the buffers it is given, loops that cannot afford cudaMalloc's
synchronisation).  It keeps its tables and scratch in a fixed static device
array instead of cudaMalloc'd buffers.  This test calls it through the C ABI
twice in a row on the same banks and checks both results against
dgfs_vhs_apply within the tolerances of the other collision tests.  It lives
in its own file, collected last, and passes both alone in a fresh process and
after the rest of the suite.
"""

import ctypes as ct

import numpy as np
import pytest
import torch

from helpers import config, random_states, rel_err
from frfs_b200 import _lib
from frfs_b200.backend import B200Backend
from frfs_b200.scattering import DGFSVHSGLLScatteringModel
from frfs_b200.velocitymesh import DGFSVelocityMesh

pytestmark = pytest.mark.gpu

TOL = {'double': 1e-10, 'single': 2e-4}


def _params(sm):
    vm = sm.vm
    return _lib.VhsParams(
        Nv=vm.Nv(), Nrho=vm.Nrho(), M=vm.M(),
        precision=sm.backend.precision, L=vm.L(),
        qz=_lib.as_dptr(sm._qz), qw=_lib.as_dptr(sm._qw),
        sz=_lib.as_dptr(sm._sz), sw=vm.sw(), prefactor=sm.prefactor,
        gamma=sm._gamma, project=sm._project, cluster=0)


@pytest.mark.parametrize('name,precision,project', [
    ('couette-n24', 'double', 0), ('couette-n24', 'single', 0),
    ('relax0d-n16', 'single', 1), ('channel-n32', 'single', 0)])
def test_noalloc_matches_allocating_entry_point(name, precision, project):
    cfg = config(name, precision)
    cfg.set('backend-b200', 'vhs-project', project)
    be = B200Backend(cfg, device='cuda:0')
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    nupts, neles = 2, 3
    f = random_states(vm.cv(), nupts*neles, seed=21)
    arr = np.ascontiguousarray(f.reshape(nupts, neles, -1).transpose(0, 2, 1))
    fin = be.matrix(arr.shape, arr)
    qref = be.matrix(arr.shape)
    sm.fs_all(fin, qref)
    sm.status()
    ref = qref.get()

    lib = _lib.load()
    p = _params(sm)
    nrow, ldim, _ = fin.traits
    for call in range(2):
        qout = be.matrix(arr.shape)
        rc = lib.dgfs_vhs_apply_noalloc(
            ct.byref(p), fin._as_parameter_, qout._as_parameter_, nupts,
            neles, ldim, be.soasz, -1, 0, be.stream)
        assert rc == 0, lib.dgfs_last_error().decode()
        torch.cuda.synchronize()
        err = rel_err(qout.get(), ref)
        assert err < TOL[precision], f'call {call}: rel err {err:.3e}'


def test_noalloc_rejects_sizes_beyond_the_static_array():
    cfg = config('couette-n24', 'single')
    be = B200Backend(cfg, device='cuda:0')
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    p = _params(sm)
    p.Nrho = 33                                    # above the static limit
    lib = _lib.load()
    fin = be.matrix((1, vm.vsize(), 1))
    fout = be.matrix((1, vm.vsize(), 1))
    nrow, ldim, _ = fin.traits
    rc = lib.dgfs_vhs_apply_noalloc(ct.byref(p), fin._as_parameter_,
                                    fout._as_parameter_, 1, 1, ldim,
                                    be.soasz, -1, 0, be.stream)
    assert rc == 1
    assert b'static limits' in lib.dgfs_last_error()
