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


def _setup(name, precision, project, nupts=2, neles=3, **kw):
    cfg = config(name, precision, **kw)
    cfg.set('backend-b200', 'vhs-project', project)
    be = B200Backend(cfg, device='cuda:0')
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    f = random_states(vm.cv(), nupts*neles, seed=21)
    arr = np.ascontiguousarray(f.reshape(nupts, neles, -1).transpose(0, 2, 1))
    fin = be.matrix(arr.shape, arr)
    qref = be.matrix(arr.shape)
    sm.fs_all(fin, qref)
    sm.status()
    return be, sm, fin, qref.get()


def _status(lib, be):
    flag = ct.c_int(-1)
    rc = lib.dgfs_vhs_noalloc_status(be.stream, ct.byref(flag))
    return rc, flag.value


@pytest.mark.parametrize('name,precision,project', [
    ('couette-n24', 'double', 0), ('couette-n24', 'single', 0),
    ('relax0d-n16', 'single', 1), ('relax0d-n16', 'double', 1),
    ('channel-n32', 'single', 0)])
def test_noalloc_matches_allocating_entry_point(name, precision, project):
    be, sm, fin, ref = _setup(name, precision, project)
    nupts, neles = 2, 3
    lib = _lib.load()
    p = _params(sm)
    nrow, ldim, _ = fin.traits
    for call in range(2):
        qout = be.matrix(fin.ioshape)
        rc = lib.dgfs_vhs_apply_noalloc(
            ct.byref(p), fin._as_parameter_, qout._as_parameter_, nupts,
            neles, ldim, be.soasz, -1, 0, be.stream)
        assert rc == 0, lib.dgfs_last_error().decode()
        assert _status(lib, be) == (0, 0)
        err = rel_err(qout.get(), ref)
        assert err < TOL[precision], f'call {call}: rel err {err:.3e}'


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_noalloc_single_point_matches_allocating_entry_point(precision):
    """elem >= 0: one point of the bank, as fs(..., elem, upt); every other
    entry of Q stays untouched."""
    be, sm, fin, ref = _setup('channel-n32', precision, 0, nupts=3, neles=5,
                              Nv=8, Nrho=4, M=6)
    lib = _lib.load()
    p = _params(sm)
    nrow, ldim, _ = fin.traits
    for call, (elem, upt) in enumerate([(3, 1), (4, 2)]):
        qout = be.matrix(fin.ioshape)
        rc = lib.dgfs_vhs_apply_noalloc(
            ct.byref(p), fin._as_parameter_, qout._as_parameter_, 3, 5, ldim,
            be.soasz, elem, upt, be.stream)
        assert rc == 0, lib.dgfs_last_error().decode()
        assert _status(lib, be) == (0, 0)
        got = qout.get()
        err = rel_err(got[upt, :, elem], ref[upt, :, elem])
        assert err < TOL[precision], f'call {call}: rel err {err:.3e}'
        mask = np.ones(got.shape, bool)
        mask[upt, :, elem] = False
        assert not np.any(got[mask])


def test_noalloc_status_reports_a_wait_that_ran_out():
    """A bounded wait that runs out (an exchange whose bytes never arrive,
    limit 1 ms) sets the allocation-free path's flag; a later call neither
    clears it nor computes differently, and dgfs_vhs_noalloc_status reports
    it once."""
    be, sm, fin, ref = _setup('relax0d-n16', 'single', 0)
    lib = _lib.load()
    p = _params(sm)
    nrow, ldim, _ = fin.traits
    qout = be.matrix(fin.ioshape)
    args = (ct.byref(p), fin._as_parameter_, qout._as_parameter_, 2, 3, ldim,
            be.soasz, -1, 0, be.stream)
    assert lib.dgfs_vhs_apply_noalloc(*args) == 0
    assert _status(lib, be) == (0, 0)
    assert lib.dgfs_vhs_check_wait(None, 1000000, be.stream) == 0
    assert lib.dgfs_vhs_apply_noalloc(*args) == 0
    rc, flag = _status(lib, be)
    assert (rc, flag) == (2, 1)
    assert b'gave up' in lib.dgfs_last_error()
    assert rel_err(qout.get(), ref) < TOL['single']
    assert _status(lib, be) == (0, 0)


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
