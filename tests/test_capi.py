# -*- coding: utf-8 -*-
"""The C-ABI library loads and exports every entry point include/*.h
declares (no compute calls; runs without a GPU)."""

import ctypes as ct
import glob
import os
import re

from conftest import ROOT
from frfs_b200 import _lib


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, 'include', '*.h')):
        src = open(h).read()
        names |= set(re.findall(r'^DGFS_API\s+[\w\s\*]+?\b(dgfs_\w+)\s*\(',
                                src, flags=re.M))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert 'dgfs_vhs_create' in names and 'dgfs_vhs_apply' in names
    assert len(names) >= 8


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in sorted(declared_symbols())
               if not hasattr(lib, n)]
    assert not missing, f'not exported: {missing}'


def test_error_path_without_gpu_work():
    lib = _lib.load()
    assert lib.dgfs_version().startswith(b'dgfs_b200')
    # null arguments are rejected before any CUDA call
    assert lib.dgfs_vhs_create(None, None) == 1
    assert b'null' in lib.dgfs_last_error()
    assert lib.dgfs_vhs_apply(None, None, None, 1, 1, 1, 32, -1, 0,
                              None) == 1


def test_surrogate_entry_points_validate_arguments_before_any_cuda_call():
    """Host-side argument checks of the surrogate's entry points (no GPU
    needed): each bad call returns an error code and a message."""
    import frfs_b200.surrogate  # noqa: F401  (declares the signatures)
    lib = _lib.load()
    p = ct.c_void_p(8)
    # reconstruct: null coefficient / moment / output arrays
    assert lib.dgfs_hermite_reconstruct(32, None, p, None, 1, 1, 32*4096, 16,
                                        5.0, 1.0, 1.0, 1.0, p, None, None,
                                        None, p, None, None, None, None) != 0
    # gate: a network list without its counter
    assert lib.dgfs_surrogate_gate(4, p, 0.05, 1e-3, None, 5.0, 3.5, p, p,
                                   p, p, None, None) != 0
    assert b'bad arguments' in lib.dgfs_last_error()
    # row-list affine without a count
    assert lib.dgfs_mlp_affine_rows(4, 8, p, None, p, p, p, p, 0, None) != 0
    # GEMM with an unknown activation
    assert lib.dgfs_mlp_gemm(4, 4, 4, p, 4, 1, p, 0, 4, 1, None, None, p, 4,
                             2, 0, None, None) != 0
    assert b'act' in lib.dgfs_last_error()
    # scale with the log column inside the scaled range
    assert lib.dgfs_surrogate_scale(4, 256, p, 1e-3, 4, 220, 100, 0, p,
                                    None) != 0


def test_tensor_core_and_graph_entry_points_validate_arguments():
    """Host-side checks of the tensor-core products and the stage-graph
    entry points (no GPU needed: each bad call is rejected before any CUDA
    call)."""
    import frfs_b200.surrogate  # noqa: F401  (declares the signatures)
    lib = _lib.load()
    p16, p8 = ct.c_void_p(16), ct.c_void_p(8)
    # TMA-fed product: leading dimensions must be multiples of 8 ...
    assert lib.dgfs_mlp_gemm_bf16(64, 64, 64, p16, 0, 12, p16, 0, 64, None,
                                  None, p16, None, 64, 0, 0, p16, None) == 1
    assert b'multiples of 8' in lib.dgfs_last_error()
    # ... operands 16-byte aligned for the tensor maps ...
    assert lib.dgfs_mlp_gemm_bf16(64, 64, 64, p8, 0, 64, p16, 0, 64, None,
                                  None, p16, None, 64, 0, 0, p16, None) == 1
    assert b'aligned' in lib.dgfs_last_error()
    # ... and an error flag is required
    assert lib.dgfs_mlp_gemm_bf16(64, 64, 64, p16, 0, 64, p16, 0, 64, None,
                                  None, p16, None, 64, 0, 0, None, None) == 1
    # staged product: unknown activation
    assert lib.dgfs_mlp_gemm_tc(4, 4, 4, p16, 4, 1, p16, 0, 4, 1, None, None,
                                p16, 4, 2, 0, p16, None) == 1
    # stage graphs: the legacy default stream cannot be captured
    lib.dgfs_graph_begin.argtypes = [ct.c_void_p]
    lib.dgfs_graph_end.argtypes = [ct.c_void_p, ct.c_void_p]
    lib.dgfs_graph_launch.argtypes = [ct.c_void_p, ct.c_void_p]
    lib.dgfs_graph_destroy.argtypes = [ct.c_void_p]
    assert lib.dgfs_graph_begin(None) == 1
    assert b'legacy default stream' in lib.dgfs_last_error()
    assert lib.dgfs_graph_end(None, None) == 1
    assert lib.dgfs_graph_launch(None, None) == 1
    assert lib.dgfs_graph_destroy(None) == 0
