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
