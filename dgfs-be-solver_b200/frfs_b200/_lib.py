# -*- coding: utf-8 -*-
"""ctypes binding of libdgfs_b200.so (the C ABI in include/dgfs_b200.h).

The library is required: there is no CPU or PyTorch fallback.  Loading
fails with a RuntimeError naming the missing file when the shared library has
not been built (``python -m frfs_b200.build`` or ``__graft_entry__.build()``).
"""

import ctypes as ct
import os

from frfs_b200.build import LIBPATH

c_int, c_ll, c_double, c_void_p = ct.c_int, ct.c_longlong, ct.c_double, ct.c_void_p
c_dp = ct.POINTER(ct.c_double)


class DgfsError(RuntimeError):
    """An error status returned by libdgfs_b200."""

    def __init__(self, code, fn, msg):
        super().__init__(f'{fn} failed (code {code}): {msg}')
        self.code = code


class VhsParams(ct.Structure):
    """dgfs_vhs_params (include/dgfs_b200.h)."""
    _fields_ = [('Nv', c_int), ('Nrho', c_int), ('M', c_int),
                ('precision', c_int), ('L', c_double), ('qz', c_dp),
                ('qw', c_dp), ('sz', c_dp), ('sw', c_double),
                ('prefactor', c_double), ('gamma', c_double),
                ('project', c_int), ('cluster', c_int)]


_SIGS = {
    'dgfs_last_error': (ct.c_char_p, []),
    'dgfs_version': (ct.c_char_p, []),
    'dgfs_vhs_create': (c_int, [ct.POINTER(VhsParams), ct.POINTER(c_void_p)]),
    'dgfs_vhs_destroy': (c_int, [c_void_p]),
    'dgfs_vhs_apply': (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int,
                               c_ll, c_int, c_int, c_int, c_void_p]),
    'dgfs_vhs_apply_range': (c_int, [c_void_p, c_void_p, c_void_p, c_int,
                                     c_int, c_ll, c_int, c_int, c_int,
                                     c_void_p]),
    'dgfs_vhs_apply_list': (c_int, [c_void_p, c_void_p, c_void_p, c_int,
                                    c_int, c_ll, c_int, c_void_p, c_void_p,
                                    c_int, c_void_p]),
    'dgfs_vhs_loss_rate': (c_int, [c_void_p, c_void_p, c_void_p, c_int,
                                   c_int, c_ll, c_int, c_void_p, c_void_p]),
    'dgfs_vhs_info': (c_int, [c_void_p, ct.POINTER(c_int),
                              ct.POINTER(c_int), ct.POINTER(c_int),
                              ct.POINTER(c_int)]),
    'dgfs_vhs_set_cluster': (c_int, [c_void_p, c_int]),
    'dgfs_vhs_num_variants': (c_int, [c_void_p, ct.POINTER(c_int)]),
    'dgfs_vhs_variant_info': (c_int, [c_void_p, c_int] +
                              [ct.POINTER(c_int)]*5),
    'dgfs_vhs_select': (c_int, [c_void_p, c_int]),
    'dgfs_vhs_variant_kind': (c_int, [c_void_p, c_int, ct.POINTER(c_int)]),
    'dgfs_vhs_status': (c_int, [c_void_p, c_void_p, ct.POINTER(c_int)]),
    'dgfs_vhs_apply_noalloc': (c_int, [ct.POINTER(VhsParams), c_void_p,
                                       c_void_p, c_int, c_int, c_ll, c_int,
                                       c_int, c_int, c_void_p]),
    'dgfs_vhs_noalloc_status': (c_int, [c_void_p, ct.POINTER(c_int)]),
    'dgfs_vhs_check_wait': (c_int, [c_void_p, c_ll, c_void_p]),
    'dgfs_moments': (c_int, [c_int, c_void_p, c_int, c_int, c_ll, c_int,
                             c_double, c_double, c_void_p, c_void_p]),
    'dgfs_probe_fma_peak': (c_int, [c_int, c_int, ct.POINTER(c_double),
                                    ct.POINTER(ct.c_float), c_void_p]),
}

_lib = None


def load(path=None):
    """Load libdgfs_b200.so and declare its signatures (cached)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    path = path or LIBPATH
    if not os.path.exists(path):
        raise RuntimeError(f'{path} not found: build the CUDA library first '
                           '(python -m frfs_b200.build); there is no '
                           'fallback implementation')
    lib = ct.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype, fn.argtypes = res, args
    _lib = lib
    return lib


def declare(name, restype, argtypes):
    """Declare an additional entry point (used by the DG module)."""
    _SIGS[name] = (restype, argtypes)
    if _lib is not None:
        fn = getattr(_lib, name)
        fn.restype, fn.argtypes = restype, argtypes


def check(code, fn):
    if code != 0:
        msg = load().dgfs_last_error().decode(errors='replace')
        raise DgfsError(code, fn, msg)


def call(name, *args):
    """Call an entry point and raise DgfsError on a non-zero status."""
    fn = getattr(load(), name)
    check(fn(*args), name)


def as_dptr(arr):
    """ctypes double* to a contiguous float64 numpy array (kept alive by the
    caller)."""
    return arr.ctypes.data_as(c_dp)
