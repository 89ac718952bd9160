# -*- coding: utf-8 -*-
"""Collision operators: the scattering-model interface of frfs.

``DGFSVHSGLLScatteringModel`` is registered under the same name as the
reference (``scattering_model = 'vhs-gll'``, frfs/solvers/dgfs/
scattering.py:44-45), is constructed the same way
(``(backend, cfg, velocitymesh)``, scattering.py:16-28) and keeps
``fs(d_arr_in, d_arr_out, elem, upt)`` (scattering.py:227).  All arithmetic
runs in libdgfs_b200.so: the fused cluster kernel evaluates Q(f) either at one
solution point (``fs``) or at every point of a bank in one persistent launch
(``fs_all``).
"""

import ctypes as ct
from abc import ABCMeta, abstractmethod
from math import gamma

import numpy as np

from frfs_b200 import _lib


def subclass_where(cls, **kwargs):
    """The subclass of ``cls`` whose attributes match ``kwargs``
    (frfs/util.py:subclass_where)."""
    for s in _subclasses(cls):
        if all(getattr(s, k, None) == v for k, v in kwargs.items()):
            return s
    raise KeyError(f'No subclass of {cls.__name__} with {kwargs}')


def _subclasses(cls):
    out = []
    for s in cls.__subclasses__():
        out.append(s)
        out.extend(_subclasses(s))
    return out


class DGFSScatteringModel(metaclass=ABCMeta):
    def __init__(self, backend, cfg, velocitymesh):
        self.backend = backend
        self.cfg = cfg
        self.vm = velocitymesh
        self.load_parameters()
        self.perform_precomputation()

    @abstractmethod
    def load_parameters(self):
        pass

    @abstractmethod
    def perform_precomputation(self):
        pass

    @abstractmethod
    def fs(self, d_arr_in, d_arr_out, elem, upt):
        pass


class DGFSVHSGLLScatteringModel(DGFSScatteringModel):
    """Fast-spectral VHS operator (frfs/solvers/dgfs/scattering.py:44-286)."""

    scattering_model = 'vhs-gll'

    def load_parameters(self):
        # scattering.py:50-65
        alpha = 1.0
        omega = self.cfg.getfloat('scattering-model', 'omega')
        self._gamma = 2.0*(1 - omega)
        dRef = self.cfg.getfloat('scattering-model', 'dRef')
        Tref = self.cfg.getfloat('scattering-model', 'Tref')
        invKn = (self.vm.H0()*np.sqrt(2.0)*np.pi*self.vm.n0()*dRef*dRef *
                 pow(Tref/self.vm.T0(), omega - 0.5))
        self._prefactor = invKn*alpha/(
            pow(2.0, 2 - omega + alpha)*gamma(2.5 - omega)*np.pi)
        self._invKn = invKn

    def perform_precomputation(self):
        vm = self.vm
        sect = 'backend-b200'
        self._project = self.cfg.getint(sect, 'vhs-project', 0)
        cluster = self.cfg.getint(sect, 'vhs-cluster', 0)
        self._qz = np.ascontiguousarray(vm.qz(), dtype=np.float64)
        self._qw = np.ascontiguousarray(vm.qw(), dtype=np.float64)
        self._sz = np.ascontiguousarray(vm.sz(), dtype=np.float64)
        self._lib = _lib.load()
        self._extra = []
        self._h = self._create_handle(cluster)

    def _create_handle(self, cluster=0):
        vm = self.vm
        p = _lib.VhsParams(
            Nv=vm.Nv(), Nrho=vm.Nrho(), M=vm.M(),
            precision=self.backend.precision, L=vm.L(),
            qz=_lib.as_dptr(self._qz), qw=_lib.as_dptr(self._qw),
            sz=_lib.as_dptr(self._sz), sw=vm.sw(),
            prefactor=self._prefactor, gamma=self._gamma,
            project=self._project, cluster=cluster)
        h = ct.c_void_p()
        _lib.check(self._lib.dgfs_vhs_create(ct.byref(p), ct.byref(h)),
                   'dgfs_vhs_create')
        return h

    def make_handle(self, exchange, largest_cluster=False):
        """A second operator handle on the same parameters with the first
        compiled launch shape of the given kind ('push', 'pull',
        'single-cta') selected -- or, with largest_cluster, the one of that
        kind with the most CTAs per point, for calls on a few points (it
        spreads each over the most SMs).  Owned and freed by this model;
        None when no shape of that kind is compiled."""
        vs = self.variants()
        idx = [i for i, v in enumerate(vs) if v['exchange'] == exchange]
        if not idx:
            return None
        pick = max(idx, key=lambda i: (vs[i]['cluster'], -i)) \
            if largest_cluster else idx[0]
        h = self._create_handle()
        _lib.check(self._lib.dgfs_vhs_select(h, pick), 'dgfs_vhs_select')
        self._extra.append(h)
        return h

    def __del__(self):
        for h in getattr(self, '_extra', []):
            self._lib.dgfs_vhs_destroy(h)
        self._extra = []
        h = getattr(self, '_h', None)
        if h:
            self._lib.dgfs_vhs_destroy(h)
            self._h = None

    @property
    def prefactor(self):
        return self._prefactor

    def _bank_args(self, d_arr_in, d_arr_out):
        nrow, ldim, dtype = d_arr_in.traits
        ncola, ncolb = d_arr_in.ioshape[1:]
        if d_arr_out.traits != d_arr_in.traits:
            raise ValueError('input and output banks differ in layout')
        if ncola != self.vm.vsize():
            raise ValueError(f'bank has {ncola} variables, expected '
                             f'{self.vm.vsize()}')
        if np.dtype(dtype).itemsize*8 != self.backend.precision:
            raise ValueError('bank precision differs from the backend')
        return nrow, ncolb, ldim

    def fs(self, d_arr_in, d_arr_out, elem, upt):
        """Q(f) at point (elem, upt) (scattering.py:227-286)."""
        nupts, neles, ldim = self._bank_args(d_arr_in, d_arr_out)
        _lib.check(self._lib.dgfs_vhs_apply(
            self._h, d_arr_in._as_parameter_, d_arr_out._as_parameter_,
            nupts, neles, ldim, self.backend.soasz, int(elem), int(upt),
            self.backend.stream), 'dgfs_vhs_apply')

    def fs_all(self, d_arr_in, d_arr_out):
        """Q(f) at every solution point of the bank in one launch."""
        nupts, neles, ldim = self._bank_args(d_arr_in, d_arr_out)
        _lib.check(self._lib.dgfs_vhs_apply(
            self._h, d_arr_in._as_parameter_, d_arr_out._as_parameter_,
            nupts, neles, ldim, self.backend.soasz, -1, 0,
            self.backend.stream), 'dgfs_vhs_apply')

    def fs_range(self, d_arr_in, d_arr_out, pt0, npts):
        """Q(f) at linear points [pt0, pt0+npts), pt = upt*neles + elem."""
        nupts, neles, ldim = self._bank_args(d_arr_in, d_arr_out)
        _lib.check(self._lib.dgfs_vhs_apply_range(
            self._h, d_arr_in._as_parameter_, d_arr_out._as_parameter_,
            nupts, neles, ldim, self.backend.soasz, int(pt0), int(npts),
            self.backend.stream), 'dgfs_vhs_apply_range')

    def launch_info(self):
        vals = [ct.c_int() for _ in range(4)]
        _lib.check(self._lib.dgfs_vhs_info(self._h, *[ct.byref(v)
                                                      for v in vals]),
                   'dgfs_vhs_info')
        return dict(zip(('cluster', 'threads', 'smem_bytes',
                         'max_clusters'), (v.value for v in vals)))

    def set_cluster(self, cluster):
        _lib.check(self._lib.dgfs_vhs_set_cluster(self._h, int(cluster)),
                   'dgfs_vhs_set_cluster')

    def variants(self):
        """Compiled launch shapes for this (Nv, precision)."""
        n = ct.c_int()
        _lib.check(self._lib.dgfs_vhs_num_variants(self._h, ct.byref(n)),
                   'dgfs_vhs_num_variants')
        out = []
        for i in range(n.value):
            vals = [ct.c_int() for _ in range(5)]
            _lib.check(self._lib.dgfs_vhs_variant_info(
                self._h, i, *[ct.byref(v) for v in vals]),
                'dgfs_vhs_variant_info')
            d = dict(zip(('cluster', 'double_buffered', 'min_ctas_per_sm',
                          'threads', 'smem_bytes'), (v.value for v in vals)))
            k = ct.c_int()
            _lib.check(self._lib.dgfs_vhs_variant_kind(self._h, i,
                                                       ct.byref(k)),
                       'dgfs_vhs_variant_kind')
            d['exchange'] = {0: 'pull', 1: 'push', 2: 'single-cta',
                             3: 'pair'}[k.value]
            out.append(d)
        return out

    def status(self):
        """Synchronise and raise if a launch gave up waiting for cluster
        data (the push kernels bound every wait)."""
        flag = ct.c_int()
        _lib.check(self._lib.dgfs_vhs_status(self._h, self.backend.stream,
                                             ct.byref(flag)),
                   'dgfs_vhs_status')

    def select(self, idx):
        _lib.check(self._lib.dgfs_vhs_select(self._h, int(idx)),
                   'dgfs_vhs_select')
        self._variant = int(idx)

    def autotune(self, d_arr_in, d_arr_out, npts=None, reps=2,
                 cache=True, verbose=False):
        """Time every compiled launch shape on this bank and keep the
        fastest.  Results are cached per (GPU, precision, Nv, Nrho, M,
        points) in $DGFS_B200_CACHE or ~/.cache/dgfs_b200/vhs_tune.json."""
        from frfs_b200 import autotune as at
        return at.tune_vhs(self, d_arr_in, d_arr_out, npts=npts, reps=reps,
                           cache=cache, verbose=verbose)

    def flops_per_point(self):
        """Algorithmic FLOPs of one Q(f) evaluation as implemented:
        5 V log2 V per complex 3D transform times (2 Nrho M + Nrho + 3)
        transforms, plus 12 Nrho M V for phase products and g*h sums."""
        V, P, M = self.vm.vsize(), self.vm.Nrho(), self.vm.M()
        return (5.0*V*np.log2(V)*(2*P*M + P + 3) + 12.0*P*M*V)
