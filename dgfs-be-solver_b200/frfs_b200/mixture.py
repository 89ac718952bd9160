# -*- coding: utf-8 -*-
"""Binary-mixture VSS collision operator (frfs's dgfsbi solver) on the B200
library.

``DGFSBiVelocityMesh`` restates frfs/solvers/dgfsbi/velocitymesh.py:27-151:
the velocity box of half width L = cmax/u0 + dev sqrt(Tmax/T0), the radial
range R = 2S with S shrunk by the largest mass ratio, the Gauss-Jacobi
radial rule on [0, R] and the full-sphere design (sw = 4 pi / M).

``DGFSBiVSSGLLScatteringModel`` keeps the interface of
frfs/solvers/dgfsbi/scattering.py:44-330 (scattering_model 'vss-gll'):
per ordered species pair pq the parameters alpha_pq, omega_pq, dRef_pq,
Tref_pq of ``[scattering-model]`` give eta = alpha - 1, gamma =
2 (1 - omega) and the prefactor (scattering.py:64-87); one library handle
per pair holds the precomputation; ``fs(elem, upt, f_0, f_1, Q_0, Q_1)``
evaluates Q_p = sum_q Q(f_p, f_q) at one point (scattering.py:317-330) and
``fs_all`` at every point of the banks in one persistent launch per pair.
"""

import ctypes as ct
import itertools as it
from math import gamma as gammafn

import numpy as np

from frfs_b200 import _lib
from frfs_b200.quadratures import zwgj, zwglj
from frfs_b200.sphericaldesign import get_sphquadrule

NA = 6.0221409e+23
R0 = 8.3144598

c_int, c_double, c_dp = ct.c_int, ct.c_double, ct.POINTER(ct.c_double)


class VssParams(ct.Structure):
    """dgfs_vss_params (include/dgfs_b200.h)."""
    _fields_ = [('Nv', c_int), ('Nrho', c_int), ('M', c_int), ('Mpre', c_int),
                ('precision', c_int), ('L', c_double), ('qz', c_dp),
                ('qw', c_dp), ('sz', c_dp), ('szpre', c_dp),
                ('mp', c_double), ('mq', c_double), ('alpha', c_double),
                ('omega', c_double), ('prefactor', c_double)]


_lib.declare('dgfs_vss_create', c_int, [ct.POINTER(VssParams),
                                        ct.POINTER(ct.c_void_p)])
_lib.declare('dgfs_vss_destroy', c_int, [ct.c_void_p])
_lib.declare('dgfs_vss_apply', c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                       ct.c_void_p, c_int, c_int,
                                       ct.c_longlong, c_int, c_int, c_int,
                                       c_int, ct.c_void_p])
_lib.declare('dgfs_vss_status', c_int, [ct.c_void_p, ct.c_void_p,
                                        ct.POINTER(c_int)])
_lib.declare('dgfs_vss_select', c_int, [ct.c_void_p, c_int])


class DGFSBiVelocityMesh:
    def __init__(self, backend, cfg, nspcs=2, sphdesign_paths=None):
        self.backend, self.cfg, self._nspcs = backend, cfg, nspcs
        g = cfg.getfloat
        self._H0, self._T0 = g('non-dim', 'H0'), g('non-dim', 'T0')
        self._rho0 = g('non-dim', 'rho0')
        self._molarMass0 = g('non-dim', 'molarMass0')
        self._n0 = self._rho0/self._molarMass0*NA                  # :33
        self._u0 = np.sqrt(2*R0/self._molarMass0*self._T0)        # :35
        self._Nv = cfg.getint('constants', 'Nv')
        self._vsize = self._Nv**3
        self._Nrho = cfg.getint('constants', 'Nrho', self._Nv//2)
        cmax = g('velocity-mesh', 'cmax')/self._u0
        Tmax = g('velocity-mesh', 'Tmax')/self._T0
        dev = g('velocity-mesh', 'dev')
        self._masses = [g('velocity-mesh', f'molarMass{p + 1}') /
                        self._molarMass0 for p in range(nspcs)]  # :60-63
        mr = max(self._masses)
        self._L = cmax + dev*np.sqrt(Tmax)                        # :70
        self._S = min(                                            # :72-75
            self._L*2.0/(max(4.*mr/(1. + mr), 2.) + np.sqrt(1. + mr) + 1.),
            self._L*2.0/(max(4./(1. + mr), 2.) + np.sqrt(1. + 1./mr) + 1.))
        self._R = 2*self._S
        Nv = self._Nv
        self._cw = (2.0*self._L/Nv)**3
        self._c0 = np.linspace(-self._L + self._L/Nv, self._L - self._L/Nv,
                               Nv)
        idx = np.arange(self._vsize)
        self._cv = np.stack([self._c0[idx//(Nv*Nv)],
                             self._c0[(idx % (Nv*Nv))//Nv],
                             self._c0[idx % Nv]])
        rule = cfg.get('velocity-mesh', 'quad-rule', 'jacobi')
        rules = {'jacobi': zwgj, 'lobatto': zwglj}
        a = g('velocity-mesh', 'quad-rule-alpha', 0.0)
        b = g('velocity-mesh', 'quad-rule-beta', 0.0)
        qz, qw = rules[rule](self._Nrho, a, b)
        self._qz = (self._R/2.0)*(1.0 + qz)                       # :139
        self._qw = (self._R/2.0)*qw                               # :140
        self._M = cfg.getint('spherical-design-rule', 'M')
        paths = sphdesign_paths or [cfg.get('spherical-design-rule', 'path',
                                            None)]
        self._sz = get_sphquadrule(
            'symmetric', cfg.get('spherical-design-rule', 'ssrule'),
            self._M, paths=[p for p in paths if p]).pts
        self._sw = 4*np.pi/self._M

    def nspcs(self): return self._nspcs
    def masses(self): return list(self._masses)
    def Nv(self): return self._Nv
    def Nrho(self): return self._Nrho
    def M(self): return self._M
    def L(self): return self._L
    def R(self): return self._R
    def vsize(self): return self._vsize
    def qz(self): return self._qz
    def qw(self): return self._qw
    def sz(self): return self._sz
    def sw(self): return self._sw
    def cv(self): return self._cv
    def cw(self): return self._cw
    def n0(self): return self._n0
    def T0(self): return self._T0
    def H0(self): return self._H0


class DGFSBiVSSGLLScatteringModel:
    scattering_model = 'vss-gll'

    def __init__(self, backend, cfg, velocitymesh):
        self.backend, self.cfg, self.vm = backend, cfg, velocitymesh
        self._nspcs = velocitymesh.nspcs()
        self._lib = _lib.load()
        self._h = {}
        self.load_parameters()
        self.perform_precomputation()

    def load_parameters(self):
        cfg, vm = self.cfg, self.vm
        self._Mpre = cfg.getint('scattering-model', 'Mpre')
        paths = [cfg.get('spherical-design-rule', 'path', None)]
        self._szpre = get_sphquadrule(
            'symmetric', cfg.get('scattering-model', 'ssrulepre'),
            self._Mpre, paths=[p for p in paths if p]).pts
        self._cases = list(it.product(range(self._nspcs), repeat=2))
        m = vm.masses()
        self._alpha, self._omega, self._prefactor = {}, {}, {}
        for p, q in self._cases:
            pq = f'{p}{q}'
            alpha = cfg.getfloat('scattering-model', 'alpha' + pq)
            omega = cfg.getfloat('scattering-model', 'omega' + pq)
            dRef = cfg.getfloat('scattering-model', 'dRef' + pq)
            Tref = cfg.getfloat('scattering-model', 'Tref' + pq)
            invKn = (np.sqrt(1. + m[p]/m[q])*np.pi*vm.n0()*dRef*dRef *
                     pow(Tref/vm.T0(), omega - 0.5)*vm.H0())   # :80-81
            mu = m[p]*m[q]/(m[p] + m[q])
            self._alpha[pq], self._omega[pq] = alpha, omega
            self._prefactor[pq] = invKn*alpha/(                  # :85-87
                np.sqrt(1. + m[p]/m[q])*pow(mu, omega - 0.5) *
                pow(2., 1 + alpha)*gammafn(2.5 - omega)*np.pi)

    def perform_precomputation(self):
        vm, m = self.vm, self.vm.masses()
        keep = dict(qz=np.ascontiguousarray(vm.qz(), dtype=np.float64),
                    qw=np.ascontiguousarray(vm.qw(), dtype=np.float64),
                    sz=np.ascontiguousarray(vm.sz(), dtype=np.float64),
                    szpre=np.ascontiguousarray(self._szpre,
                                               dtype=np.float64))
        self._keep = keep
        for p, q in self._cases:
            pq = f'{p}{q}'
            prm = VssParams(
                Nv=vm.Nv(), Nrho=vm.Nrho(), M=vm.M(), Mpre=self._Mpre,
                precision=self.backend.precision, L=vm.L(),
                qz=_lib.as_dptr(keep['qz']), qw=_lib.as_dptr(keep['qw']),
                sz=_lib.as_dptr(keep['sz']),
                szpre=_lib.as_dptr(keep['szpre']), mp=m[p], mq=m[q],
                alpha=self._alpha[pq], omega=self._omega[pq],
                prefactor=self._prefactor[pq])
            h = ct.c_void_p()
            _lib.check(self._lib.dgfs_vss_create(ct.byref(prm), ct.byref(h)),
                       'dgfs_vss_create')
            self._h[pq] = h

    def __del__(self):
        for h in getattr(self, '_h', {}).values():
            if h:
                self._lib.dgfs_vss_destroy(h)
        self._h = {}

    def select(self, pair):
        """Launch shape of every pair: 1 the two-CTA kernel (FP32, N = 24,
        the default there), 0 the cluster exchange kernel."""
        for pq, h in self._h.items():
            _lib.check(self._lib.dgfs_vss_select(h, int(pair)),
                       'dgfs_vss_select')

    def prefactor(self, pq):
        return self._prefactor[pq]

    def _apply(self, pq, fp, fq, Q, elem, upt, accumulate):
        nupts, _, neles = fp.ioshape
        _, ldim, _ = fp.traits
        _lib.check(self._lib.dgfs_vss_apply(
            self._h[pq], fp._as_parameter_, fq._as_parameter_,
            Q._as_parameter_, nupts, neles, ldim, self.backend.soasz, elem,
            upt, accumulate, self.backend.stream), 'dgfs_vss_apply')

    def fs(self, elem, upt, *args):
        """Q_p(elem, upt) = sum_q Q(f_p, f_q): args = (f_0 .. f_{n-1},
        Q_0 .. Q_{n-1}) banks (scattering.py:317-330)."""
        n = self._nspcs
        assert len(args) == 2*n, 'need n distributions and n outputs'
        for p, q in self._cases:
            self._apply(f'{p}{q}', args[p], args[q], args[p + n], elem, upt,
                        1 if q > 0 else 0)

    def fs_all(self, *args):
        """Q_p = sum_q Q(f_p, f_q) at every point of the banks."""
        self.fs(-1, 0, *args)

    def flops_per_point(self):
        """Algorithmic FLOPs of all ordered pairs' Q(f_p, f_q) at one
        point: per pair 3 Nrho M + 4 complex 3D transforms (the reference's
        count, scattering.py:227-315: F, G, two inverse and one forward
        transform per radial node and direction, the gain and loss inverse
        transforms) at 5 V log2 V each, plus 20 Nrho M V for the phase
        products, g h and the weighted gain sum."""
        V, P, M = self.vm.vsize(), self.vm.Nrho(), self.vm.M()
        per_pair = 5.0*V*np.log2(V)*(3*P*M + 4) + 20.0*P*M*V
        return len(self._cases)*per_pair

    def status(self):
        flag = c_int()
        for pq, h in self._h.items():
            _lib.check(self._lib.dgfs_vss_status(h, self.backend.stream,
                                                 ct.byref(flag)),
                       'dgfs_vss_status')
