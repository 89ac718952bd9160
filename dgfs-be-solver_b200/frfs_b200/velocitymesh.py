# -*- coding: utf-8 -*-
"""Velocity mesh of the DGFS solver.

Same construction and accessors as DGFSVelocityMesh
(frfs/solvers/dgfs/velocitymesh.py:11-162): nondimensionalisation
(n0 = rho0/m N_A, u0 = sqrt(2 R T0 / m)), the cell-centred N^3 grid on
[-L, L]^3 with index I (x) slowest, the Gauss-Jacobi radial rule on [0, R]
and the first M points of a 2M-point symmetric spherical design with weight
2 pi / M.
"""

import numpy as np

from frfs_b200.quadratures import zwgj, zwglj
from frfs_b200.sphericaldesign import get_sphquadrule


class DGFSVelocityMesh:
    R0 = 8.3144598
    NA = 6.0221409e+23

    def __init__(self, backend, cfg, sphdesign_paths=None):
        self.backend = backend
        self.cfg = cfg
        self._sphpaths = sphdesign_paths
        self._construct_velocity_mesh()
        self._load_quadrature()
        self._construct_spherical_mesh()
        self._dev = {}

    def _construct_velocity_mesh(self):
        cfg = self.cfg
        self._H0 = cfg.getfloat('non-dim', 'H0')
        self._T0 = cfg.getfloat('non-dim', 'T0')
        self._rho0 = cfg.getfloat('non-dim', 'rho0')
        self._molarMass0 = cfg.getfloat('non-dim', 'molarMass0')
        self._n0 = self._rho0/self._molarMass0*self.NA
        self._u0 = np.sqrt(2*self.R0/self._molarMass0*self._T0)

        self._Nv = cfg.getint('constants', 'Nv')
        self._vsize = self._Nv**3
        self._NvBatchSize = cfg.getint('constants', 'NvBatchSize',
                                       self._vsize)
        if self._vsize < self._NvBatchSize:
            raise ValueError('NvBatchSize larger than Nv^3')
        if self._vsize % self._NvBatchSize:
            raise ValueError('NvBatchSize must divide Nv^3')
        self._NvBatches = self._vsize // self._NvBatchSize
        self._Nrho = cfg.getint('constants', 'Nrho', int(self._Nv/2))

        cmax = cfg.getfloat('velocity-mesh', 'cmax')/self._u0
        Tmax = cfg.getfloat('velocity-mesh', 'Tmax')/self._T0
        dev = cfg.getfloat('velocity-mesh', 'dev')
        self._L = cmax + dev*np.sqrt(Tmax)
        self._S = self._L*2.0/(3.0 + np.sqrt(2.0))
        self._R = 2*self._S

        N = self._Nv
        self._cw = (2.0*self._L/N)**3
        c0 = np.linspace(-self._L + self._L/N, self._L - self._L/N, N)
        idx = np.arange(self._vsize)
        self._c0 = c0
        self._cv = np.stack([c0[idx // (N*N)], c0[(idx % (N*N)) // N],
                             c0[idx % N]])

    def _load_quadrature(self):
        rule = self.cfg.get('velocity-mesh', 'quad-rule', 'jacobi')
        rules = {'jacobi': zwgj, 'lobatto': zwglj}
        if rule not in rules:
            raise ValueError(f'Valid quads: {list(rules)}')
        a = self.cfg.getfloat('velocity-mesh', 'quad-rule-alpha', 0.0)
        b = self.cfg.getfloat('velocity-mesh', 'quad-rule-beta', 0.0)
        qz, qw = rules[rule](self._Nrho, a, b)
        self._qz = (self._R/2.0)*(1.0 + qz)
        self._qw = ((self._R - 0.0)/2.0)*qw

    def _construct_spherical_mesh(self):
        self._ssrule = self.cfg.get('spherical-design-rule', 'ssrule')
        self._M = self.cfg.getint('spherical-design-rule', 'M')
        paths = list(self._sphpaths or [])
        if self.cfg.hasopt('spherical-design-rule', 'path'):
            paths.insert(0, self.cfg.getpath('spherical-design-rule', 'path'))
        srule = get_sphquadrule('symmetric', rule=self._ssrule,
                                npts=2*self._M, paths=paths)
        self._sz = np.ascontiguousarray(srule.pts[0:self._M, :])
        self._sw = 2*np.pi/self._M

    def Nv(self): return self._Nv
    def Nrho(self): return self._Nrho
    def NvBatches(self): return self._NvBatches
    def NvBatchSize(self): return self._NvBatchSize
    def M(self): return self._M
    def L(self): return self._L
    def vsize(self): return self._vsize
    def qz(self): return self._qz
    def qw(self): return self._qw
    def cv(self): return self._cv
    def c0(self): return self._c0
    def cw(self): return self._cw
    def sz(self): return self._sz
    def sw(self): return self._sw
    def H0(self): return self._H0
    def T0(self): return self._T0
    def rho0(self): return self._rho0
    def n0(self): return self._n0
    def u0(self): return self._u0
    def molarMass0(self): return self._molarMass0
