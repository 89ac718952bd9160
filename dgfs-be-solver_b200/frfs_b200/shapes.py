# -*- coding: utf-8 -*-
"""Flux-reconstruction operators for line and quadrilateral elements.

Restates the operator construction of frfs/shapes.py:83-289 and
frfs/polys.py:9-200 for the element types the DGFS hot path runs on:

* orthonormal Legendre bases (frfs/polys.py:LinePolyBasis, QuadPolyBasis),
  nodal bases by a Vandermonde solve (polys.py:nodal_basis_at);
* M0: nodal basis at the flux points; M1: basis gradients at the solution
  points laid out (nupts, ndims*nupts); M2 = n_ref (x) M0; M3: the lifting
  operator g_k(x) = sum_j (int_face l_k phi_j) phi_j(x), with the face
  integral by the (order+1)-point Gauss-Lobatto rule (shapes.py:243-289);
* every operator passes through the same post-processing as frfs's
  ``clean`` decorator (frfs/nputil.py:22-55): entries below 1e-10 become zero
  and magnitudes within 1e-10 of each other are replaced by their median.

Point sets are computed (Gauss-Legendre by Golub-Welsch) instead of read from
frfs's tables; they agree with the tables to ~1e-16.

The line element uses a point face at xi = -1 and xi = +1 with unit weight:
frfs's LineShape has no 'point' rule for its lifting operator
(shapes.py:262-268) and maps both faces to xi = 0, so 1D elements are a
documented extension here rather than a restatement.
"""

import itertools as it
from math import sqrt

import numpy as np

from frfs_b200.quadratures import gauss_legendre, gauss_legendre_lobatto


def tol_runs(vals, tol):
    """Split an ascending sequence into runs: a run starts at the first
    value not yet taken and holds every later value that exceeds it by less
    than ``tol``.  Yields (start, stop) index pairs."""
    vals = np.asarray(vals, dtype=float)
    n, i = len(vals), 0
    while i < n:
        far = np.nonzero(vals[i + 1:] - vals[i] >= tol)[0]
        j = i + 1 + int(far[0]) if far.size else n
        yield i, j
        i = j


def clean(arr, tol=1e-10):
    """Post-processing frfs applies to every operator matrix
    (frfs/nputil.py:24-52): entries of magnitude below ``tol`` become zero;
    then the magnitudes, taken in ascending order, are grouped into runs
    that stay within ``tol`` of their first member, every run of two or more
    is replaced by its median, and the signs are restored."""
    out = np.array(arr, dtype=np.float64, copy=True)
    out[np.abs(out) < tol] = 0
    mag = np.abs(out).ravel()
    order = np.argsort(mag)
    srt = mag[order]
    for i, j in tol_runs(srt, tol):
        if j - i > 1:
            mag[order[i:j]] = np.median(srt[i:j])
    return np.copysign(mag, out.ravel()).reshape(out.shape)


def legendre(nmax, x):
    """Legendre polynomials P_0..P_nmax and their derivatives at x, from
    Bonnet's recurrence (n + 1) P_{n+1} = (2n + 1) x P_n - n P_{n-1} and
    P'_{n+1} = P'_{n-1} + (2n + 1) P_n (Abramowitz & Stegun 22.7.10 and
    22.8.5 in differentiated form)."""
    p = [1.0, x]
    dp = [0.0, 1.0]
    for n in range(1, nmax):
        p.append(((2*n + 1)*x*p[n] - n*p[n - 1])/(n + 1))
        dp.append(dp[n - 1] + (2*n + 1)*p[n])
    return p[:nmax + 1], dp[:nmax + 1]


class _Basis:
    """Orthonormal tensor-product Legendre basis of given order (number of
    modes per direction) on [-1, 1]^ndims, with nodal variants."""

    def __init__(self, ndims, order, pts):
        self.ndims, self.order = ndims, order
        self.pts = np.atleast_2d(np.asarray(pts, dtype=float))
        if self.ndims == 1 and self.pts.shape[0] == 1:
            self.pts = self.pts.T

    def _leg(self, x):
        """sqrt(k + 1/2) P_k(x), k < order: orthonormal on [-1, 1]."""
        p, _ = legendre(self.order - 1, x)
        return [sqrt(k + 0.5)*v for k, v in enumerate(p)]

    def _dleg(self, x):
        _, dp = legendre(self.order - 1, x)
        return [sqrt(k + 0.5)*v for k, v in enumerate(dp)]

    def ortho_basis_at(self, pts):
        pts = np.atleast_2d(np.asarray(pts, dtype=float))
        out = []
        for p in pts:
            if self.ndims == 1:
                out.append(self._leg(p[0]))
            else:
                pa, pb = self._leg(p[0]), self._leg(p[1])
                out.append([pi*pj for pi in pa for pj in pb])
        return clean(np.array(out, dtype=float).T)

    def jac_ortho_basis_at(self, pts):
        pts = np.atleast_2d(np.asarray(pts, dtype=float))
        J = []
        for p in pts:
            if self.ndims == 1:
                J.append([[d] for d in self._dleg(p[0])])
            else:
                pa, pb = self._leg(p[0]), self._leg(p[1])
                dpa, dpb = self._dleg(p[0]), self._dleg(p[1])
                J.append([[dpi*pj, pi*dpj] for pi, dpi in zip(pa, dpa)
                          for pj, dpj in zip(pb, dpb)])
        return clean(np.array(J, dtype=float).swapaxes(0, 2))

    @property
    def vdm(self):
        return self.ortho_basis_at(self.pts)

    def nodal_basis_at(self, epts):
        return clean(np.linalg.solve(self.vdm, self.ortho_basis_at(epts)).T)

    def jac_nodal_basis_at(self, epts):
        return clean(np.linalg.solve(self.vdm, self.jac_ortho_basis_at(epts)))


def _std_ele(ndims, sptord):
    pts1d = np.linspace(-1, 1, sptord + 1)
    return np.array([p[::-1] for p in it.product(pts1d, repeat=ndims)])


class QuadShape:
    """Quadrilateral FR element of a given order with Gauss-Legendre
    solution and flux points (the configuration the workloads use)."""

    name = 'quad'
    ndims = 2
    # (reference-to-face projection, reference normal): shapes.py QuadShape
    faces = [(lambda s: (s, -1.0), (0, -1)), (lambda s: (1.0, s), (1, 0)),
             (lambda s: (s, 1.0), (0, 1)), (lambda s: (-1.0, s), (-1, 0))]

    def __init__(self, order, nspts=4):
        self.order = order
        n = order + 1
        z, _ = gauss_legendre(n)
        self.pts1d = z
        self.upts = np.array([(z[i], z[j]) for j in range(n)
                              for i in range(n)])
        self.nupts = n*n
        self.nfacefpts = [n]*4
        self.nfpts = 4*n
        self.fpts = np.vstack([[proj(s) for s in z] for proj, _ in self.faces])
        self.norm_fpts = np.vstack([[nrm]*n for _, nrm in self.faces]).astype(
            float)
        self.facefpts = [list(range(k*n, (k + 1)*n)) for k in range(4)]
        self.ubasis = _Basis(2, n, self.upts)
        self.nspts = nspts
        self.nsptsord = int(round(sqrt(nspts)))
        self.spts = _std_ele(2, self.nsptsord - 1)
        self.sbasis = _Basis(2, self.nsptsord, self.spts)
        self.mpts = _std_ele(2, max(order, 1))
        self.nmpts = len(self.mpts)
        self.mbasis = _Basis(2, max(order + 1, 2), self.mpts)
        self._face_basis = _Basis(1, n, z[:, None])

    # -- operators -----------------------------------------------------
    @property
    def m0(self):
        return self.ubasis.nodal_basis_at(self.fpts)

    @property
    def m1(self):
        m = np.rollaxis(self.ubasis.jac_nodal_basis_at(self.upts), 2)
        return m.reshape(self.nupts, -1)

    @property
    def m2(self):
        m = self.norm_fpts[..., None]*self.m0[:, None, :]
        return m.reshape(self.nfpts, -1)

    @property
    def m3(self):
        zq, wq = gauss_legendre_lobatto(self.order + 1)
        coeffs = []
        for proj, _ in self.faces:
            L = self._face_basis.nodal_basis_at(zq[:, None])
            M = self.ubasis.ortho_basis_at(np.array([proj(s) for s in zq]))
            coeffs.append(np.einsum('i,ik,ji->kj', wq, L, M))
        coeffs = np.vstack(coeffs)
        return clean(np.dot(coeffs, self.ubasis.ortho_basis_at(self.upts)).T)

    @property
    def m12(self):
        """V^T V, V the orthonormal basis at the solution points: the
        operator of DGFSElements' 'invmass' kernel (frfs/shapes.py:164-166,
        frfs/solvers/dgfs/elements.py:161-164)."""
        vdm = self.ubasis.vdm
        return (vdm.T @ vdm).reshape(self.nupts, -1)

    def opmat(self, expr):
        if expr == 'M12':
            return self.m12
        m0, m1, m2, m3 = self.m0, self.m1, self.m2, self.m3
        if expr == 'M0':
            return clean(m0)
        if expr == 'M1':
            return clean(m1)
        if expr == 'M2':
            return clean(m2)
        if expr == 'M3':
            return clean(m3)
        if expr == 'M1 - M3*M2':
            return clean(m1 - m3 @ m2)
        if expr == 'M12':
            return self.m12
        raise ValueError(f'unsupported operator expression {expr!r}')
