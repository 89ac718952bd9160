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


def clean(arr, tol=1e-10):
    """frfs/nputil.py:clean: flush tiny entries, coalesce equal magnitudes."""
    arr = np.array(arr, dtype=np.float64, copy=True)
    arr[np.abs(arr) < tol] = 0
    if arr.size > 1:
        amfl = np.abs(arr.ravel())
        amix = np.argsort(amfl, kind='quicksort')
        i, ix = 0, amix[0]
        for j, jx in enumerate(amix[1:], start=1):
            if amfl[jx] - amfl[ix] >= tol:
                if j - i > 1:
                    amfl[amix[i:j]] = np.median(amfl[amix[i:j]])
                i, ix = j, jx
        if i != j:
            amfl[amix[i:]] = np.median(amfl[amix[i:]])
        arr = np.copysign(amfl, arr.ravel()).reshape(arr.shape)
    return arr


def jacobi(n, a, b, z):
    """P_0..P_n of the Jacobi family at z (frfs/polys.py:12-33)."""
    j = [np.ones_like(z, dtype=float) if hasattr(z, '__len__') else 1.0]
    if n >= 1:
        j.append(((a + b + 2)*z + a - b)/2)
    if n >= 2:
        apb, bbmaa = a + b, b*b - a*a
        for q in range(2, n + 1):
            qapbpq, apbp2q = q*(apb + q), apb + 2*q
            apbp2qm1, apbp2qm2 = apbp2q - 1, apbp2q - 2
            aq = apbp2q*apbp2qm1/(2*qapbpq)
            bq = apbp2qm1*bbmaa/(2*qapbpq*apbp2qm2)
            cq = apbp2q*(a + q - 1)*(b + q - 1)/(qapbpq*apbp2qm2)
            j.append((aq*z - bq)*j[-1] - cq*j[-2])
    return j


def jacobi_diff(n, a, b, z):
    dj = [0.0]
    if n >= 1:
        dj.extend(jp*(i + a + b + 2)/2
                  for i, jp in enumerate(jacobi(n - 1, a + 1, b + 1, z)))
    return dj


class _Basis:
    """Orthonormal tensor-product Legendre basis of given order (number of
    modes per direction) on [-1, 1]^ndims, with nodal variants."""

    def __init__(self, ndims, order, pts):
        self.ndims, self.order = ndims, order
        self.pts = np.atleast_2d(np.asarray(pts, dtype=float))
        if self.ndims == 1 and self.pts.shape[0] == 1:
            self.pts = self.pts.T

    def _leg(self, x):
        sk = [sqrt(k + 0.5) for k in range(self.order)]
        return [c*p for c, p in zip(sk, jacobi(self.order - 1, 0, 0, x))]

    def _dleg(self, x):
        sk = [sqrt(k + 0.5) for k in range(self.order)]
        return [c*p for c, p in zip(sk, jacobi_diff(self.order - 1, 0, 0, x))]

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

    def opmat(self, expr):
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
        raise ValueError(f'unsupported operator expression {expr!r}')
