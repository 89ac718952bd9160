# -*- coding: utf-8 -*-
"""Element geometry of the FR-DG discretisation.

Restates the numpy side of frfs/solvers/base/elements.py:83-354 for the
quadrilateral elements of the hot path: physical point locations through the
shape-point basis, Kopriva's free-stream-preserving metric terms
S = |J| J^{-1} on the order-p pseudo grid (``mpts``) interpolated to the
solution and flux points, |J|, the physical normals |S^T n| and n-hat at the
flux points, and the fuzzy coordinate sort of each face's flux points that
pairs the two sides of an interface (frfs/nputil.py:fuzzysort).
"""

import numpy as np

from frfs_b200.shapes import tol_runs


def fuzzysort(arr, idx, dim=0, tol=1e-6):
    """Order the points ``idx`` by coordinate ``dim``; points whose
    coordinate agrees within ``tol`` (runs anchored at their first member,
    as in ``clean``) are ordered among themselves by the next coordinate.
    This is the face flux-point ordering frfs pairs interfaces with
    (frfs/nputil.py:84-100).  Points that agree within ``tol`` in every
    coordinate cannot be ordered (a degenerate face): ValueError."""
    if dim == len(arr):
        raise ValueError(f'flux points of a face coincide within {tol} in '
                         'every coordinate (degenerate element)')
    key = arr[dim]
    order = sorted(idx, key=key.__getitem__)
    out = []
    for i, j in tol_runs([key[k] for k in order], tol):
        run = order[i:j]
        out.extend(fuzzysort(arr, run, dim + 1, tol) if j - i > 1 else run)
    return out


class ElementGeometry:
    def __init__(self, shape, spt):
        self.shape = shape
        self.eles = np.asarray(spt, dtype=np.float64)
        self.nspts, self.neles, self.ndims = self.eles.shape
        if self.ndims != 2:
            raise ValueError('only 2D quadrilateral meshes are supported')
        self._geom()

    def ploc_at(self, pts):
        op = self.shape.sbasis.nodal_basis_at(pts)
        ploc = op @ self.eles.reshape(self.nspts, -1)
        return ploc.reshape(-1, self.neles, self.ndims).swapaxes(1, 2)

    def _geom(self):
        sh, ndims, neles = self.shape, self.ndims, self.neles
        nmpts = sh.nmpts
        x = self.ploc_at(sh.mpts)
        jacop = np.rollaxis(sh.mbasis.jac_nodal_basis_at(sh.mpts), 2)
        jacop = jacop.reshape(-1, nmpts)
        jac = (jacop @ x.reshape(nmpts, -1)).reshape(nmpts, ndims, ndims,
                                                     neles)
        jac = jac.transpose(1, 2, 0, 3)
        a, b, c, d = jac[0, 0], jac[1, 0], jac[0, 1], jac[1, 1]
        smats = np.empty((ndims, nmpts, ndims, neles))
        smats[0, :, 0], smats[0, :, 1] = d, -b
        smats[1, :, 0], smats[1, :, 1] = -c, a
        self._smats_mpts = smats.reshape(ndims, nmpts, -1)
        self._djacs_mpts = a*d - b*c

        self.plocfpts = (sh.sbasis.nodal_basis_at(sh.fpts) @
                         self.eles.reshape(self.nspts, -1)).reshape(
            sh.nfpts, neles, ndims)
        self.ploc_upts = self.ploc_at(sh.upts)

        sm_f = self.smat_at(sh.fpts).transpose(1, 3, 0, 2)
        pnorm = np.einsum('ijlk,il->ijk', sm_f, sh.norm_fpts)
        mag = np.sqrt(np.einsum('...i,...i', pnorm, pnorm))
        if np.any(mag < 1e-10):
            raise RuntimeError('Zero face normals detected')
        self.norm_pnorm_fpts = pnorm/mag[..., None]
        self.mag_pnorm_fpts = mag

        pts = self.plocfpts.transpose(1, 2, 0)
        self.srtd_face_fpts = [
            [np.array(fuzzysort(p.tolist(), ff)) for p in pts]
            for ff in sh.facefpts]

    def smat_at(self, pts):
        m0 = self.shape.mbasis.nodal_basis_at(pts)
        smats = np.array([m0 @ s for s in self._smats_mpts])
        return smats.reshape(self.ndims, -1, self.ndims, self.neles)

    def djac_at(self, pts):
        djac = self.shape.mbasis.nodal_basis_at(pts) @ self._djacs_mpts
        if np.any(djac < -1e-5):
            raise RuntimeError('Negative mesh Jacobians detected')
        return djac

    def rcpdjac_at(self, pts):
        return 1.0/self.djac_at(pts)
