# -*- coding: utf-8 -*-
"""FP64 numpy restatement of frfs's FR-DG advection residual for DGFS.

Test infrastructure only (see ``oracle/__init__.py``).

The element operators (M0, M1-M3*M2, M3) and geometry (smats, 1/|J|, face
normals, face-point pairing) are inputs: they are pinned separately against
fixtures produced by the reference's own shapes/elements code.  This module
restates the kernels that act on the distribution banks:

  disu        uf = M0 u                         frfs/solvers/dgfs/elements.py:55-59
  tdisf       F~_i = sum_k S_ik c_k u           kernels/tflux.mako:14-24, flux.mako:10-16
  tdivtpcorf  R = (M1 - M3 M2) F~               elements.py:78-82
  comm_flux   upwind common flux, interfaces    kernels/intcflux.mako:16-24,
              and boundaries                    rsolvers/rusanov.mako:46-50,
                                                bccflux.mako:20-36, bcs/*.mako
  tdivtconf   R += M3 uf                        elements.py:85-88
  negdivconf  R = -R / |J|                      kernels/negdivconf.mako:11-13
  update_bc   diffuse-wall flux sums            bcs/dgfs-wall-diffuse-update.mako:14-36,
                                                bcs/dgfs-wall-diffuse-cyl-update.mako
  (faces shared with another partition are a boundary region of type 'mpi'
  whose ghost values are the received partner values, kernels/mpicflux.mako)

Arrays: u (nupts, V, neles); uf (nfpts, V, neles).
"""

import numpy as np


class DGOracle:
    def __init__(self, ops, geo, con, bcons, cv, cw, bcs):
        """ops: dict M0, M132, M3; geo: dict smats (D,U,D,E), rcpdjac (U,E),
        nrm (F,E,D), mag (F,E), srtd [face][ele] -> fpt indices;
        con: (lhs, rhs) lists of (eidx, fidx); bcons: name -> [(eidx, fidx)];
        cv (3, V); bcs: name -> dict(type=..., fw=(V,), uw=(3,)), and for
        'dgfs-wall-diffuse-cyl' w = (npts, 4): the wall (Ux, Uy, Uz, T) at
        each of the region's flux points in self.bpts order (may be set
        after construction)."""
        self.M0, self.M132, self.M3 = ops['M0'], ops['M132'], ops['M3']
        self.smats, self.rcpdjac = geo['smats'], geo['rcpdjac']
        self.nrm, self.mag, self.srtd = geo['nrm'], geo['mag'], geo['srtd']
        self.ndims = self.smats.shape[0]
        self.cv, self.cw = cv, cw
        self.bcs = bcs
        # interface flux point pairs (fpt_l, e_l, fpt_r, e_r)
        self.ipairs = []
        for (el, fl), (er, fr) in zip(*con):
            for jl, jr in zip(self.srtd[fl][el], self.srtd[fr][er]):
                self.ipairs.append((jl, el, jr, er))
        self.bpts = {name: [(j, e) for e, f in recs for j in self.srtd[f][e]]
                     for name, recs in bcons.items()}
        self.bcvals = {name: np.ones((2, len(p)))
                       for name, p in self.bpts.items()}
        self._refl = {}

    # -- kernels --------------------------------------------------------
    def disu(self, u):
        return np.einsum('fu,uve->fve', self.M0, u)

    def tdisf(self, u):
        D = self.ndims
        fl = np.empty((D,) + u.shape)
        for i in range(D):
            fl[i] = sum(self.smats[i, :, k, :][:, None, :]*self.cv[k][None, :,
                                                                       None]*u
                        for k in range(D))
        return fl

    def _rusanov(self, ul, ur, n):
        D = self.ndims
        nv = sum(n[j]*self.cv[j] for j in range(D))
        a = np.abs(nv)
        return 0.5*nv*(ul + ur) + 0.5*a*(ul - ur)

    def _ghost(self, name, k, j, e, ul):
        bc = self.bcs[name]
        kind = bc['type']
        n = self.nrm[j, e]
        D = self.ndims
        if kind == 'dgfs-wall-diffuse':
            fac = sum((self.cv[i] - bc['uw'][i])*n[i] for i in range(D))
            b0, b1 = self.bcvals[name][:, k]
            return np.where(fac < 0, bc['fw']*(-b0/b1), ul)
        if kind == 'dgfs-inlet':
            fac = sum((self.cv[i] - bc['uw'][i])*n[i] for i in range(D))
            return np.where(fac < 0, bc['fw'], ul)
        if kind == 'dgfs-inlet-normalshock':
            # bcs/dgfs-inlet-normalshock.mako: c.n selects the incoming half
            fac = sum(self.cv[i]*n[i] for i in range(D))
            return np.where(fac < 0, bc['fw'], ul)
        if kind == 'dgfs-wall-diffuse-cyl':
            # bcs/dgfs-wall-diffuse-cyl.mako: the wall state (Ux, Uy, Uz, T)
            # of this boundary point, unnormalised Maxwellian
            fac, mx = self._cyl_wall(bc['w'][k], n)
            b0, b1 = self.bcvals[name][:, k]
            return np.where(fac < 0, mx*(-b0/b1), ul)
        if kind == 'dgfs-outlet':
            return ul
        if kind == 'dgfs-vanish':
            fac = sum(self.cv[i]*n[i] for i in range(D))
            return np.where(fac < 0, 0.0, ul)
        if kind == 'dgfs-wall-specular':
            return ul[self.specular_map(name, j, e)]
        if kind == 'mpi':
            # a face shared with another partition: the partner's face value
            # received from it (kernels/mpicflux.mako: the Riemann solve
            # against the received ur, scaled by the local |S^T n|)
            return bc['ur'][k]
        raise ValueError(kind)

    def _cyl_wall(self, w, n):
        """(c - U).n and exp(-|c - U|^2 / T) for a cylinder-wall point."""
        D = self.ndims
        dc = self.cv - np.asarray(w[:3]).reshape(3, 1)
        fac = sum(dc[i]*n[i] for i in range(D))
        return fac, np.exp(-np.sum(dc*dc, axis=0)/w[3])

    def specular_map(self, name, j, e):
        """Reflected-velocity index (frfs/solvers/dgfs/inters.py:244-275,
        flat-wall branch)."""
        n = np.zeros(3)
        n[:self.ndims] = self.nrm[j, e]
        key = (name, tuple(np.round(n, 12)))
        if key not in self._refl:
            cv = self.cv
            dot = n @ cv
            cr = cv - 2*dot[None, :]*n[:, None]
            idx = np.empty(cv.shape[1], dtype=np.int64)
            for v in range(cv.shape[1]):
                d = cr[:, v:v + 1] - cv
                idx[v] = np.argmin(np.sum(d**2, axis=0))
            self._refl[key] = idx
        return self._refl[key]

    def update_bc(self, uf):
        """Diffuse-wall sums over all velocities (reset, then accumulate)."""
        D = self.ndims
        for name, pts in self.bpts.items():
            bc = self.bcs[name]
            if bc['type'] not in ('dgfs-wall-diffuse', 'dgfs-wall-diffuse-cyl'):
                continue
            for k, (j, e) in enumerate(pts):
                n = self.nrm[j, e]
                if bc['type'] == 'dgfs-wall-diffuse':
                    fac = sum((self.cv[i] - bc['uw'][i])*n[i] for i in range(D))
                    fw = bc['fw']
                else:
                    # bcs/dgfs-wall-diffuse-cyl-update.mako
                    fac, fw = self._cyl_wall(bc['w'][k], n)
                ul = uf[j, :, e]
                self.bcvals[name][0, k] = np.sum(np.where(fac >= 0, fac*ul*self.cw,
                                                          0.0))
                self.bcvals[name][1, k] = np.sum(np.where(fac < 0,
                                                          fac*fw*self.cw,
                                                          0.0))

    def comm_flux(self, uf):
        out = uf.copy()
        for jl, el, jr, er in self.ipairs:
            fn = self._rusanov(uf[jl, :, el], uf[jr, :, er], self.nrm[jl, el])
            m = self.mag[jl, el]
            out[jl, :, el] = m*fn
            out[jr, :, er] = -m*fn
        for name, pts in self.bpts.items():
            for k, (j, e) in enumerate(pts):
                ul = uf[j, :, e]
                ur = self._ghost(name, k, j, e, ul)
                out[j, :, e] = self.mag[j, e]*self._rusanov(ul, ur,
                                                            self.nrm[j, e])
        return out

    def rhs(self, u, uf=None):
        """-div of the FR-DG flux (DGFSSystem.rhs, system.py:140-177); uses
        the current boundary values (call update_bc first)."""
        U, V, E = u.shape
        if uf is None:
            uf = self.disu(u)
        F = self.tdisf(u).reshape(self.ndims*U, V*E)
        R = (self.M132 @ F).reshape(U, V, E)
        ufc = self.comm_flux(uf)
        R += np.einsum('uf,fve->uve', self.M3, ufc)
        return -self.rcpdjac[:, None, :]*R


def ssp_rk2_step(dg, Qfun, u0, dt):
    """StdTVDRK2DGFSStepper.step (frfs/integrators/std/steppers.py:122-225)
    with all velocities in one batch."""
    q0 = Qfun(u0)
    dg.update_bc(dg.disu(u0))
    u1 = u0 + dt*dg.rhs(u0) + dt*q0
    q1 = Qfun(u1)
    dg.update_bc(dg.disu(u1))
    return 0.5*u0 + 0.5*u1 + 0.5*dt*(dg.rhs(u1) + q1)


def euler_step(dg, Qfun, u0, dt):
    """StdEulerDGFSStepper.step (steppers.py:39-100)."""
    q0 = Qfun(u0)
    dg.update_bc(dg.disu(u0))
    return u0 + dt*dg.rhs(u0) + dt*q0
