# -*- coding: utf-8 -*-
"""FP64 numpy restatement of frfs's velocity mesh and VHS fast-spectral Q(f).

Test infrastructure only (see ``oracle/__init__.py``).
"""

from math import gamma as _gammafn
import os

import numpy as np
import scipy.fft as sfft

R0 = 8.3144598           # frfs/solvers/dgfs/velocitymesh.py:8
NA = 6.0221409e+23       # frfs/solvers/dgfs/velocitymesh.py:9


def _workers():
    """Threads of every FFT: DGFS_ORACLE_THREADS if set (the timed CPU
    baseline runs one single-threaded process per core), else all cores."""
    env = os.environ.get('DGFS_ORACLE_THREADS')
    if env:
        return max(1, int(env))
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# --------------------------------------------------------------------------
# Quadrature: frfs/quadratures.py:6-44 (Golub-Welsch via eigh)
# --------------------------------------------------------------------------
def rjacobi(n, a, b):
    """Recurrence coefficients; frfs/quadratures.py:6-30."""
    ra, rb = np.zeros(n), np.zeros(n)
    apbp2 = 2. + a + b
    ra[0] = (b - a)/apbp2
    rb[0] = 2.0**(a + b + 1)*(_gammafn(a + 1.)*_gammafn(b + 1.) /
                               _gammafn(apbp2))
    rb[1] = 4.*(a + 1.)*(b + 1.)/((apbp2 + 1.)*apbp2*apbp2)
    apbp2 += 2
    for i in range(1, n - 1):
        ra[i] = (b*b - a*a)/((apbp2 - 2.)*apbp2)
        rb[i + 1] = (4.*(i + 1)*(i + 1 + a)*(i + 1 + b)*(i + 1 + a + b) /
                     ((apbp2*apbp2 - 1)*apbp2*apbp2))
        apbp2 += 2
    ra[n - 1] = (b*b - a*a)/((apbp2 - 2.)*apbp2)
    return ra, rb


def zwgj(n, a, b):
    """Gauss-Jacobi nodes/weights; frfs/quadratures.py:32-44."""
    ra, rb = rjacobi(n, a, b)
    scal = rb[0]
    off = np.sqrt(rb[1:])
    z, V = np.linalg.eigh(np.diag(ra) + np.diag(off, -1))
    idx = np.argsort(z)
    z = z[idx]
    V = V[:, idx]
    w = scal*V[0, :]**2
    return z, w


# --------------------------------------------------------------------------
# Velocity mesh: frfs/solvers/dgfs/velocitymesh.py:25-135
# --------------------------------------------------------------------------
def velocity_mesh(Nv, Nrho, M, sz_full, H0, T0, rho0, molarMass0, cmax,
                  Tmax, dev, qa=0.0, qb=0.0):
    """Return a dict with L, cw, c0, cv, qz, qw, sz, sw, n0, u0.

    ``sz_full`` is the 2M-point symmetric design; its first M rows form the
    half sphere (velocitymesh.py:128-135).
    """
    n0 = rho0/molarMass0*NA                              # :33
    u0 = np.sqrt(2*R0/molarMass0*T0)                      # :34
    L = cmax/u0 + dev*np.sqrt(Tmax/T0)                    # :59-63
    S = L*2.0/(3.0 + np.sqrt(2.0))                        # :64
    R = 2*S                                               # :65
    cw = (2.0*L/Nv)**3                                    # :73
    c0 = np.linspace(-L + L/Nv, L - L/Nv, Nv)             # :74
    V = Nv**3
    idx = np.arange(V)
    cv = np.stack([c0[idx//(Nv*Nv)], c0[(idx % (Nv*Nv))//Nv],
                   c0[idx % Nv]])                         # :78-85, I slowest
    qz, qw = zwgj(Nrho, qa, qb)                           # :122
    qz = (R/2.0)*(1.0 + qz)                               # :124
    qw = ((R - 0.0)/2.0)*qw                               # :125
    sz = np.asarray(sz_full)[:M, :]                       # :133
    sw = 2*np.pi/M                                        # :134
    return dict(Nv=Nv, V=V, L=L, S=S, R=R, cw=cw, c0=c0, cv=cv, qz=qz,
                qw=qw, sz=sz, sw=sw, n0=n0, u0=u0, M=M, Nrho=Nrho)


def vhs_parameters(omega, dRef, Tref, H0, n0, T0):
    """gamma and prefactor; frfs/solvers/dgfs/scattering.py:50-65."""
    alpha = 1.0
    gam = 2.0*(1 - omega)
    invKn = H0*np.sqrt(2.0)*np.pi*n0*dRef*dRef*pow(Tref/T0, omega - 0.5)
    prefac = invKn*alpha/(pow(2.0, 2 - omega + alpha)*_gammafn(2.5 - omega)
                          * np.pi)
    return gam, prefac


def maxwellian(cv, rho, u, T):
    """frfs/solvers/dgfs/initcond.py:62-64 (nondimensional inputs)."""
    u = np.asarray(u, dtype=float).reshape(3, 1)
    return (rho/(np.pi*T)**1.5)*np.exp(-np.sum((cv - u)**2, axis=0)/T)


def bkw(cv, t0):
    """BKW initial state; frfs/solvers/dgfs/initcond.py:128-137."""
    K = 1.0 - np.exp(-t0/6.0)
    cSqr = np.sum(cv*cv, axis=0)
    return (1/(2*pow(2*np.pi*K, 1.5))*np.exp(-cSqr/(2.0*K)) *
            ((5*K - 3)/K + (1 - K)/(K*K)*cSqr))


# --------------------------------------------------------------------------
# VHS precomputation: scattering.py:67-126 and vhs-gll.mako:45-101
# --------------------------------------------------------------------------
def _sinc(s):
    """vhs-gll.mako:11-14 (the kernels' definition, not numpy's)."""
    return np.sin(s + 1e-15)/(s + 1e-15)


def vhs_precompute(vm, gam):
    """Return l (3,V), aa (P,M,V), bb1 (P,V), bb2 (V)."""
    Nv, V, L = vm['Nv'], vm['V'], vm['L']
    qz, qw, sz = vm['qz'], vm['qw'], vm['sz']
    P, M = len(qz), sz.shape[0]
    l0 = np.concatenate((np.arange(0, Nv/2), np.arange(-Nv/2, 0)))  # :79
    idx = np.arange(V)
    l = np.stack([l0[idx//(Nv*Nv)], l0[(idx % (Nv*Nv))//Nv],
                  l0[idx % Nv]])                                     # :82-90
    aa = np.empty((P, M, V))
    for p in range(P):
        fac = np.pi/L*qz[p]/2.
        for q in range(M):
            # vhs-gll.mako:62-65
            aa[p, q] = fac*((sz[q, 0]*l[0]) + (sz[q, 1]*l[1]) +
                            (sz[q, 2]*l[2]))
    cSqr = np.sqrt(l[0]*l[0] + l[1]*l[1] + l[2]*l[2])                 # :84-86
    bb1 = np.empty((P, V))
    bb2 = np.zeros(V)
    for p in range(P):
        bb1[p] = pow(qz[p], gam + 2.)*4*np.pi*_sinc(np.pi/L*qz[p]/2.*cSqr)
        bb2 += qw[p]*pow(qz[p], gam + 2.)*16*np.pi*np.pi*_sinc(
            np.pi/L*qz[p]*cSqr)                                       # :88-97
    return dict(l=l, aa=aa, bb1=bb1, bb2=bb2, P=P, M=M)


def _fft(x, axes):
    # cuFFT forward: unnormalised, exp(-2 pi i ...)
    return sfft.fftn(x, axes=axes, norm='backward', workers=_workers())


def _ifft(x, axes):
    # cuFFT inverse: unnormalised, exp(+2 pi i ...)
    return sfft.ifftn(x, axes=axes, norm='forward', workers=_workers())


def vhs_Q(f, vm, pre, prefac, batch_pm=None):
    """Q(f) at one point, FP64, in the reference's operation order.

    Follows DGFSVHSGLLScatteringModel.fs (scattering.py:227-286) with the
    kernels of vhs-gll.mako: cosSinMul (103-140, including the 1/V scale of
    the spectrum), batched inverse FFTs (scattering.py:250-253), magSqr
    (142-169, complex squares), batched forward FFT (260-261), computeQG
    (172-207, weight 2 qw_p sw / V), inverse FFT (272-273), ax (209-220),
    inverse FFT (280-281) and output (246-266, real parts).  That is
    exactly 3*M*Nrho + 3 three-dimensional FFTs.
    """
    Nv, V = vm['Nv'], vm['V']
    P, M = pre['P'], pre['M']
    qw, sw = vm['qw'], vm['sw']
    shp = (Nv, Nv, Nv)
    f = np.asarray(f, dtype=np.float64)

    FTf = _fft(f.reshape(shp).astype(np.complex128), (0, 1, 2)).ravel()
    FTf = FTf/V                                              # mako:120
    fC = np.zeros(V, dtype=np.complex128)
    aa = pre['aa'].reshape(P*M, V)
    nb = batch_pm or P*M
    for b0 in range(0, P*M, nb):
        b1 = min(P*M, b0 + nb)
        a = aa[b0:b1]
        t1 = np.cos(a)*FTf[None, :]                          # mako:129-133
        t2 = np.sin(a)*FTf[None, :]                          # mako:135-136
        t3 = _ifft(t1.reshape((-1,) + shp), (1, 2, 3))
        t4 = _ifft(t2.reshape((-1,) + shp), (1, 2, 3))
        t2 = (t3.real*t3.real - t3.imag*t3.imag + t4.real*t4.real -
              t4.imag*t4.imag) + 1j*(2*t3.real*t3.imag +
                                     2*t4.real*t4.imag)      # mako:162-164
        t1 = _fft(t2, (1, 2, 3)).reshape(b1 - b0, V)
        for k in range(b0, b1):
            p = k // M
            intw = 2.*qw[p]*sw/V*pre['bb1'][p]               # mako:194
            fC += intw*t1[k - b0]
    QG = _ifft(fC.reshape(shp), (0, 1, 2)).ravel()          # scattering:272
    FTf = FTf*pre['bb2']                                     # mako:216-217
    Lf = _ifft(FTf.reshape(shp), (0, 1, 2)).ravel()         # scattering:280
    return prefac*(QG.real - f*Lf.real)                      # mako:264


def vhs_Q_gain_loss(f, vm, pre, prefac):
    """Same as vhs_Q but returns (gain, loss_frequency) separately."""
    Nv, V = vm['Nv'], vm['V']
    shp = (Nv, Nv, Nv)
    Qf = vhs_Q(f, vm, pre, prefac)
    FTf = _fft(np.asarray(f, np.float64).reshape(shp).astype(np.complex128),
               (0, 1, 2)).ravel()/V
    Lf = _ifft((FTf*pre['bb2']).reshape(shp), (0, 1, 2)).ravel().real
    gain = Qf/prefac + f*Lf
    return gain*prefac, Lf*prefac


# --------------------------------------------------------------------------
# Independent direct evaluation of the same discrete formula (no FFTs)
# --------------------------------------------------------------------------
def vhs_direct(f, vm, pre, prefac):
    """Q(f) from explicit DFT matrices, for small N only.

    This evaluates the formula of scattering.py:227-286 without any FFT
    library: every 3D transform is the Kronecker product of explicit 1D DFT
    matrices applied mode by mode, and the gain sum runs over (p, q) in the
    order written in computeQG (vhs-gll.mako:186-203).  It is an independent
    check of the index order, signs and normalisation used by ``vhs_Q``.
    """
    Nv, V = vm['Nv'], vm['V']
    P, M = pre['P'], pre['M']
    n = np.arange(Nv)
    Fw = np.exp(-2j*np.pi*np.outer(n, n)/Nv)     # forward 1D DFT
    Bw = np.exp(+2j*np.pi*np.outer(n, n)/Nv)     # inverse, unnormalised

    def tr3(D, x):
        x = x.reshape(Nv, Nv, Nv)
        x = np.einsum('ai,ijk->ajk', D, x)
        x = np.einsum('bj,ajk->abk', D, x)
        x = np.einsum('ck,abk->abc', D, x)
        return x.ravel()

    FTf = tr3(Fw, np.asarray(f, np.complex128))/V
    fC = np.zeros(V, dtype=np.complex128)
    for p in range(P):
        acc = np.zeros(V, dtype=np.complex128)
        for q in range(M):
            a = pre['aa'][p, q]
            g = tr3(Bw, np.exp(1j*a)*FTf)
            h = tr3(Bw, np.exp(-1j*a)*FTf)
            # cos/sin form: t3^2 + t4^2 = g*h algebraically
            acc += tr3(Fw, g*h)
        fC += 2.*vm['qw'][p]*vm['sw']/V*pre['bb1'][p]*acc
    QG = tr3(Bw, fC)
    Lf = tr3(Bw, FTf*pre['bb2'])
    return prefac*(QG.real - np.asarray(f)*Lf.real)


def moments(f, cv, cw):
    """rho, u, T, q (3D) as in frfs/plugins/dgfsmomwriterstd.py:154-190
    (nondimensional, mr = 1)."""
    f = np.asarray(f, np.float64)
    rho = np.sum(f)*cw
    u = np.array([np.dot(f, cv[i]) for i in range(3)])*cw/rho
    c = cv - u[:, None]
    cSqr = np.sum(c*c, axis=0)
    T = np.sum(f*cSqr)*(2.0/3.0*cw)/rho
    q = np.array([np.sum(f*cSqr*c[i]) for i in range(3)])*cw
    return rho, u, T, q


def project_conservative(Q, cv):
    """Least-squares projection of Q onto zero mass, momentum and energy
    moments: Q - phi^T G^{-1} (phi Q), phi = (1, cx, cy, cz, |c|^2),
    G = phi phi^T.  The reference has no such stage; this is the FP64
    definition the B200 kernel's optional projection is checked against."""
    phi = np.vstack([np.ones(cv.shape[1]), cv, np.sum(cv*cv, axis=0)])
    G = phi @ phi.T
    lam = np.linalg.solve(G, phi @ Q)
    return Q - lam @ phi
