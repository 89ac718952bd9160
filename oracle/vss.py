# -*- coding: utf-8 -*-
"""FP64 numpy restatement of frfs's binary-mixture VSS fast-spectral
operator: the mixture velocity mesh (frfs/solvers/dgfsbi/velocitymesh.py),
the per-pair parameters and precomputation
(frfs/solvers/dgfsbi/scattering.py:44-224) and Q_ij
(scattering.py:227-330 with the kernels of
frfs/solvers/dgfsbi/kernels/scattering/vss-gll.mako).

Test infrastructure only (see ``oracle/__init__.py``): the checker of the
product's VSS kernel (tests/test_vss_gpu.py).  Conventions as the VHS
oracle: cuFFT's unnormalised forward/inverse transforms, velocity index I
slowest.
"""

from math import gamma as _gammafn

import numpy as np

from oracle.vhs import NA, R0, _fft, _ifft, zwgj


def mixture_mesh(Nv, Nrho, sz_full, masses_molar, H0, T0, rho0, molarMass0,
                 cmax, Tmax, dev, qa=0.0, qb=0.0):
    """Velocity mesh of a mixture (dgfsbi/velocitymesh.py:27-151): the radial
    range R = 2S shrinks with the largest mass ratio, and the spherical rule
    is the full-sphere design (sw = 4 pi / M)."""
    n0 = rho0/molarMass0*NA                                  # :33
    u0 = np.sqrt(2*R0/molarMass0*T0)                          # :35
    masses = [m/molarMass0 for m in masses_molar]             # :60-63
    mr = max(masses)                                          # :64
    L = cmax/u0 + dev*np.sqrt(Tmax/T0)                        # :70
    S = min(L*2.0/(max(4.*mr/(1.+mr), 2.) + np.sqrt(1.+mr) + 1.),
            L*2.0/(max(4./(1.+mr), 2.) + np.sqrt(1.+1./mr) + 1.))  # :72-75
    R = 2*S                                                   # :76
    cw = (2.0*L/Nv)**3                                        # :85
    c0 = np.linspace(-L + L/Nv, L - L/Nv, Nv)                 # :86-87
    V = Nv**3
    idx = np.arange(V)
    cv = np.stack([c0[idx//(Nv*Nv)], c0[(idx % (Nv*Nv))//Nv],
                   c0[idx % Nv]])                             # :90-96
    qz, qw = zwgj(Nrho, qa, qb)                               # :137
    qz = (R/2.0)*(1.0 + qz)                                   # :139
    qw = ((R - 0.0)/2.0)*qw                                   # :140
    sz = np.asarray(sz_full, dtype=np.float64)                # :147-150
    return dict(Nv=Nv, V=V, L=L, S=S, R=R, cw=cw, c0=c0, cv=cv, qz=qz,
                qw=qw, sz=sz, sw=4*np.pi/sz.shape[0], n0=n0, u0=u0,
                masses=masses, T0=T0, H0=H0)


def vss_parameters(mesh, alpha, omega, dRef, Tref):
    """Per ordered pair 'pq': gamma, eta = alpha - 1 and the prefactor
    (dgfsbi/scattering.py:64-87); alpha, omega, dRef, Tref are dicts keyed
    'pq'."""
    m, out = mesh['masses'], {}
    for p in range(len(m)):
        for q in range(len(m)):
            pq = f'{p}{q}'
            a, w = alpha[pq], omega[pq]
            invKn = (np.sqrt(1. + m[p]/m[q])*np.pi*mesh['n0']*dRef[pq]**2 *
                     pow(Tref[pq]/mesh['T0'], w - 0.5)*mesh['H0'])
            mu = m[p]*m[q]/(m[p] + m[q])
            prefac = invKn*a/(np.sqrt(1. + m[p]/m[q])*pow(mu, w - 0.5) *
                              pow(2., 1 + a)*_gammafn(2.5 - w)*np.pi)
            out[pq] = dict(gamma=2.0*(1. - w), eta=a - 1., prefac=prefac)
    return out


def vss_precompute(mesh, params, szpre):
    """a (Nrho, M, V) and, per pair, b (Nrho, M, V) complex and c (V)
    complex (vss-gll.mako:31-93, scattering.py:172-198)."""
    Nv, V, L = mesh['Nv'], mesh['V'], mesh['L']
    qz, qw, sz, sw = mesh['qz'], mesh['qw'], mesh['sz'], mesh['sw']
    szpre = np.asarray(szpre, dtype=np.float64)
    swpre = 4*np.pi/szpre.shape[0]
    P, M = len(qz), sz.shape[0]
    l0 = np.concatenate((np.arange(0, Nv//2), np.arange(-Nv//2, 0)))
    idx = np.arange(V)
    l = np.stack([l0[idx//(Nv*Nv)], l0[(idx % (Nv*Nv))//Nv],
                  l0[idx % Nv]]).astype(np.float64)
    a = np.empty((P, M, V))
    for x in range(P):
        fac = np.pi/L*qz[x]
        for y in range(M):
            a[x, y] = fac*(sz[y] @ l)                          # :44-47
    lpre = szpre @ l                                          # (Mpre, V)
    masses, pre = mesh['masses'], {'a': a}
    for pq, prm in params.items():
        mp, mq = masses[int(pq[0])], masses[int(pq[1])]
        mpq = mq/(mp + mq)
        # (1 + cos)^eta (vss-gll.mako:74-76); for the antipodal pairs of a
        # symmetric design 1 + cos is 0 mathematically but +-1e-16 after
        # rounding, where the reference's pow gives NaN (negative) or up to
        # (1e-16)^eta (positive) depending on the summation order: values
        # below 1e-12 in magnitude are taken as the exact 0
        d = 1. + sz @ szpre.T
        d[np.abs(d) < 1e-12] = 0.0
        B = np.maximum(d, 0.0)**prm['eta']                     # (M, Mpre)
        b = np.empty((P, M, V), dtype=np.complex128)
        c = np.zeros(V, dtype=np.complex128)
        for x in range(P):
            fac = np.pi/L*qz[x]
            fac_b = swpre*pow(qz[x], prm['gamma'] + 2)
            fac_c = qw[x]*sw*fac_b
            eb = np.exp(-1j*mpq*fac*lpre)                     # (Mpre, V)
            ec = np.exp(-1j*fac*lpre)
            b[x] = fac_b*(B @ eb)                             # :73-82
            c += fac_c*np.sum(B @ ec, axis=0)                 # :83-91
        pre[pq] = dict(b=b, c=c)
    return pre


def vss_Qpq(fp, fq, p, q, mesh, pre, params):
    """Q(f_p, f_q) at one point (scattering.py:227-315): gain from the
    mass-weighted phase products, loss f_p times IFFT(c G)."""
    Nv, V = mesh['Nv'], mesh['V']
    qw, sw = mesh['qw'], mesh['sw']
    mp, mq = mesh['masses'][p], mesh['masses'][q]
    pq = f'{p}{q}'
    sh = (Nv, Nv, Nv)
    F = _fft(np.asarray(fp, np.complex128).reshape(sh), (0, 1, 2)).reshape(V)/V
    G = _fft(np.asarray(fq, np.complex128).reshape(sh), (0, 1, 2)).reshape(V)/V
    a = pre['a']
    P, M, _ = a.shape
    t1 = np.exp(1j*a*(mq/(mp + mq)))*F                        # mako :128-135
    t2 = np.exp(-1j*a*(mp/(mp + mq)))*G                       # mako :137-140
    axes = (2, 3, 4)
    t3 = _ifft(t1.reshape(P, M, *sh), axes)
    t4 = _ifft(t2.reshape(P, M, *sh), axes)
    T = _fft(t3*t4, axes).reshape(P, M, V)
    w = (qw*sw/V)[:, None, None]                              # mako :190-198
    QGhat = np.sum(w*T*pre[pq]['b'], axis=(0, 1))
    QG = _ifft(QGhat.reshape(sh), (0, 1, 2)).reshape(V)
    fL = _ifft((pre[pq]['c']*G).reshape(sh), (0, 1, 2)).reshape(V)
    return params[pq]['prefac']*(QG.real - np.asarray(fp)*fL.real)  # :290-298


def vss_Q(fs, mesh, pre, params):
    """Q_p = sum_q Q(f_p, f_q) for every species (scattering.py:317-330)."""
    n = len(fs)
    return [sum(vss_Qpq(fs[p], fs[q], p, q, mesh, pre, params)
                for q in range(n)) for p in range(n)]


def mixture_maxwellian(cv, nden, m, u, T):
    """dgfsbi/initcond.py:67-74: n (m / (pi T))^{3/2} e^{-m |c - u|^2 / T}."""
    u = np.asarray(u, dtype=float).reshape(3, 1)
    return nden*(m/np.pi/T)**1.5*np.exp(-m*np.sum((cv - u)**2, axis=0)/T)
