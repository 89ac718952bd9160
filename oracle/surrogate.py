# -*- coding: utf-8 -*-
"""FP64 restatement of the collision surrogate's pieces -- TEST
INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The surrogate has no counterpart in the reference; these functions define
what the B200 kernels must compute so that their results and gradients can
be checked: the windowed Hermite embedding of a distribution in its local
frame, the reconstruction of Q from windowed Hermite coefficients with the
conservation projection, and the MLP forward/backward pass.  The frame moments follow
frfs/plugins/dgfsmomwriterstd.py:154-190 (nondimensional).
"""

from math import factorial

import numpy as np
from scipy.special import erfc

from oracle.vhs import project_conservative

DEG = 9
WIN_R, WIN_W = 4.0, 0.4     # window chi(c^) = erfc((|c^| - WIN_R)/WIN_W)/2


def modes(deg=DEG):
    """(i, j, k) with i+j+k <= deg, ordered by degree, then i, then j
    (descending), as the device tables."""
    out = []
    for d in range(deg + 1):
        for i in range(d, -1, -1):
            for j in range(d - i, -1, -1):
                out.append((i, j, d - i - j))
    return out


def phi(n, x):
    """phi_n(x) = He_n(sqrt(2) x)/sqrt(n!) (probabilists' Hermite)."""
    y = np.sqrt(2.0)*x
    p = [np.ones_like(y), y]
    for k in range(1, n):
        p.append(y*p[k] - k*p[k - 1])
    return p[n]/np.sqrt(factorial(n))


def frame(f, cv, cw):
    f = np.asarray(f, np.float64)
    m0 = f.sum()
    u = (cv*f).sum(axis=1)/m0
    c = cv - u[:, None]
    T = (f*np.sum(c*c, axis=0)).sum()*(2.0/3.0)/m0
    return m0*cw, u, T


def window(cv, u, T):
    ch = (cv - u[:, None])/np.sqrt(T)
    return 0.5*erfc((np.sqrt(np.sum(ch*ch, axis=0)) - WIN_R)/WIN_W)


def window_gram(nq=80):
    """Gw_kl = int chi(c^) W(c^) phi_k phi_l dc^ by a 3D Gauss-Hermite
    product rule of nq points per axis (mode by mode)."""
    x, w = np.polynomial.hermite.hermgauss(nq)
    w = w/np.sqrt(np.pi)
    P = np.stack([phi(n, x) for n in range(DEG + 1)])
    X, Y, Z = np.meshgrid(x, x, x, indexing='ij')
    cw3 = (0.5*erfc((np.sqrt(X*X + Y*Y + Z*Z) - WIN_R)/WIN_W) *
           w[:, None, None]*w[None, :, None]*w[None, None, :])
    m = modes()
    G = np.empty((len(m), len(m)))
    for p, (i, j, k) in enumerate(m):
        A = cw3*P[i][:, None, None]*P[j][None, :, None]*P[k][None, None, :]
        Ax = np.einsum('abc,la->lbc', A, P)
        Axy = np.einsum('lbc,mb->lmc', Ax, P)
        Axyz = np.einsum('lmc,nc->lmn', Axy, P)
        for q, (a, b, c) in enumerate(m):
            G[p, q] = Axyz[a, b, c]
    return G


def basis(cv, u, T, deg=DEG):
    ch = (cv - u[:, None])/np.sqrt(T)
    return np.stack([np.prod([phi(m[a], ch[a]) for a in range(3)], axis=0)
                     for m in modes(deg)])                      # (nmodes, V)


def local_maxwellian(cv, rho, u, T):
    ch2 = np.sum(((cv - u[:, None])/np.sqrt(T))**2, axis=0)
    return rho*T**-1.5*np.pi**-1.5*np.exp(-ch2)


def embed(f, cv, cw, L, Q=None, prefac=1.0, gamma=0.0, nu=None):
    """Features x (256: windowed coefficients of (f - M)/rho, sqrt(T)/L,
    u/L), frame (rho, u, T), eps and (if Q) targets b (256) of g = Q, or of
    the gain deviation g = Q + nu (f - M) given the collision frequency nu
    (M the local Maxwellian)."""
    f = np.asarray(f, np.float64)
    rho, u, T = frame(f, cv, cw)
    Phi = basis(cv, u, T)
    chi = window(cv, u, T)
    M = local_maxwellian(cv, rho, u, T)
    a = Phi @ (chi*(f - M))*cw/rho
    x = np.zeros(256)
    x[:len(a)] = a
    x[len(a)] = np.sqrt(T)/L
    x[len(a) + 1:len(a) + 4] = u/L
    deg = np.array([sum(m) for m in modes()])
    eps = np.sqrt(np.sum(a[deg >= 2]**2))
    b = None
    if Q is not None:
        g = np.asarray(Q, np.float64)
        if nu is not None:
            g = g + np.asarray(nu, np.float64)*(f - M)
        b = np.zeros(256)
        b[:len(a)] = Phi @ (chi*g)*cw/(prefac*rho*rho*T**(0.5*gamma))
    return x, (rho, u, T), eps, b


def reconstruct(b, mom, cv, prefac=1.0, gamma=0.0, Gw=None, f=None,
                nu=None):
    """Q from windowed coefficients b: d = Gw^{-1} b (Gw = window_gram();
    None: d = b), g = prefac rho^2 T^{gamma/2} T^{-3/2} W(c^) sum d_k phi_k,
    Q = g (or g - nu (f - M) given f and nu), then the conservation
    projection."""
    rho, u, T = mom
    Phi = basis(cv, u, T)
    ch2 = np.sum(((cv - u[:, None])/np.sqrt(T))**2, axis=0)
    W = np.pi**-1.5*np.exp(-ch2)
    d = np.asarray(b[:Phi.shape[0]], np.float64)
    if Gw is not None:
        d = np.linalg.solve(Gw, d)
    Q = prefac*rho*rho*T**(0.5*gamma)*T**-1.5*W*(d @ Phi)
    if nu is not None:
        Q = Q - np.asarray(nu, np.float64)*(
            np.asarray(f, np.float64) - local_maxwellian(cv, rho, u, T))
    return project_conservative(Q, cv)


# --------------------------------------------------------------------------
# MLP: x -> tanh(W1) -> tanh(W2) -> tanh(W3) -> W4 (+ Ws x); W[in][out]
# --------------------------------------------------------------------------
def bf16_round(x):
    """x rounded to FP32, then to the nearest BF16 (ties to even), as
    float64: the rounding the tensor-core products apply to their
    operands."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    u = u.astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _same(a):
    return a


def mlp_forward(params, X, rnd=None):
    """Forward pass; ``rnd`` (e.g. bf16_round) is applied to the activation
    operand of every product, as the tensor-core training products do."""
    r = rnd or _same
    W1, b1, W2, b2, W3, b3, W4, b4, Ws = params
    H1 = np.tanh(r(X) @ W1 + b1)
    H2 = np.tanh(r(H1) @ W2 + b2)
    H3 = np.tanh(r(H2) @ W3 + b3)
    Y = r(H3) @ W4 + b4 + r(X) @ Ws
    return Y, (X, H1, H2, H3)


def mlp_backward(params, cache, dY, rnd=None):
    """Backward pass; ``rnd`` is applied to both operands of every weight
    gradient and to the gradient operand of every input gradient."""
    r = rnd or _same
    W1, b1, W2, b2, W3, b3, W4, b4, Ws = params
    X, H1, H2, H3 = cache
    g = {}
    g['W4'] = r(H3).T @ r(dY)
    g['b4'] = dY.sum(axis=0)
    g['Ws'] = r(X).T @ r(dY)
    dZ3 = (r(dY) @ W4.T)*(1 - H3**2)
    g['W3'] = r(H2).T @ r(dZ3)
    g['b3'] = dZ3.sum(axis=0)
    dZ2 = (r(dZ3) @ W3.T)*(1 - H2**2)
    g['W2'] = r(H1).T @ r(dZ2)
    g['b2'] = dZ2.sum(axis=0)
    dZ1 = (r(dZ2) @ W2.T)*(1 - H1**2)
    g['W1'] = r(X).T @ r(dZ1)
    g['b1'] = dZ1.sum(axis=0)
    return g


def mse(Y, T, nused, w=None):
    d = (Y - T)[:, :nused]
    wt = np.ones(nused) if w is None else np.asarray(w)[:nused]
    M = Y.shape[0]
    loss = np.sum(wt*d*d)/(M*nused)
    dY = np.zeros_like(Y)
    dY[:, :nused] = 2*wt*d/(M*nused)
    return loss, dY
