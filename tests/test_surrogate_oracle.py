# -*- coding: utf-8 -*-
"""Self-consistency of the surrogate's FP64 oracle (CPU): the Hermite basis,
the embedding/reconstruction pair and the MLP gradients that the GPU
kernels are checked against."""

import numpy as np

from helpers import config
from frfs_b200.velocitymesh import DGFSVelocityMesh
from oracle import surrogate as osur
from oracle import vhs as ovhs


def _vm():
    return DGFSVelocityMesh(None, config('couette-n24'))


def test_modes_count_and_order():
    m = osur.modes()
    assert len(m) == 220 and len(set(m)) == 220
    deg = [sum(t) for t in m]
    assert deg == sorted(deg)
    assert m[:4] == [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]


def test_phi_orthonormal():
    x, w = np.polynomial.hermite.hermgauss(30)
    w = w/np.sqrt(np.pi)
    G = np.array([[np.sum(w*osur.phi(m, x)*osur.phi(n, x))
                   for n in range(10)] for m in range(10)])
    assert np.max(np.abs(G - np.eye(10))) < 1e-12


def test_embedding_of_a_maxwellian():
    vm = _vm()
    cv, cw = vm.cv(), vm.cw()
    f = ovhs.maxwellian(cv, 1.3, [0.2, -0.1, 0.05], 1.2)
    x, (rho, u, T), eps, _ = osur.embed(f, cv, cw, vm.L())
    assert abs(rho - 1.3) < 1e-6 and abs(T - 1.2) < 1e-6
    assert np.max(np.abs(u - [0.2, -0.1, 0.05])) < 1e-6
    # features are coefficients of f - M: zero for a Maxwellian up to the
    # grid quadrature of its moments
    assert np.max(np.abs(x[:220])) < 1e-6
    assert eps < 1e-6
    assert abs(x[220] - np.sqrt(T)/vm.L()) < 1e-15


def test_reconstruct_then_embed_round_trip():
    """Windowed coefficients with zero mass, momentum and energy survive
    reconstruction (inverse windowed Gram, projection) and re-embedding, up
    to the grid quadrature of the window integrals."""
    vm = _vm()
    cv, cw = vm.cv(), vm.cw()
    rng = np.random.default_rng(3)
    deg = np.array([sum(t) for t in osur.modes()])
    Gw = osur.window_gram()
    d = np.zeros(220)
    d[:] = rng.standard_normal(220)*0.5**deg
    d[:4] = 0.0
    tr = [osur.modes().index(t) for t in ((2, 0, 0), (0, 2, 0), (0, 0, 2))]
    d[tr] -= d[tr].mean()
    b = np.zeros(256)
    b[:220] = Gw @ d
    mom = (1.1, np.array([0.1, 0.0, -0.2]), 0.9)
    prefac, gamma = 0.7, 0.38
    Q = osur.reconstruct(b, mom, cv, prefac, gamma, Gw=Gw)
    f = ovhs.maxwellian(cv, mom[0], mom[1], mom[2])
    _, _, _, b2 = osur.embed(f, cv, cw, vm.L(), Q=Q, prefac=prefac,
                             gamma=gamma)
    # grid (spacing 0.48 in c^) against continuum window integrals
    assert np.max(np.abs(b2[:220] - b[:220])) < 3e-5*np.max(np.abs(b))
    phi = np.vstack([np.ones(cv.shape[1]), cv, np.sum(cv*cv, axis=0)])
    assert np.max(np.abs(phi @ Q)) < 1e-12*np.max(np.abs(Q))*cv.shape[1]


def test_window_gram_of_the_product_matches():
    """The host table the surrogate passes to the reconstruction kernel
    (frfs_b200.surrogate.window_gram_inverse) inverts the oracle's Gram."""
    from frfs_b200.surrogate import hermite_modes, window_gram_inverse
    assert hermite_modes() == osur.modes()
    G = osur.window_gram()
    assert np.max(np.abs(window_gram_inverse() @ G - np.eye(220))) < 1e-7
    ev = np.linalg.eigvalsh(0.5*(G + G.T))
    assert 1.7 < ev.max()/ev.min() < 1.8


def _params(rng, nin, wd, nout):
    return [rng.standard_normal((nin, wd))/np.sqrt(nin),
            0.1*rng.standard_normal(wd),
            rng.standard_normal((wd, wd))/np.sqrt(wd),
            0.1*rng.standard_normal(wd),
            rng.standard_normal((wd, wd))/np.sqrt(wd),
            0.1*rng.standard_normal(wd),
            rng.standard_normal((wd, nout))/np.sqrt(wd),
            0.1*rng.standard_normal(nout),
            0.1*rng.standard_normal((nin, nout))]


def test_mlp_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    nin, wd, nout, B = 7, 6, 5, 4
    P = _params(rng, nin, wd, nout)
    X = rng.standard_normal((B, nin))
    T = rng.standard_normal((B, nout))
    w = rng.uniform(0.5, 2.0, nout)

    def loss(P):
        Y, _ = osur.mlp_forward(P, X)
        return osur.mse(Y, T, nout - 1, w)[0]

    Y, cache = osur.mlp_forward(P, X)
    _, dY = osur.mse(Y, T, nout - 1, w)
    g = osur.mlp_backward(P, cache, dY)
    names = ['W1', 'b1', 'W2', 'b2', 'W3', 'b3', 'W4', 'b4', 'Ws']
    h = 1e-6
    for k, name in enumerate(names):
        flat = P[k].reshape(-1)
        for i in rng.choice(flat.size, size=min(5, flat.size), replace=False):
            old = flat[i]
            flat[i] = old + h
            lp = loss(P)
            flat[i] = old - h
            lm = loss(P)
            flat[i] = old
            fd = (lp - lm)/(2*h)
            assert abs(fd - g[name].reshape(-1)[i]) < 1e-7 + 1e-5*abs(fd), \
                (name, i, fd, g[name].reshape(-1)[i])


def test_bf16_round_matches_torch():
    """The oracle's BF16 rounding (FP32 first, then nearest even) is
    torch's float32 -> bfloat16 conversion, over 40 binades."""
    import torch
    rng = np.random.default_rng(0)
    x = rng.standard_normal(20000)*np.exp(rng.uniform(-20, 20, 20000))
    x = np.concatenate([x, [0.0, -0.0, 1.0, 1.00390625, 1.01171875]])
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16)
    assert np.array_equal(osur.bf16_round(x), ref.double().numpy())
