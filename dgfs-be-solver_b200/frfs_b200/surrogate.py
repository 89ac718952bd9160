# -*- coding: utf-8 -*-
"""Learned collision surrogate with the plain fast-spectral operator as
fallback and error reference (no counterpart in the reference).

Per solution point:

1. FP64 moments rho, u, T define a local frame c^ = (c - u)/sqrt(T);
2. the deviation f - M from the local Maxwellian is embedded as 220
   Hermite coefficients (total degree <= 9) in that frame, taken under the
   radial window erfc((|c^| - 4)/0.4)/2
   (the polynomials would otherwise amplify the round-off that f and Q hold
   at the corners of the velocity box), plus sqrt(T)/L and u/L (256
   features);
3. the degree >= 2 coefficients are divided by the deviation size
   s = max(eps, 1e-3) and log(s) is appended; an MLP (256 -> 512 -> 512 ->
   512 -> 256, tanh, with a linear skip from the input; BF16 weights, FP32
   accumulation) predicts the windowed Hermite coefficients of the gain
   deviation G - nu M = Q + nu (f - M) (nu the collision frequency, M the
   local Maxwellian) divided by prefac rho^2 T^{gamma/2} s: it is smooth
   even where f jumps at a diffuse wall, and near equilibrium it is linear
   in f - M, so both sides are O(1) whatever the distance from equilibrium;
4. nu(c) is computed exactly (two 3D transforms per point), Q = (G - nu M)
   - nu (f - M) is rebuilt on the velocity grid (windowed coefficients
   mapped back by the inverse windowed Gram matrix) and projected in FP64
   onto zero mass, momentum and energy moments.

A point uses the surrogate when its non-equilibrium measure eps (the norm of
its Hermite coefficients of degree >= 2, a local Knudsen indicator: Grad's
expansion deviates from the Maxwellian at O(Kn)) is below the threshold and
the velocity grid resolves its local Maxwellian ((L - |u_axis|) >=
3.5 sqrt(T); beyond that the plain operator's own truncation error, which
the features do not see, dominates Q);
below eps = 1e-3 (where the plain Q is the operator's aliasing) the
network is skipped and Q = -nu (f - M).  Every other point runs the plain
operator through a device point list, with no host round trip.  ``residual_check`` re-evaluates a sample of surrogate
points with the plain operator and reports their relative error, which the
caller compares with its tolerance to fall back to the plain operator.

All arithmetic runs in libdgfs_b200.so (embedding, gate, MLP forward and
backward, Adam, reconstruction); PyTorch allocates the buffers.
"""

import ctypes as ct

import numpy as np
import torch

from frfs_b200 import _lib

c_int, c_ll, c_double, c_float, c_void_p = (ct.c_int, ct.c_longlong,
                                            ct.c_double, ct.c_float,
                                            ct.c_void_p)
_lib.declare('dgfs_hermite_embed', c_int,
             [c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, c_ll, c_int,
              c_double, c_double, c_double, c_double, c_void_p, c_void_p,
              c_void_p, c_void_p, c_void_p])
_lib.declare('dgfs_hermite_reconstruct', c_int,
             [c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, c_ll, c_int,
              c_double, c_double, c_double, c_double, c_void_p, c_void_p,
              c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
              c_void_p])
_lib.declare('dgfs_surrogate_gate', c_int,
             [c_int, c_void_p, c_float, c_float, c_void_p, c_double,
              c_double, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
              c_void_p])
_lib.declare('dgfs_mlp_gemm', c_int,
             [c_int, c_int, c_int, c_void_p, c_ll, c_ll, c_void_p, c_int,
              c_ll, c_ll, c_void_p, c_void_p, c_void_p, c_ll, c_int, c_int,
              c_void_p, c_void_p])
_lib.declare('dgfs_mlp_gemm_tc', c_int,
             [c_int, c_int, c_int, c_void_p, c_ll, c_ll, c_void_p, c_int,
              c_ll, c_ll, c_void_p, c_void_p, c_void_p, c_ll, c_int, c_int,
              c_void_p, c_void_p])
_lib.declare('dgfs_mlp_gemm_bf16', c_int,
             [c_int, c_int, c_int, c_void_p, c_int, c_ll, c_void_p, c_int,
              c_ll, c_void_p, c_void_p, c_void_p, c_void_p, c_ll, c_int,
              c_int, c_void_p, c_void_p])
_lib.declare('dgfs_mlp_tanh_bwd', c_int, [c_ll, c_void_p, c_void_p,
                                          c_void_p, c_void_p])
_lib.declare('dgfs_mlp_tanh_bwd_bf16', c_int, [c_ll, c_void_p, c_void_p,
                                               c_void_p, c_void_p, c_void_p])
_lib.declare('dgfs_mlp_colsum', c_int, [c_int, c_int, c_void_p, c_ll,
                                        c_void_p, c_int, c_void_p])
_lib.declare('dgfs_mlp_mse', c_int, [c_int, c_int, c_int, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p, c_void_p])
_lib.declare('dgfs_mlp_adam', c_int, [c_ll, c_void_p, c_void_p, c_void_p,
                                      c_void_p, c_void_p, c_float, c_float,
                                      c_float, c_float, c_int, c_float,
                                      c_void_p])
_lib.declare('dgfs_mlp_adam_dev', c_int,
             [c_ll, c_ll, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
              c_void_p, c_float, c_float, c_float, c_float, c_void_p])
_lib.declare('dgfs_mlp_schedule', c_int,
             [c_void_p, c_void_p, c_float, c_float, c_int, c_float, c_float,
              c_void_p])
_lib.declare('dgfs_mlp_affine', c_int, [c_int, c_int, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_int, c_void_p])
_lib.declare('dgfs_mlp_affine_rows', c_int,
             [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
              c_void_p, c_int, c_void_p])
_lib.declare('dgfs_f32_to_bf16', c_int, [c_ll, c_void_p, c_void_p, c_void_p])
_lib.declare('dgfs_surrogate_scale', c_int,
             [c_int, c_int, c_void_p, c_float, c_int, c_int, c_int, c_int,
              c_void_p, c_void_p])

NFEAT = 256
NMODES = 220
WIDTH = 512
DEG = 9
EPS0 = 1e-3     # floor of the deviation scale s = max(eps, EPS0); below it
                # Q is dominated by the operator's aliasing, not by f - M
LOGCOL = 224    # feature column that carries log(max(eps, EPS0))
RMIN = 3.5      # resolved frames: (L - |u_axis|) >= RMIN sqrt(T) (the local
                # Maxwellian's mass outside the velocity box is ~e^-12)
WIN_R, WIN_W = 4.0, 0.4       # the kernels' window erfc((|c^| - 4)/0.4)/2


def hermite_modes():
    """(i, j, k), i + j + k <= 9, in the kernels' order (degree, then i,
    then j, both descending)."""
    return [(i, j, d - i - j) for d in range(DEG + 1)
            for i in range(d, -1, -1) for j in range(d - i, -1, -1)]


def window_gram_inverse(nq=100):
    """Inverse of Gw_kl = int chi(c^) W(c^) phi_k(c^) phi_l(c^) dc^, the
    Gram matrix of the windowed Hermite projection (condition number 1.75),
    by an nq-point Gauss-Hermite product rule: pair products of the 1D
    polynomials are contracted against the window one axis at a time.
    Row-major (220, 220) float64."""
    from scipy.special import erfc
    x, w = np.polynomial.hermite.hermgauss(nq)
    w = w/np.sqrt(np.pi)
    P = np.empty((DEG + 1, nq))
    P[0], P[1] = 1.0, np.sqrt(2.0)*x
    for n in range(1, DEG):
        P[n + 1] = (np.sqrt(2.0)*x*P[n] - np.sqrt(n)*P[n - 1])/np.sqrt(n + 1)
    P2 = (P[:, None, :]*P[None, :, :]*w).reshape(-1, nq)    # (100, nq)
    r = np.sqrt(x[:, None, None]**2 + x[None, :, None]**2 +
                x[None, None, :]**2)
    chi = 0.5*erfc((r - WIN_R)/WIN_W)
    T = np.einsum('abc,rc->abr', chi, P2)
    T = np.einsum('abr,qb->aqr', T, P2)
    T = np.einsum('aqr,pa->pqr', T, P2)                       # (100,)*3
    T = T.reshape((DEG + 1,)*6)                                # i i' j j' k k'
    m = hermite_modes()
    G = np.empty((len(m), len(m)))
    for p, (i, j, k) in enumerate(m):
        for q, (a, b, c) in enumerate(m):
            G[p, q] = T[i, a, j, b, k, c]
    return np.linalg.inv(G)


def _p(t):
    return None if t is None else t.data_ptr()


class _Workspace:
    """Buffers reused across calls, keyed by name, shape and dtype, so that a
    CUDA graph captured around a call keeps pointing at live memory."""

    def __init__(self, device):
        self.device = device
        self._bufs = {}

    def get(self, name, shape, dtype=torch.float32):
        key = (name, tuple(shape), dtype)
        t = self._bufs.get(key)
        if t is None:
            t = self._bufs[key] = torch.empty(shape, dtype=dtype,
                                              device=self.device)
        return t


class MLP:
    """4 layers of width 512 with a linear input->output skip; FP32 master
    weights, BF16 copies for the products, Adam optimiser; every kernel is
    libdgfs_b200's.  Weights are stored W[in][out], activations row-major
    [batch][features].

    The parameters live in one flat buffer (weights first, then biases) so
    that one Adam launch updates all of them.  ``tc`` chooses the training
    products (forward with ``keep``, backward): 'tma' (the default; True)
    keeps BF16 copies of the activations and gradients, written by the
    kernels that produce them, and multiplies them with dgfs_mlp_gemm_bf16
    (TMA loads into the tensor cores); 'staged' rounds FP32 operands as it
    stages them (dgfs_mlp_gemm_tc); False uses the SIMT product.  Both
    tensor-core modes round the same operands to BF16 and accumulate in
    FP32.  Inference keeps the FP32-activation SIMT product."""

    names = ('W1', 'b1', 'W2', 'b2', 'W3', 'b3', 'W4', 'b4', 'Ws')
    _order = ('W1', 'W2', 'W3', 'W4', 'Ws', 'b1', 'b2', 'b3', 'b4')

    def __init__(self, device, nin=NFEAT, width=WIDTH, nout=NFEAT, seed=0,
                 tc=True):
        self.device = device
        self.nin, self.width, self.nout = nin, width, nout
        self.tc = 'tma' if tc is True else (tc or False)
        assert self.tc in (False, 'staged', 'tma'), tc
        rng = np.random.default_rng(seed)
        shapes = {'W1': (nin, width), 'b1': (width,), 'W2': (width, width),
                  'b2': (width,), 'W3': (width, width), 'b3': (width,),
                  'W4': (width, nout), 'b4': (nout,), 'Ws': (nin, nout)}
        init = {}
        for k, shp in shapes.items():      # same draws as per-tensor storage
            if k in ('W1', 'W2', 'W3'):
                init[k] = rng.standard_normal(shp)/np.sqrt(shp[0])
            elif k == 'W4':
                init[k] = 0.1*rng.standard_normal(shp)/np.sqrt(shp[0])
            else:
                init[k] = np.zeros(shp)
        # flat layout: every slice starts on a multiple of 8 entries (16-byte
        # aligned BF16 views for the tensor-core loads)
        off, offs = 0, {}
        for k in self._order:
            offs[k] = off
            off += -(-int(np.prod(shapes[k]))//8)*8
        self.n = off
        self.n_decay = offs['b1']
        f32 = dict(dtype=torch.float32, device=device)
        self.flat_w = torch.zeros(off, **f32)
        self.flat_g = torch.zeros(off, **f32)
        self.flat_m1 = torch.zeros(off, **f32)
        self.flat_m2 = torch.zeros(off, **f32)
        self.flat_wb = torch.zeros(off, dtype=torch.bfloat16, device=device)
        self.w, self.g, self.m1, self.m2, self.wb = {}, {}, {}, {}, {}
        for k, shp in shapes.items():
            sl = slice(offs[k], offs[k] + int(np.prod(shp)))
            self.w[k] = self.flat_w[sl].view(shp)
            self.g[k] = self.flat_g[sl].view(shp)
            self.m1[k] = self.flat_m1[sl].view(shp)
            self.m2[k] = self.flat_m2[sl].view(shp)
            if k.startswith('W'):
                self.wb[k] = self.flat_wb[sl].view(shp)
            self.w[k].copy_(torch.tensor(init[k], dtype=torch.float32))
        self.step = 0
        self.ws = _Workspace(device)
        # {it, step} of the device learning-rate schedule, and its output
        # {lr, 1 - beta1^t, 1 - beta2^t}
        self.counters = torch.zeros(2, dtype=torch.int32, device=device)
        self.hyper = torch.zeros(3, **f32)
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self.sync_bf16()
        self._cache = None

    @property
    def _s(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def nparams(self):
        return sum(t.numel() for t in self.w.values())

    def train_flops_per_row(self):
        """Multiply-add FLOPs of one training row: the forward products,
        the weight gradients (the same sizes) and the input gradients of
        layers 4, 3 and 2."""
        nin, wd, nout = self.nin, self.width, self.nout
        fwd = 2*(nin*wd + 2*wd*wd + wd*nout + nin*nout)
        return 2*fwd + 2*(wd*nout + 2*wd*wd)

    def sync_bf16(self):
        _lib.check(_lib.load().dgfs_f32_to_bf16(
            self.n, _p(self.flat_w), _p(self.flat_wb), self._s),
            'dgfs_f32_to_bf16')

    def _gemm(self, A, B, C, M, N, K, sam, sak, sbk, sbn, bf16, bias=None,
              act=0, acc=0, mcount=None, tc=False):
        lib = _lib.load()
        if tc:
            assert mcount is None
            _lib.check(lib.dgfs_mlp_gemm_tc(
                M, N, K, _p(A), sam, sak, _p(B), 1 if bf16 else 0, sbk, sbn,
                _p(bias), None, _p(C), N, act, acc, _p(self.err), self._s),
                'dgfs_mlp_gemm_tc')
            return
        _lib.check(lib.dgfs_mlp_gemm(
            M, N, K, _p(A), sam, sak, _p(B), 1 if bf16 else 0, sbk, sbn,
            _p(bias), None, _p(C), N, act, acc, _p(mcount), self._s),
            'dgfs_mlp_gemm')

    def check_tc(self):
        """Raise if a bounded wait of a tensor-core product ran out (reads
        the device flag: synchronises the stream)."""
        if int(self.err.item()):
            raise _lib.DgfsError(2, 'dgfs_mlp_gemm_tc',
                                 'a bounded wait of the tensor-core GEMM '
                                 'ran out')

    def _gemm_bf16(self, A, a_mn, lda, B, b_mn, ldb, C, M, N, K, bias=None,
                   act=0, acc=0, Cb=None):
        _lib.check(_lib.load().dgfs_mlp_gemm_bf16(
            M, N, K, _p(A), a_mn, lda, _p(B), b_mn, ldb, _p(bias), None,
            _p(C), _p(Cb), N, act, acc, _p(self.err), self._s),
            'dgfs_mlp_gemm_bf16')

    def _to_bf16(self, X, Xb):
        _lib.check(_lib.load().dgfs_f32_to_bf16(X.numel(), _p(X), _p(Xb),
                                                self._s), 'dgfs_f32_to_bf16')

    def _forward_tma(self, X):
        """Training forward pass on BF16 operands: every layer writes its
        activations in FP32 (for the backward pass) and in BF16 (the next
        product's operand).  Weights W[in][out] are the MN-major B operand
        as stored."""
        B = X.shape[0]
        nin, wd, nout = self.nin, self.width, self.nout
        ws, wb, w = self.ws, self.wb, self.w
        Xb = ws.get('trainXb', (B, nin), torch.bfloat16)
        H = [ws.get('trainH%d' % i, (B, wd)) for i in (1, 2, 3)]
        Hb = [ws.get('trainH%db' % i, (B, wd), torch.bfloat16)
              for i in (1, 2, 3)]
        Y = ws.get('trainY', (B, nout))
        self._to_bf16(X, Xb)
        self._gemm_bf16(Xb, 0, nin, wb['W1'], 1, wd, H[0], B, wd, nin,
                        w['b1'], act=1, Cb=Hb[0])
        self._gemm_bf16(Hb[0], 0, wd, wb['W2'], 1, wd, H[1], B, wd, wd,
                        w['b2'], act=1, Cb=Hb[1])
        self._gemm_bf16(Hb[1], 0, wd, wb['W3'], 1, wd, H[2], B, wd, wd,
                        w['b3'], act=1, Cb=Hb[2])
        self._gemm_bf16(Hb[2], 0, wd, wb['W4'], 1, nout, Y, B, nout, wd,
                        w['b4'])
        self._gemm_bf16(Xb, 0, nin, wb['Ws'], 1, nout, Y, B, nout, nin,
                        acc=1)
        self._cache = (X, H[0], H[1], H[2])
        self._cache_bf16 = (Xb, Hb[0], Hb[1], Hb[2])
        return Y

    def _backward_tma(self, dY):
        """Backward pass on the BF16 copies: weight gradients g = A^T D
        read both operands MN-major (as stored), input gradients D W^T read
        W K-major (as stored)."""
        lib = _lib.load()
        X, H1, H2, H3 = self._cache
        Xb, H1b, H2b, H3b = self._cache_bf16
        B = X.shape[0]
        nin, wd, nout = self.nin, self.width, self.nout
        g, wb, ws = self.g, self.wb, self.ws
        dYb = ws.get('dYb', (B, nout), torch.bfloat16)
        dH = ws.get('dH', (B, wd))
        dZ = ws.get('dZ', (B, wd))
        dZb = ws.get('dZb', (B, wd), torch.bfloat16)
        self._to_bf16(dY, dYb)

        def wgrad(Ab, Db, name, k, n):
            self._gemm_bf16(Ab, 1, k, Db, 1, n, g[name], k, n, B)

        def bgrad(D, name, n):
            _lib.check(lib.dgfs_mlp_colsum(B, n, _p(D), n, _p(g[name]), 0,
                                           self._s), 'dgfs_mlp_colsum')

        def through(Db, nd, W, H):
            self._gemm_bf16(Db, 0, nd, W, 0, nd, dH, B, wd, nd)
            _lib.check(lib.dgfs_mlp_tanh_bwd_bf16(
                dH.numel(), _p(H), _p(dH), _p(dZ), _p(dZb), self._s),
                'dgfs_mlp_tanh_bwd_bf16')

        wgrad(H3b, dYb, 'W4', wd, nout)
        bgrad(dY, 'b4', nout)
        wgrad(Xb, dYb, 'Ws', nin, nout)
        through(dYb, nout, wb['W4'], H3)
        wgrad(H2b, dZb, 'W3', wd, wd)
        bgrad(dZ, 'b3', wd)
        through(dZb, wd, wb['W3'], H2)
        wgrad(H1b, dZb, 'W2', wd, wd)
        bgrad(dZ, 'b2', wd)
        through(dZb, wd, wb['W2'], H1)
        wgrad(Xb, dZb, 'W1', nin, wd)
        bgrad(dZ, 'b1', wd)
        return g

    def forward(self, X, keep=False, mcount=None):
        """Y = W4 tanh(W3 tanh(W2 tanh(W1 X + b1) + b2) + b3) + b4 + Ws X.
        With mcount (a device int), only the first *mcount rows."""
        if keep and self.tc == 'tma' and mcount is None:
            return self._forward_tma(X)
        B = X.shape[0]
        nin, wd, nout = self.nin, self.width, self.nout
        tag = 'train' if keep else 'infer'
        tc = keep and self.tc == 'staged' and mcount is None
        H1 = self.ws.get(tag + 'H1', (B, wd))
        H2 = self.ws.get(tag + 'H2', (B, wd))
        H3 = self.ws.get(tag + 'H3', (B, wd))
        Y = self.ws.get(tag + 'Y', (B, nout))
        wb, w = self.wb, self.w
        mc = mcount
        self._gemm(X, wb['W1'], H1, B, wd, nin, nin, 1, wd, 1, True,
                   w['b1'], act=1, mcount=mc, tc=tc)
        self._gemm(H1, wb['W2'], H2, B, wd, wd, wd, 1, wd, 1, True,
                   w['b2'], act=1, mcount=mc, tc=tc)
        self._gemm(H2, wb['W3'], H3, B, wd, wd, wd, 1, wd, 1, True,
                   w['b3'], act=1, mcount=mc, tc=tc)
        self._gemm(H3, wb['W4'], Y, B, nout, wd, wd, 1, nout, 1, True,
                   w['b4'], mcount=mc, tc=tc)
        self._gemm(X, wb['Ws'], Y, B, nout, nin, nin, 1, nout, 1, True,
                   acc=1, mcount=mc, tc=tc)
        if keep:
            self._cache = (X, H1, H2, H3)
        return Y

    def backward(self, dY):
        """Gradients of every parameter into self.g: weight gradients from
        the activations, input gradients through the BF16 weights that the
        forward pass used (on the tensor cores with ``tc``: activations and
        gradients rounded to BF16 as they are staged)."""
        if self.tc == 'tma':
            return self._backward_tma(dY)
        lib = _lib.load()
        X, H1, H2, H3 = self._cache
        B = X.shape[0]
        nin, wd, nout = self.nin, self.width, self.nout
        g, wb = self.g, self.wb
        tc = self.tc == 'staged'
        dH = self.ws.get('dH', (B, wd))
        dZ = self.ws.get('dZ', (B, wd))

        def wgrad(A, D, name, k, n):          # g = A^T D, (k x n), K = B
            self._gemm(A, D, g[name], k, n, B, 1, k, n, 1, False, tc=tc)

        def bgrad(D, name, n):
            _lib.check(lib.dgfs_mlp_colsum(B, n, _p(D), n, _p(g[name]), 0,
                                           self._s), 'dgfs_mlp_colsum')

        def through(D, nd, W, H):
            # dZ = (D W^T) o (1 - H^2); D may be dZ itself: the product is
            # complete (same stream) before dZ is overwritten
            self._gemm(D, W, dH, B, wd, nd, nd, 1, 1, nd, True, tc=tc)
            _lib.check(lib.dgfs_mlp_tanh_bwd(dH.numel(), _p(H), _p(dH),
                                             _p(dZ), self._s),
                       'dgfs_mlp_tanh_bwd')

        wgrad(H3, dY, 'W4', wd, nout)
        bgrad(dY, 'b4', nout)
        wgrad(X, dY, 'Ws', nin, nout)
        through(dY, nout, wb['W4'], H3)
        wgrad(H2, dZ, 'W3', wd, wd)
        bgrad(dZ, 'b3', wd)
        through(dZ, wd, wb['W3'], H2)
        wgrad(H1, dZ, 'W2', wd, wd)
        bgrad(dZ, 'b2', wd)
        through(dZ, wd, wb['W2'], H1)
        wgrad(X, dZ, 'W1', nin, wd)
        bgrad(dZ, 'b1', wd)
        return g

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, wd=0.0):
        lib = _lib.load()
        self.step += 1
        for k in self.names:
            _lib.check(lib.dgfs_mlp_adam(
                self.w[k].numel(), _p(self.w[k]), _p(self.wb.get(k)),
                _p(self.g[k]), _p(self.m1[k]), _p(self.m2[k]), lr, beta1,
                beta2, eps, self.step, wd if k.startswith('W') else 0.0,
                self._s), 'dgfs_mlp_adam')

    def start_schedule(self):
        """Point the device schedule at iteration 0 and this MLP's Adam
        step count."""
        self.counters.copy_(torch.tensor([0, self.step], dtype=torch.int32))

    def adam_scheduled(self, lr, lr_min, total, beta1=0.9, beta2=0.999,
                       eps=1e-8, wd=0.0):
        """One Adam step of every parameter (one launch) at the device
        schedule's rate: stream-ordered, no host values that change from
        step to step, so it can be replayed from a CUDA graph.  The caller
        advances ``self.step`` on the host."""
        lib = _lib.load()
        _lib.check(lib.dgfs_mlp_schedule(
            _p(self.counters), _p(self.hyper), lr, lr_min, total, beta1,
            beta2, self._s), 'dgfs_mlp_schedule')
        _lib.check(lib.dgfs_mlp_adam_dev(
            self.n, self.n_decay, _p(self.flat_w), _p(self.flat_wb),
            _p(self.flat_g), _p(self.flat_m1), _p(self.flat_m2),
            _p(self.hyper), beta1, beta2, eps, wd, self._s),
            'dgfs_mlp_adam_dev')

    def state(self):
        return {k: v.detach().cpu().numpy() for k, v in self.w.items()}

    def load(self, state):
        for k, v in state.items():
            self.w[k].copy_(torch.as_tensor(v, dtype=torch.float32))
        self.sync_bf16()


class VHSSurrogate:
    """Surrogate for a DGFSVHSGLLScatteringModel ``sm``.

    ``collide(fbank, qbank)`` is stream-ordered and allocation-free after
    the first call for a bank shape, so a stage that contains it can be
    captured in a CUDA graph."""

    def __init__(self, sm, threshold=0.05, seed=0):
        self.sm = sm
        self.backend = sm.backend
        self.vm = sm.vm
        self.device = sm.backend.device
        self.threshold = float(threshold)
        self.mlp = MLP(self.device, seed=seed)
        self.ws = _Workspace(self.device)
        z = lambda: torch.zeros(NFEAT, device=self.device)
        o = lambda: torch.ones(NFEAT, device=self.device)
        self.mu_x, self.is_x, self.mu_y, self.is_y = z(), o(), z(), o()
        cv = self.vm.cv()
        phi = np.vstack([np.ones(cv.shape[1]), cv, np.sum(cv*cv, axis=0)])
        self.ginv = torch.tensor(np.linalg.inv(phi @ phi.T).ravel(),
                                 dtype=torch.float64, device=self.device)
        self.gwinv = torch.tensor(window_gram_inverse().ravel(),
                                  dtype=torch.float64, device=self.device)
        self.loss_history = []
        self._last = None
        # the plain fallback runs on a few points: its own handle (it runs
        # on a side stream) with the single-CTA kernel, which splits few
        # points into one work item per radial node (42 Couette points:
        # 0.4 ms), else the cluster shape that spreads a point over the most
        # SMs
        self._plain_h = (sm.make_handle('single-cta') or
                         sm.make_handle('push', largest_cluster=True) or sm._h)
        self._side = None

    @property
    def _s(self):
        return self.backend.stream

    # -- features ------------------------------------------------------------
    def nu_bank(self, fbank):
        """Workspace bank for the collision frequency nu(c)."""
        key = ('nu',) + tuple(fbank.ioshape)
        b = self.ws._bufs.get(key)
        if b is None:
            b = self.ws._bufs[key] = self.backend.matrix(fbank.ioshape)
        return b

    def loss_rate(self, fbank, nubank, gate=None):
        """nu(c) at the points with gate != 0 (all when gate is None)."""
        nupts, _, neles = fbank.ioshape
        _, ldim, _ = fbank.traits
        _lib.check(_lib.load().dgfs_vhs_loss_rate(
            self.sm._h, fbank._as_parameter_, nubank._as_parameter_, nupts,
            neles, ldim, self.backend.soasz, _p(gate), self._s),
            'dgfs_vhs_loss_rate')
        return nubank

    def embed(self, fbank, qbank=None, out=None, nubank=None):
        """Features X, targets B (when qbank: coefficients of Q, or of the
        gain deviation Q + nu (f - M) when nubank is given), frame mom,
        measure eps."""
        nupts, _, neles = fbank.ioshape
        npts = nupts*neles
        _, ldim, _ = fbank.traits
        if out is None:
            X = torch.empty(npts, NFEAT, device=self.device)
            B = torch.empty(npts, NFEAT, device=self.device) if qbank \
                else None
            mom = torch.empty(npts, 5, dtype=torch.float64,
                              device=self.device)
            eps = torch.empty(npts, device=self.device)
        else:
            X, B, mom, eps = out
        _lib.check(_lib.load().dgfs_hermite_embed(
            self.backend.precision, fbank._as_parameter_,
            qbank._as_parameter_ if qbank else None,
            nubank._as_parameter_ if nubank else None, nupts, neles, ldim,
            self.vm.Nv(), self.vm.L(), self.vm.cw(), self.sm.prefactor,
            self.sm._gamma, _p(X), _p(B), _p(mom), _p(eps), self._s),
            'dgfs_hermite_embed')
        return X, B, mom, eps

    def _affine(self, X, mu, isg, inverse=False, out=None):
        Y = torch.empty_like(X) if out is None else out
        _lib.check(_lib.load().dgfs_mlp_affine(
            X.shape[0], X.shape[1], _p(X), _p(mu), _p(isg), _p(Y),
            1 if inverse else 0, self._s), 'dgfs_mlp_affine')
        return Y

    def _scale(self, X, eps, c0, c1, logcol=-1, inverse=False):
        _lib.check(_lib.load().dgfs_surrogate_scale(
            X.shape[0], X.shape[1], _p(eps), EPS0, c0, c1, logcol,
            1 if inverse else 0, _p(X), self._s), 'dgfs_surrogate_scale')
        return X

    def scale_features(self, X, eps):
        """In place: degree >= 2 coefficients divided by the deviation
        size s = max(eps, EPS0), log(s) into column LOGCOL."""
        return self._scale(X, eps, 4, NMODES, LOGCOL)

    def scale_targets(self, B, eps, inverse=False):
        """In place: targets divided (inverse: multiplied) by s."""
        return self._scale(B, eps, 0, NMODES, inverse=inverse)

    def embed_scaled(self, fbank, qbank):
        """Training pair rows (scaled features, scaled gain-deviation
        targets) and eps."""
        nu = self.loss_rate(fbank, self.nu_bank(fbank))
        X, B, mom, eps = self.embed(fbank, qbank, nubank=nu)
        return (self.scale_features(X, eps), self.scale_targets(B, eps), eps,
                mom)

    def resolved(self, mom):
        """Frames whose local Maxwellian the velocity grid resolves (the
        gate's condition)."""
        umax = mom[:, 1:4].abs().max(dim=1).values
        return (self.vm.L() - umax) >= RMIN*mom[:, 4].sqrt()

    def set_normalisation(self, X, B):
        """Per-feature standardisation from training data.  Features that
        are constant by construction (a_000 = 1, first-order modes) get a
        zero scale; targets are centred and divided by one global scale, so
        that the loss is the physical L2 error of Q in the orthonormal
        Hermite basis."""
        mu, sd = X.mean(dim=0), X.std(dim=0)
        self.mu_x = mu.contiguous()
        self.is_x = torch.where(sd > 1e-5, 1.0/sd.clamp(min=1e-30),
                                torch.zeros_like(sd)).contiguous()
        mu, sd = B.mean(dim=0), B.std(dim=0)
        ref = float(torch.sqrt(torch.mean(sd[:NMODES]**2)))
        ref = ref if ref > 0 else 1.0
        self.mu_y = mu.contiguous()
        self.is_y = torch.full_like(sd, 1.0/ref)

    # -- training ------------------------------------------------------------
    def train(self, X, B, epochs=20, batch=1024, lr=1e-3, seed=0,
              lr_min=0.05, weight_decay=0.0, graph=True):
        """Mini-batch Adam on normalised features/targets with the
        project's kernels (cosine learning-rate decay to lr*lr_min);
        returns the per-epoch mean loss.

        A training step gathers the batch, runs the forward pass, the loss,
        the backward pass and one Adam launch whose rate comes from the
        device schedule.  With ``graph`` the first step runs eagerly and is
        then captured in a CUDA graph that every later step replays; only
        the batch's row indices are copied in between."""
        Xn = self._affine(X, self.mu_x, self.is_x)
        Bn = self._affine(B, self.mu_y, self.is_y)
        n = X.shape[0]
        batch = min(batch, n)
        gen = torch.Generator(device='cpu').manual_seed(seed)
        lib = _lib.load()
        mlp, dev = self.mlp, self.device
        nb = n//batch
        total = max(epochs*nb, 1)
        idx = torch.empty(batch, dtype=torch.int64, device=dev)
        xb = torch.empty(batch, NFEAT, device=dev)
        yb = torch.empty(batch, NFEAT, device=dev)
        dY = torch.empty(batch, NFEAT, device=dev)
        rl = torch.empty(batch, dtype=torch.float64, device=dev)
        acc = torch.zeros((), dtype=torch.float64, device=dev)

        def step():
            torch.index_select(Xn, 0, idx, out=xb)
            torch.index_select(Bn, 0, idx, out=yb)
            Y = mlp.forward(xb, keep=True)
            _lib.check(lib.dgfs_mlp_mse(
                batch, NFEAT, NMODES, _p(Y), _p(yb), None, _p(dY), _p(rl),
                mlp._s), 'dgfs_mlp_mse')
            acc.add_(rl.sum())
            mlp.backward(dY)
            mlp.adam_scheduled(lr, lr_min, total, wd=weight_decay)

        mlp.start_schedule()
        cg = None
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen).to(dev)
            for b in range(nb):
                idx.copy_(perm[b*batch:(b + 1)*batch])
                if cg is not None:
                    cg.replay()
                    continue
                step()
                if graph and total > 1:
                    cg = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(cg):
                        step()
            hist.append(float(acc)/(nb*batch*NMODES))
            acc.zero_()
        del cg
        mlp.step += total
        mlp.check_tc()
        self.loss_history += hist
        return hist

    def predict(self, X, rows=None, count=None):
        """Predicted (scaled) targets for the rows of X; with a device row
        list rows[0 .. *count), only those rows (gathered, evaluated,
        scattered back; the other rows of the result are left as they
        are)."""
        npts = X.shape[0]
        Bp = self.ws.get('Bp', (npts, NFEAT))
        if rows is None:
            Xn = self._affine(X, self.mu_x, self.is_x,
                              out=self.ws.get('Xn', (npts, NFEAT)))
            Yn = self.mlp.forward(Xn)
            return self._affine(Yn, self.mu_y, self.is_y, inverse=True,
                                out=Bp)
        lib = _lib.load()
        Xn = self.ws.get('Xn', (npts, NFEAT))
        _lib.check(lib.dgfs_mlp_affine_rows(
            npts, NFEAT, _p(rows), _p(count), _p(X), _p(self.mu_x),
            _p(self.is_x), _p(Xn), 0, self._s), 'dgfs_mlp_affine_rows')
        Yn = self.mlp.forward(Xn, mcount=count)
        _lib.check(lib.dgfs_mlp_affine_rows(
            npts, NFEAT, _p(rows), _p(count), _p(Yn), _p(self.mu_y),
            _p(self.is_y), _p(Bp), 1, self._s), 'dgfs_mlp_affine_rows')
        return Bp

    # -- use -----------------------------------------------------------------
    def collide(self, fbank, qbank, threshold=None):
        """Q into qbank: surrogate where eps < threshold, plain operator
        elsewhere (device gate and point list).  Returns the gate tensor."""
        thr = self.threshold if threshold is None else threshold
        nupts, _, neles = fbank.ioshape
        npts = nupts*neles
        _, ldim, _ = fbank.traits
        lib = _lib.load()
        ws = self.ws
        out = (ws.get('X', (npts, NFEAT)), None,
               ws.get('mom', (npts, 5), torch.float64),
               ws.get('eps', (npts,)))
        X, _, mom, eps = self.embed(fbank, out=out)
        self.scale_features(X, eps)
        gate = ws.get('gate', (npts,), torch.int32)
        plain = ws.get('plain', (npts,), torch.int32)
        nplain = ws.get('nplain', (1,), torch.int32)
        net = ws.get('net', (npts,), torch.int32)
        nnet = ws.get('nnet', (1,), torch.int32)
        _lib.check(lib.dgfs_surrogate_gate(npts, _p(eps), thr, EPS0,
                                           _p(mom), self.vm.L(), RMIN,
                                           _p(gate), _p(plain), _p(nplain),
                                           _p(net), _p(nnet), self._s),
                   'dgfs_surrogate_gate')
        # the plain fallback (few points, on cluster shapes that leave SMs
        # idle) runs on a side stream beside the network path; both write
        # disjoint points of qbank.  Event fork/join keeps it capturable.
        main = torch.cuda.current_stream(self.device)
        if self._side is None:
            self._side = torch.cuda.Stream(device=self.device)
            self._fork = torch.cuda.Event()
            self._join = torch.cuda.Event()
        self._fork.record(main)
        self._side.wait_event(self._fork)
        _lib.check(lib.dgfs_vhs_apply_list(
            self._plain_h, fbank._as_parameter_, qbank._as_parameter_, nupts,
            neles, ldim, self.backend.soasz, _p(plain), _p(nplain), npts,
            self._side.cuda_stream), 'dgfs_vhs_apply_list')
        self._join.record(self._side)
        nu = self.loss_rate(fbank, self.nu_bank(fbank), gate)
        # the network runs on the gate-1 rows only
        Bp = self.scale_targets(self.predict(X, net, nnet), eps,
                                inverse=True)
        work = ws.get('rwork', (nupts*(-(-neles//32))*32*(32*5 + NMODES),),
                      torch.float64)
        _lib.check(lib.dgfs_hermite_reconstruct(
            self.backend.precision, _p(Bp), _p(mom), _p(gate), nupts, neles,
            ldim, self.vm.Nv(), self.vm.L(), self.vm.cw(),
            self.sm.prefactor, self.sm._gamma, _p(self.ginv),
            _p(self.gwinv), fbank._as_parameter_, nu._as_parameter_,
            qbank._as_parameter_, _p(net), _p(nnet), _p(work), self._s),
            'dgfs_hermite_reconstruct')
        main.wait_event(self._join)
        self._last = (gate, eps)
        return gate

    # kernels one collide() launches: embed, 2 scale, gate (+ counter
    # resets), loss rate, 2 row-list affine, 5 GEMMs, reconstruct (+
    # coefficients, 2 relaxation passes), plain list
    launches_per_collide = 17

    def residual_check(self, fbank, qbank, scratch, sample=16, seed=0):
        """Plain Q at a random sample of the last call's surrogate points
        (into ``scratch``) against the surrogate's values in ``qbank``.

        Returns r = sqrt(sum |dQ|^2 / sum (prefac rho T^{gamma/2} |f|)^2)
        over the sample (0 when no point used the surrogate): the error in
        units of a collision rate times f, so that r nu K dt bounds the
        relative change of f that K steps of size dt accumulate (nu, the
        dimensionless collision rate, is O(10) for VHS).  Near equilibrium
        |Q| itself tends to zero, which makes |dQ|/|Q| meaningless there.
        The caller compares r with its tolerance and drops the surrogate
        when it is exceeded."""
        gate, _ = self._last
        mom = self.ws.get('mom', (gate.numel(), 5), torch.float64)
        sur = torch.nonzero(gate).flatten()
        if sur.numel() == 0:
            return 0.0
        g = torch.Generator(device='cpu').manual_seed(seed)
        pick = sur[torch.randperm(sur.numel(), generator=g)[:sample]
                   .to(sur.device)].to(torch.int32).contiguous()
        nupts, _, neles = fbank.ioshape
        _, ldim, _ = fbank.traits
        _lib.check(_lib.load().dgfs_vhs_apply_list(
            self.sm._h, fbank._as_parameter_, scratch._as_parameter_, nupts,
            neles, ldim, self.backend.soasz, _p(pick), None, pick.numel(),
            self._s), 'dgfs_vhs_apply_list')
        qa, qb, fa = qbank.get(), scratch.get(), fbank.get()
        m = mom.cpu().numpy()
        num = den = 0.0
        for pt in pick.cpu().numpy():
            u, e = divmod(int(pt), neles)
            num += float(np.sum((qa[u, :, e].astype(np.float64) -
                                 qb[u, :, e])**2))
            rate = self.sm.prefactor*m[pt, 0]*m[pt, 4]**(0.5*self.sm._gamma)
            den += rate**2*float(np.sum(fa[u, :, e].astype(np.float64)**2))
        return float(np.sqrt(num/max(den, 1e-300)))

    def save(self, path):
        st = self.mlp.state()
        st.update(mu_x=self.mu_x.cpu().numpy(), is_x=self.is_x.cpu().numpy(),
                  mu_y=self.mu_y.cpu().numpy(), is_y=self.is_y.cpu().numpy(),
                  threshold=self.threshold)
        np.savez(path, **st)

    def load(self, path):
        d = np.load(path)
        self.mlp.load({k: d[k] for k in MLP.names})
        for k in ('mu_x', 'is_x', 'mu_y', 'is_y'):
            setattr(self, k, torch.tensor(d[k], device=self.device))
        self.threshold = float(d['threshold'])


# --------------------------------------------------------------------------
# Training data from the solver's own trajectories
# --------------------------------------------------------------------------
def _ball(rng):
    d = rng.standard_normal(3)
    return d/np.linalg.norm(d)*rng.uniform()**(1/3)


def random_uniform_state(vm, rng, bimodal):
    """A spatially uniform initial distribution: a Maxwellian with
    rho ~ U[0.5, 2], T ~ U[0.5, 3], u uniform in the unit ball, or (bimodal)
    the equal mixture of two such Maxwellians at +-u, renormalised to
    rho."""
    from frfs_b200.initcond import maxwellian_values
    rho, T = rng.uniform(0.5, 2.0), rng.uniform(0.5, 3.0)
    u = _ball(rng)
    if not bimodal:
        return maxwellian_values(vm, rho, T, u)
    f = 0.5*(maxwellian_values(vm, 1.0, T, u) +
             maxwellian_values(vm, 1.0, T, -u))
    return f*rho/(np.sum(f)*vm.cw())


def random_near_state(vm, rng, dmin=10**-1.5):
    """A spatially uniform Maxwellian at a log-uniform distance d in
    [dmin, 1] from the nondimensional reference state (rho = 1, T = 1,
    u = 0, the scales the velocity mesh is built on): u uniform in the ball
    of radius d, log rho and log T uniform in [-0.7 d, 0.7 d].  The
    parameters stay inside the ranges of random_uniform_state's box
    (rho in [0.5, 2], T in [0.5, 2], |u| <= 1) but the mismatch between
    gas and walls at the reference temperature covers every scale, so the
    wall fronts the solver grows range from weak to strong."""
    from frfs_b200.initcond import maxwellian_values
    d = 10**rng.uniform(np.log10(dmin), 0.0)
    u = d*_ball(rng)
    T = float(np.exp(d*rng.uniform(-0.7, 0.7)))
    rho = float(np.exp(d*rng.uniform(-0.7, 0.7)))
    return maxwellian_values(vm, rho, T, u)


def random_point_states(vm, n, rng):
    """n distributions spanning far from and near equilibrium: wall fronts
    (the gas Maxwellian on one side of a random plane, another Maxwellian on
    the other, as the particles a diffuse wall emits leave it), Maxwellians
    times 1 + a random degree
    2..4 Hermite polynomial of relative size 1e-3 .. 5e-2 (log-uniform),
    two-Maxwellian mixtures (random weights,
    velocities in the unit ball, temperatures in [0.5, 3]) and anisotropic
    Gaussians (one temperature per axis), with densities in [0.5, 2];
    shape (n, V)."""
    cv = vm.cv()
    out = np.empty((n, cv.shape[1]))
    modes = hermite_modes()
    for i in range(n):
        kind = rng.uniform()
        if kind < 0.3:
            # a wall front: the gas Maxwellian on one side of a random plane,
            # a different Maxwellian (another velocity, temperature and
            # density, as a diffuse wall emits) on the other; the plane
            # sits between half a thermal speed behind and three ahead of
            # the mean velocity
            T, u = rng.uniform(0.5, 3.0), _ball(rng)
            amp = 10**rng.uniform(-3, 0)
            n = rng.standard_normal(3)
            n /= np.linalg.norm(n)
            T2 = T*np.clip(1 + amp*rng.standard_normal(), 0.5, 2.0)
            u2 = u + amp*np.sqrt(T)*rng.standard_normal(3)
            r2 = np.clip(1 + amp*rng.standard_normal(), 0.3, 3.0)
            cut = np.sqrt(T)*rng.uniform(-0.5, 3.0)
            side = np.sum((cv - u[:, None])*n[:, None], axis=0) > cut
            m1 = np.exp(-np.sum((cv - u[:, None])**2, axis=0)/T)/(np.pi*T)**1.5
            m2 = np.exp(-np.sum((cv - u2[:, None])**2, axis=0)/T2) \
                / (np.pi*T2)**1.5
            f = np.where(side, r2*m2, m1)
        elif kind < 0.55:
            # near equilibrium: a random Maxwellian times 1 + a random
            # degree 2..4 Hermite polynomial of size 1e-3 .. 5e-2
            rho, T, u = 1.0, rng.uniform(0.5, 3.0), _ball(rng)
            ch = (cv - u[:, None])/np.sqrt(T)
            y = np.sqrt(2.0)*ch
            P = [np.ones_like(y), y]
            for k in range(1, 4):
                P.append((y*P[k] - np.sqrt(k)*P[k - 1])/np.sqrt(k + 1))
            h = np.zeros(cv.shape[1])
            for (a, b, c) in modes:
                if 2 <= a + b + c <= 4:
                    h += rng.standard_normal()*P[a][0]*P[b][1]*P[c][2]
            m = np.exp(-np.sum(ch*ch, axis=0))/(np.pi*T)**1.5
            h *= 10**rng.uniform(-3, np.log10(0.05))/np.sqrt(
                np.sum(m*h*h)/np.sum(m))
            f = m*(1 + h)
        elif kind < 0.8:
            w = rng.uniform(0.2, 0.8)
            f = 0.0
            for wk in (w, 1 - w):
                T = rng.uniform(0.5, 3.0)
                u = _ball(rng)
                f = f + wk*np.exp(-np.sum((cv - u[:, None])**2, axis=0)/T) \
                    / (np.pi*T)**1.5
        else:
            Tk = rng.uniform(0.5, 3.0)*rng.uniform(0.6, 1.4, 3)
            u = _ball(rng)
            f = np.exp(-np.sum((cv - u[:, None])**2/Tk[:, None], axis=0)) \
                / np.sqrt(np.pi**3*np.prod(Tk))
        out[i] = f*rng.uniform(0.5, 2.0)/(np.sum(f)*vm.cw())
    return out


class Harvester:
    """Collects the scaled (features, targets) of every (f, Q) pair it is
    called with (installed as ``system.collide_hook``), keeping points with
    eps_min <= eps < eps_max (below EPS0 the target is the operator's
    aliasing, which the features cannot predict) and a resolved frame."""

    def __init__(self, sur, eps_max, eps_min=EPS0):
        self.sur = sur
        self.eps_max, self.eps_min = eps_max, eps_min
        self.X, self.B = [], []
        self.seen = 0

    def __call__(self, fbank, qbank):
        X, B, eps, mom = self.sur.embed_scaled(fbank, qbank)
        keep = (eps < self.eps_max) & (eps >= self.eps_min) & \
            self.sur.resolved(mom)
        self.X.append(X[keep])
        self.B.append(B[keep])
        self.seen += eps.numel()

    def data(self):
        return torch.cat(self.X), torch.cat(self.B)


def _subsample(X, B, max_pairs, seed):
    if max_pairs is not None and X.shape[0] > max_pairs:
        g = torch.Generator(device='cpu').manual_seed(seed)
        idx = torch.randperm(X.shape[0], generator=g)[:max_pairs].to(X.device)
        X, B = X.index_select(0, idx), B.index_select(0, idx)
    return X, B


def harvest(system, stepper_cls, sur, runs, steps, seed=1, eps_max=0.2,
            bimodal_every=3, max_pairs=None, near=False):
    """Run ``runs`` trajectories of ``steps`` steps of the plain solver from
    random uniform initial states (seeds seed .. seed+runs-1; every
    ``bimodal_every``-th is a bimodal mixture; with ``near``, Maxwellians
    near the reference state, random_near_state) and collect the (f, Q(f))
    pairs of every collide (a seeded random subset of ``max_pairs`` when
    given).  Returns X, B on the device."""
    h = Harvester(sur, eps_max)
    vm = system.vm
    shape = system.bank[0].ioshape
    old_hook, old_sur = system.collide_hook, system.surrogate
    system.collide_hook, system.surrogate = h, None
    try:
        for r in range(runs):
            rng = np.random.default_rng(seed + r)
            if near:
                f = random_near_state(vm, rng)
            else:
                f = random_uniform_state(vm, rng, (r % bimodal_every) ==
                                         bimodal_every - 1)
            system.bank[0].set(np.broadcast_to(f[None, :, None], shape))
            st = stepper_cls(system, system.cfg)
            st.use_graphs = False
            st.advance(steps)
    finally:
        system.collide_hook, system.surrogate = old_hook, old_sur
    return _subsample(*h.data(), max_pairs, seed)


def harvest_relaxation(sm, sur, npts, steps, dt, seed=0, eps_max=0.2,
                       nupts=1, max_pairs=None):
    """(f, Q(f)) pairs along space-homogeneous relaxations (SSP-RK2 of
    df/dt = Q(f), plain operator) of ``npts`` random states
    (random_point_states), so that the data cover the whole path from far
    from equilibrium to equilibrium.  Training-data utility: its RK
    combinations are PyTorch element-wise operations on the banks."""
    be, vm = sm.backend, sm.vm
    rng = np.random.default_rng(seed)
    neles = -(-npts//nupts)
    f0 = random_point_states(vm, nupts*neles, rng)
    shape = (nupts, vm.vsize(), neles)
    f = be.matrix(shape, f0.reshape(nupts, neles, -1).transpose(0, 2, 1))
    f1, q = be.matrix(shape), be.matrix(shape)
    h = Harvester(sur, eps_max)
    for _ in range(steps):
        sm.fs_all(f, q)
        h(f, q)
        f1.data.copy_(f.data).add_(q.data, alpha=dt)
        sm.fs_all(f1, q)
        h(f1, q)
        f.data.mul_(0.5).add_(f1.data, alpha=0.5).add_(q.data, alpha=0.5*dt)
    return _subsample(*h.data(), max_pairs, seed)
