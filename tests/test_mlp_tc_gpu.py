# -*- coding: utf-8 -*-
"""The tensor-core GEMM of the surrogate's training step (GPU):
dgfs_mlp_gemm_tc against the FP64 product of the same operands rounded to
BF16 (nearest even), for every operand layout the training step uses
(activations row-major, weights as stored and transposed, both operands of
the weight gradient transposed), ragged M, N and K, bias, tanh, the
pre-activation output and accumulation into C.

Tolerance: the products of BF16 operands are exact in FP32, so the only
error is FP32 accumulation: 2e-5 of the largest output.
"""

import numpy as np
import pytest
import torch

from frfs_b200 import _lib
from frfs_b200 import surrogate  # noqa: F401  (declares the MLP entry points)

pytestmark = pytest.mark.gpu

DEV = torch.device('cuda:0')


def _rnd(t):
    return t.to(torch.bfloat16).to(torch.float64)


def _run(M, N, K, A, sam, sak, B, sbk, sbn, bias=None, act=0, acc=0,
         keep_z=False, C0=None):
    lib = _lib.load()
    C = (C0.clone() if C0 is not None else
         torch.zeros(M, N, dtype=torch.float32, device=DEV))
    Z = torch.zeros(M, N, dtype=torch.float32, device=DEV) if keep_z else None
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.dgfs_mlp_gemm_tc(
        M, N, K, A.data_ptr(), sam, sak, B.data_ptr(),
        1 if B.dtype == torch.bfloat16 else 0, sbk, sbn,
        None if bias is None else bias.data_ptr(),
        None if Z is None else Z.data_ptr(), C.data_ptr(), N, act, acc,
        err.data_ptr(), s), 'dgfs_mlp_gemm_tc')
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return C, Z


def _strided(t, M, K, sm, sk):
    """The (M, K) matrix element (m, k) = t.flatten()[m sm + k sk]."""
    return torch.as_strided(t, (M, K), (sm, sk))


def _check(C, ref, tol=2e-5):
    ref = ref.cpu().numpy()
    got = C.double().cpu().numpy()
    scale = max(np.max(np.abs(ref)), 1e-30)
    assert np.max(np.abs(got - ref))/scale < tol


@pytest.mark.parametrize('M,N,K', [(300, 512, 256), (70, 256, 512),
                                   (2400, 1024, 128)])
def test_forward_layout(M, N, K):
    """A row-major FP32 activations, B the BF16 weights W[K][N] as stored;
    bias, tanh and the pre-activation."""
    g = torch.Generator(device='cpu').manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(DEV)
    W = (torch.randn(K, N, generator=g)/np.sqrt(K)).to(DEV).to(torch.bfloat16)
    b = (0.1*torch.randn(N, generator=g)).to(DEV)
    C, Z = _run(M, N, K, A, K, 1, W, N, 1, bias=b, act=1, keep_z=True)
    z = _rnd(A) @ _rnd(W) + b.double()
    _check(Z, z)
    _check(C, torch.tanh(z))


def test_input_gradient_layout():
    """dX = dZ W^T: B is W read transposed (K contiguous, vector loads)."""
    M, N, K = 300, 256, 512                   # N = fan-in, K = fan-out
    g = torch.Generator(device='cpu').manual_seed(3)
    D = torch.randn(M, K, generator=g).to(DEV)
    W = torch.randn(N, K, generator=g).to(DEV).to(torch.bfloat16)
    C, _ = _run(M, N, K, D, K, 1, W, 1, K)
    _check(C, _rnd(D) @ _rnd(W).T)


@pytest.mark.parametrize('rows', [70, 1024])
def test_weight_gradient_layout(rows):
    """g = X^T D with both operands read transposed (FP32), accumulated
    into a C that already holds values."""
    nin, nout = 256, 512
    g = torch.Generator(device='cpu').manual_seed(rows)
    X = torch.randn(rows, nin, generator=g).to(DEV)
    D = torch.randn(rows, nout, generator=g).to(DEV)
    C0 = torch.randn(nin, nout, generator=g).to(DEV)
    C, _ = _run(nin, nout, rows, X, 1, nin, D, nout, 1, acc=1, C0=C0)
    _check(C, C0.double() + _rnd(X).T @ _rnd(D))


def test_generic_strides_and_ragged_k():
    """K not a multiple of 4 or of the slice: A takes the scalar K-pair
    path, B general strides."""
    M, N, K = 130, 96, 70
    g = torch.Generator(device='cpu').manual_seed(11)
    A = torch.randn(M, K, generator=g).to(DEV)
    Bs = torch.randn(3*K*N, generator=g).to(DEV)
    B = _strided(Bs, K, N, 3*N, 3)
    C, _ = _run(M, N, K, A, K, 1, Bs, 3*N, 3)
    _check(C, _rnd(A) @ _rnd(B.contiguous()))


def test_matches_simt_gemm_on_rounded_operands():
    """On operands already representable in BF16 the tensor-core product
    and the SIMT product agree to FP32 accumulation."""
    M, N, K = 512, 512, 512
    g = torch.Generator(device='cpu').manual_seed(5)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).float().to(DEV)
    W = torch.randn(K, N, generator=g).to(DEV).to(torch.bfloat16)
    C, _ = _run(M, N, K, A, K, 1, W, N, 1)
    C2 = torch.zeros_like(C)
    _lib.check(_lib.load().dgfs_mlp_gemm(
        M, N, K, A.data_ptr(), K, 1, W.data_ptr(), 1, N, 1, None, None,
        C2.data_ptr(), N, 0, 0, None, torch.cuda.current_stream().cuda_stream),
        'dgfs_mlp_gemm')
    torch.cuda.synchronize()
    _check(C, C2.double())
