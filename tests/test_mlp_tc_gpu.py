# -*- coding: utf-8 -*-
"""The tensor-core GEMMs of the surrogate's training step (GPU):
dgfs_mlp_gemm_tc (FP32 operands rounded as they are staged) against the
FP64 product of the same operands rounded to BF16 (nearest even), for every
operand layout the training step uses (activations row-major, weights as
stored and transposed, both operands of the weight gradient transposed);
dgfs_mlp_gemm_bf16 (BF16 operands loaded by TMA) for every combination of
K-major and MN-major operands. Ragged M, N and K, bias, tanh, the
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


def _run_bf16(M, N, K, A, a_mn, lda, B, b_mn, ldb, bias=None, act=0, acc=0,
              C0=None, keep_z=False, want_cb=False):
    lib = _lib.load()
    C = (C0.clone() if C0 is not None else
         torch.zeros(M, N, dtype=torch.float32, device=DEV))
    Z = torch.zeros(M, N, dtype=torch.float32, device=DEV) if keep_z else None
    Cb = torch.zeros(M, N, dtype=torch.bfloat16, device=DEV) if want_cb else None
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    _lib.check(lib.dgfs_mlp_gemm_bf16(
        M, N, K, A.data_ptr(), a_mn, lda, B.data_ptr(), b_mn, ldb,
        None if bias is None else bias.data_ptr(),
        None if Z is None else Z.data_ptr(), C.data_ptr(),
        None if Cb is None else Cb.data_ptr(), N, act, acc, err.data_ptr(),
        torch.cuda.current_stream().cuda_stream), 'dgfs_mlp_gemm_bf16')
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return C, Z, Cb


@pytest.mark.parametrize('a_mn', [0, 1])
@pytest.mark.parametrize('b_mn', [0, 1])
@pytest.mark.parametrize('M,N,K', [(300, 512, 256), (70, 192, 72),
                                   (2400, 1024, 128), (4096, 512, 512)])
def test_tma_gemm_layouts(a_mn, b_mn, M, N, K):
    """Every combination of K-major and MN-major BF16 operands, loaded by
    TMA, against the FP64 product; ragged M, N and K (zero fill outside the
    tensor maps); bias, tanh, the pre-activation and the BF16 copy."""
    g = torch.Generator(device='cpu').manual_seed(M + 3*N + 7*K + a_mn + 2*b_mn)
    # weights scaled by 1/sqrt(K) as in a layer, so that tanh is tested
    # where it is not saturated
    Am = torch.randn(M, K, generator=g).to(torch.bfloat16)
    Bm = (torch.randn(K, N, generator=g)/np.sqrt(K)).to(torch.bfloat16)
    lda = -(-(M if a_mn else K)//8)*8 + 8     # padded leading dimensions
    ldb = -(-(N if b_mn else K)//8)*8
    As = torch.zeros((K if a_mn else M), lda, dtype=torch.bfloat16)
    Bs = torch.zeros((K if b_mn else N), ldb, dtype=torch.bfloat16)
    if a_mn:
        As[:, :M] = Am.T
    else:
        As[:, :K] = Am
    if b_mn:
        Bs[:, :N] = Bm
    else:
        Bs[:, :K] = Bm.T
    b = (0.1*torch.randn(N, generator=g)).to(DEV)
    C, Z, Cb = _run_bf16(M, N, K, As.to(DEV), a_mn, lda, Bs.to(DEV), b_mn,
                         ldb, bias=b, act=1, keep_z=True, want_cb=True)
    z = Am.double().to(DEV) @ Bm.double().to(DEV) + b.double()
    _check(Z, z)
    _check(C, torch.tanh(z))
    assert torch.equal(Cb, C.to(torch.bfloat16))


def test_tma_gemm_accumulates():
    """The weight-gradient shape: both operands MN-major, K = 1024 rows
    (16 slices through the 4-slot ring), accumulated into C."""
    M, N, K = 256, 128, 1024
    g = torch.Generator(device='cpu').manual_seed(21)
    X = torch.randn(K, M, generator=g).to(torch.bfloat16).to(DEV)
    D = torch.randn(K, N, generator=g).to(torch.bfloat16).to(DEV)
    C0 = torch.randn(M, N, generator=g).to(DEV)
    C, _, _ = _run_bf16(M, N, K, X, 1, M, D, 1, N, acc=1, C0=C0)
    _check(C, C0.double() + X.double().T @ D.double())
