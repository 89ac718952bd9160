// Training and inference kernels of the collision surrogate's MLP
// (no counterpart in the reference).
//
// Weights are stored in BF16 for the forward and input-gradient products and
// kept in FP32 as Adam's master copy; every product accumulates in FP32.
//   dgfs_mlp_gemm    C = act(op(A) op(B) + bias) [+ C], generic strides,
//                    A FP32, B FP32 or BF16; act = identity or tanh (the
//                    pre-activation can be kept for the backward pass)
//   dgfs_mlp_tanh_bwd  dZ = dH (1 - H^2) (and its BF16 copy: _bf16)
//   dgfs_mlp_colsum  bias gradient (column sums, fixed order)
//   dgfs_mlp_mse     loss = mean over rows and the first n_used columns of
//                    w_j (Y - T)^2, and dY
//   dgfs_mlp_adam    Adam step on FP32 weights, refreshing the BF16 copy
//   dgfs_mlp_adam_dev  the same over a flat buffer, hyper-parameters from
//                    device memory (dgfs_mlp_schedule writes them)
//   dgfs_mlp_affine  y = (x - mu) * inv_sigma per column (and the inverse);
//                    dgfs_mlp_affine_rows gathers / scatters through a row list
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"

namespace {

constexpr int NTH = 256;

__device__ __forceinline__ float ld_b(const float* p) { return *p; }
__device__ __forceinline__ float ld_b(const __nv_bfloat16* p) { return __bfloat162float(*p); }

// C[m][n] (ldc) = act(sum_k A(m,k) B(k,n) + bias[n]) (+ C if accumulate);
// BM x BN tile per CTA, TM x TN outputs per thread (256 threads), BK-deep
// slices of K staged in shared memory (deeper slices for small tiles: fewer
// round trips to L2 per output).  With mcount, only the first *mcount rows
// exist (a count the device produced): tiles past it return at once.
template <typename TB, int BM, int BN, int TM, int TN, int BK>
__global__ void __launch_bounds__(NTH) gemm_kernel(int M, const int* __restrict__ mcount, int N, int K,
                                                  const float* __restrict__ A, long long sam, long long sak,
                                                  const TB* __restrict__ B, long long sbk, long long sbn,
                                                  const float* __restrict__ bias, float* __restrict__ Z,
                                                  float* __restrict__ C, long long ldc, int act, int accumulate) {
  static_assert((BM / TM) * (BN / TN) == NTH, "one output block per thread");
  __shared__ float As[BK][BM + 4];
  __shared__ float Bs[BK][BN + 4];
  constexpr int TX = BN / TN;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  if (mcount) M = min(M, *mcount);
  if (m0 >= M) return;  // uniform over the CTA
  float acc[TM][TN] = {};
  // slices of K go through registers: every global load of a slice is
  // issued before any of its shared-memory stores, and the next slice's
  // loads before this slice's products (one round trip to L2 per slice,
  // hidden behind the FMAs)
  constexpr int LA = BK * BM / NTH, LB = BK * BN / NTH;
  static_assert(LA * NTH == BK * BM && LB * NTH == BK * BN, "whole tiles per thread");
  float ra[LA], rb[LB];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int u = 0; u < LA; ++u) {
      // consecutive threads walk k when A is row-major (sak == 1), m otherwise
      const int t = threadIdx.x + u * NTH;
      const int kk = sak == 1 ? t % BK : t / BM, mm = sak == 1 ? t / BK : t % BM;
      const int m = m0 + mm, k = k0 + kk;
      ra[u] = (m < M && k < K) ? A[m * sam + k * sak] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < LB; ++u) {
      const int t = threadIdx.x + u * NTH;
      const int kk = sbn == 1 ? t / BN : t % BK, nn = sbn == 1 ? t % BN : t / BK;
      const int n = n0 + nn, k = k0 + kk;
      rb[u] = (n < N && k < K) ? ld_b(B + k * sbk + n * sbn) : 0.f;
    }
  };
  fetch(0);
  for (int k0 = 0; k0 < K; k0 += BK) {
#pragma unroll
    for (int u = 0; u < LA; ++u) {
      const int t = threadIdx.x + u * NTH;
      const int kk = sak == 1 ? t % BK : t / BM, mm = sak == 1 ? t / BK : t % BM;
      As[kk][mm] = ra[u];
    }
#pragma unroll
    for (int u = 0; u < LB; ++u) {
      const int t = threadIdx.x + u * NTH;
      const int kk = sbn == 1 ? t / BN : t % BK, nn = sbn == 1 ? t % BN : t / BK;
      Bs[kk][nn] = rb[u];
    }
    __syncthreads();
    if (k0 + BK < K) fetch(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float a[TM], b[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) a[i] = As[kk][ty * TM + i];
#pragma unroll
      for (int j = 0; j < TN; ++j) b[j] = Bs[kk][tx * TN + j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int m = m0 + ty * TM + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int n = n0 + tx * TN + j;
      if (n >= N) continue;
      float z = acc[i][j] + (bias ? bias[n] : 0.f);
      if (accumulate) z += C[m * ldc + n];
      if (Z) Z[m * ldc + n] = z;
      C[m * ldc + n] = act == 1 ? tanhf(z) : z;
    }
  }
}

__global__ void tanh_bwd_kernel(long long n, const float* __restrict__ H, const float* __restrict__ dH,
                                float* __restrict__ dZ, __nv_bfloat16* __restrict__ dZb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float z = dH[i] * (1.f - H[i] * H[i]);
    dZ[i] = z;
    if (dZb) dZb[i] = __float2bfloat16_rn(z);
  }
}

// out[n] = sum_m X[m][n] in a fixed order (deterministic): a CTA of 32 x 32
// threads takes 32 columns; thread (ty, tx) sums rows ty, ty + 32, ... of
// column tx in FP64, then each column's 32 partial sums are added in
// row-group order.
__global__ void __launch_bounds__(1024) colsum_kernel(int M, int N, const float* __restrict__ X, long long ldx,
                                                      float* __restrict__ out, int accumulate) {
  __shared__ double part[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int n = blockIdx.x * 32 + tx;
  double s = 0.0;
  if (n < N) {
#pragma unroll 4
    for (int m = ty; m < M; m += 32) s += X[m * ldx + n];
  }
  part[ty][tx] = s;
  __syncthreads();
  if (ty == 0 && n < N) {
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < 32; ++k) t += part[k][tx];
    out[n] = accumulate ? out[n] + (float)t : (float)t;
  }
}

// loss partials per row and dY = 2 w (Y - T) / (M n_used)
__global__ void mse_kernel(int M, int N, int nused, const float* __restrict__ Y, const float* __restrict__ Tg,
                           const float* __restrict__ w, float* __restrict__ dY, double* __restrict__ rowloss) {
  const int m = blockIdx.x;
  double s = 0.0;
  const double sc = 2.0 / ((double)M * nused);
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const long long i = (long long)m * N + n;
    float g = 0.f;
    if (n < nused) {
      const float d = Y[i] - Tg[i];
      const float wn = w ? w[n] : 1.f;
      s += (double)wn * d * d;
      g = (float)(sc * wn * d);
    }
    dY[i] = g;
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < (int)(blockDim.x + 31) / 32; ++k) t += red[k];
    rowloss[m] = t;
  }
}

__global__ void adam_kernel(long long n, float* __restrict__ w, __nv_bfloat16* __restrict__ wb,
                            const float* __restrict__ g, float* __restrict__ m1, float* __restrict__ m2, float lr,
                            float b1, float b2, float eps, float c1, float c2, float wd) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * w[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float wi = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

// One Adam step over a flat parameter buffer: the first n_decay entries
// take the L2 weight decay; the learning rate and the bias corrections come
// from device memory (hyper = {lr, 1 - beta1^t, 1 - beta2^t}), so that the
// step can be replayed from a CUDA graph.
__global__ void adam_dev_kernel(long long n, long long n_decay, float* __restrict__ w, __nv_bfloat16* __restrict__ wb,
                                const float* __restrict__ g, float* __restrict__ m1, float* __restrict__ m2,
                                const float* __restrict__ hyper, float b1, float b2, float eps, float wd) {
  const float lr = hyper[0], c1 = hyper[1], c2 = hyper[2];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i] + (i < n_decay ? wd * w[i] : 0.f);
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float wi = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

// Learning-rate schedule on the device: counters = {it, step}. Writes
// hyper = {lr (lr_min + (1 - lr_min) (1 + cos(pi it / total)) / 2),
// 1 - beta1^(step+1), 1 - beta2^(step+1)} and advances both counters.
__global__ void schedule_kernel(int* __restrict__ counters, float* __restrict__ hyper, float lr, float lr_min,
                                int total, float b1, float b2) {
  const int it = counters[0], step = counters[1] + 1;
  counters[0] = it + 1;
  counters[1] = step;
  const double frac = (double)it / (double)total;
  hyper[0] = (float)((double)lr * ((double)lr_min + (1.0 - (double)lr_min) * 0.5 * (1.0 + cospi(frac))));
  hyper[1] = 1.f - powf(b1, (float)step);
  hyper[2] = 1.f - powf(b2, (float)step);
}

__global__ void affine_kernel(int M, int N, const float* __restrict__ X, const float* __restrict__ mu,
                              const float* __restrict__ s, float* __restrict__ Y, int inverse) {
  const long long n = (long long)M * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % N);
    Y[i] = inverse ? X[i] / s[c] + mu[c] : (X[i] - mu[c]) * s[c];
  }
}

// Row-list form: forward (inverse = 0) gathers Y[r] = (X[rows[r]] - mu) s,
// inverse scatters Y[rows[r]] = X[r] / s + mu, for r < min(M, *count).
__global__ void affine_rows_kernel(int M, int N, const int* __restrict__ rows, const int* __restrict__ count,
                                   const float* __restrict__ X, const float* __restrict__ mu,
                                   const float* __restrict__ s, float* __restrict__ Y, int inverse) {
  const int m = min(M, *count);
  for (int r = blockIdx.x; r < m; r += gridDim.x) {
    const long long src = inverse ? r : rows[r], dst = inverse ? rows[r] : r;
    for (int c = threadIdx.x; c < N; c += blockDim.x)
      Y[dst * N + c] = inverse ? X[src * N + c] / s[c] + mu[c] : (X[src * N + c] - mu[c]) * s[c];
  }
}

__global__ void f32_to_bf16_kernel(long long n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

inline unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096); }

inline int launched(const char* what) {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DGFS_OK : dgfs::set_error(DGFS_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
}

}  // namespace

template <typename TB, int BM, int BN, int TM, int TN, int BK>
static void gemm_launch(int M, const int* mcount, int N, int K, const float* A, long long sam, long long sak,
                        const TB* B, long long sbk, long long sbn, const float* bias, float* Z, float* C,
                        long long ldc, int act, int accumulate, cudaStream_t s) {
  const dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  gemm_kernel<TB, BM, BN, TM, TN, BK><<<grid, NTH, 0, s>>>(M, mcount, N, K, A, sam, sak, B, sbk, sbn, bias, Z, C, ldc,
                                                       act, accumulate);
}

template <typename TB>
static void gemm_pick(int M, const int* mcount, int N, int K, const float* A, long long sam, long long sak,
                      const TB* B, long long sbk, long long sbn, const float* bias, float* Z, float* C,
                      long long ldc, int act, int accumulate, cudaStream_t s) {
  // 64 x 64 tiles when they fill the GPU; 32 x 32 for short products and
  // for row counts known only on the device (typically a few dozen rows)
  const long long tiles64 = (long long)((M + 63) / 64) * ((N + 63) / 64);
  if (!mcount && tiles64 >= 148)
    gemm_launch<TB, 64, 64, 4, 4, 16>(M, mcount, N, K, A, sam, sak, B, sbk, sbn, bias, Z, C, ldc, act, accumulate, s);
  else
    gemm_launch<TB, 32, 32, 2, 2, 64>(M, mcount, N, K, A, sam, sak, B, sbk, sbn, bias, Z, C, ldc, act, accumulate, s);
}

extern "C" int dgfs_mlp_gemm(int M, int N, int K, const float* A, long long sam, long long sak, const void* B,
                             int b_bf16, long long sbk, long long sbn, const float* bias, float* Z, float* C,
                             long long ldc, int act, int accumulate, const int* mcount, void* stream) {
  dgfs::clear_error();
  if (M < 1 || N < 1 || K < 1 || !A || !B || !C) return dgfs::set_error(DGFS_ERR_INVALID, "bad GEMM arguments");
  if (act != 0 && act != 1) return dgfs::set_error(DGFS_ERR_INVALID, "act must be 0 or 1");
  if ((M + 31) / 32 > 65535) return dgfs::set_error(DGFS_ERR_UNSUPPORTED, "M=%d too large", M);
  if (b_bf16)
    gemm_pick<__nv_bfloat16>(M, mcount, N, K, A, sam, sak, (const __nv_bfloat16*)B, sbk, sbn, bias, Z, C, ldc,
                             act, accumulate, (cudaStream_t)stream);
  else
    gemm_pick<float>(M, mcount, N, K, A, sam, sak, (const float*)B, sbk, sbn, bias, Z, C, ldc, act, accumulate,
                     (cudaStream_t)stream);
  return launched("gemm");
}

extern "C" int dgfs_mlp_tanh_bwd(long long n, const float* H, const float* dH, float* dZ, void* stream) {
  dgfs::clear_error();
  if (n < 1 || !H || !dH || !dZ) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  tanh_bwd_kernel<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, H, dH, dZ, nullptr);
  return launched("tanh_bwd");
}

extern "C" int dgfs_mlp_tanh_bwd_bf16(long long n, const float* H, const float* dH, float* dZ, void* dZb,
                                      void* stream) {
  dgfs::clear_error();
  if (n < 1 || !H || !dH || !dZ || !dZb) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  tanh_bwd_kernel<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, H, dH, dZ, (__nv_bfloat16*)dZb);
  return launched("tanh_bwd");
}

extern "C" int dgfs_mlp_colsum(int M, int N, const float* X, long long ldx, float* out, int accumulate,
                               void* stream) {
  dgfs::clear_error();
  if (M < 1 || N < 1 || !X || !out) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  colsum_kernel<<<(N + 31) / 32, 1024, 0, (cudaStream_t)stream>>>(M, N, X, ldx, out, accumulate);
  return launched("colsum");
}

extern "C" int dgfs_mlp_mse(int M, int N, int nused, const float* Y, const float* T, const float* w, float* dY,
                            double* rowloss, void* stream) {
  dgfs::clear_error();
  if (M < 1 || N < 1 || nused < 1 || nused > N || !Y || !T || !dY || !rowloss)
    return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  mse_kernel<<<M, 256, 0, (cudaStream_t)stream>>>(M, N, nused, Y, T, w, dY, rowloss);
  return launched("mse");
}

extern "C" int dgfs_mlp_adam(long long n, float* w, void* wbf16, const float* g, float* m1, float* m2, float lr,
                             float beta1, float beta2, float eps, int step, float weight_decay, void* stream) {
  dgfs::clear_error();
  if (n < 1 || !w || !g || !m1 || !m2 || step < 1) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, w, (__nv_bfloat16*)wbf16, g, m1, m2, lr, beta1,
                                                               beta2, eps, c1, c2, weight_decay);
  return launched("adam");
}

extern "C" int dgfs_mlp_schedule(int* counters, float* hyper, float lr, float lr_min, int total, float beta1,
                                 float beta2, void* stream) {
  dgfs::clear_error();
  if (!counters || !hyper || total < 1) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  schedule_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(counters, hyper, lr, lr_min, total, beta1, beta2);
  return launched("schedule");
}

extern "C" int dgfs_mlp_adam_dev(long long n, long long n_decay, float* w, void* wbf16, const float* g, float* m1,
                                 float* m2, const float* hyper, float beta1, float beta2, float eps,
                                 float weight_decay, void* stream) {
  dgfs::clear_error();
  if (n < 1 || n_decay < 0 || n_decay > n || !w || !g || !m1 || !m2 || !hyper)
    return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  adam_dev_kernel<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, n_decay, w, (__nv_bfloat16*)wbf16, g, m1, m2,
                                                                   hyper, beta1, beta2, eps, weight_decay);
  return launched("adam");
}

extern "C" int dgfs_mlp_affine(int M, int N, const float* X, const float* mu, const float* inv_sigma, float* Y,
                               int inverse, void* stream) {
  dgfs::clear_error();
  if (M < 1 || N < 1 || !X || !mu || !inv_sigma || !Y) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  affine_kernel<<<blocks_for((long long)M * N), 256, 0, (cudaStream_t)stream>>>(M, N, X, mu, inv_sigma, Y, inverse);
  return launched("affine");
}

extern "C" int dgfs_mlp_affine_rows(int M, int N, const int* rows, const int* count, const float* X,
                                    const float* mu, const float* inv_sigma, float* Y, int inverse, void* stream) {
  dgfs::clear_error();
  if (M < 1 || N < 1 || !rows || !count || !X || !mu || !inv_sigma || !Y)
    return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  affine_rows_kernel<<<M < 1024 ? M : 1024, 256, 0, (cudaStream_t)stream>>>(M, N, rows, count, X, mu, inv_sigma, Y,
                                                                           inverse);
  return launched("affine_rows");
}

extern "C" int dgfs_f32_to_bf16(long long n, const float* x, void* y, void* stream) {
  dgfs::clear_error();
  if (n < 1 || !x || !y) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  f32_to_bf16_kernel<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, x, (__nv_bfloat16*)y);
  return launched("f32_to_bf16");
}
