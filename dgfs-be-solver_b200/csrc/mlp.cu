// Training and inference kernels of the collision surrogate's MLP
// (no counterpart in the reference).
//
// Weights are stored in BF16 for the forward and input-gradient products and
// kept in FP32 as Adam's master copy; every product accumulates in FP32.
//   dgfs_mlp_gemm    C = act(op(A) op(B) + bias) [+ C], generic strides,
//                    A FP32, B FP32 or BF16; act = identity or tanh (the
//                    pre-activation can be kept for the backward pass)
//   dgfs_mlp_tanh_bwd  dZ = dH (1 - H^2)
//   dgfs_mlp_colsum  bias gradient (column sums, fixed order)
//   dgfs_mlp_mse     loss = mean over rows and the first n_used columns of
//                    w_j (Y - T)^2, and dY
//   dgfs_mlp_adam    Adam step on FP32 weights, refreshing the BF16 copy
//   dgfs_mlp_affine  y = (x - mu) * inv_sigma per column (and the inverse)
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"

namespace {

constexpr int BM = 64, BN = 64, BK = 16, NTH = 256;

__device__ __forceinline__ float ld_b(const float* p) { return *p; }
__device__ __forceinline__ float ld_b(const __nv_bfloat16* p) { return __bfloat162float(*p); }

// C[m][n] (ldc) = act(sum_k A(m,k) B(k,n) + bias[n]) (+ C if accumulate)
template <typename TB>
__global__ void __launch_bounds__(NTH) gemm_kernel(int M, int N, int K, const float* __restrict__ A, long long sam,
                                                  long long sak, const TB* __restrict__ B, long long sbk,
                                                  long long sbn, const float* __restrict__ bias,
                                                  float* __restrict__ Z, float* __restrict__ C, long long ldc,
                                                  int act, int accumulate) {
  __shared__ float As[BK][BM + 4];
  __shared__ float Bs[BK][BN + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int t = threadIdx.x; t < BK * BM; t += NTH) {
      // consecutive threads walk k when A is row-major (sak == 1), m otherwise
      const int kk = sak == 1 ? t % BK : t / BM, mm = sak == 1 ? t / BK : t % BM;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? A[m * sam + k * sak] : 0.f;
    }
    for (int t = threadIdx.x; t < BK * BN; t += NTH) {
      const int kk = sbn == 1 ? t / BN : t % BK, nn = sbn == 1 ? t % BN : t / BK;
      const int n = n0 + nn, k = k0 + kk;
      Bs[kk][nn] = (n < N && k < K) ? ld_b(B + k * sbk + n * sbn) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float z = acc[i][j] + (bias ? bias[n] : 0.f);
      if (accumulate) z += C[m * ldc + n];
      if (Z) Z[m * ldc + n] = z;
      C[m * ldc + n] = act == 1 ? tanhf(z) : z;
    }
  }
}

__global__ void tanh_bwd_kernel(long long n, const float* __restrict__ H, const float* __restrict__ dH,
                                float* __restrict__ dZ) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dZ[i] = dH[i] * (1.f - H[i] * H[i]);
}

// out[n] = sum_m X[m][n] (fixed summation order: deterministic)
__global__ void colsum_kernel(int M, int N, const float* __restrict__ X, long long ldx, float* __restrict__ out,
                              int accumulate) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double s = 0.0;
  for (int m = 0; m < M; ++m) s += X[m * ldx + n];
  out[n] = accumulate ? out[n] + (float)s : (float)s;
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

__global__ void affine_kernel(int M, int N, const float* __restrict__ X, const float* __restrict__ mu,
                              const float* __restrict__ s, float* __restrict__ Y, int inverse) {
  const long long n = (long long)M * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % N);
    Y[i] = inverse ? X[i] / s[c] + mu[c] : (X[i] - mu[c]) * s[c];
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

extern "C" int dgfs_mlp_gemm(int M, int N, int K, const float* A, long long sam, long long sak, const void* B,
                             int b_bf16, long long sbk, long long sbn, const float* bias, float* Z, float* C,
                             long long ldc, int act, int accumulate, void* stream) {
  dgfs::clear_error();
  if (M < 1 || N < 1 || K < 1 || !A || !B || !C) return dgfs::set_error(DGFS_ERR_INVALID, "bad GEMM arguments");
  if (act != 0 && act != 1) return dgfs::set_error(DGFS_ERR_INVALID, "act must be 0 or 1");
  if ((M + BM - 1) / BM > 65535) return dgfs::set_error(DGFS_ERR_UNSUPPORTED, "M=%d too large", M);
  const dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  if (b_bf16)
    gemm_kernel<__nv_bfloat16><<<grid, NTH, 0, (cudaStream_t)stream>>>(
        M, N, K, A, sam, sak, (const __nv_bfloat16*)B, sbk, sbn, bias, Z, C, ldc, act, accumulate);
  else
    gemm_kernel<float><<<grid, NTH, 0, (cudaStream_t)stream>>>(M, N, K, A, sam, sak, (const float*)B, sbk, sbn,
                                                                bias, Z, C, ldc, act, accumulate);
  return launched("gemm");
}

extern "C" int dgfs_mlp_tanh_bwd(long long n, const float* H, const float* dH, float* dZ, void* stream) {
  dgfs::clear_error();
  if (n < 1 || !H || !dH || !dZ) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  tanh_bwd_kernel<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, H, dH, dZ);
  return launched("tanh_bwd");
}

extern "C" int dgfs_mlp_colsum(int M, int N, const float* X, long long ldx, float* out, int accumulate,
                               void* stream) {
  dgfs::clear_error();
  if (M < 1 || N < 1 || !X || !out) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  colsum_kernel<<<(N + 127) / 128, 128, 0, (cudaStream_t)stream>>>(M, N, X, ldx, out, accumulate);
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

extern "C" int dgfs_mlp_affine(int M, int N, const float* X, const float* mu, const float* inv_sigma, float* Y,
                               int inverse, void* stream) {
  dgfs::clear_error();
  if (M < 1 || N < 1 || !X || !mu || !inv_sigma || !Y) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  affine_kernel<<<blocks_for((long long)M * N), 256, 0, (cudaStream_t)stream>>>(M, N, X, mu, inv_sigma, Y, inverse);
  return launched("affine");
}

extern "C" int dgfs_f32_to_bf16(long long n, const float* x, void* y, void* stream) {
  dgfs::clear_error();
  if (n < 1 || !x || !y) return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  f32_to_bf16_kernel<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, x, (__nv_bfloat16*)y);
  return launched("f32_to_bf16");
}
