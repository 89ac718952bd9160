// Measurement helper: sustained FMA throughput of the SIMT pipes.
//
// The fused VHS kernel is bound by FP32 (or FP64) SIMT arithmetic, a peak
// that the driver-measured table (HBM copy, bf16 tensor GEMM) does not hold.
// This probe times a register-only FMA loop over every SM with CUDA events
// so the benchmark can report its roofline against a number measured on the
// same GPU in the same run.
#include <cuda_runtime.h>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"

namespace dgfs {

template <typename T>
__global__ void __launch_bounds__(256) fma_probe_kernel(T* out, int iters, T a, T b) {
  // 8 independent chains per thread keep the FMA pipe full
  T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
  T x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == T(-1.2345e-30)) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keep live
}

}  // namespace dgfs

extern "C" int dgfs_probe_fma_peak(int precision, int iters, double* tflops, float* ms, void* stream) {
  using namespace dgfs;
  clear_error();
  if (!tflops || (precision != 32 && precision != 64) || iters < 1 || iters > (1 << 20))
    return set_error(DGFS_ERR_INVALID, "bad probe arguments");
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = nsm * 8, threads = 256;
  void* out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * threads * 8) != cudaSuccess)
    return set_error(DGFS_ERR_NOMEM, "probe buffer allocation failed");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaStream_t s = (cudaStream_t)stream;
  // warm-up launch, then the timed one
  for (int rep = 0; rep < 2; ++rep) {
    if (rep == 1) cudaEventRecord(e0, s);
    if (precision == 32)
      fma_probe_kernel<float><<<blocks, threads, 0, s>>>((float*)out, iters, 0.999999f, 1e-7f);
    else
      fma_probe_kernel<double><<<blocks, threads, 0, s>>>((double*)out, iters, 0.999999, 1e-9);
  }
  cudaEventRecord(e1, s);
  cudaError_t err = cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return set_error(DGFS_ERR_CUDA, "probe failed: %s", cudaGetErrorString(err));
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (t * 1e-3) / 1e12;
  if (ms) *ms = t;
  return DGFS_OK;
}
