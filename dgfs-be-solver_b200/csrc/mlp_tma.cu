// BF16 tensor-core GEMM fed by TMA, for the collision surrogate's training
// step (no counterpart in the reference).
//
//   dgfs_mlp_gemm_bf16  C = act(op(A) op(B) + bias) [+ C], A and B BF16 in
//                       global memory, each either K-major (row-major with
//                       K contiguous) or MN-major (row-major with M or N
//                       contiguous, i.e. the transposed matrix as stored);
//                       FP32 accumulation; C FP32 and optionally a BF16
//                       copy Cb for the next product.
//
// One CTA of 128 threads computes a 128 x BN tile. Warp 0 lane 0 issues the
// TMA loads (cp.async.bulk.tensor, 128-byte swizzle, no multicast) of a
// K slice of 64 into a ring of STAGES shared-memory slots, each completing on
// the slot's `full` mbarrier; warp 1 lane 0 waits on it, issues the slice's
// four 128 x BN x 16 tcgen05.mma (kind::f16) and commits them to the slot's
// `empty` mbarrier, which the producer waits on before refilling the slot.
// The accumulator lives in BN tensor-memory columns; after the last commit
// (`done`) the four warps read it back (warp w: rows 32w..32w+31), stage it
// in the ring's shared memory and write the epilogue row by row. Every wait is bounded (1 s); on expiry the kernel sets *err,
// stops issuing, drains what it issued (bounded) and frees its tensor
// memory.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"
#include "mbarrier.cuh"
#include "tcgen05.cuh"

namespace {

using namespace dgfs;

constexpr int TB_BM = 128;  // MMA M
constexpr int TB_BK = 64;   // K slice: one 128-byte swizzle row of BF16
constexpr int TB_UK = 16;   // K of one kind::f16 MMA
constexpr int TB_THREADS = 128;
constexpr int TB_STAGES = 4;

template <int BN>
struct TmaGeom {
  static constexpr int A_BYTES = TB_BM * TB_BK * 2;  // 16 KB
  static constexpr int B_BYTES = BN * TB_BK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int SMEM = 1024 + TB_STAGES * STAGE + 256;
  // the epilogue's staging (4 warps x 32 rows x BN + 1 floats) reuses the ring
  static_assert(4 * 32 * (BN + 1) * 4 <= TB_STAGES * STAGE, "epilogue staging fits in the ring");
};

// Issue the TMA loads of K slice kc into a slot. A K-major operand of R
// rows is one box of 64 (K) x R rows at (k0, r0); an MN-major one is R / 64
// boxes of 64 (M or N) x 64 (K rows) at (r0 + 64 g, k0), 8 KB apart.
template <int R>
__device__ __forceinline__ void tma_operand(uint32_t dst, const CUtensorMap* tm, bool mn, int r0, int k0,
                                            uint64_t* bar) {
  if (!mn) {
    tma_load_2d(dst, tm, k0, r0, bar);
  } else {
#pragma unroll
    for (int g = 0; g < R / 64; ++g) tma_load_2d(dst + g * 8192, tm, r0 + 64 * g, k0, bar);
  }
}

// Descriptor of the MMA's K step j (16 elements) inside a slot's operand.
__device__ __forceinline__ uint64_t op_desc(uint32_t base, bool mn, int j) {
  return mn ? sdesc_sw128_mn(base + (uint32_t)j * 2048, 8192) : sdesc_sw128(base + (uint32_t)j * 32);
}

template <int BN>
__global__ void __launch_bounds__(TB_THREADS, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M, int N,
                     int K, int a_mn, int b_mn, const float* __restrict__ bias, float* __restrict__ Z,
                     float* __restrict__ C, __nv_bfloat16* __restrict__ Cb, long long ldc, int act, int accumulate,
                     int* __restrict__ err) {
  using Gm = TmaGeom<BN>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + TB_STAGES * Gm::STAGE);
  uint64_t* empty = full + TB_STAGES;
  uint64_t* done = empty + TB_STAGES;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  int* gave_up = reinterpret_cast<int*>(tslot + 1);  // a wait ran out: stop issuing
  int* drain_up = gave_up + 1;                       // a drain wait ran out
  int* counts = drain_up + 1;                        // [0] slices loaded, [1] slices consumed

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * TB_BM, n0 = blockIdx.x * BN;
  const int nk = (K + TB_BK - 1) / TB_BK;
  const bool amn = a_mn != 0, bmn = b_mn != 0;

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < TB_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *gave_up = 0;
    *drain_up = 0;
    counts[0] = counts[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(tslot, BN);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t sbase = smem_u32(smem);

  if (warp == 0 && lane == 0) {
    // producer: slot s is refilled once the MMAs of slice kc - STAGES are done
    int kc = 0;
    for (; kc < nk; ++kc) {
      const int s = kc % TB_STAGES;
      if (kc >= TB_STAGES) mbar_wait_bounded(&empty[s], (uint32_t)((kc / TB_STAGES - 1) & 1), err, gave_up);
      if (*(volatile int*)gave_up) break;
      mbar_expect_tx(&full[s], (uint32_t)Gm::STAGE);
      const uint32_t sa = sbase + s * Gm::STAGE, sb = sa + Gm::A_BYTES;
      tma_operand<TB_BM>(sa, &tmA, amn, m0, kc * TB_BK, &full[s]);
      tma_operand<BN>(sb, &tmB, bmn, n0, kc * TB_BK, &full[s]);
    }
    counts[0] = kc;
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t idesc = idesc_bf16_major(TB_BM, BN, amn, bmn);
    int kc = 0;
    for (; kc < nk; ++kc) {
      const int s = kc % TB_STAGES;
      mbar_wait_bounded(&full[s], (uint32_t)((kc / TB_STAGES) & 1), err, gave_up);
      if (*(volatile int*)gave_up) break;
      tc_fence_after();
      const uint32_t sa = sbase + s * Gm::STAGE, sb = sa + Gm::A_BYTES;
#pragma unroll
      for (int j = 0; j < TB_BK / TB_UK; ++j)
        umma_f16(tmem, op_desc(sa, amn, j), op_desc(sb, bmn, j), idesc, (kc > 0 || j > 0) ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    counts[1] = kc;
    umma_commit(done);  // completes when every MMA issued above has
  }
  // everyone: the accumulator is complete (or the launch gave up)
  mbar_wait_bounded(done, 0u, err, drain_up);
  __syncthreads();
  tc_fence_after();
  // after a give-up, loads issued but never consumed may still be landing:
  // wait for them (bounded) before the shared memory is released
  if (tid == 0 && *(volatile int*)gave_up) {
    for (int kc = counts[1]; kc < counts[0]; ++kc)
      mbar_wait_bounded(&full[kc % TB_STAGES], (uint32_t)((kc / TB_STAGES) & 1), err, drain_up);
  }
  if (!*(volatile int*)gave_up && !*(volatile int*)drain_up) {
    // The ring's shared memory is free now (every MMA and every load has
    // completed): each warp stages its 32 rows x BN accumulator columns
    // there (row stride BN + 1, so both the row-wise writes and the
    // column-wise reads are free of bank conflicts), then writes whole rows
    // with consecutive lanes on consecutive columns (coalesced).
    float* stg = reinterpret_cast<float*>(smem) + warp * 32 * (BN + 1);
#pragma unroll 1
    for (int j0 = 0; j0 < BN; j0 += 16) {
      float v[16];
      __syncwarp();  // tcgen05.ld is warp-collective
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)j0, v);
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) stg[lane * (BN + 1) + j0 + jj] = v[jj];
    }
    __syncwarp();
#pragma unroll 1
    for (int r = 0; r < 32; ++r) {
      const int m = m0 + warp * 32 + r;
      if (m >= M) break;  // uniform over the warp
      const long long row = (long long)m * ldc;
#pragma unroll
      for (int c = lane; c < BN; c += 32) {
        const int n = n0 + c;
        if (n < N) {
          float z = stg[r * (BN + 1) + c] + (bias ? __ldg(bias + n) : 0.f);
          if (accumulate) z += C[row + n];
          if (Z) Z[row + n] = z;
          const float cv = act == 1 ? tanhf(z) : z;
          C[row + n] = cv;
          if (Cb) Cb[row + n] = __float2bfloat16_rn(cv);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, BN);
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links no driver library).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor map of a row-major BF16 matrix of `rows` rows of `cols` elements
// (leading dimension ld elements), box 64 elements x box_rows rows, 128-byte
// swizzle, zero fill outside the matrix.
int make_map(CUtensorMap* tm, const void* base, long long rows, long long cols, long long ld, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return set_error(DGFS_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
  const cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(DGFS_ERR_INVALID, "tensor map rejected (CUresult %d)", (int)r);
  return DGFS_OK;
}

template <int BN>
int launch_bf16(const CUtensorMap& ta, const CUtensorMap& tb, int M, int N, int K, int a_mn, int b_mn,
                const float* bias, float* Z, float* C, void* Cb, long long ldc, int act, int accumulate, int* err,
                cudaStream_t s) {
  constexpr int smem = TmaGeom<BN>::SMEM;
  static std::atomic<unsigned long long> configured{0};  // per device
  const cudaError_t attr = smem_limit_once(gemm_bf16_kernel<BN>, smem, configured);
  if (attr != cudaSuccess) return set_error(DGFS_ERR_CUDA, "BF16 GEMM attributes: %s", cudaGetErrorString(attr));
  const dim3 grid((N + BN - 1) / BN, (M + TB_BM - 1) / TB_BM);
  gemm_bf16_kernel<BN><<<grid, TB_THREADS, smem, s>>>(ta, tb, M, N, K, a_mn, b_mn, bias, Z, C,
                                                      (__nv_bfloat16*)Cb, ldc, act, accumulate, err);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DGFS_OK : set_error(DGFS_ERR_CUDA, "BF16 GEMM launch: %s", cudaGetErrorString(e));
}

}  // namespace

extern "C" int dgfs_mlp_gemm_bf16(int M, int N, int K, const void* A, int a_mn, long long lda, const void* B,
                                  int b_mn, long long ldb, const float* bias, float* Z, float* C, void* Cb,
                                  long long ldc, int act, int accumulate, int* err, void* stream) {
  clear_error();
  if (M < 1 || N < 1 || K < 1 || !A || !B || !C || !err) return set_error(DGFS_ERR_INVALID, "bad GEMM arguments");
  if (act != 0 && act != 1) return set_error(DGFS_ERR_INVALID, "act must be 0 or 1");
  if (((uintptr_t)A & 15) || ((uintptr_t)B & 15))
    return set_error(DGFS_ERR_INVALID, "A and B must be 16-byte aligned for the tensor maps");
  if (lda % 8 || ldb % 8) return set_error(DGFS_ERR_INVALID, "lda=%lld ldb=%lld must be multiples of 8", lda, ldb);
  if (lda < (a_mn ? M : K) || ldb < (b_mn ? N : K) || ldc < N)
    return set_error(DGFS_ERR_INVALID, "leading dimension smaller than a row");
  if ((M + TB_BM - 1) / TB_BM > 65535) return set_error(DGFS_ERR_UNSUPPORTED, "M=%d too large", M);
  const long long tiles128 = (long long)((M + TB_BM - 1) / TB_BM) * ((N + 127) / 128);
  const int bn = tiles128 >= 148 ? 128 : 64;
  CUtensorMap ta, tb;
  int rc = a_mn ? make_map(&ta, A, K, M, lda, 64) : make_map(&ta, A, M, K, lda, TB_BM);
  if (!rc) rc = b_mn ? make_map(&tb, B, K, N, ldb, 64) : make_map(&tb, B, N, K, ldb, bn);
  if (rc) return rc;
  const cudaStream_t s = (cudaStream_t)stream;
  if (bn == 128)
    return launch_bf16<128>(ta, tb, M, N, K, a_mn, b_mn, bias, Z, C, Cb, ldc, act, accumulate, err, s);
  return launch_bf16<64>(ta, tb, M, N, K, a_mn, b_mn, bias, Z, C, Cb, ldc, act, accumulate, err, s);
}
