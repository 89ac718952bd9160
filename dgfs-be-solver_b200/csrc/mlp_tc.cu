// Tensor-core GEMM of the collision surrogate's training step (no
// counterpart in the reference).
//
//   dgfs_mlp_gemm_tc   C = act(op(A) op(B) + bias) [+ C], the contract of
//                      dgfs_mlp_gemm (generic strides, A FP32, B FP32 or
//                      BF16), with both operands rounded to BF16 (nearest
//                      even) and the products accumulated in FP32 by
//                      tcgen05.mma (kind::f16) into tensor memory.
//
// One CTA of 256 threads computes a 128 x BN tile of C. K advances in slices
// of 64 (one 128-byte row of BF16): the eight warps load a slice of A
// (128 x 64) and of B (BN x 64) from global memory into registers, round it
// to BF16 and store it in shared memory in the K-major 128-byte-swizzled
// layout the tensor core reads (rows of 128 B, the 16-byte chunk c of row r
// at chunk c ^ (r & 7), 8-row groups 1024 B apart), then issue the next
// slice's loads. One thread issues the slice's four 128 x BN x 16 MMAs and
// commits them to the slot's mbarrier; a slot is refilled only after that
// mbarrier reports its MMAs complete.
// The accumulator lives in BN columns of tensor memory (lane = row of the
// tile); the epilogue reads it with tcgen05.ld, stages it in the ring's
// shared memory, adds the bias, applies tanh and writes C (and the
// pre-activation Z) row by row.
//
// Every mbarrier wait is bounded (1 s); on expiry the kernel sets *err,
// skips the epilogue, waits (bounded) for its MMAs in flight and frees its
// tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"
#include "mbarrier.cuh"
#include "tcgen05.cuh"

namespace {

using dgfs::fence_async_smem;
using dgfs::idesc_bf16;
using dgfs::mbar_init;
using dgfs::mbar_wait_bounded;
using dgfs::sdesc_sw128;
using dgfs::smem_u32;
using dgfs::tc_fence_after;
using dgfs::tc_fence_before;
using dgfs::tmem_ld16;
using dgfs::umma_commit;
using dgfs::umma_f16;

constexpr int TC_BM = 128;       // MMA M: one tensor-memory lane per row of the tile
constexpr int TC_BK = 64;        // K slice: one 128-byte swizzle row of BF16
constexpr int TC_UK = 16;        // K of one kind::f16 MMA
constexpr int TC_THREADS = 256;  // eight warps: warp w reads tensor-memory lanes 32 (w % 4) .. + 31
constexpr int TC_STAGES = 3;

// Operand staging modes (chosen on the host from the strides).
enum : int {
  kVec = 0,      // K contiguous and 16-byte aligned: vector loads along K
  kRowFast = 1,  // rows contiguous: lanes walk rows, two K values per thread
  kKFast = 2,    // anything else: lanes walk K pairs
};

// Byte offset of element (row, k) in a K-major SWIZZLE_128B tile.
__device__ __forceinline__ uint32_t sw128(int row, int k) {
  return (uint32_t)(row * 128 + ((((k >> 3) ^ (row & 7)) << 4) | ((k & 7) << 1)));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

// One K slice of an operand held in registers between its global loads and
// its shared-memory stores: rows [r0, r0 + ROWS) x K [k0, k0 + 64) of a
// strided matrix (element (r, k) at src[r sr + k sk]), zero outside
// [0, nr) x [0, K), stored into a swizzled BF16 tile. Loading the next slice
// while the tensor core works on this one hides the global-memory latency.
template <int ROWS, typename TS>
struct Slice;

template <int ROWS>
struct Slice<ROWS, float> {
  static constexpr int NF = ROWS * TC_BK / TC_THREADS;  // floats per thread (vectors or pairs)
  float v[NF];

  // kRowFast: lanes walk rows, two K values each; kKFast: lanes walk K pairs
  __device__ __forceinline__ static void pair_at(int q, int mode, int& row, int& kp) {
    row = mode == kRowFast ? q % ROWS : q >> 5;
    kp = mode == kRowFast ? q / ROWS : q & 31;
  }

  __device__ __forceinline__ void load(const float* __restrict__ src, long long sr, long long sk, int nr, int K,
                                       int r0, int k0, int mode) {
    const int tid = threadIdx.x;
    if (mode == kVec) {  // sk == 1, sr % 4 == 0, K % 4 == 0, 16-byte aligned
#pragma unroll
      for (int i = 0; i < NF / 4; ++i) {
        const int q = tid + TC_THREADS * i, row = q >> 4, k = k0 + (q & 15) * 4, r = r0 + row;
        const float4 x = (r < nr && k < K) ? __ldg(reinterpret_cast<const float4*>(src + r * sr + k))
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
        v[4 * i] = x.x, v[4 * i + 1] = x.y, v[4 * i + 2] = x.z, v[4 * i + 3] = x.w;
      }
    } else {
#pragma unroll
      for (int i = 0; i < NF / 2; ++i) {
        int row, kp;
        pair_at(tid + TC_THREADS * i, mode, row, kp);
        const int r = r0 + row, k = k0 + 2 * kp;
        const float* p = src + r * sr + k * sk;
        v[2 * i] = (r < nr && k < K) ? __ldg(p) : 0.f;
        v[2 * i + 1] = (r < nr && k + 1 < K) ? __ldg(p + sk) : 0.f;
      }
    }
  }

  __device__ __forceinline__ void store(uint8_t* tile, int mode) const {
    const int tid = threadIdx.x;
    if (mode == kVec) {
#pragma unroll
      for (int i = 0; i < NF / 4; ++i) {
        const int q = tid + TC_THREADS * i, row = q >> 4, kq = (q & 15) * 4;
        *reinterpret_cast<uint2*>(tile + sw128(row, kq)) =
            make_uint2(pack_bf16(v[4 * i], v[4 * i + 1]), pack_bf16(v[4 * i + 2], v[4 * i + 3]));
      }
    } else {
#pragma unroll
      for (int i = 0; i < NF / 2; ++i) {
        int row, kp;
        pair_at(tid + TC_THREADS * i, mode, row, kp);
        *reinterpret_cast<uint32_t*>(tile + sw128(row, 2 * kp)) = pack_bf16(v[2 * i], v[2 * i + 1]);
      }
    }
  }
};

template <int ROWS>
struct Slice<ROWS, __nv_bfloat16> {
  static constexpr int NU = ROWS * TC_BK / 2 / TC_THREADS;  // BF16 pairs per thread
  uint32_t v[NU];

  __device__ __forceinline__ static void pair_at(int q, int mode, int& row, int& kp) {
    row = mode == kRowFast ? q % ROWS : q >> 5;
    kp = mode == kRowFast ? q / ROWS : q & 31;
  }

  __device__ __forceinline__ void load(const __nv_bfloat16* __restrict__ src, long long sr, long long sk, int nr,
                                       int K, int r0, int k0, int mode) {
    const int tid = threadIdx.x;
    if (mode == kVec) {  // sk == 1, sr % 8 == 0, K % 8 == 0, 16-byte aligned: copied as is
#pragma unroll
      for (int i = 0; i < NU / 4; ++i) {
        const int q = tid + TC_THREADS * i, row = q >> 3, k = k0 + (q & 7) * 8, r = r0 + row;
        const uint4 x = (r < nr && k < K) ? __ldg(reinterpret_cast<const uint4*>(src + r * sr + k))
                                          : make_uint4(0u, 0u, 0u, 0u);
        v[4 * i] = x.x, v[4 * i + 1] = x.y, v[4 * i + 2] = x.z, v[4 * i + 3] = x.w;
      }
    } else {
      const uint16_t* s16 = reinterpret_cast<const uint16_t*>(src);
#pragma unroll
      for (int i = 0; i < NU; ++i) {
        int row, kp;
        pair_at(tid + TC_THREADS * i, mode, row, kp);
        const int r = r0 + row, k = k0 + 2 * kp;
        const uint16_t* p = s16 + r * sr + k * sk;
        const uint32_t lo = (r < nr && k < K) ? __ldg(p) : 0u;
        const uint32_t hi = (r < nr && k + 1 < K) ? __ldg(p + sk) : 0u;
        v[i] = lo | (hi << 16);
      }
    }
  }

  __device__ __forceinline__ void store(uint8_t* tile, int mode) const {
    const int tid = threadIdx.x;
    if (mode == kVec) {
#pragma unroll
      for (int i = 0; i < NU / 4; ++i) {
        const int q = tid + TC_THREADS * i, row = q >> 3, kq = (q & 7) * 8;
        *reinterpret_cast<uint4*>(tile + sw128(row, kq)) = make_uint4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < NU; ++i) {
        int row, kp;
        pair_at(tid + TC_THREADS * i, mode, row, kp);
        *reinterpret_cast<uint32_t*>(tile + sw128(row, 2 * kp)) = v[i];
      }
    }
  }
};

template <int BN>
constexpr int tc_smem_bytes() {
  return 1024 /* alignment slack */ + TC_STAGES * (TC_BM + BN) * 128 + 256 /* barriers, tmem slot, flag */;
}

// Row m of the tile is tensor-memory lane m; the MMA's B operand is op(B)
// transposed (BN rows of K), staged the same way as A.
template <typename TB, int BN>
__global__ void __launch_bounds__(TC_THREADS, 1)
    gemm_tc_kernel(int M, int N, int K, const float* __restrict__ A, long long sam, long long sak, int amode,
                   const TB* __restrict__ B, long long sbk, long long sbn, int bmode, const float* __restrict__ bias,
                   float* __restrict__ Z, float* __restrict__ C, long long ldc, int act, int accumulate,
                   int* __restrict__ err) {
  static_assert(BN % 16 == 0 && BN >= 32 && BN <= 256 && (BN & (BN - 1)) == 0, "MMA N and tensor-memory columns");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr int A_BYTES = TC_BM * 128, B_BYTES = BN * 128, STAGE_BYTES = A_BYTES + B_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TC_STAGES * STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + TC_STAGES);
  int* gave_up = reinterpret_cast<int*>(tmem_slot + 1);  // a wait ran out: stop issuing
  int* drain_up = gave_up + 1;                            // the final drain ran out

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * BN;

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < TC_STAGES; ++s) mbar_init(&bars[s], 1);
    *gave_up = 0;
    *drain_up = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) dgfs::tmem_alloc(tmem_slot, BN);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t IDESC = idesc_bf16(TC_BM, BN);

  const int nk = (K + TC_BK - 1) / TC_BK;
  int last = -1;  // last K slice whose MMAs were committed
  Slice<TC_BM, float> sa;
  Slice<BN, TB> sb;
  sa.load(A, sam, sak, M, K, m0, 0, amode);
  sb.load(B, sbn, sbk, N, K, n0, 0, bmode);
  for (int kc = 0; kc < nk; ++kc) {
    const int s = kc % TC_STAGES;
    // the slot's previous MMAs (slice kc - STAGES) must be done reading it
    if (kc >= TC_STAGES) mbar_wait_bounded(&bars[s], (uint32_t)((kc / TC_STAGES - 1) & 1), err, gave_up);
    uint8_t* ta = smem + s * STAGE_BYTES;
    uint8_t* tb = ta + A_BYTES;
    sa.store(ta, amode);
    sb.store(tb, bmode);
    if (kc + 1 < nk) {  // the next slice's loads fly during the barrier and the MMAs
      sa.load(A, sam, sak, M, K, m0, (kc + 1) * TC_BK, amode);
      sb.load(B, sbn, sbk, N, K, n0, (kc + 1) * TC_BK, bmode);
    }
    fence_async_smem();  // the generic-proxy stores become visible to the tensor core
    __syncthreads();
    if (*(volatile int*)gave_up) break;  // uniform: read after the barrier
    if (tid == 0) {
      tc_fence_after();
      const uint32_t sa = smem_u32(ta), sb = smem_u32(tb);
#pragma unroll
      for (int j = 0; j < TC_BK / TC_UK; ++j)
        umma_f16(tmem, sdesc_sw128(sa + j * TC_UK * 2), sdesc_sw128(sb + j * TC_UK * 2), IDESC,
                  (kc > 0 || j > 0) ? 1u : 0u);
      umma_commit(&bars[s]);
    }
    last = kc;
  }
  // the last commit completes when every MMA issued before it has; this
  // wait has its own flag so that it still drains after an earlier give-up
  if (last >= 0) mbar_wait_bounded(&bars[last % TC_STAGES], (uint32_t)((last / TC_STAGES) & 1), err, drain_up);
  __syncthreads();
  tc_fence_after();

  if (!*(volatile int*)gave_up && !*(volatile int*)drain_up && last == nk - 1) {
    // warp w: rows 32 (w % 4) .. + 31, the half (w / 4) of the columns.
    // The ring's shared memory is free now: each warp stages its 32 x BN/2
    // block there (row stride BN/2 + 1: no bank conflicts either way) and
    // writes whole row segments with consecutive lanes on consecutive
    // columns (coalesced).
    constexpr int HW = BN / 2, SP = HW + 1;
    static_assert(8 * 32 * SP * 4 <= TC_STAGES * STAGE_BYTES, "epilogue staging fits in the ring");
    const int quarter = warp & 3, half = warp >> 2;
    float* stg = reinterpret_cast<float*>(smem) + warp * 32 * SP;
#pragma unroll 1
    for (int j = 0; j < HW; j += 16) {
      float v[16];
      __syncwarp();  // tcgen05.ld is warp-collective
      tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(half * HW + j), v);
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) stg[lane * SP + j + jj] = v[jj];
    }
    __syncwarp();
#pragma unroll 1
    for (int r = 0; r < 32; ++r) {
      const int m = m0 + quarter * 32 + r;
      if (m >= M) break;  // uniform over the warp
      const long long row = (long long)m * ldc;
#pragma unroll
      for (int c = lane; c < HW; c += 32) {
        const int n = n0 + half * HW + c;
        if (n < N) {
          float z = stg[r * SP + c] + (bias ? __ldg(bias + n) : 0.f);
          if (accumulate) z += C[row + n];
          if (Z) Z[row + n] = z;
          C[row + n] = act == 1 ? tanhf(z) : z;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    dgfs::tmem_dealloc(tmem, BN);
  }
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Staging mode of an operand whose rows are r (stride sr) and K is k (stride sk).
inline int operand_mode(const void* p, long long sr, long long sk, int K, int vec) {
  if (sk == 1 && sr % vec == 0 && K % vec == 0 && aligned16(p)) return kVec;
  if (sr == 1) return kRowFast;
  return kKFast;
}

template <typename TB, int BN>
int gemm_tc_launch(int M, int N, int K, const float* A, long long sam, long long sak, const TB* B, long long sbk,
                   long long sbn, const float* bias, float* Z, float* C, long long ldc, int act, int accumulate,
                   int* err, cudaStream_t s) {
  constexpr int smem = tc_smem_bytes<BN>();
  static std::atomic<unsigned long long> configured{0};  // per device
  const cudaError_t e0 = dgfs::smem_limit_once(gemm_tc_kernel<TB, BN>, smem, configured);
  if (e0 != cudaSuccess)
    return dgfs::set_error(DGFS_ERR_CUDA, "tensor-core GEMM attributes: %s", cudaGetErrorString(e0));
  const int amode = operand_mode(A, sam, sak, K, 4);
  const int bmode = operand_mode(B, sbn, sbk, K, sizeof(TB) == 2 ? 8 : 4);
  const dim3 grid((N + BN - 1) / BN, (M + TC_BM - 1) / TC_BM);
  gemm_tc_kernel<TB, BN><<<grid, TC_THREADS, smem, s>>>(M, N, K, A, sam, sak, amode, B, sbk, sbn, bmode, bias, Z, C,
                                                         ldc, act, accumulate, err);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DGFS_OK : dgfs::set_error(DGFS_ERR_CUDA, "tensor-core GEMM launch: %s", cudaGetErrorString(e));
}

template <typename TB>
int gemm_tc_pick(int M, int N, int K, const float* A, long long sam, long long sak, const TB* B, long long sbk,
                 long long sbn, const float* bias, float* Z, float* C, long long ldc, int act, int accumulate,
                 int* err, cudaStream_t s) {
  // 128-column tiles when they cover the GPU, else 64 columns for more CTAs
  const long long tiles128 = (long long)((M + TC_BM - 1) / TC_BM) * ((N + 127) / 128);
  if (tiles128 >= 148)
    return gemm_tc_launch<TB, 128>(M, N, K, A, sam, sak, B, sbk, sbn, bias, Z, C, ldc, act, accumulate, err, s);
  return gemm_tc_launch<TB, 64>(M, N, K, A, sam, sak, B, sbk, sbn, bias, Z, C, ldc, act, accumulate, err, s);
}

}  // namespace

extern "C" int dgfs_mlp_gemm_tc(int M, int N, int K, const float* A, long long sam, long long sak, const void* B,
                                int b_bf16, long long sbk, long long sbn, const float* bias, float* Z, float* C,
                                long long ldc, int act, int accumulate, int* err, void* stream) {
  dgfs::clear_error();
  if (M < 1 || N < 1 || K < 1 || !A || !B || !C || !err) return dgfs::set_error(DGFS_ERR_INVALID, "bad GEMM arguments");
  if (act != 0 && act != 1) return dgfs::set_error(DGFS_ERR_INVALID, "act must be 0 or 1");
  if ((M + TC_BM - 1) / TC_BM > 65535) return dgfs::set_error(DGFS_ERR_UNSUPPORTED, "M=%d too large", M);
  const cudaStream_t s = (cudaStream_t)stream;
  if (b_bf16)
    return gemm_tc_pick<__nv_bfloat16>(M, N, K, A, sam, sak, (const __nv_bfloat16*)B, sbk, sbn, bias, Z, C, ldc, act,
                                       accumulate, err, s);
  return gemm_tc_pick<float>(M, N, K, A, sam, sak, (const float*)B, sbk, sbn, bias, Z, C, ldc, act, accumulate, err,
                             s);
}
