// Tensor-core form of the FR-DG residual (FP32 banks).
//
// The residual of dg_residual_kernel (dg_kernel.cuh) at one (velocity,
// element) is one product with the element operator,
//   R = Mop Phi,  Mop = [M3 | M1 - M3 M2]  (U x K, K = F + D U),
//   Phi = [|S^T n| F^ at the F flux points | F~_(i,k) at the solution points]
// (frfs/solvers/dgfs/elements.py:49-118: the 'tdivtconf' and 'tdivtpcorf'
// products).  Batched over the (velocity, element) pairs of a CTA it is a
// GEMM with M = 128 rows, N = U (padded to 16) and K padded to whole
// 128-byte rows of FP32, which this kernel runs on the tensor cores
// (tcgen05.mma kind::tf32, accumulator in tensor memory):
//
//   * each of the 128 threads computes its row Phi (the common fluxes and
//     transformed fluxes, exactly as the SIMT kernel does) and stores it in
//     shared memory, K-major with the 128-byte swizzle, split into
//     Phi = Phi_hi + Phi_lo with both parts representable in TF32;
//   * Mop is split the same way once per CTA, so three TF32 products
//     Phi_hi Mop_hi + Phi_hi Mop_lo + Phi_lo Mop_hi carry the product to
//     about 2^-21 relative (the dropped Phi_lo Mop_lo term is 2^-22): the
//     FP32 residual's accuracy, not TF32's 2^-11;
//   * one thread issues the MMAs and commits them to an mbarrier; every
//     thread then reads its own row of R back from tensor memory (warp w
//     owns lanes 32w..32w+31 = its rows) and finishes as the SIMT kernel:
//     out = a A + b B + g (-(1/|J|) R + C).
//
// A CTA of 128 threads takes one 32-element block (lane = element) and a
// chunk of 4 VPT velocities (warp w takes v = chunk + 4 it + w).  Every wait
// is bounded (1 s); on expiry the kernel sets *a.err and stops issuing.
#pragma once

#include "dg_kernel.cuh"
#include "tcgen05.cuh"

namespace dgfs {

template <int U, int F, int D> struct DgTc {
  static constexpr int K = F + D * U;             // columns of the element operator
  static constexpr int KP = (K + 31) / 32 * 32;   // padded to whole 128-byte rows of FP32
  static constexpr int NA = KP / 32;              // 128-byte K atoms
  static constexpr int N = 16;                    // MMA N: U outputs padded
  static constexpr int ROWS = 128;                // MMA M: one (velocity, element) per thread
  static constexpr int A_ATOM = ROWS * 128;       // bytes of one K atom of an A tile
  static constexpr int B_ATOM = N * 128;
  static constexpr int OFF_AHI = 0, OFF_ALO = NA * A_ATOM;
  static constexpr int OFF_BHI = 2 * NA * A_ATOM, OFF_BLO = OFF_BHI + NA * B_ATOM;
  static constexpr int TILES = OFF_BLO + NA * B_ATOM;
  static constexpr int SMEM = TILES + 1024;       // dynamic shared memory, with the 1024-byte alignment slack
  static constexpr int TMEM_COLS = 32;            // N = 16 FP32 columns, allocation granule 32
  static_assert(U <= N, "outputs of one row");
};

// Byte offset of FP32 element (row, k), k < 32, in a K-major SWIZZLE_128B
// atom (rows of 128 B, 16-byte chunk c of row r at chunk c ^ (r & 7)).
__device__ __forceinline__ uint32_t sw128f(int row, int k) {
  return (uint32_t)(row * 128 + ((((k >> 2) ^ (row & 7)) << 4) | ((k & 3) << 2)));
}

template <int U, int F, int D, int VPT, int MB>
__global__ void __launch_bounds__(128, MB)
    dg_residual_tc_kernel(const DgArgs<float> a, const __grid_constant__ DgOps<float, U, F, D> op) {
  using G = DgGeo<float, U, F, D>;
  using TC = DgTc<U, F, D>;
  __shared__ __align__(16) float sg[32 * G::GS];
  __shared__ __align__(16) int64_t sp[32 * G::PS];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  __shared__ int gave_up, drain_up;
  extern __shared__ uint8_t dyn_raw[];
  uint8_t* tiles = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(dyn_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;

  {
    const float* gs = a.geoblk + (size_t)blockIdx.x * 32 * G::GS;
    for (int i = tid; i < 32 * G::GS; i += 128) sg[i] = gs[i];
    const int64_t* ps = a.pblk + (size_t)blockIdx.x * 32 * G::PS;
    for (int i = tid; i < 32 * G::PS; i += 128) sp[i] = ps[i];
  }
  // Mop split into TF32 parts, rows r >= U and columns k >= K zero (every
  // iteration writes the whole padded row of the A tiles)
  for (int idx = tid; idx < TC::N * TC::KP; idx += 128) {
    const int r = idx / TC::KP, k = idx % TC::KP;
    float m = 0.f;
    if (r < U && k < TC::K) m = k < F ? op.m3[r][k] : op.m132[r][k - F];
    const float hi = tf32_round(m), lo = tf32_round(m - hi);
    const uint32_t off = (uint32_t)(k >> 5) * TC::B_ATOM + sw128f(r, k & 31);
    *reinterpret_cast<float*>(tiles + TC::OFF_BHI + off) = hi;
    *reinterpret_cast<float*>(tiles + TC::OFF_BLO + off) = lo;
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    gave_up = 0;
    drain_up = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (w == 0) tmem_alloc(&tslot, TC::TMEM_COLS);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tslot;
  const uint32_t sbase = smem_u32(tiles);
  constexpr uint32_t IDESC = idesc_tf32(TC::ROWS, TC::N);

  const int64_t e = (int64_t)blockIdx.x * 32 + lane;
  const bool e_ok = e < a.neles;
  const float* gl = sg + lane * G::GS;
  const int64_t* pl = sp + lane * G::PS;
  const int vend = a.v0 + a.nv;
  const int vchunk = a.v0 + (int)blockIdx.y * (4 * VPT);
  int issued = 0;  // commits issued (each completes one phase of bar)

  // the bank values of one iteration: loaded one iteration ahead, so their
  // latency hides behind the previous iteration's MMAs and epilogue
  struct In {
    int v;
    bool act;
    int64_t o;
    float u[U], Kc[U], urv[F];
  };
  auto load_bank = [&](In& in, int v) {
    in.v = v;
    in.act = e_ok && v < vend;
    const int vv = in.act ? v : a.v0;  // a valid velocity for the idle rows
    in.o = ((int64_t)blockIdx.x * a.V + vv) * 32 + (e_ok ? lane : 0);
    const float* up = a.u + in.o;
#pragma unroll
    for (int i = 0; i < U; ++i, up += a.ldim_u) in.u[i] = in.act ? __ldg(up) : 0.f;
#pragma unroll
    for (int r = 0; r < U; ++r) {
      const int64_t ro = in.o + (int64_t)r * a.ldim_u;
      float k = (in.act && a.Cq) ? a.gamma * __ldg(a.Cq + ro) : 0.f;
      if (in.act && a.A) k = fmaf(a.alpha, __ldg(a.A + ro), k);
      if (in.act && a.B) k = fmaf(a.beta, __ldg(a.B + ro), k);
      in.Kc[r] = k;
    }
  };
  auto load_faces = [&](In& in) {  // after pdl_wait: the interp kernel's face values
#pragma unroll
    for (int f = 0; f < F; f += 2) {
      const longlong2 pb = reinterpret_cast<const longlong2*>(pl)[f / 2];
      in.urv[f] = (in.act && pb.x >= 0) ? a.uf[pb.x + (int64_t)in.v * 32] : 0.f;
      if (f + 1 < F) in.urv[f + 1] = (in.act && pb.y >= 0) ? a.uf[pb.y + (int64_t)in.v * 32] : 0.f;
    }
  };

  In cur;
  load_bank(cur, vchunk + w);
  pdl_wait();
  load_faces(cur);
#pragma unroll 1
  for (int it = 0; it < VPT; ++it) {
    if (vchunk + 4 * it >= vend) break;  // uniform over the CTA
    const int v = cur.v;
    float phi[TC::KP];
#pragma unroll
    for (int k = 0; k < TC::KP; ++k) phi[k] = 0.f;
    if (cur.act) {
      const float c[3] = {__ldg(a.cvx + v), __ldg(a.cvy + v), __ldg(a.cvz + v)};
      // common normal fluxes |S^T n| F^ at the flux points
      float nm[G::NN];
#pragma unroll
      for (int f = 0; f < F; ++f) {
        if ((f * D) % G::VW == 0) lds16<float, 1>(gl + G::ON + f * D, nm + f * D);
        float ul = 0.f;
#pragma unroll
        for (int i = 0; i < U; ++i) ul = fmaf(op.m0[f][i], cur.u[i], ul);
        const float* nmv = nm + f * D;
        float nc = nmv[0] * c[0];
#pragma unroll
        for (int d = 1; d < D; ++d) nc = fmaf(nmv[d], c[d], nc);
        float ur = cur.urv[f];
        const int64_t pb = pl[f];
        if (pb < 0) {
          const int b = (int)(-pb - 1);
          ur = b >= a.nb ? a.halo[(int64_t)(b - a.nb) * a.V + v] : dg_ghost<float, D>(a, b, v, e, f, c, nmv, nc, ul);
        }
        phi[f] = 0.5f * nc * (ul + ur) + 0.5f * fabsf(nc) * (ul - ur);  // rusanov.mako:46-50
      }
      // transformed flux at the solution points F~_(i,k) = (sum_kk S_ik,kk c_kk) u_k
      float sm[G::NS];
#pragma unroll
      for (int k = 0; k < U; ++k)
#pragma unroll
        for (int i = 0; i < D; ++i) {
          if (((k * D + i) * D) % G::VW == 0) lds16<float, 1>(gl + G::OS + (k * D + i) * D, sm + (k * D + i) * D);
          float s = 0.f;
#pragma unroll
          for (int kk = 0; kk < D; ++kk) s = fmaf(sm[(k * D + i) * D + kk], c[kk], s);
          phi[F + i * U + k] = s * cur.u[k];
        }
    }
    // this thread's row of Phi_hi and Phi_lo, 16 bytes at a time
#pragma unroll
    for (int g = 0; g < TC::KP / 4; ++g) {
      float4 hi, lo;
      hi.x = tf32_round(phi[4 * g]), lo.x = tf32_round(phi[4 * g] - hi.x);
      hi.y = tf32_round(phi[4 * g + 1]), lo.y = tf32_round(phi[4 * g + 1] - hi.y);
      hi.z = tf32_round(phi[4 * g + 2]), lo.z = tf32_round(phi[4 * g + 2] - hi.z);
      hi.w = tf32_round(phi[4 * g + 3]), lo.w = tf32_round(phi[4 * g + 3] - hi.w);
      const uint32_t off = (uint32_t)(g >> 3) * TC::A_ATOM + sw128f(tid, 4 * (g & 7));
      *reinterpret_cast<float4*>(tiles + TC::OFF_AHI + off) = hi;
      *reinterpret_cast<float4*>(tiles + TC::OFF_ALO + off) = lo;
    }
    fence_async_smem();  // the generic-proxy stores become visible to the tensor core
    tc_fence_before();   // this thread's tensor-memory reads of the last iteration come first
    __syncthreads();
    if (*(volatile int*)&gave_up) break;  // uniform: read after the barrier
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int j = 0; j < TC::KP / 8; ++j) {
        const uint32_t ko = (uint32_t)(j >> 2) * TC::A_ATOM + (uint32_t)(j & 3) * 32;
        const uint32_t kb = (uint32_t)(j >> 2) * TC::B_ATOM + (uint32_t)(j & 3) * 32;
        const uint64_t ahi = sdesc_sw128(sbase + TC::OFF_AHI + ko), alo = sdesc_sw128(sbase + TC::OFF_ALO + ko);
        const uint64_t bhi = sdesc_sw128(sbase + TC::OFF_BHI + kb), blo = sdesc_sw128(sbase + TC::OFF_BLO + kb);
        umma_tf32(tmem, ahi, bhi, IDESC, j > 0 ? 1u : 0u);
        umma_tf32(tmem, ahi, blo, IDESC, 1u);
        umma_tf32(tmem, alo, bhi, IDESC, 1u);
      }
      umma_commit(&bar);
    }
    // the next iteration's loads fly while the tensor core works
    const bool more = it + 1 < VPT && vchunk + 4 * (it + 1) < vend;
    In nxt;
    if (more) {
      load_bank(nxt, v + 4);
      load_faces(nxt);
    }
    mbar_wait_bounded(&bar, (uint32_t)(issued & 1), a.err, &gave_up);
    ++issued;
    tc_fence_after();
    float R[16];
    __syncwarp();  // tcgen05.ld is warp-collective
    tmem_ld16(tmem + ((uint32_t)(w * 32) << 16), R);
    if (cur.act && !*(volatile int*)&gave_up) {
      float rj[G::NR];
      lds16<float, G::NR / G::VW>(gl + G::OR, rj);
      float* op_ = a.out + cur.o;
#pragma unroll
      for (int r = 0; r < U; ++r, op_ += a.ldim_u) *op_ = fmaf(a.gamma, -rj[r] * R[r], cur.Kc[r]);
    }
    if (more) cur = nxt;
  }
  // a wait that gave up may leave MMAs in flight: drain them (bounded, with
  // its own flag) before the tensor memory is freed
  if (*(volatile int*)&gave_up && issued > 0) mbar_wait_bounded(&bar, (uint32_t)((issued - 1) & 1), a.err, &drain_up);
  tc_fence_before();
  __syncthreads();
  if (w == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, TC::TMEM_COLS);
  }
}

}  // namespace dgfs
