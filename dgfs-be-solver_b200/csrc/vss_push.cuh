// Fused binary-mixture VSS collision kernel (push exchange).
//
// One collision pair (p, q) of frfs's DGFSBi VSS operator
// (frfs/solvers/dgfsbi/scattering.py:227-315 with the kernels of
// dgfsbi/kernels/scattering/vss-gll.mako):
//
//   F = FFT(f_p) / V,  G = FFT(f_q) / V
//   for every radial node x and direction y (full sphere):
//     g = IFFT(e^{+i kq a_xy} F),  h = IFFT(e^{-i kp a_xy} G)
//     QGhat += w_x b_xy FFT(g h)        (kp = m_p/(m_p+m_q), kq = m_q/(m_p+m_q))
//   Q_pq = prefac (Re IFFT(QGhat) - f_p Re IFFT(c G))
//
// with a_xy(l) = (pi / L) qz_x (s_y . l).  The phase factorises over the
// three axes, so each pencil pass applies per-axis phase tables (no N^3
// phase array), as in the VHS kernels.  Unlike VHS, the gain kernel b
// depends on the direction, so FFT(g h) is taken for every (x, y): three
// full transforms per (x, y), the reference's count.  b_xy (with the weight
// w_x = qw_x sw / V folded in) is a table [x][y][V] read once per (x, y)
// and point (L2 resident).
//
// Data layout, exchange and bounded waits as vhs_push.cuh: the cluster's C
// CTAs own slabs (planes x1) and pencils (l2, l3); an inverse transform is a
// pencil pass, a push of every pencil into the owners' plane buffers
// (st.async, mbarrier completion, waits bounded by %globaltimer with the
// error flag of dgfs_vss_status), then row and column passes on the planes.
// A forward transform is the 2D slab pass, a cluster barrier and a gather
// of the pencils.
#pragma once

#include "vhs_push.cuh"

namespace dgfs {

template <typename T> struct VssArgs {
  const T* fp;         // bank of species p (AoSoA)
  const T* fq;         // bank of species q (may equal fp)
  T* Q;                // output bank; accumulate != 0 adds to it
  int64_t ldim;
  int nupts, neles, soasz;
  int pt0, npts;
  int P, M;
  const cx<T>* phase;  // [P][M][2][3][N]: field 0 e^{+i kq fac s[ax] l0}, field 1 e^{-i kp fac s[ax] l0}
  const cx<T>* b;      // [P][M][V] w_x b_xy
  const cx<T>* c;      // [V] loss kernel
  cx<T>* fc;           // scratch [gridDim.x][N][NJ]: gain spectrum per CTA
  int* err;
  T prefac;
  int accumulate;
};

template <int N, int C> struct VssGeom {
  using G = VhsGeom<N, C, false>;
  static constexpr int NS = G::NS, NJ = G::NJ, NTASK = G::NTASK, NT = G::NT, RP = G::RP, V = G::V;
  static constexpr int BSZ = G::BSZ;
  // sF, sG [N][NJ] + planes [2 sets][2 fields][BSZ] + S [BSZ] + phases [2 slots][2 fields][3N]
  static constexpr int SMEM_CX = 2 * N * NJ + 5 * BSZ + 12 * N;
};

// FFT(f) / V of one bank into the pencil layout dst [N][NJ] (slab pass,
// cluster barrier, pencil gather).  Entered with one pending cluster arrive
// (the peers' last reads of this CTA's slab buffer) and left with one (this
// gather's reads of the peers' slabs), like every step of the kernel.
template <typename T, int N, int C>
__device__ __forceinline__ void vss_forward_input(const VssArgs<T>& a, const T* f, int upt, int elem, int rank,
                                                  int tid, cx<T>* sS, cx<T>* dst) {
  using P = PushGeom<N, C>;
  using CX = cx<T>;
  constexpr int NS = P::NS, NJ = P::NJ, RP = P::RP, V = P::V;
  const T invV = T(1) / T(V);
  cl_wait();  // no peer reads sS any more
  for (int i = tid; i < NS * N * N; i += P::NT) {
    const int x1l = i / (N * N), r2 = i % (N * N);
    const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
    sS[(x1l * N + r2 / N) * RP + r2 % N] = mk<CX>(f[soa_ix(upt, a.ldim, elem, v, V, a.soasz)], T(0));
  }
  __syncthreads();
  slab_forward_2d<T, N, C, false>(sS, tid);
  cl_arrive();
  cl_wait();  // every slab is transformed
  if (tid < NJ) {
    const int jl = tid;
    CX x[N];
    gather_pencil_forward<T, N, C, false>(sS, rank, jl, x);
#pragma unroll
    for (int k = 0; k < N; ++k) dst[k * NJ + jl] = cscale(x[k], invV);
  }
  __syncthreads();
  cl_arrive();  // pending: done reading the peers' slabs
}

template <typename T, int N, int C, int MINB>
__global__ void __launch_bounds__(PushGeom<N, C>::NT, MINB) vss_push_kernel(const VssArgs<T> a) {
  using P = PushGeom<N, C>;
  using CX = cx<T>;
  constexpr int NS = P::NS, NJ = P::NJ, NT = P::NT, RP = P::RP, V = P::V, BSZ = P::BSZ;
  constexpr uint32_t kPhaseBytes = 2u * NS * N * N * sizeof(CX);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  CX* sF = reinterpret_cast<CX*>(smem_raw);  // [N][NJ]
  CX* sG = sF + N * NJ;                      // [N][NJ]
  CX* sPl = sG + N * NJ;                     // [2 sets][2 fields][BSZ]
  CX* sS = sPl + 4 * BSZ;                    // [NS][N][RP]
  CX* sPh = sS + BSZ;                        // [2 slots][2 fields][3N]
  __shared__ __align__(8) uint64_t sBar[2];
  __shared__ int sGaveUp;

  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const int cid = blockIdx.x / C, ncl = gridDim.x / C;
  const bool active = tid < P::NTASK;
  const int which = active ? tid / NJ : 0, jl = tid % NJ;
  const int l2g = rank * NS + jl / N, l3 = jl % N;
  const int jglob = l2g * N + l3;
  CX* fc = a.fc + (size_t)blockIdx.x * N * NJ;
  const int npq = a.P * a.M;
  int it = 0;

  auto load_phases = [&](int pq, int slot) {
    const CX* src = a.phase + (size_t)pq * 6 * N;
    for (int i = tid; i < 6 * N; i += NT) sPh[slot * 6 * N + i] = src[i];
  };
  auto exchange = [&](const CX (&x)[N], int set) {
    cl_wait();  // every CTA is done reading this set from two exchanges ago
    if (active) push_pencil<T, N, C>(x, sPl + (set * 2 + which) * BSZ, &sBar[set], l2g, l3);
    if (tid == 0) mbar_expect_tx(&sBar[set], kPhaseBytes);
    mbar_wait_bounded(&sBar[set], (uint32_t)((it >> 1) & 1), a.err, &sGaveUp);
  };

  if (tid == 0) {
    sGaveUp = 0;
    mbar_init(&sBar[0], 1);
    mbar_init(&sBar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  cl_arrive();
  cl_wait();
  cl_arrive();  // pending: nothing to protect yet

  for (int ip = cid; ip < a.npts; ip += ncl) {
    const int pt = a.pt0 + ip;
    const int upt = pt / a.neles, elem = pt % a.neles;

    // ---- F = FFT(f_p) / V, G = FFT(f_q) / V ------------------------------
    vss_forward_input<T, N, C>(a, a.fp, upt, elem, rank, tid, sS, sF);
    vss_forward_input<T, N, C>(a, a.fq, upt, elem, rank, tid, sS, sG);
    if (tid < NJ) {
#pragma unroll
      for (int k = 0; k < N; ++k) fc[k * NJ + jl] = mk<CX>(T(0), T(0));
    }
    load_phases(0, it & 1);
    __syncthreads();

    for (int pq = 0; pq < npq; ++pq, ++it) {
      const int set = it & 1;
      const CX* ph = sPh + (it & 1) * 6 * N + which * 3 * N;
      // ---- g = IFFT(e0 F), h = IFFT(e1 G) -----------------------------------
      CX x[N];
      if (active) {
        const CX* src = which ? sG : sF;
        const CX eyz = cmul(ph[N + l2g], ph[2 * N + l3]);
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = cmul(cmul(src[k * NJ + jl], ph[k]), eyz);
        fft<T, N, +1>(x);
      }
      if (pq + 1 < npq) load_phases(pq + 1, (it + 1) & 1);
      exchange(x, set);
      CX* pset = sPl + set * 2 * BSZ;
      plane_rows_cols<T, N, C>(pset, tid);
      // ---- S = g h, then FFT(S) and QGhat += w b FFT(S) ----------------------
      for (int i = tid; i < NS * N * N; i += NT) {
        const int idx = (i / N) * RP + i % N;
        sS[idx] = cmul(pset[idx], pset[BSZ + idx]);
      }
      __syncthreads();
      cl_arrive();  // done reading this plane set
      slab_forward_2d<T, N, C, false>(sS, tid);
      cl_wait();
      cl_arrive();
      cl_wait();  // every slab is transformed
      if (tid < NJ) {
        CX y[N];
        gather_pencil_forward<T, N, C, false>(sS, rank, jl, y);
        const CX* bb = a.b + (size_t)pq * V + jglob;
#pragma unroll
        for (int k = 0; k < N; ++k) fc[k * NJ + jl] = cfma(bb[k * N * N], y[k], fc[k * NJ + jl]);
      }
      __syncthreads();
      cl_arrive();  // pending: done reading the peers' slabs
    }

    // ---- QG = IFFT(QGhat) (field 0), fL = IFFT(c G) (field 1) -------------
    {
      const int set = it & 1;
      CX x[N];
      if (active) {
        if (which) {
          const CX* cc = a.c + jglob;
#pragma unroll
          for (int k = 0; k < N; ++k) x[k] = cmul(cc[k * N * N], sG[k * NJ + jl]);
        } else {
#pragma unroll
          for (int k = 0; k < N; ++k) x[k] = fc[k * NJ + jl];
        }
        fft<T, N, +1>(x);
      }
      exchange(x, set);
      ++it;
      CX* pset = sPl + set * 2 * BSZ;
      plane_rows_cols<T, N, C>(pset, tid);
      const CX* gain = pset;
      const CX* loss = pset + BSZ;
      for (int i = tid; i < NS * N * N; i += NT) {
        const int x1l = i / (N * N), r2 = i % (N * N);
        const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
        const int idx = (i / N) * RP + i % N;
        const int64_t ai = soa_ix(upt, a.ldim, elem, v, V, a.soasz);
        const T qv = a.prefac * (gain[idx].x - a.fp[ai] * loss[idx].x);
        a.Q[ai] = a.accumulate ? a.Q[ai] + qv : qv;
      }
      __syncthreads();
      cl_arrive();  // done reading this plane set
    }
  }
  cl_wait();  // close the pending phase before exit
}

}  // namespace dgfs
