// Fused fast-spectral VHS collision operator Q(f): one thread-block cluster
// per solution point, persistent over all points of a bank.
//
// Algorithm (the reference's DGFSVHSGLLScatteringModel.fs,
// frfs/solvers/dgfs/scattering.py:227-286 with kernels
// frfs/solvers/dgfs/kernels/scattering/vhs-gll.mako:103-266):
//
//   F  = FFT(f) / V
//   for p < Nrho:  S_p = sum_q  t3_pq^2 + t4_pq^2,
//                  t3 = IFFT(cos(a_pq) F),  t4 = IFFT(sin(a_pq) F)
//   fC = sum_p (2 qw_p sw / V) b1_p FFT(S_p)
//   Q  = prefac * ( Re IFFT(fC) - f * Re IFFT(b2 F) )
//
// Two restatements keep the same discrete operator while cutting work:
//   * t3^2 + t4^2 = g h with g = IFFT(e^{+i a} F), h = IFFT(e^{-i a} F)
//     (linearity: t3 = (g+h)/2, t4 = (g-h)/2i); the phase a_pq(l) =
//     fac_p (s_q . l) factorises over the three axes, so each 1D pass
//     applies its own axis phase and no N^3 phase array exists;
//   * sum_q FFT(g h) = FFT(sum_q g h): one forward transform per radial
//     node instead of one per (p, q).
// Per point: 2*Nrho*M + Nrho + 3 3D transforms (the reference does
// 3*Nrho*M + 3).
//
// Data layout inside a cluster of C CTAs (N^3 grid, NS = N/C, NJ = N^2/C):
//   slab    CTA r owns planes x1 in [r NS, (r+1) NS)       S  [NS][N][N+1]
//   pencil  CTA r owns pencils (l2, l3), l2 in [r NS, ...)  F  [N][NJ]
// A 3D transform is a local 1D pass over pencils (along x1/l1), an
// exchange through distributed shared memory, then local 2D passes over the
// slab planes (or the reverse for forward transforms).  The gain spectrum
// fC, touched once per radial node, lives in a per-CTA global scratch slice
// (L2 resident); everything touched per (p, q) stays in shared memory.
//
// Exchange buffers: with DB (double buffering) two sets alternate between
// "exchange" (read by peers) and "plane" (local 2D passes) roles, so one
// cluster barrier per (p, q) suffices; without DB a second barrier protects
// the single set before it is overwritten.
#pragma once

#include <cooperative_groups.h>

#include "dgfs_common.cuh"
#include "fft_reg.cuh"

namespace dgfs {

namespace cg = cooperative_groups;

template <typename T> struct VhsArgs {
  const T* f;           // input bank, frfs AoSoA layout
  T* Q;                 // output bank, same layout
  int64_t ldim;         // leading dimension (elements) of one solution-point row
  int nupts, neles, soasz;
  int pt0, npts;        // linear points [pt0, pt0+npts), pt -> (pt / neles, pt % neles)
  int P, M;             // radial and half-sphere quadrature sizes
  const cx<T>* phase;   // [P][M][3][N] exp(i fac_p s_q[axis] l0[k])
  const T* w1;          // [P][V]  (2 qw_p sw / V) b1_p(l)
  const T* b2;          // [V]
  const T* w1t;         // [P][N][N*N] w1 with the last axis outermost: w1t[p][k3][k1 N + k2]
  const T* b2t;         // [N][N*N]    b2 likewise (lane-contiguous for per-line access)
  cx<T>* fc;            // scratch [gridDim.x][N][NJ]: gain spectrum per CTA
  cx<T>* fcp;           // single-CTA kernel, points split over CTAs: partial gain
                        // spectra, one [V] slice per (point, radial chunk) item
                        // (<= kCubeSlices gridDim.x)
  int* pdone;           // ... and per point the chunks finished (<= kCubeSlices / 2 gridDim.x points;
                        // zero between launches).  NULL: never split.
  int* err;             // set to 1 when a bounded wait gives up
  const int* plist;     // optional device list of linear points (NULL: pt0 + i)
  const int* pcount;    // optional device count capping npts (NULL: npts)
  T prefac;
  // optional FP64 conservation projection (mass, momentum, energy)
  int project;
  const double* ginv;   // [5][5] inverse of G_kj = sum_v phi_k(c_v) phi_j(c_v)
  const double* cvec;   // [3][V] velocity grid
};

template <int N, int C, bool DB> struct VhsGeom {
  static constexpr int NS = N / C;        // slab planes per CTA
  static constexpr int NJ = N * N / C;    // pencils per CTA
  static constexpr int NTASK = 2 * NJ;    // pencil/row/column tasks per pass
  static constexpr int NT = (NTASK + 31) / 32 * 32;  // threads per CTA (whole warps)
  static constexpr int RP = N + 1;        // padded row length
  static constexpr int V = N * N * N;
  static constexpr int BSZ = N * NS * RP; // one exchange / plane buffer
  static constexpr int NSETS = DB ? 2 : 1;
  // sF [N][NJ] + exchange sets [NSETS][2][BSZ] + S [BSZ] + phases [2][3N]
  static constexpr int SMEM_CX = N * NJ + (2 * NSETS + 1) * BSZ + 6 * N;
  static_assert(N % C == 0, "cluster size must divide N");
};

// ---- distributed shared memory access (explicit shared::cluster space) ----
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t local = (uint32_t)__cvta_generic_to_shared(p), remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
  return remote;
}
__device__ __forceinline__ float2 ld_cluster(const float2*, uint32_t a) {
  float2 v;
  asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ double2 ld_cluster(const double2*, uint32_t a) {
  double2 v;
  asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a) : "memory");
  return v;
}

// Forward 2D transform of this CTA's slab planes (rows along x3, then columns
// along x2), in place; every thread takes part (tasks are split in two halves
// so that all NT threads have work).
template <typename T, int N, int C, bool DB>
__device__ __forceinline__ void slab_forward_2d(cx<T>* __restrict__ sS, int tid) {
  using G = VhsGeom<N, C, DB>;
  using CX = cx<T>;
  if (tid < G::NJ) {
    const int x1l = tid / N, x2 = tid % N;
    CX x[N];
    CX* row = sS + (x1l * N + x2) * G::RP;
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = row[k];
    fft<T, N, -1>(x);
#pragma unroll
    for (int k = 0; k < N; ++k) row[k] = x[k];
  }
  __syncthreads();
  if (tid < G::NJ) {
    const int x1l = tid / N, x3 = tid % N;
    CX x[N];
    CX* col = sS + x1l * N * G::RP + x3;
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = col[k * G::RP];
    fft<T, N, -1>(x);
#pragma unroll
    for (int k = 0; k < N; ++k) col[k * G::RP] = x[k];
  }
  __syncthreads();
}

// Gather pencil (l2, l3) along x1 from the slab planes of every CTA of the
// cluster and transform it forward.
template <typename T, int N, int C, bool DB>
__device__ __forceinline__ void gather_pencil_forward(const cx<T>* sS, int rank, int jl, cx<T> (&x)[N]) {
  using G = VhsGeom<N, C, DB>;
  const int l2 = rank * G::NS + jl / N, l3 = jl % N;
  const cx<T>* base = sS + l2 * G::RP + l3;
#pragma unroll
  for (int r = 0; r < C; ++r) {
    const uint32_t a = cluster_addr(base, r);
#pragma unroll
    for (int k = 0; k < G::NS; ++k) x[r * G::NS + k] = ld_cluster(base, a + k * N * G::RP * sizeof(cx<T>));
  }
  fft<T, N, -1>(x);
}

// Inverse transform, second half: row pass along l3 reading the peers'
// exchange buffers (pencil layout), written to the local plane buffers, then
// the column pass along l2 in place.  On return the plane buffers hold this
// CTA's slab of both fields, [x1l][x2][x3] with row stride RP.
template <typename T, int N, int C, bool DB>
__device__ __forceinline__ void inverse_rows_cols(cg::cluster_group& cluster, const cx<T>* xg,
                                                  const cx<T>* xh, cx<T>* pg, cx<T>* ph, int rank,
                                                  int tid) {
  using G = VhsGeom<N, C, DB>;
  using CX = cx<T>;
  const bool active = tid < G::NTASK;
  const int which = active ? tid / G::NJ : 0, rem = tid % G::NJ;
  CX* pl = which ? ph : pg;
  CX x[N];
  if (active) {
    const int x1l = rem / N, l2 = rem % N;
    const int owner = l2 / G::NS, l2l = l2 % G::NS;
    const int x1 = rank * G::NS + x1l;
    const CX* src = (which ? xh : xg) + (x1 * G::NS + l2l) * G::RP;
    const uint32_t a = cluster_addr(src, owner);
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = ld_cluster(src, a + k * sizeof(CX));
    fft<T, N, +1>(x);
  }
  if constexpr (!DB) cluster.sync();  // peers have finished reading xg/xh == pg/ph
  if (active) {
    const int x1l = rem / N, l2 = rem % N;
    CX* dst = pl + (x1l * N + l2) * G::RP;
#pragma unroll
    for (int k = 0; k < N; ++k) dst[k] = x[k];
  }
  __syncthreads();
  if (active) {
    const int x1l = rem / N, x3 = rem % N;
    CX* col = pl + x1l * N * G::RP + x3;
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = col[k * G::RP];
    fft<T, N, +1>(x);
#pragma unroll
    for (int k = 0; k < N; ++k) col[k * G::RP] = x[k];
  }
  __syncthreads();
}

template <typename T, int N, int C, bool DB, int MINB>
__global__ void __launch_bounds__(VhsGeom<N, C, DB>::NT, MINB) vhs_cluster_kernel(const VhsArgs<T> a) {
  using G = VhsGeom<N, C, DB>;
  using CX = cx<T>;
  constexpr int NS = G::NS, NJ = G::NJ, NT = G::NT, RP = G::RP, V = G::V, BSZ = G::BSZ;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  CX* sF = reinterpret_cast<CX*>(smem_raw);      // [N][NJ]  spectrum / V (pencils)
  CX* sX = sF + N * NJ;                          // exchange sets [NSETS][2][BSZ]
  CX* sS = sX + 2 * G::NSETS * BSZ;              // [NS][N][RP] slab accumulator
  CX* sPh = sS + BSZ;                            // [2][3N] axis phases of (p, q)
  __shared__ double sRed[5][NT / 32];
  __shared__ double sMom[5];

  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const int cid = blockIdx.x / C, ncl = gridDim.x / C;
  const bool active = tid < G::NTASK;
  const int which = active ? tid / NJ : 0, jl = tid % NJ;
  const int l2g = rank * NS + jl / N, l3 = jl % N;  // pencil owned by task jl
  const int jglob = l2g * N + l3;
  const T invV = T(1) / T(V);
  CX* fc = a.fc + (size_t)blockIdx.x * N * NJ;  // this CTA's gain spectrum [N][NJ]
  const int npq = a.P * a.M;
  int it = 0;  // running (p, q) counter: selects buffer sets and phase slots

  auto xbuf = [&](int set, int w) -> CX* { return sX + (DB ? (set * 2 + w) : w) * BSZ; };
  auto load_phases = [&](int pq, int slot) {
    const CX* src = a.phase + (size_t)pq * 3 * N;
    for (int i = tid; i < 3 * N; i += NT) sPh[slot * 3 * N + i] = src[i];
  };

  const int npts = a.pcount ? min(a.npts, *a.pcount) : a.npts;
  for (int ip = cid; ip < npts; ip += ncl) {
    const int pt = a.plist ? a.plist[a.pt0 + ip] : a.pt0 + ip;
    // listed ids come from device memory: skip one outside the bank (every
    // CTA of the cluster reads the same entry, so all skip together and the
    // cluster barriers stay paired)
    if ((unsigned)pt >= (unsigned)(a.nupts * a.neles)) continue;
    const int upt = pt / a.neles, elem = pt % a.neles;

    // ---- F = FFT(f) / V -------------------------------------------------
    for (int i = tid; i < NS * N * N; i += NT) {
      const int x1l = i / (N * N), r2 = i % (N * N);
      const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
      const T fv = a.f[soa_ix(upt, a.ldim, elem, v, V, a.soasz)];
      sS[(x1l * N + r2 / N) * RP + r2 % N] = mk<CX>(fv, T(0));
    }
    load_phases(0, it & 1);
    __syncthreads();
    slab_forward_2d<T, N, C, DB>(sS, tid);
    cluster.sync();
    if (tid < NJ) {
      CX x[N];
      gather_pencil_forward<T, N, C, DB>(sS, rank, jl, x);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        sF[k * NJ + jl] = cscale(x[k], invV);
        fc[k * NJ + jl] = mk<CX>(T(0), T(0));
      }
    }
    __syncthreads();

    for (int p = 0; p < a.P; ++p) {
      for (int q = 0; q < a.M; ++q, ++it) {
        const int cur = DB ? (it & 1) : 0, pl = DB ? (cur ^ 1) : 0;
        const CX* ph = sPh + (it & 1) * 3 * N;
        // ---- pencil pass: g (which=0) and h (which=1) along l1 ----------
        if (active) {
          CX eyz = cmul(ph[N + l2g], ph[2 * N + l3]);
          if (which) eyz.y = -eyz.y;
          CX x[N];
#pragma unroll
          for (int k = 0; k < N; ++k) {
            CX e = ph[k];
            if (which) e.y = -e.y;
            x[k] = cmul(cmul(sF[k * NJ + jl], e), eyz);
          }
          fft<T, N, +1>(x);
          CX* sB = xbuf(cur, which);
#pragma unroll
          for (int k = 0; k < N; ++k) sB[(k * NS + jl / N) * RP + l3] = x[k];
        }
        // prefetch the next (p, q)'s axis phases into the other slot
        if (p * a.M + q + 1 < npq) load_phases(p * a.M + q + 1, (it + 1) & 1);
        cluster.sync();
        inverse_rows_cols<T, N, C, DB>(cluster, xbuf(cur, 0), xbuf(cur, 1), xbuf(pl, 0), xbuf(pl, 1),
                                       rank, tid);
        // ---- S_p (+)= g h ------------------------------------------------
        {
          const CX* g = xbuf(pl, 0);
          const CX* h = xbuf(pl, 1);
          for (int i = tid; i < NS * N * N; i += NT) {
            const int idx = (i / N) * RP + i % N;
            const CX gh = cmul(g[idx], h[idx]);
            sS[idx] = q == 0 ? gh : cadd(sS[idx], gh);
          }
        }
        __syncthreads();
      }
      // ---- fC += w1_p * FFT(S_p) ------------------------------------------
      slab_forward_2d<T, N, C, DB>(sS, tid);
      cluster.sync();
      if (tid < NJ) {
        CX x[N];
        gather_pencil_forward<T, N, C, DB>(sS, rank, jl, x);
        const T* w = a.w1 + (size_t)p * V + jglob;
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const T wk = w[k * N * N];
          CX acc = fc[k * NJ + jl];
          acc.x += wk * x[k].x;
          acc.y += wk * x[k].y;
          fc[k * NJ + jl] = acc;
        }
      }
    }

    // ---- gain = IFFT(fC) (which=0), loss = IFFT(b2 F) (which=1) -----------
    const int cur = DB ? (it & 1) : 0, pl = DB ? (cur ^ 1) : 0;
    if (active) {
      CX x[N];
      if (which) {
        const T* b = a.b2 + jglob;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = cscale(sF[k * NJ + jl], b[k * N * N]);
      } else {
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = fc[k * NJ + jl];
      }
      fft<T, N, +1>(x);
      CX* sB = xbuf(cur, which);
#pragma unroll
      for (int k = 0; k < N; ++k) sB[(k * NS + jl / N) * RP + l3] = x[k];
    }
    ++it;
    cluster.sync();
    inverse_rows_cols<T, N, C, DB>(cluster, xbuf(cur, 0), xbuf(cur, 1), xbuf(pl, 0), xbuf(pl, 1), rank,
                                   tid);
    CX* gain = xbuf(pl, 0);
    const CX* loss = xbuf(pl, 1);

    // ---- Q = prefac (Re gain - f Re loss) [+ FP64 projection] --------------
    if (!a.project) {
      for (int i = tid; i < NS * N * N; i += NT) {
        const int x1l = i / (N * N), r2 = i % (N * N);
        const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
        const int idx = (i / N) * RP + i % N;
        const int64_t ai = soa_ix(upt, a.ldim, elem, v, V, a.soasz);
        a.Q[ai] = a.prefac * (gain[idx].x - a.f[ai] * loss[idx].x);
      }
    } else {
      // Moments m_k = sum_v phi_k(c_v) Q_v, phi = (1, cx, cy, cz, |c|^2),
      // reduced in FP64 over the cluster; Q -= sum_k lambda_k phi_k with
      // lambda = Ginv m (least-squares projection onto zero moments).
      double m[5] = {0, 0, 0, 0, 0};
      for (int i = tid; i < NS * N * N; i += NT) {
        const int x1l = i / (N * N), r2 = i % (N * N);
        const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
        const int idx = (i / N) * RP + i % N;
        const int64_t ai = soa_ix(upt, a.ldim, elem, v, V, a.soasz);
        const double qv = (double)(a.prefac * (gain[idx].x - a.f[ai] * loss[idx].x));
        gain[idx].y = (T)qv;  // keep Q in the spare imaginary slot
        const double c0 = a.cvec[v], c1 = a.cvec[V + v], c2 = a.cvec[2 * V + v];
        m[0] += qv;
        m[1] += qv * c0;
        m[2] += qv * c1;
        m[3] += qv * c2;
        m[4] += qv * (c0 * c0 + c1 * c1 + c2 * c2);
      }
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        double s = m[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((tid & 31) == 0) sRed[k][tid >> 5] = s;
      }
      __syncthreads();
      if (tid < 5) {
        double s = 0;
        for (int w = 0; w < NT / 32; ++w) s += sRed[tid][w];
        sMom[tid] = s;
      }
      cluster.sync();
      double lam[5];
      {
        double mt[5] = {0, 0, 0, 0, 0};
        for (int r = 0; r < C; ++r) {
          const double* rm = cluster.map_shared_rank(sMom, r);
#pragma unroll
          for (int k = 0; k < 5; ++k) mt[k] += rm[k];
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          double s = 0;
#pragma unroll
          for (int j = 0; j < 5; ++j) s += a.ginv[k * 5 + j] * mt[j];
          lam[k] = s;
        }
      }
      for (int i = tid; i < NS * N * N; i += NT) {
        const int x1l = i / (N * N), r2 = i % (N * N);
        const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
        const int idx = (i / N) * RP + i % N;
        const double c0 = a.cvec[v], c1 = a.cvec[V + v], c2 = a.cvec[2 * V + v];
        const double corr = lam[0] + lam[1] * c0 + lam[2] * c1 + lam[3] * c2 +
                            lam[4] * (c0 * c0 + c1 * c1 + c2 * c2);
        a.Q[soa_ix(upt, a.ldim, elem, v, V, a.soasz)] = (T)((double)gain[idx].y - corr);
      }
      cluster.sync();  // sMom is read remotely above
    }
    __syncthreads();
  }
}

}  // namespace dgfs
