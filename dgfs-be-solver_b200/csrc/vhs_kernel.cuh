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
//   pencil  CTA r owns pencils (l2, l3), l2 in [r NS, ...)  F, fC [N][NJ]
// A 3D transform is a local 1D pass over pencils (along x1/l1), an
// exchange through distributed shared memory, then local 2D passes over the
// slab planes (or the reverse for forward transforms).  All state of a point
// stays in the cluster's shared memory; only f, Q and the small read-only
// tables (axis phases, radial weights) touch global memory.
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
  T prefac;
  // optional FP64 conservation projection (mass, momentum, energy)
  int project;
  const double* ginv;   // [5][5] inverse of G_kj = sum_v phi_k(c_v) phi_j(c_v)
  const double* cvec;   // [3][V] velocity grid
};

template <int N, int C> struct VhsGeom {
  static constexpr int NS = N / C;        // slab planes per CTA
  static constexpr int NJ = N * N / C;    // pencils per CTA
  static constexpr int NTASK = 2 * NJ;    // pencil/row/column tasks per pass
  static constexpr int NT = (NTASK + 31) / 32 * 32;  // threads per CTA (whole warps)
  static constexpr int RP = N + 1;        // padded row length
  static constexpr int V = N * N * N;
  static constexpr int BSZ = N * NS * RP; // exchange / plane buffer
  static constexpr int SMEM_CX = 2 * N * NJ + 3 * BSZ;
  static_assert(N % C == 0, "cluster size must divide N");
};

// Forward 2D transform of this CTA's slab planes (rows along x3, then columns
// along x2), in place.
template <typename T, int N, int C>
__device__ __forceinline__ void slab_forward_2d(cx<T>* __restrict__ sS, int tid) {
  using G = VhsGeom<N, C>;
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
template <typename T, int N, int C>
__device__ __forceinline__ void gather_pencil_forward(cg::cluster_group& cluster, cx<T>* sS, int rank,
                                                      int jl, cx<T> (&x)[N]) {
  using G = VhsGeom<N, C>;
  const int l2 = rank * G::NS + jl / N, l3 = jl % N;
#pragma unroll
  for (int r = 0; r < C; ++r) {
    const cx<T>* rs = cluster.map_shared_rank(sS, r);
#pragma unroll
    for (int k = 0; k < G::NS; ++k) x[r * G::NS + k] = rs[(k * N + l2) * G::RP + l3];
  }
  fft<T, N, -1>(x);
}

// Second half of an inverse 3D transform: row pass along l3 reading the
// pencil-layout exchange buffers of the owning CTAs, then (after the cluster
// barrier) a column pass along l2 in the local plane buffer.  On return
// sB0/sB1 hold this CTA's slab of both transformed fields,
// [x1l][x2][x3] with row stride RP.
template <typename T, int N, int C>
__device__ __forceinline__ void inverse_rows_cols(cg::cluster_group& cluster, cx<T>* sB0, cx<T>* sB1,
                                                  int rank, int tid) {
  using G = VhsGeom<N, C>;
  using CX = cx<T>;
  const bool active = tid < G::NTASK;
  const int which = active ? tid / G::NJ : 0, rem = tid % G::NJ;
  CX* sB = which ? sB1 : sB0;
  CX x[N];
  if (active) {
    const int x1l = rem / N, l2 = rem % N;
    const int owner = l2 / G::NS, l2l = l2 % G::NS;
    const CX* rB = cluster.map_shared_rank(sB, owner);
    const int x1 = rank * G::NS + x1l;
    const CX* src = rB + (x1 * G::NS + l2l) * G::RP;
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = src[k];
    fft<T, N, +1>(x);
  }
  cluster.sync();  // every remote read of the exchange buffers is complete
  if (active) {
    const int x1l = rem / N, l2 = rem % N;
    CX* dst = sB + (x1l * N + l2) * G::RP;
#pragma unroll
    for (int k = 0; k < N; ++k) dst[k] = x[k];
  }
  __syncthreads();
  if (active) {
    const int x1l = rem / N, x3 = rem % N;
    CX* col = sB + x1l * N * G::RP + x3;
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = col[k * G::RP];
    fft<T, N, +1>(x);
#pragma unroll
    for (int k = 0; k < N; ++k) col[k * G::RP] = x[k];
  }
  __syncthreads();
}

template <typename T, int N, int C>
__global__ void __launch_bounds__(VhsGeom<N, C>::NT, 1) vhs_cluster_kernel(const VhsArgs<T> a) {
  using G = VhsGeom<N, C>;
  using CX = cx<T>;
  constexpr int NS = G::NS, NJ = G::NJ, NT = G::NT, RP = G::RP, V = G::V;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  CX* sF = reinterpret_cast<CX*>(smem_raw);  // [N][NJ]  spectrum / V (pencils)
  CX* sFC = sF + N * NJ;                     // [N][NJ]  gain spectrum accumulator
  CX* sB0 = sFC + N * NJ;                    // exchange / plane buffer (g)
  CX* sB1 = sB0 + G::BSZ;                    // exchange / plane buffer (h)
  CX* sS = sB1 + G::BSZ;                     // [NS][N][RP] slab accumulator
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

  for (int pt = a.pt0 + cid; pt < a.pt0 + a.npts; pt += ncl) {
    const int upt = pt / a.neles, elem = pt % a.neles;

    // ---- F = FFT(f) / V -------------------------------------------------
    for (int i = tid; i < NS * N * N; i += NT) {
      const int x1l = i / (N * N), r2 = i % (N * N);
      const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
      const T fv = a.f[soa_ix(upt, a.ldim, elem, v, V, a.soasz)];
      sS[(x1l * N + r2 / N) * RP + r2 % N] = mk<CX>(fv, T(0));
    }
    __syncthreads();
    slab_forward_2d<T, N, C>(sS, tid);
    cluster.sync();
    if (tid < NJ) {
      CX x[N];
      gather_pencil_forward<T, N, C>(cluster, sS, rank, jl, x);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        sF[k * NJ + jl] = cscale(x[k], invV);
        sFC[k * NJ + jl] = mk<CX>(T(0), T(0));
      }
    }
    __syncthreads();

    for (int p = 0; p < a.P; ++p) {
      for (int q = 0; q < a.M; ++q) {
        // ---- pencil pass: g (which=0) and h (which=1) along l1 ----------
        if (active) {
          const CX* ph = a.phase + (size_t)(p * a.M + q) * 3 * N;
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
          CX* sB = which ? sB1 : sB0;
#pragma unroll
          for (int k = 0; k < N; ++k) sB[(k * NS + jl / N) * RP + l3] = x[k];
        }
        cluster.sync();
        inverse_rows_cols<T, N, C>(cluster, sB0, sB1, rank, tid);
        // ---- S_p (+)= g h ------------------------------------------------
        for (int i = tid; i < NS * N * N; i += NT) {
          const int idx = (i / N) * RP + i % N;
          const CX gh = cmul(sB0[idx], sB1[idx]);
          sS[idx] = q == 0 ? gh : cadd(sS[idx], gh);
        }
        __syncthreads();
      }
      // ---- fC += w1_p * FFT(S_p) ------------------------------------------
      slab_forward_2d<T, N, C>(sS, tid);
      cluster.sync();
      if (tid < NJ) {
        CX x[N];
        gather_pencil_forward<T, N, C>(cluster, sS, rank, jl, x);
        const T* w = a.w1 + (size_t)p * V + jglob;
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const T wk = w[k * N * N];
          CX acc = sFC[k * NJ + jl];
          acc.x += wk * x[k].x;
          acc.y += wk * x[k].y;
          sFC[k * NJ + jl] = acc;
        }
      }
    }

    // ---- gain = IFFT(fC) (which=0), loss = IFFT(b2 F) (which=1) -----------
    __syncthreads();
    if (active) {
      CX x[N];
      if (which) {
        const T* b = a.b2 + jglob;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = cscale(sF[k * NJ + jl], b[k * N * N]);
      } else {
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = sFC[k * NJ + jl];
      }
      fft<T, N, +1>(x);
      CX* sB = which ? sB1 : sB0;
#pragma unroll
      for (int k = 0; k < N; ++k) sB[(k * NS + jl / N) * RP + l3] = x[k];
    }
    cluster.sync();
    inverse_rows_cols<T, N, C>(cluster, sB0, sB1, rank, tid);

    // ---- Q = prefac (Re gain - f Re loss) [+ FP64 projection] --------------
    if (!a.project) {
      for (int i = tid; i < NS * N * N; i += NT) {
        const int x1l = i / (N * N), r2 = i % (N * N);
        const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
        const int idx = (i / N) * RP + i % N;
        const int64_t ai = soa_ix(upt, a.ldim, elem, v, V, a.soasz);
        a.Q[ai] = a.prefac * (sB0[idx].x - a.f[ai] * sB1[idx].x);
      }
    } else {
      // Moments m_k = cw sum_v phi_k(c_v) Q_v, phi = (1, cx, cy, cz, |c|^2),
      // reduced in FP64 over the cluster; Q -= sum_k lambda_k phi_k with
      // lambda = Ginv m (least-squares projection onto zero moments).
      double m[5] = {0, 0, 0, 0, 0};
      for (int i = tid; i < NS * N * N; i += NT) {
        const int x1l = i / (N * N), r2 = i % (N * N);
        const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
        const int idx = (i / N) * RP + i % N;
        const int64_t ai = soa_ix(upt, a.ldim, elem, v, V, a.soasz);
        const double qv = (double)(a.prefac * (sB0[idx].x - a.f[ai] * sB1[idx].x));
        sB0[idx].y = (T)qv;  // keep Q in the spare imaginary slot
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
        a.Q[soa_ix(upt, a.ldim, elem, v, V, a.soasz)] = (T)((double)sB0[idx].y - corr);
      }
      cluster.sync();  // sMom is read remotely above
    }
    __syncthreads();
  }
}

}  // namespace dgfs
