// Fused VHS collision kernel, "push" exchange.
//
// Same algorithm and data distribution as vhs_cluster_kernel
// (vhs_kernel.cuh), but the all-to-all of every inverse transform is done by
// the producers: after its pencil pass a CTA writes each result straight into
// the plane buffer of the CTA that owns that x1 plane with st.async (remote
// shared-memory stores that complete on the receiver's mbarrier), instead of
// every consumer issuing remote loads.  Plane buffers alternate between two
// sets, and the cluster barrier that protects a set from being overwritten is
// split into arrive (after the last local read) and wait (just before the next
// pushes), so its latency hides behind the next pencil FFTs.
//
// Every mbarrier wait is bounded (1 s of %globaltimer); on expiry the kernel
// records an error flag in global memory and carries on, so all cluster
// barriers are still reached and the launch always terminates; the host
// turns the flag into an error (dgfs_vhs_status).
#pragma once

#include "mbarrier.cuh"
#include "vhs_kernel.cuh"

namespace dgfs {

// ---- PTX helpers ----------------------------------------------------------
__device__ __forceinline__ void cl_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cl_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

// Failure-detection check of the bounded wait: one CTA waits on an mbarrier
// that expects 16 bytes nothing will send, so the wait runs out after
// `limit_ns` and sets `err`, exactly as a push exchange whose data never
// arrives would.  Nothing else is touched; the launch ends after one timeout.
static __global__ void __launch_bounds__(32) wait_check_kernel(int* err, uint64_t limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int gave_up;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    gave_up = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_expect_tx(&bar, 16);
  __syncthreads();
  mbar_wait_bounded(&bar, 0, err, &gave_up, limit_ns);
}
__device__ __forceinline__ void st_async(uint32_t raddr, float2 v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];" ::"r"(raddr),
               "f"(v.x), "f"(v.y), "r"(rbar)
               : "memory");
}
__device__ __forceinline__ void st_async(uint32_t raddr, double2 v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(raddr),
               "d"(v.x), "d"(v.y), "r"(rbar)
               : "memory");
}

template <int N, int C> struct PushGeom {
  using G = VhsGeom<N, C, false>;
  static constexpr int NS = G::NS, NJ = G::NJ, NTASK = G::NTASK, NT = G::NT, RP = G::RP, V = G::V;
  static constexpr int BSZ = G::BSZ;  // one plane buffer [NS][N][RP]
  // sF [N][NJ] + planes [2 sets][2 fields][BSZ] + S [BSZ] + phases [2][3N]
  static constexpr int SMEM_CX = N * NJ + 5 * BSZ + 6 * N;
};

// Pencil results x[x1] of field `which` for pencil (l2g, l3) pushed to the
// owners of the x1 planes: element (x1, l2, l3) lands at
// planes[set][which][((x1 % NS) * N + l2) * RP + l3] of CTA x1 / NS.
template <typename T, int N, int C>
__device__ __forceinline__ void push_pencil(const cx<T> (&x)[N], const cx<T>* plane_local, uint64_t* bar_local,
                                            int l2g, int l3) {
  using P = PushGeom<N, C>;
  const uint32_t off = (uint32_t)((l2g * P::RP + l3) * sizeof(cx<T>));
#pragma unroll
  for (int r = 0; r < C; ++r) {
    const uint32_t base = cluster_addr(plane_local, r) + off;
    const uint32_t rbar = cluster_addr(bar_local, r);
#pragma unroll
    for (int k = 0; k < P::NS; ++k)
      st_async(base + (uint32_t)(k * N * P::RP * sizeof(cx<T>)), x[r * P::NS + k], rbar);
  }
}

// Row pass along l3 and column pass along l2 of both fields in a local plane
// set, in place: after it the set holds this CTA's slab [x1l][x2][x3].
template <typename T, int N, int C>
__device__ __forceinline__ void plane_rows_cols(cx<T>* set, int tid) {
  using P = PushGeom<N, C>;
  using CX = cx<T>;
  const bool active = tid < P::NTASK;
  const int which = active ? tid / P::NJ : 0, rem = tid % P::NJ;
  CX* pl = set + which * P::BSZ;
  CX x[N];
  if (active) {
    CX* row = pl + rem * P::RP;  // rem = x1l * N + l2
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = row[k];
    fft<T, N, +1>(x);
#pragma unroll
    for (int k = 0; k < N; ++k) row[k] = x[k];
  }
  __syncthreads();
  if (active) {
    const int x1l = rem / N, x3 = rem % N;
    CX* col = pl + x1l * N * P::RP + x3;
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = col[k * P::RP];
    fft<T, N, +1>(x);
#pragma unroll
    for (int k = 0; k < N; ++k) col[k * P::RP] = x[k];
  }
  __syncthreads();
}

template <typename T, int N, int C, int MINB>
__global__ void __launch_bounds__(PushGeom<N, C>::NT, MINB) vhs_push_kernel(const VhsArgs<T> a) {
  using P = PushGeom<N, C>;
  using CX = cx<T>;
  constexpr int NS = P::NS, NJ = P::NJ, NT = P::NT, RP = P::RP, V = P::V, BSZ = P::BSZ;
  constexpr uint32_t kPhaseBytes = 2u * NS * N * N * sizeof(CX);  // both fields of my slab

  extern __shared__ __align__(16) unsigned char smem_raw[];
  CX* sF = reinterpret_cast<CX*>(smem_raw);  // [N][NJ]
  CX* sPl = sF + N * NJ;                     // [2 sets][2 fields][BSZ]
  CX* sS = sPl + 4 * BSZ;                    // [NS][N][RP]
  CX* sPh = sS + BSZ;                        // [2][3N]
  __shared__ __align__(8) uint64_t sBar[2];
  __shared__ int sGaveUp;
  __shared__ double sRed[5][NT / 32];
  __shared__ double sMom[5];

  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const int cid = blockIdx.x / C, ncl = gridDim.x / C;
  const bool active = tid < P::NTASK;
  const int which = active ? tid / NJ : 0, jl = tid % NJ;
  const int l2g = rank * NS + jl / N, l3 = jl % N;
  const int jglob = l2g * N + l3;
  const T invV = T(1) / T(V);
  CX* fc = a.fc + (size_t)blockIdx.x * N * NJ;
  const int npq = a.P * a.M;
  int it = 0;

  auto load_phases = [&](int pq, int slot) {
    const CX* src = a.phase + (size_t)pq * 3 * N;
    for (int i = tid; i < 3 * N; i += NT) sPh[slot * 3 * N + i] = src[i];
  };
  // One exchange: push both fields' pencils into plane set `set` of the
  // owners, then wait until this CTA's slab of that set is complete.
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
    slab_forward_2d<T, N, C, false>(sS, tid);
    cl_wait();
    cl_arrive();
    cl_wait();  // every slab is transformed
    if (tid < NJ) {
      CX x[N];
      gather_pencil_forward<T, N, C, false>(sS, rank, jl, x);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        sF[k * NJ + jl] = cscale(x[k], invV);
        fc[k * NJ + jl] = mk<CX>(T(0), T(0));
      }
    }
    __syncthreads();
    cl_arrive();  // pending: done reading the peers' slabs

    for (int p = 0; p < a.P; ++p) {
      for (int q = 0; q < a.M; ++q, ++it) {
        const int set = it & 1;
        const CX* ph = sPh + (it & 1) * 3 * N;
        CX x[N];
        if (active) {
          CX eyz = cmul(ph[N + l2g], ph[2 * N + l3]);
          if (which) eyz.y = -eyz.y;
#pragma unroll
          for (int k = 0; k < N; ++k) {
            CX e = ph[k];
            if (which) e.y = -e.y;
            x[k] = cmul(cmul(sF[k * NJ + jl], e), eyz);
          }
          fft<T, N, +1>(x);
        }
        if (p * a.M + q + 1 < npq) load_phases(p * a.M + q + 1, (it + 1) & 1);
        exchange(x, set);
        CX* pset = sPl + set * 2 * BSZ;
        plane_rows_cols<T, N, C>(pset, tid);
        const CX* g = pset;
        const CX* h = pset + BSZ;
        for (int i = tid; i < NS * N * N; i += NT) {
          const int idx = (i / N) * RP + i % N;
          const CX gh = cmul(g[idx], h[idx]);
          sS[idx] = q == 0 ? gh : cadd(sS[idx], gh);
        }
        __syncthreads();
        cl_arrive();  // done reading this plane set
      }
      // ---- fC += w1_p * FFT(S_p) ------------------------------------------
      slab_forward_2d<T, N, C, false>(sS, tid);
      cl_wait();
      cl_arrive();
      cl_wait();  // every slab is transformed
      if (tid < NJ) {
        CX x[N];
        gather_pencil_forward<T, N, C, false>(sS, rank, jl, x);
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
      cl_arrive();  // pending: done reading the peers' slabs
    }

    // ---- gain = IFFT(fC) (which=0), loss = IFFT(b2 F) (which=1) -----------
    {
      const int set = it & 1;
      CX x[N];
      if (active) {
        if (which) {
          const T* b = a.b2 + jglob;
#pragma unroll
          for (int k = 0; k < N; ++k) x[k] = cscale(sF[k * NJ + jl], b[k * N * N]);
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
      CX* gain = pset;
      const CX* loss = pset + BSZ;

      if (!a.project) {
        for (int i = tid; i < NS * N * N; i += NT) {
          const int x1l = i / (N * N), r2 = i % (N * N);
          const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
          const int idx = (i / N) * RP + i % N;
          const int64_t ai = soa_ix(upt, a.ldim, elem, v, V, a.soasz);
          a.Q[ai] = a.prefac * (gain[idx].x - a.f[ai] * loss[idx].x);
        }
        __syncthreads();
        cl_arrive();
      } else {
        double m[5] = {0, 0, 0, 0, 0};
        for (int i = tid; i < NS * N * N; i += NT) {
          const int x1l = i / (N * N), r2 = i % (N * N);
          const int64_t v = (int64_t)(rank * NS + x1l) * (N * N) + r2;
          const int idx = (i / N) * RP + i % N;
          const int64_t ai = soa_ix(upt, a.ldim, elem, v, V, a.soasz);
          const double qv = (double)(a.prefac * (gain[idx].x - a.f[ai] * loss[idx].x));
          gain[idx].y = (T)qv;
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
        cl_arrive();
        cl_wait();  // every CTA's partial moments are in place
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
        __syncthreads();
        cl_arrive();  // pending: done reading the peers' moments and this set
      }
    }
  }
  cl_wait();  // close the pending phase before exit
}

}  // namespace dgfs
