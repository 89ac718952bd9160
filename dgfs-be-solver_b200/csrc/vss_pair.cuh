// Two-CTA binary-mixture VSS kernel (FP32, N = 24).
//
// The operator of vss_push.cuh (one collision pair (p, q) of frfs's DGFSBi
// VSS model, frfs/solvers/dgfsbi/scattering.py:227-315 with the kernels of
// dgfsbi/kernels/scattering/vss-gll.mako), with the point's data in the
// shared memory of a two-CTA cluster instead of an 8-CTA exchange:
//
//   F = FFT(f_p) / V, G = FFT(f_q) / V (half spectra k3 <= N/2 in the
//   pair's L2 scratch; k3 > N/2 from the conjugate mirror, f being real)
//   for every radial node x and direction y:
//     g = IFFT(e^{+i kq a} F), h = IFFT(e^{-i kp a} G)
//     QGhat += b_xy FFT(g h)
//   Q_pq = prefac (Re IFFT(QGhat) - f_p Re IFFT(c G))
//
// Data distribution (rank r of the pair): CTA r owns the k1 values K_r of
// the two-CTA VHS kernel (vhs_pair.cuh) and the x2 half X_r = [MH r,
// MH r + MH).  An inverse transform runs along k3 on the lines (k1 in K_r,
// k2), along k2 on the lines (k1 in K_r, x3), hands the other CTA the half
// of every line it owns in x2 (a staging buffer in the L2 scratch, one
// cluster barrier), and runs along k1 on the lines (x2 in X_r, x3).  The
// forward transform of g h runs the other way: along x1, the hand-over of
// the k1 the other CTA owns, along x2, along x3; the gain spectrum QGhat
// of the CTA's k-slab accumulates in shared memory.
//
// 576 threads: 288 take the g field's lines and 288 the h field's (one line
// each per pass); the forward transform of g h uses the first 288.
// Shared memory (complex float): Wg, Wh [MH][N][N+1], QGhat [N][MH][N]
// (k3, k1l, k2), two phase slots [2 fields][3][N]: 174 KB.
#pragma once

#include "vhs_pair.cuh"
#include "vss_push.cuh"

namespace dgfs {

template <int N_> struct VssPairGeom {
  static constexpr int N = N_, H = N / 2 + 1, NY = N / 2, NN = N * N, V = N * N * N;
  static constexpr int MH = N / 2, LP = N + 1;
  static constexpr int NL = MH * N;                  // lines of a pass and field
  static constexpr int NT = 2 * NL;                  // threads: a g line and an h line each
  static constexpr int WSZ = MH * N * LP;            // cx per work cube
  static constexpr int OFF_WG = 0, OFF_WH = WSZ, OFF_QG = 2 * WSZ;
  static constexpr int OFF_PH = OFF_QG + N * MH * N;  // [2 slots][2 fields][3][N]
  static constexpr int SMEM_CX = OFF_PH + 2 * 6 * N;
  static constexpr int SLICE = H * NN;               // half spectrum in the scratch
  static constexpr int XSLAB = MH * MH * N;          // staging buffer [k1l][j][x3]
  // scratch per pair: F, G, [2 CTAs][2 alternating buffers][2 fields] staging
  static constexpr int SCRATCH = 2 * SLICE + 8 * XSLAB;
  static_assert(NT % 32 == 0 && NT <= 1024, "thread layout");
};

// Second pass of an inverse transform: the line (k1l = hi, x3 = lo) of a
// work cube W along k2; the outputs with x2 in X_r stay in W, the others go
// to the staging buffer xs for the peer ([k1l][x2 - MH (1 - r)][x3]).
template <int N>
__device__ __forceinline__ void vss_pair_pass2(cx<float>* sW, cx<float>* xs, int r, int hi, int lo) {
  constexpr int LP = N + 1, MH = N / 2;
  cx<float> x[N];
#pragma unroll
  for (int j = 0; j < N; ++j) x[j] = sW[(hi * N + j) * LP + lo];
  fft<float, N, +1>(x);
#pragma unroll
  for (int j = 0; j < MH; ++j) {
    sW[(hi * N + MH * r + j) * LP + lo] = r ? x[MH + j] : x[j];
    __stcg(xs + (hi * MH + j) * N + lo, r ? x[j] : x[MH + j]);
  }
}

template <int N>
__global__ void __launch_bounds__(VssPairGeom<N>::NT, 1) vss_pair_kernel(const VssArgs<float> a) {
  using G = VssPairGeom<N>;
  using C = cx<float>;
  constexpr int H = G::H, NY = G::NY, NN = G::NN, V = G::V, LP = G::LP, MH = G::MH, NL = G::NL;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sWg = reinterpret_cast<C*>(smem_raw) + G::OFF_WG;
  C* const sWh = reinterpret_cast<C*>(smem_raw) + G::OFF_WH;
  C* const sQG = reinterpret_cast<C*>(smem_raw) + G::OFF_QG;
  C* const sPh = reinterpret_cast<C*>(smem_raw) + G::OFF_PH;

  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  // field of this thread (0: g from F, 1: h from G) and its line in a pass:
  // hi = L / N (k1l, or x2l in the third pass), lo = L % N (k2, x3)
  const int fld = tid / NL, L = tid % NL, hi = L / N, lo = L % N;
  C* const sW = fld ? sWh : sWg;
  const int cid = blockIdx.x / 2, ncl = gridDim.x / 2;
  C* const Fg = a.fc + (size_t)cid * G::SCRATCH;
  C* const Gg = Fg + G::SLICE;
  C* const Xs = Gg + G::SLICE;  // staging: [rank][buffer][field][k1l][j][x3]
  const float invV = 1.f / (float)V;
  const int npq = a.P * a.M;
  int xb = 0;  // staging buffer of the next exchange
  auto xmine = [&](int b, int f) { return Xs + (size_t)((r * 2 + b) * 2 + f) * G::XSLAB; };
  auto xpeer = [&](int b, int f) { return (const C*)(Xs + (size_t)(((r ^ 1) * 2 + b) * 2 + f) * G::XSLAB); };
  // a spectrum value at (k1, k2, k3) from a half spectrum in the scratch
  auto at = [&](const C* S, int k1, int k2, int k3) -> C {
    if (k3 <= NY) return __ldcg(S + (k3 * N + k1) * N + k2);
    const C c = __ldcg(S + ((N - k3) * N + (N - k1) % N) * N + (N - k2) % N);
    return mk<C>(c.x, -c.y);
  };

  // Second pass of an inverse transform (vss_pair_pass2) and the exchange;
  // returns the staging buffer to read.
  auto inverse_pass2 = [&]() -> int {
    vss_pair_pass2<N>(sW, xmine(xb, fld), r, hi, lo);
    cl_arrive();
    cl_wait();  // both halves staged (cluster-scope release / acquire)
    const int b = xb;
    xb ^= 1;
    return b;
  };

#pragma unroll 1
  for (int ip = cid; ip < a.npts; ip += ncl) {
    const int pt = a.pt0 + ip;
    const int upt = pt / a.neles, elem = pt % a.neles;

    // ---- F = FFT(f_p) / V (field 0) and G = FFT(f_q) / V (field 1) -------
    // lines (x1 = MH r + hi, x2 = lo) along x3, then (x1l, k3) along x2,
    // through the staging buffers, then (k2, k3) along x1
    {
      const float* f = fld ? a.fq : a.fp;
      const int64_t b0 = soa_ix(upt, a.ldim, elem, (int64_t)((MH * r + hi) * N + lo) * N, V, a.soasz);
      C x[N];
#pragma unroll
      for (int k = 0; k < N; ++k) x[k] = mk<C>(f[b0 + (int64_t)k * a.soasz], 0.f);
      fft<float, N, -1>(x);
#pragma unroll
      for (int k = 0; k <= NY; ++k) sW[(hi * N + lo) * LP + k] = x[k];
    }
    __syncthreads();
    // exchange buffer [k3][x1][k2] of each field: the half spectrum slot
    // itself (written by both CTAs, each its x1 half)
    C* const S = fld ? Gg : Fg;
#pragma unroll 1
    for (int t = L; t < MH * H; t += NL) {
      const int x1l = t / H, k3 = t % H;
      C x[N];
#pragma unroll
      for (int j = 0; j < N; ++j) x[j] = sW[(x1l * N + j) * LP + k3];
      fft<float, N, -1>(x);
#pragma unroll
      for (int j = 0; j < N; ++j) __stcg(S + (k3 * N + MH * r + x1l) * N + j, x[j]);
    }
    cl_arrive();
    cl_wait();  // every x1 of both fields in the scratch
    // lines (k2 in this CTA's half, k3) along x1, into registers, then
    // back in place once both CTAs have read (a second barrier)
    C y[N];
    const bool fwd3 = L < MH * H;
    const int k2f = MH * r + (fwd3 ? L / H : 0), k3f = fwd3 ? L % H : 0;
    if (fwd3) {
#pragma unroll
      for (int i = 0; i < N; ++i) y[i] = __ldcg(S + (k3f * N + i) * N + k2f);
      fft<float, N, -1>(y);
    }
    cl_arrive();
    cl_wait();  // both CTAs hold their lines of the exchange buffer
    if (fwd3) {
#pragma unroll
      for (int i = 0; i < N; ++i) __stcg(S + (k3f * N + i) * N + k2f, cscale(y[i], invV));
    }
    if (tid < 6 * N) sPh[tid] = a.phase[tid];
    // the gain spectrum of this CTA's k-slab starts at zero
    for (int i = tid; i < N * MH * N; i += G::NT) sQG[i] = mk<C>(0.f, 0.f);
    cl_arrive();
    cl_wait();  // F and G complete in the scratch

#pragma unroll 1
    for (int pq = 0; pq < npq; ++pq) {
      const int slot = pq & 1;
      const C* ph = sPh + slot * 6 * N + fld * 3 * N;
      // ---- pass 1: the field's line (k1, k2 = lo) along k3 -------------------
      {
        const int k1 = pair_kmap<N>(r, hi), k2 = lo;
        const C e12 = cmul(ph[k1], ph[N + k2]);
        const C* Sf = fld ? Gg : Fg;
        C x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = cmul(at(Sf, k1, k2, k), cmul(e12, ph[2 * N + k]));
        fft<float, N, +1>(x);
#pragma unroll
        for (int k = 0; k < N; ++k) sW[(hi * N + k2) * LP + k] = x[k];
      }
      // the next (x, y)'s phases into the other slot
      const C phn = (tid < 6 * N && pq + 1 < npq) ? a.phase[(size_t)(pq + 1) * 6 * N + tid] : mk<C>(0.f, 0.f);
      __syncthreads();
      if (tid < 6 * N && pq + 1 < npq) sPh[(slot ^ 1) * 6 * N + tid] = phn;
      // ---- pass 2 and the exchange ------------------------------------------
      const int xr = inverse_pass2();
      // ---- pass 3: g or h on the line (x2 = MH r + hi, x3 = lo) --------------
      C x[N];
      pair_load3<float, N>(x, sW, xpeer(xr, fld), r, hi, lo);
      fft<float, N, +1>(x);
      __syncthreads();  // every thread has read its pass-3 inputs
      if (fld) {
#pragma unroll
        for (int i = 0; i < N; ++i) sWh[(hi * N + lo) * LP + i] = x[i];
      }
      __syncthreads();
      // ---- g h, forward along x1; the k1 the peer owns go to its buffer ------
      if (!fld) {
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] = cmul(x[i], sWh[(hi * N + lo) * LP + i]);
        fft<float, N, -1>(x);
        C* const xs = xmine(xb, 0);
        const int x2 = MH * r + hi;
#pragma unroll
        for (int k1 = 0; k1 < N; ++k1) {
          if (pair_owner<N>(k1) == r) sWg[(pair_kinv<N>(k1) * N + x2) * LP + lo] = x[k1];
          else __stcg(xs + (pair_kinv<N>(k1) * MH + hi) * N + lo, x[k1]);
        }
      }
      cl_arrive();
      cl_wait();  // both halves staged
      const int xf = xb;
      xb ^= 1;
      // ---- forward along x2 on the lines (k1l, x3) ----------------------------
      if (!fld) {
        const C* xp = xpeer(xf, 0);
#pragma unroll
        for (int j = 0; j < N; ++j)
          x[j] = j / MH == r ? sWg[(hi * N + j) * LP + lo] : __ldcg(xp + (hi * MH + j % MH) * N + lo);
        fft<float, N, -1>(x);
#pragma unroll
        for (int j = 0; j < N; ++j) sWg[(hi * N + j) * LP + lo] = x[j];
      }
      __syncthreads();
      // ---- forward along x3 on the lines (k1l, k2); QGhat += b FFT(g h) ------
      if (!fld) {
        const int k1 = pair_kmap<N>(r, hi), k2 = lo;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = sWg[(hi * N + k2) * LP + k];
        fft<float, N, -1>(x);
        const C* bb = a.b + (size_t)pq * V + (k1 * N + k2) * N;
#pragma unroll
        for (int k = 0; k < N; ++k) {
          C* q = sQG + (k * MH + hi) * N + k2;
          *q = cfma(__ldg(bb + k), x[k], *q);
        }
      }
      __syncthreads();
    }

    // ---- QG = IFFT(QGhat) (field 0), fL = IFFT(c G) (field 1) ---------------
    {
      const int k1 = pair_kmap<N>(r, hi), k2 = lo;
      C x[N];
      if (fld) {
        const C* cc = a.c + (k1 * N + k2) * N;
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = cmul(__ldg(cc + k), at(Gg, k1, k2, k));
      } else {
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = sQG[(k * MH + hi) * N + k2];
      }
      fft<float, N, +1>(x);
#pragma unroll
      for (int k = 0; k < N; ++k) sW[(hi * N + k2) * LP + k] = x[k];
    }
    __syncthreads();
    {
      const int xr = inverse_pass2();
      C x[N];
      pair_load3<float, N>(x, sW, xpeer(xr, fld), r, hi, lo);
      fft<float, N, +1>(x);
      __syncthreads();
      if (fld) {
#pragma unroll
        for (int i = 0; i < N; ++i) sWh[(hi * N + lo) * LP + i] = x[i];
      }
      __syncthreads();
      if (!fld) {
        // x2 = MH r + hi, x3 = lo: bank entries v = x1 N^2 + x2 N + x3
        const int64_t b0 = soa_ix(upt, a.ldim, elem, (int64_t)(MH * r + hi) * N + lo, V, a.soasz);
        const int64_t st = (int64_t)NN * a.soasz;
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const float qv = a.prefac * (x[i].x - a.fp[b0 + i * st] * sWh[(hi * N + lo) * LP + i].x);
          a.Q[b0 + i * st] = a.accumulate ? a.Q[b0 + i * st] + qv : qv;
        }
      }
    }
    // the next point rewrites the scratch and the work cubes: both CTAs done
    cl_arrive();
    cl_wait();
  }
  cl_arrive();
  cl_wait();  // no CTA leaves while the peer may still address its memory
}

}  // namespace dgfs
