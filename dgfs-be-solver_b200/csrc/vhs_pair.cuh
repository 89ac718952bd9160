// Two-CTA fast-spectral VHS kernel for grids that do not fit one SM's
// shared memory: FP32 at N = 32 and FP64 at N = 24.  The sizes below are
// those of N = 32 (MH = N/2 = 16); FP64 at N = 24 has MH = 12, K_0 =
// {0..5, 12, 19..23} and 201.7 KB of shared memory.
//
// The same exact restatement of the reference's operator as the single-CTA
// kernel (vhs_cube.cuh: one complex transform R = IFFT(m F) per (p, q), the
// Nyquist-plane term Nq as three 2D transforms, Re S = Re R^2 + Re Nq^2,
// fC = sum_p w1_p FFT(S_p), Q = prefac (Re IFFT(fC) - f Re IFFT(b2 F))),
// frfs/solvers/dgfs/scattering.py:227-286 and vhs-gll.mako:103-266), for a
// grid that does not fit one SM: a thread-block cluster of two CTAs per
// solution point, persistent over the bank.
//
// Data distribution (rank r of the pair):
//   k-slab   CTA r owns the k1 values K_r (16 of them, closed under
//            k1 -> -k1 mod 32, so a line's Hermitian mirror is local):
//            K_0 = {0..7, 16, 25..31}, K_1 = {8..15, 17..24};
//   x-slab   CTA r owns x2 in X_r = [16 r, 16 r + 16).
// A 3D inverse transform runs along k3 on the lines (k1 in K_r, k2), along
// k2 on the lines (k1 in K_r, x3), then along k1 on the lines (x2 in X_r,
// x3).  Between the second and third passes each CTA hands the half of its
// k-slab that the other owns in x (16 complex values per line) to the other
// through a staging buffer in the pair's global scratch (L2 resident):
// coalesced 8-byte stores, one cluster barrier (release/acquire at cluster
// scope), coalesced L2 loads straight into the third pass's registers.
// Measured per (p, q), this moves the 64 KB a CTA sends about three times
// faster than remote shared-memory stores (st.async into the peer's work
// cube, an earlier form of this kernel).  The staging buffers alternate
// between consecutive exchanges, so the barrier of one exchange also tells a
// CTA that the peer has finished reading the buffer it is about to refill.
// Forward transforms (FFT(S_p)) run the passes in the opposite order with
// the same exchange.  The spectrum F of the point (k3 <= N/2, [k3][k1][k2])
// and the gain spectrum fC live in the pair's slice of the scratch too; S_p
// accumulates in shared memory.
//
// Shared memory (complex unless noted): W [16][32][33], S [32][16][32]
// (real), the Nyquist planes T1..T3 [32][33], two phase slots.  352
// threads: 256 main threads (two of the 512 lines of every pass each, one
// after the other: a 32-point register FFT needs ~130 registers) and 96 that
// transform the Nyquist planes during the first two passes of every (p, q).
#pragma once

#include "vhs_push.cuh"

namespace dgfs {

// T, N: precision and grid (FP32 N = 32, FP64 N = 24; N a multiple of 4,
// MH = N/2 values of k1 or x2 per CTA).  LPT: lines of a pass per main
// thread.  LPT = 2: MH N / 2 main threads (lines t and t + MH N / 2, one
// after the other) and the Nyquist lines on threads of their own; LPT = 1:
// MH N threads, the first 3 N of which also take the Nyquist lines.
template <typename T, int N_, int LPT> struct PairGeom {
  static constexpr int N = N_, H = N / 2 + 1, NY = N / 2, NN = N * N, V = N * N * N;
  static constexpr int MH = N / 2;           // k1 (x2) values per CTA
  static constexpr int LP = N + 1;           // padded line stride
  static constexpr int NL = MH * N;          // lines of a pass
  static constexpr int NM = NL / LPT;        // main threads
  static constexpr int NMP = (NM + 31) / 32 * 32;  // main threads padded to whole warps
  static constexpr int HS = MH / LPT;        // step of a thread's line index hi
  static constexpr int NQ = LPT == 2 ? (3 * N + 31) / 32 * 32 : 0;  // threads for the Nyquist planes only
  static constexpr int NT = NMP + NQ;
  static constexpr int PHS = 3 * N + 4;
  static constexpr int OFF_W = 0;                        // [MH][N][LP] cx
  static constexpr int OFF_S = OFF_W + MH * N * LP;      // [N][MH][N] reals
  static constexpr int OFF_T = OFF_S + N * MH * N / 2;   // [3][N][LP] cx
  static constexpr int OFF_PH = OFF_T + 3 * N * LP;      // [2][PHS] cx
  static constexpr int SMEM_CX = OFF_PH + 2 * PHS;
  static constexpr int SLICE = H * NN;                   // cx per spectrum in the scratch
  static constexpr int XSLAB = MH * MH * N;              // cx per staging buffer [k1l][j][x3]
  static_assert(N % 4 == 0 && NM % N == 0, "line mapping");
  // F on the Nyquist planes k2 = N/2 ([k3 <= N/2][k1]) and k3 = N/2
  // ([k2][k1]), lanes (k1) fastest: a copy per CTA
  static constexpr int NQ2 = H * N, NQS = H * N + N * N;
  // scratch per pair: F, fC, [2 CTAs][2 alternating buffers] staging, then
  // [2 CTAs] Nyquist-plane copies
  static constexpr int SCRATCH = 2 * SLICE + 4 * XSLAB + 2 * NQS;
};

// k1 ownership, closed under k1 -> -k1 mod N (Q = N/4, MH = N/2):
// K_0 = {0..Q-1, MH, N-Q+1..N-1}, K_1 = {Q..MH-1, MH+1..N-Q}; for N = 32
// K_0 = {0..7, 16, 25..31}, K_1 = {8..15, 17..24}
template <int N> __device__ __forceinline__ int pair_owner(int k1) {
  constexpr int Q = N / 4, MH = N / 2;
  return (k1 < Q || k1 == MH || k1 > N - Q) ? 0 : 1;
}
template <int N> __device__ __forceinline__ int pair_kinv(int k1) {
  constexpr int Q = N / 4, MH = N / 2;
  return k1 < Q ? k1 : k1 == MH ? Q : k1 > N - Q ? k1 - N + MH : k1 < MH ? k1 - Q : k1 - Q - 1;
}
template <int N> __device__ __forceinline__ int pair_kmap(int r, int l) {
  constexpr int Q = N / 4, MH = N / 2;
  return r == 0 ? (l < Q ? l : l == Q ? MH : l + N - MH) : (l < Q ? l + Q : l + Q + 1);
}

__device__ __forceinline__ void cl_sync() {
  cl_arrive();
  cl_wait();
}

// third-pass line (x2l = hi, x3 = lo) along k1: the k1 of this CTA from its
// work cube (row kinv(k1) N + x2, x2 = MH r + hi), the others from the
// peer's staging buffer ([kinv(k1)][hi][lo], written before the barrier)
template <typename T, int N>
__device__ __forceinline__ void pair_load3(cx<T> (&x)[N], const cx<T>* sW, const cx<T>* xpeer, int r, int hi,
                                           int lo) {
  constexpr int LP = N + 1, MH = N / 2;
#pragma unroll
  for (int k1 = 0; k1 < N; ++k1)
    x[k1] = pair_owner<N>(k1) == r ? sW[(pair_kinv<N>(k1) * N + MH * r + hi) * LP + lo]
                                   : __ldcg(xpeer + (pair_kinv<N>(k1) * MH + hi) * N + lo);
}

template <typename T, int NV, int LPT>
__global__ void __launch_bounds__(PairGeom<T, NV, LPT>::NT, 1) vhs_pair_kernel(const VhsArgs<T> a) {
  using G = PairGeom<T, NV, LPT>;
  constexpr int HS = G::HS;
  using C = cx<T>;
  constexpr int N = G::N, H = G::H, NY = G::NY, NN = G::NN, V = G::V, LP = G::LP, NM = G::NM, PHS = G::PHS;
  constexpr int MH = G::MH;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sW = reinterpret_cast<C*>(smem_raw) + G::OFF_W;
  T* const sS = reinterpret_cast<T*>(reinterpret_cast<C*>(smem_raw) + G::OFF_S);
  C* const sT1 = reinterpret_cast<C*>(smem_raw) + G::OFF_T;
  C* const sT2 = sT1 + N * LP;
  C* const sT3 = sT2 + N * LP;
  C* const sPh = reinterpret_cast<C*>(smem_raw) + G::OFF_PH;
  __shared__ double sRed[5][G::NT / 32];
  __shared__ double sMom[5];

  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const bool is_main = tid < NM;
  // the Nyquist lines: own threads (LPT = 2) or the first 3 N main threads
  const int tq = G::NQ > 0 ? tid - G::NMP : tid;
  const bool has_nyq = tq >= 0 && tq < 3 * N;
  const int cid = blockIdx.x / 2, ncl = gridDim.x / 2;
  // the pair's scratch: F [H][N][N] then fC [H][N][N] (fC doubles as the
  // exchange buffer of the forward transform of f)
  C* const Fg = a.fc + (size_t)cid * G::SCRATCH;
  C* const fC = Fg + G::SLICE;
  C* const Xs = fC + G::SLICE;  // staging: [rank][buffer][k1l][j][x3]
  C* const Nq = Xs + 4 * G::XSLAB + r * G::NQS;  // this CTA's Nyquist-plane copy
  const T invV = T(1) / T(V);
  const int npq = a.P * a.M;
  // a main thread's lines in every pass: L = tid + NM h (h < LPT), with
  // hi = L / N (k1l, or x2l in the third pass) and lo = L % N (k2, x3)
  const int lo = tid % N, hi0 = tid / N;  // hi of line h: hi0 + HS h
  const uint32_t peer = (uint32_t)(r ^ 1);
  int xb = 0;  // staging buffer of the next exchange
  auto xmine = [&](int b) { return Xs + (size_t)(r * 2 + b) * G::XSLAB; };
  auto xpeer = [&](int b) { return (const C*)(Xs + (size_t)((r ^ 1) * 2 + b) * G::XSLAB); };

  // Second pass of an inverse transform (lines (k1l, x3 = lo) along k2) and
  // the exchange: of the 32 outputs (index x2) of each line the 16 with x2
  // in X_r stay, the others go to the peer, which keeps them at row
  // k1l * 32 + 16 r + (x2 - 16 (1 - r)) of its work cube -- the region it
  // has just read for its own second pass.  Nyquist threads run `nyq`
  // (their own second pass) meanwhile.
  // Second pass of an inverse transform (lines (k1l, x3 = lo) along k2) and
  // the exchange: of the 32 outputs (index x2) of each line the 16 with x2
  // in X_r stay in the work cube, the others go to this CTA's staging buffer
  // [k1l][x2 - 16 (1 - r)][x3] for the peer.  Nyquist threads run `nyq`
  // (their own second pass) meanwhile.  Returns the buffer to read.
  auto pass2_exchange = [&](auto&& nyq) -> int {
    if (has_nyq) nyq();
    if (is_main) {
      C* const xs = xmine(xb);
#pragma unroll 1
      for (int h = 0; h < LPT; ++h) {
        const int hi = hi0 + HS * h;
        C x[N];
#pragma unroll
        for (int j = 0; j < N; ++j) x[j] = sW[(hi * N + j) * LP + lo];
        fft<T, N, +1>(x);
#pragma unroll
        for (int j = 0; j < MH; ++j) {
          sW[(hi * N + MH * r + j) * LP + lo] = r ? x[MH + j] : x[j];
          __stcg(xs + (hi * MH + j) * N + lo, r ? x[j] : x[MH + j]);
        }
      }
    }
    cl_sync();  // both halves staged (cluster-scope release / acquire)
    const int b = xb;
    xb ^= 1;
    return b;
  };
  const int npts = a.pcount ? min(a.npts, *a.pcount) : a.npts;
#pragma unroll 1
  for (int ip = cid; ip < npts; ip += ncl) {
    const int pt = a.plist ? a.plist[a.pt0 + ip] : a.pt0 + ip;
    // listed ids come from device memory: both CTAs read the same entry and
    // skip together, so the cluster barriers stay paired
    if ((unsigned)pt >= (unsigned)(a.nupts * a.neles)) continue;
    const int upt = pt / a.neles, elem = pt % a.neles;

    // ---- F = FFT(f) / V into the scratch, k3 <= N/2 ------------------------
    // lines (x1 = 16 r + hi, x2 = lo) along x3, then (x1l, k3) along x2
    // (272 lines), then through the scratch to lines (k2, k3) along x1
    if (is_main) {
#pragma unroll 1
      for (int h = 0; h < LPT; ++h) {
        const int hi = hi0 + HS * h, x1 = MH * r + hi;
        const int64_t b0 = soa_ix(upt, a.ldim, elem, (int64_t)(x1 * N + lo) * N, V, a.soasz);
        C x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = mk<C>(a.f[b0 + (int64_t)k * a.soasz], T(0));
        fft<T, N, -1>(x);
#pragma unroll
        for (int k = 0; k <= NY; ++k) sW[(hi * N + lo) * LP + k] = x[k];
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int t = tid; t < MH * H; t += G::NT) {
      const int x1l = t / H, k3 = t % H;
      C x[N];
#pragma unroll
      for (int j = 0; j < N; ++j) x[j] = sW[(x1l * N + j) * LP + k3];
      fft<T, N, -1>(x);
      // exchange buffer [k3][x1][k2] (the fC slice, free until p = 0 ends)
#pragma unroll
      for (int j = 0; j < N; ++j) fC[(k3 * N + MH * r + x1l) * N + j] = x[j];
    }
    cl_sync();  // the exchange buffer is complete (cluster-scope release/acquire)
#pragma unroll 1
    for (int t = tid; t < MH * H; t += G::NT) {
      const int k2 = MH * r + t / H, k3 = t % H;
      C x[N];
#pragma unroll
      for (int i = 0; i < N; ++i) x[i] = __ldcg(fC + (k3 * N + i) * N + k2);
      fft<T, N, -1>(x);
#pragma unroll
      for (int i = 0; i < N; ++i) Fg[(k3 * N + i) * N + k2] = cscale(x[i], invV);
    }
    if (tid < 3 * N) {
      const C e = a.phase[tid];
      sPh[tid] = e;
      if (tid % N == NY) sPh[3 * N + tid / N] = cmul(mk<C>(e.x, -e.y), mk<C>(e.x, -e.y));
    }
    cl_sync();  // F complete in the scratch; the exchange buffer may be reused
    // the planes k2 = N/2 and k3 = N/2 of F with k1 fastest, so that the
    // Nyquist lines of those planes (one k1 per lane) read coalesced rows
#pragma unroll 1
    for (int t = tid; t < G::NQS; t += G::NT) {
      const bool q2 = t < G::NQ2;
      const int u = q2 ? t : t - G::NQ2, row = u / N, k1 = u % N;
      Nq[t] = __ldcg(Fg + (q2 ? (row * N + k1) * N + NY : (NY * N + k1) * N + row));
    }
    __syncthreads();

    // F at (k1, k2, k3) from the half spectrum in the scratch (written by
    // both CTAs: read through L2)
    auto Fat = [&](int k1, int k2, int k3) -> C {
      if (k3 <= NY) return __ldcg(Fg + (k3 * N + k1) * N + k2);
      const C c = __ldcg(Fg + ((N - k3) * N + (N - k1) % N) * N + (N - k2) % N);
      return mk<C>(c.x, -c.y);
    };

    int slot = 0;
#pragma unroll 1
    for (int p = 0; p < a.P; ++p) {
#pragma unroll 1
      for (int q = 0; q < a.M; ++q) {
        const int pq = p * a.M + q;
        const C* ph = sPh + slot * PHS;
        const C th1 = ph[3 * N], th2 = ph[3 * N + 1], th3 = ph[3 * N + 2];
        const C phn = (tid < 3 * N && pq + 1 < npq) ? a.phase[(size_t)(pq + 1) * 3 * N + tid] : mk<C>(T(0), T(0));
        // pass 1: lines (k1, k2 = lo) along k3 | Nyquist first axes
        if (is_main) {
#pragma unroll 1
          for (int h = 0; h < LPT; ++h) {
            const int hi = hi0 + HS * h, k1 = pair_kmap<N>(r, hi), k2 = lo;
            const C E12 = cmul(ph[k1], ph[N + k2]);
            C t12 = mk<C>(T(1), T(0));
            if (k1 == NY) t12 = th1;
            if (k2 == NY) t12 = cmul(t12, th2);
            const C E12t = cmul(E12, t12);
            const C s0 = cadd(E12, E12t), s3 = cadd(E12, cmul(E12t, th3));
            const C A = mk<C>(T(0.5) * (s0.x + s0.y), T(0.5) * (s0.y - s0.x));
            const C A3 = mk<C>(T(0.5) * (s3.x + s3.y), T(0.5) * (s3.y - s3.x));
            C x[N];
#pragma unroll
            for (int k = 0; k < N; ++k) {
              const C e3 = ph[2 * N + k];
              const C& Ak = k == NY ? A3 : A;
              x[k] = cscale(Fat(k1, k2, k), Ak.x * e3.x - Ak.y * e3.y);
            }
            fft<T, N, +1>(x);
#pragma unroll
            for (int k = 0; k < N; ++k) sW[(hi * N + k2) * LP + k] = x[k];
          }
        }
        if (has_nyq) {
          // n F on the Nyquist planes (vhs_cube.cuh): plane 1 (k1 = N/2)
          // lines over k3, plane 2 (k2 = N/2) lines over k3, plane 3
          // (k3 = N/2) lines over k2; one coefficient per line
          const int which = tq / N, j = tq % N;
          const bool p3 = which == 2;
          C Eb, tb;
          if (which == 0) {
            Eb = cmul(ph[NY], ph[N + j]);
            tb = j == NY ? cmul(th1, th2) : th1;
          } else if (which == 1) {
            Eb = cmul(ph[j], ph[N + NY]);
            tb = th2;
          } else {
            Eb = cmul(ph[j], ph[2 * N + NY]);
            tb = th3;
          }
          C B = cmul(Eb, mk<C>(T(1) - tb.x, -tb.y));
          const C tb3 = cmul(tb, th3);
          C B3 = p3 ? mk<C>(T(0), T(0)) : cmul(Eb, mk<C>(T(1) - tb3.x, -tb3.y));
          if (which != 0 && j == NY) B = B3 = mk<C>(T(0), T(0));
          const C A = mk<C>(T(0.5) * (B.x + B.y), T(0.5) * (B.y - B.x));
          const C A3 = mk<C>(T(0.5) * (B3.x + B3.y), T(0.5) * (B3.y - B3.x));
          const C* ev = ph + (p3 ? N : 2 * N);
          // the line's F values, one load each: plane 1 from the half
          // spectrum (rows k3, stride N^2), planes 2 and 3 from the copies
          // (rows k3 or k2, stride N); k3 > N/2 from the conjugate mirror
          const C* const qb = which == 0 ? Fg + NY * N : (which == 1 ? Nq : Nq + G::NQ2);
          const int rs = which == 0 ? NN : N, jm = (N - j) % N;
          const bool mir = !p3;
          C x[N];
#pragma unroll
          for (int k = 0; k < N; ++k) {
            C v;
            if (k <= NY) {
              v = __ldcg(qb + k * rs + j);
            } else {
              const C c = __ldcg(mir ? qb + (N - k) * rs + jm : qb + k * rs + j);
              v = mk<C>(c.x, mir ? -c.y : c.y);
            }
            const C& Ak = k == NY ? A3 : A;
            const C e = ev[k];
            x[k] = cscale(v, Ak.x * e.x - Ak.y * e.y);
          }
          fft<T, N, +1>(x);
          C* Tp = which == 0 ? sT1 : (which == 1 ? sT2 : sT3);
#pragma unroll
          for (int k = 0; k < N; ++k) Tp[j * LP + k] = x[k];
        }
        __syncthreads();
        if (tid < 3 * N && pq + 1 < npq) {
          C* dst = sPh + (slot ^ 1) * PHS;
          dst[tid] = phn;
          if (tid % N == NY) dst[3 * N + tid / N] = cmul(mk<C>(phn.x, -phn.y), mk<C>(phn.x, -phn.y));
        }
        // pass 2 and the exchange | Nyquist second axes (all 32 columns of
        // every plane; the third pass reads the rows of its own x2 half)
        const int xr = pass2_exchange([&]() {
          const int which = tq / N, col = tq % N;
          C* Tp = which == 0 ? sT1 : (which == 1 ? sT2 : sT3);
          C x[N];
#pragma unroll
          for (int j = 0; j < N; ++j) x[j] = Tp[j * LP + col];
          fft<T, N, +1>(x);
#pragma unroll
          for (int j = 0; j < N; ++j) Tp[j * LP + col] = x[j];
        });
        // pass 3: lines (x2 = 16 r + hi, x3 = lo) along k1;
        // S += Re R^2 + Re Nq^2
        if (is_main) {
#pragma unroll 1
          for (int h = 0; h < LPT; ++h) {
            const int hi = hi0 + HS * h, x2 = MH * r + hi, x3 = lo;
            C x[N];
            pair_load3<T, N>(x, sW, xpeer(xr), r, hi, lo);
            fft<T, N, +1>(x);
            const C t1 = sT1[x2 * LP + x3];
            const T s2 = (x2 & 1) ? T(-1) : T(1), s3 = (x3 & 1) ? T(-1) : T(1);
            T* Sl = sS + hi * N + x3;
#pragma unroll
            for (int i = 0; i < N; ++i) {
              const T s1 = (i & 1) ? T(-1) : T(1);
              const C t2 = sT2[i * LP + x3], t3 = sT3[i * LP + x2];
              const T nr = s1 * t1.x + s2 * t2.x + s3 * t3.x;
              const T ni = s1 * t1.y + s2 * t2.y + s3 * t3.y;
              const T v = x[i].x * x[i].x - x[i].y * x[i].y + nr * nr - ni * ni;
              Sl[i * MH * N] = q == 0 ? v : Sl[i * MH * N] + v;
            }
          }
        }
        slot ^= 1;
        __syncthreads();
      }

      // ---- fC += w1_p FFT(S_p) ----------------------------------------------
      // lines (x2l, x3) along x1 from S, the exchange to k-slabs, lines
      // (k1l, x3) along x2, lines (k1l, k2) along x3 into fC (k3 <= N/2).
      // An output k1 of a first-pass line is local when owned, else pushed
      // to the peer's row kinv(k1) * 32 + x2.
      if (is_main) {
        C* const xs = xmine(xb);
#pragma unroll 1
        for (int h = 0; h < LPT; ++h) {
          const int hi = hi0 + HS * h, x2 = MH * r + hi;
          C x[N];
          const T* Sl = sS + hi * N + lo;
#pragma unroll
          for (int i = 0; i < N; ++i) x[i] = mk<C>(Sl[i * MH * N], T(0));
          fft<T, N, -1>(x);
#pragma unroll
          for (int k1 = 0; k1 < N; ++k1) {
            if (pair_owner<N>(k1) == r) sW[(pair_kinv<N>(k1) * N + x2) * LP + lo] = x[k1];
            else __stcg(xs + (pair_kinv<N>(k1) * MH + hi) * N + lo, x[k1]);
          }
        }
      }
      cl_sync();  // both halves staged
      const int xr = xb;
      xb ^= 1;
      if (is_main) {
#pragma unroll 1
        for (int h = 0; h < LPT; ++h) {
          const int hi = hi0 + HS * h;
          const C* xp = xpeer(xr);
          C x[N];
#pragma unroll
          for (int j = 0; j < N; ++j)
            x[j] = j / MH == r ? sW[(hi * N + j) * LP + lo] : __ldcg(xp + (hi * MH + j % MH) * N + lo);
          fft<T, N, -1>(x);
#pragma unroll
          for (int j = 0; j < N; ++j) sW[(hi * N + j) * LP + lo] = x[j];
        }
      }
      __syncthreads();
      if (is_main) {
        const T* w1 = a.w1t + (size_t)p * V;
#pragma unroll 1
        for (int h = 0; h < LPT; ++h) {
          const int hi = hi0 + HS * h, k1 = pair_kmap<N>(r, hi), k2 = lo, L = k1 * N + k2;
          C x[N];
#pragma unroll
          for (int k = 0; k < N; ++k) x[k] = sW[(hi * N + k2) * LP + k];
          fft<T, N, -1>(x);
#pragma unroll
          for (int k = 0; k <= NY; ++k) x[k] = cscale(x[k], __ldg(w1 + k * NN + L));
          if (p > 0) {
            // read-modify-write in chunks of 6 (the loads of a chunk issued
            // together; fewer live registers than the whole line)
#pragma unroll
            for (int k0 = 0; k0 <= NY; k0 += 6) {
              C acc[6];
#pragma unroll
              for (int k = k0; k < k0 + 6 && k <= NY; ++k) acc[k - k0] = fC[k * NN + L];
#pragma unroll
              for (int k = k0; k < k0 + 6 && k <= NY; ++k) fC[k * NN + L] = cadd(acc[k - k0], x[k]);
            }
          } else {
#pragma unroll
            for (int k = 0; k <= NY; ++k) fC[k * NN + L] = x[k];
          }
        }
      }
      __syncthreads();
    }

    // ---- Q = prefac (Re IFFT(fC) - f Re IFFT(b2 F)) ----------------------------
    // Two inverse transforms over the half spectra (each line's mirror is in
    // this CTA's k-slab): Lf into S, then the gain and Q into S.
#pragma unroll 1
    for (int t = 0; t < 2; ++t) {
      if (is_main) {
#pragma unroll 1
        for (int h = 0; h < LPT; ++h) {
          const int hi = hi0 + HS * h, k1 = pair_kmap<N>(r, hi), k2 = lo, L = k1 * N + k2;
          const int m1 = (N - k1) % N, m2 = (N - k2) % N;
          C x[N];
#pragma unroll
          for (int k = 0; k < N; ++k) {
            if (t == 0) {
              x[k] = cscale(Fat(k1, k2, k), __ldg(a.b2t + k * NN + L));
            } else if (k <= NY) {
              x[k] = fC[k * NN + L];
            } else {
              const C c = fC[(N - k) * NN + m1 * N + m2];
              x[k] = mk<C>(c.x, -c.y);
            }
          }
          fft<T, N, +1>(x);
#pragma unroll
          for (int k = 0; k < N; ++k) sW[(hi * N + k2) * LP + k] = x[k];
        }
      }
      __syncthreads();
      const int xr = pass2_exchange([]() {});
      if (is_main) {
#pragma unroll 1
        for (int h = 0; h < LPT; ++h) {
          const int hi = hi0 + HS * h;
          C x[N];
          pair_load3<T, N>(x, sW, xpeer(xr), r, hi, lo);
          fft<T, N, +1>(x);
          T* Sl = sS + hi * N + lo;
          if (t == 0) {
#pragma unroll
            for (int i = 0; i < N; ++i) Sl[i * MH * N] = x[i].x;
          } else {
            // x2 = MH r + hi, x3 = lo: bank entries v = i N^2 + x2 N + x3
            const int64_t b0 = soa_ix(upt, a.ldim, elem, (int64_t)(MH * r + hi) * N + lo, V, a.soasz);
            const int64_t st = (int64_t)NN * a.soasz;
#pragma unroll
            for (int i0 = 0; i0 < N; i0 += 8) {
              T fl[8];
#pragma unroll
              for (int i = 0; i < 8; ++i) fl[i] = a.f[b0 + (i0 + i) * st];
#pragma unroll
              for (int i = 0; i < 8; ++i)
                Sl[(i0 + i) * MH * N] = a.prefac * (x[i0 + i].x - fl[i] * Sl[(i0 + i) * MH * N]);
            }
          }
        }
      }
      __syncthreads();
    }

    // write Q (this CTA's x2 half), with the optional FP64 projection onto
    // zero mass, momentum and energy over both halves
    double lam[5] = {0, 0, 0, 0, 0};
    if (a.project) {
      double mom[5] = {0, 0, 0, 0, 0};
      if (is_main) {
#pragma unroll 1
        for (int h = 0; h < LPT; ++h) {
          const int hi = hi0 + HS * h;
          const T* Sl = sS + hi * N + lo;
#pragma unroll 4
          for (int i = 0; i < N; ++i) {
            const int64_t v = (int64_t)(i * N + MH * r + hi) * N + lo;
            const double d = (double)Sl[i * MH * N];
            const double c0 = a.cvec[v], c1 = a.cvec[V + v], c2 = a.cvec[2 * V + v];
            mom[0] += d;
            mom[1] += d * c0;
            mom[2] += d * c1;
            mom[3] += d * c2;
            mom[4] += d * (c0 * c0 + c1 * c1 + c2 * c2);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        double s = mom[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((tid & 31) == 0) sRed[k][tid >> 5] = s;
      }
      __syncthreads();
      if (tid < 5) {
        double s = 0;
        for (int w = 0; w < G::NT / 32; ++w) s += sRed[tid][w];
        sMom[tid] = s;
      }
      cl_sync();  // both halves' moments in place
      double mt[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) mt[k] = sMom[k] + cluster.map_shared_rank(sMom, (int)peer)[k];
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < 5; ++j) s += a.ginv[k * 5 + j] * mt[j];
        lam[k] = s;
      }
    }
    if (is_main) {
#pragma unroll 1
      for (int h = 0; h < LPT; ++h) {
        const int hi = hi0 + HS * h;
        const T* Sl = sS + hi * N + lo;
        const int64_t b0 = soa_ix(upt, a.ldim, elem, (int64_t)(MH * r + hi) * N + lo, V, a.soasz);
        const int64_t st = (int64_t)NN * a.soasz;
#pragma unroll 4
        for (int i = 0; i < N; ++i) {
          T qq = Sl[i * MH * N];
          if (a.project) {
            const int64_t v = (int64_t)(i * N + MH * r + hi) * N + lo;
            const double c0 = a.cvec[v], c1 = a.cvec[V + v], c2 = a.cvec[2 * V + v];
            qq = (T)((double)qq - (lam[0] + lam[1] * c0 + lam[2] * c1 + lam[3] * c2 +
                                       lam[4] * (c0 * c0 + c1 * c1 + c2 * c2)));
          }
          a.Q[b0 + i * st] = qq;
        }
      }
    }
    // the next point rewrites the scratch, S and the moments: both CTAs done
    cl_sync();
  }
  cl_sync();  // no CTA leaves while the peer may still address its memory
}

}  // namespace dgfs
