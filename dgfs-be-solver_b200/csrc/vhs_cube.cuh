// Single-CTA fast-spectral VHS kernel for FP32 and N <= 24: the whole N^3
// problem of one point lives in one CTA's shared memory, so no transform
// crosses SMs, and the transform count is nearly halved by an exact
// restatement that uses the reality of f.
//
// The reference (frfs/solvers/dgfs/scattering.py:227-286, vhs-gll.mako)
// computes per radial node p and direction q
//     t3 = IFFT(cos a F), t4 = IFFT(sin a F),  S = t3^2 + t4^2 (complex),
// with F = FFT(f)/V and a(l) = fac_p s_q.l, then
//     Q = prefac (Re IFFT(sum_p w1_p FFT(sum_q S)) - f Re IFFT(b2 F)).
// w1_p and b2 depend on |l| only, and the index grid maps -l onto itself up
// to the Nyquist index (l0 holds -N/2 but not +N/2), so both are even on the
// grid: Re IFFT(w FFT(S)) = IFFT(w FFT(Re S)) and only Re S matters.
// Let l' = -l (mod N).  Real f gives F(l') = conj F(l), and
// a(l') = -a(l) - theta(l), theta = fac_p N sum over the axes where l sits on
// the Nyquist index of s_q[axis] (theta = 0 off those planes).  Splitting
// cos a F and sin a F into parts that are even and odd under l -> l'
// (conjugated) gives exactly
//     Re S = Re(R^2) + Re(Nq^2),
//     R  = IFFT(m F),  m = (cos a + cos(a+th) + sin a + sin(a+th)) / 2,
//     Nq = IFFT(n F),  n = (cos a - cos(a+th) + sin a - sin(a+th)) / 2,
// where n vanishes off the three Nyquist planes, so Nq is three 2D
// transforms broadcast along one axis with a (-1)^x sign:
//     Nq(x) = (-1)^x1 T1(x2,x3) + (-1)^x2 T2(x1,x3) + (-1)^x3 T3(x1,x2).
// Off the Nyquist planes m = cos a + sin a: one complex transform per (p, q)
// instead of two.  Per point: 1 + Nrho M + Nrho + 2 full transforms plus
// the 2D ones (reference: 3 Nrho M + 3).
//
// Layout (shared memory, complex float): F for k3 <= N/2 ([N][N][N/2+1]),
// the work cube as N^2 lines of N+1 (padding keeps line-parallel accesses
// free of bank conflicts), the three Nyquist planes, the axis phases.
// The gain spectrum fC accumulates in a global (L2-resident) slice per CTA,
// stored with the last axis outermost so that the per-line accesses of a
// warp are contiguous (w1 and b2 come in the same order, from their own
// tables).
// Main threads own two lines per pass; NQ extra threads (one line each)
// transform the Nyquist planes during the first two passes of every (p, q).
#pragma once

#include "vhs_kernel.cuh"

namespace dgfs {

template <int N> struct CubeGeom {
  static constexpr int H = N / 2 + 1;
  static constexpr int NN = N * N;
  static constexpr int LP = N + 1;                      // padded line stride
  static constexpr int NM = NN / 2;                     // main threads (2 lines)
  static constexpr int NQ = ((3 * N + 31) / 32) * 32;  // Nyquist threads, one line each
  static constexpr int NT = NM + NQ;
  static constexpr int V = N * N * N;
  static constexpr int PHS = 3 * N + 4;                 // one phase slot
  // F at (k1, k2, k3 <= N/2) sits at k1 FS + k2 H + k3: one padding entry
  // per k1 slab makes lanes that differ in k1 (the Nyquist-plane lines)
  // fall in different banks
  static constexpr int FS = N * H + 1;
  static constexpr int OFF_F = 0;                       // [N][FS]
  static constexpr int OFF_W = OFF_F + N * FS;          // [NN][LP]
  static constexpr int OFF_T = OFF_W + NN * LP;         // [3][N][LP]
  static constexpr int OFF_PH = OFF_T + 3 * N * LP;     // [2][PHS]
  static constexpr int SMEM_CX = OFF_PH + 2 * PHS;
  static_assert(NM % 32 == 0, "main threads must fill warps");
};

// Radial-node chunks per point.  A launch with few points would leave SMs
// idle with one point per CTA, so each point's P radial nodes can be split
// into P work items of one node each: cost ~ waves x (nodes per item x
// (3 M + 3) + 3) passes (the 3: every item transforms f itself).  Only 1 or
// P chunks: with one node per chunk the final sum over the chunks' slices
// adds the nodes in the same order as the unsplit accumulation, so a point's
// Q does not depend on the launch it is part of (bit for bit).  Items are
// capped at kCubeSlices per CTA of the grid (the partial-spectrum scratch:
// with P = 12 a split covers up to two waves of whole points).  Every CTA
// computes the same value.
constexpr int kCubeSlices = 24;
__device__ __forceinline__ int cube_chunks(int npts, int G, int P, int M) {
  if (P < 2 || (long long)npts * P > (long long)kCubeSlices * G) return 1;
  const double per_node = 3.0 * M + 3.0;
  const double whole = (double)((npts + G - 1) / G) * (P * per_node + 3.0);
  const double split = (double)(((long long)npts * P + G - 1) / G) * (per_node + 3.0);
  return split < whole ? P : 1;
}

template <int N, bool IL1>
__global__ void __launch_bounds__(CubeGeom<N>::NT, 1) vhs_cube_kernel(const VhsArgs<float> a) {
  using G = CubeGeom<N>;
  using C = cx<float>;
  constexpr int H = G::H, NN = G::NN, LP = G::LP, NM = G::NM, V = G::V, PHS = G::PHS, NT = G::NT, FS = G::FS;
  constexpr int NY = N / 2;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sF = reinterpret_cast<C*>(smem_raw) + G::OFF_F;
  C* const sW = reinterpret_cast<C*>(smem_raw) + G::OFF_W;
  C* const sT1 = reinterpret_cast<C*>(smem_raw) + G::OFF_T;
  C* const sT2 = sT1 + N * LP;
  C* const sT3 = sT2 + N * LP;
  C* const sPh = reinterpret_cast<C*>(smem_raw) + G::OFF_PH;
  __shared__ double sRed[5][NT / 32];
  __shared__ double sLam[5];

  const int tid = threadIdx.x;
  const bool is_main = tid < NM;
  const int tq = tid - NM;
  C* const fcg = a.fc + (size_t)blockIdx.x * V;
  const float invV = 1.f / (float)V;
  const int npq = a.P * a.M;

  // axis phases e^{i fac_p s_q[ax] l0[k]} of (p, q), and
  // Theta_ax = e^{i fac_p N s_q[ax]} = conj(e^{i fac_p s_q[ax] l0[N/2]})^2.
  // Threads tid < 3N each carry one entry: fetched from L2 at the start of
  // a pass (phase_fetch), stored to the other slot at its end
  // (phase_store), so the load latency hides behind the pass.
  static_assert(3 * N <= NT, "one phase entry per thread");
  auto phase_fetch = [&](int pq) -> C {
    return tid < 3 * N ? a.phase[(size_t)pq * 3 * N + tid] : mk<C>(0.f, 0.f);
  };
  auto phase_store = [&](C e, int slot) {
    if (tid < 3 * N) {
      C* dst = sPh + slot * PHS;
      dst[tid] = e;
      if (tid % N == NY) {
        const C ce = mk<C>(e.x, -e.y);
        dst[3 * N + tid / N] = cmul(ce, ce);
      }
    }
  };
  // F at (k1, k2, k3) from the half spectrum
  auto Fat = [&](int k1, int k2, int k3) -> C {
    if (k3 <= NY) return sF[k1 * FS + k2 * H + k3];
    const C c = sF[((N - k1) % N) * FS + ((N - k2) % N) * H + (N - k3)];
    return mk<C>(c.x, -c.y);
  };

  const int npts = a.pcount ? min(a.npts, *a.pcount) : a.npts;
  // work item = (point, chunk of radial nodes); with KP > 1 each chunk's
  // partial gain spectrum goes to its own scratch slice and the CTA that
  // finishes a point's last chunk (a counter per point) sums the slices and
  // completes the point.  No CTA waits for another.
  // The values that stay fixed over an item live in shared memory (s_kp;
  // s_it = first and end radial node, upt, elem): read where needed, they
  // hold no registers through the (p, q) loop.
  __shared__ int s_last, s_kp, s_ni, s_ga, s_it[4];
  {
    const int kp = a.pdone ? cube_chunks(npts, gridDim.x, a.P, a.M) : 1;
    const int nitems = npts * kp;
    // as few CTAs as the number of waves needs (same makespan): the SMs
    // left over stay free for kernels on other streams (the surrogate's
    // network path runs beside its plain fallback)
    const int waves = (nitems + gridDim.x - 1) / gridDim.x;
    const int gactive = waves > 0 ? (nitems + waves - 1) / waves : 0;
    if ((int)blockIdx.x >= gactive) return;  // uniform over the CTA, before any barrier
    if (tid == 0) {
      s_kp = kp;
      s_ni = nitems;
      s_ga = gactive;
    }
  }
  __syncthreads();
  for (int item = blockIdx.x; item < s_ni; item += s_ga) {
    const int ip = item / s_kp;
    const int pt = a.plist ? a.plist[a.pt0 + ip] : a.pt0 + ip;
    if ((unsigned)pt >= (unsigned)(a.nupts * a.neles)) continue;  // uniform over the CTA
    const int upt = pt / a.neles, elem = pt % a.neles;
    if (tid == 0) {
      const int ch = item % s_kp;
      s_it[0] = ch * a.P / s_kp;
      s_it[1] = (ch + 1) * a.P / s_kp;
      s_it[2] = upt;
      s_it[3] = elem;
    }

    // ---- F = FFT(f) / V, kept for k3 <= N/2 ---------------------------------
    if (is_main) {
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        const int L = tid + r * NM;  // line (x1, x2) along x3
        C x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = mk<C>(a.f[soa_ix(upt, a.ldim, elem, (int64_t)L * N + k, V, a.soasz)], 0.f);
        fft<float, N, -1>(x);
#pragma unroll
        for (int k = 0; k < N; ++k) sW[L * LP + k] = x[k];
      }
    }
    __syncthreads();
    if (is_main) {
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        const int L = tid + r * NM, x1 = L / N, k3 = L % N;  // line (x1, k3) along x2
        C x[N];
#pragma unroll
        for (int j = 0; j < N; ++j) x[j] = sW[(x1 * N + j) * LP + k3];
        fft<float, N, -1>(x);
#pragma unroll
        for (int j = 0; j < N; ++j) sW[(x1 * N + j) * LP + k3] = x[j];
      }
    }
    __syncthreads();
    if (is_main) {
#pragma unroll 1
      for (int L = tid; L < N * H; L += NM) {
        const int k2 = L / H, k3 = L % H;  // line (k2, k3) along x1, k3 <= N/2
        C x[N];
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] = sW[(i * N + k2) * LP + k3];
        fft<float, N, -1>(x);
#pragma unroll
        for (int i = 0; i < N; ++i) sF[i * FS + k2 * H + k3] = cscale(x[i], invV);
      }
    }
    phase_store(phase_fetch(s_it[0] * a.M), 0);
    __syncthreads();

    // ---- gain: fC = sum_p w1_p FFT(sum_q Re S_pq) ---------------------------
    int slot = 0;
#pragma unroll 1
    for (int p = s_it[0]; p < s_it[1]; ++p) {
      float S0[N], S1[N];
#pragma unroll
      for (int k = 0; k < N; ++k) S0[k] = S1[k] = 0.f;
#pragma unroll 1
      for (int q = 0; q < a.M; ++q) {
        const int pq = p * a.M + q;
        const C* ph = sPh + slot * PHS;
        const C th1 = ph[3 * N], th2 = ph[3 * N + 1], th3 = ph[3 * N + 2];
        const C phn = pq + 1 < npq ? phase_fetch(pq + 1) : mk<C>(0.f, 0.f);
        // pass 1: R lines (k1, k2) along k3 | Nyquist first axes.
        // m = Re((E + E t)(1 - i)) / 2 with E = E1 E2 E3[k3] and t the
        // Nyquist factor (1 off the planes): per line A = (E12 + E12 t12)
        // (1 - i) / 2 (A3 on the k3 = N/2 plane), then m = Re(A E3[k3]).
        if (is_main && !IL1) {
#pragma unroll 1
          for (int r = 0; r < 2; ++r) {
            const int L = tid + r * NM, k1 = L / N, k2 = L % N;
            const C E12 = cmul(ph[k1], ph[N + k2]);
            C t12 = mk<C>(1.f, 0.f);
            if (k1 == NY) t12 = th1;
            if (k2 == NY) t12 = cmul(t12, th2);
            const C E12t = cmul(E12, t12);
            const C s0 = cadd(E12, E12t), s3 = cadd(E12, cmul(E12t, th3));
            const C A = mk<C>(0.5f * (s0.x + s0.y), 0.5f * (s0.y - s0.x));
            const C A3 = mk<C>(0.5f * (s3.x + s3.y), 0.5f * (s3.y - s3.x));
            C x[N];
#pragma unroll
            for (int k = 0; k < N; ++k) {
              const C e3 = ph[2 * N + k];
              const C& Ak = k == NY ? A3 : A;
              x[k] = cscale(Fat(k1, k2, k), Ak.x * e3.x - Ak.y * e3.y);
            }
            fft<float, N, +1>(x);
#pragma unroll
            for (int k = 0; k < N; ++k) sW[L * LP + k] = x[k];
          }
        } else if (is_main) {  // IL1: both lines of the thread at once
          auto coef = [&](int k1, int k2, C& A, C& A3) {
            const C E12 = cmul(ph[k1], ph[N + k2]);
            C t12 = mk<C>(1.f, 0.f);
            if (k1 == NY) t12 = th1;
            if (k2 == NY) t12 = cmul(t12, th2);
            const C E12t = cmul(E12, t12);
            const C s0 = cadd(E12, E12t), s3 = cadd(E12, cmul(E12t, th3));
            A = mk<C>(0.5f * (s0.x + s0.y), 0.5f * (s0.y - s0.x));
            A3 = mk<C>(0.5f * (s3.x + s3.y), 0.5f * (s3.y - s3.x));
          };
          const int L0 = tid, L1 = tid + NM;
          const int a1 = L0 / N, a2 = L0 % N, b1 = L1 / N, b2 = L1 % N;
          C Aa, Aa3, Ab, Ab3;
          coef(a1, a2, Aa, Aa3);
          coef(b1, b2, Ab, Ab3);
          C x[N], y[N];
#pragma unroll
          for (int k = 0; k < N; ++k) {
            const C e3 = ph[2 * N + k];
            const C& A0 = k == NY ? Aa3 : Aa;
            const C& B0 = k == NY ? Ab3 : Ab;
            x[k] = cscale(Fat(a1, a2, k), A0.x * e3.x - A0.y * e3.y);
            y[k] = cscale(Fat(b1, b2, k), B0.x * e3.x - B0.y * e3.y);
          }
          fft<float, N, +1>(x);
          fft<float, N, +1>(y);
#pragma unroll
          for (int k = 0; k < N; ++k) {
            sW[L0 * LP + k] = x[k];
            sW[L1 * LP + k] = y[k];
          }
        } else {
          // n F on the Nyquist planes: plane 1 (k1 = N/2) lines over k3,
          // plane 2 (k2 = N/2, k1 != N/2) lines over k3, plane 3 (k3 = N/2,
          // k1, k2 != N/2) lines over k2.  On a line only the phase of the
          // running axis changes, so n = Re(D (1 - i)) / 2 with
          // D = E (1 - t) becomes n = Re(A e[k]) with one coefficient A per
          // line (A3 where k meets the Nyquist index of the running axis),
          // as for the main lines.  Addresses and conjugation are selects,
          // so lines of different planes share a warp without divergence.
#pragma unroll 1
          for (int line = tq; line < 3 * N; line += G::NQ) {
            const int which = line / N, j = line % N;
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
            C B = cmul(Eb, mk<C>(1.f - tb.x, -tb.y));
            const C tb3 = cmul(tb, th3);
            C B3 = p3 ? mk<C>(0.f, 0.f) : cmul(Eb, mk<C>(1.f - tb3.x, -tb3.y));
            if (which != 0 && j == NY) B = B3 = mk<C>(0.f, 0.f);
            const C A = mk<C>(0.5f * (B.x + B.y), 0.5f * (B.y - B.x));
            const C A3 = mk<C>(0.5f * (B3.x + B3.y), 0.5f * (B3.y - B3.x));
            const C* ev = ph + (p3 ? N : 2 * N);
            // element k at lo + k sl (k <= N/2, or every k on plane 3), else
            // conj(sF[hi - k]) (the mirrored point)
            const int jm = (N - j) % N;
            const int lo = which == 0 ? NY * FS + j * H : (which == 1 ? j * FS + NY * H : j * FS + NY);
            const int sl = p3 ? H : 1;
            const int hi = (which == 0 ? NY * FS + jm * H : jm * FS + NY * H) + N;
            C x[N];
#pragma unroll
            for (int k = 0; k < N; ++k) {
              C v;
              if (k <= NY) {
                v = sF[lo + k * sl];
              } else {
                const C c = sF[p3 ? lo + k * H : hi - k];
                v = mk<C>(c.x, p3 ? c.y : -c.y);
              }
              const C& Ak = k == NY ? A3 : A;
              const C e = ev[k];
              x[k] = cscale(v, Ak.x * e.x - Ak.y * e.y);
            }
            fft<float, N, +1>(x);
            C* T = which == 0 ? sT1 : (which == 1 ? sT2 : sT3);
#pragma unroll
            for (int k = 0; k < N; ++k) T[j * LP + k] = x[k];
          }
        }
        if (pq + 1 < npq) phase_store(phn, slot ^ 1);
        __syncthreads();
        // pass 2: lines (k1, x3) along k2, both lines of a thread at once |
        // Nyquist second axes (columns)
        if (is_main) {
          const int L0 = tid, L1 = tid + NM;
          C* w0 = sW + (L0 / N) * N * LP + L0 % N;
          C* w1 = sW + (L1 / N) * N * LP + L1 % N;
          C x[N], y[N];
#pragma unroll
          for (int j = 0; j < N; ++j) {
            x[j] = w0[j * LP];
            y[j] = w1[j * LP];
          }
          fft<float, N, +1>(x);
          fft<float, N, +1>(y);
#pragma unroll
          for (int j = 0; j < N; ++j) {
            w0[j * LP] = x[j];
            w1[j * LP] = y[j];
          }
        } else {
#pragma unroll 1
          for (int line = tq; line < 3 * N; line += G::NQ) {
            const int which = line / N, col = line % N;
            C* T = which == 0 ? sT1 : (which == 1 ? sT2 : sT3);
            C x[N];
#pragma unroll
            for (int j = 0; j < N; ++j) x[j] = T[j * LP + col];
            fft<float, N, +1>(x);
#pragma unroll
            for (int j = 0; j < N; ++j) T[j * LP + col] = x[j];
          }
        }
        __syncthreads();
        // pass 3: lines (x2, x3) along k1, both lines at once;
        // S += Re R^2 + Re Nq^2
        if (is_main) {
          const int L0 = tid, L1 = tid + NM;
          const int a2 = L0 / N, a3 = L0 % N, b2 = L1 / N, b3 = L1 % N;
          C x[N], y[N];
#pragma unroll
          for (int i = 0; i < N; ++i) {
            x[i] = sW[(i * N + a2) * LP + a3];
            y[i] = sW[(i * N + b2) * LP + b3];
          }
          fft<float, N, +1>(x);
          fft<float, N, +1>(y);
          const C ta = sT1[a2 * LP + a3], tb = sT1[b2 * LP + b3];
          const float sa2 = (a2 & 1) ? -1.f : 1.f, sa3 = (a3 & 1) ? -1.f : 1.f;
          const float sb2 = (b2 & 1) ? -1.f : 1.f, sb3 = (b3 & 1) ? -1.f : 1.f;
#pragma unroll
          for (int i = 0; i < N; ++i) {
            const float s1 = (i & 1) ? -1.f : 1.f;
            {
              const C t2 = sT2[i * LP + a3], t3 = sT3[i * LP + a2];
              const float nr = s1 * ta.x + sa2 * t2.x + sa3 * t3.x;
              const float ni = s1 * ta.y + sa2 * t2.y + sa3 * t3.y;
              S0[i] += x[i].x * x[i].x - x[i].y * x[i].y + nr * nr - ni * ni;
            }
            {
              const C t2 = sT2[i * LP + b3], t3 = sT3[i * LP + b2];
              const float nr = s1 * tb.x + sb2 * t2.x + sb3 * t3.x;
              const float ni = s1 * tb.y + sb2 * t2.y + sb3 * t3.y;
              S1[i] += y[i].x * y[i].x - y[i].y * y[i].y + nr * nr - ni * ni;
            }
          }
        }
        slot ^= 1;
        __syncthreads();
      }

      // FFT(S_p): lines (x2, x3) along x1 straight from the accumulators
      if (is_main) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int L = tid + r * NM, x2 = L / N, x3 = L % N;
          C x[N];
#pragma unroll
          for (int i = 0; i < N; ++i) x[i] = mk<C>(r == 0 ? S0[i] : S1[i], 0.f);
          fft<float, N, -1>(x);
#pragma unroll
          for (int i = 0; i < N; ++i) sW[(i * N + x2) * LP + x3] = x[i];
        }
      }
      __syncthreads();
      if (is_main) {
#pragma unroll 1
        for (int r = 0; r < 2; ++r) {
          const int L = tid + r * NM, k1 = L / N, x3 = L % N;
          C x[N];
#pragma unroll
          for (int j = 0; j < N; ++j) x[j] = sW[(k1 * N + j) * LP + x3];
          fft<float, N, -1>(x);
#pragma unroll
          for (int j = 0; j < N; ++j) sW[(k1 * N + j) * LP + x3] = x[j];
        }
      }
      __syncthreads();
      if (is_main) {
        const float* w1 = a.w1t + (size_t)p * V;
#pragma unroll 1
        for (int r = 0; r < 2; ++r) {
          const int L = tid + r * NM;  // line (k1, k2) along k3
          // fC and w1 with the last axis outermost ([k3][L]): a warp's
          // accesses are 32 consecutive entries.  All loads of the line are
          // issued before its first store (fC and w1 could alias as far as
          // the compiler knows, which would otherwise order each load after
          // the previous store): one round trip per line, not one per entry.
          C x[N];
#pragma unroll
          for (int k = 0; k < N; ++k) x[k] = sW[L * LP + k];
          fft<float, N, -1>(x);
#pragma unroll
          for (int k = 0; k < N; ++k) x[k] = cscale(x[k], w1[k * NN + L]);
          C* const fca = s_kp == 1 ? fcg : a.fcp + (size_t)item * V;
          if (p > s_it[0]) {
            C acc[N];
#pragma unroll
            for (int k = 0; k < N; ++k) acc[k] = fca[k * NN + L];
#pragma unroll
            for (int k = 0; k < N; ++k) fca[k * NN + L] = cadd(acc[k], x[k]);
          } else {
#pragma unroll
            for (int k = 0; k < N; ++k) fca[k * NN + L] = x[k];
          }
        }
      }
      __syncthreads();
    }

    if (s_kp > 1) {
      // publish this chunk's slice; the point's last chunk goes on
      __threadfence();
      __syncthreads();
      if (tid == 0) s_last = atomicAdd(a.pdone + item / s_kp, 1) == s_kp - 1;
      __syncthreads();
      if (!s_last) continue;  // uniform over the CTA
      __threadfence();
    }

    // ---- Q = prefac (Re IFFT(fC) - f IFFT(b2 F)) ----------------------------
    // Two transforms: fC, summed from FP32 transforms of real fields, is
    // conjugate-even only to round-off, and packing it with b2 F into one
    // transform would leak that round-off into the loss term as a constant
    // times f (a momentum error proportional to rho u).
    auto pass23 = [&]() {  // the pass along k2, in place, between barriers
      __syncthreads();
      if (is_main) {
#pragma unroll 1
        for (int r = 0; r < 2; ++r) {
          const int L = tid + r * NM;
          C* w = sW + (L / N) * N * LP + L % N;
          C x[N];
#pragma unroll
          for (int j = 0; j < N; ++j) x[j] = w[j * LP];
          fft<float, N, +1>(x);
#pragma unroll
          for (int j = 0; j < N; ++j) w[j * LP] = x[j];
        }
      }
      __syncthreads();
    };
    // Lf = IFFT(b2 F): b2 F is built conjugate-even from the half spectrum.
    // F is not needed after this transform's first pass, so its storage
    // takes the real Lf values (slot v of each thread's own lines).
    float* const sLf = reinterpret_cast<float*>(sF);
    static_assert(2 * N * FS >= V, "Lf fits in the spectrum storage");
    if (is_main) {
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        const int L = tid + r * NM, k1 = L / N, k2 = L % N;
        C x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = cscale(Fat(k1, k2, k), a.b2t[k * NN + L]);
        fft<float, N, +1>(x);
#pragma unroll
        for (int k = 0; k < N; ++k) sW[L * LP + k] = x[k];
      }
    }
    pass23();
    if (is_main) {
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        const int L = tid + r * NM, x2 = L / N, x3 = L % N;
        C x[N];
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] = sW[(i * N + x2) * LP + x3];
        fft<float, N, +1>(x);
#pragma unroll
        for (int i = 0; i < N; ++i) sLf[(i * N + x2) * N + x3] = x[i].x;
      }
    }
    __syncthreads();
    // QG = Re IFFT(fC)
    if (is_main) {
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        const int L = tid + r * NM;
        C x[N];
        if (s_kp == 1) {
#pragma unroll
          for (int k = 0; k < N; ++k) x[k] = fcg[k * NN + L];
        } else {
          // the chunks' slices, summed in a fixed order (L2 reads: other
          // CTAs wrote them)
#pragma unroll
          for (int k = 0; k < N; ++k) x[k] = mk<C>(0.f, 0.f);
#pragma unroll 1
          const int kp = s_kp, i0 = item - item % kp;
          for (int c = 0; c < kp; ++c) {
            const C* src = a.fcp + (size_t)(i0 + c) * V + L;
#pragma unroll
            for (int k = 0; k < N; ++k) x[k] = cadd(x[k], __ldcg(src + k * NN));
          }
        }
        fft<float, N, +1>(x);
#pragma unroll
        for (int k = 0; k < N; ++k) sW[L * LP + k] = x[k];
      }
    }
    pass23();
    double mom[5] = {0, 0, 0, 0, 0};
    if (is_main) {
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        const int L = tid + r * NM, x2 = L / N, x3 = L % N;
        // bank entry of v = i N^2 + L is b0 + i st (v enters the AoSoA
        // index linearly); f of this line is loaded first, every load
        // issued before the first store of Q (which may alias f as far as
        // the compiler knows)
        const int64_t b0 = soa_ix(s_it[2], a.ldim, s_it[3], L, V, a.soasz), st = (int64_t)NN * a.soasz;
        C x[N];
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] = sW[(i * N + x2) * LP + x3];
        fft<float, N, +1>(x);
        float fl[N];
#pragma unroll
        for (int i = 0; i < N; ++i) fl[i] = a.f[b0 + i * st];
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const int64_t v = (int64_t)(i * N + x2) * N + x3;
          const float qq = a.prefac * (x[i].x - fl[i] * sLf[v]);
          if (!a.project) {
            a.Q[b0 + i * st] = qq;
            continue;
          }
          sW[(i * N + x2) * LP + x3].x = qq;  // this thread's own slot
          {
            const double c0 = a.cvec[v], c1 = a.cvec[V + v], c2 = a.cvec[2 * V + v];
            const double d = (double)qq;
            mom[0] += d;
            mom[1] += d * c0;
            mom[2] += d * c1;
            mom[3] += d * c2;
            mom[4] += d * (c0 * c0 + c1 * c1 + c2 * c2);
          }
        }
      }
    }
    if (a.project) {  // uniform: every thread takes part in the reduction
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        double s = mom[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((tid & 31) == 0) sRed[k][tid >> 5] = s;
      }
      __syncthreads();
      if (tid < 5) {
        double s = 0;
        for (int w = 0; w < NT / 32; ++w) s += sRed[tid][w];
        sRed[tid][0] = s;
      }
      __syncthreads();
      if (tid < 5) {
        double l = 0;
        for (int j = 0; j < 5; ++j) l += a.ginv[tid * 5 + j] * sRed[j][0];
        sLam[tid] = l;
      }
      __syncthreads();
    }
    if (is_main && a.project) {
#pragma unroll 1
      for (int r = 0; r < 2; ++r) {
        const int L = tid + r * NM, x2 = L / N, x3 = L % N;
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const int64_t v = (int64_t)(i * N + x2) * N + x3;
          const double c0 = a.cvec[v], c1 = a.cvec[V + v], c2 = a.cvec[2 * V + v];
          const float qq = (float)((double)sW[(i * N + x2) * LP + x3].x -
                                   (sLam[0] + sLam[1] * c0 + sLam[2] * c1 + sLam[3] * c2 +
                                    sLam[4] * (c0 * c0 + c1 * c1 + c2 * c2)));
          a.Q[soa_ix(s_it[2], a.ldim, s_it[3], v, V, a.soasz)] = qq;
        }
      }
    }
    if (s_kp > 1 && tid == 0) a.pdone[item / s_kp] = 0;  // every chunk has counted: ready for the next launch
    __syncthreads();  // the work cube and fC are reused by the next point
  }
}

}  // namespace dgfs
