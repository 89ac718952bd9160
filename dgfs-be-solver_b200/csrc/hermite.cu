// Hermite embedding and reconstruction of distributions for the learned
// collision surrogate (no counterpart in the reference).
//
// Local frame of a point: rho, u, T from the FP64 moments of f (the formulas
// of frfs/plugins/dgfsmomwriterstd.py:154-190), c^ = (c - u)/sqrt(T).
// Basis: phi_n(x) = He_n(sqrt(2) x)/sqrt(n!) (probabilists' Hermite),
// orthonormal for the weight e^{-x^2}/sqrt(pi); in 3D
// phi_ijk(c^) = phi_i phi_j phi_k, weight W(c^) = pi^{-3/2} e^{-|c^|^2}, and a
// Maxwellian is rho T^{-3/2} W(c^).  Modes: total degree i+j+k <= 9
// (220 modes, ordered by degree, then i, then j, both descending).
//
//   window      chi(c^) = erfc((|c^| - 4) / 0.4) / 2: the degree-9
//               polynomials reach 1e4..1e6 at the corners of the velocity
//               box, where f and Q hold only round-off; the window keeps that
//               noise out of the coefficients
//   embedding   a_k = (1/rho) cw sum_v chi (f - M)(c_v) phi_k(c^_v), M the
//               local Maxwellian rho T^{-3/2} W(c^) (zero for a Maxwellian
//               up to round-off, whatever the window)
//   target      b_k = cw sum_v chi g(c_v) phi_k(c^_v) / (prefac rho^2 T^{gamma/2})
//               with g = Q, or, given the collision frequency nu (Q = G -
//               nu f), the gain deviation g = G - nu M = Q + nu (f - M), M
//               the local Maxwellian: smooth even where f jumps (diffuse
//               walls), and O(f - M) near equilibrium
//   reconstruct g(c) = prefac rho^2 T^{gamma/2} T^{-3/2} W(c^) sum_k d_k phi_k(c^),
//               d = Gw^{-1} b with Gw_kl = int chi W phi_k phi_l dc^ (the
//               windowed Gram matrix, condition number 1.75, passed in);
//               Q = g, or Q = g - nu (f - M) given nu; then the FP64
//               least-squares projection onto zero mass, momentum and
//               energy moments.
// The velocity grid is a tensor product, so every sum factorises into three
// 1D contractions.  One CTA per solution point.
#include <cmath>
#include <cuda_runtime.h>

#include "../../include/dgfs_b200.h"
#include "dgfs_common.cuh"
#include "dgfs_internal.h"

namespace {

constexpr int kDeg = 9;
constexpr int kP = kDeg + 1;       // 1D polynomials per axis
constexpr int kModes = 220;        // (i, j, k) with i + j + k <= 9
constexpr int kFeat = 256;         // feature vector width
constexpr int kThreads = 256;
constexpr int kMaxN = 32;
constexpr double kWinR = 4.0;      // window centre |c^|
constexpr double kWinW = 0.4;      // window width
// with a workspace, reconstruction splits every point's velocity range into
// kRelaxSplit chunks (partial moments per chunk, then one correction pass)
constexpr int kRelaxSplit = 32;  // chunks of a relaxation-only (gate 2) point
constexpr int kNetSplit = 8;     // chunks of a network (gate 1) point
constexpr int kRelaxWarps = 8;

__constant__ unsigned char c_mi[kModes], c_mj[kModes], c_mk[kModes];
// index of mode (i, j, k) in the 220-vector, -1 if degree > 9
__constant__ short c_midx[kP][kP][kP];

struct FrameArgs {
  int N, nupts, neles;
  long long ldim;
  double L, cw, prefac, gamma;
};

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0;
  for (int w = 0; w < kThreads / 32; ++w) s += red[w];
  return s;
}

// rho, u, T of the point's distribution (one pass, FP64):
// T = (2/3) (sum f |c|^2 / sum f - |u|^2); the cancellation costs
// |u|^2/T ulps, far below the FP32 bank's own rounding
template <typename T>
__device__ void point_frame(const T* f, int upt, int e, const FrameArgs& a, double* red, double* mom) {
  const int N = a.N;
  const long long V = (long long)N * N * N;
  const double h = 2.0 * a.L / N, c00 = -a.L + a.L / N;
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
  const long long b0 = dgfs::soa_ix(upt, a.ldim, e, 0, V, 32);
  // rows (I, J) along K, as project_modes reads them
  for (int r = threadIdx.x; r < N * N; r += kThreads) {
    const double cx = c00 + (r / N) * h, cy = c00 + (r % N) * h;
    double t0 = 0, tz = 0, tzz = 0;
#pragma unroll 4
    for (int K = 0; K < N; ++K) {
      const double fv = (double)f[b0 + ((long long)r * N + K) * 32];
      const double cz = c00 + K * h;
      t0 += fv;
      tz += fv * cz;
      tzz += fv * cz * cz;
    }
    s0 += t0;
    s1 += t0 * cx;
    s2 += t0 * cy;
    s3 += tz;
    s4 += t0 * (cx * cx + cy * cy) + tzz;
  }
  const double m0 = block_sum(s0, red), m1 = block_sum(s1, red), m2 = block_sum(s2, red),
               m3 = block_sum(s3, red), m4 = block_sum(s4, red);
  const double rho = m0 * a.cw, ux = m1 / m0, uy = m2 / m0, uz = m3 / m0;
  mom[0] = rho;
  mom[1] = ux;
  mom[2] = uy;
  mom[3] = uz;
  mom[4] = (m4 / m0 - (ux * ux + uy * uy + uz * uz)) * (2.0 / 3.0);
}

// H[ax][I][n] = phi_n((c0_I - u_ax)/sqrt(T)) for the three axes, and
// Ex[ax][I] = exp(-((c0_I - u_ax)/sqrt(T))^2): the Gaussian of the frame
// factorises over the axes, so e^{-|c^|^2} = Ex[0][I] Ex[1][J] Ex[2][K]
__device__ void basis_tables(const FrameArgs& a, const double* mom, double (*H)[kMaxN][kP],
                             double (*Ex)[kMaxN]) {
  const int N = a.N;
  const double h = 2.0 * a.L / N, c00 = -a.L + a.L / N, rt = rsqrt(mom[4]);
  for (int t = threadIdx.x; t < 3 * N; t += kThreads) {
    const int ax = t / N, I = t % N;
    const double d = (c00 + I * h - mom[1 + ax]) * rt;
    Ex[ax][I] = exp(-d * d);
    const double y = 1.4142135623730950488 * d;
    double p0 = 1.0, p1 = y;
    H[ax][I][0] = p0;
    H[ax][I][1] = p1;
    for (int n = 1; n < kDeg; ++n) {
      // phi_{n+1} = (y phi_n - sqrt(n) phi_{n-1}) / sqrt(n+1)
      const double p2 = (y * p1 - sqrt((double)n) * p0) * rsqrt((double)(n + 1));
      H[ax][I][n + 1] = p2;
      p0 = p1;
      p1 = p2;
    }
  }
}

// Fields projected by project_modes: a bank value, or the gain deviation
// G - nu M = Q + nu (f - M) of a collision bank Q given the collision
// frequency nu and the local Maxwellian M (value Mv at the node).
template <typename T> struct BankField {
  const T* g;
  __device__ double operator()(long long ix, double) const { return (double)g[ix]; }
};
template <typename T> struct DevField {  // f - M
  const T* f;
  __device__ double operator()(long long ix, double Mv) const { return (double)f[ix] - Mv; }
};
template <typename T> struct GainDevField {
  const T *q, *nu, *f;
  __device__ double operator()(long long ix, double Mv) const {
    return (double)q[ix] + (double)nu[ix] * ((double)f[ix] - Mv);
  }
};

// out[m] = cw sum_v chi g(c_v) phi_m(c^_v) for the 220 modes
// The window chi is evaluated in FP32 (erfcf): it only shapes the
// projection, and the coefficients leave in FP32.
template <typename Field>
__device__ void project_modes(const Field& g, int upt, int e, const FrameArgs& a, const double* mom,
                              double (*H)[kMaxN][kP], double (*Ex)[kMaxN], double* t1, double* t2,
                              double* out) {
  const int N = a.N;
  const long long V = (long long)N * N * N;
  const double h = 2.0 * a.L / N, c00 = -a.L + a.L / N, rt = rsqrt(mom[4]);
  // local Maxwellian rho T^{-3/2} pi^{-3/2} e^{-|c^|^2}
  const double m0 = mom[0] * rt * rt * rt * 0.17958712212516656;
  // t1[I][J][k] = sum_K chi g[I][J][K] Hz[K][k]
  for (int r = threadIdx.x; r < N * N; r += kThreads) {
    double acc[kP];
#pragma unroll
    for (int k = 0; k < kP; ++k) acc[k] = 0;
    const int I = r / N, J = r % N;
    const double dx = (c00 + I * h - mom[1]) * rt, dy = (c00 + J * h - mom[2]) * rt;
    const double r2xy = dx * dx + dy * dy, mxy = m0 * Ex[0][I] * Ex[1][J];
    const long long b0 = dgfs::soa_ix(upt, a.ldim, e, (long long)r * N, V, 32);
    for (int K = 0; K < N; ++K) {
      const double dz = (c00 + K * h - mom[3]) * rt;
      const float r2 = (float)(r2xy + dz * dz);
      const double chi = 0.5f * erfcf((sqrtf(r2) - (float)kWinR) * (float)(1.0 / kWinW));
      const double gv = chi * g(b0 + (long long)K * 32, mxy * Ex[2][K]);
#pragma unroll
      for (int k = 0; k < kP; ++k) acc[k] += gv * H[2][K][k];
    }
#pragma unroll
    for (int k = 0; k < kP; ++k) t1[r * kP + k] = acc[k];
  }
  __syncthreads();
  // t2[I][j][k] = sum_J t1[I][J][k] Hy[J][j]   (j + k <= 9)
  for (int t = threadIdx.x; t < N * kP * kP; t += kThreads) {
    const int I = t / (kP * kP), j = (t / kP) % kP, k = t % kP;
    if (j + k > kDeg) continue;
    double s = 0;
    for (int J = 0; J < N; ++J) s += t1[(I * N + J) * kP + k] * H[1][J][j];
    t2[(I * kP + j) * kP + k] = s;
  }
  __syncthreads();
  // out[i][j][k] = cw sum_I t2[I][j][k] Hx[I][i]
  for (int m = threadIdx.x; m < kModes; m += kThreads) {
    const int i = c_mi[m], j = c_mj[m], k = c_mk[m];
    double s = 0;
    for (int I = 0; I < N; ++I) s += t2[(I * kP + j) * kP + k] * H[0][I][i];
    out[m] = s * a.cw;
  }
  __syncthreads();
}

// Features X[pt][256] (a_k of f - M, then sqrt(T)/L and u/L), frame
// mom[pt][5], non-equilibrium measure eps[pt] = |a_k, degree >= 2|, and
// optionally the targets B[pt][256] of a collision bank Q.
template <typename T>
__global__ void __launch_bounds__(kThreads) embed_kernel(const T* __restrict__ f, const T* __restrict__ Q,
                                                         const T* __restrict__ nu,
                                                         FrameArgs a, float* __restrict__ X,
                                                         float* __restrict__ B, double* __restrict__ mom_out,
                                                         float* __restrict__ eps) {
  extern __shared__ double sm[];
  __shared__ double red[kThreads / 32];
  __shared__ double mom[5];
  __shared__ double H[3][kMaxN][kP];
  __shared__ double Ex[3][kMaxN];
  __shared__ double coef[kModes];
  const int N = a.N;
  double* t1 = sm;                    // [N*N][kP]
  double* t2 = sm + N * N * kP;       // [N][kP][kP]
  const int pt = blockIdx.x, upt = pt / a.neles, e = pt % a.neles;

  double m[5];
  point_frame<T>(f, upt, e, a, red, m);
  if (threadIdx.x < 5) mom[threadIdx.x] = m[threadIdx.x];
  __syncthreads();
  basis_tables(a, mom, H, Ex);
  __syncthreads();

  project_modes(DevField<T>{f}, upt, e, a, mom, H, Ex, t1, t2, coef);
  const double rho = mom[0];
  double ne = 0;
  for (int k = threadIdx.x; k < kFeat; k += kThreads) {
    float x = 0.f;
    if (k < kModes) {
      x = (float)(coef[k] / rho);
      if (c_mi[k] + c_mj[k] + c_mk[k] >= 2) ne += (coef[k] / rho) * (coef[k] / rho);
    } else if (k == kModes) {
      x = (float)(sqrt(mom[4]) / a.L);
    } else if (k < kModes + 4) {
      x = (float)(mom[k - kModes] / a.L);
    }
    X[(long long)pt * kFeat + k] = x;
  }
  ne = block_sum(ne, red);
  if (threadIdx.x == 0) {
    eps[pt] = (float)sqrt(ne);
    for (int k = 0; k < 5; ++k) mom_out[(long long)pt * 5 + k] = mom[k];
  }
  if (Q) {
    if (nu)
      project_modes(GainDevField<T>{Q, nu, f}, upt, e, a, mom, H, Ex, t1, t2, coef);
    else
      project_modes(BankField<T>{Q}, upt, e, a, mom, H, Ex, t1, t2, coef);
    const double s = 1.0 / (a.prefac * rho * rho * pow(mom[4], 0.5 * a.gamma));
    for (int k = threadIdx.x; k < kFeat; k += kThreads)
      B[(long long)pt * kFeat + k] = k < kModes ? (float)(coef[k] * s) : 0.f;
  }
}

// Q at the gated points from predicted coefficients Bp[pt][256]:
// reconstruction, FP64 projection onto zero mass/momentum/energy, store.
// gate[pt] != 0 selects the points written; others are left untouched.
// With part (workspace): one CTA per (point, chunk of the velocity range),
// gate-2 points left to relax_pass1_kernel; each CTA stores Q on its chunk
// and its partial moments, and relax_pass2_kernel applies the projection.
template <typename T>
__global__ void __launch_bounds__(kThreads) reconstruct_kernel(const float* __restrict__ Bp,
                                                               const double* __restrict__ mom_in,
                                                               const int* __restrict__ gate, FrameArgs a,
                                                               const double* __restrict__ ginv,
                                                               const double* __restrict__ gwinv,
                                                               const T* __restrict__ f,
                                                               const T* __restrict__ nu,
                                                               T* __restrict__ Q, double* __restrict__ part,
                                                               const int* __restrict__ rows,
                                                               const int* __restrict__ nrows,
                                                               const double* __restrict__ dcoef) {
  extern __shared__ double sm[];
  __shared__ double red[kThreads / 32];
  __shared__ double H[3][kMaxN][kP];
  __shared__ double Ex[3][kMaxN];
  __shared__ double bw[kModes];
  __shared__ double b[kModes];
  __shared__ double mom[5];
  // split mode (part): CTA = (entry r of the gate-1 list, chunk); the
  // active CTAs are the first *nrows * kNetSplit, dispatched first
  const int vs = part ? kNetSplit : 1;
  const int r = blockIdx.x / vs, chunk = blockIdx.x % vs;
  if (part && r >= *nrows) return;  // uniform over the CTA
  const int pt = part ? rows[r] : r;
  if (gate && !gate[pt]) return;
  const int N = a.N, upt = pt / a.neles, e = pt % a.neles;
  const int V = N * N * N;
  const int v0 = chunk * V / vs, v1 = (chunk + 1) * V / vs;
  double* r1 = sm;                    // [kP][kP][N]   (i, j, K)
  double* r2 = sm + kP * kP * N;      // [kP][N][N]    (i, J, K)
  if (threadIdx.x < 5) mom[threadIdx.x] = mom_in[(long long)pt * 5 + threadIdx.x];
  // relaxation only (G - nu M = 0): no modal part to evaluate
  const bool zero = gate && gate[pt] == 2;
  if (!zero && part) {
    // expansion coefficients computed once per point (coef_kernel)
    for (int k = threadIdx.x; k < kModes; k += kThreads) b[k] = dcoef[(long long)r * kModes + k];
  } else if (!zero) {
    for (int k = threadIdx.x; k < kModes; k += kThreads) bw[k] = (double)Bp[(long long)pt * kFeat + k];
    __syncthreads();
    // d = Gw^{-1} b (windowed coefficients to expansion coefficients): one
    // warp per row, lanes over the columns (coalesced rows of Gw^{-1}),
    // butterfly sum in a fixed order
    const int lane = threadIdx.x & 31;
    for (int k = threadIdx.x >> 5; k < kModes; k += kThreads / 32) {
      double s = 0;
      if (gwinv) {
        for (int l = lane; l < kModes; l += 32) s += gwinv[k * kModes + l] * bw[l];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      } else {
        s = bw[k];
      }
      if (lane == 0) b[k] = s;
    }
  }
  __syncthreads();
  basis_tables(a, mom, H, Ex);
  __syncthreads();
  if (!zero) {
    // r1[i][j][K] = sum_k b[i][j][k] Hz[K][k]
    for (int t = threadIdx.x; t < kP * kP * N; t += kThreads) {
      const int i = t / (kP * N), j = (t / N) % kP, K = t % N;
      double s = 0;
      if (i + j <= kDeg)
        for (int k = 0; k + i + j <= kDeg; ++k) s += b[c_midx[i][j][k]] * H[2][K][k];
      r1[t] = s;
    }
    __syncthreads();
    // r2[i][J][K] = sum_j r1[i][j][K] Hy[J][j]
    for (int t = threadIdx.x; t < kP * N * N; t += kThreads) {
      const int i = t / (N * N), J = (t / N) % N, K = t % N;
      double s = 0;
      for (int j = 0; j + i <= kDeg; ++j) s += r1[(i * kP + j) * N + K] * H[1][J][j];
      r2[t] = s;
    }
    __syncthreads();
  }
  const double rho = mom[0], Tt = mom[4];
  // pi^{-3/2}
  const double scale = a.prefac * rho * rho * pow(Tt, 0.5 * a.gamma) * pow(Tt, -1.5) * 0.17958712212516656;
  const double h = 2.0 * a.L / N, c00 = -a.L + a.L / N, rt = rsqrt(Tt);
  const double mscale = rho * rt * rt * rt * 0.17958712212516656;  // local Maxwellian
  // Q(c) = scale e^{-|c^|^2} sum_i r2[i][J][K] Hx[I][i]; moments for the projection
  double mm[5] = {0, 0, 0, 0, 0};
  for (int v = v0 + threadIdx.x; v < v1; v += kThreads) {
    const int I = v / (N * N), J = (v / N) % N, K = v % N;
    double s = 0;
    if (!zero)
      for (int i = 0; i < kP; ++i) s += r2[(i * N + J) * N + K] * H[0][I][i];
    const double cx = c00 + I * h, cy = c00 + J * h, cz = c00 + K * h;
    const double ex = Ex[0][I] * Ex[1][J] * Ex[2][K];
    const long long ix = dgfs::soa_ix(upt, a.ldim, e, v, V, 32);
    double q = scale * ex * s;
    if (nu) q -= (double)nu[ix] * ((double)f[ix] - mscale * ex);  // Q = dG - nu (f - M)
    Q[ix] = (T)q;
    mm[0] += q;
    mm[1] += q * cx;
    mm[2] += q * cy;
    mm[3] += q * cz;
    mm[4] += q * (cx * cx + cy * cy + cz * cz);
  }
  if (part) {
    // partial moments of this chunk (layout shared with the relaxation
    // kernels: the point's slot in its AoSoA block)
    const long long slot = ((long long)upt * ((a.neles + 31) / 32) * 32 + e) * kRelaxSplit + chunk;  // chunk < kNetSplit
    for (int k = 0; k < 5; ++k) {
      const double t = block_sum(mm[k], red);
      if (threadIdx.x == 0) part[slot * 5 + k] = t;
    }
    return;
  }
  double lam[5];
  {
    double mt[5];
    for (int k = 0; k < 5; ++k) mt[k] = block_sum(mm[k], red);
    for (int k = 0; k < 5; ++k) {
      double s = 0;
      for (int j = 0; j < 5; ++j) s += ginv[k * 5 + j] * mt[j];
      lam[k] = s;
    }
  }
  // each thread corrects the values it stored itself
  for (int v = threadIdx.x; v < V; v += kThreads) {
    const int I = v / (N * N), J = (v / N) % N, K = v % N;
    const double cx = c00 + I * h, cy = c00 + J * h, cz = c00 + K * h;
    const long long ix = dgfs::soa_ix(upt, a.ldim, e, v, V, 32);
    Q[ix] = (T)((double)Q[ix] -
                (lam[0] + lam[1] * cx + lam[2] * cy + lam[3] * cz + lam[4] * (cx * cx + cy * cy + cz * cz)));
  }
}

// Expansion coefficients of the gate-1 list, once per point: d = Gw^{-1} b.
// Gw^{-1} is symmetric, so thread k reads column k of row l (coalesced over
// k); each warp takes a range of l, and the warps' partial sums are added
// in a fixed order.
__global__ void __launch_bounds__(kThreads) coef_kernel(const int* __restrict__ rows, const int* __restrict__ nrows,
                                                       const float* __restrict__ Bp,
                                                       const double* __restrict__ gwinv,
                                                       double* __restrict__ dcoef) {
  constexpr int W = kThreads / 32, PER = (kModes + 31) / 32;
  __shared__ double bw[kModes];
  __shared__ double acc[W][kModes];
  const int r = blockIdx.x;
  if (r >= *nrows) return;
  const int pt = rows[r], w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = threadIdx.x; k < kModes; k += kThreads) bw[k] = (double)Bp[(long long)pt * kFeat + k];
  __syncthreads();
  double s[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) s[j] = 0.0;
  for (int l = w; l < kModes; l += W) {
    const double bl = bw[l];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int k = lane + 32 * j;
      if (k < kModes) s[j] += (gwinv ? gwinv[l * kModes + k] : (double)(l == k)) * bl;
    }
  }
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int k = lane + 32 * j;
    if (k < kModes) acc[w][k] = s[j];
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kModes; k += kThreads) {
    double t = 0;
    for (int ww = 0; ww < W; ++ww) t += acc[ww][k];
    dcoef[(long long)r * kModes + k] = t;
  }
}

// Points with gate 2 (relaxation only: Q = -nu (f - M), then the FP64
// projection), coalesced: a CTA takes the 32 points of one AoSoA block (lane
// = point, so every bank access is a 128-byte row) over one of kRelaxSplit
// ranges of the velocity index.  Pass 1 stores Q and the range's moments per
// point; pass 2 (for every gated point: the gate-1 partials come from
// reconstruct_kernel) sums the ranges' moments in a fixed order, solves for
// the projection and corrects its range.  The local Maxwellian comes from
// per-point 1D Gaussian tables (the Gaussian factorises over the axes).

struct RelaxPoint {
  int upt, eb, lane, e;
};

__device__ __forceinline__ RelaxPoint relax_point(const FrameArgs& a) {
  const int nb = (a.neles + 31) / 32;
  RelaxPoint r;
  r.upt = blockIdx.y / nb;
  r.eb = blockIdx.y % nb;
  r.lane = threadIdx.x & 31;
  r.e = r.eb * 32 + r.lane;
  return r;
}

template <typename T>
__global__ void __launch_bounds__(kRelaxWarps * 32) relax_pass1_kernel(const double* __restrict__ mom_in,
                                                                      const int* __restrict__ gate, FrameArgs a,
                                                                      const T* __restrict__ f,
                                                                      const T* __restrict__ nu,
                                                                      T* __restrict__ Q, double* __restrict__ part) {
  __shared__ double Ex[32][3 * kMaxN + 1];
  __shared__ double red[kRelaxWarps][32][5];
  __shared__ double ms[32];
  __shared__ int on[32];
  const int N = a.N, V = N * N * N;
  const RelaxPoint P = relax_point(a);
  const double h = 2.0 * a.L / N, c00 = -a.L + a.L / N;
  if (threadIdx.x < 32) {
    const int pt = P.upt * a.neles + P.e;
    const bool ok = P.e < a.neles && gate[pt] == 2;
    on[threadIdx.x] = ok;
    const double rt = ok ? rsqrt(mom_in[(long long)pt * 5 + 4]) : 0.0;
    ms[threadIdx.x] = ok ? mom_in[(long long)pt * 5] * rt * rt * rt * 0.17958712212516656 : 0.0;
  }
  for (int t = threadIdx.x; t < 32 * 3 * N; t += blockDim.x) {
    const int l = t / (3 * N), ax = (t / N) % 3, I = t % N;
    const int pt = P.upt * a.neles + P.eb * 32 + l;
    double v = 0.0;
    if (P.eb * 32 + l < a.neles && gate[pt] == 2) {
      const double d = (c00 + I * h - mom_in[(long long)pt * 5 + 1 + ax]) * rsqrt(mom_in[(long long)pt * 5 + 4]);
      v = exp(-d * d);
    }
    Ex[l][ax * N + I] = v;
  }
  __syncthreads();
  const int w = threadIdx.x >> 5;
  const int v0 = blockIdx.x * V / kRelaxSplit, v1 = (blockIdx.x + 1) * V / kRelaxSplit;
  double m[5] = {0, 0, 0, 0, 0};
  if (on[P.lane]) {
    const double msc = ms[P.lane];
    const long long base = (long long)P.upt * a.ldim + (long long)P.eb * V * 32 + P.lane;
    int I = (v0 + w) / (N * N), J = ((v0 + w) / N) % N, K = (v0 + w) % N;
#pragma unroll 4
    for (int v = v0 + w; v < v1; v += kRelaxWarps) {
      const long long ix = base + (long long)v * 32;
      const double M = msc * Ex[P.lane][I] * Ex[P.lane][N + J] * Ex[P.lane][2 * N + K];
      const double q = -(double)nu[ix] * ((double)f[ix] - M);
      Q[ix] = (T)q;
      const double cx = c00 + I * h, cy = c00 + J * h, cz = c00 + K * h;
      m[0] += q;
      m[1] += q * cx;
      m[2] += q * cy;
      m[3] += q * cz;
      m[4] += q * (cx * cx + cy * cy + cz * cz);
      // next v: carry K into J into I
      K += kRelaxWarps;
      while (K >= N) {
        K -= N;
        if (++J == N) {
          J = 0;
          ++I;
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) red[w][P.lane][k] = m[k];
  __syncthreads();
  if (threadIdx.x < 32 * 5 && on[threadIdx.x / 5]) {  // gate-1 slots hold reconstruct_kernel's partials
    const int l = threadIdx.x / 5, k = threadIdx.x % 5;
    double s = 0;
    for (int ww = 0; ww < kRelaxWarps; ++ww) s += red[ww][l][k];
    part[(((long long)blockIdx.y * 32 + l) * kRelaxSplit + blockIdx.x) * 5 + k] = s;
  }
}

template <typename T>
__global__ void __launch_bounds__(kRelaxWarps * 32) relax_pass2_kernel(const int* __restrict__ gate, FrameArgs a,
                                                                      const double* __restrict__ ginv,
                                                                      const double* __restrict__ part,
                                                                      T* __restrict__ Q) {
  __shared__ double lam[32][5];
  __shared__ int on[32];
  const int N = a.N, V = N * N * N;
  const RelaxPoint P = relax_point(a);
  const double h = 2.0 * a.L / N, c00 = -a.L + a.L / N;
  if (threadIdx.x < 32) {
    const int pt = P.upt * a.neles + P.e;
    const bool ok = P.e < a.neles && gate[pt] != 0;  // gate 1 (reconstruct_kernel) and 2 (pass 1)
    on[threadIdx.x] = ok;
    double mt[5] = {0, 0, 0, 0, 0};
    const int nslot = ok && gate[pt] == 1 ? kNetSplit : kRelaxSplit;
    if (ok)
      for (int c = 0; c < nslot; ++c)
#pragma unroll
        for (int k = 0; k < 5; ++k) mt[k] += part[(((long long)blockIdx.y * 32 + P.lane) * kRelaxSplit + c) * 5 + k];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      double s = 0;
#pragma unroll
      for (int j = 0; j < 5; ++j) s += ginv[k * 5 + j] * mt[j];
      lam[threadIdx.x][k] = s;
    }
  }
  __syncthreads();
  if (!on[P.lane]) return;
  const int w = threadIdx.x >> 5;
  const int v0 = blockIdx.x * V / kRelaxSplit, v1 = (blockIdx.x + 1) * V / kRelaxSplit;
  const double l0 = lam[P.lane][0], l1 = lam[P.lane][1], l2 = lam[P.lane][2], l3 = lam[P.lane][3],
               l4 = lam[P.lane][4];
  const long long base = (long long)P.upt * a.ldim + (long long)P.eb * V * 32 + P.lane;
  int I = (v0 + w) / (N * N), J = ((v0 + w) / N) % N, K = (v0 + w) % N;
#pragma unroll 4
  for (int v = v0 + w; v < v1; v += kRelaxWarps) {
    const long long ix = base + (long long)v * 32;
    const double cx = c00 + I * h, cy = c00 + J * h, cz = c00 + K * h;
    Q[ix] = (T)((double)Q[ix] - (l0 + l1 * cx + l2 * cy + l3 * cz + l4 * (cx * cx + cy * cy + cz * cz)));
    K += kRelaxWarps;
    while (K >= N) {
      K -= N;
      if (++J == N) {
        J = 0;
        ++I;
      }
    }
  }
}

// gate[pt] = 1 when eps[pt] < threshold (2 when also eps[pt] < eps_zero:
// the reconstruction then takes G - nu M = 0) and, given the frames mom,
// the local Maxwellian is resolved by the grid:
// min_axis (L - |u_axis|)/sqrt(T) >= rmin; gate 0 points go to the plain
// list (order irrelevant: every point is independent)
__global__ void gate_kernel(int npts, const float* __restrict__ eps, float threshold, float eps_zero,
                            const double* __restrict__ mom, double L, double rmin, int* __restrict__ gate,
                            int* __restrict__ plain, int* __restrict__ nplain, int* __restrict__ net,
                            int* __restrict__ nnet) {
  const int pt = blockIdx.x * blockDim.x + threadIdx.x;
  if (pt >= npts) return;
  int g = (eps[pt] < threshold) ? (eps[pt] < eps_zero ? 2 : 1) : 0;
  if (mom) {
    const double* m = mom + (long long)pt * 5;
    const double umax = fmax(fabs(m[1]), fmax(fabs(m[2]), fabs(m[3])));
    if (!((L - umax) >= rmin * sqrt(m[4]))) g = 0;
  }
  gate[pt] = g;
  if (!g) plain[atomicAdd(nplain, 1)] = pt;
  if (g == 1 && net) net[atomicAdd(nnet, 1)] = pt;
}

bool g_modes_ready[64];

int init_modes() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && g_modes_ready[dev]) return DGFS_OK;
  unsigned char mi[kModes], mj[kModes], mk[kModes];
  short idx[kP][kP][kP];
  for (int i = 0; i < kP; ++i)
    for (int j = 0; j < kP; ++j)
      for (int k = 0; k < kP; ++k) idx[i][j][k] = -1;
  int m = 0;
  for (int d = 0; d <= kDeg; ++d)
    for (int i = d; i >= 0; --i)
      for (int j = d - i; j >= 0; --j) {
        const int k = d - i - j;
        mi[m] = (unsigned char)i;
        mj[m] = (unsigned char)j;
        mk[m] = (unsigned char)k;
        idx[i][j][k] = (short)m;
        ++m;
      }
  if (cudaMemcpyToSymbol(c_mi, mi, sizeof(mi)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_mj, mj, sizeof(mj)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_mk, mk, sizeof(mk)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_midx, idx, sizeof(idx)) != cudaSuccess)
    return dgfs::set_error(DGFS_ERR_CUDA, "mode table upload failed");
  if (dev >= 0 && dev < 64) g_modes_ready[dev] = true;
  return DGFS_OK;
}

int check_frame(int precision, int N, int nupts, int neles, long long ldim, double L, double cw) {
  using dgfs::set_error;
  if (precision != 32 && precision != 64) return set_error(DGFS_ERR_INVALID, "precision must be 32 or 64");
  if (N < 4 || N > kMaxN) return set_error(DGFS_ERR_UNSUPPORTED, "Nv=%d outside 4..%d", N, kMaxN);
  if (nupts < 1 || neles < 1 || !(L > 0) || !(cw > 0)) return set_error(DGFS_ERR_INVALID, "bad sizes");
  const long long V = (long long)N * N * N;
  if (ldim < (neles + 31) / 32 * 32 * V) return set_error(DGFS_ERR_INVALID, "ldim too small");
  if ((long long)nupts * neles > 0x7fffffffLL) return set_error(DGFS_ERR_UNSUPPORTED, "too many points");
  return DGFS_OK;
}

}  // namespace

extern "C" int dgfs_hermite_embed(int precision, const void* f, const void* Q, const void* nu, int nupts,
                                  int neles, long long ldim, int Nv, double L, double cw, double prefactor,
                                  double gamma, float* X, float* B, double* mom, float* eps, void* stream) {
  dgfs::clear_error();
  if (!f || !X || !mom || !eps || (Q && !B) || (nu && !Q)) return dgfs::set_error(DGFS_ERR_INVALID, "null pointer");
  int rc = check_frame(precision, Nv, nupts, neles, ldim, L, cw);
  if (!rc) rc = init_modes();
  if (rc) return rc;
  FrameArgs a{Nv, nupts, neles, ldim, L, cw, prefactor, gamma};
  const size_t smem = ((size_t)Nv * Nv * kP + (size_t)Nv * kP * kP) * sizeof(double);
  const void* fn = precision == 64 ? (const void*)embed_kernel<double> : (const void*)embed_kernel<float>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return dgfs::set_error(DGFS_ERR_CUDA, "smem attribute");
  const unsigned grid = (unsigned)(nupts * neles);
  if (precision == 64)
    embed_kernel<double><<<grid, kThreads, smem, (cudaStream_t)stream>>>((const double*)f, (const double*)Q,
                                                                          (const double*)nu, a, X, B, mom, eps);
  else
    embed_kernel<float><<<grid, kThreads, smem, (cudaStream_t)stream>>>((const float*)f, (const float*)Q,
                                                                         (const float*)nu, a, X, B, mom, eps);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return dgfs::set_error(DGFS_ERR_CUDA, "embed launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_hermite_reconstruct(int precision, const float* B, const double* mom, const int* gate,
                                        int nupts, int neles, long long ldim, int Nv, double L, double cw,
                                        double prefactor, double gamma, const double* ginv,
                                        const double* gwinv, const void* f, const void* nu, void* Q,
                                        const int* rows, const int* nrows, double* work, void* stream) {
  dgfs::clear_error();
  if (!B || !mom || !ginv || !Q || (nu && !f)) return dgfs::set_error(DGFS_ERR_INVALID, "null pointer");
  int rc = check_frame(precision, Nv, nupts, neles, ldim, L, cw);
  if (!rc) rc = init_modes();
  if (rc) return rc;
  FrameArgs a{Nv, nupts, neles, ldim, L, cw, prefactor, gamma};
  const size_t smem = ((size_t)kP * kP * Nv + (size_t)kP * Nv * Nv) * sizeof(double);
  const void* fn =
      precision == 64 ? (const void*)reconstruct_kernel<double> : (const void*)reconstruct_kernel<float>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return dgfs::set_error(DGFS_ERR_CUDA, "smem attribute");
  // with a workspace, the gate-1 list, gate and nu: gate-1 points from the
  // list in kNetSplit chunks (coefficients once per point), gate-2 points on
  // the coalesced relaxation kernels, the projection in one coalesced pass
  const bool split = work && rows && nrows && gate && nu;
  const long long npad = (long long)nupts * ((neles + 31) / 32) * 32;
  double* part = split ? work : nullptr;
  double* dcoef = split ? work + npad * kRelaxSplit * 5 : nullptr;
  const unsigned npts = (unsigned)(nupts * neles);
  const unsigned grid = npts * (split ? kNetSplit : 1);
  cudaStream_t s = (cudaStream_t)stream;
  if (split) coef_kernel<<<npts, kThreads, 0, s>>>(rows, nrows, B, gwinv, dcoef);
  if (precision == 64)
    reconstruct_kernel<double><<<grid, kThreads, smem, s>>>(B, mom, gate, a, ginv, gwinv, (const double*)f,
                                                           (const double*)nu, (double*)Q, part, rows, nrows,
                                                           dcoef);
  else
    reconstruct_kernel<float><<<grid, kThreads, smem, s>>>(B, mom, gate, a, ginv, gwinv, (const float*)f,
                                                          (const float*)nu, (float*)Q, part, rows, nrows, dcoef);
  if (split) {
    const dim3 rg(kRelaxSplit, (unsigned)(nupts * ((neles + 31) / 32)));
    if (precision == 64) {
      relax_pass1_kernel<double><<<rg, kRelaxWarps * 32, 0, s>>>(mom, gate, a, (const double*)f, (const double*)nu,
                                                                  (double*)Q, work);
      relax_pass2_kernel<double><<<rg, kRelaxWarps * 32, 0, s>>>(gate, a, ginv, work, (double*)Q);
    } else {
      relax_pass1_kernel<float><<<rg, kRelaxWarps * 32, 0, s>>>(mom, gate, a, (const float*)f, (const float*)nu,
                                                                 (float*)Q, work);
      relax_pass2_kernel<float><<<rg, kRelaxWarps * 32, 0, s>>>(gate, a, ginv, work, (float*)Q);
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return dgfs::set_error(DGFS_ERR_CUDA, "reconstruct launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_surrogate_gate(int npts, const float* eps, float threshold, float eps_zero,
                                   const double* mom, double L, double rmin, int* gate, int* plain, int* nplain,
                                   int* net, int* nnet, void* stream) {
  dgfs::clear_error();
  if (npts < 1 || !eps || !gate || !plain || !nplain || (!net != !nnet))
    return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  cudaError_t e = cudaMemsetAsync(nplain, 0, sizeof(int), (cudaStream_t)stream);
  if (e == cudaSuccess && nnet) e = cudaMemsetAsync(nnet, 0, sizeof(int), (cudaStream_t)stream);
  if (e != cudaSuccess) return dgfs::set_error(DGFS_ERR_CUDA, "gate counter reset: %s", cudaGetErrorString(e));
  gate_kernel<<<(npts + 255) / 256, 256, 0, (cudaStream_t)stream>>>(npts, eps, threshold, eps_zero, mom, L, rmin,
                                                                     gate, plain, nplain, net, nnet);
  e = cudaGetLastError();
  return e == cudaSuccess ? DGFS_OK : dgfs::set_error(DGFS_ERR_CUDA, "gate launch: %s", cudaGetErrorString(e));
}

namespace {

// In place on rows of X[M][ld]: columns [c0, c1) divided (inverse: multiplied)
// by s = max(eps[m], eps0); column logcol (when >= 0, forward only) := log(s).
__global__ void scale_rows_kernel(int M, int ld, const float* __restrict__ eps, float eps0, int c0, int c1,
                                  int logcol, int inverse, float* __restrict__ X) {
  const int m = blockIdx.x;
  if (m >= M) return;
  const float s = fmaxf(eps[m], eps0);
  const float k = inverse ? s : 1.f / s;
  for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) X[(long long)m * ld + c] *= k;
  if (!inverse && logcol >= 0 && threadIdx.x == 0) X[(long long)m * ld + logcol] = logf(s);
}

}  // namespace

extern "C" int dgfs_surrogate_scale(int M, int ld, const float* eps, float eps0, int c0, int c1, int logcol,
                                    int inverse, float* X, void* stream) {
  dgfs::clear_error();
  if (M < 1 || ld < 1 || !eps || !X || !(eps0 > 0.f) || c0 < 0 || c1 > ld || c0 > c1 || logcol >= ld ||
      (logcol >= c0 && logcol < c1))
    return dgfs::set_error(DGFS_ERR_INVALID, "bad arguments");
  scale_rows_kernel<<<M, 128, 0, (cudaStream_t)stream>>>(M, ld, eps, eps0, c0, c1, logcol, inverse, X);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DGFS_OK : dgfs::set_error(DGFS_ERR_CUDA, "scale launch: %s", cudaGetErrorString(e));
}
