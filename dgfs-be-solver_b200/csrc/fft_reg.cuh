// Register-resident complex FFTs of compile-time length N (mixed radix
// 2/3/4/8, Cooley-Tukey decimation in time, natural order in and out).
//
//   fft<T, N, S>(x):  x[k] <- sum_n x[n] exp(S * 2 pi i n k / N)
//
// S = -1 is the unnormalised forward transform and S = +1 the unnormalised
// inverse, the conventions of the cuFFT Z2Z calls the reference makes
// (frfs/solvers/dgfs/scattering.py:239-281).  All indices are compile-time
// constants, so the whole transform lives in registers.  Twiddle factors
// exp(2 pi i m / 96) come from a constant-memory table filled on the host
// with long-double cosl/sinl (96 = lcm of the supported lengths 8,16,24,32).
#pragma once

#include "dgfs_common.cuh"

namespace dgfs {

constexpr int kTwBase = 96;

static __constant__ double c_tw64[2 * kTwBase];
static __constant__ float c_tw32[2 * kTwBase];

template <typename T> __device__ __forceinline__ T tw_cos(int i);
template <typename T> __device__ __forceinline__ T tw_sin(int i);
template <> __device__ __forceinline__ double tw_cos<double>(int i) { return c_tw64[2 * i]; }
template <> __device__ __forceinline__ double tw_sin<double>(int i) { return c_tw64[2 * i + 1]; }
template <> __device__ __forceinline__ float tw_cos<float>(int i) { return c_tw32[2 * i]; }
template <> __device__ __forceinline__ float tw_sin<float>(int i) { return c_tw32[2 * i + 1]; }

// Multiply by i*S (S = +-1)
template <int S, typename C> __device__ __forceinline__ C mul_si(C v) {
  if constexpr (S > 0) return mk<C>(-v.y, v.x);
  else return mk<C>(v.y, -v.x);
}

// v * exp(S * 2 pi i m / N)
template <typename T, int N, int S, int m> __device__ __forceinline__ cx<T> twiddle(cx<T> v) {
  using C = cx<T>;
  constexpr int mm = ((m % N) + N) % N;
  if constexpr (mm == 0) {
    return v;
  } else if constexpr (2 * mm == N) {
    return mk<C>(-v.x, -v.y);
  } else if constexpr (4 * mm == N) {
    return mul_si<S>(v);
  } else if constexpr (4 * mm == 3 * N) {
    return mul_si<-S>(v);
  } else {
    static_assert(kTwBase % N == 0, "unsupported FFT length");
    constexpr int idx = mm * (kTwBase / N);
    const T c = tw_cos<T>(idx);
    const T s = S > 0 ? tw_sin<T>(idx) : -tw_sin<T>(idx);
    return mk<C>(v.x * c - v.y * s, v.x * s + v.y * c);
  }
}

__host__ __device__ constexpr int pick_radix(int n) {
  return (n % 8 == 0 && n > 8) ? 8
       : (n % 4 == 0 && n > 4) ? 4
       : (n % 2 == 0 && n > 2) ? 2
       : (n % 3 == 0 && n > 3) ? 3
       : n;
}

template <typename T, int N, int S> __device__ __forceinline__ void fft(cx<T> (&x)[N]) {
  using C = cx<T>;
  if constexpr (N == 1) {
  } else if constexpr (N == 2) {
    const C a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if constexpr (N == 3) {
    // X1,2 = a - (b+c)/2 +- i S (sqrt(3)/2)(b - c)
    const T h = T(0.86602540378443864676);
    const C a = x[0], b = x[1], c = x[2];
    const C t1 = cadd(b, c);
    const C t2 = mk<C>(a.x - T(0.5) * t1.x, a.y - T(0.5) * t1.y);
    const C d = csub(b, c);
    const C t3 = S > 0 ? mk<C>(h * d.x, h * d.y) : mk<C>(-h * d.x, -h * d.y);
    x[0] = cadd(a, t1);
    x[1] = mk<C>(t2.x - t3.y, t2.y + t3.x);
    x[2] = mk<C>(t2.x + t3.y, t2.y - t3.x);
  } else if constexpr (N == 4) {
    const C s0 = cadd(x[0], x[2]), d0 = csub(x[0], x[2]);
    const C s1 = cadd(x[1], x[3]), d1 = csub(x[1], x[3]);
    const C r = mul_si<S>(d1);
    x[0] = cadd(s0, s1);
    x[2] = csub(s0, s1);
    x[1] = cadd(d0, r);
    x[3] = csub(d0, r);
  } else {
    // N = R*Q; n = r*Q + q; k = k1 + R*k2
    // X[k1 + R k2] = sum_q w_Q^{q k2} w_N^{q k1} sum_r w_R^{r k1} x[r Q + q]
    constexpr int R = pick_radix(N), Q = N / R;
    static_assert(R > 1 && Q > 1, "FFT length has no supported factorisation");
    C y[N];
    sfor<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      C t[R];
      sfor<0, R>([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        t[r] = x[r * Q + q];
      });
      fft<T, R, S>(t);
      sfor<0, R>([&](auto kc) {
        constexpr int k1 = decltype(kc)::value;
        y[k1 * Q + q] = twiddle<T, N, S, q * k1>(t[k1]);
      });
    });
    sfor<0, R>([&](auto kc) {
      constexpr int k1 = decltype(kc)::value;
      C t[Q];
      sfor<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        t[q] = y[k1 * Q + q];
      });
      fft<T, Q, S>(t);
      sfor<0, Q>([&](auto k2c) {
        constexpr int k2 = decltype(k2c)::value;
        x[k1 + R * k2] = t[k2];
      });
    });
  }
}

}  // namespace dgfs
