// Common device helpers for the DGFS B200 kernels: complex arithmetic on
// float2/double2, compile-time loops and the frfs AoSoA addressing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace dgfs {

template <typename T> struct cplx_of;
template <> struct cplx_of<float> { using type = float2; };
template <> struct cplx_of<double> { using type = double2; };
template <typename T> using cx = typename cplx_of<T>::type;

template <typename C> __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C r; r.x = a; r.y = b; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return mk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mk<C>(a.x * s, a.y * s); }
// acc + a*b
template <typename C> __device__ __forceinline__ C cfma(C a, C b, C acc) {
  return mk<C>(acc.x + a.x * b.x - a.y * b.y, acc.y + a.x * b.y + a.y * b.x);
}

// Compile-time loop: f(std::integral_constant<int, I>) for I in [B, E)
template <int B, int E, typename F> __device__ __forceinline__ void sfor(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    sfor<B + 1, E>(f);
  }
}

// frfs AoSoA(soasz) address of (upt, var v, element e) in a bank of leading
// dimension ldim (frfs/backends/cuda/kernels/base.mako:4-6):
//   upt*ldim + ((e/soasz)*nvar + v)*soasz + e%soasz
__device__ __forceinline__ int64_t soa_ix(int64_t upt, int64_t ldim, int64_t e, int64_t v,
                                          int64_t nvar, int64_t soasz) {
  return upt * ldim + ((e / soasz) * nvar + v) * soasz + e % soasz;
}

}  // namespace dgfs
