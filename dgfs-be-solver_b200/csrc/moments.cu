// Macroscopic moments of the distribution at every solution point, in FP64.
//
// Restates the 3D moment formulas of frfs's moment writer
// (frfs/plugins/dgfsmomwriterstd.py:154-214) in nondimensional form (mass
// ratio 1):
//   rho = cw sum f,  u = cw sum f c / rho,
//   T = (2/3) cw sum f |c-u|^2 / rho,  q = cw sum f |c-u|^2 (c-u),
//   P_ij = 2 cw sum f (c_i-u_i)(c_j-u_j)
// on the cell-centred grid c0_i = -L + L/N + i 2L/N.  The writer copies the
// whole bank to the host and reduces in numpy; here one CTA reduces 32
// elements of one solution-point row (one AoSoA block, coalesced) in two
// passes over the velocities (mean velocity, then central moments).
#include <cuda_runtime.h>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"

namespace {

constexpr int kW = 8;  // warps per CTA; lane = element of the AoSoA block

template <typename T>
__global__ void __launch_bounds__(32 * kW) moments_kernel(const T* __restrict__ f, int nupts, int neles,
                                                          long long ldim, int N, double L, double cw,
                                                          double* __restrict__ out) {
  __shared__ double red[kW][32][4];
  __shared__ double red2[kW][32][10];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nblk = (neles + 31) / 32;
  const int upt = blockIdx.x / nblk, eb = blockIdx.x % nblk;
  const int e = eb * 32 + lane;
  const long long V = (long long)N * N * N;
  const double h = 2.0 * L / N, c00 = -L + L / N;
  const T* row = f + (long long)upt * ldim + (long long)eb * V * 32 + lane;

  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  if (e < neles)
    for (long long v = w; v < V; v += kW) {
      const double fv = (double)row[v * 32];
      const double cx = c00 + (double)(v / (N * N)) * h, cy = c00 + (double)((v / N) % N) * h,
                   cz = c00 + (double)(v % N) * h;
      s0 += fv;
      s1 += fv * cx;
      s2 += fv * cy;
      s3 += fv * cz;
    }
  red[w][lane][0] = s0;
  red[w][lane][1] = s1;
  red[w][lane][2] = s2;
  red[w][lane][3] = s3;
  __syncthreads();
  double m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  for (int k = 0; k < kW; ++k) {
    m0 += red[k][lane][0];
    m1 += red[k][lane][1];
    m2 += red[k][lane][2];
    m3 += red[k][lane][3];
  }
  const double rho = m0 * cw;
  const double ux = m1 * cw / rho, uy = m2 * cw / rho, uz = m3 * cw / rho;

  double a[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // |c'|^2, q(3), P(6)
  if (e < neles)
    for (long long v = w; v < V; v += kW) {
      const double fv = (double)row[v * 32];
      const double cx = c00 + (double)(v / (N * N)) * h - ux, cy = c00 + (double)((v / N) % N) * h - uy,
                   cz = c00 + (double)(v % N) * h - uz;
      const double c2 = cx * cx + cy * cy + cz * cz;
      a[0] += fv * c2;
      a[1] += fv * c2 * cx;
      a[2] += fv * c2 * cy;
      a[3] += fv * c2 * cz;
      a[4] += fv * cx * cx;
      a[5] += fv * cx * cy;
      a[6] += fv * cx * cz;
      a[7] += fv * cy * cy;
      a[8] += fv * cy * cz;
      a[9] += fv * cz * cz;
    }
#pragma unroll
  for (int k = 0; k < 10; ++k) red2[w][lane][k] = a[k];
  __syncthreads();
  if (w == 0 && e < neles) {
    double t[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < kW; ++k)
#pragma unroll
      for (int j = 0; j < 10; ++j) t[j] += red2[k][lane][j];
    double* o = out + ((long long)upt * neles + e) * 14;
    o[0] = rho;
    o[1] = ux;
    o[2] = uy;
    o[3] = uz;
    o[4] = t[0] * (2.0 / 3.0 * cw) / rho;
    o[5] = t[1] * cw;
    o[6] = t[2] * cw;
    o[7] = t[3] * cw;
#pragma unroll
    for (int j = 0; j < 6; ++j) o[8 + j] = 2.0 * t[4 + j] * cw;
  }
}

}  // namespace

extern "C" int dgfs_moments(int precision, const void* f, int nupts, int neles, long long ldim, int Nv, double L,
                            double cw, double* out, void* stream) {
  using dgfs::set_error;
  dgfs::clear_error();
  if (!f || !out) return set_error(DGFS_ERR_INVALID, "null pointer");
  if (precision != 32 && precision != 64) return set_error(DGFS_ERR_INVALID, "precision must be 32 or 64");
  if (nupts < 1 || neles < 1 || Nv < 1 || !(L > 0) || !(cw > 0))
    return set_error(DGFS_ERR_INVALID, "bad sizes");
  const long long V = (long long)Nv * Nv * Nv;
  const long long nblk = (neles + 31) / 32;
  if (ldim < nblk * 32 * V) return set_error(DGFS_ERR_INVALID, "ldim %lld smaller than one AoSoA row", ldim);
  const unsigned grid = (unsigned)(nupts * nblk);
  if (precision == 64)
    moments_kernel<double><<<grid, 32 * kW, 0, (cudaStream_t)stream>>>((const double*)f, nupts, neles, ldim, Nv, L,
                                                                       cw, out);
  else
    moments_kernel<float><<<grid, 32 * kW, 0, (cudaStream_t)stream>>>((const float*)f, nupts, neles, ldim, Nv, L,
                                                                      cw, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "moments launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}
