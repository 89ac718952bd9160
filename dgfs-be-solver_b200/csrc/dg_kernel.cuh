// FR-DG advection residual over all discrete velocities.
//
// One thread per (velocity v, element e); a warp covers the 32 elements of
// one AoSoA block at one velocity, so every bank access is a coalesced
// 32-element row.  The element operators travel in the kernel parameters
// (constant bank) and every loop over them is unrolled, so matrix entries are
// FMA operands, not loads.
//
//   dg_interp_kernel    uf = M0 u at the flux points (frfs/solvers/dgfs/
//                        elements.py:55-59, 'disu')
//   dg_bcsum_kernel     diffuse-wall sums over velocities in FP64
//                        (kernels/bcs/dgfs-wall-diffuse-update.mako:14-36)
//   dg_residual_kernel  R = -(1/|J|)[(M1 - M3 M2) F~ + M3 F^] with the upwind
//                        common flux at every flux point (interfaces and
//                        boundaries), fused with the Runge-Kutta combination
//                        out = a A + b B + g (R + C)
//                        (elements.py:49-118, intcflux.mako, bccflux.mako,
//                        rusanov.mako:46-50, negdivconf.mako, axnpby.mako)
#pragma once

#include "dgfs_common.cuh"

namespace dgfs {

enum DgBcKind {
  BC_WALL_DIFFUSE = 0,
  BC_INLET = 1,
  BC_OUTLET = 2,
  BC_VANISH = 3,
  BC_WALL_SPECULAR = 4,
  BC_WALL_DIFFUSE_CYL = 5
};

template <typename T, int U, int F, int D> struct DgOps {
  T m0[F][U];
  T m132[U][D * U];
  T m3[U][F];
};

template <typename T> struct DgArgs {
  int V, neles, v0, nv;
  int64_t ldim_u;          // leading dimension of solution banks
  int64_t ldim_f;          // leading dimension of the flux-point scratch
  const T* u;              // solution bank [U][V][E] (AoSoA 32)
  T* uf;                   // flux-point values [F][V][E] (AoSoA 32)
  T* out;                  // residual / RK output bank
  const T* A;              // optional terms of out = a A + b B + g (R + C)
  const T* B;
  const T* Cq;
  T alpha, beta, gamma;
  // geometry (SoA over elements)
  const T* smats;          // [D][U][D][E]
  const T* rcpdjac;        // [U][E]
  const T* nrm;            // [F][D][E] unit outward normals
  const T* mag;            // [F][E]    |S^T n|
  const int* part;         // [F][E]    fpt_r*E + e_r, or -(b+1) for boundary b
  const int64_t* pbase;    // [F][E]    partner's flux-bank offset at v = 0 (-1: boundary)
  const T* cvx;            // [V] velocity grid
  const T* cvy;
  const T* cvz;
  // boundaries
  const int* bkind;        // [nb]
  const int* bgroup;       // [nb]
  const T* guw;            // [ngroups][3]
  const T* gfw;            // [ngroups][V]
  const int* grefl;        // [ngroups][V]
  const T* bwall;          // [nb][4] wall Ux, Uy, Uz, T per boundary point (cylinder wall)
  const double* bcvals;    // [nb][2]
};

template <typename T, int U> struct DgMassOps {
  T m12[U][U];
};

__device__ __forceinline__ int64_t aos32(int64_t row, int64_t ldim, int64_t e, int64_t v, int64_t V) {
  return row * ldim + ((e >> 5) * V + v) * 32 + (e & 31);
}

template <typename T, int U, int F, int D>
__global__ void __launch_bounds__(256) dg_interp_kernel(const DgArgs<T> a, const DgOps<T, U, F, D> op) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = (int)(t & 31);
  const int64_t w = t >> 5;
  const int v = a.v0 + (int)(w % a.nv);
  const int64_t e = (w / a.nv) * 32 + lane;
  if (e >= a.neles) return;
  T u[U];
#pragma unroll
  for (int i = 0; i < U; ++i) u[i] = a.u[aos32(i, a.ldim_u, e, v, a.V)];
#pragma unroll
  for (int f = 0; f < F; ++f) {
    T s = T(0);
#pragma unroll
    for (int i = 0; i < U; ++i) s = fma(op.m0[f][i], u[i], s);
    a.uf[aos32(f, a.ldim_f, e, v, a.V)] = s;
  }
}

// out = M12 u at the solution points of velocities [v0, v0 + nv): the
// 'invmass' kernel of DGFSElements (frfs/solvers/dgfs/elements.py:161-164),
// M12 = V^T V with V the orthonormal basis at the solution points.
template <typename T, int U>
__global__ void __launch_bounds__(256) dg_invmass_kernel(const DgArgs<T> a, const DgMassOps<T, U> op) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = (int)(t & 31);
  const int64_t w = t >> 5;
  const int v = a.v0 + (int)(w % a.nv);
  const int64_t e = (w / a.nv) * 32 + lane;
  if (e >= a.neles) return;
  T u[U];
#pragma unroll
  for (int i = 0; i < U; ++i) u[i] = a.u[aos32(i, a.ldim_u, e, v, a.V)];
#pragma unroll
  for (int r = 0; r < U; ++r) {
    T s = T(0);
#pragma unroll
    for (int i = 0; i < U; ++i) s = fma(op.m12[r][i], u[i], s);
    a.out[aos32(r, a.ldim_u, e, v, a.V)] = s;
  }
}

// Diffuse-wall sums, pass 1: block (chunk, group) reduces 32 boundary flux
// points over one chunk of the velocity range in FP64 (8 velocity lanes per
// point) and writes partials[chunk][b] = (sum_{c.n>=0} (c-Uw).n f cw,
// sum_{c.n<0} (c-Uw).n fw cw).
template <typename T, int D>
__global__ void __launch_bounds__(256) dg_bcsum_kernel(const DgArgs<T> a, const int* __restrict__ bfpt,
                                                      const int* __restrict__ bele, int nb, double cw,
                                                      int chunk, double* __restrict__ partials) {
  __shared__ double s0[8][32], s1[8][32];
  const int bl = threadIdx.x & 31, vg = threadIdx.x >> 5;
  const int b = blockIdx.y * 32 + bl;
  const int vbeg = a.v0 + blockIdx.x * chunk;
  const int vend = min(a.v0 + a.nv, vbeg + chunk);
  double acc0 = 0.0, acc1 = 0.0;
  const int kind = b < nb ? a.bkind[b] : -1;
  if (kind == BC_WALL_DIFFUSE || kind == BC_WALL_DIFFUSE_CYL) {
    const int j = bfpt[b], e = bele[b], g = a.bgroup[b];
    const bool cyl = kind == BC_WALL_DIFFUSE_CYL;
    double n[D], uw[3], tw = 1.0;
#pragma unroll
    for (int d = 0; d < D; ++d) n[d] = (double)a.nrm[((int64_t)j * D + d) * a.neles + e];
#pragma unroll
    for (int d = 0; d < 3; ++d) uw[d] = cyl ? (double)a.bwall[b * 4 + d] : (double)a.guw[g * 3 + d];
    if (cyl) tw = (double)a.bwall[b * 4 + 3];
    for (int v = vbeg + vg; v < vend; v += 8) {
      const double dc[3] = {(double)a.cvx[v] - uw[0], (double)a.cvy[v] - uw[1], (double)a.cvz[v] - uw[2]};
      const double dx = dc[0], dy = dc[1], dz = dc[2];
      double fac = 0.0;
#pragma unroll
      for (int d = 0; d < D; ++d) fac += dc[d] * n[d];
      if (fac >= 0.0) {
        acc0 += fac * (double)a.uf[aos32(j, a.ldim_f, e, v, a.V)] * cw;
      } else {
        // the cylinder wall's Maxwellian exp(-|c - U|^2 / T), unnormalised
        // like the reference's (the ratio of the two sums normalises it;
        // bcs/dgfs-wall-diffuse-cyl-update.mako)
        const double fw = cyl ? exp(-(dx * dx + dy * dy + dz * dz) / tw) : (double)a.gfw[(int64_t)g * a.V + v];
        acc1 += fac * fw * cw;
      }
    }
  }
  s0[vg][bl] = acc0;
  s1[vg][bl] = acc1;
  __syncthreads();
  if (vg == 0 && b < nb) {
    double r0 = 0.0, r1 = 0.0;
    for (int k = 0; k < 8; ++k) {
      r0 += s0[k][bl];
      r1 += s1[k][bl];
    }
    partials[((int64_t)blockIdx.x * nb + b) * 2] = r0;
    partials[((int64_t)blockIdx.x * nb + b) * 2 + 1] = r1;
  }
}

// Pass 2: one warp per boundary point sums the chunks into bcvals in a
// fixed order (lane-strided partial sums, then a fixed butterfly), so the
// result is the same on every run.
__global__ void __launch_bounds__(256) dg_bcsum_finish_kernel(const int* __restrict__ bkind, int nb, int nchunks,
                                                             const double* __restrict__ partials,
                                                             double* __restrict__ bcvals, int reset) {
  const int b = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b >= nb || (bkind[b] != BC_WALL_DIFFUSE && bkind[b] != BC_WALL_DIFFUSE_CYL)) return;  // uniform per warp
  double r0 = 0.0, r1 = 0.0;
  for (int c = lane; c < nchunks; c += 32) {
    r0 += partials[((int64_t)c * nb + b) * 2];
    r1 += partials[((int64_t)c * nb + b) * 2 + 1];
  }
  for (int o = 16; o > 0; o >>= 1) {
    r0 += __shfl_xor_sync(0xffffffffu, r0, o);
    r1 += __shfl_xor_sync(0xffffffffu, r1, o);
  }
  if (lane == 0) {
    if (reset) {
      bcvals[2 * b] = r0;
      bcvals[2 * b + 1] = r1;
    } else {
      bcvals[2 * b] += r0;
      bcvals[2 * b + 1] += r1;
    }
  }
}

// FP32 up to p = 2: 4 CTAs per SM (<= 64 registers; measured 0.132 ms per
// Couette stage against 0.145 ms at 2 CTAs per SM): the kernel is bound by
// the latency of its partner loads, issued together up front from
// precomputed offsets.  p = 3 (16 solution and flux points) holds too many
// values for 64 registers: no occupancy bound there.
template <typename T, int U, int F, int D>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 && U <= 9) ? 4 : 1) dg_residual_kernel(const DgArgs<T> a, const DgOps<T, U, F, D> op) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = (int)(t & 31);
  const int64_t w = t >> 5;
  const int v = a.v0 + (int)(w % a.nv);
  const int64_t e = (w / a.nv) * 32 + lane;
  if (e >= a.neles) return;
  const int64_t E = a.neles;

  T u[U];
#pragma unroll
  for (int i = 0; i < U; ++i) u[i] = a.u[aos32(i, a.ldim_u, e, v, a.V)];
  const T c[3] = {a.cvx[v], a.cvy[v], a.cvz[v]};

  // partner values first: every load independent of the others, so their
  // latencies overlap (offsets precomputed per (flux point, element))
  T urv[F];
#pragma unroll
  for (int f = 0; f < F; ++f) {
    const int64_t pb = a.pbase[(int64_t)f * E + e];
    urv[f] = pb >= 0 ? a.uf[pb + (int64_t)v * 32] : T(0);
  }

  // common normal fluxes at this element's flux points
  T fh[F];
#pragma unroll
  for (int f = 0; f < F; ++f) {
    T ul = T(0);
#pragma unroll
    for (int i = 0; i < U; ++i) ul = fma(op.m0[f][i], u[i], ul);
    T n[D];
#pragma unroll
    for (int d = 0; d < D; ++d) n[d] = a.nrm[((int64_t)f * D + d) * E + e];
    T nc = n[0] * c[0];
#pragma unroll
    for (int d = 1; d < D; ++d) nc = fma(n[d], c[d], nc);
    const int p = a.part[(int64_t)f * E + e];
    T ur;
    if (p >= 0) {
      ur = urv[f];
    } else {
      const int b = -p - 1;
      const int kind = a.bkind[b], g = a.bgroup[b];
      if (kind == BC_WALL_DIFFUSE || kind == BC_INLET) {
        T fac = (c[0] - a.guw[g * 3]) * n[0];
#pragma unroll
        for (int d = 1; d < D; ++d) fac = fma(c[d] - a.guw[g * 3 + d], n[d], fac);
        if (fac < T(0)) {
          const T fw = a.gfw[(int64_t)g * a.V + v];
          ur = kind == BC_INLET ? fw : fw * (T)(-a.bcvals[2 * b] / a.bcvals[2 * b + 1]);
        } else {
          ur = ul;
        }
      } else if (kind == BC_WALL_DIFFUSE_CYL) {
        // bcs/dgfs-wall-diffuse-cyl.mako: wall state of this boundary point
        const T* w = a.bwall + (int64_t)b * 4;
        const T dc[3] = {c[0] - w[0], c[1] - w[1], c[2] - w[2]};
        T fac = dc[0] * n[0];
#pragma unroll
        for (int d = 1; d < D; ++d) fac = fma(dc[d], n[d], fac);
        if (fac < T(0)) {
          const T mx = exp(-(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]) / w[3]);
          ur = mx * (T)(-a.bcvals[2 * b] / a.bcvals[2 * b + 1]);
        } else {
          ur = ul;
        }
      } else if (kind == BC_VANISH) {
        ur = nc < T(0) ? T(0) : ul;
      } else if (kind == BC_WALL_SPECULAR) {
        const int vr = a.grefl[(int64_t)g * a.V + v];
        ur = a.uf[aos32(f, a.ldim_f, e, vr, a.V)];
      } else {
        ur = ul;  // outlet
      }
    }
    // upwind flux 0.5 (n.c)(ul + ur) + 0.5 |n.c| (ul - ur)  (rusanov.mako:46-50)
    const T fn = T(0.5) * nc * (ul + ur) + T(0.5) * fabs(nc) * (ul - ur);
    fh[f] = a.mag[(int64_t)f * E + e] * fn;
  }

  // transformed flux at the solution points F~_i = sum_k S_ik c_k u
  T ft[D * U];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int k = 0; k < U; ++k) {
      T s = T(0);
#pragma unroll
      for (int kk = 0; kk < D; ++kk) s = fma(a.smats[(((int64_t)i * U + k) * D + kk) * E + e], c[kk], s);
      ft[i * U + k] = s * u[k];
    }

#pragma unroll
  for (int r = 0; r < U; ++r) {
    T s = T(0);
#pragma unroll
    for (int j = 0; j < D * U; ++j) s = fma(op.m132[r][j], ft[j], s);
#pragma unroll
    for (int f = 0; f < F; ++f) s = fma(op.m3[r][f], fh[f], s);
    const T R = -a.rcpdjac[(int64_t)r * E + e] * s;
    const int64_t o = aos32(r, a.ldim_u, e, v, a.V);
    T res = a.gamma * (a.Cq ? R + a.Cq[o] : R);
    if (a.A) res = fma(a.alpha, a.A[o], res);
    if (a.B) res = fma(a.beta, a.B[o], res);
    a.out[o] = res;
  }
}

}  // namespace dgfs
