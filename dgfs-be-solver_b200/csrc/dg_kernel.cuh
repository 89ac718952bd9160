// FR-DG advection residual over all discrete velocities.
//
// Banks are frfs's AoSoA(32) layout: value (row i, velocity v, element e) at
// i*ldim + ((e/32)*V + v)*32 + e%32, so the 32 elements of one block at one
// velocity form one coalesced 128-byte row.  A CTA of 256 threads takes one
// 32-element block (lane = element) and a chunk of 8*VPT velocities (warp w
// takes v = chunk + 8*it + w): consecutive warps read consecutive rows.  The
// element operators travel in the kernel parameters (constant bank) and every
// loop over them is unrolled, so matrix entries are FMA operands, not loads.
// The residual stages the block's element geometry (metric terms, 1/|J|,
// scaled normals, partner offsets) in shared memory once per CTA, one row of
// GS values per lane read with 16-byte loads, and reuses it for every
// velocity of the chunk.
//
//   dg_interp_kernel    uf = M0 u at the flux points (frfs/solvers/dgfs/
//                        elements.py:55-59, 'disu')
//   dg_bcsum_kernel     diffuse-wall sums over velocities in FP64
//                        (kernels/bcs/dgfs-wall-diffuse-update.mako:14-36)
//   dg_residual_kernel  R = -(1/|J|)[(M1 - M3 M2) F~ + M3 F^] with the upwind
//                        common flux at every flux point (interfaces,
//                        boundaries and faces shared with another partition),
//                        fused with the Runge-Kutta combination
//                        out = a A + b B + g (R + C)
//                        (elements.py:49-118, intcflux.mako, bccflux.mako,
//                        mpicflux.mako, rusanov.mako:46-50, negdivconf.mako,
//                        axnpby.mako)
//   dg_pack_kernel      face values at the flux points on partition faces
//                        into a send buffer (the 'pack' kernel of frfs's MPI
//                        interfaces, inters.py:61-112)
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
  int nb;                  // boundary flux points
  // per element block: geometry rows [nblk][32][GS] and partner offsets
  // [nblk][32][PS] (>= 0: flux-bank offset of the partner at v = 0;
  // -1-b: boundary point b < nb; -1-(nb+h): row h of the halo)
  const T* geoblk;
  const int64_t* pblk;
  const T* halo;           // [nhalo][V] partner face values from other partitions
  int* err;                // set to 1 when a bounded wait of the tensor-core residual ran out
};

// Shared-memory row of one element (T values): metric terms S[k][i][kk]
// (k-major, D*D per solution point), 1/|J| (padded to a 16-byte multiple),
// |S^T n| n at the flux points [F][D]; GS pads the row so that the 16-byte
// loads of 8 consecutive lanes fall in distinct bank quads.  Partner offsets
// [F] int64 per lane, padded to PS likewise.
template <typename T, int U, int F, int D> struct DgGeo {
  static constexpr int VW = 16 / (int)sizeof(T);
  static constexpr int OS = 0, NS = U * D * D;
  static constexpr int OR = NS, NR = ((U + VW - 1) / VW) * VW;
  static constexpr int ON = OR + NR, NN = F * D;
  static constexpr int G = ON + NN;
  static constexpr int GS = sizeof(T) == 4 ? G + ((4 - G % 8) + 8) % 8 : G + ((2 - G % 4) + 4) % 4;
  static constexpr int PS = F + ((2 - F % 4) + 4) % 4;
  static_assert(NS % VW == 0 && NN % VW == 0, "16-byte sections");
};

template <typename T, int U> struct DgMassOps {
  T m12[U][U];
};

__device__ __forceinline__ int64_t aos32(int64_t row, int64_t ldim, int64_t e, int64_t v, int64_t V) {
  return row * ldim + ((e >> 5) * V + v) * 32 + (e & 31);
}

// Programmatic dependent launch.  The interp and boundary-sum kernels wait
// for their predecessor in the stream to complete (a no-op when they were
// not launched as dependents), then let their own dependent start: a
// dependent that starts early therefore finds everything before them
// complete and may read the banks (u and the Runge-Kutta terms) before its
// own wait; it reads their outputs (face values, boundary sums) only after
// that wait.  The residual never triggers early: whatever follows it starts
// after it has completed.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename T, int U, int F, int D, int VPT>
__global__ void __launch_bounds__(256) dg_interp_kernel(const DgArgs<T> a, const DgOps<T, U, F, D> op) {
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t e = (int64_t)blockIdx.x * 32 + lane;
  if (e >= a.neles) return;
  const int vend = a.v0 + a.nv;
  const int vbeg = a.v0 + (int)blockIdx.y * (8 * VPT) + w;
#pragma unroll 1
  for (int it = 0; it < VPT; ++it) {
    const int v = vbeg + 8 * it;
    if (v >= vend) break;
    const int64_t o = ((int64_t)blockIdx.x * a.V + v) * 32 + lane;
    T u[U];
    const T* up = a.u + o;
#pragma unroll
    for (int i = 0; i < U; ++i, up += a.ldim_u) u[i] = __ldg(up);
    T* fp = a.uf + o;
#pragma unroll
    for (int f = 0; f < F; ++f, fp += a.ldim_f) {
      T s = T(0);
#pragma unroll
      for (int i = 0; i < U; ++i) s = fma(op.m0[f][i], u[i], s);
      *fp = s;
    }
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
  pdl_wait();
  pdl_trigger();
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
  pdl_wait();
  pdl_trigger();
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

template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; };
template <> struct Vec16<double> { using type = double2; };

// n 16-byte loads from shared memory into r[0 .. n*VW)
template <typename T, int N> __device__ __forceinline__ void lds16(const T* src, T* r) {
  using V4 = typename Vec16<T>::type;
  constexpr int VW = 16 / (int)sizeof(T);
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const V4 q = reinterpret_cast<const V4*>(src)[j];
    if constexpr (VW == 4) {
      r[4 * j] = q.x; r[4 * j + 1] = q.y; r[4 * j + 2] = q.z; r[4 * j + 3] = q.w;
    } else {
      r[2 * j] = q.x; r[2 * j + 1] = q.y;
    }
  }
}

// Ghost value of boundary point b at velocity v (bccflux.mako with the
// bcs/*.mako kinds); nmv = |S^T n| n, whose sign tests equal the unit
// normal's; ul the interior face value.
template <typename T, int D>
__device__ __forceinline__ T dg_ghost(const DgArgs<T>& a, int b, int v, int64_t e, int f, const T* c, const T* nmv,
                                   T nc, T ul) {
  const int kind = a.bkind[b], g = a.bgroup[b];
  if (kind == BC_WALL_DIFFUSE || kind == BC_INLET) {
    T fac = (c[0] - a.guw[g * 3]) * nmv[0];
#pragma unroll
    for (int d = 1; d < D; ++d) fac = fma(c[d] - a.guw[g * 3 + d], nmv[d], fac);
    if (fac < T(0)) {
      const T fw = a.gfw[(int64_t)g * a.V + v];
      return kind == BC_INLET ? fw : fw * (T)(-a.bcvals[2 * b] / a.bcvals[2 * b + 1]);
    }
    return ul;
  }
  if (kind == BC_WALL_DIFFUSE_CYL) {
    // bcs/dgfs-wall-diffuse-cyl.mako: wall state of this boundary point
    const T* w = a.bwall + (int64_t)b * 4;
    const T dc[3] = {c[0] - w[0], c[1] - w[1], c[2] - w[2]};
    T fac = dc[0] * nmv[0];
#pragma unroll
    for (int d = 1; d < D; ++d) fac = fma(dc[d], nmv[d], fac);
    if (fac < T(0)) {
      const T mx = exp(-(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]) / w[3]);
      return mx * (T)(-a.bcvals[2 * b] / a.bcvals[2 * b + 1]);
    }
    return ul;
  }
  if (kind == BC_VANISH) return nc < T(0) ? T(0) : ul;
  if (kind == BC_WALL_SPECULAR) {
    const int vr = a.grefl[(int64_t)g * a.V + v];
    return a.uf[aos32(f, a.ldim_f, e, vr, a.V)];
  }
  return ul;  // outlet
}

// Launch shapes (the autotuner's choice, dgfs_dg_select): VPT velocities per
// warp and CTA chunk; PF = 1 loads the Runge-Kutta terms A, B, C of an
// iteration together with u, before the flux work, as one combination
// K = a A + b B + g C (U more registers); MB CTAs of 256 per SM the
// register budget is compiled for (FP32 p <= 2 needs 80 registers at
// PF = 0, FP32 p = 3 and FP64 p <= 2 128, FP64 p = 3 160).
template <typename T, int U, int F, int D, int VPT, int PF, int MB>
__global__ void __launch_bounds__(256, MB)
    dg_residual_kernel(const DgArgs<T> a, const DgOps<T, U, F, D> op) {
  using G = DgGeo<T, U, F, D>;
  __shared__ __align__(16) T sg[32 * G::GS];
  __shared__ __align__(16) int64_t sp[32 * G::PS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  {
    const T* gs = a.geoblk + (size_t)blockIdx.x * 32 * G::GS;
    for (int i = threadIdx.x; i < 32 * G::GS; i += 256) sg[i] = gs[i];
    const int64_t* ps = a.pblk + (size_t)blockIdx.x * 32 * G::PS;
    for (int i = threadIdx.x; i < 32 * G::PS; i += 256) sp[i] = ps[i];
  }
  __syncthreads();
  const int64_t e = (int64_t)blockIdx.x * 32 + lane;
  if (e >= a.neles) return;
  const T* gl = sg + lane * G::GS;
  const int64_t* pl = sp + lane * G::PS;
  const int vend = a.v0 + a.nv;
  const int vbeg = a.v0 + (int)blockIdx.y * (8 * VPT) + w;

#pragma unroll 1
  for (int it = 0; it < VPT; ++it) {
    const int v = vbeg + 8 * it;
    if (v >= vend) break;
    const int64_t o = ((int64_t)blockIdx.x * a.V + v) * 32 + lane;

    // every bank value of this (v, e) first, so the loads overlap
    T u[U];
    {
      const T* up = a.u + o;
#pragma unroll
      for (int i = 0; i < U; ++i, up += a.ldim_u) u[i] = __ldg(up);
    }
    T K[PF ? U : 1];
    if constexpr (PF != 0) {
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const int64_t ro = o + (int64_t)r * a.ldim_u;
        T k = a.Cq ? a.gamma * __ldg(a.Cq + ro) : T(0);
        if (a.A) k = fma(a.alpha, __ldg(a.A + ro), k);
        if (a.B) k = fma(a.beta, __ldg(a.B + ro), k);
        K[r] = k;
      }
    }
    // the face values come from the interp kernel: wait for it (returns at
    // once after the first iteration)
    pdl_wait();
    T urv[F];
#pragma unroll
    for (int f = 0; f < F; f += 2) {
      const longlong2 pb = reinterpret_cast<const longlong2*>(pl)[f / 2];
      urv[f] = pb.x >= 0 ? a.uf[pb.x + (int64_t)v * 32] : T(0);
      if (f + 1 < F) urv[f + 1] = pb.y >= 0 ? a.uf[pb.y + (int64_t)v * 32] : T(0);
    }
    const T c[3] = {__ldg(a.cvx + v), __ldg(a.cvy + v), __ldg(a.cvz + v)};

    // R = (M1 - M3 M2) F~ + M3 F^, accumulated term by term so that only
    // the U partial sums and u stay live
    T R[U];
#pragma unroll
    for (int r = 0; r < U; ++r) R[r] = T(0);

    // common normal fluxes |S^T n| F^ at this element's flux points
    {
      T nm[G::NN];
#pragma unroll
      for (int f = 0; f < F; ++f) {
        // scaled normals fetched where first used (16 bytes at a time)
        if ((f * D) % G::VW == 0) lds16<T, 1>(gl + G::ON + f * D, nm + f * D);
        T ul = T(0);
#pragma unroll
        for (int i = 0; i < U; ++i) ul = fma(op.m0[f][i], u[i], ul);
        const T* nmv = nm + f * D;
        T nc = nmv[0] * c[0];
#pragma unroll
        for (int d = 1; d < D; ++d) nc = fma(nmv[d], c[d], nc);
        T ur = urv[f];
        const int64_t pb = pl[f];
        if (pb < 0) {
          const int b = (int)(-pb - 1);
          ur = b >= a.nb ? a.halo[(int64_t)(b - a.nb) * a.V + v] : dg_ghost<T, D>(a, b, v, e, f, c, nmv, nc, ul);
        }
        // upwind flux (rusanov.mako:46-50) with the scaled normal
        const T fh = T(0.5) * nc * (ul + ur) + T(0.5) * fabs(nc) * (ul - ur);
#pragma unroll
        for (int r = 0; r < U; ++r) R[r] = fma(op.m3[r][f], fh, R[r]);
      }
    }

    // transformed flux at the solution points F~_(i,k) = (sum_kk S_ik,kk c_kk) u_k
    {
      T sm[G::NS];
#pragma unroll
      for (int k = 0; k < U; ++k)
#pragma unroll
        for (int i = 0; i < D; ++i) {
          if (((k * D + i) * D) % G::VW == 0) lds16<T, 1>(gl + G::OS + (k * D + i) * D, sm + (k * D + i) * D);
          T s = T(0);
#pragma unroll
          for (int kk = 0; kk < D; ++kk) s = fma(sm[(k * D + i) * D + kk], c[kk], s);
          const T ft = s * u[k];
#pragma unroll
          for (int r = 0; r < U; ++r) R[r] = fma(op.m132[r][i * U + k], ft, R[r]);
        }
    }

    T rj[G::NR];
    lds16<T, G::NR / G::VW>(gl + G::OR, rj);
    if constexpr (PF != 0) {
      T* op_ = a.out + o;
#pragma unroll
      for (int r = 0; r < U; ++r, op_ += a.ldim_u) *op_ = fma(a.gamma, -rj[r] * R[r], K[r]);
    } else {
      const T* ap = a.A ? a.A + o : nullptr;
      const T* bp = a.B ? a.B + o : nullptr;
      const T* cp = a.Cq ? a.Cq + o : nullptr;
      T* op_ = a.out + o;
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const T Rr = -rj[r] * R[r];
        T res = a.gamma * (cp ? Rr + __ldg(cp) : Rr);
        if (ap) res = fma(a.alpha, __ldg(ap), res);
        if (bp) res = fma(a.beta, __ldg(bp), res);
        *op_ = res;
        op_ += a.ldim_u;
        if (ap) ap += a.ldim_u;
        if (bp) bp += a.ldim_u;
        if (cp) cp += a.ldim_u;
      }
    }
  }
}

// send[s][v] = uf[sfpt[s]][v][sele[s]] for every velocity: the face values a
// neighbouring partition needs, one row per shared flux point.
template <typename T>
__global__ void __launch_bounds__(256) dg_pack_kernel(const T* __restrict__ uf, int64_t ldim_f, int V,
                                                     const int* __restrict__ sfpt, const int* __restrict__ sele,
                                                     int nsend, T* __restrict__ send) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nsend * V) return;
  const int s = (int)(t / V), v = (int)(t % V);
  send[t] = uf[aos32(sfpt[s], ldim_f, sele[s], v, V)];
}

}  // namespace dgfs
