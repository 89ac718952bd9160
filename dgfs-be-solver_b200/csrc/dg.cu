// Host side of the FR-DG residual: validation, device copies of geometry and
// boundary data, the flux-point scratch and the launches behind the C ABI.
#include <utility>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/dgfs_b200.h"
#include "dg_kernel.cuh"
#include "dg_tc.cuh"
#include "dgfs_internal.h"

using namespace dgfs;

struct dgfs_dg {
  int prec, D, U, F, V, E, nb, ngroups, device, nhalo, nsend;
  int shape;  // residual launch shape (kDgShapes)
  long long ldim_u, ldim_f;
  double cw;
  std::vector<double> m0, m132, m3, m12;  // host copies (operators travel as params)
  void *smats, *rcpdjac, *nrm, *mag, *cvx, *cvy, *cvz, *guw, *gfw, *bwall;
  int *part, *bkind, *bgroup, *bfpt, *bele, *grefl;
  double* bcvals;
  double* bcpart;  // [kBcChunks][nb][2] partial wall sums
  void* uf;        // flux-point scratch [F][ldim_f]
  void* geoblk;    // [nblk][32][GS] per-block geometry rows (T)
  int64_t* pblk;   // [nblk][32][PS] partner offsets, boundary and halo codes
  int *sfpt, *sele;  // [nsend] flux point and element of each send row
  const void* halo;  // caller's [nhalo][V] received values (dgfs_dg_set_halo)
  int* err;          // bounded-wait flag of the tensor-core residual (dgfs_dg_status)
};

constexpr int kBcChunks = 256;  // velocity chunks of the wall-sum reduction
constexpr int kVpt = 8;         // velocities per warp in the interp kernel (largest)

// Residual launch shapes: (velocities per warp, prefetch of the RK terms,
// CTAs per SM of the register budget); MB 0 = the precision's default
// (3 for FP32 p <= 2, 2 for FP32 p = 3 and FP64 p <= 2, 1 for FP64 p = 3).
struct DgShape {
  int vpt, pf, mb;
};
constexpr DgShape kDgShapes[] = {{8, 0, 0}, {8, 1, 0}, {8, 1, 2}, {16, 1, 2}, {4, 0, 0}, {4, 1, 0}, {2, 1, 0}};
constexpr int kDgNumShapes = sizeof(kDgShapes) / sizeof(kDgShapes[0]);
// Tensor-core residual shapes (FP32 only; dg_tc.cuh), numbered after the
// SIMT shapes: velocities per warp of a 128-thread CTA, Runge-Kutta terms
// always loaded ahead, CTAs per SM (0: 4 for p <= 2, 2 for p = 3, what the
// operand tiles' shared memory allows).
constexpr DgShape kDgTcShapes[] = {{8, 1, 0}, {16, 1, 0}, {4, 1, 0}, {32, 1, 0}};
constexpr int kDgNumTc = sizeof(kDgTcShapes) / sizeof(kDgTcShapes[0]);

inline int num_shapes(const dgfs_dg* h) { return kDgNumShapes + (h->prec == 32 ? kDgNumTc : 0); }
inline bool tc_shape(int idx) { return idx >= kDgNumShapes; }
inline const DgShape& shape_of(int idx) { return tc_shape(idx) ? kDgTcShapes[idx - kDgNumShapes] : kDgShapes[idx]; }
// velocities of one CTA's chunk: 8 warps x vpt (SIMT), 4 warps x vpt (tensor cores)
inline int chunk_of(int idx) { return (tc_shape(idx) ? 4 : 8) * shape_of(idx).vpt; }

namespace {

template <typename T> int upload_as(void** dst, const double* src, size_t n) {
  std::vector<T> h(n);
  for (size_t i = 0; i < n; ++i) h[i] = (T)src[i];
  if (cudaMalloc(dst, n * sizeof(T) + 16) != cudaSuccess) {
    *dst = nullptr;
    return set_error(DGFS_ERR_NOMEM, "cudaMalloc(%zu) failed", n * sizeof(T));
  }
  if (n && cudaMemcpy(*dst, h.data(), n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(cudaGetLastError()));
  return DGFS_OK;
}

int upload_int(int** dst, const int* src, size_t n) {
  if (cudaMalloc((void**)dst, n * sizeof(int) + 16) != cudaSuccess) {
    *dst = nullptr;
    return set_error(DGFS_ERR_NOMEM, "cudaMalloc(%zu) failed", n * sizeof(int));
  }
  if (n && cudaMemcpy(*dst, src, n * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(cudaGetLastError()));
  return DGFS_OK;
}

template <typename T> int upload_geom(dgfs_dg* h, const dgfs_dg_params* p) {
  const size_t D = h->D, U = h->U, F = h->F, E = h->E, V = h->V;
  int rc;
  if ((rc = upload_as<T>(&h->smats, p->smats, D * U * D * E))) return rc;
  if ((rc = upload_as<T>(&h->rcpdjac, p->rcpdjac, U * E))) return rc;
  if ((rc = upload_as<T>(&h->nrm, p->nrm, F * D * E))) return rc;
  if ((rc = upload_as<T>(&h->mag, p->mag, F * E))) return rc;
  if ((rc = upload_as<T>(&h->cvx, p->cv, V))) return rc;
  if ((rc = upload_as<T>(&h->cvy, p->cv + V, V))) return rc;
  if ((rc = upload_as<T>(&h->cvz, p->cv + 2 * V, V))) return rc;
  const size_t G = h->ngroups;
  std::vector<double> uw(3 * (G ? G : 1), 0.0), fw(V * (G ? G : 1), 0.0);
  if (G) {
    std::memcpy(uw.data(), p->guw, 3 * G * sizeof(double));
    std::memcpy(fw.data(), p->gfw, V * G * sizeof(double));
  }
  if ((rc = upload_as<T>(&h->guw, uw.data(), uw.size()))) return rc;
  if ((rc = upload_as<T>(&h->gfw, fw.data(), fw.size()))) return rc;
  // per-point wall states (cylinder walls); a neutral placeholder otherwise
  const size_t nb = h->nb;
  std::vector<double> bw(4 * (nb ? nb : 1), 1.0);
  if (nb && p->bwall) std::memcpy(bw.data(), p->bwall, 4 * nb * sizeof(double));
  if ((rc = upload_as<T>(&h->bwall, bw.data(), bw.size()))) return rc;
  return DGFS_OK;
}

// Per-block geometry rows of the residual kernel (DgGeo layout): for each
// element S[k][i][kk] = smats[i][k][kk][e], 1/|J| (zero padded), and
// |S^T n| n at the flux points; partner codes: the partner's flux-bank
// offset at v = 0 (interior), -1-b (boundary point b), -1-(nb+h) (halo row
// h).  Lanes past the last element are zero.
template <typename T, int U, int F, int D> int build_blocks(dgfs_dg* h, const dgfs_dg_params* p) {
  using G = DgGeo<T, U, F, D>;
  const int E = h->E;
  const size_t nblk = (E + 31) / 32;
  std::vector<T> g(nblk * 32 * G::GS, T(0));
  std::vector<int64_t> pb(nblk * 32 * G::PS, 0);
  for (int e = 0; e < E; ++e) {
    T* row = g.data() + (size_t)e * G::GS;
    for (int k = 0; k < U; ++k)
      for (int i = 0; i < D; ++i)
        for (int kk = 0; kk < D; ++kk)
          row[G::OS + (k * D + i) * D + kk] = (T)p->smats[(((size_t)i * U + k) * D + kk) * E + e];
    for (int k = 0; k < U; ++k) row[G::OR + k] = (T)p->rcpdjac[(size_t)k * E + e];
    for (int f = 0; f < F; ++f)
      for (int d = 0; d < D; ++d)
        row[G::ON + f * D + d] = (T)(p->mag[(size_t)f * E + e] * p->nrm[((size_t)f * D + d) * E + e]);
    int64_t* prow = pb.data() + (size_t)e * G::PS;
    for (int f = 0; f < F; ++f) {
      const int q = p->partner[(size_t)f * E + e];
      prow[f] = q >= 0 ? (int64_t)(q / E) * h->ldim_f + (int64_t)((q % E) >> 5) * h->V * 32 + ((q % E) & 31)
                       : (int64_t)q;
    }
  }
  if (cudaMalloc(&h->geoblk, g.size() * sizeof(T)) != cudaSuccess ||
      cudaMalloc((void**)&h->pblk, pb.size() * sizeof(int64_t)) != cudaSuccess)
    return set_error(DGFS_ERR_NOMEM, "block geometry allocation failed");
  if (cudaMemcpy(h->geoblk, g.data(), g.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->pblk, pb.data(), pb.size() * sizeof(int64_t), cudaMemcpyHostToDevice) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "block geometry upload: %s", cudaGetErrorString(cudaGetLastError()));
  return DGFS_OK;
}

template <typename T> DgArgs<T> make_args(const dgfs_dg* h) {
  DgArgs<T> a{};
  a.V = h->V;
  a.neles = h->E;
  a.ldim_u = h->ldim_u;
  a.ldim_f = h->ldim_f;
  a.uf = (T*)h->uf;
  a.err = h->err;
  a.smats = (const T*)h->smats;
  a.rcpdjac = (const T*)h->rcpdjac;
  a.nrm = (const T*)h->nrm;
  a.mag = (const T*)h->mag;
  a.part = h->part;
  a.cvx = (const T*)h->cvx;
  a.cvy = (const T*)h->cvy;
  a.cvz = (const T*)h->cvz;
  a.bkind = h->bkind;
  a.bgroup = h->bgroup;
  a.guw = (const T*)h->guw;
  a.gfw = (const T*)h->gfw;
  a.grefl = h->grefl;
  a.bwall = (const T*)h->bwall;
  a.bcvals = h->bcvals;
  a.nb = h->nb;
  a.geoblk = (const T*)h->geoblk;
  a.pblk = h->pblk;
  a.halo = (const T*)h->halo;
  return a;
}

template <typename T, int U, int F, int D> DgOps<T, U, F, D> make_ops(const dgfs_dg* h) {
  DgOps<T, U, F, D> o;
  for (int f = 0; f < F; ++f)
    for (int i = 0; i < U; ++i) o.m0[f][i] = (T)h->m0[f * U + i];
  for (int r = 0; r < U; ++r)
    for (int j = 0; j < D * U; ++j) o.m132[r][j] = (T)h->m132[r * D * U + j];
  for (int r = 0; r < U; ++r)
    for (int f = 0; f < F; ++f) o.m3[r][f] = (T)h->m3[r * F + f];
  return o;
}

template <typename T, int U> DgMassOps<T, U> make_mass_ops(const dgfs_dg* h) {
  DgMassOps<T, U> o;
  for (int r = 0; r < U; ++r)
    for (int i = 0; i < U; ++i) o.m12[r][i] = (T)h->m12[r * U + i];
  return o;
}

// Launch as a programmatic dependent of the previous kernel in the stream
// (dg_kernel.cuh: pdl_wait / pdl_trigger say what each kernel may do before
// its predecessor has completed); pdl = false launches in plain stream order.
template <typename... P, typename... A>
cudaError_t launch_pdl_shape(bool pdl, void (*kern)(P...), dim3 grid, int threads, int smem, cudaStream_t s,
                             A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3((unsigned)threads, 1, 1);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

template <typename... P, typename... A>
cudaError_t launch_pdl(bool pdl, void (*kern)(P...), dim3 grid, cudaStream_t s, A&&... args) {
  return launch_pdl_shape(pdl, kern, grid, 256, 0, s, std::forward<A>(args)...);
}

inline unsigned grid_for(const dgfs_dg* h, int nv) {
  const long long nblk = (h->E + 31) / 32;
  return (unsigned)((nblk * nv * 32 + 255) / 256);
}

// (element block, velocity chunk of 8 * kVpt) grid of the interp/residual
inline dim3 grid_blk(const dgfs_dg* h, int nv) {
  return dim3((unsigned)((h->E + 31) / 32), (unsigned)((nv + 8 * kVpt - 1) / (8 * kVpt)));
}

template <typename T, int U, int F, int D>
cudaError_t run_interp(const dgfs_dg* h, const void* u, int v0, int nv, cudaStream_t s) {
  DgArgs<T> a = make_args<T>(h);
  a.u = (const T*)u;
  a.v0 = v0;
  a.nv = nv;
  // the interp kernel takes the velocity chunk of the selected residual
  // shape (small meshes: more CTAs)
  const int vs = chunk_of(h->shape) / 8, vpt = vs <= 2 ? 2 : vs <= 4 ? 4 : kVpt;
  const dim3 grid((unsigned)((h->E + 31) / 32), (unsigned)((nv + 8 * vpt - 1) / (8 * vpt)));
  const DgOps<T, U, F, D> ops = make_ops<T, U, F, D>(h);
  if (vpt <= 2) return launch_pdl(true, dg_interp_kernel<T, U, F, D, 2>, grid, s, a, ops);
  if (vpt <= 4) return launch_pdl(true, dg_interp_kernel<T, U, F, D, 4>, grid, s, a, ops);
  return launch_pdl(true, dg_interp_kernel<T, U, F, D, kVpt>, grid, s, a, ops);
}

template <typename T, int U, int F, int D>
constexpr int dg_default_mb() {
  return sizeof(T) == 4 ? (U <= 9 ? 3 : 2) : (U <= 9 ? 2 : 1);
}

template <typename T, int U, int F, int D, int VPT, int PF, int MB>
cudaError_t launch_rhs(const dgfs_dg* h, const DgArgs<T>& a, int nv, cudaStream_t s) {
  constexpr int mb = MB ? MB : dg_default_mb<T, U, F, D>();
  const dim3 grid((unsigned)((h->E + 31) / 32), (unsigned)((nv + 8 * VPT - 1) / (8 * VPT)));
  // with halo rows the face values of other partitions arrive by a
  // collective on another stream: the residual then waits in plain stream
  // order for everything before it
  return launch_pdl(h->nhalo == 0, dg_residual_kernel<T, U, F, D, VPT, PF, mb>, grid, s, a,
                    make_ops<T, U, F, D>(h));
}

template <int U, int F, int D, int VPT>
cudaError_t launch_rhs_tc(const dgfs_dg* h, const DgArgs<float>& a, int nv, cudaStream_t s) {
  using TC = DgTc<U, F, D>;
  constexpr int mb = U <= 9 ? 4 : 2;
  auto kern = dg_residual_tc_kernel<U, F, D, VPT, mb>;
  static std::atomic<unsigned long long> configured{0};  // per instantiation and device
  const cudaError_t e = smem_limit_once(kern, TC::SMEM, configured);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)((h->E + 31) / 32), (unsigned)((nv + 4 * VPT - 1) / (4 * VPT)));
  return launch_pdl_shape(h->nhalo == 0, kern, grid, 128, TC::SMEM, s, a, make_ops<float, U, F, D>(h));
}

template <typename T, int U, int F, int D>
cudaError_t run_rhs(const dgfs_dg* h, const void* u, void* out, int v0, int nv, double alpha, const void* A,
                    double beta, const void* B, double gamma, const void* C, cudaStream_t s) {
  DgArgs<T> a = make_args<T>(h);
  a.u = (const T*)u;
  a.out = (T*)out;
  a.A = (const T*)A;
  a.B = (const T*)B;
  a.Cq = (const T*)C;
  a.alpha = (T)alpha;
  a.beta = (T)beta;
  a.gamma = (T)gamma;
  a.v0 = v0;
  a.nv = nv;
  if constexpr (sizeof(T) == 4) {
    switch (h->shape - kDgNumShapes) {
      case 0: return launch_rhs_tc<U, F, D, 8>(h, a, nv, s);
      case 1: return launch_rhs_tc<U, F, D, 16>(h, a, nv, s);
      case 2: return launch_rhs_tc<U, F, D, 4>(h, a, nv, s);
      case 3: return launch_rhs_tc<U, F, D, 32>(h, a, nv, s);
      default: break;
    }
  }
  switch (h->shape) {
    case 1: return launch_rhs<T, U, F, D, 8, 1, 0>(h, a, nv, s);
    case 2: return launch_rhs<T, U, F, D, 8, 1, 2>(h, a, nv, s);
    case 3: return launch_rhs<T, U, F, D, 16, 1, 2>(h, a, nv, s);
    case 4: return launch_rhs<T, U, F, D, 4, 0, 0>(h, a, nv, s);
    case 5: return launch_rhs<T, U, F, D, 4, 1, 0>(h, a, nv, s);
    case 6: return launch_rhs<T, U, F, D, 2, 1, 0>(h, a, nv, s);
    default: return launch_rhs<T, U, F, D, 8, 0, 0>(h, a, nv, s);
  }
}

template <typename T, int U, int F, int D>
cudaError_t run_invmass(const dgfs_dg* h, const void* u, void* out, int v0, int nv, cudaStream_t s) {
  DgArgs<T> a = make_args<T>(h);
  a.u = (const T*)u;
  a.out = (T*)out;
  a.v0 = v0;
  a.nv = nv;
  dg_invmass_kernel<T, U><<<grid_for(h, nv), 256, 0, s>>>(a, make_mass_ops<T, U>(h));
  return cudaGetLastError();
}

// (U, F, D) shapes compiled in: quadrilaterals of order 1, 2, 3
#define DG_DISPATCH(PREC, CALL)                                         \
  do {                                                                  \
    if (h->D == 2 && h->U == 4 && h->F == 8) {                          \
      CALL(PREC, 4, 8, 2);                                              \
    } else if (h->D == 2 && h->U == 9 && h->F == 12) {                  \
      CALL(PREC, 9, 12, 2);                                             \
    } else if (h->D == 2 && h->U == 16 && h->F == 16) {                 \
      CALL(PREC, 16, 16, 2);                                            \
    } else {                                                            \
      return set_error(DGFS_ERR_UNSUPPORTED, "no DG kernel for D=%d U=%d F=%d", h->D, h->U, h->F); \
    }                                                                   \
  } while (0)

bool supported_shape(int D, int U, int F) {
  return D == 2 && ((U == 4 && F == 8) || (U == 9 && F == 12) || (U == 16 && F == 16));
}

int check_bank(const dgfs_dg* h, const void* p, const char* what) {
  if (!p) return set_error(DGFS_ERR_INVALID, "null %s bank", what);
  const size_t esz = h->prec == 64 ? 8 : 4;
  if ((uintptr_t)p % esz) return set_error(DGFS_ERR_INVALID, "misaligned %s bank", what);
  return DGFS_OK;
}

int check_range(const dgfs_dg* h, int v0, int nv) {
  if (v0 < 0 || nv < 1 || (long long)v0 + nv > h->V)
    return set_error(DGFS_ERR_INVALID, "velocity range [%d, %d) outside 0..%d", v0, v0 + nv, h->V);
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != h->device)
    return set_error(DGFS_ERR_INVALID, "handle built on device %d used on device %d", h->device, dev);
  return DGFS_OK;
}

void free_dg(dgfs_dg* h) {
  if (!h) return;
  void* ptrs[] = {h->smats, h->rcpdjac, h->nrm, h->mag, h->cvx, h->cvy, h->cvz, h->guw, h->gfw, h->bwall,
                  h->part, h->bkind, h->bgroup, h->bfpt, h->bele, h->grefl, h->bcvals, h->bcpart,
                  h->uf, h->geoblk, h->pblk, h->sfpt, h->sele, h->err};
  for (void* q : ptrs) cudaFree(q);
  delete h;
}

}  // namespace

extern "C" int dgfs_dg_create(const dgfs_dg_params* p, dgfs_dg** out) {
  clear_error();
  if (!p || !out) return set_error(DGFS_ERR_INVALID, "null argument");
  *out = nullptr;
  if (p->precision != 32 && p->precision != 64) return set_error(DGFS_ERR_INVALID, "precision must be 32 or 64");
  if (!supported_shape(p->ndims, p->nupts, p->nfpts))
    return set_error(DGFS_ERR_UNSUPPORTED, "no DG kernel for ndims=%d nupts=%d nfpts=%d", p->ndims, p->nupts,
                     p->nfpts);
  if (p->nvars < 1 || p->neles < 1) return set_error(DGFS_ERR_INVALID, "bad sizes nvars=%d neles=%d", p->nvars, p->neles);
  if (p->soasz != 32) return set_error(DGFS_ERR_UNSUPPORTED, "DG kernels need soasz = 32, got %d", p->soasz);
  const long long nblk = (p->neles + 31) / 32;
  if (p->ldim < nblk * 32 * (long long)p->nvars)
    return set_error(DGFS_ERR_INVALID, "ldim %lld smaller than one AoSoA row", p->ldim);
  if (!p->m0 || !p->m132 || !p->m3 || !p->smats || !p->rcpdjac || !p->nrm || !p->mag || !p->partner || !p->cv)
    return set_error(DGFS_ERR_INVALID, "null operator or geometry array");
  if (p->nbfpts < 0 || p->ngroups < 0 || (p->nbfpts && (!p->bkind || !p->bgroup || !p->bfpt || !p->bele)))
    return set_error(DGFS_ERR_INVALID, "bad boundary description");
  if (p->ngroups && (!p->guw || !p->gfw)) return set_error(DGFS_ERR_INVALID, "null boundary group data");
  const int U = p->nupts, F = p->nfpts, D = p->ndims, E = p->neles;
  if (p->nhalo < 0 || p->nsend < 0 || (p->nsend && (!p->sfpt || !p->sele)))
    return set_error(DGFS_ERR_INVALID, "bad partition halo description");
  for (int i = 0; i < F * E; ++i) {
    const int q = p->partner[i];
    if (q >= 0 ? (long long)q >= (long long)F * E : (long long)(-(long long)q - 1) >= (long long)p->nbfpts + p->nhalo)
      return set_error(DGFS_ERR_INVALID, "partner entry %d = %d out of range", i, q);
  }
  for (int s = 0; s < p->nsend; ++s)
    if (p->sfpt[s] < 0 || p->sfpt[s] >= F || p->sele[s] < 0 || p->sele[s] >= E)
      return set_error(DGFS_ERR_INVALID, "bad send row %d", s);
  for (int b = 0; b < p->nbfpts; ++b) {
    if (p->bkind[b] < 0 || p->bkind[b] > BC_WALL_DIFFUSE_CYL) return set_error(DGFS_ERR_INVALID, "bad boundary kind");
    if (p->bkind[b] == BC_WALL_DIFFUSE_CYL && (!p->bwall || !(p->bwall[4 * b + 3] > 0.0)))
      return set_error(DGFS_ERR_INVALID, "cylinder wall point %d without a positive wall temperature", b);
    if (p->bgroup[b] < 0 || p->bgroup[b] >= p->ngroups) return set_error(DGFS_ERR_INVALID, "bad boundary group");
    if (p->bfpt[b] < 0 || p->bfpt[b] >= F || p->bele[b] < 0 || p->bele[b] >= E)
      return set_error(DGFS_ERR_INVALID, "bad boundary flux point");
    if (p->bkind[b] == BC_WALL_SPECULAR && !p->grefl)
      return set_error(DGFS_ERR_INVALID, "specular wall without a reflection map");
  }
  if (p->grefl)
    for (long long i = 0; i < (long long)p->ngroups * p->nvars; ++i)
      if (p->grefl[i] < 0 || p->grefl[i] >= p->nvars) return set_error(DGFS_ERR_INVALID, "bad reflection map");

  dgfs_dg* h = new dgfs_dg();
  h->prec = p->precision;
  h->D = D;
  h->U = U;
  h->F = F;
  h->V = p->nvars;
  h->E = E;
  h->nb = p->nbfpts;
  h->ngroups = p->ngroups;
  h->nhalo = p->nhalo;
  h->nsend = p->nsend;
  h->ldim_u = p->ldim;
  h->cw = p->cw;
  h->m0.assign(p->m0, p->m0 + F * U);
  h->m132.assign(p->m132, p->m132 + U * D * U);
  h->m3.assign(p->m3, p->m3 + U * F);
  if (p->m12) h->m12.assign(p->m12, p->m12 + U * U);
  const size_t esz = h->prec == 64 ? 8 : 4;
  const long long row = nblk * 32 * (long long)h->V;
  const long long ldmod = 128 / (long long)esz;
  h->ldim_f = (row + ldmod - 1) / ldmod * ldmod;
  int rc = cudaGetDevice(&h->device) == cudaSuccess ? DGFS_OK : set_error(DGFS_ERR_CUDA, "no CUDA device");
  if (!rc) rc = h->prec == 64 ? upload_geom<double>(h, p) : upload_geom<float>(h, p);
  if (!rc) rc = upload_int(&h->part, p->partner, (size_t)F * E);
  if (!rc) {
#define CALL(P, U_, F_, D_) rc = build_blocks<P, U_, F_, D_>(h, p)
    if (h->prec == 64)
      DG_DISPATCH(double, CALL);
    else
      DG_DISPATCH(float, CALL);
#undef CALL
  }
  if (!rc && h->nsend) {
    if ((rc = upload_int(&h->sfpt, p->sfpt, h->nsend)) == DGFS_OK) rc = upload_int(&h->sele, p->sele, h->nsend);
  }
  const int nb = h->nb ? h->nb : 1;
  std::vector<int> zeros(nb, 0);
  if (!rc) rc = upload_int(&h->bkind, h->nb ? p->bkind : zeros.data(), nb);
  if (!rc) rc = upload_int(&h->bgroup, h->nb ? p->bgroup : zeros.data(), nb);
  if (!rc) rc = upload_int(&h->bfpt, h->nb ? p->bfpt : zeros.data(), nb);
  if (!rc) rc = upload_int(&h->bele, h->nb ? p->bele : zeros.data(), nb);
  if (!rc) {
    const size_t n = (size_t)(p->ngroups ? p->ngroups : 1) * h->V;
    std::vector<int> refl(n, 0);
    if (p->grefl) std::memcpy(refl.data(), p->grefl, (size_t)p->ngroups * h->V * sizeof(int));
    rc = upload_int(&h->grefl, refl.data(), n);
  }
  if (!rc) {
    std::vector<double> ones(2 * nb, 1.0);  // frfs initialises bc_vals to 1 (inters.py:203)
    if (cudaMalloc((void**)&h->bcvals, 2 * nb * sizeof(double)) != cudaSuccess ||
        cudaMemcpy(h->bcvals, ones.data(), 2 * nb * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc((void**)&h->bcpart, (size_t)kBcChunks * 2 * nb * sizeof(double)) != cudaSuccess)
      rc = set_error(DGFS_ERR_NOMEM, "boundary value allocation failed");
  }
  if (!rc) {
    if (cudaMalloc((void**)&h->err, sizeof(int)) != cudaSuccess || cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess)
      rc = set_error(DGFS_ERR_NOMEM, "error flag allocation failed");
  }
  if (!rc) {
    const size_t bytes = (size_t)F * h->ldim_f * esz;
    if (cudaMalloc(&h->uf, bytes) != cudaSuccess)
      rc = set_error(DGFS_ERR_NOMEM, "cudaMalloc(%zu) for the flux-point scratch failed", bytes);
    else
      cudaMemset(h->uf, 0, bytes);
  }
  if (rc) {
    free_dg(h);
    return rc;
  }
  *out = h;
  return DGFS_OK;
}

extern "C" int dgfs_dg_destroy(dgfs_dg* h) {
  clear_error();
  free_dg(h);
  return DGFS_OK;
}

extern "C" int dgfs_dg_interp(dgfs_dg* h, const void* u, int v0, int nv, void* stream) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  int rc = check_bank(h, u, "solution");
  if (!rc) rc = check_range(h, v0, nv);
  if (rc) return rc;
  cudaError_t e = cudaSuccess;
#define CALL(P, U, F, D) e = run_interp<P, U, F, D>(h, u, v0, nv, (cudaStream_t)stream)
  if (h->prec == 64)
    DG_DISPATCH(double, CALL);
  else
    DG_DISPATCH(float, CALL);
#undef CALL
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "DG interp launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_dg_updatebc(dgfs_dg* h, int v0, int nv, int reset, void* stream) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  int rc = check_range(h, v0, nv);
  if (rc) return rc;
  if (h->nb == 0) return DGFS_OK;
  const int chunk = (nv + kBcChunks - 1) / kBcChunks;
  const int nchunks = (nv + chunk - 1) / chunk;
  const dim3 grid((unsigned)nchunks, (unsigned)((h->nb + 31) / 32));
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if (h->prec == 64) {
    DgArgs<double> a = make_args<double>(h);
    a.v0 = v0;
    a.nv = nv;
    e = launch_pdl(true, dg_bcsum_kernel<double, 2>, grid, s, a, (const int*)h->bfpt, (const int*)h->bele, h->nb, h->cw,
                   chunk, h->bcpart);
  } else {
    DgArgs<float> a = make_args<float>(h);
    a.v0 = v0;
    a.nv = nv;
    e = launch_pdl(true, dg_bcsum_kernel<float, 2>, grid, s, a, (const int*)h->bfpt, (const int*)h->bele, h->nb, h->cw,
                   chunk, h->bcpart);
  }
  if (e == cudaSuccess)
    e = launch_pdl(true, dg_bcsum_finish_kernel, dim3((unsigned)((h->nb + 7) / 8)), s, (const int*)h->bkind, h->nb,
                   nchunks, (const double*)h->bcpart, h->bcvals, reset);
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "DG boundary update launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_dg_rhs(dgfs_dg* h, const void* u, void* out, int v0, int nv, double alpha, const void* A,
                           double beta, const void* B, double gamma, const void* C, void* stream) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  int rc = check_bank(h, u, "solution");
  if (!rc) rc = check_bank(h, out, "output");
  if (!rc) rc = check_range(h, v0, nv);
  if (rc) return rc;
  if (out == u) return set_error(DGFS_ERR_INVALID, "output bank must differ from the solution bank");
  if (h->nhalo && !h->halo) return set_error(DGFS_ERR_INVALID, "partition faces without a halo buffer (dgfs_dg_set_halo)");
  if (!std::isfinite(alpha) || !std::isfinite(beta) || !std::isfinite(gamma))
    return set_error(DGFS_ERR_INVALID, "non-finite combination coefficient");
  cudaError_t e = cudaSuccess;
#define CALL(P, U, F, D) e = run_rhs<P, U, F, D>(h, u, out, v0, nv, alpha, A, beta, B, gamma, C, (cudaStream_t)stream)
  if (h->prec == 64)
    DG_DISPATCH(double, CALL);
  else
    DG_DISPATCH(float, CALL);
#undef CALL
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "DG residual launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_dg_invmass(dgfs_dg* h, const void* u, void* out, int v0, int nv, void* stream) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  if (h->m12.empty()) return set_error(DGFS_ERR_INVALID, "handle created without the M12 operator");
  int rc = check_bank(h, u, "solution");
  if (!rc) rc = check_bank(h, out, "output");
  if (!rc) rc = check_range(h, v0, nv);
  if (rc) return rc;
  if (out == u) return set_error(DGFS_ERR_INVALID, "output bank must differ from the solution bank");
  cudaError_t e = cudaSuccess;
#define CALL(P, U, F, D) e = run_invmass<P, U, F, D>(h, u, out, v0, nv, (cudaStream_t)stream)
  if (h->prec == 64)
    DG_DISPATCH(double, CALL);
  else
    DG_DISPATCH(float, CALL);
#undef CALL
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "DG invmass launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_dg_pack(dgfs_dg* h, void* send, void* stream) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  if (!h->nsend) return DGFS_OK;
  int rc = check_bank(h, send, "send");
  if (rc) return rc;
  const long long n = (long long)h->nsend * h->V;
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (h->prec == 64)
    dg_pack_kernel<double><<<grid, 256, 0, (cudaStream_t)stream>>>((const double*)h->uf, h->ldim_f, h->V, h->sfpt,
                                                                    h->sele, h->nsend, (double*)send);
  else
    dg_pack_kernel<float><<<grid, 256, 0, (cudaStream_t)stream>>>((const float*)h->uf, h->ldim_f, h->V, h->sfpt,
                                                                   h->sele, h->nsend, (float*)send);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "DG pack launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_dg_set_halo(dgfs_dg* h, const void* recv) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  if (h->nhalo && !recv) return set_error(DGFS_ERR_INVALID, "null halo buffer");
  int rc = recv ? check_bank(h, recv, "halo") : DGFS_OK;
  if (rc) return rc;
  h->halo = recv;
  return DGFS_OK;
}

extern "C" int dgfs_dg_num_variants(const dgfs_dg* h, int* count) {
  clear_error();
  if (!h || !count) return set_error(DGFS_ERR_INVALID, "null argument");
  *count = num_shapes(h);
  return DGFS_OK;
}

extern "C" int dgfs_dg_variant_info(const dgfs_dg* h, int idx, int* vpt, int* prefetch, int* min_ctas_per_sm) {
  clear_error();
  if (!h || !vpt || !prefetch || !min_ctas_per_sm) return set_error(DGFS_ERR_INVALID, "null argument");
  if (idx < 0 || idx >= num_shapes(h))
    return set_error(DGFS_ERR_INVALID, "variant %d outside 0..%d", idx, num_shapes(h) - 1);
  const DgShape& sh = shape_of(idx);
  *vpt = sh.vpt;
  *prefetch = sh.pf;
  if (tc_shape(idx))
    *min_ctas_per_sm = h->U <= 9 ? 4 : 2;
  else
    *min_ctas_per_sm = sh.mb ? sh.mb : (h->prec == 32 ? (h->U <= 9 ? 3 : 2) : (h->U <= 9 ? 2 : 1));
  return DGFS_OK;
}

extern "C" int dgfs_dg_variant_tc(const dgfs_dg* h, int idx, int* tensor_cores) {
  clear_error();
  if (!h || !tensor_cores) return set_error(DGFS_ERR_INVALID, "null argument");
  if (idx < 0 || idx >= num_shapes(h))
    return set_error(DGFS_ERR_INVALID, "variant %d outside 0..%d", idx, num_shapes(h) - 1);
  *tensor_cores = tc_shape(idx) ? 1 : 0;
  return DGFS_OK;
}

extern "C" int dgfs_dg_status(dgfs_dg* h, void* stream, int* flag) {
  clear_error();
  if (!h || !flag) return set_error(DGFS_ERR_INVALID, "null argument");
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
  int v = 0;
  if (cudaMemcpy(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "error flag: %s", cudaGetErrorString(cudaGetLastError()));
  *flag = v;
  if (v) return set_error(DGFS_ERR_CUDA, "a tensor-core DG residual launch gave up waiting for its MMAs (flag %d)", v);
  return DGFS_OK;
}

extern "C" int dgfs_dg_select(dgfs_dg* h, int idx) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  if (idx < 0 || idx >= num_shapes(h))
    return set_error(DGFS_ERR_INVALID, "variant %d outside 0..%d", idx, num_shapes(h) - 1);
  h->shape = idx;
  return DGFS_OK;
}

extern "C" int dgfs_dg_bcvals(const dgfs_dg* h, double* host, int n) {
  clear_error();
  if (!h || !host) return set_error(DGFS_ERR_INVALID, "null argument");
  if (n < 2 * h->nb) return set_error(DGFS_ERR_INVALID, "buffer holds %d values, need %d", n, 2 * h->nb);
  if (h->nb && cudaMemcpy(host, h->bcvals, 2 * h->nb * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(cudaGetLastError()));
  return DGFS_OK;
}

extern "C" int dgfs_dg_fpts(const dgfs_dg* h, void** ptr, long long* ldim) {
  clear_error();
  if (!h || !ptr || !ldim) return set_error(DGFS_ERR_INVALID, "null argument");
  *ptr = h->uf;
  *ldim = h->ldim_f;
  return DGFS_OK;
}
