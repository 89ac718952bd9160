// Host side of the fast-spectral VHS operator: parameter validation, the
// precomputed tables of frfs's perform_precomputation
// (frfs/solvers/dgfs/scattering.py:67-224, vhs-gll.mako:45-101) and the
// cluster-kernel dispatch behind the C ABI in include/dgfs_b200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"
#include "vhs_push.cuh"
#include "vhs_cube.cuh"
#include "vhs_pair.cuh"

namespace dgfs {

// ---------------------------------------------------------------------------
// Twiddle table: exp(2 pi i m / 96), m < 96, computed in long double
// ---------------------------------------------------------------------------
static std::mutex g_tw_mutex;
static bool g_tw_ready[64];

static int init_twiddles(int dev) {
  std::lock_guard<std::mutex> lk(g_tw_mutex);
  if (dev >= 0 && dev < 64 && g_tw_ready[dev]) return DGFS_OK;
  double t64[2 * kTwBase];
  float t32[2 * kTwBase];
  const long double twopi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < kTwBase; ++m) {
    const long double ang = twopi * (long double)m / (long double)kTwBase;
    t64[2 * m] = (double)cosl(ang);
    t64[2 * m + 1] = (double)sinl(ang);
    t32[2 * m] = (float)cosl(ang);
    t32[2 * m + 1] = (float)sinl(ang);
  }
  if (cudaMemcpyToSymbol(c_tw64, t64, sizeof(t64)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_tw32, t32, sizeof(t32)) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "twiddle upload failed: %s", cudaGetErrorString(cudaGetLastError()));
  if (dev >= 0 && dev < 64) g_tw_ready[dev] = true;
  return DGFS_OK;
}

// ---------------------------------------------------------------------------
// Kernel variants
// ---------------------------------------------------------------------------
struct VhsVariant {
  int prec, N, C, db, minb, threads, push;
  size_t smem;
  size_t scratch_cx;  // two-CTA kernel: complex scratch per cluster
  const void* fn;
  cudaError_t (*launch32)(const VhsArgs<float>&, int, cudaStream_t);
  cudaError_t (*launch64)(const VhsArgs<double>&, int, cudaStream_t);
};

template <typename T, int N, int C, bool DB, int MINB>
static cudaError_t launch_vhs(const VhsArgs<T>& a, int nclusters, cudaStream_t s) {
  using G = VhsGeom<N, C, DB>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nclusters * C, 1, 1);
  cfg.blockDim = dim3(G::NT, 1, 1);
  cfg.dynamicSmemBytes = G::SMEM_CX * sizeof(cx<T>);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, vhs_cluster_kernel<T, N, C, DB, MINB>, a);
}

template <typename T, int N, int C, bool DB, int MINB> static VhsVariant make_variant() {
  using G = VhsGeom<N, C, DB>;
  VhsVariant v{};
  v.prec = sizeof(T) == 8 ? 64 : 32;
  v.N = N;
  v.C = C;
  v.db = DB ? 1 : 0;
  v.minb = MINB;
  v.threads = G::NT;
  v.smem = G::SMEM_CX * sizeof(cx<T>);
  v.fn = (const void*)vhs_cluster_kernel<T, N, C, DB, MINB>;
  if constexpr (sizeof(T) == 8) v.launch64 = launch_vhs<double, N, C, DB, MINB>;
  else v.launch32 = launch_vhs<float, N, C, DB, MINB>;
  return v;
}

template <typename T, int N, int C, int MINB>
static cudaError_t launch_push(const VhsArgs<T>& a, int nclusters, cudaStream_t s) {
  using P = PushGeom<N, C>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nclusters * C, 1, 1);
  cfg.blockDim = dim3(P::NT, 1, 1);
  cfg.dynamicSmemBytes = P::SMEM_CX * sizeof(cx<T>);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, vhs_push_kernel<T, N, C, MINB>, a);
}

template <typename T, int N, int C, int MINB> static VhsVariant make_push() {
  using P = PushGeom<N, C>;
  VhsVariant v{};
  v.prec = sizeof(T) == 8 ? 64 : 32;
  v.N = N;
  v.C = C;
  v.db = 1;
  v.push = 1;
  v.minb = MINB;
  v.threads = P::NT;
  v.smem = P::SMEM_CX * sizeof(cx<T>);
  v.fn = (const void*)vhs_push_kernel<T, N, C, MINB>;
  if constexpr (sizeof(T) == 8) v.launch64 = launch_push<double, N, C, MINB>;
  else v.launch32 = launch_push<float, N, C, MINB>;
  return v;
}

template <int N, bool IL1> static cudaError_t launch_cube(const VhsArgs<float>& a, int nctas, cudaStream_t s) {
  using G = CubeGeom<N>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nctas, 1, 1);
  cfg.blockDim = dim3(G::NT, 1, 1);
  cfg.dynamicSmemBytes = G::SMEM_CX * sizeof(cx<float>);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 1;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, vhs_cube_kernel<N, IL1>, a);
}

// single-CTA kernel (FP32; kind 2 in dgfs_vhs_variant_kind); IL1: the
// first pass of every (p, q) transforms a thread's two lines together
// (more ILP, more registers; db reports it)
template <int N, bool IL1> static VhsVariant make_cube() {
  using G = CubeGeom<N>;
  VhsVariant v{};
  v.prec = 32;
  v.N = N;
  v.C = 1;
  v.db = IL1 ? 1 : 0;
  v.push = 2;
  v.minb = 1;
  v.threads = G::NT;
  v.smem = G::SMEM_CX * sizeof(cx<float>);
  v.fn = (const void*)vhs_cube_kernel<N, IL1>;
  v.launch32 = launch_cube<N, IL1>;
  return v;
}

template <typename T, int N, int LPT>
static cudaError_t launch_pair(const VhsArgs<T>& a, int nclusters, cudaStream_t s) {
  using G = PairGeom<T, N, LPT>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nclusters * 2, 1, 1);
  cfg.blockDim = dim3(G::NT, 1, 1);
  cfg.dynamicSmemBytes = G::SMEM_CX * sizeof(cx<T>);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, vhs_pair_kernel<T, N, LPT>, a);
}

// two-CTA kernel (FP32 N = 32, FP64 N = 24; kind 3 in dgfs_vhs_variant_kind);
// LPT lines per main thread and pass (db reports LPT - 1)
template <typename T, int N, int LPT> static VhsVariant make_pair() {
  using G = PairGeom<T, N, LPT>;
  VhsVariant v{};
  v.prec = sizeof(T) == 8 ? 64 : 32;
  v.N = N;
  v.C = 2;
  v.db = LPT - 1;
  v.push = 3;
  v.minb = 1;
  v.threads = G::NT;
  v.smem = G::SMEM_CX * sizeof(cx<T>);
  v.scratch_cx = G::SCRATCH;
  v.fn = (const void*)vhs_pair_kernel<T, N, LPT>;
  if constexpr (sizeof(T) == 8) v.launch64 = launch_pair<T, N, LPT>;
  else v.launch32 = launch_pair<T, N, LPT>;
  return v;
}

// Compiled launch shapes: (precision, N, cluster size, double-buffered
// exchange, minimum CTAs per SM for the register budget).  The first entry
// of each (precision, N) family is the default (FP32 N = 24: the single-CTA
// kernel, 5.2 ms against 20 ms for the best cluster shape on 576 points;
// FP64 N = 24 and FP32 N = 32: the two-CTA kernel, 15 ms against 50 ms and
// 552 ms against 1,695 ms); the autotuner times the rest.
static const std::vector<VhsVariant>& variants() {
  static const std::vector<VhsVariant> v = {
      make_push<double, 8, 1, 4>(),             make_push<double, 16, 4, 2>(),
      make_push<double, 16, 2, 1>(),            make_pair<double, 24, 1>(),
      make_pair<double, 24, 2>(),               make_push<double, 24, 8, 1>(),
      make_push<double, 24, 12, 1>(),           make_push<double, 32, 16, 1>(),
      make_push<float, 8, 1, 4>(),              make_push<float, 16, 2, 2>(),
      make_push<float, 16, 4, 4>(),             make_cube<24, false>(),
      make_push<float, 24, 8, 2>(),             make_push<float, 24, 4, 1>(),
      make_push<float, 24, 12, 3>(),            make_pair<float, 32, 2>(),
      make_pair<float, 32, 1>(),
      make_push<float, 32, 16, 2>(),
      make_push<float, 32, 8, 1>(),             make_cube<8, false>(),
      make_cube<16, false>(),                   make_cube<16, true>(),
      make_cube<24, true>(),
      make_variant<double, 8, 1, true, 4>(),    make_variant<double, 8, 2, true, 8>(),
      make_variant<double, 16, 4, true, 2>(),   make_variant<double, 16, 2, true, 1>(),
      make_variant<double, 16, 4, false, 3>(),
      make_variant<double, 24, 8, true, 1>(),   make_variant<double, 24, 8, false, 1>(),
      make_variant<double, 24, 12, false, 2>(), make_variant<double, 24, 6, false, 1>(),
      make_variant<double, 32, 16, true, 1>(),  make_variant<double, 32, 16, false, 1>(),
      make_variant<float, 8, 1, true, 4>(),     make_variant<float, 8, 2, true, 8>(),
      make_variant<float, 16, 2, true, 2>(),    make_variant<float, 16, 1, true, 1>(),
      make_variant<float, 16, 4, true, 4>(),    make_variant<float, 16, 4, false, 6>(),
      make_variant<float, 24, 8, true, 2>(),    make_variant<float, 24, 4, true, 1>(),
      make_variant<float, 24, 4, false, 2>(),   make_variant<float, 24, 6, false, 2>(),
      make_variant<float, 24, 8, false, 3>(),   make_variant<float, 24, 12, false, 4>(),
      make_variant<float, 32, 16, true, 2>(),   make_variant<float, 32, 8, true, 1>(),
      make_variant<float, 32, 8, false, 1>(),   make_variant<float, 32, 16, false, 3>(),
  };
  return v;
}

static std::vector<const VhsVariant*> family(int prec, int N) {
  std::vector<const VhsVariant*> out;
  for (const auto& v : variants())
    if (v.prec == prec && v.N == N) out.push_back(&v);
  return out;
}

}  // namespace dgfs

using namespace dgfs;

struct dgfs_vhs {
  int N, P, M, prec, V, device, project;
  double prefac;
  std::vector<const VhsVariant*> fam;  // compiled shapes for (prec, N)
  int vidx;                            // selected entry of fam
  const VhsVariant* var;
  int max_clusters;
  void* phase;   // cx<T> [P][M][3][N]
  void* w1;      // T [P][V]
  void* b2;      // T [V]
  void* w1t;     // T [P][N][N*N] (w1 with the last axis outermost)
  void* b2t;     // T [N][N*N]
  double* ginv;  // [25]
  double* cvec;  // [3][V]
  void* fc;      // scratch: gain spectrum, one N^3 complex slice per cluster
  size_t fc_bytes;
  void* fcp;     // single-CTA kernel: partial gain spectra of split points (kCubeSlices per CTA)
  size_t fcp_bytes;
  int* pdone;    // ... and the chunk counters (kCubeSlices / 2 per CTA, zero between launches)
  int pdone_n;
  int* err;      // device flag: a bounded wait in the kernel gave up
};

// Occupancy of variant v (clusters that can be resident at once), or an
// error if it cannot run on this device.
static int variant_clusters(const dgfs_vhs* h, const VhsVariant* v, int* ncl) {
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  if ((int)v->smem > maxsm)
    return set_error(DGFS_ERR_UNSUPPORTED, "VHS kernel Nv=%d cluster=%d needs %zu B shared memory (device max %d)",
                     h->N, v->C, v->smem, maxsm);
  if (cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v->smem) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "cudaFuncSetAttribute(smem): %s", cudaGetErrorString(cudaGetLastError()));
  if (v->C > 8 && cudaFuncSetAttribute(v->fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "non-portable cluster size %d refused: %s", v->C,
                     cudaGetErrorString(cudaGetLastError()));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(v->C, 1, 1);
  cfg.blockDim = dim3(v->threads, 1, 1);
  cfg.dynamicSmemBytes = v->smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = v->C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  *ncl = 0;
  if (cudaOccupancyMaxActiveClusters(ncl, v->fn, &cfg) != cudaSuccess || *ncl <= 0) {
    cudaGetLastError();
    return set_error(DGFS_ERR_UNSUPPORTED, "cluster size %d cannot be scheduled", v->C);
  }
  return DGFS_OK;
}

static int select_index(dgfs_vhs* h, int idx) {
  if (idx < 0 || idx >= (int)h->fam.size())
    return set_error(DGFS_ERR_INVALID, "variant %d outside 0..%d", idx, (int)h->fam.size() - 1);
  const VhsVariant* v = h->fam[idx];
  int ncl = 0, rc = variant_clusters(h, v, &ncl);
  if (rc) return rc;
  const size_t esz = h->prec == 64 ? 16 : 8;
  // gain-spectrum scratch: one N^3 complex slice per cluster, or for the
  // two-CTA kernel the half spectra of F and fC and the staging buffers
  const size_t need = v->push == 3 ? (size_t)ncl * v->scratch_cx * esz
                                   : (size_t)ncl * v->C * (size_t)h->N * h->N * h->N / v->C * esz;
  if (need > h->fc_bytes) {
    cudaFree(h->fc);
    h->fc = nullptr;
    h->fc_bytes = 0;
    if (cudaMalloc(&h->fc, need) != cudaSuccess)
      return set_error(DGFS_ERR_NOMEM, "cudaMalloc(%zu) for the gain-spectrum scratch failed", need);
    h->fc_bytes = need;
  }
  if (v->push == 2) {
    // a launch on few points splits them into radial-node chunks: up to
    // kCubeSlices items per CTA, each with its own partial-spectrum slice,
    // and (at least 2 chunks per point) up to kCubeSlices / 2 points per CTA
    // with a chunk counter
    const size_t needp = (size_t)kCubeSlices * ncl * (size_t)h->N * h->N * h->N * esz;
    if (needp > h->fcp_bytes) {
      cudaFree(h->fcp);
      h->fcp = nullptr;
      h->fcp_bytes = 0;
      if (cudaMalloc(&h->fcp, needp) != cudaSuccess)
        return set_error(DGFS_ERR_NOMEM, "cudaMalloc(%zu) for the partial-spectrum scratch failed", needp);
      h->fcp_bytes = needp;
    }
    const int npd = kCubeSlices / 2 * ncl;
    if (npd > h->pdone_n) {
      cudaFree(h->pdone);
      h->pdone = nullptr;
      h->pdone_n = 0;
      if (cudaMalloc((void**)&h->pdone, (size_t)npd * sizeof(int)) != cudaSuccess)
        return set_error(DGFS_ERR_NOMEM, "cudaMalloc for the chunk counters failed");
      if (cudaMemset(h->pdone, 0, (size_t)npd * sizeof(int)) != cudaSuccess)
        return set_error(DGFS_ERR_CUDA, "cudaMemset of the chunk counters failed");
      h->pdone_n = npd;
    }
  }
  h->vidx = idx;
  h->var = v;
  h->max_clusters = ncl;
  return DGFS_OK;
}

// First runnable variant, or the first with the requested cluster size.
static int select_variant(dgfs_vhs* h, int C) {
  int first_err = 0;
  for (int i = 0; i < (int)h->fam.size(); ++i) {
    if (C > 0 && h->fam[i]->C != C) continue;
    int rc = select_index(h, i);
    if (!rc) return DGFS_OK;
    if (!first_err) first_err = rc;
  }
  if (first_err) return first_err;
  return set_error(DGFS_ERR_UNSUPPORTED, "no VHS kernel for Nv=%d precision=%d cluster=%d", h->N, h->prec, C);
}

template <typename T> static int upload(void** dst, const std::vector<T>& src) {
  if (cudaMalloc(dst, src.size() * sizeof(T)) != cudaSuccess) {
    *dst = nullptr;
    return set_error(DGFS_ERR_NOMEM, "cudaMalloc(%zu) failed", src.size() * sizeof(T));
  }
  if (cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "cudaMemcpy failed: %s", cudaGetErrorString(cudaGetLastError()));
  return DGFS_OK;
}

// sinc as defined by the reference kernels (vhs-gll.mako:11-14)
static double ref_sinc(double s) { return std::sin(s + 1e-15) / (s + 1e-15); }

static bool invert5(const double* A, double* X) {
  double a[5][10];
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 10; ++j) a[i][j] = j < 5 ? A[i * 5 + j] : (j - 5 == i ? 1.0 : 0.0);
  for (int c = 0; c < 5; ++c) {
    int piv = c;
    for (int r = c + 1; r < 5; ++r)
      if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
    if (std::fabs(a[piv][c]) < 1e-300) return false;
    if (piv != c)
      for (int j = 0; j < 10; ++j) std::swap(a[c][j], a[piv][j]);
    const double d = a[c][c];
    for (int j = 0; j < 10; ++j) a[c][j] /= d;
    for (int r = 0; r < 5; ++r)
      if (r != c) {
        const double f = a[r][c];
        for (int j = 0; j < 10; ++j) a[r][j] -= f * a[c][j];
      }
  }
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) X[i * 5 + j] = a[i][j + 5];
  return true;
}

template <typename T> static int build_tables(dgfs_vhs* h, const dgfs_vhs_params* p) {
  const int N = h->N, P = h->P, M = h->M, V = h->V;
  const double L = p->L, pi = 3.14159265358979323846;
  std::vector<double> l0(N);
  for (int k = 0; k < N; ++k) l0[k] = k < N / 2 ? k : k - N;  // scattering.py:79

  std::vector<cx<T>> phase((size_t)P * M * 3 * N);
  for (int ip = 0; ip < P; ++ip) {
    const double fac = pi / L * p->qz[ip] / 2.;  // vhs-gll.mako:58
    for (int iq = 0; iq < M; ++iq)
      for (int ax = 0; ax < 3; ++ax)
        for (int k = 0; k < N; ++k) {
          const double ang = fac * (p->sz[iq * 3 + ax] * l0[k]);
          cx<T> e;
          e.x = (T)std::cos(ang);
          e.y = (T)std::sin(ang);
          phase[((size_t)(ip * M + iq) * 3 + ax) * N + k] = e;
        }
  }
  std::vector<T> w1((size_t)P * V), b2(V);
  for (int v = 0; v < V; ++v) {
    const double lx = l0[v / (N * N)], ly = l0[(v % (N * N)) / N], lz = l0[v % N];
    const double cSqr = std::sqrt(lx * lx + ly * ly + lz * lz);  // vhs-gll.mako:84-86
    double bsum = 0.;
    for (int ip = 0; ip < P; ++ip) {
      const double qz = p->qz[ip], qw = p->qw[ip];
      const double b1 = std::pow(qz, p->gamma + 2.) * 4 * pi * ref_sinc(pi / L * qz / 2. * cSqr);
      bsum += qw * std::pow(qz, p->gamma + 2.) * 16 * pi * pi * ref_sinc(pi / L * qz * cSqr);
      w1[(size_t)ip * V + v] = (T)(2. * qw * p->sw / V * b1);  // computeQG, vhs-gll.mako:194
    }
    b2[v] = (T)bsum;
  }
  // the same tables with the last axis outermost: a thread that owns line
  // (k1, k2) reads element k3 at k3 N^2 + k1 N + k2, so a warp's 32 lines
  // read 32 consecutive entries
  std::vector<T> w1t((size_t)P * V), b2t(V);
  for (int ip = 0; ip < P; ++ip)
    for (int l = 0; l < N * N; ++l)
      for (int k = 0; k < N; ++k) w1t[((size_t)ip * N + k) * N * N + l] = w1[(size_t)ip * V + (size_t)l * N + k];
  for (int l = 0; l < N * N; ++l)
    for (int k = 0; k < N; ++k) b2t[(size_t)k * N * N + l] = b2[(size_t)l * N + k];
  int rc;
  if ((rc = upload(&h->phase, phase)) || (rc = upload(&h->w1, w1)) || (rc = upload(&h->b2, b2)) ||
      (rc = upload(&h->w1t, w1t)) || (rc = upload(&h->b2t, b2t)))
    return rc;

  if (h->project) {
    // velocity grid (frfs/solvers/dgfs/velocitymesh.py:73-85) and the Gram
    // matrix of phi = (1, cx, cy, cz, |c|^2) over it
    std::vector<double> c0(N), cv((size_t)3 * V);
    for (int i = 0; i < N; ++i) c0[i] = -L + L / N + i * (2.0 * L / N);
    double G[25] = {0}, Gi[25];
    for (int v = 0; v < V; ++v) {
      const double c[3] = {c0[v / (N * N)], c0[(v % (N * N)) / N], c0[v % N]};
      for (int a = 0; a < 3; ++a) cv[(size_t)a * V + v] = c[a];
      const double phi[5] = {1.0, c[0], c[1], c[2], c[0] * c[0] + c[1] * c[1] + c[2] * c[2]};
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) G[i * 5 + j] += phi[i] * phi[j];
    }
    if (!invert5(G, Gi)) return set_error(DGFS_ERR_INVALID, "singular moment Gram matrix");
    std::vector<double> gi(Gi, Gi + 25);
    if ((rc = upload((void**)&h->ginv, gi)) || (rc = upload((void**)&h->cvec, cv))) return rc;
  }
  return DGFS_OK;
}

static void free_handle(dgfs_vhs* h) {
  if (!h) return;
  cudaFree(h->phase);
  cudaFree(h->w1);
  cudaFree(h->b2);
  cudaFree(h->w1t);
  cudaFree(h->b2t);
  cudaFree(h->ginv);
  cudaFree(h->cvec);
  cudaFree(h->fc);
  cudaFree(h->fcp);
  cudaFree(h->pdone);
  cudaFree(h->err);
  delete h;
}

extern "C" int dgfs_vhs_create(const dgfs_vhs_params* p, dgfs_vhs** out) {
  clear_error();
  if (!p || !out) return set_error(DGFS_ERR_INVALID, "null argument");
  *out = nullptr;
  if (p->Nv != 8 && p->Nv != 16 && p->Nv != 24 && p->Nv != 32)
    return set_error(DGFS_ERR_UNSUPPORTED, "Nv=%d not supported (8, 16, 24, 32)", p->Nv);
  if (p->precision != 32 && p->precision != 64)
    return set_error(DGFS_ERR_INVALID, "precision must be 32 or 64, got %d", p->precision);
  if (p->Nrho < 1 || p->M < 1 || p->Nrho > 4096 || p->M > 4096)
    return set_error(DGFS_ERR_INVALID, "bad quadrature sizes Nrho=%d M=%d", p->Nrho, p->M);
  if (!p->qz || !p->qw || !p->sz) return set_error(DGFS_ERR_INVALID, "null quadrature array");
  if (!(p->L > 0) || !std::isfinite(p->L)) return set_error(DGFS_ERR_INVALID, "bad L");
  if (!std::isfinite(p->prefactor) || !std::isfinite(p->gamma) || !std::isfinite(p->sw))
    return set_error(DGFS_ERR_INVALID, "non-finite scalar parameter");
  for (int i = 0; i < p->Nrho; ++i)
    if (!std::isfinite(p->qz[i]) || !std::isfinite(p->qw[i]))
      return set_error(DGFS_ERR_INVALID, "non-finite radial quadrature");
  for (int i = 0; i < 3 * p->M; ++i)
    if (!std::isfinite(p->sz[i])) return set_error(DGFS_ERR_INVALID, "non-finite spherical design");

  dgfs_vhs* h = new dgfs_vhs();
  h->N = p->Nv;
  h->P = p->Nrho;
  h->M = p->M;
  h->prec = p->precision;
  h->V = p->Nv * p->Nv * p->Nv;
  h->prefac = p->prefactor;
  h->project = p->project ? 1 : 0;
  if (cudaGetDevice(&h->device) != cudaSuccess) {
    delete h;
    return set_error(DGFS_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(cudaGetLastError()));
  }
  h->fam = family(h->prec, h->N);
  int rc = init_twiddles(h->device);
  if (!rc && (cudaMalloc((void**)&h->err, sizeof(int)) != cudaSuccess ||
              cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess))
    rc = set_error(DGFS_ERR_NOMEM, "error flag allocation failed");
  if (!rc) rc = select_variant(h, p->cluster);
  if (!rc) rc = h->prec == 64 ? build_tables<double>(h, p) : build_tables<float>(h, p);
  if (rc) {
    free_handle(h);
    return rc;
  }
  *out = h;
  return DGFS_OK;
}

extern "C" int dgfs_vhs_destroy(dgfs_vhs* h) {
  clear_error();
  free_handle(h);
  return DGFS_OK;
}

extern "C" int dgfs_vhs_set_cluster(dgfs_vhs* h, int cluster) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  const int old = h->vidx;
  int rc = select_variant(h, cluster);
  if (rc) {
    const int keep = rc;
    std::string msg = dgfs_last_error();
    select_index(h, old);
    return set_error(keep, "%s", msg.c_str());
  }
  return DGFS_OK;
}

extern "C" int dgfs_vhs_status(dgfs_vhs* h, void* stream, int* flag) {
  clear_error();
  if (!h || !flag) return set_error(DGFS_ERR_INVALID, "null argument");
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
  int v = 0;
  if (cudaMemcpy(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "error flag: %s", cudaGetErrorString(cudaGetLastError()));
  *flag = v;
  if (v) return set_error(DGFS_ERR_CUDA, "a VHS launch gave up waiting for cluster data (flag %d)", v);
  return DGFS_OK;
}

extern "C" int dgfs_vhs_check_wait(dgfs_vhs* h, long long limit_ns, void* stream) {
  clear_error();
  if (limit_ns < 0 || limit_ns > 10000000000ll) return set_error(DGFS_ERR_INVALID, "limit_ns=%lld outside [0, 1e10]", limit_ns);
  if (!h) return noalloc_check_wait((unsigned long long)limit_ns, stream);
  wait_check_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(h->err, (uint64_t)limit_ns);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "wait check launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_vhs_num_variants(const dgfs_vhs* h, int* count) {
  clear_error();
  if (!h || !count) return set_error(DGFS_ERR_INVALID, "null argument");
  *count = (int)h->fam.size();
  return DGFS_OK;
}

extern "C" int dgfs_vhs_variant_kind(const dgfs_vhs* h, int idx, int* push) {
  clear_error();
  if (!h || !push) return set_error(DGFS_ERR_INVALID, "null argument");
  if (idx < 0 || idx >= (int)h->fam.size()) return set_error(DGFS_ERR_INVALID, "variant %d out of range", idx);
  *push = h->fam[idx]->push;
  return DGFS_OK;
}

extern "C" int dgfs_vhs_variant_info(const dgfs_vhs* h, int idx, int* cluster, int* double_buffered,
                                     int* min_ctas_per_sm, int* threads, int* smem_bytes) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  if (idx < 0 || idx >= (int)h->fam.size()) return set_error(DGFS_ERR_INVALID, "variant %d out of range", idx);
  const VhsVariant* v = h->fam[idx];
  if (cluster) *cluster = v->C;
  if (double_buffered) *double_buffered = v->db;
  if (min_ctas_per_sm) *min_ctas_per_sm = v->minb;
  if (threads) *threads = v->threads;
  if (smem_bytes) *smem_bytes = (int)v->smem;
  return DGFS_OK;
}

extern "C" int dgfs_vhs_select(dgfs_vhs* h, int idx) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  const int old = h->vidx;
  int rc = select_index(h, idx);
  if (rc) {
    const int keep = rc;
    std::string msg = dgfs_last_error();
    select_index(h, old);
    return set_error(keep, "%s", msg.c_str());
  }
  return DGFS_OK;
}

extern "C" int dgfs_vhs_info(const dgfs_vhs* h, int* cluster, int* threads, int* smem_bytes, int* max_clusters) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  if (cluster) *cluster = h->var->C;
  if (threads) *threads = h->var->threads;
  if (smem_bytes) *smem_bytes = (int)h->var->smem;
  if (max_clusters) *max_clusters = h->max_clusters;
  return DGFS_OK;
}

static int vhs_launch(dgfs_vhs* h, const void* f, void* Q, int nupts, int neles, long long ldim, int soasz,
                      int pt0, int npts, void* stream, const int* plist = nullptr, const int* pcount = nullptr) {
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  if (!f || !Q) return set_error(DGFS_ERR_INVALID, "null bank pointer");
  if (nupts < 1 || neles < 1 || soasz < 1)
    return set_error(DGFS_ERR_INVALID, "bad bank shape nupts=%d neles=%d soasz=%d", nupts, neles, soasz);
  const long long nblk = (neles + soasz - 1) / soasz;
  if (ldim < nblk * soasz * (long long)h->V)
    return set_error(DGFS_ERR_INVALID, "ldim=%lld smaller than one AoSoA row (%lld)", ldim,
                     nblk * soasz * (long long)h->V);
  if (!plist && (pt0 < 0 || npts < 0 || (long long)pt0 + npts > (long long)nupts * neles))
    return set_error(DGFS_ERR_INVALID, "point range [%d, %d) outside 0..%lld", pt0, pt0 + npts,
                     (long long)nupts * neles);
  if (plist && (npts < 0 || npts > nupts * neles))
    return set_error(DGFS_ERR_INVALID, "point list of %d entries for a bank of %d points", npts, nupts * neles);
  const size_t esz = h->prec == 64 ? 8 : 4;
  const char* fb = (const char*)f;
  const char* qb = (const char*)Q;
  const size_t bytes = (size_t)nupts * (size_t)ldim * esz;
  if (fb < qb + bytes && qb < fb + bytes) return set_error(DGFS_ERR_INVALID, "f and Q overlap");
  if (((uintptr_t)f % esz) || ((uintptr_t)Q % esz)) return set_error(DGFS_ERR_INVALID, "misaligned bank");
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != h->device)
    return set_error(DGFS_ERR_INVALID, "handle built on device %d used on device %d", h->device, dev);
  if (npts == 0) return DGFS_OK;

  // the single-CTA kernel may split a point over up to P CTAs
  const long long want = h->var->push == 2 ? (long long)npts * h->P : npts;
  const int ncl = want < h->max_clusters ? (int)want : h->max_clusters;
  cudaError_t e;
  if (h->prec == 64) {
    VhsArgs<double> a{};
    a.f = (const double*)f;
    a.Q = (double*)Q;
    a.ldim = ldim;
    a.nupts = nupts;
    a.neles = neles;
    a.soasz = soasz;
    a.pt0 = pt0;
    a.npts = npts;
    a.P = h->P;
    a.M = h->M;
    a.phase = (const double2*)h->phase;
    a.w1 = (const double*)h->w1;
    a.b2 = (const double*)h->b2;
    a.w1t = (const double*)h->w1t;
    a.b2t = (const double*)h->b2t;
    a.fc = (double2*)h->fc;
    a.err = h->err;
    a.plist = plist;
    a.pcount = pcount;
    a.prefac = h->prefac;
    a.project = h->project;
    a.ginv = h->ginv;
    a.cvec = h->cvec;
    e = h->var->launch64(a, ncl, (cudaStream_t)stream);
  } else {
    VhsArgs<float> a{};
    a.f = (const float*)f;
    a.Q = (float*)Q;
    a.ldim = ldim;
    a.nupts = nupts;
    a.neles = neles;
    a.soasz = soasz;
    a.pt0 = pt0;
    a.npts = npts;
    a.P = h->P;
    a.M = h->M;
    a.phase = (const float2*)h->phase;
    a.w1 = (const float*)h->w1;
    a.b2 = (const float*)h->b2;
    a.w1t = (const float*)h->w1t;
    a.b2t = (const float*)h->b2t;
    a.fc = (float2*)h->fc;
    if (h->var->push == 2) {
      a.fcp = (float2*)h->fcp;
      a.pdone = h->pdone;
    }
    a.err = h->err;
    a.plist = plist;
    a.pcount = pcount;
    a.prefac = (float)h->prefac;
    a.project = h->project;
    a.ginv = h->ginv;
    a.cvec = h->cvec;
    e = h->var->launch32(a, ncl, (cudaStream_t)stream);
  }
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "VHS launch failed: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_vhs_apply(dgfs_vhs* h, const void* f, void* Q, int nupts, int neles, long long ldim, int soasz,
                              int elem, int upt, void* stream) {
  clear_error();
  if (elem >= 0) {
    if (elem >= neles || upt < 0 || upt >= nupts)
      return set_error(DGFS_ERR_INVALID, "point (elem=%d, upt=%d) outside bank (%d, %d)", elem, upt, neles, nupts);
    return vhs_launch(h, f, Q, nupts, neles, ldim, soasz, upt * neles + elem, 1, stream);
  }
  return vhs_launch(h, f, Q, nupts, neles, ldim, soasz, 0, nupts * neles, stream);
}

extern "C" int dgfs_vhs_apply_range(dgfs_vhs* h, const void* f, void* Q, int nupts, int neles, long long ldim,
                                    int soasz, int pt0, int npts, void* stream) {
  clear_error();
  return vhs_launch(h, f, Q, nupts, neles, ldim, soasz, pt0, npts, stream);
}

extern "C" int dgfs_vhs_apply_list(dgfs_vhs* h, const void* f, void* Q, int nupts, int neles, long long ldim,
                                   int soasz, const int* pts, const int* count, int max_points, void* stream) {
  clear_error();
  if (!pts) return set_error(DGFS_ERR_INVALID, "null point list");
  return vhs_launch(h, f, Q, nupts, neles, ldim, soasz, 0, max_points, stream, pts, count);
}

// ---------------------------------------------------------------------------
// Collision frequency nu(c) = prefac Re IFFT(b2 FFT(f) / V)(c), the loss rate
// of Q = prefac (gain - f Re IFFT(b2 F)) (vhs-gll.mako:209-220, 246-266).
// One CTA per point; FP32 arithmetic whatever the bank precision (the
// surrogate needs nu to ~1e-6 relative).  f is real, so the transform along
// the last axis keeps the N/2+1 non-negative frequencies; b2 is even on the
// index grid (its Nyquist index maps onto itself), so b2 F stays Hermitian
// and the complex-to-real inverse along that axis returns the real part the
// reference takes.  Shared memory: N^2 (N/2+1) complex floats.
// ---------------------------------------------------------------------------
namespace {

template <typename TB, int N>
__global__ void __launch_bounds__(256) loss_rate_kernel(const TB* __restrict__ f, TB* __restrict__ nu, int64_t ldim,
                                                        int nupts, int neles, int soasz, const TB* __restrict__ b2,
                                                        float prefac, const int* __restrict__ gate) {
  using C = cx<float>;
  constexpr int H = N / 2 + 1, V = N * N * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);  // [N][N][H]
  const int pt = blockIdx.x;
  if (gate && !gate[pt]) return;  // uniform over the CTA
  const int upt = pt / neles, elem = pt % neles;
  const int tid = threadIdx.x, NT = blockDim.x;

  // forward along k (real to half spectrum)
  for (int line = tid; line < N * N; line += NT) {
    C x[N];
#pragma unroll
    for (int k = 0; k < N; ++k)
      x[k] = mk<C>((float)f[soa_ix(upt, ldim, elem, (int64_t)line * N + k, V, soasz)], 0.f);
    fft<float, N, -1>(x);
#pragma unroll
    for (int k = 0; k < H; ++k) s[line * H + k] = x[k];
  }
  __syncthreads();
  // forward along j, then along i
  for (int line = tid; line < N * H; line += NT) {
    const int i = line / H, k = line % H;
    C x[N];
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = s[(i * N + j) * H + k];
    fft<float, N, -1>(x);
#pragma unroll
    for (int j = 0; j < N; ++j) s[(i * N + j) * H + k] = x[j];
  }
  __syncthreads();
  for (int line = tid; line < N * H; line += NT) {
    const int j = line / H, k = line % H;
    C x[N];
#pragma unroll
    for (int i = 0; i < N; ++i) x[i] = s[(i * N + j) * H + k];
    fft<float, N, -1>(x);
    // b2 / V, then the inverse along i
#pragma unroll
    for (int i = 0; i < N; ++i) x[i] = cscale(x[i], (float)b2[(i * N + j) * N + k] * (1.f / V));
    fft<float, N, +1>(x);
#pragma unroll
    for (int i = 0; i < N; ++i) s[(i * N + j) * H + k] = x[i];
  }
  __syncthreads();
  for (int line = tid; line < N * H; line += NT) {
    const int i = line / H, k = line % H;
    C x[N];
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = s[(i * N + j) * H + k];
    fft<float, N, +1>(x);
#pragma unroll
    for (int j = 0; j < N; ++j) s[(i * N + j) * H + k] = x[j];
  }
  __syncthreads();
  // complex-to-real inverse along k
  for (int line = tid; line < N * N; line += NT) {
    C x[N];
#pragma unroll
    for (int k = 0; k < H; ++k) x[k] = s[line * H + k];
#pragma unroll
    for (int k = H; k < N; ++k) {
      const C c = s[line * H + (N - k)];
      x[k] = mk<C>(c.x, -c.y);
    }
    fft<float, N, +1>(x);
#pragma unroll
    for (int k = 0; k < N; ++k) nu[soa_ix(upt, ldim, elem, (int64_t)line * N + k, V, soasz)] = (TB)(prefac * x[k].x);
  }
}

template <typename TB, int N>
cudaError_t launch_loss_rate(const dgfs_vhs* h, const void* f, void* nu, long long ldim, int nupts, int neles,
                             int soasz, const int* gate, cudaStream_t st) {
  const size_t smem = (size_t)N * N * (N / 2 + 1) * sizeof(cx<float>);
  static bool attr[64];
  const auto fn = loss_rate_kernel<TB, N>;
  if (h->device >= 0 && h->device < 64 && !attr[h->device]) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr[h->device] = true;
  }
  fn<<<(unsigned)(nupts * neles), 256, smem, st>>>((const TB*)f, (TB*)nu, ldim, nupts, neles, soasz,
                                                  (const TB*)h->b2, (float)h->prefac, gate);
  return cudaGetLastError();
}

}  // namespace

extern "C" int dgfs_vhs_loss_rate(dgfs_vhs* h, const void* f, void* nu, int nupts, int neles, long long ldim,
                                  int soasz, const int* gate, void* stream) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  if (!f || !nu) return set_error(DGFS_ERR_INVALID, "null bank pointer");
  if (nupts < 1 || neles < 1 || soasz < 1) return set_error(DGFS_ERR_INVALID, "bad bank shape");
  const long long nblk = (neles + soasz - 1) / soasz;
  if (ldim < nblk * soasz * (long long)h->V) return set_error(DGFS_ERR_INVALID, "ldim too small");
  if ((long long)nupts * neles > 0x7fffffffLL) return set_error(DGFS_ERR_UNSUPPORTED, "too many points");
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != h->device)
    return set_error(DGFS_ERR_INVALID, "handle built on device %d used on device %d", h->device, dev);
  const size_t esz = h->prec == 64 ? 8 : 4;
  const char* fb = (const char*)f;
  const char* nb = (const char*)nu;
  const size_t bytes = (size_t)nupts * (size_t)ldim * esz;
  if (fb < nb + bytes && nb < fb + bytes) return set_error(DGFS_ERR_INVALID, "f and nu overlap");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaErrorInvalidValue;
#define LR(TB, NN) e = launch_loss_rate<TB, NN>(h, f, nu, ldim, nupts, neles, soasz, gate, st)
  if (h->prec == 64) {
    switch (h->N) {
      case 8: LR(double, 8); break;
      case 16: LR(double, 16); break;
      case 24: LR(double, 24); break;
      case 32: LR(double, 32); break;
      default: return set_error(DGFS_ERR_UNSUPPORTED, "Nv=%d", h->N);
    }
  } else {
    switch (h->N) {
      case 8: LR(float, 8); break;
      case 16: LR(float, 16); break;
      case 24: LR(float, 24); break;
      case 32: LR(float, 32); break;
      default: return set_error(DGFS_ERR_UNSUPPORTED, "Nv=%d", h->N);
    }
  }
#undef LR
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "loss-rate launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}
