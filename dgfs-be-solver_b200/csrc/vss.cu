// Host side of the binary-mixture VSS collision operator: the per-pair
// precomputation of frfs's DGFSBiVSSGLLScatteringModel
// (frfs/solvers/dgfsbi/scattering.py:44-224, vss-gll.mako:31-93) and the
// launches of the fused kernel (vss_push.cuh) behind the C ABI.
#include <cmath>
#include <complex>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"
#include "vss_push.cuh"
#include "vss_pair.cuh"

using namespace dgfs;

namespace {

// This translation unit's copy of the FFT twiddle table (fft_reg.cuh keeps
// it in file-scope constant memory), exp(2 pi i m / 96) in long double,
// uploaded once per device.
std::mutex g_tw_mutex;
bool g_tw_ready[64];

int init_twiddles_current() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return set_error(DGFS_ERR_CUDA, "no CUDA device");
  std::lock_guard<std::mutex> lk(g_tw_mutex);
  if (g_tw_ready[dev]) return DGFS_OK;
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
  g_tw_ready[dev] = true;
  return DGFS_OK;
}

struct VssShape {
  int prec, N, C, threads;
  int pair;           // 1: the two-CTA kernel (vss_pair.cuh)
  size_t smem;
  size_t scratch_cx;  // complex scratch per cluster
  const void* fn;
  cudaError_t (*launch32)(const VssArgs<float>&, int, cudaStream_t);
  cudaError_t (*launch64)(const VssArgs<double>&, int, cudaStream_t);
};

template <typename T, int N, int C, int MINB>
cudaError_t launch_vss(const VssArgs<T>& a, int nclusters, cudaStream_t s) {
  using P = PushGeom<N, C>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nclusters * C, 1, 1);
  cfg.blockDim = dim3(P::NT, 1, 1);
  cfg.dynamicSmemBytes = VssGeom<N, C>::SMEM_CX * sizeof(cx<T>);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, vss_push_kernel<T, N, C, MINB>, a);
}

template <typename T, int N, int C, int MINB> VssShape make_vss() {
  VssShape v{};
  v.prec = sizeof(T) == 8 ? 64 : 32;
  v.N = N;
  v.C = C;
  v.threads = PushGeom<N, C>::NT;
  v.smem = VssGeom<N, C>::SMEM_CX * sizeof(cx<T>);
  v.scratch_cx = (size_t)N * N * N;
  v.fn = (const void*)vss_push_kernel<T, N, C, MINB>;
  if constexpr (sizeof(T) == 8) v.launch64 = launch_vss<double, N, C, MINB>;
  else v.launch32 = launch_vss<float, N, C, MINB>;
  return v;
}

template <int N> cudaError_t launch_vss_pair(const VssArgs<float>& a, int nclusters, cudaStream_t s) {
  using P = VssPairGeom<N>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nclusters * 2, 1, 1);
  cfg.blockDim = dim3(P::NT, 1, 1);
  cfg.dynamicSmemBytes = P::SMEM_CX * sizeof(cx<float>);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, vss_pair_kernel<N>, a);
}

template <int N> VssShape make_vss_pair() {
  using P = VssPairGeom<N>;
  VssShape v{};
  v.prec = 32;
  v.N = N;
  v.C = 2;
  v.pair = 1;
  v.threads = P::NT;
  v.smem = P::SMEM_CX * sizeof(cx<float>);
  v.scratch_cx = P::SCRATCH;
  v.fn = (const void*)vss_pair_kernel<N>;
  v.launch32 = launch_vss_pair<N>;
  return v;
}

// Launch shapes per (precision, N): the cluster push kernel everywhere
// (FP64 N = 32 does not fit the shared memory of a 16-CTA cluster's CTA),
// and at FP32 N = 24 the two-CTA kernel, which is the default there.
// pair < 0: the default shape; 0 / 1: the push / two-CTA kernel.
const VssShape* vss_shape(int prec, int N, int pair = -1) {
  static const VssShape s[] = {
      make_vss_pair<24>(),          make_vss<float, 8, 1, 2>(),   make_vss<float, 16, 4, 2>(),
      make_vss<float, 24, 8, 2>(),  make_vss<float, 32, 16, 1>(), make_vss<double, 8, 1, 2>(),
      make_vss<double, 16, 4, 1>(), make_vss<double, 24, 8, 1>()};
  for (const auto& v : s)
    if (v.prec == prec && v.N == N && (pair < 0 || v.pair == pair)) return &v;
  return nullptr;
}

}  // namespace

struct dgfs_vss {
  int N, P, M, prec, V, device;
  int Mh;  // like pair on an antipodally symmetric design: M / 2 (one
           // direction of each antipodal pair, tables phase_h and b_h), else 0
  double prefac;
  const VssShape* shape;
  int max_clusters;
  void* phase;  // cx<T> [P][M][2][3][N]
  void* b;      // cx<T> [P][M][V], weight w_x folded in
  void* phase_h;  // cx<T> [P][Mh][2][3][N] (Mh > 0)
  void* b_h;      // cx<T> [P][Mh][V]: b(y) + b(-y)
  void* c;      // cx<T> [V]
  void* fc;     // scratch: [clusters * C][V / C] cx<T> (push), per pair (two-CTA)
  size_t fc_bytes;
  int* err;
};

namespace {

template <typename T> int upload_cx(void** dst, const std::vector<std::complex<double>>& src) {
  std::vector<cx<T>> h(src.size());
  for (size_t i = 0; i < src.size(); ++i) {
    h[i].x = (T)src[i].real();
    h[i].y = (T)src[i].imag();
  }
  if (cudaMalloc(dst, h.size() * sizeof(cx<T>)) != cudaSuccess) {
    *dst = nullptr;
    return set_error(DGFS_ERR_NOMEM, "cudaMalloc(%zu) failed", h.size() * sizeof(cx<T>));
  }
  if (cudaMemcpy(*dst, h.data(), h.size() * sizeof(cx<T>), cudaMemcpyHostToDevice) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(cudaGetLastError()));
  return DGFS_OK;
}

// The reference's precomputation for one ordered pair (vss-gll.mako:31-93,
// scattering.py:172-198): with l the index grid (0..N/2-1, -N/2..-1 per
// axis, I slowest), fac_x = pi / L qz_x and the full-sphere designs sz (M
// directions, sw = 4 pi / M) and szpre (Mpre, swpre = 4 pi / Mpre):
//   B[y][y'] = (1 + sz_y . szpre_y')^eta           (1 + cos below 1e-12 in
//              magnitude is the exact 0 of an antipodal pair of the
//              symmetric designs: rounding leaves +-1e-16 there, where pow
//              would give NaN or up to (1e-16)^eta)
//   b_xy(l)  = swpre qz_x^(gamma+2) sum_y' B[y][y'] e^{-i mq/(mp+mq) fac_x szpre_y'.l}
//   c(l)     = sum_x qw_x sw swpre qz_x^(gamma+2) sum_y sum_y' B[y][y'] e^{-i fac_x szpre_y'.l}
// and the weight of computeQG, w_x = qw_x sw / V, folded into b_xy.
template <typename T> int build(dgfs_vss* h, const dgfs_vss_params* p) {
  const int N = h->N, P = h->P, M = h->M, V = h->V, Mp = p->Mpre;
  const double pi = 3.14159265358979323846, L = p->L;
  const double sw = 4 * pi / M, swpre = 4 * pi / Mp;
  const double eta = p->alpha - 1.0, gam = 2.0 * (1.0 - p->omega);
  const double kp = p->mp / (p->mp + p->mq), kq = p->mq / (p->mp + p->mq);
  std::vector<double> l0(N);
  for (int k = 0; k < N; ++k) l0[k] = k < N / 2 ? k : k - N;
  std::vector<double> B((size_t)M * Mp);
  for (int y = 0; y < M; ++y)
    for (int y2 = 0; y2 < Mp; ++y2) {
      double d = 1.0;
      for (int ax = 0; ax < 3; ++ax) d += p->sz[y * 3 + ax] * p->szpre[y2 * 3 + ax];
      if (std::fabs(d) < 1e-12) d = 0.0;
      B[(size_t)y * Mp + y2] = std::pow(d > 0.0 ? d : 0.0, eta);
    }
  // szpre_y' . l for every grid point
  std::vector<double> lpre((size_t)Mp * V);
  for (int y2 = 0; y2 < Mp; ++y2)
    for (int v = 0; v < V; ++v)
      lpre[(size_t)y2 * V + v] = p->szpre[y2 * 3] * l0[v / (N * N)] + p->szpre[y2 * 3 + 1] * l0[(v / N) % N] +
                                 p->szpre[y2 * 3 + 2] * l0[v % N];

  // A like pair (equal masses, so kp = kq = 1/2) applied to one
  // distribution twice, on a design that holds every direction's antipode:
  // the antipode turns e^{+i a/2} F into e^{-i a/2} F and back, so its
  // product g h and FFT(g h) are the direction's own.  A second set of
  // tables loops over one direction of each antipodal pair with the gain
  // kernel b(y) + b(-y): exact, with half the transforms and half the table
  // reads; dgfs_vss_apply uses it when fp == fq.
  std::vector<int> rep, anti(M, -1);
  if (p->mp == p->mq) {
    for (int y = 0; y < M; ++y) {
      if (anti[y] >= 0) continue;
      for (int z = y + 1; z < M; ++z) {
        if (anti[z] >= 0) continue;
        double d = 0.0;
        for (int ax = 0; ax < 3; ++ax) d = std::fmax(d, std::fabs(p->sz[y * 3 + ax] + p->sz[z * 3 + ax]));
        if (d < 1e-9) {
          anti[y] = z;
          anti[z] = y;
          rep.push_back(y);
          break;
        }
      }
      if (anti[y] < 0) break;
    }
  }
  const bool halve = p->mp == p->mq && 2 * (int)rep.size() == M;
  std::vector<int> all(M);
  for (int y = 0; y < M; ++y) all[y] = y;

  // axis phases [P][K][2][3][N] and weighted gain kernels [P][K][V] of the
  // directions `dirs` (each with its antipode's b added when `pairs`)
  std::vector<std::complex<double>> eb((size_t)Mp * V), row(V);
  auto tables = [&](const std::vector<int>& dirs, bool pairs, std::vector<std::complex<double>>& phase,
                    std::vector<std::complex<double>>& b) {
    const int K = (int)dirs.size();
    phase.assign((size_t)P * K * 6 * N, 0.0);
    b.assign((size_t)P * K * V, 0.0);
    for (int x = 0; x < P; ++x) {
      const double fac = pi / L * p->qz[x];
      const double fac_b = swpre * std::pow(p->qz[x], gam + 2.0);
      const double w = p->qw[x] * sw / V;
      for (int j = 0; j < K; ++j)
        for (int f = 0; f < 2; ++f)
          for (int ax = 0; ax < 3; ++ax)
            for (int k = 0; k < N; ++k) {
              const double ang = (f == 0 ? kq : -kp) * fac * p->sz[dirs[j] * 3 + ax] * l0[k];
              phase[((((size_t)x * K + j) * 2 + f) * 3 + ax) * N + k] = std::polar(1.0, ang);
            }
      for (size_t i = 0; i < eb.size(); ++i) eb[i] = std::polar(1.0, -kq * fac * lpre[i]);
      for (int j = 0; j < K; ++j) {
        std::complex<double>* dst = b.data() + ((size_t)x * K + j) * V;
        for (int t = 0; t < (pairs ? 2 : 1); ++t) {
          const int y = t == 0 ? dirs[j] : anti[dirs[j]];
          for (int v = 0; v < V; ++v) row[v] = 0.0;
          for (int y2 = 0; y2 < Mp; ++y2) {
            const double bb = B[(size_t)y * Mp + y2];
            const std::complex<double>* e = eb.data() + (size_t)y2 * V;
            for (int v = 0; v < V; ++v) row[v] += bb * e[v];
          }
          for (int v = 0; v < V; ++v) dst[v] += row[v] * (w * fac_b);
        }
      }
    }
  };

  // the loss kernel c (every direction of the design)
  std::vector<std::complex<double>> c(V, 0.0), ec((size_t)Mp * V);
  std::vector<double> Bsum(Mp, 0.0);
  for (int y2 = 0; y2 < Mp; ++y2)
    for (int y = 0; y < M; ++y) Bsum[y2] += B[(size_t)y * Mp + y2];
  for (int x = 0; x < P; ++x) {
    const double fac = pi / L * p->qz[x];
    const double fac_b = swpre * std::pow(p->qz[x], gam + 2.0);
    const double fac_c = p->qw[x] * sw * fac_b;
    for (size_t i = 0; i < ec.size(); ++i) ec[i] = std::polar(1.0, -fac * lpre[i]);
    for (int y2 = 0; y2 < Mp; ++y2) {
      const std::complex<double>* e = ec.data() + (size_t)y2 * V;
      const double s = fac_c * Bsum[y2];
      for (int v = 0; v < V; ++v) c[v] += s * e[v];
    }
  }
  std::vector<std::complex<double>> phase, b;
  tables(all, false, phase, b);
  int rc;
  if ((rc = upload_cx<T>(&h->phase, phase)) || (rc = upload_cx<T>(&h->b, b)) || (rc = upload_cx<T>(&h->c, c)))
    return rc;
  h->Mh = 0;
  if (halve) {
    tables(rep, true, phase, b);
    if ((rc = upload_cx<T>(&h->phase_h, phase)) || (rc = upload_cx<T>(&h->b_h, b))) return rc;
    h->Mh = (int)rep.size();
  }
  return DGFS_OK;
}

void free_vss(dgfs_vss* h) {
  if (!h) return;
  cudaFree(h->phase);
  cudaFree(h->b);
  cudaFree(h->phase_h);
  cudaFree(h->b_h);
  cudaFree(h->c);
  cudaFree(h->fc);
  cudaFree(h->err);
  delete h;
}

}  // namespace

namespace {

// Kernel attributes, the clusters that fit the device and the scratch of a
// launch shape (the scratch grows, never shrinks).
int set_shape(dgfs_vss* h, const VssShape* shape) {
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  if ((int)shape->smem > maxsm)
    return set_error(DGFS_ERR_UNSUPPORTED, "VSS kernel Nv=%d needs %zu B shared memory", h->N, shape->smem);
  if (cudaFuncSetAttribute(shape->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shape->smem) !=
          cudaSuccess ||
      (shape->C > 8 &&
       cudaFuncSetAttribute(shape->fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess))
    return set_error(DGFS_ERR_CUDA, "VSS kernel attributes: %s", cudaGetErrorString(cudaGetLastError()));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(shape->C, 1, 1);
  cfg.blockDim = dim3(shape->threads, 1, 1);
  cfg.dynamicSmemBytes = shape->smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = shape->C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int ncl = 0;
  const cudaError_t oe = cudaOccupancyMaxActiveClusters(&ncl, shape->fn, &cfg);
  if (oe != cudaSuccess || ncl < 1) {
    cudaGetLastError();
    return set_error(DGFS_ERR_UNSUPPORTED, "VSS cluster of %d CTAs x %d threads, %zu B shared memory cannot be "
                     "scheduled (%s, %d clusters)", shape->C, shape->threads, shape->smem, cudaGetErrorString(oe), ncl);
  }
  const size_t esz = h->prec == 64 ? 16 : 8;
  const size_t need = (size_t)ncl * shape->scratch_cx * esz;
  if (need > h->fc_bytes) {
    cudaFree(h->fc);
    h->fc = nullptr;
    h->fc_bytes = 0;
    if (cudaMalloc(&h->fc, need) != cudaSuccess)
      return set_error(DGFS_ERR_NOMEM, "VSS scratch allocation of %zu B failed", need);
    h->fc_bytes = need;
  }
  h->shape = shape;
  h->max_clusters = ncl;
  return DGFS_OK;
}

}  // namespace

extern "C" int dgfs_vss_create(const dgfs_vss_params* p, dgfs_vss** out) {
  clear_error();
  if (!p || !out) return set_error(DGFS_ERR_INVALID, "null argument");
  *out = nullptr;
  if (p->precision != 32 && p->precision != 64)
    return set_error(DGFS_ERR_INVALID, "precision must be 32 or 64, got %d", p->precision);
  const VssShape* shape = vss_shape(p->precision, p->Nv);
  if (!shape) return set_error(DGFS_ERR_UNSUPPORTED, "no VSS kernel for Nv=%d precision=%d", p->Nv, p->precision);
  if (p->Nrho < 1 || p->M < 1 || p->Mpre < 1 || p->Nrho > 4096 || p->M > 4096 || p->Mpre > 4096)
    return set_error(DGFS_ERR_INVALID, "bad quadrature sizes Nrho=%d M=%d Mpre=%d", p->Nrho, p->M, p->Mpre);
  if (!p->qz || !p->qw || !p->sz || !p->szpre) return set_error(DGFS_ERR_INVALID, "null quadrature array");
  if (!(p->L > 0) || !std::isfinite(p->L) || !(p->mp > 0) || !(p->mq > 0) || !std::isfinite(p->alpha) ||
      !std::isfinite(p->omega) || !std::isfinite(p->prefactor))
    return set_error(DGFS_ERR_INVALID, "bad scalar parameter");
  dgfs_vss* h = new dgfs_vss();
  h->N = p->Nv;
  h->P = p->Nrho;
  h->M = p->M;
  h->prec = p->precision;
  h->V = p->Nv * p->Nv * p->Nv;
  h->prefac = p->prefactor;
  int rc = DGFS_OK;
  if (cudaGetDevice(&h->device) != cudaSuccess) rc = set_error(DGFS_ERR_CUDA, "no CUDA device");
  if (!rc) rc = init_twiddles_current();
  if (!rc) rc = set_shape(h, shape);
  if (!rc && (cudaMalloc((void**)&h->err, sizeof(int)) != cudaSuccess ||
              cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess))
    rc = set_error(DGFS_ERR_NOMEM, "error flag allocation failed");
  if (!rc) rc = h->prec == 64 ? build<double>(h, p) : build<float>(h, p);
  if (rc) {
    free_vss(h);
    return rc;
  }
  *out = h;
  return DGFS_OK;
}

extern "C" int dgfs_vss_destroy(dgfs_vss* h) {
  clear_error();
  free_vss(h);
  return DGFS_OK;
}

extern "C" int dgfs_vss_apply(dgfs_vss* h, const void* fp, const void* fq, void* Q, int nupts, int neles,
                              long long ldim, int soasz, int elem, int upt, int accumulate, void* stream) {
  clear_error();
  if (!h || !fp || !fq || !Q) return set_error(DGFS_ERR_INVALID, "null argument");
  if (nupts < 1 || neles < 1 || soasz < 1)
    return set_error(DGFS_ERR_INVALID, "bad bank shape nupts=%d neles=%d soasz=%d", nupts, neles, soasz);
  const long long nblk = (neles + soasz - 1) / soasz;
  if (ldim < nblk * soasz * (long long)h->V) return set_error(DGFS_ERR_INVALID, "ldim=%lld smaller than one row", ldim);
  const size_t esz = h->prec == 64 ? 8 : 4;
  const size_t bytes = (size_t)nupts * (size_t)ldim * esz;
  const char *qb = (const char*)Q, *pb = (const char*)fp, *fb = (const char*)fq;
  if ((pb < qb + bytes && qb < pb + bytes) || (fb < qb + bytes && qb < fb + bytes))
    return set_error(DGFS_ERR_INVALID, "the output bank overlaps an input bank");
  int pt0, npts;
  if (elem >= 0) {
    if (elem >= neles || upt < 0 || upt >= nupts)
      return set_error(DGFS_ERR_INVALID, "point (elem=%d, upt=%d) outside bank (%d, %d)", elem, upt, neles, nupts);
    pt0 = upt * neles + elem;
    npts = 1;
  } else {
    pt0 = 0;
    npts = nupts * neles;
  }
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != h->device) return set_error(DGFS_ERR_INVALID, "handle built on device %d used on device %d", h->device, dev);
  const int ncl = npts < h->max_clusters ? npts : h->max_clusters;
  // the halved tables need the same distribution on both sides
  const bool half = h->Mh > 0 && fp == fq;
  cudaError_t e;
  if (h->prec == 64) {
    VssArgs<double> a{};
    a.fp = (const double*)fp;
    a.fq = (const double*)fq;
    a.Q = (double*)Q;
    a.ldim = ldim;
    a.nupts = nupts;
    a.neles = neles;
    a.soasz = soasz;
    a.pt0 = pt0;
    a.npts = npts;
    a.P = h->P;
    a.M = half ? h->Mh : h->M;
    a.phase = (const double2*)(half ? h->phase_h : h->phase);
    a.b = (const double2*)(half ? h->b_h : h->b);
    a.c = (const double2*)h->c;
    a.fc = (double2*)h->fc;
    a.err = h->err;
    a.prefac = h->prefac;
    a.accumulate = accumulate ? 1 : 0;
    e = h->shape->launch64(a, ncl, (cudaStream_t)stream);
  } else {
    VssArgs<float> a{};
    a.fp = (const float*)fp;
    a.fq = (const float*)fq;
    a.Q = (float*)Q;
    a.ldim = ldim;
    a.nupts = nupts;
    a.neles = neles;
    a.soasz = soasz;
    a.pt0 = pt0;
    a.npts = npts;
    a.P = h->P;
    a.M = half ? h->Mh : h->M;
    a.phase = (const float2*)(half ? h->phase_h : h->phase);
    a.b = (const float2*)(half ? h->b_h : h->b);
    a.c = (const float2*)h->c;
    a.fc = (float2*)h->fc;
    a.err = h->err;
    a.prefac = (float)h->prefac;
    a.accumulate = accumulate ? 1 : 0;
    e = h->shape->launch32(a, ncl, (cudaStream_t)stream);
  }
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "VSS launch failed: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_vss_select(dgfs_vss* h, int pair) {
  clear_error();
  if (!h) return set_error(DGFS_ERR_INVALID, "null handle");
  const VssShape* shape = vss_shape(h->prec, h->N, pair ? 1 : 0);
  if (!shape)
    return set_error(DGFS_ERR_UNSUPPORTED, "no %s VSS kernel for Nv=%d precision=%d", pair ? "two-CTA" : "cluster",
                     h->N, h->prec);
  return set_shape(h, shape);
}

extern "C" int dgfs_vss_status(dgfs_vss* h, void* stream, int* flag) {
  clear_error();
  if (!h || !flag) return set_error(DGFS_ERR_INVALID, "null argument");
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
  int v = 0;
  if (cudaMemcpy(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "error flag: %s", cudaGetErrorString(cudaGetLastError()));
  *flag = v;
  if (v) return set_error(DGFS_ERR_CUDA, "a VSS launch gave up waiting for cluster data (flag %d)", v);
  return DGFS_OK;
}
