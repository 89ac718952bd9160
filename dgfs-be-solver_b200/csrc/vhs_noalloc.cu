// Allocation-free entry point for the VHS collision operator.
//
// Who needs it: callers that must not allocate device memory while they
// run -- host applications whose memory manager owns the whole device heap,
// plugins that may only touch the buffers they are handed, or code that runs
// between steady-state iterations where a cudaMalloc (which synchronises the
// device) is not acceptable.  dgfs_vhs_create allocates its tables and the
// gain-spectrum scratch with cudaMalloc; this path keeps all of that in one
// file-scope __device__ array of fixed size instead and never calls an
// allocator.
//
// The array (kScratchBytes = 24 MiB) lives in this translation unit's own
// module, so with the CUDA runtime's lazy module loading only processes that
// call this entry point hold it, on every GPU they call it on, until exit.
// Host code cannot use the array's name as a device address: on each device
// the first call looks its address up with cudaGetSymbolAddress, uploads the
// FFT twiddles and clears the error flag, and the first call for each
// (precision, Nv) sets that kernel's attributes; those first calls should
// come before any stream capture.  The addresses are kept for the life of
// the process: a cudaDeviceReset invalidates them and is not supported.
// Every call rebuilds the tables it needs and zeroes the accumulators that
// must start at zero, but all calls share the array: calls whose launches
// can overlap on the GPU (different streams without ordering) race on it.
// The kernel's bounded-wait flag also lives in the array; it is sticky until
// dgfs_vhs_noalloc_status reads and clears it.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"

// Private copy of the kernels (internal linkage: this module's constants and
// launch registrations never mix with the ones of the allocating path).
namespace {
#include "vhs_push.cuh"
}  // namespace

namespace {

using dgfs::cx;
using dgfs::PushGeom;
using dgfs::VhsArgs;

constexpr size_t kScratchBytes = 24ull << 20;
constexpr int kMaxNrho = 32;
constexpr int kMaxM = 128;

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct TableArgs {
  int N, P, M, project;
  double L, sw, gamma;
  double qz[kMaxNrho], qw[kMaxNrho], sz[3 * kMaxM], ginv[25];
  void* phase;   // cx<T> [P][M][3][N]
  void* w1;      // T [P][V]
  void* b2;      // T [V]
  double* cvec;  // [3][V]
  double* ginv_out;
};

__device__ __forceinline__ double ref_sinc(double s) { return sin(s + 1e-15) / (s + 1e-15); }

// The tables of dgfs_vhs_create (scattering.py:67-126, vhs-gll.mako:45-101),
// computed on the device into the static array.
template <typename T> __global__ void noalloc_tables_kernel(const TableArgs a) {
  const double pi = 3.14159265358979323846;
  const int N = a.N, V = N * N * N;
  const int nph = a.P * a.M * 3 * N;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = tid; i < nph; i += stride) {
    const int k = (int)(i % N), ax = (int)((i / N) % 3), q = (int)((i / (3 * N)) % a.M), p = (int)(i / (3 * N * a.M));
    const double l0 = k < N / 2 ? k : k - N;
    const double ang = pi / a.L * a.qz[p] / 2. * (a.sz[q * 3 + ax] * l0);
    double s, c;
    sincos(ang, &s, &c);
    cx<T> e;
    e.x = (T)c;
    e.y = (T)s;
    ((cx<T>*)a.phase)[i] = e;
  }
  for (int64_t v = tid; v < V; v += stride) {
    const int i1 = (int)(v / (N * N)), i2 = (int)((v % (N * N)) / N), i3 = (int)(v % N);
    const double lx = i1 < N / 2 ? i1 : i1 - N, ly = i2 < N / 2 ? i2 : i2 - N, lz = i3 < N / 2 ? i3 : i3 - N;
    const double cSqr = sqrt(lx * lx + ly * ly + lz * lz);
    double bsum = 0.;
    for (int p = 0; p < a.P; ++p) {
      const double qz = a.qz[p], qw = a.qw[p];
      const double b1 = pow(qz, a.gamma + 2.) * 4 * pi * ref_sinc(pi / a.L * qz / 2. * cSqr);
      bsum += qw * pow(qz, a.gamma + 2.) * 16 * pi * pi * ref_sinc(pi / a.L * qz * cSqr);
      ((T*)a.w1)[(int64_t)p * V + v] = (T)(2. * qw * a.sw / V * b1);
    }
    ((T*)a.b2)[v] = (T)bsum;
    if (a.project) {
      const double L = a.L;
      a.cvec[v] = -L + L / N + i1 * (2.0 * L / N);
      a.cvec[V + v] = -L + L / N + i2 * (2.0 * L / N);
      a.cvec[2 * V + v] = -L + L / N + i3 * (2.0 * L / N);
    }
  }
  if (tid < 25) a.ginv_out[tid] = a.ginv[tid];
}

struct Shape {
  const void* fn;
  int C, threads;
  size_t smem;
  cudaError_t (*launch32)(const VhsArgs<float>&, int, cudaStream_t);
  cudaError_t (*launch64)(const VhsArgs<double>&, int, cudaStream_t);
};

template <typename T, int N, int C, int MINB>
cudaError_t launch_shape(const VhsArgs<T>& a, int nclusters, cudaStream_t s) {
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
  return cudaLaunchKernelEx(&cfg, dgfs::vhs_push_kernel<T, N, C, MINB>, a);
}

template <typename T, int N, int C, int MINB> Shape make_shape() {
  using P = PushGeom<N, C>;
  Shape s{};
  s.fn = (const void*)dgfs::vhs_push_kernel<T, N, C, MINB>;
  s.C = C;
  s.threads = P::NT;
  s.smem = P::SMEM_CX * sizeof(cx<T>);
  if constexpr (sizeof(T) == 8) s.launch64 = launch_shape<double, N, C, MINB>;
  else s.launch32 = launch_shape<float, N, C, MINB>;
  return s;
}

// One push-exchange launch shape per (precision, Nv): index [prec64][n]
const Shape& shape_for(int prec, int N) {
  static const Shape s[2][4] = {
      {make_shape<float, 8, 1, 4>(), make_shape<float, 16, 2, 2>(), make_shape<float, 24, 8, 2>(),
       make_shape<float, 32, 16, 2>()},
      {make_shape<double, 8, 1, 4>(), make_shape<double, 16, 4, 2>(), make_shape<double, 24, 8, 1>(),
       make_shape<double, 32, 16, 1>()}};
  return s[prec == 64 ? 1 : 0][N == 8 ? 0 : N == 16 ? 1 : N == 24 ? 2 : 3];
}

// Per-device set-up state: the array's device address, and per (precision,
// Nv) shape whether its attributes are set and its resident cluster count.
struct DeviceState {
  bool ready;
  unsigned char* base;
  bool shape_ready[2][4];
  int max_clusters[2][4];
};
std::mutex g_mutex;
DeviceState g_dev[64];

// The error flag sits at offset 0 of the array.
int* flag_ptr(DeviceState* st) { return (int*)st->base; }

int setup_device(int dev, DeviceState** out) {
  using ::dgfs::set_error;
  if (dev < 0 || dev >= 64) return set_error(DGFS_ERR_UNSUPPORTED, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_mutex);
  DeviceState& st = g_dev[dev];
  if (st.ready) {
    *out = &st;
    return DGFS_OK;
  }
  void* base = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&base, g_scratch);
  if (e != cudaSuccess || !base)
    return set_error(DGFS_ERR_CUDA, "cudaGetSymbolAddress(static scratch): %s", cudaGetErrorString(e));
  // FFT twiddles of this module, exp(2 pi i m / 96) in long double
  double t64[2 * dgfs::kTwBase];
  float t32[2 * dgfs::kTwBase];
  const long double twopi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < dgfs::kTwBase; ++m) {
    const long double ang = twopi * (long double)m / (long double)dgfs::kTwBase;
    t64[2 * m] = (double)cosl(ang);
    t64[2 * m + 1] = (double)sinl(ang);
    t32[2 * m] = (float)cosl(ang);
    t32[2 * m + 1] = (float)sinl(ang);
  }
  if ((e = cudaMemcpyToSymbol(dgfs::c_tw64, t64, sizeof(t64))) != cudaSuccess ||
      (e = cudaMemcpyToSymbol(dgfs::c_tw32, t32, sizeof(t32))) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "twiddle upload: %s", cudaGetErrorString(e));
  if ((e = cudaMemset(base, 0, sizeof(int))) != cudaSuccess)
    return set_error(DGFS_ERR_CUDA, "error flag reset: %s", cudaGetErrorString(e));
  st.base = (unsigned char*)base;
  st.ready = true;
  *out = &st;
  return DGFS_OK;
}

// Attributes and resident cluster count of one (precision, Nv) shape, set
// up on its first use only, so a shape that cannot run on this device fails
// the calls that need it and no others.
int setup_shape(DeviceState* st, int pi, int ni) {
  using ::dgfs::set_error;
  std::lock_guard<std::mutex> lk(g_mutex);
  if (st->shape_ready[pi][ni]) return DGFS_OK;
  const int N = ni == 0 ? 8 : ni == 1 ? 16 : ni == 2 ? 24 : 32;
  const Shape& s = shape_for(pi ? 64 : 32, N);
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(s.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem)) != cudaSuccess ||
      (s.C > 8 && (e = cudaFuncSetAttribute(s.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess))
    return set_error(DGFS_ERR_CUDA, "kernel attributes (Nv=%d, precision %d): %s", N, pi ? 64 : 32,
                     cudaGetErrorString(e));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(s.C, 1, 1);
  cfg.blockDim = dim3(s.threads, 1, 1);
  cfg.dynamicSmemBytes = s.smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = s.C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int ncl = 0;
  if ((e = cudaOccupancyMaxActiveClusters(&ncl, s.fn, &cfg)) != cudaSuccess || ncl < 1)
    return set_error(DGFS_ERR_UNSUPPORTED, "cluster of %d CTAs (Nv=%d, precision %d) cannot be scheduled: %s", s.C,
                     N, pi ? 64 : 32, cudaGetErrorString(e));
  st->max_clusters[pi][ni] = ncl;
  st->shape_ready[pi][ni] = true;
  return DGFS_OK;
}

cudaError_t launch_wait_check(int* flag, uint64_t limit_ns, cudaStream_t stream) {
  dgfs::wait_check_kernel<<<1, 32, 0, stream>>>(flag, limit_ns);
  return cudaGetLastError();
}

int current_state(DeviceState** st) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return ::dgfs::set_error(DGFS_ERR_CUDA, "no CUDA device");
  return setup_device(dev, st);
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

bool invert5(const double* A, double* X) {
  double a[5][10];
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 10; ++j) a[i][j] = j < 5 ? A[i * 5 + j] : (j - 5 == i ? 1.0 : 0.0);
  for (int c = 0; c < 5; ++c) {
    int piv = c;
    for (int r = c + 1; r < 5; ++r)
      if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
    if (std::fabs(a[piv][c]) < 1e-300) return false;
    if (piv != c)
      for (int j = 0; j < 10; ++j) {
        const double t = a[c][j];
        a[c][j] = a[piv][j];
        a[piv][j] = t;
      }
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

template <typename T>
int run(const dgfs_vhs_params* p, DeviceState* st, const void* f, void* Q, int nupts, int neles, long long ldim,
        int soasz, int pt0, int npts, cudaStream_t stream) {
  using ::dgfs::set_error;
  const int N = p->Nv, P = p->Nrho, M = p->M, V = N * N * N;
  // layout of the static array
  size_t off = 0;
  int* err = (int*)(st->base + off);
  off = align256(off + sizeof(int));
  double* ginv = (double*)(st->base + off);
  off = align256(off + 25 * sizeof(double));
  void* phase = st->base + off;
  off = align256(off + (size_t)P * M * 3 * N * sizeof(cx<T>));
  void* w1 = st->base + off;
  off = align256(off + (size_t)P * V * sizeof(T));
  void* b2 = st->base + off;
  off = align256(off + (size_t)V * sizeof(T));
  double* cvec = (double*)(st->base + off);
  if (p->project) off = align256(off + (size_t)3 * V * sizeof(double));
  const size_t per_cluster = (size_t)V * sizeof(cx<T>);  // gain spectrum of C CTAs
  if (off + per_cluster > kScratchBytes)
    return set_error(DGFS_ERR_INVALID,
                     "Nv=%d Nrho=%d M=%d precision=%d needs %zu bytes of static scratch, more than the %zu "
                     "this allocation-free entry point holds",
                     N, P, M, p->precision, off + per_cluster, kScratchBytes);
  const int fit = (int)((kScratchBytes - off) / per_cluster);
  cx<T>* fc = (cx<T>*)(st->base + off);

  TableArgs ta{};
  ta.N = N;
  ta.P = P;
  ta.M = M;
  ta.project = p->project ? 1 : 0;
  ta.L = p->L;
  ta.sw = p->sw;
  ta.gamma = p->gamma;
  std::memcpy(ta.qz, p->qz, P * sizeof(double));
  std::memcpy(ta.qw, p->qw, P * sizeof(double));
  std::memcpy(ta.sz, p->sz, 3 * M * sizeof(double));
  if (ta.project) {
    // Gram matrix of phi = (1, cx, cy, cz, |c|^2) over the velocity grid
    double G[25] = {0};
    const double L = p->L;
    for (int v = 0; v < V; ++v) {
      const double c[3] = {-L + L / N + (v / (N * N)) * (2.0 * L / N), -L + L / N + ((v % (N * N)) / N) * (2.0 * L / N),
                           -L + L / N + (v % N) * (2.0 * L / N)};
      const double phi[5] = {1.0, c[0], c[1], c[2], c[0] * c[0] + c[1] * c[1] + c[2] * c[2]};
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) G[i * 5 + j] += phi[i] * phi[j];
    }
    if (!invert5(G, ta.ginv)) return set_error(DGFS_ERR_INVALID, "singular moment Gram matrix");
  }
  ta.phase = phase;
  ta.w1 = w1;
  ta.b2 = b2;
  ta.cvec = cvec;
  ta.ginv_out = ginv;
  const int work = P * M * 3 * N > V ? P * M * 3 * N : V;
  noalloc_tables_kernel<T><<<(work + 255) / 256, 256, 0, stream>>>(ta);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "table kernel launch: %s", cudaGetErrorString(e));

  const int pi = sizeof(T) == 8 ? 1 : 0, ni = N == 8 ? 0 : N == 16 ? 1 : N == 24 ? 2 : 3;
  int rc = setup_shape(st, pi, ni);
  if (rc) return rc;
  const Shape& s = shape_for(p->precision, N);
  int ncl = st->max_clusters[pi][ni];
  if (ncl > fit) ncl = fit;
  if (ncl > npts) ncl = npts;

  VhsArgs<T> a{};
  a.f = (const T*)f;
  a.Q = (T*)Q;
  a.ldim = ldim;
  a.nupts = nupts;
  a.neles = neles;
  a.soasz = soasz;
  a.pt0 = pt0;
  a.npts = npts;
  a.P = P;
  a.M = M;
  a.phase = (const cx<T>*)phase;
  a.w1 = (const T*)w1;
  a.b2 = (const T*)b2;
  a.fc = fc;
  a.err = err;
  a.prefac = (T)p->prefactor;
  a.project = p->project ? 1 : 0;
  a.ginv = ginv;
  a.cvec = cvec;
  if constexpr (sizeof(T) == 8) e = s.launch64(a, ncl, stream);
  else e = s.launch32(a, ncl, stream);
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "VHS launch failed: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

}  // namespace

extern "C" int dgfs_vhs_apply_noalloc(const dgfs_vhs_params* p, const void* f, void* Q, int nupts, int neles,
                                      long long ldim, int soasz, int elem, int upt, void* stream) {
  using ::dgfs::set_error;
  ::dgfs::clear_error();
  if (!p) return set_error(DGFS_ERR_INVALID, "null parameters");
  if (p->Nv != 8 && p->Nv != 16 && p->Nv != 24 && p->Nv != 32)
    return set_error(DGFS_ERR_UNSUPPORTED, "Nv=%d not supported (8, 16, 24, 32)", p->Nv);
  if (p->precision != 32 && p->precision != 64)
    return set_error(DGFS_ERR_INVALID, "precision must be 32 or 64, got %d", p->precision);
  if (p->Nrho < 1 || p->Nrho > kMaxNrho || p->M < 1 || p->M > kMaxM)
    return set_error(DGFS_ERR_INVALID, "Nrho=%d M=%d outside the static limits (Nrho <= %d, M <= %d)", p->Nrho, p->M,
                     kMaxNrho, kMaxM);
  if (!p->qz || !p->qw || !p->sz) return set_error(DGFS_ERR_INVALID, "null quadrature array");
  if (!(p->L > 0) || !std::isfinite(p->L) || !std::isfinite(p->prefactor) || !std::isfinite(p->gamma) ||
      !std::isfinite(p->sw))
    return set_error(DGFS_ERR_INVALID, "bad scalar parameter");
  if (!f || !Q) return set_error(DGFS_ERR_INVALID, "null bank pointer");
  if (nupts < 1 || neles < 1 || soasz < 1)
    return set_error(DGFS_ERR_INVALID, "bad bank shape nupts=%d neles=%d soasz=%d", nupts, neles, soasz);
  const long long V = (long long)p->Nv * p->Nv * p->Nv;
  const long long nblk = (neles + soasz - 1) / soasz;
  if (ldim < nblk * soasz * V) return set_error(DGFS_ERR_INVALID, "ldim=%lld smaller than one AoSoA row", ldim);
  const size_t esz = p->precision == 64 ? 8 : 4;
  const char *fb = (const char*)f, *qb = (const char*)Q;
  const size_t bytes = (size_t)nupts * (size_t)ldim * esz;
  if (fb < qb + bytes && qb < fb + bytes) return set_error(DGFS_ERR_INVALID, "f and Q overlap");
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
  DeviceState* st = nullptr;
  int rc = current_state(&st);
  if (rc) return rc;
  if (p->precision == 64)
    return run<double>(p, st, f, Q, nupts, neles, ldim, soasz, pt0, npts, (cudaStream_t)stream);
  return run<float>(p, st, f, Q, nupts, neles, ldim, soasz, pt0, npts, (cudaStream_t)stream);
}

namespace dgfs {
int noalloc_check_wait(unsigned long long limit_ns, void* stream) {
  DeviceState* st = nullptr;
  int rc = current_state(&st);
  if (rc) return rc;
  const cudaError_t e = launch_wait_check(flag_ptr(st), (uint64_t)limit_ns, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "wait check launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}
}  // namespace dgfs

extern "C" int dgfs_vhs_noalloc_status(void* stream, int* flag) {
  using ::dgfs::set_error;
  ::dgfs::clear_error();
  if (!flag) return set_error(DGFS_ERR_INVALID, "null argument");
  *flag = 0;
  DeviceState* st = nullptr;
  int rc = current_state(&st);
  if (rc) return rc;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
  int v = 0;
  if ((e = cudaMemcpy(&v, flag_ptr(st), sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (v && (e = cudaMemset(flag_ptr(st), 0, sizeof(int))) != cudaSuccess))
    return set_error(DGFS_ERR_CUDA, "error flag: %s", cudaGetErrorString(e));
  *flag = v;
  if (v) return set_error(DGFS_ERR_CUDA, "an allocation-free VHS launch gave up waiting for cluster data (flag %d)", v);
  return DGFS_OK;
}
