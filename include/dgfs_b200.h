/*
 * dgfs_b200 -- C ABI of the B200-native DGFS hot path.
 *
 * Two operators of the DGFS solver (Ehsan-Roohi/DGFS-BE-Solver, package
 * frfs) are provided as hand-written sm_100a CUDA behind plain C entry points:
 *
 *   - the fast-spectral VHS collision operator Q(f) at every solution point
 *     (dgfs_vhs_*), replacing DGFSVHSGLLScatteringModel
 *     (frfs/solvers/dgfs/scattering.py:44-286);
 *   - the flux-reconstruction DG advection residual with its interface
 *     and boundary kernels over all N^3 velocities (dgfs_dg_*), replacing
 *     DGFSSystem.rhs / updatebc (frfs/solvers/dgfs/system.py:140-196) and
 *     the integrator's axnpby glue (frfs/backends/cuda/blasext.py:14-43).
 *
 * Conventions
 *   - All arrays passed to *_apply / *_rhs are DEVICE pointers owned by the
 *     caller.  Distribution banks use frfs's AoSoA layout
 *     (frfs/backends/base/types.py:26-47, frfs/backends/cuda/kernels/base.mako:4-6):
 *     value (upt, v, ele) lives at  upt*ldim + ((ele/soasz)*nv + v)*soasz + ele%soasz.
 *   - Host arrays passed to *_create are copied; the library owns its
 *     device tables and frees them in *_destroy.
 *   - precision: 64 = FP64 throughout; 32 = FP32 bulk arithmetic with FP64
 *     moment sums in the optional conservation projection.
 *   - stream: a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Work is stream-ordered; nothing synchronises the host.
 *   - Every function returns 0 on success and a DGFS_ERR_* code otherwise;
 *     dgfs_last_error() returns a message for the calling thread.  The
 *     library never aborts the process.
 *   - A handle is not thread-safe; distinct handles are independent.
 */
#ifndef DGFS_B200_H
#define DGFS_B200_H

#if defined(__GNUC__)
#define DGFS_API __attribute__((visibility("default")))
#else
#define DGFS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define DGFS_OK 0
#define DGFS_ERR_INVALID 1     /* bad argument (size, pointer, range)        */
#define DGFS_ERR_CUDA 2        /* a CUDA runtime call failed                 */
#define DGFS_ERR_UNSUPPORTED 3 /* size/precision/cluster not compiled in     */
#define DGFS_ERR_NOMEM 4       /* device allocation failed                   */

/* Message describing the last error on this thread ("" if none). */
DGFS_API const char* dgfs_last_error(void);

/* Library version string. */
DGFS_API const char* dgfs_version(void);

/* ------------------------------------------------------------------------
 * Fast-spectral VHS collision operator
 *
 * Replaces: DGFSVHSGLLScatteringModel.__init__ / load_parameters /
 * perform_precomputation (frfs/solvers/dgfs/scattering.py:44-224) and
 * fs(d_arr_in, d_arr_out, elem, upt) (scattering.py:227-286).
 * ---------------------------------------------------------------------- */
typedef struct dgfs_vhs dgfs_vhs;

typedef struct dgfs_vhs_params {
  int Nv;             /* velocity points per direction (8, 16, 24, 32)       */
  int Nrho;           /* Gauss radial nodes                                  */
  int M;              /* half-sphere directions                              */
  int precision;      /* 64 or 32                                            */
  double L;           /* velocity domain half width (velocitymesh.py:62)     */
  const double* qz;   /* [Nrho] radial nodes on [0, R]  (velocitymesh.py:124) */
  const double* qw;   /* [Nrho] radial weights           (velocitymesh.py:125) */
  const double* sz;   /* [M*3] half-sphere directions, row-major (:133)      */
  double sw;          /* spherical weight 2 pi / M       (velocitymesh.py:134) */
  double prefactor;   /* scattering.py:61-62                                 */
  double gamma;       /* 2 (1 - omega)                   (scattering.py:53)  */
  int project;        /* 1: FP64 mass/momentum/energy projection of Q        */
  int cluster;        /* CTAs per point (0 = default for Nv/precision)       */
} dgfs_vhs_params;

/* Build the operator: validates sizes, precomputes the axis phases,
 * radial weights b1 and loss kernel b2 (vhs-gll.mako:45-101) on the device
 * current at call time.  Replaces scattering.py:67-224. */
DGFS_API int dgfs_vhs_create(const dgfs_vhs_params* params, dgfs_vhs** out);

DGFS_API int dgfs_vhs_destroy(dgfs_vhs* h);

/* Q(f) for solution points of one element-type bank.
 *   f, Q     : device banks (precision of the handle), AoSoA layout with
 *              nv = Nv^3 variables, nupts rows of leading dimension ldim.
 *   elem,upt : one point (elem >= 0), as fs(..., elem, upt)
 *              (scattering.py:227); elem < 0 applies Q at all
 *              nupts*neles points in one persistent launch, as
 *              DGFSSystem.collide (frfs/solvers/dgfs/system.py:199-218).
 * f and Q must not overlap. */
DGFS_API int dgfs_vhs_apply(dgfs_vhs* h, const void* f, void* Q, int nupts, int neles,
                   long long ldim, int soasz, int elem, int upt, void* stream);

/* Same as dgfs_vhs_apply with elem < 0, restricted to the linear point
 * range [pt0, pt0 + npts), point id = upt*neles + elem. */
DGFS_API int dgfs_vhs_apply_range(dgfs_vhs* h, const void* f, void* Q, int nupts,
                         int neles, long long ldim, int soasz, int pt0,
                         int npts, void* stream);

/* Q(f) at the points of a device list pts[0 .. n), point id =
 * upt*neles + elem, n = min(max_points, *count) when `count` (a device int
 * written by an earlier kernel) is given, else max_points.  Listed ids
 * outside the bank are skipped.  The count is read on the device, so a gate
 * kernel can choose the points without a host round trip.  Used by the
 * learned surrogate's plain fallback; no counterpart in the reference. */
DGFS_API int dgfs_vhs_apply_list(dgfs_vhs* h, const void* f, void* Q, int nupts,
                                 int neles, long long ldim, int soasz,
                                 const int* pts, const int* count,
                                 int max_points, void* stream);

/* Collision frequency nu(c) = prefactor Re IFFT(b2 FFT(f) / V)(c), the loss
 * rate of Q = prefactor (gain - f Re IFFT(b2 F)) (vhs-gll.mako:209-220,
 * 246-266), into a bank of the same layout and precision, at the points
 * with gate[pt] != 0 (all when gate is NULL).  Computed in FP32 whatever
 * the precision (two 3D transforms per point).  Used by the learned
 * surrogate, which keeps the loss term exact; no counterpart in the
 * reference. */
DGFS_API int dgfs_vhs_loss_rate(dgfs_vhs* h, const void* f, void* nu,
                                int nupts, int neles, long long ldim,
                                int soasz, const int* gate, void* stream);

/* Launch geometry chosen by the handle (for reporting and tuning). */
DGFS_API int dgfs_vhs_info(const dgfs_vhs* h, int* cluster, int* threads,
                  int* smem_bytes, int* max_clusters);

/* Change the cluster size (autotuning); 0 restores the default. */
DGFS_API int dgfs_vhs_set_cluster(dgfs_vhs* h, int cluster);

/* Compiled launch shapes for the handle's (Nv, precision): count, and per
 * index the cluster size, whether the exchange buffers are double-buffered
 * (one cluster barrier per (p, q) instead of two), the CTAs per SM the
 * register budget was compiled for, threads per CTA and shared memory. */
DGFS_API int dgfs_vhs_num_variants(const dgfs_vhs* h, int* count);
DGFS_API int dgfs_vhs_variant_info(const dgfs_vhs* h, int idx, int* cluster,
                                   int* double_buffered, int* min_ctas_per_sm,
                                   int* threads, int* smem_bytes);
/* Use launch shape idx for subsequent applies (the autotuner's knob). */
DGFS_API int dgfs_vhs_select(dgfs_vhs* h, int idx);

/* 1 if launch shape idx exchanges by remote pushes (st.async into the
 * owner's shared memory, mbarrier completion), 0 if by remote loads, 2 for
 * the single-CTA kernel (FP32, Nv <= 24: the whole point in one CTA's
 * shared memory, one complex transform per (p, q)), 3 for the two-CTA
 * kernel (FP32, Nv = 32: the same transforms on a pair of CTAs that swap
 * half of the work cube through distributed shared memory once per
 * transform). */
DGFS_API int dgfs_vhs_variant_kind(const dgfs_vhs* h, int idx, int* push);

/* Synchronise `stream`, then report and clear the kernel error flag: the
 * push kernels bound every wait on cluster data (1 s) and set the flag
 * instead of hanging.  Returns DGFS_ERR_CUDA when it was set. */
DGFS_API int dgfs_vhs_status(dgfs_vhs* h, void* stream, int* flag);

/* Allocation-free variant of dgfs_vhs_apply (no counterpart in the
 * reference).  For callers that cannot allocate device memory while they
 * run -- a host whose memory manager owns the device heap, a plugin that may
 * only touch the buffers it is handed, a loop where cudaMalloc's implicit
 * synchronisation is not acceptable.  It takes the same parameters as
 * dgfs_vhs_create and the same bank arguments as dgfs_vhs_apply, builds the
 * tables itself and keeps them and its scratch in one file-scope device array
 * of 24 MiB (held on every GPU that uses this entry point until the process
 * exits); it never calls cudaMalloc or cudaFree.  Limits: Nrho <= 32 and
 * M <= 128 (every such size, up to Nv = 32 in FP64 with the projection,
 * fits in the array); larger sizes are rejected with DGFS_ERR_INVALID.
 * The first call on a device sets it up (symbol address, twiddles, error
 * flag) and the first call for each (precision, Nv) sets that kernel's
 * attributes; those first calls should come before any stream capture.
 * cudaDeviceReset invalidates the set-up and is not supported.  All calls
 * share the array: calls that can overlap on the GPU race.  A bounded wait
 * that gives up sets a flag in the array that stays set until
 * dgfs_vhs_noalloc_status reads it. */
DGFS_API int dgfs_vhs_apply_noalloc(const dgfs_vhs_params* params,
                                    const void* f, void* Q, int nupts,
                                    int neles, long long ldim, int soasz,
                                    int elem, int upt, void* stream);

/* Synchronise `stream`, then report and clear the error flag of the
 * allocation-free path (set by any earlier dgfs_vhs_apply_noalloc launch on
 * the current device whose bounded wait gave up; a Q computed by such a
 * launch is invalid).  Returns DGFS_ERR_CUDA with *flag = 1 when it was
 * set.  No counterpart in the reference. */
DGFS_API int dgfs_vhs_noalloc_status(void* stream, int* flag);

/* Failure-detection check (no counterpart in the reference): one CTA runs
 * the push kernels' bounded wait on an exchange whose 16 bytes never
 * arrive, with a limit of limit_ns nanoseconds (0 .. 1e10), so the wait runs
 * out and sets the error flag of h (reported by dgfs_vhs_status) or, with h
 * NULL, the allocation-free path's flag (dgfs_vhs_noalloc_status).  The
 * wait returns and the launch ends normally; nothing else is touched. */
DGFS_API int dgfs_vhs_check_wait(dgfs_vhs* h, long long limit_ns,
                                 void* stream);

/* ------------------------------------------------------------------------
 * Binary-mixture VSS collision operator
 *
 * Replaces: DGFSBiVSSGLLScatteringModel (frfs/solvers/dgfsbi/
 * scattering.py:44-330): one handle per ordered species pair (p, q) holds
 * the pair's precomputation (scattering.py:172-198, vss-gll.mako:31-93);
 * dgfs_vss_apply evaluates Qij (scattering.py:227-315).  fs(elem, upt,
 * f_0, f_1, Q_0, Q_1) of the reference is Q_p = sum_q Q(f_p, f_q): apply
 * the pair (p, 0) without and (p, 1) with accumulation.
 * ---------------------------------------------------------------------- */
typedef struct dgfs_vss dgfs_vss;

typedef struct dgfs_vss_params {
  int Nv;             /* velocity points per direction (8, 16, 24, 32)      */
  int Nrho;           /* Gauss radial nodes                                 */
  int M;              /* full-sphere directions of the transforms           */
  int Mpre;           /* full-sphere directions of the precomputation       */
  int precision;      /* 64 or 32 (Nv = 32: 32 only)                        */
  double L;           /* velocity domain half width                         */
  const double* qz;   /* [Nrho] radial nodes on [0, R] (dgfsbi/velocitymesh.py:137-140) */
  const double* qw;   /* [Nrho] radial weights                              */
  const double* sz;   /* [M*3] full-sphere design (sw = 4 pi / M)           */
  const double* szpre;/* [Mpre*3] design of the precomputation              */
  double mp, mq;      /* nondimensional masses of species p and q           */
  double alpha;       /* VSS scattering exponent (eta = alpha - 1)          */
  double omega;       /* viscosity exponent (gamma = 2 (1 - omega))         */
  double prefactor;   /* the pair's prefactor (scattering.py:64-87)         */
} dgfs_vss_params;

DGFS_API int dgfs_vss_create(const dgfs_vss_params* params, dgfs_vss** out);
DGFS_API int dgfs_vss_destroy(dgfs_vss* h);

/* Q(f_p, f_q) for one point (elem >= 0) or every point of a bank (elem < 0,
 * one persistent launch); fp, fq, Q device banks of the handle's precision
 * in the AoSoA layout of dgfs_vhs_apply (fp may equal fq; Q overlaps
 * neither); accumulate != 0 adds to Q instead of overwriting it. */
DGFS_API int dgfs_vss_apply(dgfs_vss* h, const void* fp, const void* fq,
                            void* Q, int nupts, int neles, long long ldim,
                            int soasz, int elem, int upt, int accumulate,
                            void* stream);

/* Synchronise `stream`, then report and clear the kernel's bounded-wait
 * error flag (DGFS_ERR_CUDA when a wait gave up). */
DGFS_API int dgfs_vss_status(dgfs_vss* h, void* stream, int* flag);

/* No counterpart in the reference: the launch shape of a handle.  pair = 1
 * selects the two-CTA kernel (FP32, Nv = 24; the default there), pair = 0
 * the cluster exchange kernel.  DGFS_ERR_UNSUPPORTED when the shape does
 * not exist for the handle's precision and Nv. */
DGFS_API int dgfs_vss_select(dgfs_vss* h, int pair);

/* ------------------------------------------------------------------------
 * FR-DG advection residual over all velocities
 *
 * Replaces: the element/interface kernels behind DGFSSystem.rhs and
 * DGFSSystem.updatebc (frfs/solvers/dgfs/system.py:140-196; elements.py:49-118;
 * inters.py:17-229; kernels/{tflux,flux,intcflux,bccflux,bccupdate,
 * negdivconf}.mako, rsolvers/rusanov.mako, bcs/dgfs-*.mako) and the
 * integrator's axnpby combination (frfs/backends/cuda/blasext.py:14-43).
 * The flux-point values live in a library-owned scratch bank.
 * ---------------------------------------------------------------------- */
typedef struct dgfs_dg dgfs_dg;

#define DGFS_BC_WALL_DIFFUSE 0  /* dgfs-wall-diffuse  (inters.py:175-229)  */
#define DGFS_BC_INLET 1         /* dgfs-inlet         (inters.py:312-350)  */
#define DGFS_BC_OUTLET 2        /* dgfs-outlet        (inters.py:386-413)  */
#define DGFS_BC_VANISH 3        /* dgfs-vanish        (inters.py:416-443)  */
#define DGFS_BC_WALL_SPECULAR 4 /* dgfs-wall-specular (inters.py:232-309)  */
#define DGFS_BC_WALL_DIFFUSE_CYL 5 /* dgfs-wall-diffuse-cyl (inters.py:446-492):
                                      diffuse wall whose velocity and
                                      temperature vary along it (bwall)     */
/* dgfs-inlet-normalshock (inters.py:353-383) is DGFS_BC_INLET with a zero
 * guw: the incoming half is selected by c.n alone. */

typedef struct dgfs_dg_params {
  int precision;          /* 64 or 32                                       */
  int ndims;              /* 2 (quadrilaterals)                             */
  int nupts, nfpts;       /* solution / flux points per element             */
  int nvars;              /* discrete velocities V = Nv^3                   */
  int neles;              /* elements                                       */
  int soasz;              /* AoSoA width of the banks (32)                  */
  long long ldim;         /* leading dimension of the solution banks        */
  const double* m0;       /* [nfpts][nupts]            operator M0          */
  const double* m132;     /* [nupts][ndims*nupts]      operator M1 - M3*M2  */
  const double* m3;       /* [nupts][nfpts]            operator M3          */
  const double* smats;    /* [ndims][nupts][ndims][neles] metric terms      */
  const double* rcpdjac;  /* [nupts][neles]            1/|J|                */
  const double* nrm;      /* [nfpts][ndims][neles]     unit outward normals */
  const double* mag;      /* [nfpts][neles]            |S^T n|              */
  const int* partner;     /* [nfpts][neles]: fpt'*neles + ele' of the other
                             side, or -(b+1) for boundary flux point b      */
  const double* cv;       /* [3][nvars] velocity grid                       */
  double cw;              /* velocity cell weight                           */
  int nbfpts;             /* boundary flux points                           */
  const int* bkind;       /* [nbfpts] DGFS_BC_*                             */
  const int* bgroup;      /* [nbfpts] boundary region index                 */
  const int* bfpt;        /* [nbfpts] flux point within its element         */
  const int* bele;        /* [nbfpts] element                               */
  int ngroups;            /* boundary regions                               */
  const double* guw;      /* [ngroups][3] wall / inlet velocity             */
  const double* gfw;      /* [ngroups][nvars] wall / inlet Maxwellian       */
  const int* grefl;       /* [ngroups][nvars] specular reflection map, or NULL */
  const double* bwall;    /* [nbfpts][4] (Ux, Uy, Uz, T) of the wall at each
                             boundary flux point (nondimensional), read for
                             DGFS_BC_WALL_DIFFUSE_CYL points; NULL if none  */
  const double* m12;      /* [nupts][nupts] operator M12 = V^T V for
                             dgfs_dg_invmass (frfs/shapes.py:164-166), or
                             NULL                                           */
  /* Faces shared with other partitions of the mesh (frfs's MPI interfaces,
   * DGFSMPIInters, frfs/solvers/dgfs/inters.py:61-112): a flux point whose
   * partner lives in another partition has partner = -(nbfpts + 1 + h), h
   * the row of the halo buffer that receives the partner's face values
   * (dgfs_dg_set_halo); the send rows list this partition's flux points
   * that others need (dgfs_dg_pack).  Zero / NULL for a whole mesh.        */
  int nhalo;              /* halo rows (received flux points)               */
  int nsend;              /* send rows                                      */
  const int* sfpt;        /* [nsend] flux point of each send row            */
  const int* sele;        /* [nsend] element of each send row               */
} dgfs_dg_params;

DGFS_API int dgfs_dg_create(const dgfs_dg_params* params, dgfs_dg** out);
DGFS_API int dgfs_dg_destroy(dgfs_dg* h);

/* Face values uf = M0 u for velocities [v0, v0+nv) into the scratch bank
 * ('disu', frfs/solvers/dgfs/elements.py:55-59). */
DGFS_API int dgfs_dg_interp(dgfs_dg* h, const void* u, int v0, int nv,
                            void* stream);

/* Diffuse-wall sums over velocities [v0, v0+nv) of the current face values,
 * accumulated in FP64; reset != 0 starts from zero (the vidx == 0 reset of
 * bcs/dgfs-wall-diffuse-update.mako:21-24). */
DGFS_API int dgfs_dg_updatebc(dgfs_dg* h, int v0, int nv, int reset,
                              void* stream);

/* out = alpha*A + beta*B + gamma*(L(u) + C) on velocities [v0, v0+nv),
 * L(u) = -div of the upwind FR-DG flux (DGFSSystem.rhs,
 * frfs/solvers/dgfs/system.py:140-177).  A, B, C may be NULL (term absent)
 * and may alias out; out must differ from u.  Needs dgfs_dg_interp of the
 * same u first (and dgfs_dg_updatebc when diffuse walls are present). */
DGFS_API int dgfs_dg_rhs(dgfs_dg* h, const void* u, void* out, int v0, int nv,
                         double alpha, const void* A, double beta,
                         const void* B, double gamma, const void* C,
                         void* stream);

/* Pack the current face values (dgfs_dg_interp) of the send rows for all
 * velocities: send[s*nvars + v] = uf(sfpt[s], v, sele[s]), a device buffer
 * of nsend*nvars values of the handle's precision (the 'pack' kernel of
 * frfs's MPI interfaces, frfs/solvers/dgfs/inters.py:83-85).  The caller
 * exchanges the rows with the neighbouring partitions (NCCL send/recv). */
DGFS_API int dgfs_dg_pack(dgfs_dg* h, void* send, void* stream);

/* Device buffer of nhalo*nvars received face values (row h = halo row h,
 * all velocities), read by every later dgfs_dg_rhs; required when the
 * handle has partition faces.  The buffer stays owned by the caller. */
DGFS_API int dgfs_dg_set_halo(dgfs_dg* h, const void* recv);

/* out = M12 u on velocities [v0, v0+nv): DGFSSystem.invmass
 * (frfs/solvers/dgfs/system.py:221-231), the 'invmass' kernel of
 * frfs/solvers/dgfs/elements.py:161-164.  Needs m12 at create time; out must
 * differ from u. */
DGFS_API int dgfs_dg_invmass(dgfs_dg* h, const void* u, void* out, int v0,
                             int nv, void* stream);

/* Launch shapes of the residual kernel (the autotuner's knob): count; per
 * index the velocities per warp, whether the Runge-Kutta terms are loaded
 * ahead of the flux work, and the CTAs per SM the register budget was
 * compiled for; dgfs_dg_select sets the shape of later dgfs_dg_rhs calls
 * (index 0 by default).  No counterpart in the reference. */
DGFS_API int dgfs_dg_num_variants(const dgfs_dg* h, int* count);
DGFS_API int dgfs_dg_variant_info(const dgfs_dg* h, int idx, int* vpt,
                                  int* prefetch, int* min_ctas_per_sm);
DGFS_API int dgfs_dg_select(dgfs_dg* h, int idx);
/* 1 when shape idx runs the element-operator contraction on the tensor
 * cores (FP32 handles: tcgen05.mma kind::tf32 with operands split into
 * two TF32 parts, FP32 accuracy), 0 for the SIMT shapes. */
DGFS_API int dgfs_dg_variant_tc(const dgfs_dg* h, int idx, int* tensor_cores);
/* Synchronise the stream and read (and clear) the bounded-wait flag of the
 * tensor-core residual: *flag = 1 and DGFS_ERR_CUDA when a launch gave up
 * waiting for its MMAs. */
DGFS_API int dgfs_dg_status(dgfs_dg* h, void* stream, int* flag);

/* Copy the 2*nbfpts diffuse-wall sums to host memory (synchronous). */
DGFS_API int dgfs_dg_bcvals(const dgfs_dg* h, double* host, int n);

/* Device pointer and leading dimension of the face-value scratch bank. */
DGFS_API int dgfs_dg_fpts(const dgfs_dg* h, void** ptr, long long* ldim);

/* ------------------------------------------------------------------------
 * Stage graphs at the C ABI
 *
 * Replaces the per-kernel launches of a Runge-Kutta stage of
 * StdTVDRK2DGFSStepper / StdEulerDGFSStepper
 * (frfs/integrators/std/steppers.py:39-225) with one graph launch, for
 * callers that reach the library through these entry points only.
 * dgfs_graph_begin starts capturing `stream` (a created stream; capture
 * mode thread-local); the dgfs_* calls that follow on that stream are
 * recorded, not run; dgfs_graph_end stops the capture and instantiates the
 * graph; dgfs_graph_launch replays it on any stream.  Every call inside a
 * capture must have been made once before with the same handles and sizes
 * (first calls set up kernel attributes and scratch), and the captured
 * pointers must stay valid while the graph lives.  If a call inside the
 * capture fails, dgfs_graph_end still ends the capture and reports it.
 * ---------------------------------------------------------------------- */
typedef struct dgfs_graph dgfs_graph;

DGFS_API int dgfs_graph_begin(void* stream);
DGFS_API int dgfs_graph_end(void* stream, dgfs_graph** out);
DGFS_API int dgfs_graph_launch(dgfs_graph* g, void* stream);
DGFS_API int dgfs_graph_destroy(dgfs_graph* g);

/* ------------------------------------------------------------------------
 * Macroscopic moments
 *
 * Replaces: the 3D moment formulas of DGFSMomWriterStdPlugin
 * (frfs/plugins/dgfsmomwriterstd.py:154-214), which copy the whole bank to
 * the host.  For every solution point of a bank (AoSoA, soasz 32, Nv^3
 * variables on the cell-centred grid of half width L, weight cw) writes 14
 * FP64 values out[(upt*neles + ele)*14 + k]: rho, ux, uy, uz, T, qx, qy, qz,
 * Pxx, Pxy, Pxz, Pyy, Pyz, Pzz (nondimensional).  `out` is a device array.
 * ---------------------------------------------------------------------- */
DGFS_API int dgfs_moments(int precision, const void* f, int nupts, int neles,
                          long long ldim, int Nv, double L, double cw,
                          double* out, void* stream);

/* ------------------------------------------------------------------------
 * Learned collision surrogate (no counterpart in the reference)
 *
 * Per point: FP64 frame rho, u, T (the formulas of dgfs_moments);
 * c^ = (c - u)/sqrt(T); phi_n(x) = He_n(sqrt(2) x)/sqrt(n!); 220 modes
 * (i, j, k), i + j + k <= 9, ordered by degree, then i, then j (both
 * descending); window chi(c^) = erfc((|c^| - 4)/0.4)/2; M the local
 * Maxwellian rho T^{-3/2} pi^{-3/2} e^{-|c^|^2}.  Feature row X[pt][256]:
 * a_k = cw/rho sum_v chi (f - M) phi_k(c^_v) (k < 220), sqrt(T)/L,
 * ux/L, uy/L, uz/L, zeros.  Target row B[pt][256]:
 * b_k = cw sum_v chi g phi_k(c^_v) / (prefactor rho^2 T^{gamma/2}), g = Q,
 * or g = Q + nu (f - M) (the gain deviation G - nu M, M the local
 * Maxwellian) when the collision-frequency bank nu is given.  mom[pt][5]
 * = rho, ux, uy, uz, T; eps[pt] = |a_k, degree >= 2| (non-equilibrium
 * measure).  Nv <= 32, soasz 32.  All pointers are device pointers; point
 * id pt = upt*neles + elem.
 * ---------------------------------------------------------------------- */
DGFS_API int dgfs_hermite_embed(int precision, const void* f, const void* Q,
                                const void* nu, int nupts, int neles,
                                long long ldim, int Nv, double L, double cw,
                                double prefactor, double gamma, float* X,
                                float* B, double* mom, float* eps,
                                void* stream);

/* g(c) = prefactor rho^2 T^{gamma/2} T^{-3/2} pi^{-3/2} e^{-|c^|^2}
 * sum_k d_k phi_k(c^) with d = gwinv B[pt] (gwinv: 220x220 row-major
 * inverse of the windowed Gram matrix int chi W phi_k phi_l dc^; NULL uses
 * d = B[pt]); Q = g, or Q = g - nu (f - M) when the banks f and nu are
 * given; then the FP64 projection onto zero mass, momentum and energy with
 * the 5x5 inverse Gram matrix ginv of (1, c, |c|^2) on the grid; written
 * only where gate[pt] != 0 (all points when gate is NULL).  Split mode,
 * with gate, nu, the list rows[0 .. *nrows) of the gate-1 points (device
 * memory, as dgfs_surrogate_gate's net list) and work (device memory of
 * nupts * ceil(neles/32) * 32 * (32 * 5 + 220) doubles): the gate-1 points'
 * coefficients are computed once and their velocity ranges split over 8
 * CTAs each, the gate-2 points (B ignored, Q = -nu (f - M)) go to
 * coalesced kernels that take the 32 points of an AoSoA block at a time,
 * and the projection runs as one coalesced pass. */
DGFS_API int dgfs_hermite_reconstruct(int precision, const float* B,
                                      const double* mom, const int* gate,
                                      int nupts, int neles, long long ldim,
                                      int Nv, double L, double cw,
                                      double prefactor, double gamma,
                                      const double* ginv, const double* gwinv,
                                      const void* f, const void* nu, void* Q,
                                      const int* rows, const int* nrows,
                                      double* work, void* stream);

/* gate[pt] = 1 where eps[pt] < threshold (2 where also eps[pt] < eps_zero:
 * dgfs_hermite_reconstruct then uses zero coefficients, i.e. Q = -nu (f - M)
 * when nu is given) and, when the frames mom are given, the local
 * Maxwellian is resolved by the grid of half width L: min over axes of
 * (L - |u_axis|) >= rmin sqrt(T); gate 0 points are appended to
 * plain[0 .. *nplain) (unordered) for dgfs_vhs_apply_list, and, when net
 * and nnet are given, gate 1 points to net[0 .. *nnet) (the rows the
 * network evaluates). */
DGFS_API int dgfs_surrogate_gate(int npts, const float* eps, float threshold,
                                 float eps_zero, const double* mom, double L,
                                 double rmin, int* gate, int* plain,
                                 int* nplain, int* net, int* nnet,
                                 void* stream);

/* Scale-free surrogate rows, in place on X[M][ld]: columns [c0, c1) are
 * divided (inverse != 0: multiplied) by s = max(eps[m], eps0); forward
 * only, column logcol (>= 0, outside [c0, c1)) receives log(s).  Near
 * equilibrium Q is linear in the deviation f - M, so features and targets
 * divided by the deviation size eps are O(1) across the whole range. */
DGFS_API int dgfs_surrogate_scale(int M, int ld, const float* eps, float eps0,
                                  int c0, int c1, int logcol, int inverse,
                                  float* X, void* stream);

/* Surrogate MLP kernels (FP32 accumulation; B operand FP32 or BF16):
 * C[m*ldc+n] = act(sum_k A[m*sam+k*sak] B[k*sbk+n*sbn] + bias[n]) (+ C),
 * act 0 identity, 1 tanh; Z (optional) receives the pre-activation.
 * mcount (optional, device memory): only rows m < min(M, *mcount) are
 * computed, for row counts the device produced (no host round trip). */
DGFS_API int dgfs_mlp_gemm(int M, int N, int K, const float* A, long long sam,
                           long long sak, const void* B, int b_bf16,
                           long long sbk, long long sbn, const float* bias,
                           float* Z, float* C, long long ldc, int act,
                           int accumulate, const int* mcount, void* stream);
/* The same product on the tensor cores (tcgen05.mma, kind::f16): A and B
 * are rounded to BF16 (nearest even) as they are staged, products
 * accumulate in FP32 in tensor memory. No mcount. err (device int) is set
 * to 1 when a bounded wait of the kernel ran out; the kernel never clears
 * it. */
DGFS_API int dgfs_mlp_gemm_tc(int M, int N, int K, const float* A,
                              long long sam, long long sak, const void* B,
                              int b_bf16, long long sbk, long long sbn,
                              const float* bias, float* Z, float* C,
                              long long ldc, int act, int accumulate,
                              int* err, void* stream);
/* BF16 operands already in memory, loaded by TMA into the tensor cores'
 * swizzled layout (tcgen05.mma kind::f16, FP32 accumulation): op(A) is
 * M x K, element (m, k) at A[m lda + k] (a_mn = 0) or A[k lda + m]
 * (a_mn = 1); op(B) is K x N, element (k, n) at B[n ldb + k] (b_mn = 0) or
 * B[k ldb + n] (b_mn = 1). A and B 16-byte aligned, lda and ldb multiples
 * of 8. C[m ldc + n] = act(sum + bias[n]) (+ C); Z (optional) the
 * pre-activation; Cb (optional) C rounded to BF16, with the same ldc. err
 * as for dgfs_mlp_gemm_tc. */
DGFS_API int dgfs_mlp_gemm_bf16(int M, int N, int K, const void* A, int a_mn,
                                long long lda, const void* B, int b_mn,
                                long long ldb, const float* bias, float* Z,
                                float* C, void* Cb, long long ldc, int act,
                                int accumulate, int* err, void* stream);
/* dZ = dH (1 - H^2) */
DGFS_API int dgfs_mlp_tanh_bwd(long long n, const float* H, const float* dH,
                               float* dZ, void* stream);
/* The same, also writing dZ rounded to BF16 into dZb (the operand of the
 * next tensor-core product). */
DGFS_API int dgfs_mlp_tanh_bwd_bf16(long long n, const float* H,
                                    const float* dH, float* dZ, void* dZb,
                                    void* stream);
/* out[n] (+)= sum_m X[m*ldx+n], fixed order */
DGFS_API int dgfs_mlp_colsum(int M, int N, const float* X, long long ldx,
                             float* out, int accumulate, void* stream);
/* rowloss[m] = sum_{n<nused} w_n (Y-T)^2, dY = 2 w (Y-T)/(M nused) (0 for
 * n >= nused); w may be NULL. */
DGFS_API int dgfs_mlp_mse(int M, int N, int nused, const float* Y,
                          const float* T, const float* w, float* dY,
                          double* rowloss, void* stream);
/* Adam with bias correction; L2 weight decay is added to the gradient
 * (g + wd w); refreshes the BF16 copy wbf16 when not NULL. */
DGFS_API int dgfs_mlp_adam(long long n, float* w, void* wbf16, const float* g,
                           float* m1, float* m2, float lr, float beta1,
                           float beta2, float eps, int step,
                           float weight_decay, void* stream);
/* Adam over a flat buffer of n parameters whose first n_decay take the
 * weight decay; hyper (device) = {lr, 1 - beta1^t, 1 - beta2^t}. */
DGFS_API int dgfs_mlp_adam_dev(long long n, long long n_decay, float* w,
                               void* wbf16, const float* g, float* m1,
                               float* m2, const float* hyper, float beta1,
                               float beta2, float eps, float weight_decay,
                               void* stream);
/* Cosine learning-rate schedule on the device: counters (device) =
 * {it, step}; writes hyper = {lr (lr_min + (1 - lr_min)(1 + cos(pi it /
 * total))/2), 1 - beta1^(step+1), 1 - beta2^(step+1)} and advances both
 * counters by one, so a captured training step replays with the right
 * rate. */
DGFS_API int dgfs_mlp_schedule(int* counters, float* hyper, float lr,
                               float lr_min, int total, float beta1,
                               float beta2, void* stream);
/* Y = (X - mu) inv_sigma per column, or X / inv_sigma + mu (inverse). */
DGFS_API int dgfs_mlp_affine(int M, int N, const float* X, const float* mu,
                             const float* inv_sigma, float* Y, int inverse,
                             void* stream);
/* Through a device row list, for r < min(M, *count): Y[r] =
 * (X[rows[r]] - mu) inv_sigma (gather), or with inverse Y[rows[r]] =
 * X[r] / inv_sigma + mu (scatter); N columns, rows of N floats. */
DGFS_API int dgfs_mlp_affine_rows(int M, int N, const int* rows,
                                  const int* count, const float* X,
                                  const float* mu, const float* inv_sigma,
                                  float* Y, int inverse, void* stream);
DGFS_API int dgfs_f32_to_bf16(long long n, const float* x, void* y,
                              void* stream);

/* ------------------------------------------------------------------------
 * Measurement helper (no counterpart in the reference)
 * ---------------------------------------------------------------------- */

/* Sustained SIMT FMA throughput of the current device (precision 32 or 64),
 * measured with an FMA loop over every SM and CUDA events; the roofline
 * denominator for the SIMT-bound collision kernel.  Blocks the host. */
DGFS_API int dgfs_probe_fma_peak(int precision, int iters, double* tflops,
                                 float* ms, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DGFS_B200_H */
