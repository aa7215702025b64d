/*
 * rgf.h -- C ABI of the B200 (sm_100a) recursive Green's function library.
 *
 * The library replaces the per-energy Fortran subroutines
 *
 *   green_RGF_RS   src/green_rgf.f90:3950-3958   (module green_rgf)
 *   RGF_G          src/rgf_mod.f90:26-35         (module rgf_mod, same math)
 *
 * of liteQT / eXcitonQT, and the loops that call them once per energy
 * (`do ik / !$omp do ie` at src/green_rgf.f90:2914-2925, :733-742, :968-977,
 * :3174-3178, src/gw_sparse.f90:283-294) with one batched launch.
 *
 * Conventions (identical to the Fortran callers, so ISO_C_BINDING binds them
 * with no copies):
 *   - every matrix array is complex(8), column-major, dimension (nm,nm,nx):
 *     element (i,j) of block l (all 0-based) sits at i + j*nm + l*nm*nm;
 *     rgf_c16 is bit-compatible with complex(8), double _Complex and
 *     std::complex<double>;
 *   - `cur` is real(8) with the same (nm,nm,nx) layout;
 *   - dimensions are int64_t so that `-i8` (ILP64, Makefile.intel:6) and
 *     default-integer builds both bind through integer(c_int64_t);
 *   - pointers may be host or device memory; the library detects which with
 *     cudaPointerGetAttributes and stages host arrays itself;
 *   - a NULL output pointer means "not requested" (the optional Fortran
 *     arguments GRi1 / GLi1 / GGi1, and outputs a batched caller skips).
 *
 * Error behaviour: the reference has no error return; it prints
 * "SEVERE warning" and substitutes a zero block for a singular inverse
 * (green_rgf.f90:4429-4437) and drops the lead self-energy when Sancho does
 * not converge in nmax iterations (:4513-4518).  The library reproduces both
 * and in addition reports them: every entry point returns RGF_OK or an
 * RGF_E* code, and per-task status words carry RGF_ST_* bits.
 */
#ifndef LITEQT_B200_RGF_H
#define LITEQT_B200_RGF_H

#include <stdint.h>

#if defined(__GNUC__)
#define RGF_API __attribute__((visibility("default")))
#else
#define RGF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rgf_c16 { double re, im; } rgf_c16;

/* return codes */
#define RGF_OK             0
#define RGF_E_ARG         -1   /* invalid argument (sizes, pointers) */
#define RGF_E_CUDA        -2   /* a CUDA call failed; see rgf_last_error() */
#define RGF_E_NOMEM       -3   /* device allocation failed */
#define RGF_E_UNSUPPORTED -4   /* option or size not supported by this build */
#define RGF_E_STATUS      -5   /* solve ran; some task has a non-zero status word */

/* per-task status bits */
#define RGF_ST_SINGULAR    1   /* a block inverse hit a zero pivot; block set to 0 (compat) */
#define RGF_ST_SANCHO_NC   2   /* Sancho-Rubio hit nmax; lead self-energy dropped (compat) */
#define RGF_ST_BAD_TASK    4   /* task descriptor rejected on the device */
#define RGF_ST_REFINE_NC   8   /* mixed precision, informational: a refined inverse did not converge
                                  and that block was inverted in FP64 instead (results unaffected;
                                  not an error: RGF_E_STATUS ignores this bit) */
#define RGF_ST_TIMEOUT    16   /* mixed precision: a bounded tensor-core wait gave up; the task's
                                  outputs are invalid and its CTA stopped */

/* precision modes */
#define RGF_PREC_FP64  0       /* complex FP64 throughout: the drop-in */
#define RGF_PREC_MIXED 1       /* nb = 128: split-integer block products on the int8 tensor cores
                                  (tcgen05), FP32 inverses refined against FP64 residuals;
                                  Sancho-Rubio and the lead self-energies in FP64 */

typedef struct rgf_opts {
  int32_t struct_size;     /* sizeof(rgf_opts); filled by rgf_opts_default */
  int32_t device;          /* CUDA device ordinal */
  double eta_dev;          /* device broadening; 0 = z = dcmplx(E,0.0d-6) (green_rgf.f90:3974) */
  double eta_lead;         /* Sancho broadening; 1e-3 (green_rgf.f90:4474) */
  double boltz;            /* 8.61734e-5 eV/K (green_rgf.f90:3968); RGF_G uses 8.617333262e-5 */
  double sancho_tol;       /* 1e-100 (green_rgf.f90:4457) */
  int32_t sancho_nmax;     /* 100 (green_rgf.f90:4473) */
  int32_t consistent;      /* 0: backward sweep couples with H1i(:,:,l) as the reference does
                              (green_rgf.f90:4070); 1: with H1i(:,:,l+1) = H_{l+1,l} */
  int32_t precision;       /* RGF_PREC_FP64 or RGF_PREC_MIXED */
  int32_t want_T;          /* also compute Caroli T(E) (green.f90:2571-2580) */
  int32_t verbose;         /* 1: print "SEVERE warning" lines like the reference */
  int32_t zero_copy;       /* 1 (default): outputs in pinned host memory that the solver only
                              writes (all but `cur`) are written by the kernels through their
                              device mapping, so the transfer overlaps the solve; 0: staged in
                              device memory and copied back after the launch */
  int32_t pipelined;       /* 1: rgf_solve_batch / rgf_solve_energies called with info = NULL
                              return once the solve is queued: outputs are staged in one of two
                              device buffers (taken in turn); a copier thread of the context
                              queues the host copies of each task's blocks as the kernel reports
                              them written, on the context's copy stream, so the copies run
                              while the solve runs and overlap the next call's solve.
                              Host outputs (and tr, tre, T) hold the results after
                              rgf_ctx_synchronize(ctx), which also completes the statistics;
                              until then the host arrays must not be read or reused.
                              Pageable host outputs are copied by the same thread through
                              pinned bounce buffers (below), also while the solve runs.  A
                              call with info != NULL runs as with 0.
                              Pageable (not page-locked) host arrays, in either mode, move
                              through pinned bounce slots of the context (16 x 8 MB) with the
                              host side split over a process-wide pool of host threads, at
                              the host link's speed rather than the driver's one-thread
                              pageable path. */
  int32_t reserved[5];
} rgf_opts;

typedef struct rgf_ctx rgf_ctx;

/* One device (Hamiltonian) shared by many energy points.  Hii and H1i are
 * (nm,nm,nx); H1i(:,:,l) couples block l-1 to block l (forward-sweep meaning),
 * H1i(:,:,1) and Hii(:,:,1) / Hii(:,:,nx), H1i(:,:,nx) also define the two
 * semi-infinite leads, exactly as in green_RGF_RS.
 * Sii: NULL for an orthogonal basis (green_RGF_RS / RGF_G); otherwise the
 * (nm,nm,nx) overlap blocks of a non-orthogonal basis, which selects
 * green_RGF_CMS (src/green_rgf.f90:4167-4383): z*Sii(:,:,l) in place of z*I,
 * sigma_r_ph(:,:,l)*Sii(:,:,l) and sigma_lesser_ph(:,:,l)*Sii(:,:,l) in place
 * of the self-energies, Sancho-Rubio leads with the end blocks' overlap, and
 * G^>_ll (pdens, l < nx) and GGi1 from that routine's own recursion through
 * the never-filled Glp (zero) instead of G^> = G^< + G^R - G^A. */
typedef struct rgf_device {
  int64_t nm, nx;
  const rgf_c16* Hii;
  const rgf_c16* H1i;
  double mu[2];            /* (muL, muR) eV */
  double temp[2];          /* (TL, TR) K */
  const rgf_c16* Sii;      /* overlap blocks, or NULL = identity */
} rgf_device;

/* One (device, k, E) task: one call of green_RGF_RS.  Inputs and outputs are
 * (nm,nm,nx) arrays of the task's device, or NULL. */
typedef struct rgf_task {
  int32_t device;          /* index into the rgf_device array */
  int32_t reserved;
  double E;                /* energy, eV */
  const rgf_c16* sigma_lesser;   /* sigma_lesser_ph, or NULL = 0 */
  const rgf_c16* sigma_r;        /* sigma_r_ph, or NULL = 0 */
  rgf_c16* ldos;           /* G^R_ll        (ldos)   */
  rgf_c16* ndens;          /* G^<_ll        (ndens)  */
  rgf_c16* pdens;          /* G^>_ll        (pdens)  */
  rgf_c16* GRi1;           /* G^R_{l,l+1}   (GRi1)   */
  rgf_c16* GLi1;           /* G^<_{l,l+1}   (GLi1)   */
  rgf_c16* GGi1;           /* GGi1 exactly as the reference fills it (green_rgf.f90:4094-4103) */
  double* cur;             /* bond-current matrix cur(:,:,l) */
  double* tr;              /* right-contact current spectrum (scalar) */
  double* tre;             /* left-contact current spectrum (scalar) */
  double* T;               /* Caroli transmission (scalar; needs opts.want_T) */
} rgf_task;

/* Per-task diagnostics written by rgf_solve_batch when `info` is non-NULL. */
typedef struct rgf_task_info {
  int32_t status;          /* RGF_ST_* bits */
  int32_t sancho_iters_left;
  int32_t sancho_iters_right;
  int32_t n_gemm;          /* nb^3 complex products executed in FP64 */
  int32_t n_inv;           /* nb x nb inversions executed in FP64 */
  int32_t mixed_pairs;     /* RGF_PREC_MIXED: digit-pair products of the split-integer form
                              (products and refinement steps; each is 4 real nb^3 int8
                              products on the tensor cores) */
} rgf_task_info;

/* Measurements of the last rgf_solve_batch on a context. */
typedef struct rgf_stats {
  double last_kernel_ms;   /* device time of its solver launches (CUDA events on its stream) */
  double last_flops;       /* executed FP64 real flops: 8 nb^3 (n_gemm + n_inv) summed over tasks */
  int64_t last_tasks;      /* tasks in it */
  int64_t launches;        /* solver kernel launches since the context was created */
  double last_int8_ops;    /* RGF_PREC_MIXED: int8 tensor-core operations (2 per multiply-add) of
                              the split-integer products: 8 nb^3 per digit pair */
  int64_t reserved[3];
} rgf_stats;

/* Options with the reference's behaviour (compat mode). */
RGF_API void rgf_opts_default(rgf_opts* opts);

/* Context: owns the device workspace and streams.  Not thread-safe: use one
 * context per host thread, or serialise calls. */
RGF_API int rgf_ctx_create(const rgf_opts* opts, rgf_ctx** ctx);
RGF_API int rgf_ctx_destroy(rgf_ctx* ctx);
RGF_API int rgf_ctx_set_opts(rgf_ctx* ctx, const rgf_opts* opts);
RGF_API int rgf_ctx_get_stats(const rgf_ctx* ctx, rgf_stats* stats);
/* Waits until every solve and output copy the context has queued
 * (rgf_opts.pipelined) is complete and fills the last call's statistics. */
RGF_API int rgf_ctx_synchronize(rgf_ctx* ctx);

/* Batched solve: replaces the whole `do ik / !$omp do ie / call green_RGF_RS`
 * loop.  All tasks run in one persistent launch that drains a work queue.
 * `stream` is a cudaStream_t (NULL = the context's stream).  The call returns
 * when all outputs are written (host outputs copied back; when a call stages
 * 64 MB or more of host outputs, they are copied while the solve runs, block
 * by block as the kernel reports them written).  Returns RGF_OK,
 * RGF_E_STATUS if any task status is non-zero, or an error code. */
RGF_API int rgf_solve_batch(rgf_ctx* ctx, const rgf_device* devices, int32_t n_devices,
                    const rgf_task* tasks, int64_t n_tasks, rgf_task_info* info, void* stream);

/* Reusable batched solve captured in a CUDA graph.  No counterpart in the
 * reference: for drivers that solve the same task list again and again (the
 * self-consistent GW and Poisson loops re-solve every energy with new
 * self-energies or potentials written in place).  rgf_plan_create checks the
 * task list, builds the device task table and workspace once and captures the
 * launch (queue reset + one persistent launch over all tasks, any mix of
 * block sizes) in a CUDA graph; rgf_plan_execute replays it on `stream`.
 * Every array the devices and tasks reference must be device memory and stay
 * valid while the plan exists; their contents may change between executions
 * (they are read when the graph runs), the energies and addresses may not.
 * The plan keeps the context's options and kernel choices of creation time. */
typedef struct rgf_plan rgf_plan;
RGF_API int rgf_plan_create(rgf_ctx* ctx, const rgf_device* devices, int32_t n_devices,
                            const rgf_task* tasks, int64_t n_tasks, rgf_plan** plan);
/* Replay.  info == NULL: returns once the graph is launched (stream-ordered).
 * info != NULL (host, n_tasks entries): waits for the solve, copies the
 * per-task diagnostics, updates the context's stats and returns
 * RGF_E_STATUS if any status word is non-zero. */
RGF_API int rgf_plan_execute(rgf_plan* plan, rgf_task_info* info, void* stream);
RGF_API int rgf_plan_destroy(rgf_plan* plan);

/* Autotuner.  No counterpart in the reference.  For the block size of
 * `device`, times every kernel variant that supports it (staged GEMM with
 * blocked inverse for nb = 32, 64, 128, 256; register-direct GEMMs with 8x8,
 * 8x16 and 16x16 warp tiles for any multiple of 8 / 16) at 1 and at the
 * largest number of resident CTAs per SM, each on a probe batch of the
 * device's first min(nx, 12) blocks with one energy per resident CTA
 * (outputs G^R_ll, G^<_ll, T; energies spread over [-3, 3] eV), and keeps the
 * fastest per energy in the context for later solves of that block size.
 * Inputs may be host or device memory.  result may be NULL. */
typedef struct rgf_tune_result {
  int32_t nb;
  int32_t variant;              /* chosen kernel variant (rgf_variant_name) */
  int32_t ctas_per_sm;          /* chosen resident CTAs per SM */
  int32_t n_candidates;
  int32_t cand_variant[16];
  int32_t cand_ctas_per_sm[16];
  double cand_us_per_energy[16];
} rgf_tune_result;
RGF_API int rgf_autotune(rgf_ctx* ctx, const rgf_device* device, rgf_tune_result* result);
/* Name of a kernel variant id ("staged128", "generic2x2", ...). */
RGF_API const char* rgf_variant_name(int32_t variant);

/* Drop-in for green_RGF_RS (src/green_rgf.f90:3950): same arguments in the
 * same order, scalars by reference.  sigma_greater_ph is accepted and unused,
 * as in the reference.  GRi1 / GLi1 / GGi1 may be NULL (absent optional). */
RGF_API int rgf_green_rgf_rs(rgf_ctx* ctx, const double* temp, const int64_t* nm, const int64_t* nx,
                     const double* E, const double* mu, const rgf_c16* Hii, const rgf_c16* H1i,
                     const rgf_c16* sigma_lesser_ph, const rgf_c16* sigma_greater_ph,
                     const rgf_c16* sigma_r_ph, rgf_c16* ndens, rgf_c16* pdens, rgf_c16* ldos,
                     double* tr, double* tre, double* cur, rgf_c16* GRi1, rgf_c16* GLi1,
                     rgf_c16* GGi1);

/* Drop-in for RGF_G (src/rgf_mod.f90:26): its argument order (tr, tre before
 * the density arrays) and its BOLTZ (8.617333262e-5, parameters.f90:38). */
RGF_API int rgf_rgf_g(rgf_ctx* ctx, const double* temperature, const int64_t* nm, const int64_t* nx,
              const double* E, const double* mu, const rgf_c16* Hii, const rgf_c16* H1i,
              const rgf_c16* sigma_lesser_ph, const rgf_c16* sigma_greater_ph,
              const rgf_c16* sigma_r_ph, double* tr, double* tre, rgf_c16* ndens,
              rgf_c16* pdens, rgf_c16* ldos, double* cur, rgf_c16* GRi1, rgf_c16* GLi1,
              rgf_c16* GGi1);

/* Drop-in for green_RGF_CMS (src/green_rgf.f90:4167): green_RGF_RS's
 * arguments with the overlap blocks Sii before Hii, as in the reference. */
RGF_API int rgf_green_rgf_cms(rgf_ctx* ctx, const double* temp, const int64_t* nm, const int64_t* nx,
                      const double* E, const double* mu, const rgf_c16* Sii, const rgf_c16* Hii,
                      const rgf_c16* H1i, const rgf_c16* sigma_lesser_ph,
                      const rgf_c16* sigma_greater_ph, const rgf_c16* sigma_r_ph, rgf_c16* ndens,
                      rgf_c16* pdens, rgf_c16* ldos, double* tr, double* tre, double* cur,
                      rgf_c16* GRi1, rgf_c16* GLi1, rgf_c16* GGi1);

/* Strided batch over the energies of one device, in the layout the reference
 * drivers allocate: g(nm,nm,nx,nen) (green_rgf.f90:2880-2890, one ik slice).
 * Any array may be NULL.  Equivalent to nen calls of green_RGF_RS. */
RGF_API int rgf_solve_energies(rgf_ctx* ctx, const rgf_device* device, int64_t nen, const double* E,
                       const rgf_c16* sigma_lesser, const rgf_c16* sigma_r, rgf_c16* ldos,
                       rgf_c16* ndens, rgf_c16* pdens, rgf_c16* GRi1, double* cur, double* tr,
                       double* tre, double* T, rgf_task_info* info, void* stream);

/* Adjoint RGF (no counterpart in the reference; the Jacobian a Newton-Poisson
 * loop needs).  For every energy of one ballistic device (no scattering
 * self-energy) it returns the Caroli transmission T(E) and its derivatives
 *   dTdV[e*nx + l] = dT(E_e)/dV_l,  V_l adding V_l * I to Hii(:,:,l+1)
 *                    (the end blocks also shift their semi-infinite leads,
 *                    which are the continuation of Hii(:,:,1) / Hii(:,:,nx));
 *   dTds[e]        = dT(E_e)/ds,    s scaling the interior couplings
 *                    H1i(:,:,m), m = 2..nx-1 (1-based),
 * from one reverse sweep with sqrt(nx) checkpoints of the left-connected
 * Green's functions.  If dIdV (nx values) / dIds (1 value) are non-NULL they
 * receive the derivatives of the Landauer current
 *   I = spindeg * e0^2/(2 pi hbar) * dE * sum_e T(E_e) (f_L(E_e) - f_R(E_e)),
 * with dE = E[1] - E[0] and the constants of green_rgf.f90:18-24.  T, dTdV and
 * dTds may be host or device memory; E, dIdV and dIds are host memory.
 * Orthogonal basis only (device->Sii must be NULL). */
RGF_API int rgf_adjoint_energies(rgf_ctx* ctx, const rgf_device* device, int64_t nen,
                                 const double* E, double* T, double* dTdV, double* dTds,
                                 double spindeg, double* dIdV, double* dIds,
                                 rgf_task_info* info, void* stream);

/* Screened interaction W (green_rgf_calc_w, src/green_rgf.f90:3399-3831 ==
 * RGF_W, src/rgf_mod.f90:242-674) for the GW loop: W^R = (I - V P^R)^-1 V and
 * W^<, W^> from W^R and P^<, P^> by the routine's own formula, per
 * (q, energy) task, all tasks in one persistent launch.  This is the form
 * every call site uses (green_rgf.f90:846, :1551, :3008): NBC = 0 and no
 * off-diagonal P blocks.  V is the device's bare interaction: Vii diagonal
 * blocks, V1i(:,:,l) = V_{l+1,l} (and V_{l,l+1} = V1i(:,:,l)^H); its W^R
 * off-diagonal block formula assumes V real symmetric and P^R complex
 * symmetric, as the physical inputs are. */
typedef struct rgf_w_device {
  int64_t nm, nx;
  const rgf_c16* Vii;
  const rgf_c16* V1i;
} rgf_w_device;

typedef struct rgf_w_task {
  int32_t device;          /* index into the rgf_w_device array */
  int32_t reserved;
  const rgf_c16* PL;       /* P^< diagonal blocks (nm,nm,nx) */
  const rgf_c16* PG;       /* P^> */
  const rgf_c16* PR;       /* P^R */
  rgf_c16* WL;             /* W^< diagonal blocks (nm,nm,nx) */
  rgf_c16* WG;             /* W^> */
  rgf_c16* WR;             /* W^R */
  rgf_c16* WRi1;           /* W^R_{l,l+1} (blocks 1..nx-1; block nx untouched), or NULL */
} rgf_w_task;

RGF_API int rgf_w_solve_batch(rgf_ctx* ctx, const rgf_w_device* devices, int32_t n_devices,
                              const rgf_w_task* tasks, int64_t n_tasks, rgf_task_info* info,
                              void* stream);

/* All energies of one q-point in the drivers' layout p(nm,nm,nx,nen)
 * (green_rgf.f90:836-850): PL/PG/PR and WL/WG/WR strided by nm*nm*nx;
 * WRi1 may be NULL. */
RGF_API int rgf_w_solve_energies(rgf_ctx* ctx, const rgf_w_device* device, int64_t nen,
                                 const rgf_c16* PL, const rgf_c16* PG, const rgf_c16* PR,
                                 rgf_c16* WL, rgf_c16* WG, rgf_c16* WR, rgf_c16* WRi1,
                                 rgf_task_info* info, void* stream);

/* Drop-in for green_rgf_calc_w / RGF_W with the reference's argument list
 * (scalars by reference).  NBC other than 0 or present PL1i / PG1i / PR1i
 * (never used by the reference's drivers) return RGF_E_UNSUPPORTED; WLi1 /
 * WGi1 are not written, as in the reference. */
RGF_API int rgf_green_rgf_calc_w(rgf_ctx* ctx, const int64_t* NBC, const int64_t* nm, const int64_t* nx,
                                 const rgf_c16* Vii, const rgf_c16* V1i, const rgf_c16* PL,
                                 const rgf_c16* PG, const rgf_c16* PR, rgf_c16* WL, rgf_c16* WG,
                                 rgf_c16* WR, const rgf_c16* PL1i, const rgf_c16* PG1i,
                                 const rgf_c16* PR1i, rgf_c16* WLi1, rgf_c16* WGi1, rgf_c16* WRi1);

/* The energy / k convolutions of the GW loop of green_rgf_solve_gw_3d
 * (src/green_rgf.f90:2944-3092), as the reference computes them: direct
 * banded sums (|i - j| <= ndiag) over energies and k-points, with
 * nopmax = nen/2 - 10 energy offsets, k - q taken with the reference's nk/2
 * shift, dE = En(2) - En(1).  All arrays (nm,nm,nx,nen,nk), nk = nky*nkz,
 * host or device memory.  imag_only = 1 reads G with its real part zeroed, as
 * the reference zeroes it before these steps (:2940-2942).
 *
 * rgf_gw_polarization: P^<, P^>, P^R (:2944-2999), zero outside the band and
 * outside the nopmax window.
 * rgf_gw_self_energy: the new Sigma^<, Sigma^>, Sigma^R from G and W
 * (:3020-3065), Sigma^R's imaginary part from Sigma^> - Sigma^< (:3068),
 * symmetrisation (:3070-3081), mixing into Sigma_*_gw with alpha_mix
 * (:3083-3085) and the copies of blocks 3 / nx-2 into the two edge blocks of
 * each side (:3087-3092); Sigma_*_gw are updated in place (nx >= 3).
 * Error text: rgf_gw_last_error(). */
RGF_API int rgf_gw_polarization(rgf_ctx* ctx, int64_t nm, int64_t nx, int64_t nen, int64_t nky,
                                int64_t nkz, int64_t ndiag, double dE, double spindeg,
                                int32_t imag_only, const rgf_c16* G_lesser, const rgf_c16* G_greater,
                                const rgf_c16* G_r, rgf_c16* P_lesser, rgf_c16* P_greater,
                                rgf_c16* P_retarded, void* stream);
RGF_API int rgf_gw_self_energy(rgf_ctx* ctx, int64_t nm, int64_t nx, int64_t nen, int64_t nky,
                               int64_t nkz, int64_t ndiag, double dE, double alpha_mix,
                               int32_t imag_only, const rgf_c16* G_lesser, const rgf_c16* G_greater,
                               const rgf_c16* G_r, const rgf_c16* W_lesser, const rgf_c16* W_greater,
                               const rgf_c16* W_retarded, rgf_c16* Sigma_lesser_gw,
                               rgf_c16* Sigma_greater_gw, rgf_c16* Sigma_r_gw, void* stream);
RGF_API const char* rgf_gw_last_error(void);

/* FFT form of the GW convolutions as the production loop with energy <-> (i,j)
 * redistribution computes them (green_rgf_solve_gw_ephoton_3d_ijs,
 * src/green_rgf.f90:1397-1473 and :1598-1678; corr1d2 / conv1d2 with method
 * 'fft', src/fft_mod.f90:56-89, :175-212): the rank's slice of nij (i,j)
 * elements, global indices first_ij .. first_ij+nij-1 (1-based, column-major
 * (i,j) of an nm x nm block), after energies_to_ijs_2.  Arrays are device
 * memory in the *_by_blocks layout (nen, nk, nx, nij) complex(8), nk = nky*nkz,
 * ik = ikz + nkz*(iky-1); nen even.  Elements outside the band |i-j| <= ndiag
 * are written as zeros.  dEn = En(2) - En(1).
 *   rgf_gw_polarization_fft: P^< = sum_k corr(G^<_k, G^>_t,kd), P^> likewise,
 *     P^R = sum_k corr(G^<_k, conj(G^R_kd)) + corr(G^R_k, G^<_t,kd), times
 *     -i dEn/(2 pi) spindeg/nk; G^<_t, G^>_t are the transposed G^<, G^>
 *     (element (j,i)) in the same layout;
 *   rgf_gw_self_energy_fft: Sigma^< = sum_q conv(G^<_kd, W^<_q), Sigma^>
 *     likewise, Sigma^R = conv(G^<, W^R) + conv(G^R, W^<) + conv(G^R, W^R),
 *     times i dEn/(2 pi)/nk, then Sigma^R = Re + i Im(Sigma^> - Sigma^<)/2.
 * The transforms are cuFFT's, in chunks of (i,j, ix) lines within at most
 * 4 GB of device scratch (RGF_GW_FFT_CHUNK sets the lines per chunk); the
 * context keeps the scratch and the cuFFT plans of the last shape between
 * calls and frees them in rgf_ctx_destroy.
 * Stream-ordered on `stream`; returns when the results are written.  Error
 * text: rgf_gw_fft_last_error(). */
RGF_API int rgf_gw_polarization_fft(rgf_ctx* ctx, int64_t nm, int64_t nx, int64_t nen, int64_t nky,
                                    int64_t nkz, int64_t ndiag, int64_t nij, int64_t first_ij, double dEn,
                                    double spindeg, const rgf_c16* G_lesser, const rgf_c16* G_greater,
                                    const rgf_c16* G_r, const rgf_c16* G_lesser_t, const rgf_c16* G_greater_t,
                                    rgf_c16* P_lesser, rgf_c16* P_greater, rgf_c16* P_retarded, void* stream);
RGF_API int rgf_gw_self_energy_fft(rgf_ctx* ctx, int64_t nm, int64_t nx, int64_t nen, int64_t nky,
                                   int64_t nkz, int64_t ndiag, int64_t nij, int64_t first_ij, double dEn,
                                   const rgf_c16* G_lesser, const rgf_c16* G_greater, const rgf_c16* G_r,
                                   const rgf_c16* W_lesser, const rgf_c16* W_greater, const rgf_c16* W_retarded,
                                   rgf_c16* Sigma_lesser_new, rgf_c16* Sigma_greater_new, rgf_c16* Sigma_r_new,
                                   void* stream);
RGF_API const char* rgf_gw_fft_last_error(void);

/* Local transpose of the GW loop's energy <-> (i,j) redistribution
 * (energies_to_ijs_2 / ijs_to_energies_2, src/green_rgf.f90:243-329):
 * dst = RESHAPE(src, dst_shape, ORDER=order) with Fortran's meaning, for pure
 * transposes (dst_shape(order(k)) = src_shape(k)); order is 1-based, ndim <= 8.
 * src and dst are device arrays of complex(8); stream-ordered, returns after
 * the launch.  The MPI_Alltoall between the two transposes is NCCL's
 * all-to-all (liteqt_b200/redistribute.py). */
RGF_API int rgf_permute_c16(rgf_ctx* ctx, const rgf_c16* src, rgf_c16* dst, int32_t ndim,
                            const int64_t* src_shape, const int32_t* order, void* stream);
RGF_API const char* rgf_permute_last_error(void);

/* Terminal current of one energy sweep: sum(tr)*dE*e0/tpi/hbar*e0*spindeg/nk
 * (green_rgf.f90:2938), summed on the device in a fixed order. */
RGF_API int rgf_terminal_current(rgf_ctx* ctx, const double* tr, int64_t nen, double dE, double spindeg,
                         int64_t nk, double* current);

/* Electron / hole densities from Im G^<_jj and Im G^>_jj split at midgap
 * (calc_n_electron, green_rgf.f90:3920-3945).  G arrays (nm,nm,nx,nen,nk). */
RGF_API int rgf_calc_n_electron(rgf_ctx* ctx, const rgf_c16* G_lesser, const rgf_c16* G_greater,
                        int64_t nen, const double* E, int64_t nm, int64_t nk, int64_t nx,
                        double* nelec, double* pelec, const double* midgap);

/* Batched FP64 solve that allocates no device memory.  No counterpart in the
 * reference: it exists for callers that cannot let a library call cudaMalloc
 * -- host codes whose own memory pool owns all of HBM, or that call the solver
 * inside a loop where cudaMalloc's implicit device synchronisation is not
 * acceptable.  Same meaning as rgf_solve_energies, except:
 *   - every array (device->Hii, H1i and all inputs / outputs) must be device
 *     memory; E (nen energies) and info (nen entries, may be NULL) are host
 *     memory; there is no context: options come per call, `stream` is a
 *     cudaStream_t (NULL = the default stream), and the call returns when the
 *     results are written;
 *   - every array must be on the current device, which must be opts->device;
 *   - its workspace is a fixed 256 MiB array inside the library, reserved on
 *     every GPU that loads the library until the process exits; problems
 *     whose one solver slot plus task tables exceed it ((2 nx + 32) nm^2 * 16
 *     bytes + about 200 bytes per energy) are rejected with RGF_E_ARG;
 *   - the array holds as many solver slots as fit, and one CTA runs per slot:
 *     floor((256 MiB - tables) / ((2 nx + 32) nm^2 * 16 B)) of them, at most
 *     2 per SM.  Small problems run on most of the GPU (nm = 32, nx = 50:
 *     2.2 MB a slot, 124 CTAs); large ones on few SMs (nm = 128, nx = 100:
 *     61 MB a slot, 4 CTAs, about 1/70 of rgf_solve_energies' throughput on
 *     a 148-SM B200);
 *   - the first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current, so make that first
 *     call before any stream capture;
 *   - all calls share the array, which keeps the last call's contents; calls
 *     from one process are serialised by a lock, and calls whose GPU work
 *     overlaps (for example from several processes sharing a device through
 *     MPS, which each see their own copy) must not be assumed to be
 *     independent of that.
 * The error text of a failed call is rgf_noalloc_last_error(). */
RGF_API int rgf_solve_energies_noalloc(const rgf_opts* opts, const rgf_device* device,
                                       int64_t nen, const double* E,
                                       const rgf_c16* sigma_lesser, const rgf_c16* sigma_r,
                                       rgf_c16* ldos, rgf_c16* ndens, rgf_c16* pdens,
                                       rgf_c16* GRi1, double* cur, double* tr, double* tre,
                                       double* T, rgf_task_info* info, void* stream);
RGF_API const char* rgf_noalloc_last_error(void);

/* Bond current between the sub-blocks of every block (calc_block_current,
 * green_rgf.f90:4602-4640): nm = nb*ns orbitals per block as ns sub-blocks
 * of nb; tot_cur / tot_ecur (nb,nb,nx*ns) are the energy sums of the current
 * and energy current, jdens (nb,nb,nx*ns,nen) the energy-resolved current
 * (tot_ecur, jdens may be NULL).  The last sub-block of each block repeats
 * the previous sub-block's value, as in the reference.  Host outputs. */
RGF_API int rgf_calc_block_current(rgf_ctx* ctx, const rgf_c16* H, const rgf_c16* G_lesser,
                                   int64_t nen, const double* E, double spindeg, int64_t nb,
                                   int64_t ns, int64_t nm, int64_t nx, double* tot_cur,
                                   double* tot_ecur, double* jdens);

/* The reference's output writers, so a driver keeps writing identical files
 * (src/green_rgf.f90:4541-4896, :2937-2939).  Sums run on the GPU in each
 * routine's loop order; text follows the routine's FORMAT ('(4E18.4)',
 * '(3E18.4)', '(2E18.4)', '(I4,2E16.6)'; a blank line for `write(11,*)`);
 * files are named dataset // STRING(i) // '.dat' (STRING: 4 digits,
 * zero-padded) or dataset // '_' // STRING(i) // '.dat' as each routine does.
 * Arrays host or device; append as the optional argument.
 *   rgf_write_spectrum: write_spectrum (summed_over_k = 0, nk = 1) and
 *     write_spectrum_summed_over_k (summed_over_k = 1), G(NB*NS,NB*NS,length,nen,nk);
 *   rgf_write_dos: write_dos_summed_over_k;
 *   rgf_write_current_spectrum: write_current_spectrum (kz_summed = 0,
 *     cur(NB,NB,length,nen), name with '_') and ..._summed_over_kz (kz_summed = 1,
 *     cur(NB,NB,length,nen,nk));
 *   rgf_write_current_summed_over_k: cur(NB,NB,nx,nk);
 *   rgf_write_transmission_spectrum: write_transmission_spectrum (nk = 0,
 *     tr(nen), name with '_') and write_transmission_spectrum_k (tr(nen,nk));
 *   rgf_write_id_iteration: one line of Id_iteration.dat (appended). */
RGF_API int rgf_write_spectrum(rgf_ctx* ctx, const char* dataset, int32_t iter, const rgf_c16* G, int64_t nen,
                               const double* en, int64_t nk, int64_t length, int64_t NB, int64_t NS, double Lx,
                               const double* coeff, int32_t summed_over_k, int32_t append);
RGF_API int rgf_write_dos(rgf_ctx* ctx, const char* dataset, int32_t iter, const rgf_c16* G, int64_t nen,
                          const double* en, int64_t nk, int64_t length, int64_t NB, int64_t NS, double Lx,
                          int32_t append);
RGF_API int rgf_write_current_spectrum(rgf_ctx* ctx, const char* dataset, int32_t iter, const double* cur,
                                       int64_t nen, const double* en, int64_t nk, int64_t length, int64_t NB,
                                       double Lx, int32_t kz_summed, int32_t append);
RGF_API int rgf_write_current_summed_over_k(rgf_ctx* ctx, const char* dataset, int32_t iter, const double* cur,
                                            int64_t nx, int64_t NB, double Lx, int64_t nk);
RGF_API int rgf_write_transmission_spectrum(const char* dataset, int32_t iter, const double* tr, int64_t nen,
                                            const double* en, int64_t nk, int32_t append);
RGF_API int rgf_write_id_iteration(const char* path, int32_t iter, double current_left, double current_right);
RGF_API const char* rgf_io_last_error(void);

/* Reader of the Wannier Hamiltonian file (w90_load_from_file,
 * src/wannierHam.f90:68-130): nvb and spin degeneracy, the three cell vectors,
 * n entries (x, y, z cell offsets, orbital m, orbital n, Re H, Im H) read as
 * Fortran list-directed input; with axis (3 values, 1-based, or NULL) the cell
 * vectors and the first three columns are permuted as the reference's
 * lreorder_axis does.  info receives the dimensions (nb, nx, ny, x/y ranges)
 * and the derived Lx, Ly, Lz, b1, b2; Hr (NULL: dimensions only) receives
 * Hr(nb,nb,nx,ny), complex(8) column-major, zero where the file has no entry.
 * Host-only. */
typedef struct rgf_ham_info {
  int32_t nvb, spin_deg, nb, nx, ny, xmin, xmax, ymin, ymax, n_entries;
  double cell[9];          /* (alpha, beta, gamm) as columns, Angstrom */
  double Lx, Ly, Lz;
  double b1[3], b2[3];
} rgf_ham_info;
RGF_API int rgf_read_ham_dat(const char* path, const int32_t* axis, rgf_ham_info* info, rgf_c16* Hr);

/* Last error message of the calling thread ("" if none). */
RGF_API const char* rgf_last_error(void);

/* Batched block operations of either precision form on device arrays of
 * `count` nb x nb complex(8) column-major blocks (no counterpart in the
 * reference; the building blocks of the solver, exposed for callers that
 * assemble their own recursions and for accuracy checks of the mixed form).
 * rgf_block_product: C_b = op(A_b) op(B_b), op = conjugate transpose when
 *   conj_a / conj_b is non-zero; nb = 128.  RGF_PREC_MIXED: the split-integer
 *   product on the int8 tensor cores (absolute error below about
 *   2^-44 nb max_k |op(A)_ik| max_k |op(B)_kj|: operands are scaled per row of
 *   op(A) and per column of op(B)); RGF_PREC_FP64: the FP64 DMMA product.
 * rgf_block_inverse: Xinv_b = X_b^-1.  RGF_PREC_FP64 (nb = 32, 64, 128): the
 *   Gauss-Jordan inverse of the plain form (partial pivoting; a zero pivot
 *   gives the zero block and RGF_ST_SINGULAR); RGF_PREC_MIXED (nb = 128): the
 *   FP32 inverse refined by Newton-Schulz steps against FP64 residuals
 *   (RGF_ST_REFINE_NC when a block fell back to the FP64 inverse).
 *   status (host, count entries) may be NULL.
 * Both return after the results are written (on `stream`, NULL = the
 * context's). */
RGF_API int rgf_block_product(rgf_ctx* ctx, int32_t precision, int64_t nb, int64_t count, const rgf_c16* A,
                            int32_t conj_a, const rgf_c16* B, int32_t conj_b, rgf_c16* C, void* stream);
RGF_API int rgf_block_inverse(rgf_ctx* ctx, int32_t precision, int64_t nb, int64_t count, const rgf_c16* X,
                           rgf_c16* Xinv, int32_t* status, void* stream);

/* Library version string. */
RGF_API const char* rgf_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LITEQT_B200_RGF_H */
