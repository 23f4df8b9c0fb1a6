/* deeptime_gpu.h - the C ABI of the B200 backend for deep-time's per-timestep elliptic solves.
 *
 * Two solves, each behind an opaque handle that owns its device buffers, FFT tables, multigrid
 * levels and CUDA graphs for one raster shape (w x h cells of dx metres; x wraps, the first and
 * last rows are closed):
 *
 *   flexure    (L D L + C) x = b, L the 5-point Laplacian; PCG with a spectral preconditioner.
 *              Replaces flexure::Solver (crates/deeptime-core/src/surface/flexure.rs:1471-1741):
 *              dt_flex_create      <- Solver::with_metric   (flexure.rs:1528)
 *              dt_flex_solve       <- Solver::solve         (flexure.rs:1680-1687)
 *              dt_flex_operator    <- Solver::operator      (flexure.rs:1606)
 *              dt_flex_bend        <- Solver::bend          (flexure.rs:1598)
 *   diffusion  (I + dt L_kd) h' = h, L_kd the variable-coefficient 5-point flux Laplacian; CG
 *              preconditioned by one multigrid V-cycle.
 *              dt_diff_solve       <- diffusion::solve      (crates/deeptime-core/src/surface/diffusion.rs:77-85)
 *                                     with DiffusionSolver::Multigrid (multigrid::cg_on,
 *                                     surface/diffusion/multigrid.rs:562-763)
 *
 * Conventions. Host arrays are row-major (x fastest), w*h doubles, borrowed for the call. The
 * `_dev` variants take device pointers and run on the handle's stream. Every call returns a status;
 * no exception crosses the boundary; dt_last_error() gives the calling thread's last message.
 * A handle is not thread-safe: use one per thread (or per stream).
 * There is no CPU fallback: without a usable CUDA device every entry point returns
 * DT_DEVICE_ERROR.
 */
#ifndef DEEPTIME_GPU_H
#define DEEPTIME_GPU_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DT_OK = 0,
  DT_NOT_CONVERGED = 1, /* the iteration cap was reached (the reference's converged = false) */
  DT_NONFINITE = 2,     /* a non-finite value appeared (flexure.rs:2571-2575 maps this to InvalidState) */
  DT_OOM = 3,
  DT_BAD_ARG = 4,
  DT_DEVICE_ERROR = 5,
  DT_UNSUPPORTED = 6    /* a shape or option this build does not handle; see dt_last_error() */
} dt_status;

enum { DT_PRECOND_REFERENCE = 0, /* 3-level ln(alpha) bank inside damped Jacobi sweeps, flexure.rs:1352-1468 */
       DT_PRECOND_MEAN_D = 1 };  /* one spectral solve at the mean rigidity and mean restoring density */
enum { DT_STOP_MAX_Z = 0,        /* the reference's: max |z| < tol metres (flexure.rs:1727-1732) */
       DT_STOP_REL_RESIDUAL = 1, /* ||b - A x||_2 / ||b||_2 <= tol */
       DT_STOP_RMS_RESIDUAL = 2 };/* the reference diffusion's: ||r||_2^2 <= tol^2 n (multigrid.rs:620) */
enum { DT_PREC_FP64 = 0,         /* PCG entirely in FP64 */
       DT_PREC_MIXED = 1,        /* FP32 inner PCG inside FP64 iterative refinement */
       DT_PREC_MIXED_RELIABLE = 2 }; /* one FP32 PCG whose residual is replaced by the FP64 b - A x
                                        (and its correction added to the FP64 x) each time it has
                                        fallen tenfold; the FP64 residual decides convergence */
enum { DT_WARM_NONE = 0,         /* start from x = 0 (the reference) */
       DT_WARM_GIVEN = 1,        /* start from x_inout's contents */
       DT_WARM_UNET = 2 };       /* start from the attached U-Net's prediction (dt_flex_set_unet);
                                    a first guess is kept only when its preconditioned residual is
                                    below the zero guess's (see warm_start_rel_residual) */
enum { DT_CYCLE_JACOBI = 0,      /* the reference's V-cycle: damped Jacobi, omega 0.8, nu 2, to <= 64 cells */
       DT_CYCLE_RBGS = 1 };      /* red-black Gauss-Seidel V(2,2) to a 16 x 8 coarsest level */
enum { DT_DIFF_FP64_CG_FP32_CYCLE = 0, /* the reference's split: FP64 CG, FP32 cycle */
       DT_DIFF_FP64 = 1,               /* FP64 CG and FP64 cycle */
       DT_DIFF_MIXED = 2,              /* FP32 inner CG + FP32 cycle inside FP64 refinement */
       DT_DIFF_MIXED_RELIABLE = 3 };   /* one FP32 CG + FP32 cycle, FP64 reliable updates of x and r */

typedef struct {
  int precond;          /* DT_PRECOND_* */
  int stop;             /* DT_STOP_MAX_Z or DT_STOP_REL_RESIDUAL */
  int precision;        /* DT_PREC_* */
  int warm_start;       /* DT_WARM_* */
  double tol;           /* metres (MAX_Z) or relative residual */
  int max_iterations;   /* PCG iterations (summed over refinements in MIXED) */
  double inner_tol;     /* MIXED: inner relative residual, at least this (default 1e-5) */
  int max_refinements;  /* MIXED: outer FP64 refinements (default 8) */
  int host_loop;        /* diagnostics: 1 = drive the PCG loop from the host, one sync per
                           iteration, instead of the device-side graph loop (for profilers that
                           do not see inside conditional graph nodes); 2 = also print each
                           iteration's scalars to stderr. Default 0. */
} dt_flex_params;

typedef struct {
  /* the reference's SolveReport (flexure.rs:947-952) */
  int iterations;       /* PCG iterations (all refinements) */
  double error_m;       /* the last max |z| (the reference's error estimate), metres */
  int converged;
  /* additions */
  double rel_residual;  /* ||b - A x|| / ||b|| at exit (recomputed in FP64) */
  int refinements;      /* MIXED: FP64 refinement steps taken */
  int warm_start_accepted;
  double warm_start_rel_residual; /* sqrt(r0.M^-1 r0 / b.M^-1 b) of the offered first guess, r0 = b - A x0,
                                     M the solve's preconditioner: the guess is kept when it is below 1 */
  double device_ms;     /* device time of the solve (CUDA events on the handle's stream) */
  long long kernel_launches; /* this backend's kernels that ran for the solve */
} dt_report;

typedef struct dt_flex dt_flex;
typedef struct dt_diff dt_diff;

void dt_flex_default_params(dt_flex_params* p);

/* metric_a (h values) and metric_b (h + 1 values) select the sphere's row metric (RowMetric,
 * flexure.rs:954-1010, Solver::with_metric :1528); pass NULL for both for the block metric, and
 * one without the other is DT_BAD_ARG. On the row metric the operator runs the per-block stencil
 * with the rows' couplings, the Jacobi weights take (L D L)'s diagonal on the metric, and the
 * spectral pass solves d L_k^2 + c per wavenumber along y (RowSolve, :1012-1099) in place of the
 * cosine transform, so h need not be a power of two. On the block metric a height that is not a
 * power of two takes the same row solve with the block couplings (RowMetric::block: a = 1, b = 1
 * inside and 0 at the edges), the cosine transform's inverse; the operator and the Jacobi weights
 * stay the block metric's. Any width from 2 to 65536 is taken, as the reference plans its FFT at
 * any length (Spectral::new, flexure.rs:1139-1170): w/2 a power of two up to 8192 through one
 * shared-memory kernel a pass, every other width through mixed-radix passes (prime factors up to
 * 64) or Bluestein's chirp z-transform. h is at most 8192; larger rasters are DT_UNSUPPORTED. */
dt_status dt_flex_create(int w, int h, double dx, const double* metric_a, const double* metric_b, dt_flex** out);
dt_status dt_flex_destroy(dt_flex* s);
/* Binds the handle to a CUDA stream (cudaStream_t passed as void*); NULL = the handle's own. */
dt_status dt_flex_set_stream(dt_flex* s, void* stream);
/* d = D/g (kg m), c = restoring density (kg/m^3), b = load (kg/m^2); x in metres. With
 * DT_WARM_GIVEN, x_inout holds the first guess on entry. */
dt_status dt_flex_solve(dt_flex* s, const double* d, const double* c, const double* b, double* x_inout,
                        const dt_flex_params* p, dt_report* rep);
dt_status dt_flex_solve_dev(dt_flex* s, const double* d, const double* c, const double* b, double* x_inout,
                            const dt_flex_params* p, dt_report* rep);
/* y = (L D L + C) v and y = L (D L v) (host arrays). */
dt_status dt_flex_operator(dt_flex* s, const double* d, const double* c, const double* v, double* y);
dt_status dt_flex_bend(dt_flex* s, const double* d, const double* v, double* y);
/* z = M^-1 r with the chosen preconditioner (host arrays); for tests of the transforms. */
dt_status dt_flex_precondition(dt_flex* s, const double* d, const double* c, const double* r, double* z, int precond,
                               int precision);

/* y = (L D L + C) v and *vav = v . y on an FP64 raster of w x h cells (device arrays), with no
 * allocation and no solver handle. No counterpart in the reference: it is for callers that cannot
 * allocate device memory at the point of use (a host code that gives the whole device to its own
 * fixed arena, or one that must not synchronise the device, as cudaMalloc and cudaFree can). The
 * reduction's scratch is a fixed device array inside this library: rasters up to
 * DT_NOALLOC_MAX_TILES tiles of 64 x 16 cells (134,217,728 cells, e.g. 16384 x 8192) and at most
 * 65535 rows of tiles (h <= 1,048,560); larger ones return DT_UNSUPPORTED. vav is a device pointer, written on `stream` (cudaStream_t as
 * void*; NULL = the legacy default stream) in stream order; the call does not synchronise.
 * The first call on each device looks the scratch up (this can load the library's device code),
 * so make it before any stream capture that contains the call. The address found is kept for the
 * life of the process: after a cudaDeviceReset by the caller it is stale, so a process that
 * resets a device must not call this entry point on that device again. The scratch is shared by every
 * call on a device: calls that can overlap (other streams, other threads) race on it and must be
 * ordered by the caller. */
#define DT_NOALLOC_MAX_TILES 131072
dt_status dt_flex_operator_dot_noalloc(int w, int h, double dx, const double* d, const double* c, const double* v,
                                       double* y, double* vav, void* stream);

/* ---- diffusion ------------------------------------------------------------------------------ */

typedef struct {
  int cycle;            /* DT_CYCLE_JACOBI (the reference's, default) or DT_CYCLE_RBGS */
  int precision;        /* DT_DIFF_FP64_CG_FP32_CYCLE (the reference's, default), DT_DIFF_FP64, DT_DIFF_MIXED,
                           DT_DIFF_MIXED_RELIABLE */
  int stop;             /* DT_STOP_RMS_RESIDUAL (the reference's: RMS residual < tol metres) or DT_STOP_REL_RESIDUAL */
  double tol;           /* default 1e-5 m (surface.numerics.diffusion_tol_m, params.rs:197-200) */
  int max_iterations;   /* default 400 (CG_MAX_ITER, diffusion.rs:497) */
  int first_guess;      /* 1: the LOD splitting's first guess (the reference, diffusion.rs:101-110); 0: h itself */
  double inner_tol;     /* MIXED: inner relative residual, at least this (default 1e-5) */
  int max_refinements;  /* MIXED: outer FP64 refinements (default 8) */
  int host_loop;        /* diagnostics, as dt_flex_params.host_loop */
} dt_diff_params;

void dt_diff_default_params(dt_diff_params* p);
/* A w x h raster of dx metres, x wrapping when wrap_x (Dims, crates/deeptime-core/src/surface/grid.rs:11-17). */
dt_status dt_diff_create(int w, int h, double dx, int wrap_x, dt_diff** out);
dt_status dt_diff_destroy(dt_diff* s);
dt_status dt_diff_set_stream(dt_diff* s, void* stream);
/* One implicit step: h_inout holds h (m) on entry and h' on return; kd the diffusivity per cell
 * (m^2/yr), dt the step (yr). Iterations in rep->iterations (diffusion::solve's return value);
 * rep->error_m is the final RMS residual (m). */
dt_status dt_diff_solve(dt_diff* s, double* h_inout, const double* kd, double dt, const dt_diff_params* p, dt_report* rep);
dt_status dt_diff_solve_dev(dt_diff* s, double* h_inout, const double* kd, double dt, const dt_diff_params* p, dt_report* rep);
/* y = (I + dt L_kd) x (host arrays). */
dt_status dt_diff_operator(dt_diff* s, const double* kd, double dt, const double* x, double* y);
/* x = the LOD splitting's first guess (diffusion.rs:370-489) from h (host arrays; the solve's own
 * first guess, for tests) */
dt_status dt_diff_lod(dt_diff* s, const double* h, const double* kd, double dt, double* x);
/* z = M^-1 r, one V-cycle from z = 0 (FP32 levels), for tests of the cycle; `levels` receives
 * the hierarchy's depth. */
dt_status dt_diff_vcycle(dt_diff* s, const double* kd, double dt, int cycle, const double* r, float* z, int* levels);
/* Benchmark support (no counterpart in the reference): the average device time (ms) of the
 * finest level's hot kernels for the operator of kd and dt (host array), each launch timed alone
 * with CUDA events on the handle's stream after a write of a buffer twice the L2, and each
 * kernel's algorithmic bytes per launch. Kernel ids, DT_DIFF_PROFILE_KERNELS of them: 0 the CG
 * operator y = A x with x.y in FP64, 1 the same in FP32, 2 the Gauss-Seidel pre-smoothing (two
 * red-black sweeps from z = 0, the residual's restriction fused) in FP32, 3 the post-smoothing
 * (the coarse correction fused, two sweeps) in FP32, 4 and 5 those two in FP64. Rasters whose
 * finest level does not take the tiled sweeps (odd periodic widths, widths under 42) return
 * DT_UNSUPPORTED. */
#define DT_DIFF_PROFILE_KERNELS 6
dt_status dt_diff_profile_kernels(dt_diff* s, const double* kd, double dt, int reps, double* ms, double* bytes);

/* ---- learned warm start ----------------------------------------------------------------------
 * No counterpart in the reference: a 4-level U-Net (32/64/128/256 channels, 3 x 3 convolutions,
 * BF16 weights and activations, FP32 accumulation) that predicts the normalised deflection
 * w * c / rms(b) from (b / rms(b), (log10(d g) - 22.5) / 1.5). Trained by dt_unet_train_step_dev
 * (Adam, MSE) on this library's own tensor-core convolution kernels. Shapes: H a multiple of 8,
 * W a multiple of 512. Device arrays: x [B][H][W][2], targets and predictions [B][H][W] (FP32). */
typedef struct dt_unet dt_unet;
dt_status dt_unet_create(int base_channels, unsigned long long seed, dt_unet** out);
dt_status dt_unet_destroy(dt_unet* u);
size_t dt_unet_num_params(const dt_unet* u);
dt_status dt_unet_set_stream(dt_unet* u, void* stream);
dt_status dt_unet_predict_dev(dt_unet* u, const float* x, float* y, int B, int H, int W);
dt_status dt_unet_train_step_dev(dt_unet* u, const float* x, const float* t, int B, int H, int W, float lr, double* loss);
dt_status dt_unet_loss_and_grad_dev(dt_unet* u, const float* x, const float* t, int B, int H, int W, double* loss);
dt_status dt_unet_gradients(dt_unet* u, float* out, size_t n);
dt_status dt_unet_get_params(dt_unet* u, float* out, size_t n);
dt_status dt_unet_set_params(dt_unet* u, const float* in, size_t n);
dt_status dt_unet_save(dt_unet* u, const char* path);
dt_status dt_unet_load(dt_unet* u, const char* path);
/* Attach a model to a flexure handle for DT_WARM_UNET: its first guess is predicted on the model's
 * cells (model_dx metres, a power-of-two multiple of the raster's dx; block means of b and
 * log10 D), prolonged by Catmull-Rom cubic interpolation (C1, unlike the reference's bilinear
 * prolong_linear, flexure.rs:1816-1844, whose kinks the operator's curvature energy penalises),
 * and kept only when r0.M^-1 r0 < b.M^-1 b. NULL detaches. */
dt_status dt_flex_set_unet(dt_flex* s, dt_unet* u, double model_dx);

/* Benchmark support: the average device time (ms) of each hot kernel of one PCG iteration,
 * launched `reps` times back to back on the handle's stream between CUDA events, on the
 * handle's current data (call after a solve; the solve's output was already returned), and each
 * kernel's algorithmic bytes per launch. Kernel ids, DT_PROFILE_KERNELS of them: 0 operator +
 * p.Ap, 1 x/r update + r.r, 2 direction, 3 rows forward, 4 column DCT-divide-IDCT, 5 rows
 * inverse + r.z, 6 Jacobi left, 7 Jacobi final, 8 rows forward weighted, 9 rows inverse of
 * the bank (its three levels' weighted sum). Kernels 4 and 8 are timed as the bank's solve
 * launches them: where it takes the three levels in one launch (power-of-two transforms), one
 * launch of the three levels, with three levels' bytes; 10 is the column pass of one level, the
 * constant-mean-D preconditioner's. `precision` selects the FP64 or the FP32 lane. */
#define DT_PROFILE_KERNELS 11
dt_status dt_flex_profile_kernels(dt_flex* s, int precision, int reps, double* ms, double* bytes);

/* Implicit diffusion on the cube grid (surface/cube/diffusion.rs::solve with
 * DiffusionSolver::Multigrid, diffusion.rs:244-313): (mu + sum K) x - K x_neighbours = mu h on
 * the 6 n^2 cells, K = dt / mean_area * D * w per neighbour slot, D the side pair's mean
 * diffusivity or a diagonal's least quad side mean; the LOD first guess, CG preconditioned by one
 * FP32 multigrid V-cycle on 2 x 2 face blocks (surface/cube/multigrid.rs), stop at an RMS
 * residual of tol_m over every cell or after 400 iterations, then the residual's sum put back so
 * that sum(area h) is kept. The grid's geometry comes from the caller's CubeGrid at create:
 * slots (6 n^2 x 8, CubeTopology::slots in OFFSETS order, 0xFFFFFFFF where there is none), lap
 * (6 n^2 x 8, CubeGrid::lap) and areas (6 n^2, CubeGrid::areas). The report's error_m is the
 * final RMS residual (m), rel_residual ||mu h - A x|| / ||mu h||. Status DT_NOT_CONVERGED after
 * 400 iterations (h still holds the last iterate, as the reference leaves it). */
typedef struct dt_cube dt_cube;
dt_status dt_cube_create(int n, const uint32_t* slots, const double* lap, const double* areas, dt_cube** out);
dt_status dt_cube_destroy(dt_cube* s);
dt_status dt_cube_set_stream(dt_cube* s, void* stream);
int dt_cube_levels(const dt_cube* s); /* the V-cycle's levels, -1 for NULL */
dt_status dt_cube_diff_solve(dt_cube* s, double* h, const double* kd, double dt, double tol_m, dt_report* rep);
dt_status dt_cube_diff_solve_dev(dt_cube* s, double* h, const double* kd, double dt, double tol_m, dt_report* rep);
/* host arrays: y = A x of the operator for kd and dt; z = one V-cycle of r; the LOD first guess */
dt_status dt_cube_operator(dt_cube* s, const double* kd, double dt, const double* x, double* y);
dt_status dt_cube_vcycle(dt_cube* s, const double* kd, double dt, const double* r, double* z);
dt_status dt_cube_lod(dt_cube* s, const double* kd, double dt, const double* h, double* x);

/* The flexure step's grid helpers on device arrays (row-major, x fastest), enqueued on `stream`
 * (NULL: the legacy default stream) without a host sync; each result is bit-for-bit the
 * reference's.
 *   restrict:       coarse (w/f x h/f) = the mean of each f x f block of fine (w x h); the
 *                   cells of a block summed row by row, then times 1/(f f); f = 1 copies
 *                   (restrict_by, flexure.rs:1773-1795).
 *   prolong_const:  fine (ws f x hs f) = each coarse cell's value on its f x f cells
 *                   (coarse_cell / prolong_const, flexure.rs:1797-1813).
 *   prolong_linear: fine = bilinear interpolation from the coarse cells' centres, x wrapping,
 *                   rows clamped (prolong_linear / linear_at, flexure.rs:1815-1844).
 *   binomial:       `passes` of [1/4, 1/2, 1/4] along x (wrapping) then y (rows clamped), in
 *                   place; scratch holds w h values (binomial, flexure.rs:1745-1762).
 *   box_blur:       `passes` of the radius-r running-sum box along x (wrapping when wrap_x,
 *                   else clamped) then y (rows reflected), in place; scratch holds w h values
 *                   (box_blur, grid.rs:224-270). */
dt_status dt_grid_restrict_dev(int w, int h, int f, const double* fine, double* coarse, void* stream);
dt_status dt_grid_prolong_const_dev(int ws, int hs, int f, const double* coarse, double* fine, void* stream);
dt_status dt_grid_prolong_linear_dev(int ws, int hs, int f, const double* coarse, double* fine, void* stream);
dt_status dt_grid_binomial_dev(int w, int h, int passes, double* v, double* scratch, void* stream);
dt_status dt_grid_box_blur_dev(int w, int h, int wrap_x, int r, int passes, double* v, double* scratch, void* stream);

const char* dt_last_error(void);
/* Library and device facts: 1 when a CUDA device is usable, with its name. */
int dt_device_info(char* name, int len);

#ifdef __cplusplus
}
#endif
#endif
