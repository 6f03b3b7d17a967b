/*
 * gd_poisson.h - C ABI of the B200 gradient-domain Poisson solver.
 *
 * The reference (gradient-domain, pure Python) exposes the Poisson path as
 * Python functions; this library is what those functions bind to through
 * ctypes.  Every pointer argument named *_dev is a device pointer owned by the
 * caller; the library never allocates device memory on a solve.  Every call is
 * ordered on the given CUDA stream and returns GD_OK (0) or a negative error
 * code; gd_last_error() gives the message of the calling thread's last error.
 * A plan is not thread-safe: one host thread drives it at a time.
 *
 * Conventions shared by all entry points:
 *   - grids are row-major (rows = height, cols = width) with a row pitch given
 *     in elements; FP64 arrays are double, masks are uint8 (non-zero = unknown);
 *   - the system solved is A x = f with A the positive five-point operator
 *     (A u = d_p u_p - sum of neighbour values), so the reference's
 *     laplacian(u) = b with spacing h maps to f = -h^2 b.
 */
#ifndef GD_POISSON_H
#define GD_POISSON_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GD_OK 0
#define GD_ERR_ARG (-1)
#define GD_ERR_CUDA (-2)
#define GD_ERR_STATE (-3)
#define GD_ERR_UNSUPPORTED (-4)

/* Boundary of one solve instance. */
enum gd_boundary {
  GD_DIRICHLET = 0, /* rectangle, zero values outside (solvers.py:171 system)   */
  GD_NEUMANN = 1,   /* rectangle, edge-replicated ghosts (solvers.py:224 system) */
  GD_MASKED = 2     /* unknowns where mask != 0, Dirichlet elsewhere (poisson.py:154) */
};

/* Arithmetic of a plan. */
enum gd_precision {
  GD_MIXED = 0, /* FP32 V-cycle and Krylov vectors, FP64 residual/scalars/solution */
  GD_FP64 = 1   /* everything in FP64 */
};

/* Per-instance status words reported by a solve. */
enum gd_status {
  GD_CONVERGED = 0,
  GD_MAX_ITERATIONS = 1,
  GD_BREAKDOWN = 2,  /* p.Ap <= 0 or a non-finite scalar */
  GD_ACTIVE = 3,     /* internal: still iterating */
  GD_STAGNATED = 4   /* the FP64 residual stopped decreasing above the tolerance
                        (the tolerance is below the attainable accuracy) */
};

typedef struct gd_grid_desc {
  int32_t height;   /* unknown rows    */
  int32_t width;    /* unknown columns */
  int32_t boundary; /* enum gd_boundary */
  int32_t flags;    /* bit 0 (Neumann): drop the mean of f, return the zero-mean x (solvers.py:258-262) */
} gd_grid_desc;

typedef struct gd_params {
  int32_t precision;      /* enum gd_precision                                   */
  int32_t pre_sweeps;     /* RB-GS sweeps before restriction (1..3)               */
  int32_t post_sweeps;    /* RB-GS sweeps after prolongation (1..3)               */
  int32_t max_iterations; /* PCG iteration budget (solvers.py:176 default 2000)    */
  double tolerance;       /* target ||f - A x|| / ||f|| (solvers.py:175 default 1e-8) */
  double reliable_delta;  /* mixed precision: residual drop between FP64 refreshes */
  int32_t check_every;    /* host poll interval of solves on direct launches         */
  int32_t use_graph;      /* from a plan's second solve on, run the whole solve as   *
                           * one CUDA graph whose while node loops on the device     */
  int32_t strip_target_warps; /* smoother strips: > 0: warps wanted per level launch,
                                 all instances together (the tallest of 64/32/16/8
                                 rows that gives them); 0: level 0 as for 1800,
                                 coarse levels the height with the fewest waves x
                                 rows (occupancy queried per kernel)               */
  int32_t bottom_cells;       /* largest level the one-CTA bottom takes (0 = 4096)   */
  int32_t tile_cells;         /* largest coarse level on shared-memory tiles (0 = 262144) */
  int32_t zero_start;         /* nonzero: every solve starts from x = 0 and x is only
                                 written (it need not be initialised), as the
                                 reference's solvers start (solvers.py:143)           */
  int32_t persistent_coarse;  /* 1: the V-cycle levels below the strips whose tiles are
                                 fewer than the SMs, the bottom, and those levels again on
                                 the way up run as one persistent cooperative launch per
                                 V-cycle, a grid barrier between levels (per-level launches
                                 where the device or the graph cannot take it); 0 (the
                                 default): one launch per level, measured faster on the
                                 B200 inside the solve graph                            */
  int32_t dependent_launch;   /* 1: the kernels of a solve are launched as programmatic
                                 dependents of the kernel ahead of them (each waits for it
                                 inside), so a launch and its table reads may overlap the
                                 previous kernel's tail; 0 (the default): plain stream
                                 order, measured faster on the B200 inside the solve graph */
} gd_params;

typedef struct gd_report {
  int32_t iterations;        /* PCG iterations taken                      */
  int32_t status;            /* enum gd_status                            */
  double relative_residual;  /* true FP64 ||f - A x|| / ||f|| at exit      */
  double initial_norm;       /* ||f||                                      */
  int32_t refreshes;         /* FP64 residual refreshes after the first    */
  int32_t reserved;
} gd_report;

typedef struct gd_plan_s *gd_plan;

/* Thread-local message of the last failed call ("" if none). */
const char *gd_last_error(void);

/* Library build identification, e.g. "gd_poisson sm_100a". */
const char *gd_version(void);

/* ---------------------------------------------------------------------------
 * Batched MG-preconditioned CG (the B200 replacement of the reference's
 * solve_system(method="mgcg") loop, solvers.py:134-160, its per-channel loops
 * poisson.py:137-145 and :216-242, and the DCT solve_neumann, solvers.py:224-262).
 * -------------------------------------------------------------------------*/

/* Build the multigrid hierarchy and work lists for n instances. */
int gd_plan_create(const gd_grid_desc *grids, int32_t n, const gd_params *params,
                   gd_plan *out);
void gd_plan_destroy(gd_plan plan);

/* Device workspace the caller must provide (bytes, 256-byte aligned). */
size_t gd_plan_workspace_bytes(gd_plan plan);

/* Attach the workspace and upload descriptors; zeroes the hierarchy arrays. */
int gd_plan_bind(gd_plan plan, void *workspace_dev, size_t bytes, cudaStream_t stream);

/* Masked instances only: mask_dev[r*pitch+c] != 0 marks an unknown.  Builds the
 * per-level cell classes; call before gd_plan_prepare. */
int gd_plan_set_mask(gd_plan plan, int32_t instance, const uint8_t *mask_dev,
                     int32_t pitch, cudaStream_t stream);

/* Factor the coarsest grid of every instance (FP64 dense inverse on device). */
int gd_plan_prepare(gd_plan plan, cudaStream_t stream);

/* Solve A x_i = scale_i * f_i for every instance.  f_dev[i], x_dev[i] point to
 * height x width FP64 arrays with row pitch pitch[i] (elements); x_dev[i] holds
 * the initial guess on entry (zero it for the reference's x0 = 0) and the
 * solution on exit.  Unknown-free cells of masked instances are written 0.
 * Blocks until every instance has converged or stopped; fills reports[n]. */
int gd_solve(gd_plan plan, const double *const *f_dev, double *const *x_dev,
             const int32_t *pitch, const double *scale, cudaStream_t stream,
             gd_report *reports);

/* gd_solve in two halves, so that copies and other work can overlap a solve
 * (no counterpart in the reference, whose solves are synchronous Python calls,
 * solvers.py:171-221).
 * gd_solve_async enqueues the solve on `stream` and, once the plan has been
 * solved before (its whole solve is then one CUDA graph with a device-side
 * loop), returns without waiting; a plan's first solve and profiled solves
 * still poll the host and return with the stream drained.  gd_solve_finish
 * waits for that solve and fills reports[n].  One solve per plan may be in
 * flight; gd_solve on a plan with an unfinished solve returns GD_ERR_STATE. */
int gd_solve_async(gd_plan plan, const double *const *f_dev, double *const *x_dev,
                   const int32_t *pitch, const double *scale, cudaStream_t stream);
int gd_solve_finish(gd_plan plan, gd_report *reports);

/* One application of the preconditioner (a single V-cycle from zero) to the
 * FP64 residual r of instance i: z = M r.  Test and inspection hook. */
int gd_plan_apply_vcycle(gd_plan plan, int32_t instance, const double *r_dev,
                         double *z_dev, int32_t pitch, cudaStream_t stream);

/* Exact Neumann solve by the discrete cosine transform, the algorithm of
 * solvers.py:224-262 (replaces scipy dctn / idctn; the FFTs are this
 * library's own shared-memory kernels): u = zero-mean solution of
 * laplacian(u) = b with edge-replicated (Neumann) boundaries, any constant
 * component of b dropped.  Sides of 2 to 8192 cells (GD_ERR_UNSUPPORTED
 * beyond).  Three passes: rows, columns (with the eigenvalue division) and
 * rows again, through one coefficient buffer.  The plan allocates nothing on
 * the device; the caller binds a 256-byte aligned workspace of
 * gd_dct_workspace_bytes (the coefficient buffer and the twiddle and
 * eigenvalue tables, filled at bind on `stream`, which bind then waits for)
 * before solving.  b and u have row pitch
 * `pitch` (elements) and may alias (u = b solves in place). */
typedef struct gd_dct_plan_s *gd_dct_plan;
int gd_dct_plan_create(int32_t h, int32_t w, gd_dct_plan *out);
size_t gd_dct_workspace_bytes(gd_dct_plan plan);
int gd_dct_plan_bind(gd_dct_plan plan, void *workspace_dev, size_t bytes, cudaStream_t stream);
int gd_dct_solve_neumann(gd_dct_plan plan, const double *b_dev, double *u_dev, int32_t pitch,
                         cudaStream_t stream);
void gd_dct_plan_destroy(gd_dct_plan plan);

/* Tone mapping around the Neumann solve (hdr.py:73-185), all FP64 row-major;
 * `scratch` is gd_tm_scratch_bytes() of device memory owned by the caller.
 *   gd_tm_log_luminance: lum = max(radiance . (0.2126, 0.7152, 0.0722), tiny),
 *     logl = log(lum); radiance is (h, w, 3) interleaved          (hdr.py:168-170)
 *   gd_tm_downsample: binomial blur + every other sample, out ceil(h/2) x ceil(w/2)
 *                                                                   (hdr.py:73-80)
 *   gd_tm_level_factor: the attenuation factor of one pyramid level (spacing
 *     2^level), times the bilinear upsampling of the coarser level's factor
 *     (coarse = NULL on the coarsest level)                     (hdr.py:83-134)
 *   gd_tm_compose: out = clip(image / percentile(image, q), 0, 1) with
 *     image = (radiance / lum)^saturation * exp(c - max c); `image` is an
 *     (h, w, 3) buffer of the caller                            (hdr.py:178-185) */
size_t gd_tm_scratch_bytes(void);
int gd_tm_log_luminance(double *logl_dev, double *lum_dev, const double *radiance_dev,
                        int32_t h, int32_t w, cudaStream_t stream);
int gd_tm_downsample(double *out_dev, const double *in_dev, int32_t h, int32_t w,
                     cudaStream_t stream);
int gd_tm_level_factor(double *factor_dev, const double *level_dev, const double *coarse_dev,
                       int32_t h, int32_t w, int32_t coarse_h, int32_t coarse_w, double spacing,
                       double alpha, double beta, double epsilon, void *scratch_dev,
                       cudaStream_t stream);
int gd_tm_compose(double *out_dev, double *image_dev, const double *radiance_dev,
                  const double *lum_dev, const double *compressed_dev, int32_t h, int32_t w,
                  double saturation, double percentile, void *scratch_dev, cudaStream_t stream);

/* Kernel kinds reported by gd_plan_kernel_times. */
enum gd_kernel_kind {
  GD_K_DOWN0 = 0,   /* level-0 pre-smooth + residual + restriction      */
  GD_K_DOWN = 1,    /* same on levels >= 1                              */
  GD_K_BOTTOM = 2,  /* small levels of every instance, one CTA each      */
  GD_K_UP = 3,      /* prolongation + correction + post-smooth, levels >= 1 */
  GD_K_UP0 = 4,     /* same on level 0, with the r.z reduction           */
  GD_K_PUPDATE = 5, /* p = z + beta p and p.Ap                           */
  GD_K_CGUPDATE = 6,/* d += alpha p, r -= alpha A p and r.r              */
  GD_K_FOLD = 7,    /* x += d on FP64 refresh iterations                 */
  GD_K_RESID = 8,   /* FP64 residual refresh and convergence test        */
  GD_K_INIT = 9,    /* right-hand-side mean and initial FP64 residual    */
  GD_K_MEAN = 10,   /* zero-mean projection of Neumann solutions         */
  GD_K_COARSE = 11, /* the persistent launch of the coarse levels and bottom */
  GD_KERNEL_KINDS = 12
};

typedef struct gd_kernel_time {
  long long launches;  /* launches since profiling was enabled              */
  double milliseconds; /* summed CUDA-event durations on the solve stream    */
  double cells;        /* summed grid cells covered by those launches        */
} gd_kernel_time;

/* Record CUDA events around every launch of subsequent solves (graphs are
 * bypassed while enabled); resets the totals. */
int gd_plan_set_profiling(gd_plan plan, int32_t enable);

/* Per-kind totals since gd_plan_set_profiling; out has GD_KERNEL_KINDS entries. */
int gd_plan_kernel_times(gd_plan plan, gd_kernel_time *out, int32_t n);

/* The same totals split by multigrid level: out[kind * GD_PROFILE_LEVELS + level]
 * (n >= GD_KERNEL_KINDS * GD_PROFILE_LEVELS).  Level-wise kinds (down, up, their
 * level-0 forms) use the level they run on, the bottom uses the deepest level
 * above it, and the Krylov, refresh, init, mean and persistent kinds level 0. */
#define GD_PROFILE_LEVELS 32
int gd_plan_level_times(gd_plan plan, gd_kernel_time *out, int32_t n);

/* Self-test of the bounded waits (no counterpart in the reference).  The
 * streaming kernels wait for their bulk copies on mbarriers with a limit; a
 * wait that gives up sets bit 0 of an error word (a solve then fails with
 * GD_ERR_CUDA) instead of hanging the GPU.  This launches one warp that arms an
 * mbarrier for 16 bytes no copy will deliver and waits with `tries` attempts
 * (1 .. 1<<22): afterwards *err (device int32) has bit 0 set and *completed
 * (device int32) is 0, and the context stays usable.  Nothing is allocated. */
int gd_selftest_bounded_wait(int32_t tries, int32_t *err, int32_t *completed, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Reference-exact vertex-centred FP64 multigrid (multigrid.py:147-215), used by
 * v_cycle, multigrid.solve and solve_system("multigrid" | "cg" | "mgcg_fp64").
 * Arrays are m x n FP64, contiguous (pitch = n).
 * -------------------------------------------------------------------------*/

/* Scratch bytes needed by gd_ref_vcycle for an m x n interior grid. */
size_t gd_ref_workspace_bytes(int32_t m, int32_t n, int32_t coarsest_size);

/* u <- v_cycle(u, b, spacing, options) (multigrid.py:184-215). */
int gd_ref_vcycle(double *u_dev, const double *b_dev, int32_t m, int32_t n, double spacing,
                  int32_t pre, int32_t post, int32_t coarsest_size, int32_t coarsest_sweeps,
                  void *workspace_dev, size_t bytes, cudaStream_t stream);

/* Size of the file-scope device scratch array used by gd_ref_vcycle_static. */
#define GD_STATIC_SCRATCH_BYTES (4u << 20)

/* Allocation-free u <- v_cycle(u, b, spacing, options).  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory when
 * they need a cycle (inside CUDA stream capture, in allocation-free real-time
 * loops, or as a plug-in of an application that owns the memory budget).  The
 * coarse-level scratch is a GD_STATIC_SCRATCH_BYTES (4 MiB) static device
 * array that every GPU loading this library holds until exit; grids needing
 * more (gd_ref_workspace_bytes > 4 MiB, about 500 x 500 and up) are rejected
 * with GD_ERR_ARG (a grid whose hierarchy is a single level, the coarsest solve
 * in place, uses no scratch and is never rejected).  The first call on a device
 * that needs the scratch looks up the array's address (cudaGetSymbolAddress)
 * and keeps it for the life of the process, so make that call before any
 * stream capture; after cudaDeviceReset on that device the kept address is
 * stale and the entry point must not be called again.  All calls
 * share the array: calls that overlap on the GPU (different streams or
 * threads) race and must be serialised by the caller.  Nothing is allocated
 * or freed; the coarse iterates are zeroed on every call. */
int gd_ref_vcycle_static(double *u_dev, const double *b_dev, int32_t m, int32_t n,
                         double spacing, int32_t pre, int32_t post, int32_t coarsest_size,
                         int32_t coarsest_sweeps, cudaStream_t stream);

/* out <- sweeps (1-4) red-black Gauss-Seidel sweeps of multigrid._smooth
 * (multigrid.py:147-165) on laplacian(u) = b with zeros outside the array:
 * cells with (i + j) % 2 == 0 first, each u = 0.25 * (((up + down) + left) +
 * right - spacing^2 b).  One temporally blocked pass: u and b are read once
 * and out written once, whatever the number of sweeps.  fp64 = 1: double
 * arrays, bitwise the reference's result; fp64 = 0: float arrays, bitwise the
 * same expression evaluated in float32.  All three arrays are ny x nx with row
 * pitch `pitch` elements; out must not overlap u or b (u and b may be the same
 * array).  More sweeps: call again with u and out exchanged. */
int gd_rbgs_smooth(const void *u_dev, void *out_dev, const void *b_dev, int32_t ny, int32_t nx,
                   int32_t pitch, int32_t fp64, double spacing, int32_t sweeps,
                   cudaStream_t stream);

/* r <- b - laplacian(u, spacing) (multigrid.py:210, operators.py:86-107). */
int gd_ref_residual(double *r_dev, const double *u_dev, const double *b_dev, int32_t m,
                    int32_t n, double spacing, cudaStream_t stream);

/* out[0] <- sum(a*b) over m*n elements, deterministic (solvers.py:146,151,157). */
int gd_ref_dot(double *out_dev, const double *a_dev, const double *b_dev, int64_t count,
               void *workspace_dev, size_t bytes, cudaStream_t stream);

/* y <- alpha * x + beta * y over count elements (solvers.py:152-158). */
int gd_ref_axpby(double *y_dev, const double *x_dev, double alpha, double beta,
                 int64_t count, cudaStream_t stream);

/* rc ((m-1)/2 x (n-1)/2) <- _restrict(r) = 0.25 Rows^T r Cols, full weighting
 * (multigrid.py:169-174); r is m x n contiguous, m, n >= 3. */
int gd_ref_restrict(double *rc_dev, const double *r_dev, int32_t m, int32_t n,
                    cudaStream_t stream);

/* u (m x n) += _prolong(e, (m, n)) = Rows e Cols^T, bilinear with zeros outside
 * the coarse grid (multigrid.py:177-181, _prolongation_1d :111-133); e is
 * mc x nc contiguous. */
int gd_ref_prolong_add(double *u_dev, const double *e_dev, int32_t m, int32_t n, int32_t mc,
                       int32_t nc, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Right-hand-side assembly (operators.py:53-83, :139-169; poisson.py:210-224).
 * -------------------------------------------------------------------------*/

/* (gx, gy) <- gradient(u) (operators.py:30-50); all arrays h x w contiguous FP64. */
int gd_gradient(double *gx_dev, double *gy_dev, const double *u_dev, int32_t h, int32_t w,
                cudaStream_t stream);

/* div_dev (h x w) <- divergence(gx, gy); all arrays contiguous FP64. */
int gd_divergence(double *div_dev, const double *gx_dev, const double *gy_dev, int32_t h,
                  int32_t w, cudaStream_t stream);

/* f_dev ((h-2) x (w-2)) <- scale * fold_boundary(div[1:-1,1:-1], boundary, 1)
 * (solve_dirichlet's per-channel system, poisson.py:131-143). */
int gd_fold_dirichlet(double *f_dev, const double *div_dev, const double *boundary_dev,
                      int32_t h, int32_t w, double scale, cudaStream_t stream);

/* out_dev <- fold_boundary(rhs, boundary, spacing) (operators.py:139-169) for any
 * spacing and channel count: rhs and out are (h-2, w-2, channels), boundary is
 * (h, w, channels), contiguous with channels interleaved (channels = 1 for 2-D
 * arrays).  Each cell next to the ring subtracts (1 / spacing^2) * ring value,
 * first row, last row, first column, last column in that order, as the
 * reference does.  out may be rhs (in place). */
int gd_fold_boundary(double *out_dev, const double *rhs_dev, const double *boundary_dev,
                     int32_t h, int32_t w, int32_t channels, double spacing,
                     cudaStream_t stream);

/* Guidance fields of the editing entry points, built on the device from the
 * images themselves (poisson.py:52-92 and the field set-up of seamless_clone,
 * texture_flatten, illumination_change, poisson.py:306-431). */
enum gd_field_kind {
  GD_FIELD_IMPORT = 0,       /* source gradient inside `select`, target outside     */
  GD_FIELD_MIXED = 1,        /* inside: the larger of source / target per component */
  GD_FIELD_AVERAGE = 2,      /* inside: the mean of source and target gradients     */
  GD_FIELD_WEIGHTED = 3,     /* target gradient times per-pixel `weights`           */
  GD_FIELD_ILLUMINATION = 4  /* target gradient times alpha^beta max(|g|,eps)^-beta */
};

typedef struct gd_field_desc {
  int32_t kind;                 /* enum gd_field_kind */
  int32_t height, width;        /* image size */
  int32_t channels, channel;    /* interleaved (height, width, channels) images; channel used */
  int32_t edges;                /* non-zero: the window's outer ring follows operators.py's
                                   edge rules (for a window that is the whole image) */
  const double *target;         /* the image whose gradient is the base field */
  const double *source;         /* cloning: source placed on a target-sized canvas */
  const uint8_t *select;        /* cloning: height x width, non-zero where the source field applies */
  const double *weights;        /* weighted: height x width */
  double alpha_pow_beta, beta, epsilon;  /* illumination parameters (alpha^beta precomputed) */
} gd_field_desc;

/* div (h x w, row pitch w) = divergence of the field over the interior cells
 * of the window whose corner is image cell (row0, col0); the window's outer
 * ring is written 0, or with `edges` follows the edge rules of
 * operators.divergence (tone mapping integrates the whole image).  Replaces GuidanceField construction + operators.divergence
 * as seamless_clone / texture_flatten / illumination_change use them; feed the
 * result to gd_masked_rhs or gd_fold_dirichlet. */
int gd_guidance_divergence(double *div_dev, const gd_field_desc *field, int32_t row0,
                           int32_t col0, int32_t h, int32_t w, cudaStream_t stream);

/* Masked system on the whole h x w image: f <- scale * (div - sum of known
 * neighbour values) at unknowns, 0 elsewhere (poisson.py:216-224). */
int gd_masked_rhs(double *f_dev, const double *div_dev, const double *image_dev,
                  const uint8_t *unknown_dev, int32_t h, int32_t w, double scale,
                  cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* GD_POISSON_H */
