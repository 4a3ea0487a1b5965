/*
 * sdot_gpu.h -- C ABI of the B200-native power-diagram library (libsdot_b200.so).
 *
 * Drop-in for the power-diagram hot path of sdot (Laguerre cells of weighted
 * Diracs clipped to a domain; cell integrals, centroids and the weight
 * Hessian; Newton on the weights).  Plain pointers and sizes only.
 *
 * Conventions
 *  - Positions are AoS `double[n * dim]` (x0, y0[, z0], x1, ...), the layout
 *    of the reference's Point2/Point3 arrays (src/sdot/Geometry/Point2.h:13-30).
 *  - Indices are int64 (the reference's TI = std::size_t).
 *  - `mem_space` says where a caller buffer lives: SDOT_HOST or SDOT_DEVICE
 *    (a device pointer of the current CUDA device).
 *  - Every call returns an sdot_status; sdot_last_error() gives the text.
 *    No call aborts the process or traps the GPU.
 *  - One context per stream; contexts are independent and may be used from
 *    different threads.  A context is not re-entrant.
 */
#ifndef SDOT_GPU_H
#define SDOT_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sdot_ctx sdot_ctx;

typedef enum sdot_status {
    SDOT_OK = 0,
    SDOT_VOID_CELL = 1,       /* reference: for_each_laguerre_cell(stop_if_void) returns 1 */
    SDOT_CAPACITY = 2,        /* a cell has more than 1024 vertices (2D) */
    SDOT_NOT_CONVERGED = 3,   /* Newton / PCG did not reach the tolerance */
    SDOT_ITER_CAP = 4,        /* an iteration cap was reached */
    SDOT_OOM = 5,
    SDOT_BAD_ARG = 6,
    SDOT_CUDA_ERROR = 7,
    SDOT_UNSUPPORTED = 8,
    SDOT_PENDING = 9          /* a served request is still queued or running */
} sdot_status;

enum { SDOT_HOST = 0, SDOT_DEVICE = 1 };
enum { SDOT_FP64 = 0, SDOT_MIXED = 1 };

typedef struct sdot_options {
    int64_t max_diracs_per_cell; /* SpZGrid( max_diracs_per_cell = 11 ), SpZGrid.h:37; 0 -> 11 */
    void *stream;                /* cudaStream_t to run on; NULL -> the context creates its own */
    int device;                  /* CUDA device ordinal; -1 -> current device */
} sdot_options;

/* ---- context ------------------------------------------------------------
 * Replaces the pair (SpZGrid<Pc> grid, ConvexPolyhedronAssembly<Pc> bounds)
 * that every reference entry point takes (SpZGrid.h:16-53,
 * ConvexPolyhedronAssembly.h:12-51), with Pc::dim = dim and Pc::TF = double.
 * precision: SDOT_FP64 (all arithmetic in double) or SDOT_MIXED (FP32
 * clipping, FP64 re-clip and accumulation).                                  */
sdot_ctx *sdot_create(int dim, int precision, const sdot_options *opt);
void sdot_destroy(sdot_ctx *ctx);
const char *sdot_last_error(const sdot_ctx *ctx);
/* Moves the context's device work to `stream` (a cudaStream_t created on the
 * context's device; NULL: a stream of the context's own).  Work already queued
 * on the previous stream is waited for first.  No reference counterpart: the
 * serving loop uses it to run its largest requests on a high-priority stream. */
int sdot_set_stream(sdot_ctx *ctx, void *stream);

/* ---- Diracs --------------------------------------------------------------
 * Replaces SpZGrid::update( positions, weights, nb_diracs, ... )
 * (SpZGrid.tcc:24-38): the Z-order tree is rebuilt on the device.            */
int sdot_set_diracs(sdot_ctx *ctx, const double *positions, const double *weights, int64_t n, int mem_space);
/* New weights, same positions: only the per-node maximum weights change
 * (SpZGrid::update with positions_have_changed = false).                     */
int sdot_set_weights(sdot_ctx *ctx, const double *weights, int mem_space);

/* ---- domain (cumulative, like PowerDiagram.add_..._shape) ---------------
 * ConvexPolyhedronAssembly::add_box            (ConvexPolyhedronAssembly.tcc:46-50)
 * ConvexPolyhedronAssembly::add_convex_polyhedron (:7-33): m (point, normal) half-planes
 * ConvexPolyhedronAssembly::add_simplex        (:36-43): dim + 1 points
 * ConvexPolyhedronAssembly::normalize          (:53-57)
 * ConvexPolyhedronAssembly::measure            (:115-120) / ScaledImage::measure (ScaledImage.tcc:36-69)
 * ScaledImage( min_pt, max_pt, data, sizes, nb_coeffs ) (ScaledImage.tcc:8-10): data is
 *   x-fastest; nb_coeffs = 1 (piecewise constant).  Replaces the domain.   */
int sdot_add_box_shape(sdot_ctx *ctx, const double *p0, const double *p1, double coeff);
int sdot_add_convex_polyhedron_shape(sdot_ctx *ctx, const double *points, const double *normals, int64_t m,
                                     double coeff);
int sdot_add_simplex_shape(sdot_ctx *ctx, const double *points, double coeff);
int sdot_set_image_density(sdot_ctx *ctx, const double *min_pt, const double *max_pt, const double *data,
                           const int64_t *sizes, int nb_coeffs);
/* Multilinear density factor (3D): the domain's density becomes
 *   coeff * (c0 + c1 x + c2 y + c3 z + c4 xy + c5 xz + c6 yz + c7 xyz)
 * in absolute coordinates (nb_coeffs = 8; nb_coeffs = 1 restores a constant
 * factor).  No reference counterpart: the reference's 3D densities are
 * piecewise constant (ScaledImage with nb_coeffs = 1, Polynomial.h:53-58);
 * this one integrates exactly the smooth density 1 + 0.3 xyz of the 3D
 * benchmark workload.  Cleared by sdot_clear_domain; counted by
 * sdot_domain_measure and sdot_normalize_domain.  2D: SDOT_UNSUPPORTED.     */
int sdot_set_polynomial_density(sdot_ctx *ctx, const double *coeffs, int nb_coeffs);
int sdot_clear_domain(sdot_ctx *ctx);
int sdot_normalize_domain(sdot_ctx *ctx);
int sdot_domain_measure(sdot_ctx *ctx, double *measure);

/* ---- periodicity ------------------------------------------------------------
 * SpZGrid::translations (SpZGrid.h:53, with Pc::allow_translations): count
 * translation vectors (x, y pairs; 2D, at most 64).  Each cell is also cut by
 * the images x_j + t_k of every Dirac (its own images included), as the
 * reference's traversal does (SpZGrid.tcc:558-561, :608-611); the image of
 * Dirac j under translation k has the cut id j + (k + 1) n in the neighbour
 * lists, and its Hessian entry goes to column j, the distance taken to the
 * image (get_der_integrals_wrt_weights.h:61-62).  count = 0 removes them.
 * The mixed-precision context runs its periodic cells in FP64.             */
int sdot_set_translations(sdot_ctx *ctx, const double *translations, int64_t count);

/* ---- radial function ------------------------------------------------------
 * on = 0: FunctionEnum::Unit (Unit.h:10-30); on = 1: FunctionEnum::InBallW05
 * (InBallW05.h:8-28): each cell is also clipped by the disc of radius sqrt(w_i). */
int sdot_set_ball_cut(sdot_ctx *ctx, int on);

/* ---- per-cell results -----------------------------------------------------
 * All three share one fused device evaluation (traversal + clipping +
 * integrals + centroids + Hessian rows); it is recomputed only when the
 * Diracs, weights, domain or radial function changed.
 *
 * get_integrals( res, grid, bounds, positions, weights, n, rf )   get_integrals.h:12-21
 *   out: double[n] cell masses.                                               */
int sdot_get_integrals(sdot_ctx *ctx, double *out, int mem_space);
/* get_centroids( grid, bounds, positions, weights, n, rf, cb )     get_centroids.h:13-56
 *   out_c: double[n * dim] centroids, out_m: double[n] masses (may be NULL). */
int sdot_get_centroids(sdot_ctx *ctx, double *out_c, double *out_m, int mem_space);
/* get_der_integrals_wrt_weights( offsets, columns, values, v_values, grid,
 *   bounds, positions, weights, n, rf, stop_if_void )  get_der_integrals_wrt_weights.h:15-122
 * Two-phase: call with columns == NULL to get *nnz_inout; then call with
 * buffers of offsets[n + 1], columns[nnz], values[nnz], masses[n].
 * Returns SDOT_VOID_CELL when stop_if_void and a cell is empty (the
 * buffers are still filled).                                                  */
int sdot_get_der_integrals_wrt_weights(sdot_ctx *ctx, int64_t *offsets, int64_t *columns, double *values,
                                       double *masses, int64_t *nnz_inout, int stop_if_void, int mem_space);
/* Cut ids of each final cell boundary, in vertex order (the CP2 cut_ids the
 * traversal hands to its callback, SpZGrid.tcc:643): Dirac index, -1 for a
 * domain edge, -2 for a disc arc.  Two-phase like the Hessian.               */
int sdot_get_neighbors(sdot_ctx *ctx, int64_t *offsets, int64_t *ids, int64_t *count_inout, int mem_space);

/* get_der_centroids_and_integrals_wrt_weight_and_positions( m_offsets,
 *   m_columns, m_values, v_values, grid, bounds, positions, weights, n, rf )
 *   (get_der_centroids_and_integrals_wrt_weight_and_positions.h:17-216), 2D:
 * the derivatives of (centroid x, centroid y, mass) of every cell with
 * respect to (x, y, weight) of every Dirac, as CSR over 3 n rows and columns
 * (row 3 i + d: output d of cell i; column 3 j + e: input e of Dirac j), and
 * v_values[3 n] = (centroid x, centroid y, mass).  The blocks are the
 * reference's, including its division of the centroid rows by
 * mass + (mass == 1).  Two-phase like the Hessian (columns == NULL: *nnz_inout
 * receives nnz).  Box / convex one-shape domains (periodic translations
 * allowed), without the disc clip; cells of at most 64 vertices
 * (SDOT_CAPACITY beyond).                                                    */
int sdot_get_der_centroids_and_integrals_wrt_weight_and_positions(sdot_ctx *ctx, int64_t *offsets,
                                                                   int64_t *columns, double *values,
                                                                   double *v_values, int64_t *nnz_inout,
                                                                   int mem_space);

/* ---- rasterisation ----------------------------------------------------------
 * get_image_integrals( res, grid, bounds, positions, weights, n, rf, min_pt,
 *   max_pt, nbp )  (get_image_integrals.h:16-78): for the raster of
 * nb_pixels[0] x nb_pixels[1] pixels over the box [min_pt, max_pt], out
 * (double[3 * pixels], pixel index x-fastest) receives per pixel
 * (sum_i m_i x_i, sum_i m_i y_i, sum_i m_i), m_i the integral of cell i (with
 * the domain's density, after the disc clip with InBallW05) over the pixel.
 * The per-pixel sums run in no fixed order (atomic additions): results agree
 * with the reference to rounding, not bit for bit.  2D, box / convex-shape
 * domains (SDOT_UNSUPPORTED with an image density).                          */
int sdot_get_image_integrals(sdot_ctx *ctx, const double *min_pt, const double *max_pt, const int64_t *nb_pixels,
                             double *out, int mem_space);
/* get_image_of_cell_nums( res, grid, bounds, positions, weights, n, rf,
 *   min_pt, max_pt, nbp )  (get_image_of_cell_nums.h:13-80): out (int64[pixels])
 * receives the index of a cell of non-zero integral over the pixel, -1 when
 * there is none.  Where several cells meet a pixel the reference keeps the one
 * its threads wrote last; this keeps the largest index, so that the result
 * does not depend on the order of the work.                                  */
int sdot_get_image_of_cell_nums(sdot_ctx *ctx, const double *min_pt, const double *max_pt, const int64_t *nb_pixels,
                                int64_t *out, int mem_space);

/* ---- Newton on the weights -------------------------------------------------
 * Replaces OptimalTransportSolver::solve( positions, weights, n, masses, rf )
 * (OptimalTransportSolver.tcc:27-119) and its sparse direct solve
 * EigenSolver::solve (EigenSolver.cpp:9-41).  Each iteration evaluates the
 * masses and the CSR Hessian on the device, applies the reference's gauge fix
 * (the Hessian entry (0,0) doubled when there is no ball cut, .tcc:62-63),
 * solves H dw = m - target by preconditioned conjugate gradients on the
 * device and sets w -= tau dw.  The preconditioner is a multilevel V-cycle
 * over aggregates of 8 consecutive cells in Morton order (damped Jacobi
 * smoothing, exact coarsest solve) or plain Jacobi.
 *   damping = 0: the reference rule: tau = 1; when a cell is empty the step
 *                is undone as w = 0.9 w_old + 0.1 w (.tcc:72-79).
 *   damping = 1: Kitagawa-Merigot-Thibert damping: tau halves until every
 *                cell keeps at least half of min(min target, min starting
 *                mass) and |m - target| drops by the factor (1 - tau / 2);
 *                a trial step whose cells overflow the kernels' capacity is
 *                rejected like one that fails these tests, and each search
 *                starts from min(1, 4 x the last accepted tau).
 * Stops when max_i |m_i - target_i| / target_i <= rel_mass_tol (the
 * reference stops on max |dw| < 1e-6, .tcc:111-112).  The solved weights
 * stay in the context (sdot_get_weights).                                    */
typedef struct sdot_newton_opts {
    int max_iter;          /* Newton iterations (reference: max_nb_iter = 150, .tcc:16) */
    double rel_mass_tol;   /* stopping tolerance on the relative mass error */
    int pcg_max_iter;      /* conjugate-gradient iterations per Newton step */
    double pcg_rel_tol;    /* |H dw - b| <= pcg_rel_tol |b| */
    int damping;           /* 0: reference rule, 1: KMT step halving */
    int verbosity;         /* > 0: one line per Newton iteration on stderr */
    int preconditioner;    /* 0: multilevel (default), 1: Jacobi */
    int pcg_fp32;          /* 1: each linear solve by FP32 PCG on an FP32 copy of the Hessian
                              with FP64 iterative refinement (FP64 residuals, FP64 weights;
                              steps that do not halve the residual hand over to FP64 PCG);
                              0: FP64 PCG */
} sdot_newton_opts;

typedef struct sdot_newton_report {
    int iterations;            /* Newton iterations done */
    int64_t pcg_iterations;    /* conjugate-gradient iterations, all steps */
    double max_rel_mass_error; /* at the returned weights */
    double min_mass;           /* smallest cell mass at the returned weights */
    double time_ms;            /* wall time of the solve */
    int evaluations;           /* fused cell evaluations done */
    int pcg_levels;            /* multilevel levels of the last solve (0: Jacobi) */
} sdot_newton_report;

/* target: double[n] masses (mem_space says where).  opts may be NULL for the
 * defaults {150, 1e-10, 20000, 1e-12, 1, 0, 0, 0}; report may be NULL.
 * Returns SDOT_OK, SDOT_NOT_CONVERGED (iteration or step-halving cap),
 * SDOT_VOID_CELL (damping = 1 and a cell is empty at the start weights) or
 * an evaluation error.                                                        */
int sdot_solve(sdot_ctx *ctx, const double *target, int mem_space, const sdot_newton_opts *opts,
               sdot_newton_report *report);
/* Current weights, double[n] in the caller's Dirac order. */
int sdot_get_weights(sdot_ctx *ctx, double *out, int mem_space);

/* EigenSolver::solve( x, offsets, columns, values, b ) (EigenSolver.cpp:9-41):
 * solves H x = b for the n x n CSR matrix H (offsets[n + 1], columns[nnz],
 * values[nnz], symmetric positive definite; the output of
 * sdot_get_der_integrals_wrt_weights after the gauge fix).  gauge_fix != 0
 * doubles the diagonal entry of row 0 first, as the reference does before
 * its solve (m_values[0] *= 2, OptimalTransportSolver.tcc:62-63).  Jacobi-
 * preconditioned conjugate gradients on the device from x = 0, stopping at
 * |H x - b| <= rel_tol |b| or after max_iter iterations (the reference uses a
 * sparse Cholesky factorisation).  All buffers in mem_space; work buffers
 * are allocated for the call.  iterations / rel_residual may be NULL;
 * errbuf (may be NULL) receives the message of a failure.
 * Returns SDOT_OK, SDOT_NOT_CONVERGED, SDOT_BAD_ARG, SDOT_OOM or SDOT_CUDA_ERROR. */
int sdot_csr_solve(const int64_t *offsets, const int64_t *columns, const double *values, int64_t n,
                   const double *b, double *x, int gauge_fix, double rel_tol, int max_iter, int mem_space,
                   int64_t *iterations, double *rel_residual, char *errbuf, int64_t errbuf_len);

/* Allocation-free variant of sdot_csr_solve.  No reference counterpart.
 *
 * Meant for callers that cannot allocate device memory while they solve: a
 * process whose free device memory is held by another allocator (a
 * framework's caching allocator, say) would see an allocation fail or split
 * that pool, and a latency-bound loop running one small solve per step cannot
 * afford the device-wide synchronisation that cudaMalloc and cudaFree bring
 * on every call.  The work vectors live in a fixed array compiled into the
 * library (2.65 MB of device memory on each device), hence:
 *   - n may not exceed SDOT_NOALLOC_MAX_ROWS; a larger n returns SDOT_BAD_ARG
 *     with the limit in errbuf, before anything runs;
 *   - offsets, columns, values, b and x are DEVICE pointers; stream is a
 *     cudaStream_t (NULL: the default stream); the call returns once the
 *     solve has finished on that stream;
 *   - the first call on each device looks up that device's scratch array
 *     (cudaGetSymbolAddress, with the device current), so make the first call
 *     on a device before any stream capture on that device;
 *   - that address is kept for the life of the process: resetting the device
 *     (cudaDeviceReset) between calls is not supported, since the array may
 *     then move and the kept address would be stale;
 *   - calls whose work overlaps on one device (several threads or streams)
 *     race on the shared scratch: the caller serialises them.
 * Other arguments and results as sdot_csr_solve.                            */
#define SDOT_NOALLOC_MAX_ROWS 65536
int sdot_csr_solve_noalloc(const int64_t *offsets, const int64_t *columns, const double *values, int64_t n,
                           const double *b, double *x, int gauge_fix, double rel_tol, int max_iter, void *stream,
                           int64_t *iterations, double *rel_residual, char *errbuf, int64_t errbuf_len);

/* ---- serving: continuously batched solves ---------------------------------
 * No single reference counterpart: each request is one
 * OptimalTransportSolver::solve (positions, starting weights, target masses,
 * unit-density box domain).  A server runs `slots` requests at once, each on
 * its own worker, contexts and CUDA stream (grids, weights, Hessian rows and
 * solver buffers stay resident on the device and are reused); requests are
 * admitted in arrival order as soon as a slot is free and the estimated
 * device memory of the requests in flight fits hbm_budget_bytes (a request
 * larger than the budget runs alone).  The device work of requests in flight
 * overlaps.  slots = 1 runs the same solves one after the other.            */
typedef struct sdot_server sdot_server;
typedef struct sdot_server_opts {
    int slots;                 /* requests in flight at once (1..64) */
    int64_t hbm_budget_bytes;  /* admission budget for the requests in flight */
    int device;                /* CUDA device; -1 -> current */
    sdot_newton_opts newton;   /* per-request Newton options */
} sdot_server_opts;
typedef struct sdot_request_report {
    int status;                /* SDOT_PENDING until done, then the solve's status */
    double submit_ms, start_ms, end_ms;  /* since the server was created */
    int iterations;            /* Newton iterations */
    double max_rel_mass_error;
} sdot_request_report;

sdot_server *sdot_server_create(const sdot_server_opts *opts);
/* Copies the inputs: positions double[n * dim], weights double[n] (NULL:
 * zeros), target double[n], box corners double[dim] (NULL: unit box).
 * Returns the request id (>= 0) or minus a status.                          */
int64_t sdot_server_submit(sdot_server *srv, int dim, int64_t n, const double *positions, const double *weights,
                           const double *target, const double *box_lo, const double *box_hi);
/* SDOT_PENDING while the request is queued or running; then its status, the
 * solved weights in weights_out (double[n], may be NULL) and its report.    */
int sdot_server_poll(sdot_server *srv, int64_t id, double *weights_out, sdot_request_report *report);
/* Blocks until every submitted request is done. */
int sdot_server_drain(sdot_server *srv);
/* Finishes the requests still queued, then stops the workers. */
void sdot_server_destroy(sdot_server *srv);

/* Fused evaluation only, results kept on the device (for timing). */
int sdot_evaluate(sdot_ctx *ctx);
/* Device time in milliseconds of the last evaluation stages:
 * t[0] tree build, t[1] cell kernel, t[2] Hessian assembly.                  */
int sdot_last_timings(const sdot_ctx *ctx, double *t3);
/* Number of cells rebuilt by the large-capacity fallback in the last evaluation. */
int sdot_last_overflow_count(const sdot_ctx *ctx, int64_t *count);
/* Number of kernels this library has launched in the process so far.
 * No reference counterpart (instrumentation).                               */
int sdot_kernel_launches(uint64_t *count);
/* Measured FP64 and FP32 non-tensor FMA throughput of the current device in
 * TFLOP/s (tflops2[0], tflops2[1]): the roofline denominators of the cell
 * kernels.  No reference counterpart (measurement utility).                 */
int sdot_measure_fma_peaks(double *tflops2);
/* Debug builds (-DSDOT_CHECKS) only: first failed bounds check of the cell
 * kernels (out6[0..2] = code, source line, value) and of the Hessian
 * assembly (out6[3..5]).  Release builds report zeros.                       */
int sdot_debug_checks(uint64_t *out6);

/* Counting builds (-DSDOT_COUNT) only: the work of the 2D fast tier's walks
 * since the last reset: out8[0] cut attempts, [1] vertices classified at
 * them, [2] node (eviction) tests, [3] vertices tested at them, [4] effective
 * cuts, [5] final vertices, [6] cells.  The operands of the operation count
 * of the roofline.  Release builds report zeros.  No reference counterpart. */
int sdot_debug_work_counts(uint64_t *out8, int reset);

#ifdef __cplusplus
}
#endif

#endif /* SDOT_GPU_H */
