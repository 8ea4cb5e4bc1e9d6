/*
 * svp3d.h -- C ABI of libsvp3d, the B200 (sm_100a) implementation of the certified-registration hot path of
 * seq_vp_3d (Python package jd_curl): the whole-cell Jacobian-determinant certificate, the cubic B-spline image
 * sampler, the per-cell Q1 energy/gradient/GGN kernels and the DST-I Poisson preconditioner.
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer unless its comment says "host".
 *  - Node fields are C-order (nz, ny, nx, 3) float64 with components x, y, z (x fastest in memory); cell c has
 *    coordinates x0 = c % cx, y0 = (c / cx) % cy, z0 = c / (cx cy) with (cx, cy, cz) = (nx-1, ny-1, nz-1) and vertex
 *    a = x + 2y + 4z.  Free-node vectors ("theta") are component-major (3, nz-2, ny-2, nx-2).
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are stream-ordered; a call that returns host
 *    results (marked "synchronizes") waits for its stream.
 *  - Every function returns SVP_OK (0) or an error code; svp_last_error() gives the calling thread's message.
 *    No function frees memory it did not allocate.  Handles are not shared between threads without external
 *    locking; separate handles may be used concurrently on separate streams.
 */
#ifndef SVP3D_H
#define SVP3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SVP_OK 0
#define SVP_EINVAL 1   /* invalid argument (shape, size, pointer, configuration) */
#define SVP_ECUDA 2    /* CUDA runtime error (launch, copy, device) */
#define SVP_ENOMEM 3   /* device allocation failed */
#define SVP_ENUMERIC 4 /* a numerical precondition failed (non-finite value, non-positive scale) */

/* Rectangular node grid: nx, ny, nz nodes (each >= 2), spacing and origin per axis (x, y, z).
 * Replaces jd_curl/three_d/grid.py:11 Grid3D / :49 make_grid_3d (the node axes are origin + h * arange(n)). */
typedef struct svp_grid {
    int64_t nx, ny, nz;
    double hx, hy, hz;
    double x0, y0, z0;
} svp_grid;

/* Copies the calling thread's last error message into buf (always NUL-terminated); returns its full length. */
int svp_last_error(char *buf, size_t len);
/* Library ABI version (major * 10000 + minor * 100 + patch). */
int svp_version(void);
/* Number of kernel launches this library made in the process so far (host counter).  No reference counterpart:
 * the launch accounting of the measurement harness. */
int svp_counters(int64_t *launches);
/* Opt-in CUDA-event timing of the named hot kernels on their launch streams (resets the totals).  No reference
 * counterpart (the reference times its backend methods with device syncs, backends/hybrid.py:23 timed). */
int svp_timers_enable(int on);
/* Launch count and summed device time (ms) of one named kernel since svp_timers_enable; synchronizes its events. */
int svp_timer_read(const char *name, int64_t *count, double *total_ms);

/* ============================================================================================ certificate
 * Status codes: 0 certified_feasible, 1 infeasible, 2 uncertain.  Reason codes (index into this list):
 *  0 positive_enclosure_cover  1 positive_bernstein_cover  2 JACOBIAN_VIOLATION  3 arithmetic_uncertain
 *  4 subdivision_budget  5 NONFINITE_STATE  6 NONZERO_BOUNDARY  7 INVALID_DOMAIN  8 unsupported_arithmetic
 *  9 sample_witness  10 subdivision_witness  11 box_budget  12 depth_budget
 * Arithmetic: binary64 round-to-nearest with one outward ulp step (bit steps) after every interval operation, no
 * FMA contraction, IEEE division -- the reference's exact operation sequence, so margins, verdicts and records are
 * bit-identical to jd_curl's CPU certifier. */
/* Execution flags of svp_cert_config.execution, one per member of the reference's config family
 * (feasibility.py:22-121):
 *   0                                          EnclosureCertificateConfig and its compiled/parallel/prescreen
 *                                              subclasses: edge-hull preproof, lowest-bound-first subdivision
 *   SVP_CERT_NO_HULL                           AdaptiveCertificateConfig: every cell to the interval fallback,
 *                                              lowest-bound-first subdivision
 *   SVP_CERT_NO_HULL | SVP_CERT_DEPTH_FIRST    CertificateConfig (the bare class): every cell to the fallback,
 *                                              depth-first subdivision (feasibility.py:353, left child first) */
#define SVP_CERT_NO_HULL 1
#define SVP_CERT_DEPTH_FIRST 2
/* SVP_CERT_DIRECTED (combinable with the above): the mixed form's arithmetic.  Every interval operation of the edge
 * hull, the interval fallback and the Bernstein subdivision rounds its lower end toward -inf and its upper end toward
 * +inf (__dadd_rd / __dmul_ru ...), one rounding per end, instead of round-to-nearest plus one outward ulp.  Each
 * end lies inside the reference's, so every enclosure is valid and at least as tight: cells the reference proves stay
 * proven, witnesses are true violations in both, and only cells the reference leaves undecided can change (to a
 * decision).  The prescreen keeps its a-priori bound on nearest rounding; min_jd_lower_bound = lowest + delta is
 * stepped one ulp down as in the plain form.  No counterpart in the reference (whose intervals step after rounding to
 * nearest, interval.py:52-54). */
#define SVP_CERT_DIRECTED 4
typedef struct svp_cert_config {
    double delta;       /* J > delta is proven; 0 <= delta < 1 */
    int64_t max_depth;  /* subdivision depth budget */
    int64_t max_boxes;  /* boxes per cell budget */
    int64_t tile_size;  /* cells per tile (edge-hull flag rule, arithmetic-failure rule) */
    int32_t prescreen;  /* 1: float Bernstein prescreen between hull and interval fallback (PrescreenCertificateConfig);
                           requires the edge-hull execution */
    int32_t execution;  /* SVP_CERT_* flags above (0 = edge-hull execution) */
} svp_cert_config;

/* Mirrors feasibility.py:148-179 FeasibilityResult / PrescreenFeasibilityResult (state_hash and ids excluded). */
typedef struct svp_cert_result {
    int32_t status, reason;
    int64_t n_cells_checked, n_uncertain, n_infeasible, n_boxes, max_depth, witness_cell; /* witness_cell -1: none */
    int64_t n_fast_cells, n_fallback_cells, n_prescreen_cells;
    int32_t has_min_jd, has_sampled_min;
    double min_jd_lower_bound, min_margin_lower_bound, sampled_min_jd; /* NaN when absent */
    double witness_point[3];                                           /* reference coordinates in [0,1]^3 or NaN */
} svp_cert_result;

/* One cell's subdivision verdict, mirrors feasibility.py:136 CellCertificate (status, reason, boxes, depth,
 * min_margin_lower_bound, witness_reference_point). */
typedef struct svp_cell_verdict {
    int32_t status, reason, has_margin, has_witness;
    int64_t boxes, depth;
    double margin, witness[3];
} svp_cell_verdict;

/* Per-cell lo(J - delta) of the edge-hull enclosure and an invalid-step flag (1 = some operation non-finite or
 * inverted).  Replaces compiled_enclosure.py:303 parallel_margins and backends/edge_hull_gpu.py:317
 * GpuEdgeHull.margins.  margin: (ncell,) float64, flag: (ncell,) uint8. */
int svp_edge_hull_margins(const svp_grid *g, const double *u, double delta, double *margin, uint8_t *flag,
                          void *stream);
/* The same margins in the directed-rounding arithmetic (SVP_CERT_DIRECTED): margin >= svp_edge_hull_margins' margin
 * wherever neither is flagged. */
int svp_edge_hull_margins_directed(const svp_grid *g, const double *u, double delta, double *margin, uint8_t *flag,
                                   void *stream);

/* Rigorous float Bernstein lower bounds of J over the listed cells (NaN where not finite).
 * Replaces certificate_prescreen.py:125 prescreen_lower_bounds.  cells: (n,) int64 cell ids; out: (n,) float64. */
int svp_prescreen_lower_bounds(const svp_grid *g, const double *u, const int64_t *cells, int64_t n, double *out,
                               void *stream);

/* Interval J - delta at the closed27 points, its interval Bernstein coefficients and float64 samples of standalone
 * cells.  Replaces compiled_fallback.py:177 fallback_arrays (per cell: ok[i] = 0 where the reference returns None).
 * vertices: (n, 8, 3) displacements; spacing3: host (3,) hx, hy, hz; the five outputs are (n, 27) float64 in
 * storage order 9 iz + 3 iy + ix; ok: (n,) uint8. */
int svp_fallback_arrays(const double *vertices, int64_t n, const double *spacing3, double delta, double *p_lo,
                        double *p_hi, double *c_lo, double *c_hi, double *samples, uint8_t *ok, void *stream);
/* svp_fallback_arrays in the directed-rounding arithmetic (SVP_CERT_DIRECTED); the float64 samples are unchanged. */
int svp_fallback_arrays_directed(const double *vertices, int64_t n, const double *spacing3, double delta,
                                 double *p_lo, double *p_hi, double *c_lo, double *c_hi, double *samples, uint8_t *ok,
                                 void *stream);

/* Lowest-bound-first Bernstein subdivision of n cells (one warp per cell, heap in a stream-ordered scratch
 * allocation).  Replaces feasibility.py:295 _classify.  Inputs (n, 27) from svp_fallback_arrays; out: (n,). */
int svp_classify_cells(const double *c_lo, const double *c_hi, const double *p_lo, const double *p_hi, int64_t n,
                       double delta, int64_t max_depth, int64_t max_boxes, svp_cell_verdict *out, void *stream);

/* svp_classify_cells with the subdivision order chosen as the reference's _classify chooses it from the config class
 * (feasibility.py:309-312, :351-357): SVP_SUBDIVIDE_LOWEST_FIRST (AdaptiveCertificateConfig and subclasses; the
 * order of svp_classify_cells) or SVP_SUBDIVIDE_DEPTH_FIRST (the bare CertificateConfig: pending boxes as a stack,
 * the left child first). */
#define SVP_SUBDIVIDE_LOWEST_FIRST 0
#define SVP_SUBDIVIDE_DEPTH_FIRST 1
#define SVP_SUBDIVIDE_DIRECTED 2      /* or-ed in: Bernstein splits in the directed-rounding arithmetic */
int svp_classify_cells_policy(const double *c_lo, const double *c_hi, const double *p_lo, const double *p_hi,
                              int64_t n, double delta, int64_t max_depth, int64_t max_boxes, int32_t policy,
                              svp_cell_verdict *out, void *stream);

/* svp_classify_cells without any device allocation.  No counterpart in the reference (whose subdivision runs in
 * Python on the host): it is for callers that cannot allocate device memory once they are running -- a host whose
 * device memory is owned by another allocator (a framework's caching pool, a fixed budget set at start-up) or a
 * latency-critical loop where an allocation's implicit synchronisation or pool growth is not acceptable.  The box
 * heaps live in one file-scope device array of 4,317,184 bytes (32 cells in flight x 257 heap slots), which every
 * device that loads the library keeps until process exit.  Limit: max_boxes <= 255 (larger is rejected with
 * SVP_EINVAL); n is unbounded (cells are processed 32 at a time).  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress), so make that first call before any stream capture; the address is cached per
 * device together with the id of the context it belongs to, and looked up again when that context was replaced
 * (e.g. after cudaDeviceReset).  All calls share the array:
 * calls that overlap on the GPU (concurrent streams) race and must be serialised by the caller.  Results equal
 * svp_classify_cells' bit for bit. */
int svp_classify_cells_noalloc(const double *c_lo, const double *c_hi, const double *p_lo, const double *p_hi,
                               int64_t n, double delta, int64_t max_depth, int64_t max_boxes, svp_cell_verdict *out,
                               void *stream);

/* Whole-map certificate with owned workspace.  svp_certify_map replaces feasibility.py:393 certify_map and :558
 * certify_map_owned (PrescreenCertificateConfig execution) and synchronizes; out is a host struct. */
typedef struct svp_certifier svp_certifier;
int svp_certifier_create(const svp_grid *g, const svp_cert_config *cfg, svp_certifier **out);
int svp_certifier_destroy(svp_certifier *c);
int svp_certify_map(svp_certifier *c, const double *u, svp_cert_result *out, void *stream);

/* ============================================================================================ registration pair
 * One frozen subproblem's device constants: grid, fixed image, not-a-knot cubic spline of the moving image, the
 * reference displacement u_ref of the proximal controls, the weights and the localized barrier.
 * Replaces jd_curl/three_d/problem.py:284 Problem3D / :333 make_problem / :381 with_controls on the device side
 * (backends/accelerated.py:363 AcceleratedHybridBackend owns the same constants). */
typedef struct svp_weights {
    double lam, mu, nu, kappa; /* problem.py:190 Weights3D */
    double activation;         /* localized barrier activation a (0.05 in the reference's default route) */
    double delta;              /* certificate delta (barrier domain J > delta) */
} svp_weights;

typedef struct svp_pair svp_pair;

/* fixed, moving: (nz, ny, nx) float64; u_ref: (nz, ny, nx, 3).  The spline coefficients are computed on the device
 * (interpolation.py:29 build_image_sampler: per-axis not-a-knot collocation, z then y then x). */
int svp_pair_create(const svp_grid *g, const svp_weights *w, const double *fixed, const double *moving,
                    const double *u_ref, svp_pair **out, void *stream);
/* New proximal reference (problem.py:381 with_controls / :397 make_self_reference), copied from u_ref. */
int svp_pair_set_reference(svp_pair *p, const double *u_ref, void *stream);
int svp_pair_destroy(svp_pair *p);
/* Replace the pair's spline coefficients (nz, ny, nx) by coeff (device): for a host that already holds the moving
 * image's not-a-knot coefficients on the pair's own knots (the reference's ImageSampler3D, interpolation.py:29-40,
 * whose NdBSpline keeps the coefficients and not the image). */
int svp_pair_set_spline_coefficients(svp_pair *p, const double *coeff, void *stream);
/* Copy of the spline coefficients (nz, ny, nx) into out (device). */
int svp_pair_spline_coefficients(const svp_pair *p, double *out, void *stream);

/* Arithmetic of the search direction.  SVP_PRECISION_PLAIN (the default): everything in float64, the reference's
 * binary64 results within 1e-12.  SVP_PRECISION_MIXED: svp_gradient, svp_outer_gradients, svp_ggn_diagonal and
 * svp_poisson_apply compute in float32 (edge differences, grad u, cofactors, fluxes, the folded DST-I passes), with
 * the localized barrier evaluated in float64 wherever the float32 J comes within 1e-3 of the activation, and their
 * sums and outputs in float64; energies, stable differences, the certificate, the node JD measure and the JD root
 * stay float64, so every acceptance decision is taken on float64 values (the north star's mixed form). */
#define SVP_PRECISION_PLAIN 0
#define SVP_PRECISION_MIXED 1
int svp_pair_set_precision(svp_pair *p, int32_t precision);

/* Moving image at X + u (and its physical xyz gradient when image_grad != NULL) at every node.
 * Replaces interpolation.py:72 sample_points / :109 sample_value_gradient and backends/spline.py:81 TorchSpline.
 * warped: (nz, ny, nx); image_grad: (nz, ny, nx, 3).  The caller certifies the sampling domain first. */
int svp_warp(const svp_pair *p, const double *u, double *warped, double *image_grad, void *stream);
/* Arbitrary points (n, 3) xyz inside the closed box: value (n,), gradient (n, 3) or NULL. */
int svp_sample_points(const svp_pair *p, const double *points, int64_t n, double *value, double *gradient,
                      void *stream);

/* Energy terms (image, proximity, jd, curl, barrier) of u with its warped image, summed in double-double.
 * Replaces residuals.py:189 _energy and backends/accelerated.py:1574 _energy.  terms5: host; barrier_violations:
 * host count of closed27 points with J <= delta (the reference raises there).  Synchronizes. */
int svp_energy(svp_pair *p, const double *u, const double *warped, double *terms5, int64_t *barrier_violations,
               void *stream);
/* Stable differences trial - base of E and of F = image + barrier, cancellation-free per residual and per
 * barrier point (energy_comparison.py:92 _differences; backends/accelerated.py:3062 _compare).  diff2 host. */
int svp_energy_difference(svp_pair *p, const double *base_u, const double *base_warped, const double *trial_u,
                          const double *trial_warped, double *diff2, void *stream);

/* A line-search trial against its base in one node pass and one cell pass (one synchronisation): warps
 * trial_u into trial_warped (and trial_image_grad when not NULL, the gradient promotion needs), and returns the
 * trial's terms5 and barrier_violations exactly as svp_energy and diff2 = trial - base exactly as
 * svp_energy_difference (bitwise: same sums in the same order).  Replaces the evaluate_trial -> _energy ->
 * stable_energy_reductions sequence of the reference's line search (solvers/poisson_gradient.py:1245-1290;
 * backends/accelerated.py:1667 evaluate_trial, :3062 _compare).  The caller certifies trial_u first. */
int svp_trial_energy(svp_pair *p, const double *base_u, const double *base_warped, const double *trial_u,
                     double *trial_warped, double *trial_image_grad, double *terms5, double *diff2,
                     int64_t *barrier_violations, void *stream);

/* The same two evaluations with per-cell barrier activity masks (uint8, one per cell: 1 where some closed27 J of
 * the cell is below the barrier activation).  trial_active (optional) receives the trial's mask;
 * svp_energy_difference_masked, given both states' masks, skips the closed27 sweep of cells inactive in both
 * fields.  The results are bitwise those of svp_trial_energy / svp_energy_difference (the skipped points contribute
 * nothing). */
int svp_trial_energy_masked(svp_pair *p, const double *base_u, const double *base_warped, const double *trial_u,
                            double *trial_warped, double *trial_image_grad, uint8_t *trial_active, double *terms5,
                            double *diff2, int64_t *barrier_violations, void *stream);
int svp_energy_difference_masked(svp_pair *p, const double *base_u, const double *base_warped, const double *trial_u,
                                 const double *trial_warped, const uint8_t *base_active, const uint8_t *trial_active,
                                 double *diff2, void *stream);
/* svp_trial_energy_masked given also the base's mask (base_active: the mask its own evaluation returned, or NULL):
 * the base's closed27 sweep then runs only in cells where some point of the base or of the trial is below the
 * activation, the only cells whose barrier difference is not zero.  Values bitwise those of
 * svp_trial_energy_masked. */
int svp_trial_energy_active(svp_pair *p, const double *base_u, const double *base_warped, const double *trial_u,
                            double *trial_warped, double *trial_image_grad, const uint8_t *base_active,
                            uint8_t *trial_active, double *terms5, double *diff2, int64_t *barrier_violations,
                            void *stream);

/* svp_trial_energy_active with the JD and curl penalties of the trial and of its differences evaluated in float32
 * (the mixed form's float32 energy screen; the reference screens trial energies in float32 in its default execution,
 * backends/accelerated.py:66-77).  The node terms (image, proximity), the barrier violations and the activity mask
 * are those of svp_trial_energy_active bit for bit, the localized barrier and its difference equal within rounding
 * (a cell with some float32 closed27 J within 1e-3 of the activation takes the float64 closed27 sweep); terms5[2..3]
 * and the JD/curl parts of
 * diff2[0] carry float32 rounding.  band (host) receives an estimate of that error's magnitude: the residuals'
 * absolute float32 errors (a Gauss-point J: 256 units of 2^-24, a curl component: 32) times the summed residual
 * magnitudes, plus 64 units of relative rounding of both states' squared-residual sums.  The caller resolves a
 * decision that falls within the band with svp_energy_difference_masked (float64) and checks the band against float64
 * evaluations at run time.  diff2[1] (F = image + barrier) is exact as in the float64 call. */
int svp_trial_energy_screened(svp_pair *p, const double *base_u, const double *base_warped, const double *trial_u,
                              double *trial_warped, double *trial_image_grad, const uint8_t *base_active,
                              uint8_t *trial_active, double *terms5, double *diff2, double *band,
                              int64_t *barrier_violations, void *stream);
/* The same screen for two evaluated states (energy_comparison.py:135 stable_energy_reductions, as the outer commit
 * compares its start and candidate): diff2 as svp_energy_difference_masked with the JD and curl penalty differences
 * in float32 and the band of diff2[0]; diff2[1] (F) is exact. */
int svp_energy_difference_screened(svp_pair *p, const double *base_u, const double *base_warped,
                                   const double *trial_u, const double *trial_warped, const uint8_t *base_active,
                                   double *diff2, double *band, void *stream);

/* Gradient terms mask (linearization.py:180 energy_gradient term selection). */
#define SVP_TERM_IMAGE 1
#define SVP_TERM_PROXIMITY 2
#define SVP_TERM_JD 4
#define SVP_TERM_CURL 8
#define SVP_TERM_BARRIER 16
#define SVP_TERM_TOTAL 31
#define SVP_TERM_OUTER 17
/* out: free-node vector (3 (nz-2)(ny-2)(nx-2)), component-major. */
int svp_gradient(svp_pair *p, const double *u, const double *warped, const double *image_grad, int32_t terms,
                 double *out, void *stream);
/* gF (image + barrier), gD (image), gE (total) in one cell pass (linearization.py:217 outer_gradient_vectors). */
int svp_outer_gradients(svp_pair *p, const double *u, const double *warped, const double *image_grad, double *gF,
                        double *gD, double *gE, void *stream);
/* Exact diagonal of the frozen barrier GGN (linearization.py:357) and its action on a free vector p (:327). */
int svp_ggn_diagonal(svp_pair *p, const double *u, const double *image_grad, double *out, void *stream);
/* svp_gradient, svp_outer_gradients and svp_ggn_diagonal with the state's barrier activity mask (the mask
 * svp_trial_energy_masked returned for this u, or NULL): cells inactive in it skip the closed27 barrier sweep, which
 * contributes nothing there; the values are bitwise those of the unmasked calls. */
int svp_gradient_masked(svp_pair *p, const double *u, const double *warped, const double *image_grad, int32_t terms,
                        const uint8_t *active, double *out, void *stream);
int svp_outer_gradients_masked(svp_pair *p, const double *u, const double *warped, const double *image_grad,
                               const uint8_t *active, double *gF, double *gD, double *gE, void *stream);
int svp_ggn_diagonal_masked(svp_pair *p, const double *u, const double *image_grad, const uint8_t *active,
                            double *out, void *stream);
int svp_ggn_hvp(svp_pair *p, const double *u, const double *image_grad, const double *pvec, double *out,
                void *stream);

/* Node JD measure J_a = min over the cells containing node a of (closed27 values and edge-quadratic minima)
 * (solvers/jd_affine.py:205 node_min_jd without the face/interior extension).  node: (nz, ny, nx). */
int svp_node_min_jd(svp_pair *p, const double *u, double *node, void *stream);
/* The same measure with the T69/T73 face/interior extension (solvers/jd_affine.py:205 node_min_jd with
 * extension_activation; :173 extend_minima): cells whose closed27 Bernstein coefficients allow a value below
 * min(m_c, extension_activation) take m_c = min(m_c, mu_c), mu_c the minimum over the 9^3 grid and a bounded Newton
 * descent from its 4 lowest points (a value the cell's J attains: a metric estimate, never a bound).
 * extension_activation 0 gives svp_node_min_jd exactly.  candidates (host, optional; synchronizes) receives the
 * number of candidate cells. */
int svp_node_min_jd_extended(svp_pair *p, const double *u, double extension_activation, double *node,
                             int64_t *candidates, void *stream);
/* First root tau in (0, limit] of det(I + grad u + tau grad p) - delta over all closed27 points
 * (solvers/global_jd_step.py:107 global_root_cpu; backends/torch_ops.py:636 global_jd_root).  root: host, +inf when
 * no root; invalid: host count of points with det(I + grad u) - delta <= 0.  Synchronizes. */
int svp_jd_root(svp_pair *p, const double *u, const double *pvec, double limit, double *root, int64_t *invalid,
                void *stream);

/* ============================================================================================ DST-I Poisson metric
 * out = sign * s * M^-1 (s * rhs), M^-1 = DST . diag(1 / (omega (a + b lambda))) . DST per component (poisson.py:99
 * PoissonInverse3D.apply; solvers/poisson_gradient.py:287 EquilibratedInverse; backends/hybrid.py:262
 * apply_equilibrated).  metric: 0 = q1 spectrum, 1 = seven-point.  scale: free vector or NULL (s = 1);
 * sign: +1 or -1 (the PG direction is -P^-1 g).  The per-axis DST-I is a dense GEMM with the orthonormal sine
 * matrix; rhs and out may alias. */
int svp_poisson_apply(svp_pair *p, double a, double b, int32_t metric, const double *scale, const double *rhs,
                      double sign, double *out, void *stream);

/* ============================================================================================ vector kernels
 * Deterministic (fixed-order double-double) reductions and elementwise steps of the PG solver. */
/* out (host) = sum a_i b_i. */
int svp_dot(const double *a, const double *b, int64_t n, double *out, void *stream);
/* y = x + tau p (free vectors). */
int svp_axpy(const double *x, double tau, const double *pvec, int64_t n, double *y, void *stream);
/* u (nz, ny, nx, 3) <- inject(theta) with exact zero faces (boundary.py:8 inject_free). */
int svp_inject(const svp_grid *g, const double *theta, double *u, void *stream);
/* theta <- restrict(field) (boundary.py:15 restrict_free). */
int svp_restrict(const svp_grid *g, const double *field, double *theta, void *stream);
/* Largest tau keeping every free node of X + u + tau p in the closed box: min of the quotients
 * (solvers/poisson_gradient.py:993 sampling_step_bound; fast_checks.py:85 _step_bound_xu).  bound: host. */
int svp_step_bound(const svp_grid *g, const double *u, const double *pvec, double *bound, void *stream);

/* BB2 secant products of the PG step (solvers/poisson_gradient.py:785 _step_proposal_fast): with s = theta -
 * theta_old, y = g - g_old, iy = p_old - p, out4 (host) = (s.y, s.s, y.y, y.iy). */
int svp_bb2_dots(const double *theta, const double *theta_old, const double *g, const double *g_old,
                 const double *p_old, const double *pvec, int64_t n, double *out4, void *stream);
/* out2 (host) = (max |a - b|, max |b|), NaN-propagating (fast_checks.py:120 _max_abs_diff, :111 _max_abs):
 * the inputs of the relative step max|candidate - theta| / max(L, max|theta|) (solvers/common.py:70 step_ratio). */
int svp_max_abs_diff(const double *a, const double *b, int64_t n, double *out2, void *stream);

/* Deferred forms of svp_dot, svp_bb2_dots, svp_max_abs_diff and svp_step_bound: the same values written to device
 * memory (out_dev: 1, 4, 2 and 1 doubles), stream-ordered and without synchronisation, so that a caller gathers the
 * scalars of a whole step with one copy. */
int svp_dot_dev(const double *a, const double *b, int64_t n, double *out_dev, void *stream);
int svp_bb2_dots_dev(const double *theta, const double *theta_old, const double *g, const double *g_old,
                     const double *p_old, const double *pvec, int64_t n, double *out4_dev, void *stream);
int svp_max_abs_diff_dev(const double *a, const double *b, int64_t n, double *out2_dev, void *stream);
int svp_step_bound_dev(const svp_grid *g, const double *u, const double *pvec, double *bound_dev, void *stream);
/* The scalars of one PG step in one pass over the free vectors: out_dev[0] = g.g, out_dev[1] = g.pvec and, when the
 * previous step is given (theta, theta_old, g_old, p_old all non-NULL), out_dev[2..5] = the BB2 products of
 * svp_bb2_dots_dev (poisson_gradient.py:785 _step_proposal_fast).  Each value is bitwise the one svp_dot_dev /
 * svp_bb2_dots_dev returns. */
int svp_step_dots_dev(const double *g, const double *pvec, const double *theta, const double *theta_old,
                      const double *g_old, const double *p_old, int64_t n, double *out_dev, void *stream);
/* One line-search trial point in one pass: candidate = fl(theta + fl(tau pvec)) exactly as svp_axpy, u = inject
 * (candidate) exactly as svp_inject, and out2_dev (device) = (max |candidate - theta|, max |theta|) exactly as
 * svp_max_abs_diff_dev(candidate, theta) (poisson_gradient.py:1245 trial theta; fast_checks.py:120 step ratio). */
int svp_trial_point(const svp_grid *g, const double *theta, double tau, const double *pvec, double *candidate,
                    double *u, double *out2_dev, void *stream);

/* Image-curvature shift alpha = factor * mean over free nodes of (q/omega) |grad I(X+u)|^2 / 3
 * (solvers/poisson_gradient.py:269 image_curvature_shift).  alpha: host. */
int svp_image_shift(svp_pair *p, const double *image_grad, double factor, double *alpha, void *stream);
/* Equilibrated, JD-affine damped PG scale S~ = sqrt(m) / sqrt(d) * r with r = min(1, max(J_a, floor) / activation)
 * on the free nodes (solvers/poisson_gradient.py:473-533; solvers/jd_affine.py:228 affine_factors).
 * diag: GGN diagonal (free vector), node_jd: (nz, ny, nx); scale: free vector out.  bad (host): number of entries
 * where d <= 0 or the scale is not finite and positive (the reference raises there).  Synchronizes. */
int svp_pg_scale(svp_pair *p, const double *diag, const double *node_jd, double m, double activation, double floor_,
                 double *scale, int64_t *bad, void *stream);

/* ---------------------------------------------------------------- float32 pyramid pre-optimizer (uncertified) */
/* Pre-objective weights and Adam settings of one level (preopt.py:32 PreoptConfig, the level's mu and alpha). */
typedef struct svp_pre_params {
    double mu, alpha, kappa, j0;      /* geometry weight, curvature weight, positivity-floor weight and floor */
    double lr, cap;                   /* Adam step (voxels) and the largest node move per iteration (voxels) */
    double sigma_grad, sigma_field;   /* Gaussian smoothing of the gradient / of the field after a step (0: off) */
    double beta1, beta2, eps;
} svp_pre_params;
/* Pre-objective terms (data, geometry, floor, curvature, min cell-centre det, total; terms6 host) and its gradient
 * with respect to the interior displacement u_int (3, D-2, H-2, W-2), voxel units, float32 (preopt.py:157
 * _pre_energy_tensors and its autograd gradient; preopt_grad.py:358 TritonPreGrad).  fixed, moving: (D, H, W). */
int svp_pre_energy_grad(const float *fixed, const float *moving, int32_t D, int32_t H, int32_t W, double hx, double hy,
                        double hz, const float *u_int, double mu, double alpha, double kappa, double j0, float *grad,
                        float *terms6, void *stream);
/* `iterations` Adam iterations of one level on the device (preopt.py:217 _run_level_default): u_int, m, v updated in
 * place; the Adam step counter starts at first_iteration + 1.  terms_first / terms_last (host, 6 each, optional):
 * the terms at the first and the last iteration; cap_hits (host, optional): iterations whose step was capped. */
int svp_pre_level(const float *fixed, const float *moving, int32_t D, int32_t H, int32_t W, double hx, double hy,
                  double hz, const svp_pre_params *params, int32_t first_iteration, int32_t iterations, float *u_int,
                  float *m, float *v, float *terms_first, float *terms_last, int64_t *cap_hits, void *stream);
/* Pyramid image (nifti.py:128 downsample_array): Gaussian sigma = .5 sqrt(ratio^2 - 1) per axis (mode nearest,
 * truncate 4) then linear resampling at linspace(0, n - 1, m) per axis.  src (nz, ny, nx), dst (mz, my, mx). */
int svp_image_downsample(const double *src, int32_t nz, int32_t ny, int32_t nx, double *dst, int32_t mz, int32_t my,
                         int32_t mx, void *stream);
/* Q1 transfer of a displacement (nz, ny, nx, 3) between pyramid grids (multiresolution.py:55 prolong_displacement):
 * separable linear interpolation z, then y, then x with the per-axis (left index, weight) tables the host derives
 * from the two grids' axes (left_zyx, weight_zyx: tz + ty + tx entries, host).  Synchronizes. */
int svp_field_prolong(const double *u, int32_t sz, int32_t sy, int32_t sx, double *out, int32_t tz, int32_t ty,
                      int32_t tx, const int32_t *left_zyx, const double *weight_zyx, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SVP3D_H */
