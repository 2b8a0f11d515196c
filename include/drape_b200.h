/* drape_b200: the GPU stage of the quasi-static drape solve (pseudo-transient continuation, regularised inexact
 * Newton, block-Jacobi PCG, IPC contact with a CCD-bounded Armijo line search) on one NVIDIA B200.
 *
 * C ABI: plain pointers and sizes, status codes, no exceptions across the boundary. A context is used from one
 * host thread; its work is ordered on one CUDA stream. Host arrays passed in are copied; the caller keeps them.
 *
 * The reference runs this stage as a process (engine/gpu/src/node/run-e7.ts:116-138) over problem.json /
 * problem.bin written by `oracle e7-generate` (engine/oracle/src/e7_run.rs:41-50), and in-process through the
 * TypeScript functions cited beside each entry point below.
 */
#ifndef DRAPE_B200_H
#define DRAPE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct drape_ctx drape_ctx;

typedef enum {
  DRAPE_OK = 0,
  DRAPE_E_ARG = 1,      /* invalid argument or inconsistent problem arrays */
  DRAPE_E_CUDA = 2,     /* a CUDA call failed (message in drape_last_error) */
  DRAPE_E_DIVERGED = 3, /* the solve stalled (no PTC step could be taken) or produced a non-finite state */
  DRAPE_E_TIMEOUT = 4,  /* a device-side wait gave up (bounded grid barrier) or the time budget ran out */
  DRAPE_E_IO = 5,       /* problem or state file could not be read or written */
  DRAPE_E_STATE = 6     /* called in the wrong state (e.g. no context) */
} drape_status;

/* One drape, borrowed arrays in the problem.bin layout (e3_generate.rs:84-104, e5_checks.rs:80-86):
 *   start_xyz       [3V]  cold-start vertex positions (rest_positions)
 *   elem_vertices   [3T]  triangle vertex ids                       elem_geom [7T] dN_k/dX (k=0..2) and rest area
 *   hinge_vertices  [4H]  [left opposite, right opposite, edge a, edge b]   hinge_stiffness [H]
 *   row_vertex      [R]   vertex of each unknown row                row_unit_mass [R] lumped masses (kg)
 *   row_ptr [R+1], col_idx [B]  BSR(3x3) pattern over rows (sorted columns, diagonal present)
 *   collider_data   [8 * colliders]  kind (1 plane n.x = w, 2 sphere |x - c| = w), a, b, c, w, 0, 0, 0 */
typedef struct {
  int32_t columns, vertices, triangles, hinges, rows, blocks;
  const double* start_xyz;
  const uint32_t* elem_vertices;
  const double* elem_geom;
  const uint32_t* hinge_vertices;
  const double* hinge_stiffness;
  const uint32_t* row_vertex;
  const double* row_unit_mass;
  const uint32_t* row_ptr;
  const uint32_t* col_idx;
  double wale, course, coupling, shear; /* membrane law, N/m (material.rs:28-45) */
  double gravity[3];                    /* m/s^2 */
  int32_t colliders;
  const double* collider_data;
  double dhat, kappa; /* IPC barrier activation distance (m) and stiffness */
} drape_problem_view;

/* Solver rules (the problem.json "ptc", "newton", "pcg", "robust" blocks: e7_run.rs:28-33, e3_generate.rs:199-226). */
typedef struct {
  int32_t controller;          /* 0: x2 below the inner cap, x0.5 at it (e7_ptc.rs:30-35); 1: x2 after every step */
  double h0, h_max, h_min_factor, growth, shrink;
  double inner_tolerance;      /* inner Newton stop: |g| / |g(x_n)| <= this */
  int32_t inner_max, max_rejections, max_steps;
  double equilibrium_relative; /* stop at |grad E_s| / |m g| <= this (0: off) */
  double equilibrium_absolute; /* stop at |grad E_s| <= this, N (0: off) */
  double pcg_rtol;             /* PCG relative tolerance (forcing 0) */
  int32_t pcg_max_iterations;
  int32_t forcing;             /* 0: fixed pcg_rtol; 1: Eisenstat-Walker (e4_rules.rs:15-22) */
  int32_t replace_every;       /* PCG residual replacement period (0: never) */
  double replace_above;
  int32_t refine;              /* 1: one f64 residual refinement of every Newton direction: r = -g - A d in f64
                                  and a correction solve on it */
  double refine_rtol;          /* the correction solve stops once |r| <= eta |g| (the direction's forcing target)
                                  or r has fallen by this factor, whichever comes first; no solve when the target
                                  already holds */
  int32_t curvature;           /* 1: keep the barrier's b'(I - nn^T)/|x - c| Hessian term (not SPD) */
  int32_t preconditioner;      /* 0: block Jacobi (the reference's); 1: multilevel V-cycle over the structured grid with
                                  omega-Jacobi smoothing, in flexible PCG; 2: the same V-cycle with the fine-level
                                  smoother predicted by the preconditioner network (drape_load_network). 1 and 2 need
                                  every vertex free (rows = vertices) on an n x n grid with n - 1 even; block-Jacobi
                                  PCG takes over whenever their residual stops falling (drape_run_log.fallbacks) */
  double armijo;
  int32_t max_halvings;
  double time_budget_s;        /* 0: none */
  int32_t pcg_grid, pcg_threads, pcg_lanes; /* 0: automatic */
  int32_t progress;            /* 1: one stderr line per accepted PTC step */
  int32_t newton_start;        /* inner Newton start: 0 the current state x_k (feasible; grad Phi(x_k) = grad E_s);
                                  1 the reference's prediction x_k + h^2 g cut back by the CCD bound
                                  (drape-e4.ts:55-62, e7_ptc.rs:129-133) */
  int32_t tangent;             /* 0: exact tangent (drape.rs:15-21 TangentKind::Exact) with Levenberg-Marquardt mu;
                                  1: projected (clamped membrane stress, Gauss-Newton hinge): SPD up to the barrier */
  double smoother_omega;       /* multilevel: damping of the Jacobi smoothers; 0 (default): per level
                                  2 / (1.1 lambda (1 + 1/30)) from the power method on D^{-1} A (stable) */
  int32_t prolongation;        /* multilevel fine-to-coarse prolongation: 0 (default) bilinear; 1 bilinear smoothed
                                  once, (I - (4/3) lambda^{-1} D^{-1} A) P (smoothed aggregation's prolongation
                                  smoothing; level 1 becomes a 7 x 7 stencil) */
  int32_t pcg_single_reduction; /* block-Jacobi PCG iteration form: 1 (default) one grid reduction per iteration
                                    (Chronopoulos-Gear recurrences), used when replace_every == 0; 0 the
                                    reference's two-reduction iteration (pcg.rs:271-296) */
} drape_options;

/* Outcome of drape_solve_equilibrium (gpu-result.json fields, run-e7.ts:100-106). */
typedef struct {
  int32_t ptc_steps, newton_iterations, pcg_iterations, rejected_attempts, mu_retries;
  int32_t reason; /* 0 tolerance, 1 step cap, 2 stalled, 3 time budget */
  double final_residual, final_relative_residual, final_h, gravity_load, static_energy, seconds;
  double ms_assembly, ms_pcg, ms_line_search, ms_ccd, ms_other;
  int32_t pcg_launches; /* persistent PCG kernel launches (one per linear solve) */
  int32_t pcg_grid;     /* CTAs of each PCG launch */
  double device_seconds; /* CUDA events on the context's stream around the whole solve */
  int32_t kernel_launches; /* kernels the solve launched (all of this library's own) */
  int32_t fallbacks;       /* multilevel solves handed to block-Jacobi PCG (breakdown or stalled residual) */
  int32_t mg_levels;       /* levels of the multilevel hierarchy (0: block Jacobi) */
  int32_t pad;
} drape_run_log;

/* Outcome of drape_time_step (the reference's TimeStep, drape.rs:403-408, and the step's StepSolution status,
 * newton.ts:8): status 1 converged, 2 iteration limit, 3 line search failed, 5 regularisation (mu) cap, 6 non-finite
 * residual. */
typedef struct {
  int32_t iterations, status, pcg_iterations, mu_retries;
  double scale;                  /* |grad Phi(x_n)|, the residual's scale */
  double final_relative_residual; /* |grad Phi(x)| / scale at the end */
  double max_mu, seconds;
} drape_time_step_log;

/* One accepted PTC step (gpu-ptc.bin columns, run-e7.ts:96). residual is |grad E_s| at the step's start;
 * seconds is the solve's host time at the step's end (the solve synchronizes its stream there), so a solve run to
 * a tight tolerance also tells when it passed a looser one: the first step whose starting residual is below that
 * tolerance starts at the previous step's `seconds`. */
typedef struct {
  int32_t step, inner, rejected, pcg_iterations;
  double h, residual, min_distance, seconds;
} drape_step_record;

/* One Newton iterate of a solve: the reference's IterationRecord and the RobustRecord fields this solver has
 * (newton.ts:12-22, robust-newton.ts; gpu-iterations.bin and gpu-robust.bin rows, outputs.ts:8-10). The last iterate
 * of an attempt takes no solve: pcg_iterations = -1 there (the reference's NaN). status: 0 running (an update was
 * taken), 1 converged, 2 iteration limit, 3 line search failed, 5 regularisation (mu) cap (newton.ts:8), 6 non-finite
 * residual. */
typedef struct {
  int32_t step, iteration, pcg_iterations, pcg_status, halvings, status, retries, pad;
  double relative_residual, linear_residual, step_length; /* |g| / |g(x_n)|, PCG recursive residual, alpha */
  double eta, mu, alpha_max, delta_sum, slope, norm_squared; /* forcing, regularisation, CCD bound, accepted
                                                                 energy change, g.d, |g|^2 */
  double resolution; /* probe runs: f32 spacing of the iterate's largest |x| (e4_rules.rs:35-39); else NaN */
} drape_newton_record;

/* One attempt at a step size (AttemptLog, drape-e7.ts:26-32; gpu-attempts.bin rows): its Newton records are
 * [record_start, record_end) of drape_newton_records. reason (drape-e7.ts:11): 0 accepted, 1 regularisation cap,
 * 2 line search failed, 3 non-finite, 4 curvature retry (superseded by a run without the barrier's b'd2d term). */
typedef struct {
  int32_t step, attempt, reason, record_start, record_end, pad;
  double h;
} drape_attempt_record;

/* Library version string. */
const char* drape_version(void);

/* Fills the sheet-over-sphere rules: h0 = 1e-3 s doubled after each accepted step whose inner Newton stayed below
 * its cap (halved at the cap), |grad E_s| <= 1e-6 N, PCG rtol 1e-6 with at most 2000 iterations, inner Newton
 * tol 0.1 and 10 updates from the current state (replaces parsePtcRules/parseRobustRules, ptc.ts:28-32,
 * robust-newton.ts:208-214). */
void drape_default_options(drape_options* out);

/* Creates a context on `device` from borrowed arrays (replaces prepareDrapeGpu, drape-gpu.ts:141-162). */
drape_status drape_create(const drape_problem_view* problem, const drape_options* options, int32_t device,
                          drape_ctx** out);
/* Builds the problem from a problem.json / problem.bin directory (replaces load + parseDrapeProblem,
 * run-e7.ts:51-57, drape.ts:44-63). */
drape_status drape_create_from_files(const char* dir, const drape_options* options, int32_t device, drape_ctx** out);
/* Builds the 1 m sheet over a sphere (optional ground plane at y = -0.25) with the product's scene builder. */
drape_status drape_create_sheet(int32_t columns, uint64_t seed, double radius, double young, int32_t plane,
                                const drape_options* options, int32_t device, drape_ctx** out);
/* Builds the reference's 0.5 m knit sphere-on-floor scene, edit "base" | "w1" | "w2" | "w3" (e7_run.rs:18-26). */
drape_status drape_create_reference(int32_t columns, const char* edit, const drape_options* options, int32_t device,
                                    drape_ctx** out);
void drape_destroy(drape_ctx* ctx);

/* Host-only (no GPU needed): write the problem.json / problem.bin pair of the product's scene builders (replaces
 * `oracle e7-generate`, e7_run.rs:41-50, for the GPU stage's inputs), and read + validate a pair, returning
 * [V, T, H, R, B, colliders]. */
drape_status drape_write_sheet_problem(int32_t columns, uint64_t seed, double radius, double young, int32_t plane,
                                       const char* dir);
drape_status drape_write_reference_problem(int32_t columns, const char* edit, const char* dir);
drape_status drape_inspect_problem(const char* dir, int64_t* sizes6);

/* Last error message of a context, or of the last failed create when ctx is NULL. */
const char* drape_last_error(const drape_ctx* ctx);

/* [V, T, H, R, B, colliders] */
drape_status drape_sizes(const drape_ctx* ctx, int64_t* out6);
drape_status drape_set_options(drape_ctx* ctx, const drape_options* options);

/* Current state (f64 master positions, 3V) and the step size the last solve ended with (e7_state.rs:9-40). */
drape_status drape_set_state(drape_ctx* ctx, const double* xyz);
drape_status drape_get_state(const drape_ctx* ctx, double* xyz, double* final_h);

/* PTC to equilibrium from `start_xyz` (NULL: the current state) with first step `h0` (<= 0: options.h0)
 * (replaces solveEquilibrium, drape-e7.ts:156-180; oracle ptc_solve, e7_ptc.rs:170-189). */
drape_status drape_solve_equilibrium(drape_ctx* ctx, const double* start_xyz, double h0, drape_run_log* log);
/* One dynamic (backward-Euler) step of size h s from the context's state x_n with velocity v (3V m/s, NULL: at
 * rest), the reference's time_step (drape.rs:410-417; GPU: drape-e4.ts:45-52 timeStep): prediction
 * x_hat = x_n + h v + h^2 g on the free vertices, Newton on Phi(x) = (x - x_hat)^T M (x - x_hat) / (2 h^2) + E(x)
 * from the CCD-cut prediction x_n + alpha_max (x_hat - x_n), regularised like the PTC's inner Newton, until
 * |grad Phi| / |grad Phi(x_n)| <= tolerance or max_iterations updates. The context's state becomes the step's
 * result; v_out (3V, may be NULL) receives (x - x_n) / h. The Newton records of the step are then in
 * drape_newton_records (step 1). Returns DRAPE_OK whatever the Newton's status (see log). */
drape_status drape_time_step(drape_ctx* ctx, double h, const double* v, double tolerance, int32_t max_iterations,
                             double* v_out, drape_time_step_log* log);

/* Coarse-to-fine start state for the prolong mode, in place of `oracle e7-prolong` (e7_prolong.rs:7-64): the
 * (2n - 1)^2 vertices of `ctx`'s mesh from the n^2 coarse positions `coarse` (3 n^2, n = coarse_columns), each the
 * average of its four (possibly repeated) coarse corners, then every vertex closer than d_hat to one of ctx's
 * colliders moved along that collider's normal to d = d_hat (one pass, colliders in order). fine_out: 3V;
 * *moved (may be NULL): vertices moved; *infeasible (may be NULL): vertices still at or inside a collider (the
 * reference refuses such a start). DRAPE_E_ARG when the grids do not match. */
drape_status drape_prolong_state(const drape_ctx* ctx, const double* coarse, int32_t coarse_columns, double* fine_out,
                                 int32_t* moved, int32_t* infeasible);
/* Many independent drapes at once: each of `count` distinct contexts runs drape_solve_equilibrium(ctx, NULL, 0, ...)
 * from its current state, on `workers` host threads that take the next unsolved drape in turn. Every context keeps
 * its own stream, so the kernels of up to `workers` drapes share the GPU; the threads block on events rather than
 * spin while they wait for it. Contexts may share one attached network (it is only read). Per drape (each array may
 * be NULL): logs[i], statuses[i] (drape_solve_equilibrium's status) and solve_seconds[i] (host time from the start
 * of drape i's solve to its end); total_seconds (may be NULL) = host time of the whole batch. Returns DRAPE_OK when
 * every drape ended without error, else the first failing drape's status with its message in
 * drape_last_error(NULL). Streams share the GPU's hardware queues, 8 unless CUDA_DEVICE_MAX_CONNECTIONS (read when
 * CUDA starts in the process) says more: with 32, 32 workers ran 1.8x the Newton steps per second of the default.
 * No counterpart in the reference, whose run-e7.ts solves one drape per process. */
drape_status drape_solve_batch(drape_ctx* const* ctxs, int32_t count, int32_t workers, drape_run_log* logs,
                               drape_status* statuses, double* solve_seconds, double* total_seconds);
/* Copies up to `capacity` accepted-step records of the last solve; returns their total count in *count. */
drape_status drape_step_records(const drape_ctx* ctx, drape_step_record* out, int32_t capacity, int32_t* count);
/* The same for the last solve's Newton iterates (ctx.records of robust-newton.ts, gpu-iterations.bin and
 * gpu-robust.bin) and its attempts (drape-e7.ts:116,138, gpu-attempts.bin). */
drape_status drape_newton_records(const drape_ctx* ctx, drape_newton_record* out, int32_t capacity, int32_t* count);
drape_status drape_attempt_records(const drape_ctx* ctx, drape_attempt_record* out, int32_t capacity, int32_t* count);
/* keep = 1: later solves keep every accepted PTC state (f32), the reference's keepStates (drape-e7.ts:156-178, on
 * for grids of at most 65 columns, run-e7.ts:29,133). drape_step_states copies up to `capacity` floats of the last
 * solve's states (3V per accepted step, in step order; the start state is not among them) and returns their total
 * count in *count. */
drape_status drape_keep_states(drape_ctx* ctx, int32_t keep);
/* PTC probes (runPtcProbes, drape-e7.ts:190-200; run-e7.ts:146-152): drape_probe_begin clears the Newton records and
 * the probe logs; each drape_probe_step runs one Newton attempt of PTC step `step` from `xyz` (3V f64) with step size
 * h, recording its Newton iterates (drape_newton_records) and logging, per iterate, its positions (f32 3V), per
 * update the pair (positions, direction) (f32 2 x 3V) and per line-search trial the row (step, iteration, halving,
 * alpha, energy-change sum, NaN, g.d, accepted 0/1) (f64 8; TRIAL_FIELDS of outputs.ts:11). drape_probe_logs copies
 * up to the given capacities (floats / doubles, each buffer may be NULL) and returns the totals. */
drape_status drape_probe_begin(drape_ctx* ctx);
drape_status drape_probe_step(drape_ctx* ctx, const double* xyz, double h, int32_t step);
drape_status drape_probe_logs(const drape_ctx* ctx, float* iterates, int64_t iterates_capacity, int64_t* iterates_count,
                              float* directions, int64_t directions_capacity, int64_t* directions_count,
                              double* trials, int64_t trials_capacity, int64_t* trials_count);
drape_status drape_step_states(const drape_ctx* ctx, float* out, int64_t capacity, int64_t* count);

/* Kernel-level entry points on host buffers (the parity checks of run-e7.ts:140-145 --checks):
 * g = grad Phi(x) with x_hat and step h (mode 0; Phi = (1/2h^2)(x - x_hat)^T M (x - x_hat) + Pi) or
 * grad E_s (mode 1), 3R f64; blocks = K + mu M/h^2 (mode 0) as 9B f32 row-major blocks, NULL to skip
 * (replaces evaluateKernelsWithInertia, drape-e4.ts; oracle DrapeStep::residual/tangent, drape.rs:304-322). */
drape_status drape_assemble(drape_ctx* ctx, const double* x, const double* x_hat, double h, double mu, int32_t mode,
                            int32_t curvature, double* grad, float* blocks);
/* PCG from 0 on the given f32 blocks (NULL: the last assembled matrix) and f64 rhs (3R, rounded to f32), with
 * the configured preconditioner (block Jacobi unless options.preconditioner selects the multilevel one); info = [iterations, status (1 converged, 2 iteration limit, 3 breakdown, 4 timeout), replacements],
 * relative = recursive sqrt(rr/rr0) (replaces solveOnce, solver.ts:179-191; oracle pcg::solve, pcg.rs:271-291). */
drape_status drape_pcg(drape_ctx* ctx, const float* blocks, const double* rhs, double rtol, int32_t max_iterations,
                       double* solution, int32_t* info, double* relative);
/* Phi(x + alpha d) - Phi(x) (mode 0) or E_s(x + alpha d) - E_s(x) (mode 1), f64 sum of per-element changes
 * (replaces gpuEnergy, newton-ops.ts:360-365; oracle DrapeStep::energy_change, drape.rs:325-335). */
drape_status drape_energy_change(drape_ctx* ctx, const double* x, const double* x_hat, double h, const double* d,
                                 double alpha, int32_t mode, double* out);
/* Largest alpha <= 1 keeping every vertex at >= 0.1 of its collider distances (replaces maxStepOnGpu,
 * contact-host.ts:36-41; oracle DrapeStep::max_step, drape.rs:344-346). */
drape_status drape_max_step(drape_ctx* ctx, const double* x, const double* d, double* out);
/* |grad E_s| and E_s at x (NULL: the current state), f64 (oracle static_gradient / static_energy,
 * e7_ptc.rs:43-51). */
drape_status drape_static_residual(drape_ctx* ctx, const double* x, double* out);
drape_status drape_static_energy(drape_ctx* ctx, const double* x, double* out);
/* Element terms at x (3V f64) in the reference's per-element layout, f32 (each may be NULL): grad [9T + 12H] with
 * triangle e at 9e + 3k + i and hinge h at 9T + 12h + 3k + i; hess [81T + 144H] with triangle block (k, l) at
 * 81e + 9(3k + l) and hinge block (k, l) at 81T + 144h + 9(4k + l), 3x3 row-major. exact 1: StVK stress and the
 * hinge's 2c(grad grad^T + theta d2 theta); 0: positive-part stress in the geometric term and Gauss-Newton hinge
 * (replaces the exactElements / projectedElements passes of evaluateDrapeKernels, drape-step.ts:83-97;
 * membrane_element.wgsl, hinge_element.wgsl). */
drape_status drape_element_terms(drape_ctx* ctx, const double* x, int32_t exact, float* grad, float* hess);
/* Row terms at x with prediction x_hat (3V f64 each), f32 (each may be NULL): grad [3R] = m_r (x - x_hat) +
 * sum b'(d) n, hess [9R] = m_r (1 + mu) I + sum b''(d) n n^T + b'(d) kappa (I - n n^T) over the active colliders
 * when `contact` (the kappa term when `curvature`), with row_mass [R] the per-row mass over h^2 (NULL: 0)
 * (replaces the inertia pass of evaluateKernelsWithInertia, evaluateContactKernel and evaluateInertiaAtSteps,
 * drape-e4.ts:108-120, contact-host.ts:76-90, drape-e7.ts:203-218; inertia.wgsl). */
drape_status drape_row_terms(drape_ctx* ctx, const double* x, const double* x_hat, const double* row_mass, double mu,
                             int32_t contact, int32_t curvature, float* grad, float* hess);

/* The multilevel preconditioner (no counterpart in the reference): z = M r, one V-cycle for the given f32 blocks
 * (NULL: the last assembled matrix) and rhs r (3R f64, rounded to f32); z is 3R f64. */
drape_status drape_precondition(drape_ctx* ctx, const float* blocks, const double* r, double* z);
/* Level `level` of the hierarchy for the current matrix: *columns = its grid columns, *width (may be NULL) its
 * stencil width w (5, or 7 for level 1 under the smoothed prolongation; 0 for the fine level), op (level >= 1, may
 * be NULL) the f64 Galerkin stencil [w^2 * 9][rows] (offset o = (dy + w/2) * w + dx + w/2, entry e = 3 * row + col),
 * smoother (may be NULL) the f32 blocks [9][rows]. DRAPE_E_ARG when the problem has no hierarchy or level is out of
 * range. */
drape_status drape_multilevel_view(drape_ctx* ctx, int32_t level, int32_t* columns, int32_t* width, double* op,
                                   float* smoother);

/* Timed stand-alone launches for the roofline: average device ms per launch of the BSR SpMV on the last
 * assembled matrix (lanes per row 4/8/16/32) and of the row assembly at the current state. */
drape_status drape_time_spmv(drape_ctx* ctx, int32_t launches, int32_t lanes_per_row, int32_t threads, float* ms);
drape_status drape_time_assembly(drape_ctx* ctx, int32_t launches, float* ms);
/* Stand-alone BSR(3x3) SpMV y = A x on any matrix given by host arrays (row_ptr [rows+1], col_idx [blocks],
 * values [9 blocks] f32 row-major, x [3 rows]), e.g. the block-diagonal concatenation of many drapes (the batched
 * configuration, per-instance row offsets folded into col_idx): uploads, runs 3 warm-up and `launches` timed
 * launches of the lanes_per_row (4/8/16/32) x threads (<= 256) kernel shape, *ms = device ms per launch, y
 * (3 rows, may be NULL) = the result. No counterpart in the reference (its SpMV is spmv_dot.wgsl). */
drape_status drape_spmv_benchmark(int32_t device, int32_t rows, int64_t blocks, const int32_t* row_ptr,
                                  const int32_t* col_idx, const float* values, const float* x, int32_t launches,
                                  int32_t lanes_per_row, int32_t threads, float* y, float* ms);
/* Multilevel timings on the last assembled matrix and right-hand side: out6 = [ms per stand-alone V-cycle,
 * ms per flexible PCG iteration inside the solve graph (exactly `iterations` iterations), 1 if the graph's kernels
 * are linked by programmatic dependent launch, ms per iteration of the same iterations launched kernel by kernel
 * on the stream (the launches a profiler sees one by one), ms of one hierarchy set-up with fresh spectral
 * estimates, ms of one reusing them]. */
drape_status drape_time_multilevel(drape_ctx* ctx, int32_t iterations, float* out6);
/* SM-clock cycles CTA 0 of the PCG kernel spent per phase since the last clear: [phase A (p, q = A p),
 * its CTA sum, its grid reduction, phase B (x, r, z), its CTA sum, its grid reduction, iterations]; clear != 0
 * zeroes the counters. */
drape_status drape_pcg_profile(drape_ctx* ctx, int64_t* out7, int32_t clear);

/* The preconditioner network (no counterpart in the reference): a 4-layer mesh message-passing network (hidden
 * width 64, BF16 weights, FP32 accumulation) that predicts, per fine-level row, a factor f in (0.8, 1) on the
 * multilevel preconditioner's Jacobi smoother; options.preconditioner = 2 uses the network attached to the
 * context. Parameters: DRAPE_NETWORK_PARAMETERS f32 values, layout W_in[16][64] b_in[64], 4 x (W[128][64] b[64]),
 * w_out[64] b_out. The file format is "DRAPENN1", an int32 count, then the f32 values (little-endian). */
#define DRAPE_NETWORK_PARAMETERS 34177
typedef struct drape_network drape_network;
/* Glorot-uniform weights from `seed`, zero biases and a zero output layer (f = 0.9: the untrained network gives
 * a little under the multilevel preconditioner's spectral smoother). */
drape_status drape_network_create(int32_t device, uint64_t seed, drape_network** out);
void drape_network_destroy(drape_network* net);
drape_status drape_network_load(drape_network* net, const char* path);
drape_status drape_network_save(drape_network* net, const char* path);
/* get (may be NULL) receives the parameters; set (may be NULL) replaces them (and clears the Adam moments). */
drape_status drape_network_parameters(drape_network* net, float* get, const float* set);
/* Attach (NULL: detach) the network the context's preconditioner 2 uses; the context does not own it. */
drape_status drape_set_network(drape_ctx* ctx, drape_network* net);
/* Loss ||x - M b||_A^2 / ||x||_A^2 of one V-cycle M with the network's smoother on one tuple (blocks 9B f32,
 * rhs b and solution x 3R f64, A x = b), the gradient of the loss (DRAPE_NETWORK_PARAMETERS, may be NULL) and the
 * factors f (R, may be NULL). */
drape_status drape_network_gradient(drape_ctx* ctx, drape_network* net, const float* blocks, const double* rhs,
                                    const double* solution, double* loss, float* grad, float* factors);
/* Trains on `tuples` tuples of this context's pattern: `steps` Adam steps (learning rate lr), step k on tuple
 * k % tuples; losses[k] (may be NULL) is step k's loss before its update. */
drape_status drape_network_train(drape_ctx* ctx, drape_network* net, int32_t tuples, const float* const* blocks,
                                 const double* const* rhs, const double* const* solutions, int32_t steps, double lr,
                                 double* losses);

/* Block-Jacobi PCG that allocates nothing, for callers that cannot call cudaMalloc: applications whose device
 * memory all comes from their own pool, or that must not enter the driver's allocator once they are running.
 * This entry point has no counterpart in the reference; it is the persistent PCG of drape_pcg with its work space
 * (search directions, diagonal index, grid-reduction words) in one fixed device array of about 3.4 MB that the
 * library holds on every GPU that loads it, until exit. Limit: 1 to DRAPE_NOALLOC_MAX_ROWS block rows.
 * All pointers are device memory on the current device, owned by the caller:
 *   row_ptr [rows+1], col_idx [B]   BSR(3x3) pattern, every row with its diagonal block
 *   a0, a1 [4B] and a2 [B]          blocks as the assembly writes them: a0 = (m00,m01,m02,m10),
 *                                   a1 = (m11,m12,m20,m21), a2 = m22 (a0, a1 16-byte aligned)
 *   rhs, x [4 * rows]               one 16-byte row each (x, y, z, unused); x receives the solution from 0
 * info (host, may be NULL) = int32_t[3]: [iterations, status (1 converged, 2 iteration limit, 3 breakdown),
 * residual replacements]; relative (host, may be NULL) = sqrt(rr/rr0).
 * Every call looks up the array's device address in the current context (cudaGetSymbolAddress; no allocation),
 * so the address stays right after cudaDeviceReset or a context switch. The first call on a device also loads
 * the library's device code there and should come before any stream capture. Calls share the one array and run
 * on `stream` (NULL: the default stream) and return after synchronizing it; calls that overlap on the GPU (other
 * host threads, other streams) race on the array. */
#define DRAPE_NOALLOC_MAX_ROWS 65536
drape_status drape_pcg_noalloc(int32_t rows, const int32_t* row_ptr, const int32_t* col_idx, const float* a0,
                               const float* a1, const float* a2, const float* rhs, float* x, double rtol,
                               int32_t max_iterations, void* stream, int32_t* info, double* relative);

#ifdef __cplusplus
}
#endif

#endif /* DRAPE_B200_H */
