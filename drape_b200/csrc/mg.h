// Multilevel (geometric V-cycle) preconditioner over the sheet's structured grid and the flexible PCG that uses
// it. This preconditioner has no counterpart in the reference, whose only direction solver is block-Jacobi PCG
// (engine/oracle/src/pcg.rs:37-281, engine/gpu/src/solver.ts:126-191); block-Jacobi stays the fallback.
//
// Hierarchy. The fine level is the drape's BSR(3x3) matrix over an n x n vertex grid (row = vertex, vertex =
// y * n + x). Level l + 1 has (n_l - 1) / 2 + 1 columns; the prolongation P is bilinear per displacement component
// (fine vertex 2X + a takes coarse X with weight 1 if a == 0 and X, X + 1 with 1/2 if a == 1), restriction is
// P^T, and coarse operators are Galerkin products A_{l+1} = P^T A_l P, summed in f64. Every coarse operator is a
// 5 x 5 stencil of 3x3 blocks (a fine coupling reaches 2 vertices away, a hinge's opposite vertices); the
// coarsest level (n <= 5) is solved exactly through its dense inverse.
//
// Coarse stencil layouts, w the level's stencil width (5, or 7 for level 1 under the smoothed prolongation),
// h = w / 2, o = (dy + h) * w + (dx + h) the offset of column vertex J = I + (dx, dy), e = 3 * row + col within the
// block, entries outside the grid zero:
//   A64[(o * 9 + e) * rows + I]        f64 master (the next Galerkin product, the coarsest inverse)
//   A[(I * w^2 + o) * 3 + q], q < 3    f32 copy read by the cycle: one 48-byte block per (row, offset) as three
//                                      float4 (m00 m01 m02 m10 | m11 m12 m20 m21 | m22 0 0 0)
// Smoother blocks (one 3x3 per row, any level): S[e * rows + I].
//
// One V-cycle z = M r (pre-smoothing S, post-smoothing S^T, so M is symmetric when S is symmetric or the post
// step uses the transpose of the pre step):
//   level l:  z_l = S_l r_l;  r_{l+1} = P_l^T (r_l - A_l z_l);  ...;  e_L = A_L^{-1} r_L;
//             y_l = z_l + P_l e_{l+1};  e_l = y_l + S_l^T (r_l - A_l y_l).
//
// Smoothed prolongation (MgDevice::smoothed): from the fine level to level 1 the bilinear P is smoothed once,
// P_0 = (I - omega_P D^{-1} A) P with omega_P = (4/3) / lambda, lambda the power-method estimate of
// lambda_max(D^{-1} A) (the prolongation smoothing of smoothed aggregation: Vanek, Mandel and Brezina, Computing 56
// (1996) 179-196). Level 1 = P_0^T A P_0 reaches four coarse steps; the ring at four is at rounding level (~1e-12 of
// the largest entry) and level 1 keeps the 7 x 7 stencil. The cycle's fine steps become
//   r_1 = P^T (t - A Sp t), t = r - A z_0, Sp = omega_P D^{-1};    y_0 = z_0 + v - Sp A v, v = P e_1.
#pragma once
#include <cuda_runtime.h>

#include "device_problem.h"

namespace drape {

constexpr int kMgMaxLevels = 10;
constexpr int kMgStencil = 25;         // 5 x 5 coarse stencil
constexpr int kMgStencilWide = 49;     // 7 x 7: level 1 under the smoothed prolongation
constexpr float kMgProlongC = 4.0f / 3.0f;  // omega_P = kMgProlongC / lambda
constexpr int kMgCoarsestMax = 5;      // coarsen while n > 5 and n - 1 is even
constexpr int kMgCoarsestRowsMax = 25; // dense coarse inverse of at most 75 x 75 (n <= 5)

struct MgLevel {
  int n = 0, rows = 0;
  int w = 5;              // stencil width of a coarse level (5 or 7)
  // coarse levels (l >= 1)
  double* A64 = nullptr;  // [w^2 * 9][rows]
  float4* A = nullptr;    // [rows][w^2][3] f32 blocks, 48 B each (see the layout above)
  // every level
  float* S = nullptr;     // smoother [9][rows]
  float4* r = nullptr;    // level right-hand side (level 0: the PCG residual, owned by the solver)
  float4* z = nullptr;    // pre-smoothed correction
  float4* e = nullptr;    // correction after post-smoothing (level 0: the preconditioned residual)
};

// Flexible PCG state (device). Written by CTA 0 of the kernels; every CTA computes the same sums.
// status: 1 converged, 2 iteration limit, 3 breakdown (p.q <= 0: the matrix or the preconditioner is not positive
// definite), 4 stalled (|r| fell by less than 10% over stall_window iterations).
// stall_rr[w & 1] holds rr at the end of stall window w: the test at the end of window w reads slot (w - 1) & 1
// while CTA 0 writes slot w & 1, so no CTA reads a word another CTA of the same kernel writes.
struct MgState {
  float rr0, rr, zr, pq, alpha, beta, rz_old, tol2;
  int iterations, status, done, max_iterations, stall_window;
  int has_direction;  // set by the first direction kernel: the fused update-restriction has a direction to apply
  float stall_rr[2];
};

struct MgFine {
  int R, n;
  const int* row_ptr;
  const int* col_idx;
  const int* diag_pos;
  DevBsr A;
};

// The device side of one hierarchy; every pointer is owned by the context.
struct MgDevice {
  MgFine fine;
  int levels = 0;
  MgLevel lv[kMgMaxLevels];
  float* coarse_inv = nullptr;   // dense f32 inverse of the coarsest operator, [m][m], m = 3 rows
  float* omega = nullptr;        // [kMgMaxLevels] damping of each level's Jacobi smoother (set-up output)
  // flexible PCG vectors (level 0, float4 rows)
  const float4* b = nullptr;
  float4* x = nullptr;
  float4* r[2] = {};   // residual, double-buffered (current, previous)
  float4* p[2] = {};   // search direction, double-buffered
  float4* q = nullptr;
  float* partial = nullptr;  // [4][kMgPartials]: zr, z.r_prev, pq, rr per CTA
  MgState* state = nullptr;
  int* error = nullptr;      // coarse factorisation found a zero pivot
  // smoothed prolongation from the fine level (see above); null pointers: the bilinear P everywhere
  int smoothed = 0;
  float* Sp = nullptr;       // omega_P D^{-1}, [9][R]
  float4* t = nullptr;       // fine residual after pre-smoothing, r - A z_0
  float4* u = nullptr;       // Sp t
  float4* y = nullptr;       // z_0 + P_0 e_1
};

constexpr int kMgRowsPerCta = 32;  // level-0 row kernels: 8 lanes per row, 256 threads
constexpr int kMgPartials = 4096;  // capacity of each partial array (the power method's: R < 24 x 4096 rows)

// Number of levels for an n x n grid (1 if it cannot be coarsened).
int mg_level_count(int n);

// Set-up after every assembly: Galerkin products down the hierarchy, smoothers omega_l D_l^{-1} (from level 1 when
// `fine_smoother` is false: a network supplies level 0), the coarsest dense inverse. omega > 0 fixes every
// level's damping; omega == 0 takes omega_l = 2 / (1.1 lambda_l (1 + 1/30)), the degree-1 Chebyshev smoother on
// [lambda_l / 30, 1.1 lambda_l], with lambda_l = max eigenvalue of D_l^{-1} A_l from kMgPowerSteps steps of the
// power method (all levels in one launch per step). A damping above 2 / lambda_l makes the smoother diverge on
// the highest modes; the sheet drape's fine level has lambda ~ 3.4, so a fixed 0.6 is already unstable there.
// `reuse_omega` skips the power method and scales by the omega_l of the last one (systems of one PTC attempt
// change little from one Newton update to the next).
// With a `side` stream the coarsest inverse runs there, after `fork` (recorded on s behind the last Galerkin
// product), and `join` is recorded behind it: the caller makes s wait for `join` before the cycle reads the inverse,
// so that the smoother scaling and whatever the caller queues next (the network) overlap the inverse.
constexpr int kMgPowerSteps = 10;
// With `fine_ready`, a set-up that reuses the spectral estimates scales the fine smoother first and records the
// event behind it (*fine_ready_recorded = true): the fine level's smoother is final there.
cudaError_t mg_setup(const MgDevice& d, float omega, bool fine_smoother, bool reuse_omega, cudaStream_t s,
                     cudaStream_t side = nullptr, cudaEvent_t fork = nullptr, cudaEvent_t join = nullptr,
                     cudaEvent_t fine_ready = nullptr, bool* fine_ready_recorded = nullptr);

// Flexible PCG: clear the state and start from x = 0, r = b.
cudaError_t mg_pcg_init(const MgDevice& d, float tol2, int max_iterations, int stall_window, cudaStream_t s);
// The whole flexible PCG loop as one executable graph: a conditional WHILE node whose body is two iterations
// (the double buffers return to parity 0); the body's last kernel clears the condition once state->done is set
// (convergence, iteration limit, breakdown or stall), so one graph launch runs the solve to its end on the device.
// `launches_per_body` receives the kernels of one body execution. With `pdl` the body's kernels are linked by
// programmatic dependencies (each launches while its predecessor finishes).
cudaError_t mg_build_solve_graph(const MgDevice& d, cudaStream_t s, cudaGraphExec_t* exec, int* launches_per_body,
                                 bool pdl);
// `pairs` x 2 flexible PCG iterations launched one kernel at a time on the stream (programmatic dependent launch,
// no graph): the kernels a profiler sees individually; the state must come from mg_pcg_init.
cudaError_t mg_launch_iterations(const MgDevice& d, int pairs, cudaStream_t s);
// One V-cycle z = M r on level 0 alone (r in d.r[0], z in d.lv[0].e): the preconditioner check.
cudaError_t mg_apply(const MgDevice& d, cudaStream_t s);

}  // namespace drape
