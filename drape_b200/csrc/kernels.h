// Kernel argument blocks and launchers of the drape GPU stage (elem.cu, pcg.cu).
#pragma once
#include <cuda_runtime.h>

#include "device_problem.h"

namespace drape {

// Incident elements (triangles + hinges) one warp evaluates per BSR row; the context rejects meshes above it.
constexpr int kMaxRowEntries = 32;
// Blocks per BSR row one warp writes (one lane per block).
constexpr int kMaxRowBlocks = 32;

struct AssembleArgs {
  DevProblem p;
  const double* x;
  const double* x_hat;
  double inv_h2;    // 1/h^2 (mode 0)
  double mu;        // the diagonal carries (1 + mu) m/h^2 (mode 0)
  int mode;         // 0: grad Phi = m/h^2 (x - x_hat) + grad Pi;  1: grad E_s = grad Pi - m g (no inertia block)
  int curvature;    // 1 keeps the barrier's b' (I - n n^T)/|x - c| term (negative semidefinite)
  int exact;        // 1: exact tangent (StVK stress, 2c(grad grad^T + theta d2 theta)); 0: clamped stress + Gauss-Newton
  double* grad;     // f64 [3R]
  DevBsr bsr;       // f32 blocks; a0 == nullptr computes the gradient only
  double* partial;  // f64 [assemble_grid(R)]: per-CTA sum of |grad_row|^2 (may be null)
};

struct EnergyArgs {
  DevProblem p;
  const double* x;
  const double* x_hat;
  const double* d;
  double alpha, inv_h2;
  int mode;         // 0: Phi (inertia term), 1: E_s (gravity potential)
  double* partial;  // f64 [grid]
};

int assemble_grid(int R);
cudaError_t launch_assemble(const AssembleArgs& a, cudaStream_t s);
cudaError_t launch_energy_change(const EnergyArgs& a, int grid, cudaStream_t s);
cudaError_t launch_max_step(const DevProblem& p, const double* x, const double* d, double* partial, int grid,
                            cudaStream_t s);
cudaError_t launch_slope(const DevProblem& p, const double* g, const double* d, double* partial, int grid,
                         cudaStream_t s);
cudaError_t launch_inf_norm(const DevProblem& p, const double* d, double* partial, int grid, cudaStream_t s);
// out[slot] = sum (op 0) or min (op 1) of n partials.
cudaError_t launch_reduce(const double* partial, int n, int op, double* out, int slot, cudaStream_t s);
// x_hat = x + h v + h^2 g on the free vertices (v null: x + h^2 g), x elsewhere.
cudaError_t launch_predict(const DevProblem& p, const double* x, const double* vel, double h, double* x_hat,
                           cudaStream_t s);
// v = (x - x_prev) / h over n values.
cudaError_t launch_velocity(int n, const double* x, const double* x_prev, double h, double* v, cudaStream_t s);
cudaError_t launch_axpy(int n, const double* x, double alpha, const double* d, double* out, cudaStream_t s);
cudaError_t launch_sub(int n, const double* a, const double* b, double* out, cudaStream_t s);
cudaError_t launch_scatter_direction(const DevProblem& p, const float4* sol, double* d, cudaStream_t s);
cudaError_t launch_rhs(int R, const double* g, float4* b, cudaStream_t s);

// ---------------------------------------------------------------- PCG
enum PcgStatus { kPcgRunning = 0, kPcgConverged = 1, kPcgIterationLimit = 2, kPcgBreakdown = 3, kPcgTimeout = 4 };

// Device-resident solver result (the reference's 16-word State, state.wgsl:4-9).
struct PcgState {
  float rz, rr, rr0, pq, alpha, beta;
  int iterations, status;
  int replacements, pad;
};

struct PcgArgs {
  int R;
  const int* row_ptr;
  const int* col_idx;
  const int* diag_pos;  // absolute block index of each row's diagonal
  DevBsr A;
  const float4* b;
  float4* x;            // solution (and the published x of a residual replacement)
  float4* z;            // published z (gathered by the fused direction update)
  float4* p0;           // published p, double-buffered
  float4* p1;
  unsigned long long* slots;  // [2 parities][2 values; 5 single-reduction][grid] (generation, partial) words
  unsigned long long* bcast;  // unused (kept for the layout of PcgSyncHeader)
  int* error;           // set when a wait gave up (the kernel returned early)
  PcgState* state;
  int cap_rows, cap_blocks;   // shared-memory capacity per CTA
  float tol2;           // tolerance^2 on rr / rr0
  int max_iterations;
  int replace_every;    // residual replacement period (0 = never)
  float replace_above2; // only while rr > replace_above^2 rr0
  long long spin_limit; // clock cycles a wait lasts before giving up
  long long* timing;    // optional [8]: CTA 0's cycles in phase A, its CTA sum, barrier A, phase B, CTA sum,
                        // barrier B, iterations (null: not recorded)
  int bulk;             // stage the rows with bulk copies (set by launch_pcg when the planes are 16-byte aligned)
  // single-reduction form only: published M w and M s, double-buffered (p0 / p1 carry u)
  float4* mw[2];
  float4* ms[2];
};

// One allocation per context, cleared before every launch: the result, the error flag, the broadcast words,
// then the per-CTA partial words (2 * grid).
struct PcgSyncHeader {
  PcgState state;
  int error;
  int pad[3];
  unsigned long long bcast[2];
};

struct PcgLaunch {
  int grid = 0, threads = 1024, lanes_per_row = 8;
  bool matrix_in_smem = true;
  bool single_reduction = false;  // one grid reduction per iteration (needs PcgArgs::mw, ms; no replacement)
  size_t smem = 0;
};

// Cooperative launch of the whole PCG solve; `cfg.grid` <= co-resident CTAs (see pcg_max_grid).
cudaError_t launch_pcg(const PcgArgs& a, const PcgLaunch& cfg, cudaStream_t s);
size_t pcg_smem_bytes(int cap_rows, int cap_blocks, bool matrix_in_smem, bool single_reduction = false);
// Words of shared memory each 4-byte matrix plane (a2, column indices) takes: cap_blocks plus the up to 3 words
// before a CTA's first block that a 16-byte aligned bulk copy brings along, rounded up to 16 bytes.
__host__ __device__ inline int pcg_word_plane(int cap_blocks) { return ((cap_blocks + 3) & ~3) + 4; }
int pcg_max_grid(int threads, int lanes_per_row, size_t smem, bool matrix_in_smem, bool single_reduction = false);

// y = A p (f32 BSR times float4-per-row vector): the stand-alone SpMV of the roofline measurement.
cudaError_t launch_spmv(int R, const int* row_ptr, const int* col_idx, DevBsr A, const float4* p, float4* y,
                        int lanes_per_row, int threads, cudaStream_t s);

// r = b64 - A d in f64 (A the f32 blocks, d float4 rows), written as the f32 right-hand side of a refinement
// solve; partial gets per-CTA |r|^2 (f64).
cudaError_t launch_refine_residual(int R, const int* row_ptr, const int* col_idx, DevBsr A, const double* b64_neg_g,
                                   const float4* d, float4* r_out, double* partial, int grid, cudaStream_t s);
// d += e (float4 rows).
cudaError_t launch_add_rows(int R, float4* d, const float4* e, cudaStream_t s);

// Kernel checks (checks.cu): element terms in the reference's per-element layout and per-row inertia/barrier terms.
cudaError_t launch_element_terms(const DevProblem& p, const double* x, int exact, float* grad, float* hess,
                                 cudaStream_t s);
cudaError_t launch_row_terms(const DevProblem& p, const double* x, const double* x_hat, const double* row_mass,
                             double mu, int contact, int curvature, float* grad, float* hess, cudaStream_t s);

}  // namespace drape
