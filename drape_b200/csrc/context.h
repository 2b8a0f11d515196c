// One drape on one GPU: device buffers, the Newton step operations (assembly, PCG direction, CCD bound, line
// search) and the pseudo-transient continuation driver. The host makes every decision from a few scalars read
// back per operation; all vectors stay resident in HBM.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/drape_b200.h"
#include "kernels.h"
#include "mg.h"
#include "nn.h"
#include "problem.h"

namespace drape {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const std::string& where)
      : std::runtime_error(where + ": " + cudaGetErrorString(c)), code(c) {}
};

void check(cudaError_t e, const char* where);

template <class T> struct DeviceArray {
  T* ptr = nullptr;
  size_t n = 0;
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  ~DeviceArray() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
  }
  void alloc(size_t count);
  void upload(const T* host, size_t count, cudaStream_t s);
  void download(T* host, size_t count, cudaStream_t s) const;
};

struct PcgResult {
  int iterations = 0, status = 0, replacements = 0;
  double relative = 0.0;  // recursive sqrt(rr / rr0)
  float ms = 0.0f;
};

struct AttemptResult {
  int updates = 0, pcg_iterations = 0, mu_retries = 0, halvings = 0;
  int status = 0;  // 0 converged, 1 iteration limit, 2 line search failed, 3 regularisation cap
  bool non_finite = false;
  double max_mu = 0.0;
};

// The preconditioner network's parameters on one device: f32 master weights, their transposed bf16 copies (the
// tensor-core operands) and Adam moments. Contexts on that device use it for preconditioner 2 and train it.
struct Network {
  int device = 0;
  DeviceArray<float> master, adam_m, adam_v;
  DeviceArray<unsigned short> bf16;
  int adam_t = 0;
  Network(int device, uint64_t seed);
  NnWeights view();
  void set(const float* params);
  void get(float* params);
};

class Context {
 public:
  Context(const HostProblem& problem, const drape_options& options, int device);
  ~Context();

  const HostProblem& problem() const { return host_; }
  const drape_options& options() const { return opt_; }
  drape_options& options() { return opt_; }

  // ---- state
  void set_positions(const double* xyz);           // host -> current state x
  void get_positions(double* xyz) const;           // current state -> host
  double final_h() const { return final_h_; }

  // ---- kernel-level operations on host buffers (parity entry points)
  // g = grad Phi at x with x_hat and step h (mode 0) or grad E_s (mode 1); optional f32 blocks (9B row-major).
  double assemble_host(const double* x, const double* x_hat, double h, double mu, int mode, int curvature,
                       double* grad, float* blocks);
  PcgResult pcg_host(const float* blocks, const double* rhs, double rtol, int max_iterations, double* solution);
  double energy_change_host(const double* x, const double* x_hat, double h, const double* d, double alpha, int mode);
  double max_step_host(const double* x, const double* d);
  double static_energy_host(const double* x);
  // Kernel checks in the reference's per-element layout (checks.cu): element terms at x; row terms at x, x_hat.
  void element_terms_host(const double* x, int exact, float* grad, float* hess);
  void row_terms_host(const double* x, const double* x_hat, const double* row_mass, double mu, int contact,
                      int curvature, float* grad, float* hess);

  // ---- device-resident operations
  double gravity_load() const { return gravity_load_; }
  double static_residual();                        // |grad E_s(x)| at the current state
  double static_energy();                          // E_s(x) at the current state
  int solve_equilibrium(const double* start, double h0, drape_run_log* log);
  // One backward-Euler step of size h from the current state and velocity v_in (3V, host; null: at rest); the
  // state advances, v_out (3V, host, may be null) receives the new velocity. Returns the log's status.
  int time_step(double h, const double* v_in, double tolerance, int max_iterations, double* v_out,
                drape_time_step_log* log);
  const std::vector<drape_step_record>& steps() const { return steps_; }
  const std::vector<drape_newton_record>& newton_records() const { return records_; }
  const std::vector<drape_attempt_record>& attempt_records() const { return attempts_; }
  // With `on`, every accepted PTC state of a solve is kept in f32 (3V floats per step, in step order).
  void set_keep_states(bool on) { keep_states_ = on; }
  const std::vector<float>& step_states() const { return states_; }
  // PTC probes: one logged Newton attempt of step `step` from x with step size h (records, iterates, directions,
  // line-search trials); probe_begin clears the records and the logs.
  void probe_begin();
  void probe_step(const double* x, double h, int step);
  const std::vector<float>& probe_iterates() const { return probe_iterates_; }
  const std::vector<float>& probe_directions() const { return probe_directions_; }
  const std::vector<double>& probe_trials() const { return probe_trials_; }

  // Stand-alone timed SpMV of the assembled matrix (roofline measurement): average ms per launch.
  float time_spmv(int launches, int lanes_per_row, int threads);
  // Stand-alone timed assembly at the current state (ms per launch).
  float time_assembly(int launches);
  // Multilevel timings on the last assembled matrix: [ms per stand-alone V-cycle (plain launches), ms per flexible
  // PCG iteration inside the solve graph (a fixed number of iterations), 1 if the graph links its kernels by
  // programmatic dependent launch]; out3_stream (may be null): ms per iteration launched kernel by kernel;
  // out_setup (may be null): ms of one hierarchy set-up with fresh spectral estimates and of one reusing them.
  void time_multilevel(int iterations, float* out3, float* out3_stream, float* out_setup);

  // ---- multilevel preconditioner
  // Levels of the hierarchy the grid allows (0: not a structured grid of free vertices; only block Jacobi).
  int mg_levels() const { return mg_levels_; }
  // One V-cycle z = M r for the given f32 blocks (9B row-major) and right-hand side (the preconditioner check).
  void precondition_host(const float* blocks, const double* r, double* z);
  // Level `level`'s grid columns, stencil width (width, 0 on the fine level), f64 Galerkin stencil
  // [width^2 * 9][rows] (level >= 1) and smoother [9][rows].
  int multilevel_view(int level, int* width, double* op, float* smoother);

  // ---- preconditioner network
  void attach_network(Network* net) { net_ = net; mg_stale_ = true; }
  // The preconditioner or its damping may have changed: rebuild the hierarchy's smoothers before the next use.
  void options_changed() {
    mg_stale_ = true;
    mg_setups_since_power_ = 1 << 20;
  }
  // Loss ||x - M b||_A^2 / ||x||_A^2 of one V-cycle with the network's smoother on one (blocks, b, x) tuple, its
  // parameter gradient (kNnParams, may be null) and the smoother factors f (R, may be null).
  double network_gradient_host(Network& net, const float* blocks, const double* rhs, const double* solution,
                               float* grad, float* factors);
  // Adam on the tuples: `steps` steps, each over one tuple in turn; losses[k] of step k (before its update).
  void network_train_host(Network& net, int tuples, const float* const* blocks, const double* const* rhs,
                          const double* const* solutions, int steps, double lr, double* losses);

  // ---- concurrent solves of many contexts (one host thread each)
  int device() const { return device_; }
  // With `on`, every wait for this context's stream blocks its host thread on an event (cudaEventBlockingSync)
  // instead of spinning in cudaStreamSynchronize, so that many solving threads share the host cores.
  void set_blocking_sync(bool on);

  std::string last_error;

 private:
  void upload_problem();
  void sync();
  void wait_stream() const;
  double read_scalar(int slot);
  double assemble(const double* x, double inv_h2, double mu, int mode, bool hessian);
  double reduce_partials(int n, int op, int slot);
  PcgResult pcg(double rtol, int max_iterations);
  // The Newton direction solve: the configured preconditioner, block-Jacobi PCG as its fallback.
  PcgResult direction_solve(double rtol, int max_iterations);
  PcgResult mg_pcg(double rtol, int max_iterations, bool* stalled);
  void configure_mg();
  void build_mg_graph();
  void mg_prepare();
  void upload_blocks(const float* blocks);
  double direction_slope();
  double max_step(const double* x, const double* d);
  double energy_change(const double* x, const double* d, double alpha, double inv_h2, int mode);
  AttemptResult attempt(double h, double scale);
  AttemptResult newton(double h, double scale, double tolerance, int max_updates, bool feasible_start);
  void record_phase(int phase, cudaEvent_t a, cudaEvent_t b);

  HostProblem host_;
  drape_options opt_;
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  // the hierarchy set-up's second stream: the coarsest inverse runs there beside the smoother scaling and the
  // network (fork after the last Galerkin product, join before the solve)
  cudaStream_t side_stream_ = nullptr;
  cudaEvent_t setup_fork_ = nullptr, setup_join_ = nullptr;
  // ... and the network's stream, when the set-up reuses its spectral estimates: the network needs only the fine
  // level, so it runs beside the Galerkin products (from fine_ready_ to net_done_)
  cudaStream_t net_stream_ = nullptr;
  cudaEvent_t fine_ready_ = nullptr, net_done_ = nullptr;
  cudaEvent_t sync_event_ = nullptr;  // set_blocking_sync's event (null: cudaStreamSynchronize)
  bool blocking_sync_ = false;
  DevProblem dp_{};
  double gravity_load_ = 0.0, final_h_ = 0.0;
  PcgLaunch pcg_cfg_;
  int pcg_caps_[2] = {0, 0};
  long long pcg_launches_ = 0;
  DeviceArray<long long> pcg_timing_;

 public:
  const PcgLaunch& pcg_launch() const { return pcg_cfg_; }
  long long pcg_launches() const { return pcg_launches_; }
  // CTA 0's accumulated cycles per PCG phase since the last reset (see PcgArgs::timing); reset when `clear`.
  void pcg_profile(long long* out8, bool clear) {
    pcg_timing_.download(out8, 8, stream_);
    if (clear) check_reset_timing();
    cudaStreamSynchronize(stream_);
  }
  void check_reset_timing() { cudaMemsetAsync(pcg_timing_.ptr, 0, 8 * sizeof(long long), stream_); }

 private:
  void configure_pcg();
  // check() for a kernel launcher, counting the launch.
  void kcheck(cudaError_t e, const char* where) {
    check(e, where);
    ++kernels_;
  }
  long long kernels_ = 0;

  // multilevel hierarchy (allocated when the grid allows it)
  MgDevice mg_{};
  int mg_levels_ = 0;
  bool mg_stale_ = true;
  int mg_setups_since_power_ = 1 << 20;  // the power method reruns at a new attempt and every 4th set-up
  int fallbacks_ = 0;
  // multilevel solve outcomes: converged, limit, breakdown, stalled, coarse pivot failure, then the block-Jacobi
  // fallback's converged, limit, breakdown
  long long mg_outcome_[8] = {};
  long long mg_iterations_ = 0;
  DeviceArray<double> mg_a64_;
  DeviceArray<float> mg_s_, mg_inv_, mg_partial_, mg_state_, mg_omega_;
  DeviceArray<float4> mg_a_;
  DeviceArray<float4> mg_vec_;
  DeviceArray<int> mg_error_;
  MgState* pinned_mg_ = nullptr;
  cudaGraphExec_t mg_graph_ = nullptr;
  int mg_prolongation_ = -1;  // the prolongation (0 bilinear, 1 smoothed) mg_ and mg_graph_ are built for
  int mg_graph_launches_ = 0;
  bool mg_graph_pdl_ = false;

  // preconditioner network (attached, not owned) and its per-row buffers
  Network* net_ = nullptr;
  NnBuffers nnb_{};
  DeviceArray<float> nn_feat_, nn_w_, nn_h_, nn_o_, nn_dh_, nn_dx_, nn_partial_, nn_grad_, nn_dfac_, nn_s0_, nn_zero_,
      nn_fscale_;
  DeviceArray<int> nn_transpose_;
  DeviceArray<float4> nn_vec_;
  DeviceArray<double> nn_dot_partial_, nn_scalars_;
  void ensure_nn_buffers();
  double network_pass(Network& net, bool backward);
  void upload_tuple(const float* blocks, const double* rhs, const double* solution);

  // static problem arrays
  DeviceArray<double> geom_, hinge_k_, unit_mass_, colliders_;
  DeviceArray<int> tri_, hinge_, row_vertex_, row_ptr_, col_idx_, diag_slot_, diag_pos_;
  DeviceArray<int> rt_ptr_, rt_ent_, rt_pos_, rh_ptr_, rh_ent_, rh_pos_;
  // state and work (vertex layout f64)
  DeviceArray<double> x_, xn_, xhat_, xt_, d_, towards_;
  DeviceArray<double> vel_;  // backward-Euler velocity (time_step)
  DeviceArray<double> g_, partial_, scalars_;
  // BSR f32 planes and PCG vectors (float4 rows)
  DeviceArray<float4> a0_, a1_;
  DeviceArray<float> a2_;
  DeviceArray<float4> b_, px_, pz_, pp0_, pp1_, pq_, sol_, corr_;
  DeviceArray<float4> pmw_[2], pms_[2];  // the single-reduction PCG's published M w and M s
  DeviceArray<unsigned long long> pcg_sync_;  // PcgSyncHeader + 2 * grid partial words
  double* pinned_ = nullptr;
  PcgSyncHeader* pinned_state_ = nullptr;
  cudaEvent_t ev_[8] = {};
  std::vector<drape_step_record> steps_;
  std::vector<drape_newton_record> records_;
  std::vector<drape_attempt_record> attempts_;
  bool keep_states_ = false;
  std::vector<float> states_;
  bool probe_log_ = false;
  std::vector<float> probe_iterates_, probe_directions_;
  std::vector<double> probe_trials_;
  void log_probe_iterate(drape_newton_record& rec);
  int record_step_ = 0;  // PTC step the Newton records of the running attempt belong to
  double phase_ms_[6] = {};
  int partial_grid_ = 0;
};

void check(cudaError_t e, const char* where);

}  // namespace drape
