// The drape GPU stage on one device: problem upload, Newton-step operations and the PTC driver.
// Host-side rules follow the reference's GPU host loop and oracle:
//   PTC step / attempts / rejection   drape-e7.ts:97-180, e7_ptc.rs:129-189
//   regularised inexact Newton        robust-newton.ts:312-441 (mu schedule newton.rs:113-125, forcing
//                                     e4_rules.rs:15-22), Armijo from the CCD bound newton.rs:158-167
//   controller                        e7_ptc.rs:30-35 (inner-count) or x2 per accepted step (doubling)
#include "context.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>

namespace drape {

// Energy, minimum-distance kernels live in elem.cu.
cudaError_t launch_static_energy(const DevProblem& p, const double* x, double* partial, int grid, cudaStream_t s);
cudaError_t launch_min_distance(const DevProblem& p, const double* x, double* partial, int grid, cudaStream_t s);

void check(cudaError_t e, const char* where) {
  if (e != cudaSuccess) throw CudaError(e, where);
}

template <class T> void DeviceArray<T>::alloc(size_t count) {
  release();
  n = count;
  if (count) check(cudaMalloc(&ptr, count * sizeof(T)), "cudaMalloc");
}
template <class T> void DeviceArray<T>::upload(const T* host, size_t count, cudaStream_t s) {
  if (count > n) throw std::runtime_error("upload larger than the device array");
  if (count) check(cudaMemcpyAsync(ptr, host, count * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
}
template <class T> void DeviceArray<T>::download(T* host, size_t count, cudaStream_t s) const {
  if (count > n) throw std::runtime_error("download larger than the device array");
  if (count) check(cudaMemcpyAsync(host, ptr, count * sizeof(T), cudaMemcpyDeviceToHost, s), "download");
}

namespace {

constexpr int kReduceGrid = 296;
enum Slot { kNorm = 0, kSlope, kAlpha, kDelta, kEnergy, kMinDist, kRefine, kInf, kSlots = 16 };
enum Phase { kAssembly = 0, kPcg, kLineSearch, kCcd, kOther };

double raise_mu(double mu) { return std::min(std::max(10.0 * mu, 1e-3), 1e3); }
double relax_mu(double mu) { return mu / 10.0 < 1e-3 ? 0.0 : mu / 10.0; }

// Eisenstat-Walker choice 2 (e4_rules.rs:15-22).
double next_forcing(double previous, double ratio) {
  double eta = 0.9 * ratio * ratio, safeguard = 0.9 * previous * previous;
  double guarded = safeguard > 0.1 ? std::max(eta, safeguard) : eta;
  return std::min(std::max(guarded, 1e-7), 1e-2);
}

}  // namespace

// Levels of the multilevel hierarchy the problem allows: every vertex a row in vertex order on an n x n grid,
// couplings within 2 vertices per axis (coarse operators are then 5 x 5 stencils), partial sums within capacity.
int structured_levels(const HostProblem& p) {
  const int n = p.columns;
  // the power method's partial sums cover the row CTAs of every smoothed level (< R / 24 in all)
  if (n <= 0 || p.R != p.V || n * n != p.V || (p.R + 23) / 24 > kMgPartials) return 0;
  for (int r = 0; r < p.R; ++r)
    if (p.row_vertex[r] != r) return 0;
  for (int r = 0; r < p.R; ++r)
    for (int k = p.row_ptr[r]; k < p.row_ptr[r + 1]; ++k) {
      const int c = p.col_idx[k];
      if (std::abs(c % n - r % n) > 2 || std::abs(c / n - r / n) > 2) return 0;
    }
  const int levels = mg_level_count(n);
  return levels >= 2 ? levels : 0;
}

Context::Context(const HostProblem& problem, const drape_options& options, int device)
    : host_(problem), opt_(options), device_(device) {
  std::string err = validate(host_);
  if (!err.empty()) throw std::invalid_argument("inconsistent problem: " + err);
  mg_levels_ = structured_levels(host_);
  if (opt_.preconditioner != 0 && mg_levels_ == 0)
    throw std::invalid_argument("the multilevel preconditioner needs every vertex free on an n x n grid with n - 1 even");
  check(cudaSetDevice(device_), "cudaSetDevice");
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  for (auto& e : ev_) check(cudaEventCreate(&e), "cudaEventCreate");
  check(cudaStreamCreateWithFlags(&side_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaEventCreateWithFlags(&setup_fork_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&setup_join_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaStreamCreateWithFlags(&net_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaEventCreateWithFlags(&fine_ready_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&net_done_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaMallocHost(&pinned_, kSlots * sizeof(double)), "cudaMallocHost");
  check(cudaMallocHost(&pinned_state_, sizeof(PcgSyncHeader)), "cudaMallocHost");
  check(cudaMallocHost(&pinned_mg_, sizeof(MgState) + 16), "cudaMallocHost");
  upload_problem();
}

Context::~Context() {
  if (stream_) cudaStreamSynchronize(stream_);
  if (side_stream_) cudaStreamSynchronize(side_stream_);
  if (net_stream_) cudaStreamSynchronize(net_stream_);
  for (auto& e : ev_)
    if (e) cudaEventDestroy(e);
  if (setup_fork_) cudaEventDestroy(setup_fork_);
  if (setup_join_) cudaEventDestroy(setup_join_);
  if (fine_ready_) cudaEventDestroy(fine_ready_);
  if (net_done_) cudaEventDestroy(net_done_);
  if (sync_event_) cudaEventDestroy(sync_event_);
  if (pinned_) cudaFreeHost(pinned_);
  if (pinned_state_) cudaFreeHost(pinned_state_);
  if (pinned_mg_) cudaFreeHost(pinned_mg_);
  if (mg_graph_) cudaGraphExecDestroy(mg_graph_);
  if (side_stream_) cudaStreamDestroy(side_stream_);
  if (net_stream_) cudaStreamDestroy(net_stream_);
  if (stream_) cudaStreamDestroy(stream_);
}

void Context::upload_problem() {
  const HostProblem& p = host_;
  const int V = p.V, T = p.T, H = p.H, R = p.R, B = p.B;
  // Row-centric element maps: for every row, its incident triangles and hinges in element order, each with the
  // block slot (within the row) of every element vertex.
  std::vector<int> vertex_row(V, -1);
  for (int r = 0; r < R; ++r) vertex_row[p.row_vertex[r]] = r;
  auto slot_of = [&](int r, int c) -> int {
    if (c < 0) return -1;
    auto b = p.col_idx.begin() + p.row_ptr[r], e = p.col_idx.begin() + p.row_ptr[r + 1];
    auto it = std::lower_bound(b, e, c);
    if (it == e || *it != c) throw std::invalid_argument("element coupling outside the BSR pattern");
    return int(it - b);
  };
  std::vector<std::vector<int>> rt(R), rh(R);
  for (int t = 0; t < T; ++t)
    for (int k = 0; k < 3; ++k) {
      int r = vertex_row[p.tri[3 * t + k]];
      if (r >= 0) rt[r].push_back(t << 2 | k);
    }
  for (int h = 0; h < H; ++h)
    for (int k = 0; k < 4; ++k) {
      int r = vertex_row[p.hinge[4 * h + k]];
      if (r >= 0) rh[r].push_back(h << 2 | k);
    }
  std::vector<int> rt_ptr{0}, rt_ent, rt_pos, rh_ptr{0}, rh_ent, rh_pos, diag_slot(R), diag_pos(R);
  int max_entries = 0, max_blocks = 0;
  for (int r = 0; r < R; ++r) {
    for (int ent : rt[r]) {
      rt_ent.push_back(ent);
      for (int l = 0; l < 3; ++l) rt_pos.push_back(slot_of(r, vertex_row[p.tri[3 * (ent >> 2) + l]]));
    }
    for (int ent : rh[r]) {
      rh_ent.push_back(ent);
      for (int l = 0; l < 4; ++l) rh_pos.push_back(slot_of(r, vertex_row[p.hinge[4 * (ent >> 2) + l]]));
    }
    rt_ptr.push_back(int(rt_ent.size()));
    rh_ptr.push_back(int(rh_ent.size()));
    max_entries = std::max(max_entries, int(rt[r].size() + rh[r].size()));
    max_blocks = std::max(max_blocks, p.row_ptr[r + 1] - p.row_ptr[r]);
    diag_slot[r] = slot_of(r, r);
    diag_pos[r] = p.row_ptr[r] + diag_slot[r];
  }
  if (max_entries > kMaxRowEntries)
    throw std::invalid_argument("a row has " + std::to_string(max_entries) + " incident elements (limit " +
                                std::to_string(kMaxRowEntries) + ")");
  if (max_blocks > kMaxRowBlocks)
    throw std::invalid_argument("a row has " + std::to_string(max_blocks) + " blocks (limit " +
                                std::to_string(kMaxRowBlocks) + ")");

  geom_.alloc(7 * size_t(T));
  geom_.upload(p.tri_geom.data(), geom_.n, stream_);
  tri_.alloc(3 * size_t(T));
  tri_.upload(p.tri.data(), tri_.n, stream_);
  hinge_.alloc(4 * size_t(H));
  hinge_.upload(p.hinge.data(), hinge_.n, stream_);
  hinge_k_.alloc(H);
  hinge_k_.upload(p.hinge_k.data(), H, stream_);
  row_vertex_.alloc(R);
  row_vertex_.upload(p.row_vertex.data(), R, stream_);
  unit_mass_.alloc(R);
  unit_mass_.upload(p.unit_mass.data(), R, stream_);
  row_ptr_.alloc(R + 1);
  row_ptr_.upload(p.row_ptr.data(), R + 1, stream_);
  col_idx_.alloc(B);
  col_idx_.upload(p.col_idx.data(), B, stream_);
  diag_slot_.alloc(R);
  diag_slot_.upload(diag_slot.data(), R, stream_);
  diag_pos_.alloc(R);
  diag_pos_.upload(diag_pos.data(), R, stream_);
  auto up = [&](DeviceArray<int>& d, const std::vector<int>& h) {
    d.alloc(std::max<size_t>(h.size(), 1));
    d.upload(h.data(), h.size(), stream_);
  };
  up(rt_ptr_, rt_ptr);
  up(rt_ent_, rt_ent);
  up(rt_pos_, rt_pos);
  up(rh_ptr_, rh_ptr);
  up(rh_ent_, rh_ent);
  up(rh_pos_, rh_pos);
  colliders_.alloc(std::max<size_t>(p.colliders.size(), 8));
  colliders_.upload(p.colliders.data(), p.colliders.size(), stream_);

  const size_t nv = 3 * size_t(V);
  for (auto* a : {&x_, &xn_, &xhat_, &xt_, &d_, &towards_}) a->alloc(nv);
  x_.upload(p.start.data(), nv, stream_);
  g_.alloc(3 * size_t(R));
  partial_grid_ = std::max(assemble_grid(R), kReduceGrid);
  partial_.alloc(partial_grid_);
  scalars_.alloc(kSlots);
  a0_.alloc(B);
  a1_.alloc(B);
  a2_.alloc(B);
  for (auto* a : {&b_, &px_, &pz_, &pp0_, &pp1_, &pq_, &sol_, &corr_}) a->alloc(R);
  for (auto* a : {&b_, &px_, &pz_, &pp0_, &pp1_, &pq_, &sol_, &corr_})
    check(cudaMemsetAsync(a->ptr, 0, sizeof(float4) * a->n, stream_), "memset");

  dp_ = DevProblem{};
  dp_.V = V;
  dp_.T = T;
  dp_.H = H;
  dp_.R = R;
  dp_.B = B;
  dp_.ncol = p.collider_count();
  dp_.max_row_blocks = max_blocks;
  dp_.max_row_entries = max_entries;
  dp_.geom = geom_.ptr;
  dp_.tri = tri_.ptr;
  dp_.hinge = hinge_.ptr;
  dp_.hinge_k = hinge_k_.ptr;
  dp_.row_vertex = row_vertex_.ptr;
  dp_.unit_mass = unit_mass_.ptr;
  dp_.row_ptr = row_ptr_.ptr;
  dp_.col_idx = col_idx_.ptr;
  dp_.diag_slot = diag_slot_.ptr;
  dp_.rt_ptr = rt_ptr_.ptr;
  dp_.rt_ent = rt_ent_.ptr;
  dp_.rt_pos = rt_pos_.ptr;
  dp_.rh_ptr = rh_ptr_.ptr;
  dp_.rh_ent = rh_ent_.ptr;
  dp_.rh_pos = rh_pos_.ptr;
  dp_.colliders = colliders_.ptr;
  dp_.wale = p.wale;
  dp_.course = p.course;
  dp_.coupling = p.coupling;
  dp_.shear = p.shear;
  for (int k = 0; k < 3; ++k) dp_.gravity[k] = p.gravity[k];
  dp_.dhat = p.dhat;
  dp_.kappa = p.kappa;

  double gn = std::sqrt(p.gravity[0] * p.gravity[0] + p.gravity[1] * p.gravity[1] + p.gravity[2] * p.gravity[2]);
  double s = 0;
  for (double m : p.unit_mass) s += (m * gn) * (m * gn);
  gravity_load_ = std::sqrt(s);

  configure_pcg();
  configure_mg();
  sync();
}

// PCG launch shape: 1024-thread CTAs whose lane groups cover each CTA's rows in one pass where possible, at most
// one CTA per SM (fewer CTAs = fewer barrier words), and each CTA's matrix rows in shared memory when they fit.
void Context::configure_pcg() {
  const int R = host_.R;
  PcgLaunch c;
  c.lanes_per_row = opt_.pcg_lanes > 0 ? opt_.pcg_lanes : 8;
  c.threads = opt_.pcg_threads > 0 ? opt_.pcg_threads : 1024;
  if (c.threads % 32 || c.threads > 1024 || c.threads < c.lanes_per_row)
    throw std::invalid_argument("unsupported PCG thread count");
  int sms = 0;
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "attribute");
  const int groups = c.threads / c.lanes_per_row;
  int grid = opt_.pcg_grid > 0 ? opt_.pcg_grid : std::min(sms, (R + groups - 1) / groups);
  grid = std::max(1, std::min({grid, R, c.threads}));  // the master CTA polls one partial word per thread
  for (;;) {
    int cap_rows = 0, cap_blocks = 0;
    for (int b = 0; b < grid; ++b) {
      const int r0 = int((long long)R * b / grid), r1 = int((long long)R * (b + 1) / grid);
      cap_rows = std::max(cap_rows, r1 - r0);
      cap_blocks = std::max(cap_blocks, host_.row_ptr[r1] - host_.row_ptr[r0]);
    }
    // sized for the single-reduction form (three more row vectors), which the two-reduction form fits in too
    c.matrix_in_smem = pcg_smem_bytes(cap_rows, cap_blocks, true, true) <= 200 * 1024;
    c.smem = pcg_smem_bytes(cap_rows, cap_blocks, c.matrix_in_smem, true);
    const int fit = std::min(pcg_max_grid(c.threads, c.lanes_per_row, c.smem, c.matrix_in_smem, true),
                             pcg_max_grid(c.threads, c.lanes_per_row, c.smem, c.matrix_in_smem, false));
    if (fit <= 0) throw std::invalid_argument("the PCG rows of one CTA do not fit in shared memory");
    if (grid <= fit) {
      c.grid = grid;
      pcg_caps_[0] = cap_rows;
      pcg_caps_[1] = cap_blocks;
      break;
    }
    grid = fit;
  }
  pcg_cfg_ = c;
  pcg_sync_.alloc((sizeof(PcgSyncHeader) + 80 * size_t(c.grid) + 7) / 8);  // 2 parities x 5 words x grid
  pcg_timing_.alloc(8);
  check(cudaMemsetAsync(pcg_timing_.ptr, 0, 8 * sizeof(long long), stream_), "memset");
}

void Context::sync() { wait_stream(); }

void Context::wait_stream() const {
  if (!blocking_sync_) {
    check(cudaStreamSynchronize(stream_), "stream synchronize");
    return;
  }
  check(cudaEventRecord(sync_event_, stream_), "event");
  check(cudaEventSynchronize(sync_event_), "event synchronize");
}

void Context::set_blocking_sync(bool on) {
  if (on && !sync_event_) {
    check(cudaSetDevice(device_), "cudaSetDevice");
    check(cudaEventCreateWithFlags(&sync_event_, cudaEventBlockingSync | cudaEventDisableTiming), "cudaEventCreate");
  }
  blocking_sync_ = on;
}

double Context::read_scalar(int slot) {
  check(cudaMemcpyAsync(pinned_ + slot, scalars_.ptr + slot, sizeof(double), cudaMemcpyDeviceToHost, stream_), "read");
  sync();
  return pinned_[slot];
}

double Context::reduce_partials(int n, int op, int slot) {
  kcheck(launch_reduce(partial_.ptr, n, op, scalars_.ptr, slot, stream_), "reduce");
  return read_scalar(slot);
}

void Context::set_positions(const double* xyz) {
  x_.upload(xyz, 3 * size_t(host_.V), stream_);
  sync();
}

void Context::get_positions(double* xyz) const {
  x_.download(xyz, 3 * size_t(host_.V), stream_);
  wait_stream();
}

double Context::assemble(const double* x, double inv_h2, double mu, int mode, bool hessian) {
  AssembleArgs a{};
  a.p = dp_;
  a.x = x;
  a.x_hat = xhat_.ptr;
  a.inv_h2 = inv_h2;
  a.mu = mu;
  a.mode = mode;
  a.curvature = opt_.curvature;
  a.exact = opt_.tangent == 0;
  a.grad = g_.ptr;
  a.bsr = hessian ? DevBsr{a0_.ptr, a1_.ptr, a2_.ptr} : DevBsr{nullptr, nullptr, nullptr};
  a.partial = partial_.ptr;
  if (hessian) mg_stale_ = true;
  kcheck(launch_assemble(a, stream_), "assemble");
  return std::sqrt(reduce_partials(assemble_grid(host_.R), 0, kNorm));
}

PcgResult Context::pcg(double rtol, int max_iterations) {
  PcgArgs a{};
  a.R = host_.R;
  a.row_ptr = row_ptr_.ptr;
  a.col_idx = col_idx_.ptr;
  a.diag_pos = diag_pos_.ptr;
  a.A = DevBsr{a0_.ptr, a1_.ptr, a2_.ptr};
  a.b = b_.ptr;
  a.x = px_.ptr;
  a.z = pz_.ptr;
  a.p0 = pp0_.ptr;
  a.p1 = pp1_.ptr;
  auto* head = reinterpret_cast<PcgSyncHeader*>(pcg_sync_.ptr);
  a.state = &head->state;
  a.error = &head->error;
  a.bcast = head->bcast;
  a.slots = reinterpret_cast<unsigned long long*>(head + 1);
  a.cap_rows = pcg_caps_[0];
  a.cap_blocks = pcg_caps_[1];
  a.tol2 = float(rtol * rtol);
  a.max_iterations = max_iterations;
  a.replace_every = opt_.replace_every;
  a.replace_above2 = float(opt_.replace_above * opt_.replace_above);
  a.spin_limit = 4000000000LL;  // ~2 s of SM clock per wait
  a.timing = pcg_timing_.ptr;
  PcgLaunch cfg = pcg_cfg_;
  cfg.single_reduction = opt_.pcg_single_reduction != 0 && opt_.replace_every == 0;
  if (cfg.single_reduction) {
    if (pmw_[0].n < size_t(host_.R))
      for (auto* v : {&pmw_[0], &pmw_[1], &pms_[0], &pms_[1]}) v->alloc(host_.R);
    a.mw[0] = pmw_[0].ptr;
    a.mw[1] = pmw_[1].ptr;
    a.ms[0] = pms_[0].ptr;
    a.ms[1] = pms_[1].ptr;
  }
  check(cudaMemsetAsync(pcg_sync_.ptr, 0, pcg_sync_.n * sizeof(unsigned long long), stream_), "memset");
  check(cudaEventRecord(ev_[0], stream_), "event");
  kcheck(launch_pcg(a, cfg, stream_), "pcg launch");
  check(cudaEventRecord(ev_[1], stream_), "event");
  check(cudaMemcpyAsync(pinned_state_, pcg_sync_.ptr, sizeof(PcgSyncHeader), cudaMemcpyDeviceToHost, stream_), "read");
  sync();
  PcgResult r;
  cudaEventElapsedTime(&r.ms, ev_[0], ev_[1]);
  phase_ms_[kPcg] += r.ms;
  pcg_launches_++;
  const PcgState& s = pinned_state_->state;
  if (pinned_state_->error) throw CudaError(cudaErrorLaunchTimeout, "PCG grid wait gave up");
  r.iterations = s.iterations;
  r.status = s.status;
  r.replacements = s.replacements;
  r.relative = s.rr0 > 0 ? std::sqrt(double(s.rr) / double(s.rr0)) : 0.0;
  return r;
}

double Context::max_step(const double* x, const double* d) {
  kcheck(launch_max_step(dp_, x, d, partial_.ptr, kReduceGrid, stream_), "max_step");
  return reduce_partials(kReduceGrid, 1, kAlpha);
}

double Context::energy_change(const double* x, const double* d, double alpha, double inv_h2, int mode) {
  EnergyArgs a{dp_, x, xhat_.ptr, d, alpha, inv_h2, mode, partial_.ptr};
  kcheck(launch_energy_change(a, kReduceGrid, stream_), "energy_change");
  return reduce_partials(kReduceGrid, 0, kDelta);
}

double Context::static_residual() { return assemble(x_.ptr, 0.0, 0.0, 1, false); }

double Context::static_energy() {
  kcheck(launch_static_energy(dp_, x_.ptr, partial_.ptr, kReduceGrid, stream_), "static_energy");
  return reduce_partials(kReduceGrid, 0, kEnergy);
}

// One attempt at step size h from xn_ (into x_): the PTC prediction x_n + h^2 g, the feasible start, then the
// regularised inexact Newton to the inner tolerance.
AttemptResult Context::attempt(double h, double scale) {
  kcheck(launch_predict(dp_, xn_.ptr, nullptr, h, xhat_.ptr, stream_), "predict");
  return newton(h, scale, opt_.inner_tolerance, opt_.inner_max, opt_.newton_start == 1);
}

// The regularised inexact Newton on Phi(x) = 1/(2h^2)(x - x_hat)^T M (x - x_hat) + E_s(x) with x_hat in xhat_,
// from xn_ (feasible_start: from x_n + alpha_max (x_hat - x_n), the CCD-cut prediction) into x_, until
// |grad Phi| / scale <= tolerance or `max_updates` updates.
AttemptResult Context::newton(double h, double scale, double tolerance, int max_updates, bool feasible_start) {
  AttemptResult res;
  const double inv_h2 = 1.0 / (h * h);
  const size_t nv = 3 * size_t(host_.V);
  auto t_phase = [&](int phase, auto&& fn) {
    auto t0 = std::chrono::steady_clock::now();
    auto out = fn();
    phase_ms_[phase] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return out;
  };
  mg_setups_since_power_ = 1 << 20;  // a new step size: fresh spectral estimates at the first set-up
  if (feasible_start) {
    // The reference's start: x_n + alpha_max (x_hat - x_n).
    kcheck(launch_sub(int(nv), xhat_.ptr, xn_.ptr, towards_.ptr, stream_), "towards");
    double a0 = t_phase(kCcd, [&] { return max_step(xn_.ptr, towards_.ptr); });
    kcheck(launch_axpy(int(nv), xn_.ptr, a0, towards_.ptr, x_.ptr, stream_), "start");
  } else {
    check(cudaMemcpyAsync(x_.ptr, xn_.ptr, nv * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "start");
  }
  double mu = 0.0, eta = opt_.forcing ? 1e-2 : opt_.pcg_rtol, prev_norm = 0.0;
  constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();
  for (int it = 0;; ++it) {
    double norm = t_phase(kAssembly, [&] { return assemble(x_.ptr, inv_h2, mu, 0, true); });
    double rel = norm / scale;
    // this iterate's record (robust-newton.ts records): completed below as the iterate proceeds
    drape_newton_record rec{};
    rec.step = record_step_;
    rec.iteration = it;
    rec.pcg_iterations = -1;
    rec.halvings = -1;
    rec.relative_residual = rel;
    rec.norm_squared = norm * norm;
    rec.linear_residual = rec.step_length = rec.eta = rec.alpha_max = rec.delta_sum = rec.slope = kNaN;
    rec.resolution = kNaN;
    rec.mu = mu;
    auto finish = [&](int status) {
      rec.status = status;
      if (probe_log_) log_probe_iterate(rec);
      records_.push_back(rec);
    };
    if (!std::isfinite(rel)) {
      finish(6);
      res.non_finite = true;
      return res;
    }
    if (rel <= tolerance) {
      finish(1);
      res.status = 0;
      return res;
    }
    if (it == max_updates) {
      finish(2);
      res.status = 1;
      return res;
    }
    if (opt_.forcing) eta = it == 0 ? 1e-2 : next_forcing(eta, norm / prev_norm);
    prev_norm = norm;
    rec.eta = eta;
    rec.pcg_iterations = 0;
    double slope = 0.0;
    for (;;) {
      res.max_mu = std::max(res.max_mu, mu);
      kcheck(launch_rhs(host_.R, g_.ptr, b_.ptr, stream_), "rhs");
      PcgResult pr = direction_solve(eta, opt_.pcg_max_iterations);
      res.pcg_iterations += pr.iterations;
      rec.pcg_iterations += pr.iterations;
      rec.pcg_status = pr.status;
      rec.linear_residual = pr.relative;
      check(cudaMemcpyAsync(sol_.ptr, px_.ptr, sizeof(float4) * host_.R, cudaMemcpyDeviceToDevice, stream_), "copy");
      if (opt_.refine && pr.status != kPcgBreakdown) {
        kcheck(launch_refine_residual(host_.R, row_ptr_.ptr, col_idx_.ptr, DevBsr{a0_.ptr, a1_.ptr, a2_.ptr}, g_.ptr,
                                     sol_.ptr, b_.ptr, partial_.ptr, kReduceGrid, stream_),
              "refine");
        // The correction solve on the f64 residual r = -g - A d stops once the direction meets its forcing target
        // (|r| <= eta |g|) or r has fallen by refine_rtol, whichever comes first: it fixes what the f32 solve left
        // above the target, and takes no iteration when the target already holds.
        const double rn = std::sqrt(reduce_partials(kReduceGrid, 0, kRefine));
        const double target = rn > 0.0 ? eta * norm / rn : 1.0;
        const double rtol = std::max(opt_.refine_rtol, target);
        if (rtol < 1.0) {
          PcgResult pc = direction_solve(rtol, opt_.pcg_max_iterations);
          res.pcg_iterations += pc.iterations;
          rec.pcg_iterations += pc.iterations;
          if (pc.status != kPcgBreakdown) kcheck(launch_add_rows(host_.R, sol_.ptr, px_.ptr, stream_), "add");
        }
      }
      if (host_.R < host_.V)  // fixed vertices keep a zero direction
        check(cudaMemsetAsync(d_.ptr, 0, nv * sizeof(double), stream_), "memset");
      kcheck(launch_scatter_direction(dp_, sol_.ptr, d_.ptr, stream_), "scatter");
      kcheck(launch_slope(dp_, g_.ptr, d_.ptr, partial_.ptr, kReduceGrid, stream_), "slope");
      slope = reduce_partials(kReduceGrid, 0, kSlope);
      rec.slope = slope;
      bool failed = pr.status == kPcgBreakdown || !(slope < 0.0);
      if (!failed) break;
      if (mu >= 1e3) {
        finish(5);
        res.status = 3;
        return res;
      }
      mu = raise_mu(mu);
      res.mu_retries++;
      rec.retries++;
      rec.mu = mu;
      t_phase(kAssembly, [&] { return assemble(x_.ptr, inv_h2, mu, 0, true); });
    }
    double amax = t_phase(kCcd, [&] { return max_step(x_.ptr, d_.ptr); });
    rec.alpha_max = amax;
    int halvings = -1;
    double alpha = 0.0;
    t_phase(kLineSearch, [&] {
      for (int k = 0; k <= opt_.max_halvings; ++k) {
        double a = amax * std::ldexp(1.0, -k);
        double delta = energy_change(x_.ptr, d_.ptr, a, inv_h2, 0);
        if (probe_log_) {  // TRIAL_FIELDS: step, iteration, halving, alpha, sum, abs, slope, accepted
          const double row[8] = {double(record_step_), double(it), double(k), a, delta, kNaN, slope,
                                 delta <= opt_.armijo * a * slope ? 1.0 : 0.0};
          probe_trials_.insert(probe_trials_.end(), row, row + 8);
        }
        if (delta <= opt_.armijo * a * slope) {
          halvings = k;
          alpha = a;
          rec.delta_sum = delta;
          break;
        }
      }
      return 0;
    });
    if (halvings < 0) {
      finish(3);
      res.status = 2;
      return res;
    }
    rec.halvings = halvings;
    rec.step_length = alpha;
    finish(0);
    kcheck(launch_axpy(int(nv), x_.ptr, alpha, d_.ptr, x_.ptr, stream_), "advance");
    res.updates++;
    res.halvings += halvings;
    mu = halvings == 0 ? relax_mu(mu) : mu;
  }
}

// The iterate x_k in f32, its f32 spacing (2^(exponent of max |x_i| over the rows' vertices - 23), e4_rules.rs:35-39)
// and, after a direction solve, the pair (x_k, d_k) in f32.
void Context::log_probe_iterate(drape_newton_record& rec) {
  const size_t nv = 3 * size_t(host_.V);
  std::vector<double> xs(nv), ds;
  x_.download(xs.data(), nv, stream_);
  if (rec.pcg_iterations >= 0) {
    ds.resize(nv);
    d_.download(ds.data(), nv, stream_);
  }
  sync();
  double largest = 0.0;
  for (int r = 0; r < host_.R; ++r)
    for (int c = 0; c < 3; ++c) largest = std::max(largest, std::fabs(xs[3 * size_t(host_.row_vertex[r]) + c]));
  const float m = float(largest);
  uint32_t bits;
  std::memcpy(&bits, &m, sizeof bits);
  rec.resolution = std::ldexp(1.0, int((bits >> 23) & 0xffu) - 127 - 23);
  probe_iterates_.insert(probe_iterates_.end(), xs.begin(), xs.end());
  if (rec.pcg_iterations >= 0) {
    probe_directions_.insert(probe_directions_.end(), xs.begin(), xs.end());
    probe_directions_.insert(probe_directions_.end(), ds.begin(), ds.end());
  }
}

void Context::probe_begin() {
  records_.clear();
  attempts_.clear();
  probe_iterates_.clear();
  probe_directions_.clear();
  probe_trials_.clear();
}

// runPtcProbes (drape-e7.ts:190-200): x_n = x, x_hat = x_n + h^2 g, scale = |grad E_s(x_n)|, one attempt.
void Context::probe_step(const double* x, double h, int step) {
  set_positions(x);
  check(cudaMemcpyAsync(xn_.ptr, x_.ptr, 3 * size_t(host_.V) * sizeof(double), cudaMemcpyDeviceToDevice, stream_),
        "save");
  const double scale = static_residual();
  record_step_ = step;
  probe_log_ = true;
  try {
    attempt(h, scale);
  } catch (...) {
    probe_log_ = false;
    throw;
  }
  probe_log_ = false;
}

int Context::solve_equilibrium(const double* start, double h0, drape_run_log* log) {
  if (start) set_positions(start);
  const size_t nv = 3 * size_t(host_.V);
  const double L = gravity_load_;
  double h = h0 > 0 ? h0 : opt_.h0;
  const double h_floor = opt_.h0 * opt_.h_min_factor;
  std::memset(phase_ms_, 0, sizeof phase_ms_);
  pcg_launches_ = 0;
  kernels_ = 0;
  fallbacks_ = 0;
  std::memset(mg_outcome_, 0, sizeof mg_outcome_);
  mg_iterations_ = 0;
  steps_.clear();
  records_.clear();
  attempts_.clear();
  states_.clear();
  check(cudaEventRecord(ev_[4], stream_), "event");
  drape_run_log out{};
  out.gravity_load = L;
  auto t_start = std::chrono::steady_clock::now();
  auto elapsed = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count(); };
  int reason = 1;
  double r = 0.0;
  for (;;) {
    r = static_residual();
    if ((opt_.equilibrium_absolute > 0 && r <= opt_.equilibrium_absolute) ||
        (opt_.equilibrium_relative > 0 && r / L <= opt_.equilibrium_relative)) {
      reason = 0;
      break;
    }
    if (!std::isfinite(r)) {
      reason = 2;
      break;
    }
    if (int(steps_.size()) >= opt_.max_steps) {
      reason = 1;
      break;
    }
    if (opt_.time_budget_s > 0 && elapsed() > opt_.time_budget_s) {
      reason = 3;
      break;
    }
    check(cudaMemcpyAsync(xn_.ptr, x_.ptr, nv * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "save");
    bool accepted = false;
    AttemptResult res;
    double h_try = h;
    int rejected = 0;
    record_step_ = int(steps_.size()) + 1;
    auto log_attempt = [&](int index, double ht, int reason, int start) {
      drape_attempt_record a{};
      a.step = record_step_;
      a.attempt = index;
      a.reason = reason;
      a.record_start = start;
      a.record_end = int(records_.size());
      a.h = ht;
      attempts_.push_back(a);
    };
    // attempt outcome as the reference's REJECTION code (drape-e7.ts:11)
    auto reason_of = [](const AttemptResult& a) {
      if (a.non_finite) return 3;
      if (a.updates == 0 && a.status == 3) return 1;
      if (a.updates == 0 && a.status == 2) return 2;
      return 0;
    };
    for (; rejected <= opt_.max_rejections; ++rejected) {
      h_try = std::max(h * std::pow(opt_.shrink, rejected), h_floor);
      int start = int(records_.size());
      res = attempt(h_try, r);
      bool failed = res.non_finite || (res.updates == 0 && (res.status == 2 || res.status == 3));
      if (!failed && opt_.curvature && res.status == 3 && res.updates > 0) {
        // mu-cap trigger: solve again without the b' d2d barrier term (drape-e7.ts:113-123).
        log_attempt(rejected, h_try, 4, start);
        start = int(records_.size());
        opt_.curvature = 0;
        AttemptResult again = attempt(h_try, r);
        opt_.curvature = 1;
        res = again;
        failed = res.non_finite || (res.updates == 0 && (res.status == 2 || res.status == 3));
      }
      log_attempt(rejected, h_try, reason_of(res), start);
      if (!failed) {
        accepted = true;
        break;
      }
      check(cudaMemcpyAsync(x_.ptr, xn_.ptr, nv * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "restore");
      out.rejected_attempts++;
    }
    if (!accepted) {
      reason = 2;
      break;
    }
    drape_step_record rec{};
    rec.step = int(steps_.size()) + 1;
    rec.h = h_try;
    rec.residual = r;
    rec.inner = res.updates;
    rec.rejected = rejected;
    rec.pcg_iterations = res.pcg_iterations;
    kcheck(launch_min_distance(dp_, x_.ptr, partial_.ptr, kReduceGrid, stream_), "min_distance");
    rec.min_distance = reduce_partials(kReduceGrid, 1, kMinDist);
    rec.seconds = elapsed();
    steps_.push_back(rec);
    if (keep_states_) {  // the accepted state in f32 (drape-e7.ts:175)
      std::vector<double> xs(nv);
      x_.download(xs.data(), nv, stream_);
      sync();
      states_.insert(states_.end(), xs.begin(), xs.end());
    }
    out.newton_iterations += res.updates;
    out.pcg_iterations += res.pcg_iterations;
    out.mu_retries += res.mu_retries;
    if (opt_.progress)
      std::fprintf(stderr, "step %d h %.3e r/L %.3e inner %d rej %d pcg %d %.2f s\n", rec.step, h_try, r / L,
                   res.updates, rejected, res.pcg_iterations, elapsed());
    double factor = opt_.controller == 1 ? opt_.growth : (res.updates < opt_.inner_max ? opt_.growth : opt_.shrink);
    h = std::min(std::max(h_try * factor, h_floor), opt_.h_max);
  }
  final_h_ = h;
  out.ptc_steps = int(steps_.size());
  out.reason = reason;
  out.final_residual = r;
  out.final_relative_residual = r / L;
  out.final_h = h;
  out.seconds = elapsed();
  out.static_energy = static_energy();
  out.ms_assembly = phase_ms_[kAssembly];
  out.ms_pcg = phase_ms_[kPcg];
  out.ms_line_search = phase_ms_[kLineSearch];
  out.ms_ccd = phase_ms_[kCcd];
  out.ms_other = out.seconds * 1e3 - out.ms_assembly - out.ms_pcg - out.ms_line_search - out.ms_ccd;
  out.pcg_launches = int(pcg_launches_);
  out.pcg_grid = pcg_cfg_.grid;
  check(cudaEventRecord(ev_[5], stream_), "event");
  sync();
  float dev_ms = 0.0f;
  check(cudaEventElapsedTime(&dev_ms, ev_[4], ev_[5]), "event time");
  out.device_seconds = dev_ms / 1e3;
  out.kernel_launches = int(kernels_);
  out.fallbacks = fallbacks_;
  out.mg_levels = opt_.preconditioner != 0 ? mg_levels_ : 0;
  if (opt_.progress && out.mg_levels)
    std::fprintf(stderr,
                 "multilevel: %lld iterations; solves converged %lld, limit %lld, breakdown %lld, stalled %lld, "
                 "coarse pivot %lld; block-Jacobi fallback converged %lld, limit %lld, breakdown %lld\n",
                 mg_iterations_, mg_outcome_[0], mg_outcome_[1], mg_outcome_[2], mg_outcome_[3], mg_outcome_[4],
                 mg_outcome_[5], mg_outcome_[6], mg_outcome_[7]);
  if (log) *log = out;
  return reason;
}

// One backward-Euler step of size h from the current state x_n with velocity v (drape.rs:410-417,
// drape-e4.ts:45-52): x_hat = x_n + h v + h^2 g, the scale |grad Phi(x_n)|, the regularised Newton from the
// CCD-cut prediction x_n + alpha_max (x_hat - x_n) to |grad Phi| / scale <= tolerance, then v = (x - x_n) / h.
int Context::time_step(double h, const double* v_in, double tolerance, int max_iterations, double* v_out,
                       drape_time_step_log* log) {
  const size_t nv = 3 * size_t(host_.V);
  if (!(h > 0) || !(tolerance > 0) || max_iterations < 1) throw std::invalid_argument("invalid time step arguments");
  std::memset(phase_ms_, 0, sizeof phase_ms_);
  records_.clear();
  attempts_.clear();
  record_step_ = 1;
  auto t0 = std::chrono::steady_clock::now();
  if (vel_.n != nv) vel_.alloc(nv);
  if (v_in) vel_.upload(v_in, nv, stream_);
  else check(cudaMemsetAsync(vel_.ptr, 0, nv * sizeof(double), stream_), "memset");
  check(cudaMemcpyAsync(xn_.ptr, x_.ptr, nv * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "save");
  kcheck(launch_predict(dp_, xn_.ptr, vel_.ptr, h, xhat_.ptr, stream_), "predict");
  const double scale = assemble(xn_.ptr, 1.0 / (h * h), 0.0, 0, false);
  AttemptResult res = newton(h, scale, tolerance, max_iterations, true);
  kcheck(launch_velocity(int(nv), x_.ptr, xn_.ptr, h, vel_.ptr, stream_), "velocity");
  if (v_out) vel_.download(v_out, nv, stream_);
  sync();
  drape_time_step_log out{};
  out.iterations = res.updates;
  out.status = res.non_finite ? 6 : res.status == 0 ? 1 : res.status == 1 ? 2 : res.status == 2 ? 3 : 5;
  out.pcg_iterations = res.pcg_iterations;
  out.mu_retries = res.mu_retries;
  out.scale = scale;
  out.final_relative_residual = records_.empty() ? 0.0 : records_.back().relative_residual;
  out.max_mu = res.max_mu;
  out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (log) *log = out;
  return out.status;
}

// ---------------------------------------------------------------- host-buffer entry points
double Context::assemble_host(const double* x, const double* x_hat, double h, double mu, int mode, int curvature,
                              double* grad, float* blocks) {
  const size_t nv = 3 * size_t(host_.V);
  xt_.upload(x, nv, stream_);
  if (x_hat) xhat_.upload(x_hat, nv, stream_);
  int saved = opt_.curvature;
  opt_.curvature = curvature;
  double norm = assemble(xt_.ptr, h > 0 ? 1.0 / (h * h) : 0.0, mu, mode, blocks != nullptr);
  opt_.curvature = saved;
  if (grad) g_.download(grad, 3 * size_t(host_.R), stream_);
  if (blocks) {
    std::vector<float4> h0(host_.B), h1(host_.B);
    std::vector<float> h2(host_.B);
    a0_.download(h0.data(), host_.B, stream_);
    a1_.download(h1.data(), host_.B, stream_);
    a2_.download(h2.data(), host_.B, stream_);
    sync();
    for (int k = 0; k < host_.B; ++k) {
      float* o = blocks + 9 * size_t(k);
      o[0] = h0[k].x;
      o[1] = h0[k].y;
      o[2] = h0[k].z;
      o[3] = h0[k].w;
      o[4] = h1[k].x;
      o[5] = h1[k].y;
      o[6] = h1[k].z;
      o[7] = h1[k].w;
      o[8] = h2[k];
    }
  }
  sync();
  return norm;
}

void Context::upload_blocks(const float* blocks) {
  const int B = host_.B;
  std::vector<float4> h0(B), h1(B);
  std::vector<float> h2(B);
  for (int k = 0; k < B; ++k) {
    const float* v = blocks + 9 * size_t(k);
    h0[k] = make_float4(v[0], v[1], v[2], v[3]);
    h1[k] = make_float4(v[4], v[5], v[6], v[7]);
    h2[k] = v[8];
  }
  a0_.upload(h0.data(), B, stream_);
  a1_.upload(h1.data(), B, stream_);
  a2_.upload(h2.data(), B, stream_);
  mg_stale_ = true;
  mg_setups_since_power_ = 1 << 20;  // an unrelated matrix: fresh spectral estimates
  sync();
}

PcgResult Context::pcg_host(const float* blocks, const double* rhs, double rtol, int max_iterations, double* solution) {
  const int R = host_.R;
  if (blocks) upload_blocks(blocks);
  std::vector<float4> b(R);
  for (int r = 0; r < R; ++r)
    b[r] = make_float4(float(rhs[3 * r]), float(rhs[3 * r + 1]), float(rhs[3 * r + 2]), 0.0f);
  b_.upload(b.data(), R, stream_);
  PcgResult res = direction_solve(rtol, max_iterations);
  std::vector<float4> x(R);
  px_.download(x.data(), R, stream_);
  sync();
  for (int r = 0; r < R; ++r) {
    solution[3 * r] = x[r].x;
    solution[3 * r + 1] = x[r].y;
    solution[3 * r + 2] = x[r].z;
  }
  return res;
}

double Context::energy_change_host(const double* x, const double* x_hat, double h, const double* d, double alpha,
                                   int mode) {
  const size_t nv = 3 * size_t(host_.V);
  xt_.upload(x, nv, stream_);
  if (x_hat) xhat_.upload(x_hat, nv, stream_);
  d_.upload(d, nv, stream_);
  return energy_change(xt_.ptr, d_.ptr, alpha, h > 0 ? 1.0 / (h * h) : 0.0, mode);
}

double Context::max_step_host(const double* x, const double* d) {
  const size_t nv = 3 * size_t(host_.V);
  xt_.upload(x, nv, stream_);
  d_.upload(d, nv, stream_);
  return max_step(xt_.ptr, d_.ptr);
}

void Context::element_terms_host(const double* x, int exact, float* grad, float* hess) {
  xt_.upload(x, 3 * size_t(host_.V), stream_);
  const size_t ng = 9 * size_t(host_.T) + 12 * size_t(host_.H), nh = 81 * size_t(host_.T) + 144 * size_t(host_.H);
  DeviceArray<float> g, h;
  g.alloc(ng);
  h.alloc(nh);
  kcheck(launch_element_terms(dp_, xt_.ptr, exact, g.ptr, h.ptr, stream_), "element terms");
  if (grad) g.download(grad, ng, stream_);
  if (hess) h.download(hess, nh, stream_);
  sync();
}

void Context::row_terms_host(const double* x, const double* x_hat, const double* row_mass, double mu, int contact,
                             int curvature, float* grad, float* hess) {
  const size_t nv = 3 * size_t(host_.V), R = size_t(host_.R);
  xt_.upload(x, nv, stream_);
  d_.upload(x_hat, nv, stream_);
  DeviceArray<double> m;
  if (row_mass) {
    m.alloc(R);
    m.upload(row_mass, R, stream_);
  }
  DeviceArray<float> g, h;
  g.alloc(3 * R);
  h.alloc(9 * R);
  kcheck(launch_row_terms(dp_, xt_.ptr, d_.ptr, row_mass ? m.ptr : nullptr, mu, contact, curvature, g.ptr, h.ptr,
                          stream_),
         "row terms");
  if (grad) g.download(grad, 3 * R, stream_);
  if (hess) h.download(hess, 9 * R, stream_);
  sync();
}

double Context::static_energy_host(const double* x) {
  xt_.upload(x, 3 * size_t(host_.V), stream_);
  kcheck(launch_static_energy(dp_, xt_.ptr, partial_.ptr, kReduceGrid, stream_), "static_energy");
  return reduce_partials(kReduceGrid, 0, kEnergy);
}

float Context::time_spmv(int launches, int lanes_per_row, int threads) {
  DevBsr A{a0_.ptr, a1_.ptr, a2_.ptr};
  for (int i = 0; i < 3; ++i)
    kcheck(launch_spmv(host_.R, row_ptr_.ptr, col_idx_.ptr, A, pp0_.ptr, pq_.ptr, lanes_per_row, threads, stream_), "spmv");
  check(cudaEventRecord(ev_[2], stream_), "event");
  for (int i = 0; i < launches; ++i)
    kcheck(launch_spmv(host_.R, row_ptr_.ptr, col_idx_.ptr, A, pp0_.ptr, pq_.ptr, lanes_per_row, threads, stream_), "spmv");
  check(cudaEventRecord(ev_[3], stream_), "event");
  sync();
  float ms = 0;
  cudaEventElapsedTime(&ms, ev_[2], ev_[3]);
  return ms / launches;
}

float Context::time_assembly(int launches) {
  AssembleArgs a{};
  a.p = dp_;
  a.x = x_.ptr;
  a.x_hat = x_.ptr;
  a.inv_h2 = 1.0;
  a.mode = 0;
  a.exact = opt_.tangent == 0;
  a.curvature = opt_.curvature;
  a.grad = g_.ptr;
  a.bsr = DevBsr{a0_.ptr, a1_.ptr, a2_.ptr};
  a.partial = partial_.ptr;
  for (int i = 0; i < 3; ++i) kcheck(launch_assemble(a, stream_), "assemble");
  check(cudaEventRecord(ev_[2], stream_), "event");
  for (int i = 0; i < launches; ++i) kcheck(launch_assemble(a, stream_), "assemble");
  check(cudaEventRecord(ev_[3], stream_), "event");
  sync();
  float ms = 0;
  cudaEventElapsedTime(&ms, ev_[2], ev_[3]);
  return ms / launches;
}

}  // namespace drape

namespace drape {
// ------------------------------------------------------------------------------------ multilevel preconditioner

namespace {
constexpr int kMgStallWindow = 128; // block Jacobi takes over when |r| fell by < 10% over this many iterations
}  // namespace

// Hierarchy storage, pointers and the solve graph (the pointers never change).
void Context::configure_mg() {
  if (mg_levels_ == 0) return;
  const int L = mg_levels_, R = host_.R;
  int n[kMgMaxLevels], rows[kMgMaxLevels];
  n[0] = host_.columns;
  rows[0] = R;
  // Level 1 is stored for the 7 x 7 stencil of the smoothed prolongation (the bilinear one uses its first 25
  // offsets per row); the fine level adds Sp (9R floats) and the vectors t, u, y of the smoothed fine steps.
  size_t a_count = 0, s_count = 18 * size_t(R), v_count = 10 * size_t(R);
  for (int l = 1; l < L; ++l) {
    n[l] = (n[l - 1] - 1) / 2 + 1;
    rows[l] = n[l] * n[l];
    a_count += size_t(l == 1 ? kMgStencilWide : kMgStencil) * 9 * rows[l];
    s_count += 9 * size_t(rows[l]);
    v_count += 3 * size_t(rows[l]);
  }
  mg_a64_.alloc(a_count);
  mg_a_.alloc(a_count / 9 * 3);  // one 48-byte block (3 float4) per (row, offset)
  mg_s_.alloc(s_count);
  mg_vec_.alloc(v_count);
  check(cudaMemsetAsync(mg_vec_.ptr, 0, v_count * sizeof(float4), stream_), "memset");
  check(cudaMemsetAsync(mg_s_.ptr, 0, s_count * sizeof(float), stream_), "memset");
  const int m = 3 * rows[L - 1];
  mg_inv_.alloc(size_t(m) * m);
  mg_partial_.alloc(4 * size_t(kMgPartials));
  check(cudaMemsetAsync(mg_partial_.ptr, 0, mg_partial_.n * sizeof(float), stream_), "memset");
  mg_state_.alloc((sizeof(MgState) + sizeof(float) - 1) / sizeof(float));
  mg_error_.alloc(1);

  MgDevice d{};
  d.fine = MgFine{R, n[0], row_ptr_.ptr, col_idx_.ptr, diag_pos_.ptr, DevBsr{a0_.ptr, a1_.ptr, a2_.ptr}};
  d.levels = L;
  double* a64 = mg_a64_.ptr;
  float4* a32 = mg_a_.ptr;
  float* sm = mg_s_.ptr;
  float4* v = mg_vec_.ptr;
  for (int l = 0; l < L; ++l) {
    MgLevel& lv = d.lv[l];
    lv.n = n[l];
    lv.rows = rows[l];
    lv.S = sm;
    sm += 9 * size_t(rows[l]);
    if (l > 0) {
      const int cap = l == 1 ? kMgStencilWide : kMgStencil;
      lv.A64 = a64;
      lv.A = a32;
      a64 += size_t(cap) * 9 * rows[l];
      a32 += size_t(cap) * 3 * rows[l];
      lv.r = v;
      v += rows[l];
    }
    lv.z = v;
    v += rows[l];
    lv.e = v;
    v += rows[l];
  }
  d.r[0] = v;
  d.r[1] = v + R;
  d.p[0] = v + 2 * size_t(R);
  d.p[1] = v + 3 * size_t(R);
  d.q = v + 4 * size_t(R);
  d.t = v + 5 * size_t(R);
  d.u = v + 6 * size_t(R);
  d.y = v + 7 * size_t(R);
  d.Sp = sm;
  d.b = b_.ptr;
  d.x = px_.ptr;
  d.coarse_inv = mg_inv_.ptr;
  mg_omega_.alloc(kMgMaxLevels);
  d.omega = mg_omega_.ptr;
  d.partial = mg_partial_.ptr;
  d.state = reinterpret_cast<MgState*>(mg_state_.ptr);
  d.error = mg_error_.ptr;
  mg_ = d;
  mg_prolongation_ = -1;
  build_mg_graph();
}

// The solve graph for the prolongation the options ask for (the kernel sequence differs): level 1's stencil width
// and the smoothed flag follow it. Rebuilt when the option changes.
void Context::build_mg_graph() {
  const int smoothed = opt_.prolongation != 0 ? 1 : 0;
  if (mg_prolongation_ == smoothed) return;
  sync();
  if (mg_graph_) {
    cudaGraphExecDestroy(mg_graph_);
    mg_graph_ = nullptr;
  }
  mg_.smoothed = smoothed;
  mg_.lv[1].w = smoothed ? 7 : 5;
  // Programmatic dependent launch inside the loop body where the driver accepts it, plain edges otherwise.
  mg_graph_pdl_ = mg_build_solve_graph(mg_, stream_, &mg_graph_, &mg_graph_launches_, true) == cudaSuccess;
  if (!mg_graph_pdl_) {
    cudaGetLastError();
    mg_graph_ = nullptr;
    check(mg_build_solve_graph(mg_, stream_, &mg_graph_, &mg_graph_launches_, false), "multilevel solve graph");
  }
  mg_prolongation_ = smoothed;
  mg_stale_ = true;
}

// Set-up for the matrix now in the BSR planes: smoothers, Galerkin products, coarsest inverse.
void Context::mg_prepare() {
  build_mg_graph();
  if (!mg_stale_) return;
  check(cudaMemsetAsync(mg_error_.ptr, 0, sizeof(int), stream_), "memset");
  const float omega = opt_.smoother_omega > 0 ? float(opt_.smoother_omega) : 0.0f;  // 0: spectral damping
  const bool reuse = omega == 0.0f && mg_setups_since_power_ < 4;
  mg_setups_since_power_ = reuse ? mg_setups_since_power_ + 1 : 1;
  const bool network = opt_.preconditioner == 2;
  bool fine_ready = false;
  kcheck(mg_setup(mg_, omega, true, reuse, stream_, side_stream_, setup_fork_, setup_join_,
                  network ? fine_ready_ : nullptr, &fine_ready),
         "multilevel set-up");
  // fine smoother, Galerkin products, coarse smoothers, coarsest inverse; the power method (twice with the
  // smoothed prolongation: the fine level first) and its scaling; Sp
  kernels_ += 2 * (mg_levels_ - 1) + (omega > 0 ? 0 : (reuse ? 0 : (kMgPowerSteps + 1) * (mg_.smoothed ? 2 : 1)) +
                                                       mg_levels_ - 1) + mg_.smoothed;
  if (opt_.preconditioner == 2) {
    if (!net_) throw std::invalid_argument("preconditioner 2 needs a preconditioner network (drape_set_network)");
    ensure_nn_buffers();
    if (fine_ready) {  // beside the Galerkin products, joined before the solve
      check(cudaStreamWaitEvent(net_stream_, fine_ready_, 0), "wait");
      kcheck(nn_forward(nnb_, net_->view(), mg_.omega, mg_.lv[0].S, net_stream_), "preconditioner network");
      check(cudaEventRecord(net_done_, net_stream_), "event");
      check(cudaStreamWaitEvent(stream_, net_done_, 0), "join");
    } else {
      kcheck(nn_forward(nnb_, net_->view(), mg_.omega, mg_.lv[0].S, stream_), "preconditioner network");
    }
    kernels_ += 2 + kNnLayers;  // features, input layer, message-passing layers, head
  }
  // the coarsest inverse (side stream) before anything that follows on the main stream
  check(cudaStreamWaitEvent(stream_, setup_join_, 0), "join");
  mg_stale_ = false;
}

PcgResult Context::mg_pcg(double rtol, int max_iterations, bool* stalled) {
  *stalled = false;
  mg_prepare();
  check(cudaEventRecord(ev_[0], stream_), "event");
  kcheck(mg_pcg_init(mg_, float(rtol * rtol), max_iterations, kMgStallWindow, stream_), "multilevel init");
  // The whole loop runs on the device (a conditional WHILE node); one read-back at the end.
  check(cudaGraphLaunch(mg_graph_, stream_), "graph launch");
  check(cudaMemcpyAsync(pinned_mg_, mg_.state, sizeof(MgState), cudaMemcpyDeviceToHost, stream_), "read");
  check(cudaMemcpyAsync(pinned_mg_ + 1, mg_.error, sizeof(int), cudaMemcpyDeviceToHost, stream_), "read");
  check(cudaEventRecord(ev_[1], stream_), "event");
  sync();
  const MgState& st = *pinned_mg_;
  const bool coarse_error = *reinterpret_cast<const int*>(pinned_mg_ + 1) != 0;
  *stalled = coarse_error || st.status == 4;
  // body executions: one per two iterations, plus the one that found the end
  kernels_ += (long long)(st.iterations / 2 + 1) * mg_graph_launches_;
  PcgResult r;
  cudaEventElapsedTime(&r.ms, ev_[0], ev_[1]);
  phase_ms_[kPcg] += r.ms;
  pcg_launches_++;
  r.iterations = st.iterations;
  // device status 1 converged, 2 iteration limit, 3 breakdown, 4 stalled (reported as the limit)
  r.status = st.status == 1 ? kPcgConverged : st.status == 3 ? kPcgBreakdown : kPcgIterationLimit;
  r.relative = st.rr0 > 0 ? std::sqrt(double(st.rr) / double(st.rr0)) : 0.0;
  return r;
}

PcgResult Context::direction_solve(double rtol, int max_iterations) {
  if (opt_.preconditioner == 0 || mg_levels_ == 0) return pcg(rtol, max_iterations);
  bool stalled = false;
  PcgResult r = mg_pcg(rtol, max_iterations, &stalled);
  mg_iterations_ += r.iterations;
  const bool coarse_failed = stalled && *reinterpret_cast<const int*>(pinned_mg_ + 1);
  mg_outcome_[coarse_failed ? 4 : stalled ? 3 : r.status == kPcgConverged ? 0 : r.status == kPcgBreakdown ? 2 : 1]++;
  // A breakdown is the Newton's signal to raise mu (as with block Jacobi); only a stalled residual or a failed
  // coarse factorisation hands the system to block-Jacobi PCG.
  if (!stalled) return r;
  ++fallbacks_;
  PcgResult j = pcg(rtol, max_iterations);
  mg_outcome_[j.status == kPcgConverged ? 5 : j.status == kPcgBreakdown ? 7 : 6]++;
  j.iterations += r.iterations;
  j.ms += r.ms;
  return j;
}

void Context::precondition_host(const float* blocks, const double* rhs, double* z) {
  if (mg_levels_ == 0) throw std::invalid_argument("no multilevel hierarchy for this problem");
  const int R = host_.R;
  if (blocks) upload_blocks(blocks);
  mg_prepare();
  std::vector<float4> r(R);
  for (int i = 0; i < R; ++i) r[i] = make_float4(float(rhs[3 * i]), float(rhs[3 * i + 1]), float(rhs[3 * i + 2]), 0.f);
  check(cudaMemcpyAsync(mg_.r[0], r.data(), R * sizeof(float4), cudaMemcpyHostToDevice, stream_), "upload");
  kcheck(mg_apply(mg_, stream_), "V-cycle");
  check(cudaMemcpyAsync(r.data(), mg_.lv[0].e, R * sizeof(float4), cudaMemcpyDeviceToHost, stream_), "download");
  sync();
  for (int i = 0; i < R; ++i) {
    z[3 * i] = r[i].x;
    z[3 * i + 1] = r[i].y;
    z[3 * i + 2] = r[i].z;
  }
}

void Context::time_multilevel(int iterations, float* out3, float* out3_stream, float* out_setup) {
  if (mg_levels_ == 0) throw std::invalid_argument("no multilevel hierarchy for this problem");
  if (out_setup) {  // one set-up with fresh spectral estimates (power method), one that reuses them
    for (int k = 0; k < 2; ++k) {
      mg_prepare();
      mg_stale_ = true;
      mg_setups_since_power_ = k == 0 ? (1 << 20) : 1;
      check(cudaEventRecord(ev_[2], stream_), "event");
      mg_prepare();
      check(cudaEventRecord(ev_[3], stream_), "event");
      sync();
      cudaEventElapsedTime(&out_setup[k], ev_[2], ev_[3]);
    }
  }
  mg_prepare();
  check(cudaMemcpyAsync(mg_.r[0], b_.ptr, host_.R * sizeof(float4), cudaMemcpyDeviceToDevice, stream_), "copy");
  for (int k = 0; k < 3; ++k) kcheck(mg_apply(mg_, stream_), "V-cycle");
  check(cudaEventRecord(ev_[2], stream_), "event");
  for (int k = 0; k < iterations; ++k) kcheck(mg_apply(mg_, stream_), "V-cycle");
  check(cudaEventRecord(ev_[3], stream_), "event");
  sync();
  cudaEventElapsedTime(&out3[0], ev_[2], ev_[3]);
  out3[0] /= iterations;
  // exactly `iterations` iterations: tolerance 0, no stall test
  kcheck(mg_pcg_init(mg_, 0.0f, 2, 0, stream_), "multilevel init");
  check(cudaGraphLaunch(mg_graph_, stream_), "graph launch");
  kcheck(mg_pcg_init(mg_, 0.0f, iterations, 0, stream_), "multilevel init");
  check(cudaEventRecord(ev_[2], stream_), "event");
  check(cudaGraphLaunch(mg_graph_, stream_), "graph launch");
  check(cudaEventRecord(ev_[3], stream_), "event");
  check(cudaMemcpyAsync(pinned_mg_, mg_.state, sizeof(MgState), cudaMemcpyDeviceToHost, stream_), "read");
  sync();
  cudaEventElapsedTime(&out3[1], ev_[2], ev_[3]);
  out3[1] /= std::max(1, pinned_mg_->iterations);
  out3[2] = mg_graph_pdl_ ? 1.0f : 0.0f;
  if (out3_stream) {  // the same iterations launched kernel by kernel on the stream (what ncu captures)
    kcheck(mg_pcg_init(mg_, 0.0f, iterations, 0, stream_), "multilevel init");
    check(cudaEventRecord(ev_[2], stream_), "event");
    kcheck(mg_launch_iterations(mg_, (iterations + 1) / 2, stream_), "multilevel iterations");
    check(cudaEventRecord(ev_[3], stream_), "event");
    check(cudaMemcpyAsync(pinned_mg_, mg_.state, sizeof(MgState), cudaMemcpyDeviceToHost, stream_), "read");
    sync();
    cudaEventElapsedTime(out3_stream, ev_[2], ev_[3]);
    *out3_stream /= std::max(1, pinned_mg_->iterations);
  }
}

int Context::multilevel_view(int level, int* width, double* op, float* smoother) {
  if (level < 0 || level >= mg_levels_) return -1;
  mg_prepare();
  const MgLevel& lv = mg_.lv[level];
  if (width) *width = level > 0 ? lv.w : 0;
  if (op && level > 0)
    check(cudaMemcpyAsync(op, lv.A64, size_t(lv.w) * lv.w * 9 * lv.rows * sizeof(double), cudaMemcpyDeviceToHost,
                          stream_), "download");
  if (smoother)
    check(cudaMemcpyAsync(smoother, lv.S, 9 * size_t(lv.rows) * sizeof(float), cudaMemcpyDeviceToHost, stream_),
          "download");
  sync();
  return lv.n;
}

// ------------------------------------------------------------------------------------ preconditioner network

Network::Network(int dev, uint64_t seed) : device(dev) {
  check(cudaSetDevice(device), "cudaSetDevice");
  master.alloc(kNnParams);
  adam_m.alloc(kNnParams);
  adam_v.alloc(kNnParams);
  bf16.alloc(kNnBf16);
  // Glorot-uniform weights from a 64-bit LCG, zero biases, a zero output layer (f = 0.9: the untrained network
  // is a little under the multilevel preconditioner's spectral smoother).
  std::vector<float> p(kNnParams, 0.0f);
  uint64_t state = seed * 6364136223846793005ULL + 1442695040888963407ULL;
  auto uniform = [&]() {
    state = state * 6364136223846793005ULL + 1442695040888963407ULL;
    return double(state >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  };
  auto fill = [&](int off, int fan_in, int fan_out) {
    const double a = std::sqrt(6.0 / (fan_in + fan_out));
    for (int t = 0; t < fan_in * fan_out; ++t) p[off + t] = float(a * uniform());
  };
  fill(kNnOffWin, kNnIn, kNnHidden);
  for (int l = 0; l < kNnLayers; ++l) fill(kNnOffLayer0 + l * kNnLayerSize, 2 * kNnHidden, kNnHidden);
  set(p.data());
}

NnWeights Network::view() {
  return NnWeights{master.ptr, reinterpret_cast<__nv_bfloat16*>(bf16.ptr), adam_m.ptr, adam_v.ptr};
}

void Network::set(const float* params) {
  check(cudaSetDevice(device), "cudaSetDevice");
  check(cudaMemcpy(master.ptr, params, kNnParams * sizeof(float), cudaMemcpyHostToDevice), "upload");
  check(cudaMemset(adam_m.ptr, 0, kNnParams * sizeof(float)), "memset");
  check(cudaMemset(adam_v.ptr, 0, kNnParams * sizeof(float)), "memset");
  adam_t = 0;
  check(nn_refresh_bf16(view(), nullptr), "bf16 weights");
  check(cudaDeviceSynchronize(), "synchronize");
}

void Network::get(float* params) {
  check(cudaSetDevice(device), "cudaSetDevice");
  check(cudaMemcpy(params, master.ptr, kNnParams * sizeof(float), cudaMemcpyDeviceToHost), "download");
}

namespace {
enum NnVec { kNb = 0, kNx, kZ1, kT, kC, kY, kU, kZ, kE, kAe, kAx, kGz, kSg, kGy, kGz1, kNnVecs };
}  // namespace

void Context::ensure_nn_buffers() {
  if (nnb_.R) return;
  if (mg_levels_ == 0) throw std::invalid_argument("the preconditioner network needs the multilevel hierarchy");
  const int R = host_.R, B = host_.B;
  nn_feat_.alloc(size_t(R) * kNnIn);
  nn_w_.alloc(B);
  nn_h_.alloc(size_t(kNnLayers + 1) * R * kNnHidden);
  nn_o_.alloc(R);
  nn_dh_.alloc(2 * size_t(R) * kNnHidden);
  nn_dx_.alloc(2 * size_t(R) * kNnHidden);
  nn_partial_.alloc(size_t(nn_back_ctas(R)) * kNnParams);
  nn_grad_.alloc(kNnParams);
  nn_dfac_.alloc(R);
  nn_s0_.alloc(9 * size_t(R));
  nn_zero_.alloc(9 * size_t(R));
  check(cudaMemsetAsync(nn_zero_.ptr, 0, 9 * size_t(R) * sizeof(float), stream_), "memset");
  nn_fscale_.alloc(4);
  nn_vec_.alloc(kNnVecs * size_t(R));
  check(cudaMemsetAsync(nn_vec_.ptr, 0, nn_vec_.n * sizeof(float4), stream_), "memset");
  nn_dot_partial_.alloc(256);
  nn_scalars_.alloc(8);
  // transpose map of the (symmetric) BSR pattern: entry of (j, i) for every entry (i, j)
  std::vector<int> tmap(B);
  for (int i = 0; i < R; ++i)
    for (int k = host_.row_ptr[i]; k < host_.row_ptr[i + 1]; ++k) {
      const int j = host_.col_idx[k];
      auto b0 = host_.col_idx.begin() + host_.row_ptr[j], b1 = host_.col_idx.begin() + host_.row_ptr[j + 1];
      auto it = std::lower_bound(b0, b1, i);
      if (it == b1 || *it != i) throw std::invalid_argument("the preconditioner network needs a symmetric pattern");
      tmap[k] = int(it - host_.col_idx.begin());
    }
  nn_transpose_.alloc(B);
  nn_transpose_.upload(tmap.data(), B, stream_);
  NnBuffers b{};
  b.R = R;
  b.B = B;
  b.row_ptr = row_ptr_.ptr;
  b.col_idx = col_idx_.ptr;
  b.diag_pos = diag_pos_.ptr;
  b.transpose = nn_transpose_.ptr;
  b.A = DevBsr{a0_.ptr, a1_.ptr, a2_.ptr};
  b.feat = nn_feat_.ptr;
  b.w = nn_w_.ptr;
  b.h = nn_h_.ptr;
  b.o = nn_o_.ptr;
  b.dh = nn_dh_.ptr;
  b.dx = nn_dx_.ptr;
  b.partial = nn_partial_.ptr;
  b.grad = nn_grad_.ptr;
  sync();
  nnb_ = b;
}

void Context::upload_tuple(const float* blocks, const double* rhs, const double* solution) {
  const int R = host_.R;
  upload_blocks(blocks);
  std::vector<float4> v(R);
  for (int pass = 0; pass < 2; ++pass) {
    const double* src = pass ? solution : rhs;
    for (int i = 0; i < R; ++i) v[i] = make_float4(float(src[3 * i]), float(src[3 * i + 1]), float(src[3 * i + 2]), 0.f);
    check(cudaMemcpyAsync(nn_vec_.ptr + size_t(pass ? kNx : kNb) * R, v.data(), R * sizeof(float4),
                          cudaMemcpyHostToDevice, stream_), "upload");
  }
  sync();
}

// One V-cycle with the network's smoother S = f S0 on (A, b, x) as separate steps (the cycle kernels with a zero
// fine smoother give the coarse correction C = P V_1 P^T), the loss ||x - z||_A^2 / ||x||_A^2 and, with
// `backward`, dL/df through the cycle (g_z = -2 A (x - z) / N; g_y = g_z - A S g_z; g_z1 = g_y - A C g_y) and
// the network's parameter gradient in nnb_.grad.
double Context::network_pass(Network& net, bool backward) {
  const int R = host_.R;
  auto V = [&](int k) { return nn_vec_.ptr + size_t(k) * R; };
  const DevBsr A{a0_.ptr, a1_.ptr, a2_.ptr};
  auto spmv = [&](const float4* x, float4* y) {
    kcheck(launch_spmv(R, row_ptr_.ptr, col_idx_.ptr, A, x, y, 8, 256, stream_), "spmv");
  };
  MgDevice coarse = mg_;
  coarse.lv[0].S = nn_zero_.ptr;
  auto C = [&](const float4* v, float4* out) {
    check(cudaMemcpyAsync(mg_.r[0], v, R * sizeof(float4), cudaMemcpyDeviceToDevice, stream_), "copy");
    kcheck(mg_apply(coarse, stream_), "coarse correction");
    check(cudaMemcpyAsync(out, mg_.lv[0].e, R * sizeof(float4), cudaMemcpyDeviceToDevice, stream_), "copy");
  };
  // hierarchy with the spectral smoother S0, then S = f S0 from the network
  mg_setups_since_power_ = 1 << 20;
  mg_stale_ = true;
  Network* keep = net_;
  net_ = nullptr;
  mg_prepare();
  net_ = keep;
  check(cudaMemcpyAsync(nn_s0_.ptr, mg_.lv[0].S, 9 * size_t(R) * sizeof(float), cudaMemcpyDeviceToDevice, stream_),
        "copy");
  kcheck(nn_forward(nnb_, net.view(), mg_.omega, mg_.lv[0].S, stream_), "network");
  const float* S = mg_.lv[0].S;
  float* fs = nn_fscale_.ptr;
  check(nn_block_apply(R, S, V(kNb), V(kZ1), stream_), "z1");        // z1 = S b
  spmv(V(kZ1), V(kT));
  check(nn_vec(R, V(kNb), V(kT), V(kT), 1.f, -1.f, nullptr, stream_), "t");  // t = b - A z1
  C(V(kT), V(kC));
  check(nn_vec(R, V(kZ1), V(kC), V(kY), 1.f, 1.f, nullptr, stream_), "y");    // y = z1 + C t
  spmv(V(kY), V(kU));
  check(nn_vec(R, V(kNb), V(kU), V(kU), 1.f, -1.f, nullptr, stream_), "u");   // u = b - A y
  check(nn_block_apply(R, S, V(kU), V(kZ), stream_), "Su");
  check(nn_vec(R, V(kY), V(kZ), V(kZ), 1.f, 1.f, nullptr, stream_), "z");     // z = y + S u
  check(nn_vec(R, V(kNx), V(kZ), V(kE), 1.f, -1.f, nullptr, stream_), "e");   // e = x - z
  spmv(V(kE), V(kAe));
  spmv(V(kNx), V(kAx));
  check(nn_dot(R, V(kNx), V(kAx), nn_dot_partial_.ptr, nn_scalars_.ptr, 0, fs, stream_), "x.Ax");  // fs = -2/N
  check(nn_dot(R, V(kE), V(kAe), nn_dot_partial_.ptr, nn_scalars_.ptr, 1, nullptr, stream_), "e.Ae");
  if (backward) {
    check(nn_vec(R, V(kAe), nullptr, V(kGz), 1.f, 0.f, fs, stream_), "g_z");    // g_z = -2 A e / N
    check(nn_block_apply(R, S, V(kGz), V(kSg), stream_), "S g_z");
    spmv(V(kSg), V(kT));
    check(nn_vec(R, V(kGz), V(kT), V(kGy), 1.f, -1.f, nullptr, stream_), "g_y");  // g_y = g_z - A S g_z
    C(V(kGy), V(kC));
    spmv(V(kC), V(kT));
    check(nn_vec(R, V(kGy), V(kT), V(kGz1), 1.f, -1.f, nullptr, stream_), "g_z1");  // g_z1 = g_y - A C g_y
    check(nn_dfactor(R, nn_s0_.ptr, V(kGz), V(kU), V(kGz1), V(kNb), nn_dfac_.ptr, stream_), "dL/df");
    kcheck(nn_backward(nnb_, net.view(), nn_dfac_.ptr, stream_), "network backward");
  }
  double sc[2];
  check(cudaMemcpyAsync(sc, nn_scalars_.ptr, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_), "read");
  sync();
  mg_stale_ = true;  // the hierarchy's fine smoother now holds this tuple's S
  return sc[0] != 0.0 ? sc[1] / sc[0] : 0.0;
}

double Context::network_gradient_host(Network& net, const float* blocks, const double* rhs, const double* solution,
                                      float* grad, float* factors) {
  ensure_nn_buffers();
  upload_tuple(blocks, rhs, solution);
  const double loss = network_pass(net, grad != nullptr);
  if (grad) check(cudaMemcpyAsync(grad, nn_grad_.ptr, kNnParams * sizeof(float), cudaMemcpyDeviceToHost, stream_),
                  "download");
  if (factors) {
    std::vector<float> o(host_.R);
    check(cudaMemcpyAsync(o.data(), nn_o_.ptr, host_.R * sizeof(float), cudaMemcpyDeviceToHost, stream_), "download");
    sync();
    for (int i = 0; i < host_.R; ++i)
      factors[i] = kNnFactorLow + kNnFactorSpan / (1.0f + std::exp(-(o[i] + kNnFactorShift)));
  }
  sync();
  return loss;
}

void Context::network_train_host(Network& net, int tuples, const float* const* blocks, const double* const* rhs,
                                 const double* const* solutions, int steps, double lr, double* losses) {
  ensure_nn_buffers();
  for (int k = 0; k < steps; ++k) {
    const int t = k % tuples;
    upload_tuple(blocks[t], rhs[t], solutions[t]);
    const double loss = network_pass(net, true);
    if (losses) losses[k] = loss;
    check(nn_adam(net.view(), nn_grad_.ptr, float(lr), ++net.adam_t, stream_), "adam");
    sync();
  }
}

template struct DeviceArray<double>;
template struct DeviceArray<int>;
template struct DeviceArray<unsigned short>;
template struct DeviceArray<float>;
template struct DeviceArray<float4>;
template struct DeviceArray<long long>;
template struct DeviceArray<unsigned long long>;
}  // namespace drape
