// Test infrastructure only (see core.h). C entry points the pytest suite and bench.py's CPU-baseline leg use
// (through ctypes) to ask the f64 oracle for the same quantities the CUDA path computes.
#include <chrono>
#include <cstring>
#include <memory>

#include "cases.h"
#include "drape.h"
#include "io.h"

using namespace oracle;

namespace {
thread_local std::string g_error;
struct Handle {
  Scene scene;
  std::unique_ptr<Drape> drape;
};
std::vector<Vec3> to_vec3(const double* x, size_t n) {
  std::vector<Vec3> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  return v;
}
void from_vec3(const std::vector<Vec3>& v, double* out) {
  for (size_t i = 0; i < v.size(); ++i)
    for (int k = 0; k < 3; ++k) out[3 * i + k] = v[i][k];
}
}  // namespace

extern "C" {

const char* oracle_last_error() { return g_error.c_str(); }

// kind 0: the reference sphere-on-floor scene with `edit` (base|w1|w2|w3|e5); 1: the sheet over a sphere
// (seed, radius, young, plane); 2: the pinned sheet. tangent 0 exact, 1 projected.
void* oracle_scene_create(int kind, int columns, const char* edit, uint64_t seed, double radius, double young,
                          int plane, int tangent) {
  try {
    auto h = std::make_unique<Handle>();
    if (kind == 0) h->scene = reference_scene(columns, edit ? edit : "base");
    else if (kind == 1) h->scene = sheet_scene(columns, seed, radius, young, plane != 0);
    else if (kind == 2) h->scene = pinned_scene(columns);
    else throw std::runtime_error("unknown scene kind");
    h->drape = std::make_unique<Drape>(h->scene, tangent ? TangentKind::Projected : TangentKind::Exact);
    return h.release();
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

void oracle_scene_free(void* p) { delete static_cast<Handle*>(p); }

// [V, T, H, R, B, colliders]
void oracle_scene_sizes(void* p, int64_t* out) {
  auto& d = *static_cast<Handle*>(p)->drape;
  out[0] = int64_t(d.mesh.rest.size());
  out[1] = int64_t(d.membranes.size());
  out[2] = int64_t(d.hinges.size());
  out[3] = d.rows();
  out[4] = d.pattern.blocks();
  out[5] = int64_t(d.contact.colliders.size());
}

// [dhat, kappa, |g|, gravity_load, gx, gy, gz]
void oracle_scene_scalars(void* p, double* out) {
  auto& d = *static_cast<Handle*>(p)->drape;
  out[0] = d.contact.barrier.dhat;
  out[1] = d.contact.barrier.kappa;
  out[2] = d.g_norm();
  out[3] = gravity_load(d);
  out[4] = d.gravity[0];
  out[5] = d.gravity[1];
  out[6] = d.gravity[2];
}

void oracle_scene_start(void* p, double* x) { from_vec3(static_cast<Handle*>(p)->drape->start, x); }
void oracle_scene_mass(void* p, double* m) {
  auto& d = *static_cast<Handle*>(p)->drape;
  std::memcpy(m, d.mass.data(), d.mass.size() * sizeof(double));
}
void oracle_scene_pattern(void* p, int32_t* row_ptr, int32_t* col_idx) {
  auto& d = *static_cast<Handle*>(p)->drape;
  for (size_t i = 0; i < d.pattern.row_ptr.size(); ++i) row_ptr[i] = d.pattern.row_ptr[i];
  for (size_t i = 0; i < d.pattern.col_idx.size(); ++i) col_idx[i] = d.pattern.col_idx[i];
}
// Topology: triangles [3T], hinges [4H], hinge stiffness [H].
void oracle_scene_topology(void* p, int32_t* tris, int32_t* hinges, double* stiffness) {
  auto& d = *static_cast<Handle*>(p)->drape;
  for (size_t e = 0; e < d.membranes.size(); ++e)
    for (int k = 0; k < 3; ++k) tris[3 * e + k] = d.membranes[e].vertices[k];
  for (size_t e = 0; e < d.hinges.size(); ++e) {
    for (int k = 0; k < 4; ++k) hinges[4 * e + k] = d.hinges[e].vertices[k];
    stiffness[e] = d.hinges[e].stiffness;
  }
}
void oracle_kernel_state(void* p, double* x) {
  Lcg rng(97);
  from_vec3(bent_state(*static_cast<Handle*>(p)->drape, rng), x);
}
void oracle_contact_state(void* p, double* x) { from_vec3(contact_state(*static_cast<Handle*>(p)->drape), x); }

// Residual g = grad Phi (3R) and regularised tangent K + mu M/h^2 (9B, BSR of the pattern) at x with x_hat and
// step h; curvature 0 drops the barrier's b' d2d term. Either output may be null.
int oracle_assemble(void* p, const double* x, const double* x_hat, double h, double mu, int curvature, double* grad,
                    double* vals) {
  try {
    auto& d = *static_cast<Handle*>(p)->drape;
    size_t V = d.mesh.rest.size();
    d.time_step = h;
    d.barrier_curvature = curvature != 0;
    DrapeStep s{&d, to_vec3(x_hat, V)};
    auto xv = to_vec3(x, V);
    if (grad) {
      auto r = s.residual(xv);
      std::memcpy(grad, r.data(), r.size() * sizeof(double));
    }
    if (vals) {
      Bsr m = s.regularized_tangent(xv, mu);
      std::memcpy(vals, m.vals.data(), m.vals.size() * sizeof(double));
    }
    d.barrier_curvature = true;
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

double oracle_energy_change(void* p, const double* x, const double* x_hat, double h, const double* dir, double alpha) {
  auto& d = *static_cast<Handle*>(p)->drape;
  size_t V = d.mesh.rest.size();
  d.time_step = h;
  DrapeStep s{&d, to_vec3(x_hat, V)};
  return s.energy_change(to_vec3(x, V), to_vec3(dir, V), alpha);
}

double oracle_max_step(void* p, const double* x, const double* dir) {
  auto& d = *static_cast<Handle*>(p)->drape;
  size_t V = d.mesh.rest.size();
  DrapeStep s{&d, to_vec3(x, V)};
  return s.max_step(to_vec3(x, V), to_vec3(dir, V));
}

void oracle_static_gradient(void* p, const double* x, double* out) {
  auto& d = *static_cast<Handle*>(p)->drape;
  auto g = static_gradient(d, to_vec3(x, d.mesh.rest.size()));
  std::memcpy(out, g.data(), g.size() * sizeof(double));
}
double oracle_static_energy(void* p, const double* x) {
  auto& d = *static_cast<Handle*>(p)->drape;
  return static_energy(d, to_vec3(x, d.mesh.rest.size()));
}

// PTC to equilibrium from `start` (null: the scene's cold start). controller 0 inner-count (reference), 1 doubling.
// direction 0 band Cholesky, 1 f64 block-Jacobi PCG (rtol, maxit). predicted_start 1: the reference's CCD-cut
// prediction as the inner Newton start, 0: the current state. Stops at r/L <= equilibrium, r <= absolute
// (when > 0), the floor rule (floor != 0), max_steps, or a stall. stats: [steps, newton, rejected, pcg, final_r,
// final_h, seconds, converged, reason code (0 tolerance 1 floor 2 cap 3 stalled)].
int oracle_ptc(void* p, const double* start, double h0, int controller, double equilibrium, double absolute, int floor,
               int max_steps, int direction, double rtol, int maxit, int progress, int predicted_start, double budget_s,
               double* x_out, double* stats) {
  try {
    auto& d = *static_cast<Handle*>(p)->drape;
    PtcRules r = PtcRules::reference();
    r.h0 = h0;
    r.controller = controller ? Controller::Doubling : Controller::InnerCount;
    r.equilibrium = equilibrium;
    r.absolute = absolute;
    r.floor_rule = floor != 0;
    r.predicted_start = predicted_start != 0;
    r.max_steps = max_steps;
    r.time_budget_s = budget_s;
    DirectionSolver dir{direction != 0, rtol, maxit};
    auto x0 = start ? to_vec3(start, d.mesh.rest.size()) : d.start;
    auto t0 = std::chrono::steady_clock::now();
    PtcRun run = ptc_solve(d, x0, h0, r, dir, false, progress != 0);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    from_vec3(run.states.back(), x_out);
    int newton = 0, rejected = 0, pcg = 0;
    for (auto& s : run.steps) {
      newton += s.inner_iterations;
      rejected += s.rejected_attempts;
      pcg += s.pcg_iterations;
    }
    int code = run.reason == "tolerance" ? 0 : run.reason == "floor" ? 1 : run.reason == "cap" ? 2 : 3;
    double v[9] = {double(run.steps.size()), double(newton), double(rejected), double(pcg), run.final_residual,
                   run.final_h, secs, run.converged() ? 1.0 : 0.0, double(code)};
    std::memcpy(stats, v, sizeof v);
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

// One backward-Euler step (drape.rs:410-417) of size h from (x, v): Newton (regularised) to |grad Phi| / scale <=
// tolerance or max_iterations updates, direction 0 band Cholesky / 1 f64 block-Jacobi PCG (rtol, maxit). Writes
// the new positions and velocity; stats: [updates, status (1 converged, 2 limit, 3 line search, 5 mu cap), final
// relative residual, scale, max mu].
int oracle_time_step(void* p, const double* x, const double* v, double h, double tolerance, int max_iterations,
                     int direction, double rtol, int maxit, double* x_out, double* v_out, double* stats) {
  try {
    auto& d = *static_cast<Handle*>(p)->drape;
    size_t V = d.mesh.rest.size();
    NewtonSettings set{tolerance, max_iterations, 1e-4, 30};
    DirectionSolver dir{direction != 0, rtol, maxit};
    TimeStepResult r = time_step(d, to_vec3(x, V), v ? to_vec3(v, V) : std::vector<Vec3>(V, Vec3{0, 0, 0}), h, set, dir);
    from_vec3(r.solution.positions, x_out);
    from_vec3(r.velocity, v_out);
    const StepStatus st = r.solution.status;
    int code = st == StepStatus::Converged ? 1 : st == StepStatus::IterationLimit ? 2
             : st == StepStatus::LineSearchFailed ? 3 : st == StepStatus::RegularizationCap ? 5 : 1;
    double out[5] = {double(r.solution.halvings.size()), double(code), r.solution.residuals.back(), r.scale,
                     r.solution.regularization.max_mu};
    std::memcpy(stats, out, sizeof out);
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

// Block-Jacobi PCG on a BSR system (f64, or f32 emulating the GPU's operation order when single != 0).
// info: [iterations, converged, breakdown, recursive relative residual].
void oracle_pcg(int rows, const int32_t* row_ptr, const int32_t* col_idx, const double* vals, const double* rhs,
                double tol, int maxit, int replace_every, double replace_above, int single, int detect_breakdown,
                double* x_out, double* info) {
  Bsr m;
  m.row_ptr.assign(row_ptr, row_ptr + rows + 1);
  m.col_idx.assign(col_idx, col_idx + row_ptr[rows]);
  m.vals.assign(vals, vals + 9 * size_t(row_ptr[rows]));
  std::vector<double> b(rhs, rhs + 3 * size_t(rows));
  PcgSettings s;
  s.tolerance = tol;
  s.max_iterations = maxit;
  s.history_stride = 0;
  s.replace_every = replace_every;
  s.replace_above = replace_above;
  s.detect_breakdown = detect_breakdown != 0;
  PcgReport rep = single ? pcg_solve<float>(m, b, s) : pcg_solve<double>(m, b, s);
  std::memcpy(x_out, rep.solution.data(), rep.solution.size() * sizeof(double));
  info[0] = rep.iterations;
  info[1] = rep.converged;
  info[2] = rep.breakdown;
  info[3] = rep.recursive_relative_residual;
}

// E1 linear case (kind 0 tension, 1 slack, 2 dynamic): sizes [rows, blocks], then the arrays.
void oracle_case_sizes(int kind, int columns, int64_t* out) {
  auto c = build_case(CaseKind(kind), columns);
  out[0] = c.matrix.rows();
  out[1] = c.matrix.blocks();
}
void oracle_case_build(int kind, int columns, int32_t* row_ptr, int32_t* col_idx, double* vals, double* rhs) {
  auto c = build_case(CaseKind(kind), columns);
  for (size_t i = 0; i < c.matrix.row_ptr.size(); ++i) row_ptr[i] = c.matrix.row_ptr[i];
  for (size_t i = 0; i < c.matrix.col_idx.size(); ++i) col_idx[i] = c.matrix.col_idx[i];
  std::memcpy(vals, c.matrix.vals.data(), c.matrix.vals.size() * sizeof(double));
  std::memcpy(rhs, c.rhs.data(), c.rhs.size() * sizeof(double));
}

int oracle_band_bandwidth(int rows, const int32_t* row_ptr, const int32_t* col_idx) {
  int w = 0;
  for (int r = 0; r < rows; ++r)
    for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k)
      if (col_idx[k] <= r) w = std::max(w, 3 * (r - col_idx[k]) + 2);
  return w;
}

void oracle_prolong(const double* coarse, int coarse_columns, double* fine) {
  auto f = prolong(to_vec3(coarse, size_t(coarse_columns) * coarse_columns), coarse_columns);
  from_vec3(f, fine);
}

}  // extern "C"
