// Test infrastructure only (see core.h). Implementation of drape.h.
#include "drape.h"

#include <chrono>
#include <cstdio>
#include <cstring>

namespace oracle {

// ---------------------------------------------------------------- scenes
Scene reference_scene(int columns, const std::string& edit) {
  // e7_run.rs:18-26 edits; drape.rs:53-84 contact and lift; drape.rs:108-123 scaled material and mesh.
  double mat = 1.0, radius_f = 1.0, rest_f = 1.0;
  bool placed = true;
  if (edit == "base") {
  } else if (edit == "w1") {
    mat = 1.25;
  } else if (edit == "w2") {
    radius_f = 0.96;
  } else if (edit == "w3") {
    rest_f = 1.03;
  } else if (edit == "e5") {
    placed = false;
  } else {
    throw std::runtime_error("unknown edit '" + edit + "' (base|w1|w2|w3|e5)");
  }
  const double sheet = 0.5;
  Scene s;
  s.name = "reference-" + edit;
  s.mesh = Mesh::grid(columns, columns, sheet, sheet);
  if (rest_f != 1.0) {
    double c = 0.5 * sheet;
    for (auto& p : s.mesh.rest) p = {c + rest_f * (p[0] - c), c + rest_f * (p[1] - c)};
  }
  Material base = Material::knit_baseline();
  s.material = base;
  s.material.wale *= mat;
  s.material.course *= mat;
  s.material.coupling *= mat;
  s.material.shear *= mat;
  s.material.bend_wale *= mat;
  s.material.bend_course *= mat;
  double radius = 0.25 * sheet * radius_f, dhat = 1e-3 * sheet;
  auto areas = s.mesh.vertex_areas();
  double heaviest = 0;
  for (double a : areas) heaviest = std::max(heaviest, s.material.density * a);
  s.contact.colliders = {Collider::plane({0, 0, 1}, 0.0), Collider::sphere({0.5 * sheet, 0.5 * sheet, radius}, radius)};
  s.contact.barrier = Barrier{dhat, Barrier::resting_kappa(dhat, heaviest, 9.81)};
  double lift = 2.0 * radius + (placed ? 2.0 * dhat : 0.02 * sheet);
  for (auto& p : s.mesh.rest) s.start.push_back({p[0], p[1], lift});
  s.gravity = {0, 0, -9.81};
  return s;
}

Scene pinned_scene(int columns) {
  Scene s;
  s.name = "pinned";
  s.mesh = Mesh::grid(columns, columns, 0.5, 0.5);
  s.material = Material::knit_baseline();
  s.fixed = {(s.mesh.rows - 1) * s.mesh.columns, s.mesh.rows * s.mesh.columns - 1};
  for (auto& p : s.mesh.rest) s.start.push_back({p[0], p[1], 0.0});
  return s;
}

Scene sheet_scene(int columns, uint64_t seed, double radius, double young, bool with_plane, double plane_y) {
  Scene s;
  s.name = "sheet";
  s.mesh = Mesh::grid(columns, columns, 1.0, 1.0);
  s.material = Material::isotropic(young, 0.3, 5e-4, 1e-5, 0.15);
  s.gravity = {0, -9.81, 0};
  s.contact.colliders = {Collider::sphere({0, 0, 0}, radius)};
  if (with_plane) s.contact.colliders.push_back(Collider::plane({0, 1, 0}, plane_y));
  s.contact.barrier = Barrier{2e-3, 1e3};
  Lcg rng(seed);
  for (auto& p : s.mesh.rest) s.start.push_back({p[0] - 0.5, 0.35 + 1e-5 * rng.uniform(), p[1] - 0.5});
  return s;
}

// ---------------------------------------------------------------- drape
Drape::Drape(const Scene& s, TangentKind kind)
    : mesh(s.mesh), material(s.material), fixed(s.fixed), tangent_kind(kind), contact(s.contact),
      gravity(s.gravity), start(s.start) {
  int V = int(mesh.rest.size());
  for (auto& t : mesh.triangles) membranes.push_back(MembraneElement::make(t, mesh.rest));
  hinges = hinge_elements(mesh, material);
  row_of.assign(V, -1);
  for (int v = 0; v < V; ++v)
    if (std::find(fixed.begin(), fixed.end(), v) == fixed.end()) {
      row_of[v] = int(free_.size());
      free_.push_back(v);
    }
  std::vector<std::vector<int>> groups;
  auto to_rows = [&](const int* vs, int n) {
    std::vector<int> g;
    for (int k = 0; k < n; ++k)
      if (row_of[vs[k]] >= 0) g.push_back(row_of[vs[k]]);
    return g;
  };
  for (auto& t : mesh.triangles) groups.push_back(to_rows(t.data(), 3));
  for (auto& h : mesh.hinges) groups.push_back(to_rows(h.data(), 4));
  pattern = Bsr::with_pattern(int(free_.size()), groups);
  auto areas = mesh.vertex_areas();
  for (double a : areas) mass.push_back(material.density * a);
}

double Drape::barrier_energy(const std::vector<Vec3>& x) const {
  double s = 0;
  for (int i : free_) s += contact.energy(x[i]);
  return s;
}

double Drape::potential(const std::vector<Vec3>& x) const {
  double m = 0;
  for (auto& e : membranes) m += e.energy(x, material);
  double h = 0;
  for (auto& e : hinges) h += e.energy(x);
  double el = m + h;
  return has_contact() ? el + barrier_energy(x) : el;
}

std::vector<Vec3> Drape::potential_gradient(const std::vector<Vec3>& x) const {
  std::vector<Vec3> g(x.size(), Vec3{0, 0, 0});
  for (auto& e : membranes) {
    auto ge = e.gradient(x, material);
    for (int k = 0; k < 3; ++k)
      for (int d = 0; d < 3; ++d) g[e.vertices[k]][d] += ge[k][d];
  }
  if (has_contact())
    for (int i : free_) {
      auto c = contact.gradient(x[i]);
      for (int d = 0; d < 3; ++d) g[i][d] += c[d];
    }
  for (auto& h : hinges) {
    auto gh = h.gradient(x);
    for (int k = 0; k < 4; ++k)
      for (int d = 0; d < 3; ++d) g[h.vertices[k]][d] += gh[k][d];
  }
  return g;
}

// ---------------------------------------------------------------- drape step
double DrapeStep::value(const std::vector<Vec3>& x) const {
  double inertia = 0;
  for (int i : drape->free_) {
    Vec3 o = sub(x[i], x_hat[i]);
    inertia += 0.5 * drape->mass_over_h2(i) * dot(o, o);
  }
  return inertia + drape->potential(x);
}

std::vector<double> DrapeStep::residual(const std::vector<Vec3>& x) const {
  auto g = drape->potential_gradient(x);
  std::vector<double> r;
  r.reserve(3 * drape->free_.size());
  for (int i : drape->free_)
    for (int d = 0; d < 3; ++d) r.push_back(drape->mass_over_h2(i) * (x[i][d] - x_hat[i][d]) + g[i][d]);
  return r;
}

Bsr DrapeStep::tangent(const std::vector<Vec3>& x) const {
  const Drape& d = *drape;
  Bsr m = d.pattern;
  for (size_t row = 0; row < d.free_.size(); ++row) m.add(int(row), int(row), identity_scaled(d.mass_over_h2(d.free_[row])));
  for (auto& e : d.membranes)
    d.add_blocks(m, e.vertices, d.tangent_kind == TangentKind::Exact ? e.tangent(x, d.material) : e.hessian(x, d.material));
  for (auto& h : d.hinges) d.add_blocks(m, h.vertices, d.tangent_kind == TangentKind::Exact ? h.tangent(x) : h.hessian(x));
  if (d.has_contact())
    for (size_t row = 0; row < d.free_.size(); ++row)
      m.add(int(row), int(row), d.contact.hessian_with(x[d.free_[row]], d.barrier_curvature));
  return m;
}

Bsr DrapeStep::regularized_tangent(const std::vector<Vec3>& x, double mu) const {
  Bsr m = tangent(x);
  for (size_t row = 0; row < drape->free_.size(); ++row)
    m.add(int(row), int(row), identity_scaled(mu * drape->mass_over_h2(drape->free_[row])));
  return m;
}

double DrapeStep::barrier_change(const std::vector<Vec3>& x, const std::vector<Vec3>& d, double alpha) const {
  double s = 0;
  for (int i : drape->free_) s += drape->contact.energy(add(x[i], scale(d[i], alpha))) - drape->contact.energy(x[i]);
  return s;
}

double DrapeStep::energy_change(const std::vector<Vec3>& x, const std::vector<Vec3>& d, double alpha) const {
  const Drape& D = *drape;
  double inertia = 0;
  for (int i : D.free_) {
    Vec3 st = scale(d[i], alpha), o = sub(x[i], x_hat[i]);
    inertia += D.mass_over_h2(i) * (dot(o, st) + 0.5 * dot(st, st));
  }
  double membrane = 0;
  for (auto& e : D.membranes) membrane += e.energy_change(x, d, alpha, D.material);
  double hinge = 0;
  for (auto& h : D.hinges) hinge += h.energy_change(x, d, alpha);
  double el = inertia + membrane + hinge;
  return D.has_contact() ? el + barrier_change(x, d, alpha) : el;
}

std::vector<Vec3> DrapeStep::scatter(const std::vector<double>& rows) const {
  std::vector<Vec3> v(drape->mesh.rest.size(), Vec3{0, 0, 0});
  for (size_t row = 0; row < drape->free_.size(); ++row)
    v[drape->free_[row]] = {rows[3 * row], rows[3 * row + 1], rows[3 * row + 2]};
  return v;
}

std::vector<double> DrapeStep::gather(const std::vector<Vec3>& v) const {
  std::vector<double> r;
  for (int i : drape->free_) r.insert(r.end(), v[i].begin(), v[i].end());
  return r;
}

double DrapeStep::max_step(const std::vector<Vec3>& x, const std::vector<Vec3>& d) const {
  double a = 1.0;
  for (int i : drape->free_) a = std::min(a, drape->contact.max_step(x[i], d[i]));
  return a;
}

std::vector<double> DrapeStep::absolute_contributions(const std::vector<Vec3>& x) const {
  const Drape& D = *drape;
  std::vector<Vec3> sums(x.size(), Vec3{0, 0, 0});
  for (auto& e : D.membranes) {
    auto g = e.gradient(x, D.material);
    for (int k = 0; k < 3; ++k)
      for (int c = 0; c < 3; ++c) sums[e.vertices[k]][c] += std::fabs(g[k][c]);
  }
  for (auto& h : D.hinges) {
    auto g = h.gradient(x);
    for (int k = 0; k < 4; ++k)
      for (int c = 0; c < 3; ++c) sums[h.vertices[k]][c] += std::fabs(g[k][c]);
  }
  for (int i : D.free_) {
    auto g = D.contact.gradient(x[i]);
    for (int c = 0; c < 3; ++c) sums[i][c] += std::fabs(g[c]);
  }
  std::vector<double> out;
  for (int i : D.free_)
    for (int c = 0; c < 3; ++c) out.push_back(std::fabs(D.mass_over_h2(i) * (x[i][c] - x_hat[i][c])) + sums[i][c]);
  return out;
}

std::vector<Vec3> feasible_start(const DrapeStep& step, const std::vector<Vec3>& x) {
  std::vector<Vec3> towards(x.size());
  for (size_t i = 0; i < x.size(); ++i) towards[i] = sub(step.x_hat[i], x[i]);
  double alpha = step.max_step(x, towards);
  std::vector<Vec3> out(x.size());
  for (size_t i = 0; i < x.size(); ++i) out[i] = add(x[i], scale(towards[i], alpha));
  return out;
}

// ---------------------------------------------------------------- Newton
const char* status_name(StepStatus s) {
  switch (s) {
    case StepStatus::Converged: return "converged";
    case StepStatus::IterationLimit: return "iteration_limit";
    case StepStatus::LineSearchFailed: return "line_search_failed";
    case StepStatus::RegularizationCap: return "regularization_cap";
    case StepStatus::ConvergedAtFloor: return "converged_at_floor";
  }
  return "?";
}

static double free_dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}

int line_search(const DrapeStep& s, const std::vector<Vec3>& x, const std::vector<double>& g,
                const std::vector<Vec3>& d, const NewtonSettings& set, double* length) {
  double slope = free_dot(g, s.gather(d));
  if (!(slope < 0.0)) return -1;
  double start = s.max_step(x, d);
  for (int h = 0; h <= set.max_halvings; ++h) {
    double a = start * std::pow(0.5, h);
    if (s.energy_change(x, d, a) <= set.armijo * a * slope) {
      *length = a;
      return h;
    }
  }
  return -1;
}

// newton.rs:240-258: the first mu >= start whose shifted tangent gives a descent direction.
static bool regularized_direction(const DrapeStep& s, const std::vector<Vec3>& x, const std::vector<double>& g,
                                  double start, const DirectionSolver& dir, Regularization& rec,
                                  std::vector<Vec3>& out, double& used, int& pcg_its) {
  std::vector<double> neg(g.size());
  for (size_t i = 0; i < g.size(); ++i) neg[i] = -g[i];
  double mu = start;
  pcg_its = 0;
  for (;;) {
    rec.max_mu = std::max(rec.max_mu, mu);
    Bsr A = s.regularized_tangent(x, mu);
    bool ok = false;
    std::vector<double> rows;
    if (dir.pcg) {
      PcgSettings ps;
      ps.tolerance = dir.rtol;
      ps.max_iterations = dir.max_iterations;
      ps.history_stride = 0;
      ps.detect_breakdown = true;
      PcgReport rep = pcg_solve<double>(A, neg, ps);
      pcg_its += rep.iterations;
      ok = !rep.breakdown;
      rows = std::move(rep.solution);
    } else {
      BandCholesky f;
      ok = BandCholesky::factor(A, f);
      if (ok) rows = f.solve(neg);
    }
    if (ok) {
      out = s.scatter(rows);
      if (free_dot(g, s.gather(out)) < 0.0) {
        used = mu;
        return true;
      }
    }
    if (mu >= MU_CAP) {
      rec.cap_hit = true;
      return false;
    }
    mu = raise_mu(mu);
    rec.retries++;
  }
}

StepSolution solve_step_regularized(const DrapeStep& s, std::vector<Vec3> start, double scale_,
                                    const NewtonSettings& set, const DirectionSolver& dir) {
  StepSolution st;
  st.positions = std::move(start);
  double mu = 0.0;
  for (;;) {
    auto g = s.residual(st.positions);
    st.residuals.push_back(vector_norm(g) / scale_);
    if (st.residuals.back() <= set.tolerance) {
      st.status = StepStatus::Converged;
      return st;
    }
    if (int(st.halvings.size()) == set.max_iterations) return st;
    std::vector<Vec3> d;
    double used = 0;
    int its = 0;
    if (!regularized_direction(s, st.positions, g, mu, dir, st.regularization, d, used, its)) {
      st.status = StepStatus::RegularizationCap;
      return st;
    }
    double len = 0;
    int halvings = line_search(s, st.positions, g, d, set, &len);
    if (halvings < 0) {
      st.status = StepStatus::LineSearchFailed;
      return st;
    }
    for (size_t i = 0; i < st.positions.size(); ++i)
      for (int k = 0; k < 3; ++k) st.positions[i][k] += len * d[i][k];
    st.halvings.push_back(halvings);
    st.step_lengths.push_back(len);
    st.pcg_iterations.push_back(its);
    mu = halvings == 0 ? relax_mu(used) : used;
  }
}

// drape.rs:177-185 (x_hat = x + h v + h^2 g on free vertices, pinned ones stay), with this scene's gravity vector.
std::vector<Vec3> dynamic_prediction(const Drape& d, const std::vector<Vec3>& x, const std::vector<Vec3>& v, double h) {
  std::vector<Vec3> p = x;
  for (int i : d.free_)
    for (int k = 0; k < 3; ++k) p[i][k] = x[i][k] + h * v[i][k] + h * h * d.gravity[k];
  return p;
}

// drape.rs:410-417 with the regularised solver (the E4 scheme's; e3_generate.rs:46).
TimeStepResult time_step(const Drape& d, const std::vector<Vec3>& x, const std::vector<Vec3>& v, double h,
                         const NewtonSettings& set, const DirectionSolver& dir) {
  d.time_step = h;
  DrapeStep step{&d, dynamic_prediction(d, x, v, h)};
  TimeStepResult out;
  out.scale = vector_norm(step.residual(x));
  auto start = d.has_contact() ? feasible_start(step, x) : step.x_hat;
  out.solution = solve_step_regularized(step, start, out.scale, set, dir);
  out.velocity.resize(x.size());
  for (size_t i = 0; i < x.size(); ++i)
    for (int k = 0; k < 3; ++k) out.velocity[i][k] = (out.solution.positions[i][k] - x[i][k]) / h;
  return out;
}

// e4_rules.rs:15-44
double next_forcing(double previous, double ratio) {
  double eta = 0.9 * ratio * ratio, safeguard = 0.9 * previous * previous;
  double guarded = safeguard > 0.1 ? std::max(eta, safeguard) : eta;
  return std::min(std::max(guarded, 1e-7), 1e-2);
}

double f32_spacing(double max_abs) {
  float f = float(max_abs);
  uint32_t bits;
  std::memcpy(&bits, &f, 4);
  int exponent = int((bits >> 23) & 0xff);
  return std::ldexp(1.0, exponent - 127 - 23);
}

bool update_is_small(double update_inf, double step_inf, double resolution) {
  return update_inf <= std::max(1e-4 * step_inf, 2.0 * resolution);
}

// ---------------------------------------------------------------- PTC
double next_step_size(const PtcRules& r, double h, int inner) {
  double factor = r.controller == Controller::Doubling ? r.growth : (inner < r.inner_max ? r.growth : r.shrink);
  return std::min(std::max(h * factor, r.h0 * r.h_min_factor), r.h_max);
}

double gravity_load(const Drape& d) {
  double s = 0, g = d.g_norm();
  for (int i : d.free_) s += (d.mass[i] * g) * (d.mass[i] * g);
  return std::sqrt(s);
}

std::vector<double> static_gradient(const Drape& d, const std::vector<Vec3>& x) {
  auto g = d.potential_gradient(x);
  std::vector<double> out;
  for (int i : d.free_)
    for (int k = 0; k < 3; ++k) out.push_back(g[i][k] - d.mass[i] * d.gravity[k]);
  return out;
}

double static_energy(const Drape& d, const std::vector<Vec3>& x) {
  double s = 0;
  for (size_t i = 0; i < x.size(); ++i) s += -d.mass[i] * dot(d.gravity, x[i]);
  return d.potential(x) + s;
}

std::vector<Vec3> ptc_prediction(const Drape& d, const std::vector<Vec3>& x, double h) {
  std::vector<Vec3> p = x;
  for (int i : d.free_)
    for (int k = 0; k < 3; ++k) p[i][k] = x[i][k] + h * h * d.gravity[k];
  return p;
}

double static_floor(const Drape& d, const std::vector<Vec3>& x) {
  DrapeStep step{&d, x};
  auto contrib = step.absolute_contributions(x);
  for (size_t row = 0; row < d.free_.size(); ++row) {
    int i = d.free_[row];
    for (int k = 0; k < 3; ++k)
      contrib[3 * row + k] += d.mass[i] * std::fabs(d.gravity[k]) - std::fabs(d.mass_over_h2(i) * (x[i][k] - step.x_hat[i][k]));
  }
  Bsr t = step.tangent(x);
  for (size_t row = 0; row < d.free_.size(); ++row) t.add(int(row), int(row), identity_scaled(-d.mass_over_h2(d.free_[row])));
  for (auto& v : t.vals) v = std::fabs(v);
  auto ax = step.gather(x);
  for (auto& v : ax) v = std::fabs(v);
  auto stiff = t.multiply(ax);
  return std::numeric_limits<double>::epsilon() * (vector_norm(contrib) + vector_norm(stiff));
}

bool attempt_failed(StepStatus status, int iterations, const std::vector<Vec3>& positions) {
  bool stuck = iterations == 0 && (status == StepStatus::RegularizationCap || status == StepStatus::LineSearchFailed);
  if (stuck) return true;
  for (auto& p : positions)
    for (double v : p)
      if (!std::isfinite(v)) return true;
  return false;
}

static StepSolution inner_solve(const Drape& d, const std::vector<Vec3>& x, double h, double residual,
                                const PtcRules& rules, const DirectionSolver& dir) {
  d.time_step = h;
  DrapeStep sys{&d, ptc_prediction(d, x, h)};
  NewtonSettings set{rules.inner_tolerance, rules.inner_max, 1e-4, 30};
  return solve_step_regularized(sys, rules.predicted_start ? feasible_start(sys, x) : x, residual, set, dir);
}

static bool attempt(const Drape& d, const std::vector<Vec3>& x, double h, double residual, const PtcRules& rules,
                    const DirectionSolver& dir, std::vector<Vec3>& next, PtcStep& step) {
  StepSolution sol = inner_solve(d, x, h, residual, rules, dir);
  bool capped = sol.regularization.cap_hit && !sol.halvings.empty();
  if (capped) {
    d.barrier_curvature = false;
    sol = inner_solve(d, x, h, residual, rules, dir);
    d.barrier_curvature = true;
  }
  int its = int(sol.halvings.size());
  if (attempt_failed(sol.status, its, sol.positions)) return false;
  int pcg = 0;
  for (int p : sol.pcg_iterations) pcg += p;
  step = PtcStep{h, residual, its, 0, pcg, sol.regularization.max_mu, sol.regularization.cap_hit, capped};
  next = std::move(sol.positions);
  return true;
}

bool take_step(const Drape& d, const std::vector<Vec3>& x, double h, double residual, const PtcRules& rules,
               const DirectionSolver& dir, std::vector<Vec3>& next, PtcStep& step) {
  double size = h;
  for (int rejected = 0; rejected <= rules.max_rejections; ++rejected) {
    if (attempt(d, x, size, residual, rules, dir, next, step)) {
      step.rejected_attempts = rejected;
      return true;
    }
    size = std::max(size * rules.shrink, rules.h0 * rules.h_min_factor);
  }
  return false;
}

static const char* equilibrium_reason(const Drape& d, const std::vector<Vec3>& x, double residual, const PtcRules& r) {
  double load = gravity_load(d);
  if (r.absolute > 0.0 && residual <= r.absolute) return "tolerance";
  if (residual / load <= r.equilibrium) return "tolerance";
  if (r.floor_rule && residual / load <= r.floor_guard && residual <= r.floor_factor * static_floor(d, x)) return "floor";
  return nullptr;
}

PtcRun ptc_solve(const Drape& d, std::vector<Vec3> start, double h_start, const PtcRules& rules,
                 const DirectionSolver& dir, bool keep_states, bool progress) {
  double load = gravity_load(d);
  PtcRun run;
  run.final_h = h_start;
  run.states.push_back(std::move(start));
  std::vector<Vec3> x = run.states.back();
  auto t0 = std::chrono::steady_clock::now();
  int newton_total = 0;
  for (;;) {
    run.final_residual = vector_norm(static_gradient(d, x));
    double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (progress)
      std::fprintf(stderr, "state after %zu steps: residual %.6e N at %.3f s, %d Newton iterations\n", run.steps.size(),
                   run.final_residual, elapsed, newton_total);
    if (rules.time_budget_s > 0 && elapsed > rules.time_budget_s) {
      run.reason = "time_budget";
      break;
    }
    if (const char* reason = equilibrium_reason(d, x, run.final_residual, rules)) {
      run.reason = reason;
      break;
    }
    if (int(run.steps.size()) == rules.max_steps) break;
    double h = run.steps.empty() ? h_start : next_step_size(rules, run.steps.back().h, run.steps.back().inner_iterations);
    std::vector<Vec3> next;
    PtcStep step{};
    if (!take_step(d, x, h, run.final_residual, rules, dir, next, step)) {
      run.reason = "stalled";
      break;
    }
    if (progress)
      std::fprintf(stderr, "ptc step %zu h=%.3e r/L=%.3e inner=%d rejected=%d mu=%g pcg=%d\n", run.steps.size() + 1,
                   step.h, run.final_residual / load, step.inner_iterations, step.rejected_attempts, step.max_mu,
                   step.pcg_iterations);
    newton_total += step.inner_iterations;
    run.steps.push_back(step);
    x = std::move(next);
    if (keep_states)
      run.states.push_back(x);
  }
  if (!keep_states) run.states.push_back(x);
  run.final_h = run.steps.empty() ? h_start : next_step_size(rules, run.steps.back().h, run.steps.back().inner_iterations);
  return run;
}

// ---------------------------------------------------------------- kernel-check states
// e3_checks.rs:40-44's fold plus noise, applied on top of the scene's start state with the fold along the up
// axis (-gravity): the reference evaluated it on the contact-free pinned sheet lying at z = 0; placing it over the
// start state keeps every vertex of a contact scene outside its colliders (the barrier is checked separately at
// contact_state). The noise draws keep the reference's order (x, y, z per vertex).
std::vector<Vec3> bent_state(const Drape& d, Lcg& rng) {
  double w = d.mesh.width, h = d.mesh.height, s = d.mesh.width / (d.mesh.columns - 1);
  double gn = d.g_norm();
  Vec3 up{-d.gravity[0] / gn, -d.gravity[1] / gn, -d.gravity[2] / gn};
  std::vector<Vec3> x;
  for (size_t v = 0; v < d.mesh.rest.size(); ++v) {
    auto& p = d.mesh.rest[v];
    double a = 0.1 * s * rng.uniform();
    double b = 0.1 * s * rng.uniform();
    double fold = 0.05 * std::sin(M_PI * p[0] / w) * std::cos(2.0 * M_PI * p[1] / h);
    double c = 0.1 * s * rng.uniform();
    Vec3 base = d.start[v];
    x.push_back({base[0] + a + fold * up[0], base[1] + b + fold * up[1], base[2] + c + fold * up[2]});
  }
  return x;
}

// e5_checks.rs:60-78, written for any up axis (-gravity): vertices whose horizontal position lies within
// 0.6 r of a sphere's axis sit radially outside it, the rest above the first plane, at distances log-uniform
// in [0.05 d_hat, d_hat] drawn in vertex order from Lcg(131).
std::vector<Vec3> contact_state(const Drape& d) {
  Lcg rng(131);
  double dhat = d.contact.barrier.dhat;
  double g = d.g_norm();
  Vec3 up{-d.gravity[0] / g, -d.gravity[1] / g, -d.gravity[2] / g};
  std::vector<Vec3> out;
  for (size_t v = 0; v < d.mesh.rest.size(); ++v) {
    double dist = dhat * std::pow(0.05, 0.5 * (1.0 + rng.uniform()));
    Vec3 s = d.start[v];
    Vec3 hz = sub(s, scale(up, dot(s, up)));
    bool placed = false;
    Vec3 x{};
    for (auto& c : d.contact.colliders) {
      if (c.kind != 2) continue;
      Vec3 ch = sub(c.a, scale(up, dot(c.a, up)));
      Vec3 q = sub(hz, ch);
      double r2 = dot(q, q);
      if (std::sqrt(r2) >= 0.6 * c.w) continue;
      Vec3 n = add(scale(q, 1.0 / c.w), scale(up, std::sqrt(1.0 - r2 / (c.w * c.w))));
      x = add(c.a, scale(n, c.w + dist));
      placed = true;
      break;
    }
    if (!placed) {
      double offset = 0;
      for (auto& c : d.contact.colliders)
        if (c.kind == 1) {
          offset = c.w;
          break;
        }
      x = add(hz, scale(up, offset + dist));
    }
    out.push_back(x);
  }
  return out;
}

// ---------------------------------------------------------------- prolongation (e7_prolong.rs:9-47)
std::vector<Vec3> prolong(const std::vector<Vec3>& coarse, int cc) {
  int fc = 2 * (cc - 1) + 1;
  std::vector<Vec3> fine;
  for (int v = 0; v < fc * fc; ++v) {
    int i = v % fc, j = v / fc;
    int i0 = i / 2, i1 = (i + 1) / 2, j0 = j / 2, j1 = (j + 1) / 2;
    int corners[4][2] = {{i0, j0}, {i1, j0}, {i0, j1}, {i1, j1}};
    Vec3 s{0, 0, 0};
    for (auto& c : corners)
      for (int k = 0; k < 3; ++k) s[k] += coarse[c[1] * cc + c[0]][k];
    fine.push_back({s[0] / 4.0, s[1] / 4.0, s[2] / 4.0});
  }
  return fine;
}

int project_out(const Drape& d, std::vector<Vec3>& positions) {
  double dhat = d.contact.barrier.dhat;
  int moved = 0;
  for (auto& x : positions) {
    Vec3 before = x;
    for (auto& c : d.contact.colliders) {
      double dist = c.distance(x);
      if (dist < dhat) {
        Vec3 n = c.normal(x);
        for (int k = 0; k < 3; ++k) x[k] += (dhat - dist) * n[k];
      }
    }
    moved += (x != before);
  }
  return moved;
}

}  // namespace oracle
