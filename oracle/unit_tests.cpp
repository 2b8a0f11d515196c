// Test infrastructure only (see core.h). The reference crate's #[test] functions, restated against this
// oracle. Each is registered by name and run from tests/test_oracle_unit.py through the C API.
// Sources: membrane.rs:142-234, hinge.rs:122-207, dual.rs:92-103, contact.rs:179-234, pcg.rs:283-323,
// band.rs:105-118, cases.rs:163-197, newton.rs:286-341, drape.rs:441-489, e7_ptc.rs:191-243,
// e4_rules.rs:57-89, e5_checks.rs:208-247, e7_prolong.rs:66-81, jsonscan.rs:28-41.
// The coupon-based Newton tests (newton.rs: armijo, assembled derivatives) are restated on the pinned drape;
// the coupon patch/unloading tests and the Lanczos spectrum test belong to experiments E1/E2 outside this path.
#include <functional>
#include <sstream>

#include "cases.h"
#include "drape.h"
#include "io.h"

namespace oracle {
namespace {

struct Failure : std::runtime_error {
  using std::runtime_error::runtime_error;
};
#define CHECK(cond, msg)                                                          \
  do {                                                                            \
    if (!(cond)) {                                                                \
      std::ostringstream os_;                                                     \
      os_ << __LINE__ << ": " << #cond << " | " << msg;                           \
      throw Failure(os_.str());                                                   \
    }                                                                             \
  } while (0)

// testing.rs:4-37
std::vector<Vec3> random_positions(const std::vector<Vec2>& rest, Lcg& rng, double stretch, double noise) {
  std::vector<Vec3> x;
  for (auto& p : rest) {
    double a = stretch * p[0] + noise * rng.uniform();
    double b = p[1] + noise * rng.uniform();
    double c = noise * rng.uniform();
    x.push_back({a, b, c});
  }
  return x;
}
std::vector<Vec3> stretched(const std::vector<Vec2>& rest, double w, double c, Lcg& rng, double noise) {
  std::vector<Vec3> x;
  for (auto& p : rest) {
    double a = w * p[0] + noise * rng.uniform();
    double b = c * p[1] + noise * rng.uniform();
    double z = noise * rng.uniform();
    x.push_back({a, b, z});
  }
  return x;
}
template <class F> double central(const std::vector<Vec3>& x, int v, int axis, double h, F f) {
  auto p = x, m = x;
  p[v][axis] += h;
  m[v][axis] -= h;
  return (f(p) - f(m)) / (2.0 * h);
}
template <size_t N, class G>
std::array<Vec3, N> gradient_derivative(const std::vector<Vec3>& x, int v, int axis, double h, G g) {
  auto p = x, m = x;
  p[v][axis] += h;
  m[v][axis] -= h;
  auto gp = g(p), gm = g(m);
  std::array<Vec3, N> out;
  for (size_t k = 0; k < N; ++k)
    for (int r = 0; r < 3; ++r) out[k][r] = (gp[k][r] - gm[k][r]) / (2.0 * h);
  return out;
}

// ---------------------------------------------------------------- membrane
std::pair<MembraneElement, std::vector<Vec2>> sample_element() {
  std::vector<Vec2> rest{{0.0, 0.0}, {0.004, 0.0005}, {0.001, 0.0045}};
  return {MembraneElement::make({0, 1, 2}, rest), rest};
}
void membrane_rest_state_is_stress_free() {
  auto [e, rest] = sample_element();
  std::vector<Vec3> x;
  for (auto& p : rest) x.push_back({p[0], p[1], 0.0});
  auto g = e.gradient(x, Material::knit_baseline());
  for (auto& v : g)
    for (double c : v) CHECK(std::fabs(c) < 1e-14, c);
}
void membrane_gradient_matches_energy_finite_difference() {
  auto [e, rest] = sample_element();
  Material m = Material::knit_baseline();
  Lcg rng(7);
  auto x = random_positions(rest, rng, 1.15, 0.0008);
  auto g = e.gradient(x, m);
  for (int v = 0; v < 3; ++v)
    for (int d = 0; d < 3; ++d) {
      double fd = central(x, v, d, 1e-8, [&](const std::vector<Vec3>& y) { return e.energy(y, m); });
      CHECK(std::fabs(fd - g[v][d]) <= 1e-6 * (1.0 + std::fabs(g[v][d])), fd << " vs " << g[v][d]);
    }
}
void membrane_hessian_check(bool tension) {
  auto [e, rest] = sample_element();
  Material m = Material::knit_baseline();
  Lcg rng(tension ? 3 : 11);
  auto x = tension ? stretched(rest, 1.04, 1.07, rng, 1e-5) : stretched(rest, 0.93, 1.05, rng, 1e-5);
  auto H = tension ? e.hessian(x, m) : e.tangent(x, m);
  for (int l = 0; l < 3; ++l)
    for (int d = 0; d < 3; ++d) {
      auto fd = gradient_derivative<3>(x, l, d, 1e-8, [&](const std::vector<Vec3>& y) { return e.gradient(y, m); });
      for (int k = 0; k < 3; ++k)
        for (int r = 0; r < 3; ++r) {
          double ex = H[k][l][r][d];
          CHECK(std::fabs(fd[k][r] - ex) <= 1e-5 * (1.0 + std::fabs(ex)), k << l << r << d);
        }
    }
}
void membrane_hessian_matches_gradient_finite_difference_in_tension() { membrane_hessian_check(true); }
void membrane_exact_tangent_matches_gradient_finite_difference_in_compression() { membrane_hessian_check(false); }
void membrane_energy_change_equals_energy_difference() {
  auto [e, rest] = sample_element();
  Material m = Material::knit_baseline();
  Lcg r5(5), r6(6);
  auto x = random_positions(rest, r5, 1.1, 0.0005);
  auto d = random_positions(rest, r6, 0.0, 0.0003);
  std::vector<Vec3> moved;
  for (size_t i = 0; i < x.size(); ++i) moved.push_back(add(x[i], scale(d[i], 0.7)));
  double direct = e.energy(moved, m) - e.energy(x, m);
  double change = e.energy_change(x, d, 0.7, m);
  CHECK(std::fabs(direct - change) <= 1e-12 * std::max(std::fabs(direct), e.energy(x, m)), direct << " vs " << change);
}
void membrane_rigid_rotation_is_stress_free() {
  auto [e, rest] = sample_element();
  double c = 0.6, s = 0.8;
  std::vector<Vec3> x;
  for (auto& p : rest) x.push_back({c * p[0] - s * p[1], s * p[0] + c * p[1], 0.3});
  for (double v : e.strain(x)) CHECK(std::fabs(v) < 1e-13, v);
}

// ---------------------------------------------------------------- hinge
std::pair<HingeElement, std::vector<Vec3>> bent_hinge(double height) {
  return {HingeElement{{0, 1, 2, 3}, 1.3}, {{0.5, 0.9, height}, {0.45, -1.1, -0.2 * height}, {0, 0, 0}, {1.0, 0.05, 0.0}}};
}
void hinge_flat_hinge_has_zero_angle() {
  auto [h, x] = bent_hinge(0.0);
  CHECK(std::fabs(h.angle(x)) < 1e-14, h.angle(x));
}
void hinge_angle_gradient_matches_finite_difference() {
  auto [h, x] = bent_hinge(0.4);
  auto g = h.angle_gradient(x);
  for (int v = 0; v < 4; ++v)
    for (int d = 0; d < 3; ++d) {
      double fd = central(x, v, d, 1e-7, [&](const std::vector<Vec3>& y) { return h.angle(y); });
      CHECK(std::fabs(fd - g[v][d]) < 1e-6, fd << " vs " << g[v][d]);
    }
}
void hinge_generic_angle_gradient_matches_the_f64_one() {
  auto [h, x] = bent_hinge(0.4);
  std::array<V3<Dual>, 4> p;
  for (int k = 0; k < 4; ++k)
    for (int d = 0; d < 3; ++d) p[k][d] = Dual{x[k][d], 0.0};
  auto gd = angle_gradient_of<Dual>(p);
  auto g = h.angle_gradient(x);
  for (int k = 0; k < 4; ++k)
    for (int d = 0; d < 3; ++d) CHECK(gd[k][d].v == g[k][d], k << d);
}
void hinge_exact_tangent_matches_gradient_finite_difference_when_bent() {
  auto [h, x] = bent_hinge(0.4);
  auto t = h.tangent(x);
  for (int l = 0; l < 4; ++l)
    for (int d = 0; d < 3; ++d) {
      auto fd = gradient_derivative<4>(x, l, d, 1e-7, [&](const std::vector<Vec3>& y) { return h.gradient(y); });
      for (int k = 0; k < 4; ++k)
        for (int r = 0; r < 3; ++r) {
          double ex = t[k][l][r][d];
          CHECK(std::fabs(fd[k][r] - ex) < 1e-6 * (1.0 + std::fabs(ex)), k << l << r << d);
        }
    }
}
void hinge_angle_hessian_is_symmetric() {
  auto [h, x] = bent_hinge(0.3);
  auto H = h.angle_hessian(x);
  for (int k = 0; k < 4; ++k)
    for (int l = 0; l < 4; ++l)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) CHECK(std::fabs(H[k][l][r][c] - H[l][k][c][r]) < 1e-10, k << l << r << c);
}
void hinge_energy_change_equals_energy_difference() {
  auto [h, x] = bent_hinge(0.4);
  std::vector<Vec3> d{{0.01, -0.02, 0.03}, {0.0, 0.01, -0.02}, {0.005, 0.0, 0.01}, {-0.01, 0.02, 0.0}};
  std::vector<Vec3> moved;
  for (int i = 0; i < 4; ++i) moved.push_back(add(x[i], scale(d[i], 0.6)));
  double direct = h.energy(moved) - h.energy(x);
  CHECK(std::fabs(h.energy_change(x, d, 0.6) - direct) < 1e-14, direct);
}
void hinge_gauss_newton_hessian_is_exact_at_flat_state() {
  auto [h, x] = bent_hinge(0.0);
  auto H = h.hessian(x);
  for (int l = 0; l < 4; ++l)
    for (int d = 0; d < 3; ++d) {
      auto fd = gradient_derivative<4>(x, l, d, 1e-7, [&](const std::vector<Vec3>& y) { return h.gradient(y); });
      for (int k = 0; k < 4; ++k)
        for (int r = 0; r < 3; ++r) CHECK(std::fabs(fd[k][r] - H[k][l][r][d]) < 1e-5, k << l << r << d);
    }
}

// ---------------------------------------------------------------- dual
void dual_derivatives_match_calculus() {
  Dual x{2.0, 1.0};
  Dual y = (x * x + constant<Dual>(3.0)) / dsqrt(x);
  double exact = (2.0 * 2.0 * std::sqrt(2.0) - (4.0 + 3.0) / (2.0 * std::sqrt(2.0))) / 2.0;
  CHECK(std::fabs(y.t - exact) < 1e-14, y.t << " vs " << exact);
}

// ---------------------------------------------------------------- contact
Contact test_contact() {
  Contact c;
  c.colliders = {Collider::plane({0, 0, 1}, 0.0), Collider::sphere({0.25, 0.25, 0.125}, 0.125)};
  c.barrier = Barrier{5e-4, 2.0};
  return c;
}
void contact_barrier_derivatives_match_finite_differences() {
  Barrier b{5e-4, 3.0};
  for (double d : {3e-5, 1e-4, 2.5e-4, 4.9e-4}) {
    double h = 1e-9;
    double first = (b.value(d + h) - b.value(d - h)) / (2 * h), second = (b.first(d + h) - b.first(d - h)) / (2 * h);
    CHECK(std::fabs(first - b.first(d)) <= 1e-6 * std::fabs(b.first(d)), d);
    CHECK(std::fabs(second - b.second(d)) <= 1e-6 * std::fabs(b.second(d)), d);
  }
}
void contact_resting_kappa_balances_gravity_at_half_dhat() {
  double kappa = Barrier::resting_kappa(5e-4, 2e-5, 9.81);
  CHECK(std::fabs(Barrier{5e-4, kappa}.first(2.5e-4) + 2e-5 * 9.81) < 1e-18, kappa);
}
void contact_gradient_and_hessian_match_finite_differences() {
  auto c = test_contact();
  Vec3 x{0.27, 0.24, 0.2502};
  double h = 1e-9;
  for (int k = 0; k < 3; ++k) {
    Vec3 p = x, m = x;
    p[k] += h;
    m[k] -= h;
    double fd = (c.energy(p) - c.energy(m)) / (2 * h);
    CHECK(std::fabs(fd - c.gradient(x)[k]) <= 1e-6 * std::max(std::fabs(c.gradient(x)[k]), 1e-9), k);
    for (int i = 0; i < 3; ++i) {
      double col = (c.gradient(p)[i] - c.gradient(m)[i]) / (2 * h);
      CHECK(std::fabs(col - c.hessian(x)[i][k]) <= 1e-5 * std::fabs(c.hessian(x)[k][k]), i << k);
    }
  }
}
void contact_max_step_keeps_a_tenth_of_the_distance() {
  auto c = test_contact();
  Vec3 x{0.4, 0.4, 2e-4};
  double a = c.max_step(x, {0, 0, -1e-3});
  CHECK(std::fabs(x[2] - a * 1e-3 - 2e-5) < 1e-15, a);
  Vec3 top{0.25, 0.25, 0.25 + 1e-4};
  double b = c.max_step(top, {0, 0, -1e-3});
  CHECK(std::fabs(c.colliders[1].distance({0.25, 0.25, top[2] - b * 1e-3}) - 1e-5) < 1e-14, b);
  CHECK(c.max_step(top, {0, 0, 1e-3}) == 1.0, "");
}

// ---------------------------------------------------------------- pcg / band / cases
void pcg_f64_pcg_matches_cholesky_on_tension_case() {
  auto p = build_case(CaseKind::Tension, 13);
  BandCholesky f;
  CHECK(BandCholesky::factor(p.matrix, f), "factor");
  auto exact = f.solve(p.rhs);
  PcgSettings s;
  s.tolerance = 1e-12;
  s.max_iterations = 5000;
  auto rep = pcg_solve<double>(p.matrix, p.rhs, s);
  CHECK(rep.converged, "");
  double err = difference_norm(rep.solution, exact) / vector_norm(exact);
  CHECK(err < 1e-9, err);
}
void pcg_residual_replacement_keeps_f32_pcg_on_the_true_residual() {
  auto p = build_case(CaseKind::Tension, 33);
  auto settings = [](int every) {
    PcgSettings s;
    s.tolerance = 1e-7;
    s.max_iterations = 5000;
    s.replace_every = every;
    s.replace_above = 1e-2;
    return s;
  };
  auto true_res = [&](const PcgReport& r) {
    return difference_norm(p.matrix.multiply(r.solution), p.rhs) / vector_norm(p.rhs);
  };
  auto plain = pcg_solve<float>(p.matrix, p.rhs, settings(0));
  auto replaced = pcg_solve<float>(p.matrix, p.rhs, settings(10));
  CHECK(replaced.converged, "");
  CHECK(true_res(replaced) < true_res(plain), true_res(replaced) << " vs " << true_res(plain));
}
void pcg_inverse_times_matrix_is_identity() {
  double m[9] = {4.0, 1.0, 0.5, 1.0, 3.0, 0.2, 0.5, 0.2, 2.0};
  auto inv = invert3<double>(m);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double v = 0;
      for (int k = 0; k < 3; ++k) v += m[3 * r + k] * inv[3 * k + c];
      CHECK(std::fabs(v - (r == c ? 1.0 : 0.0)) < 1e-14, r << c);
    }
}
void band_cholesky_solves_tension_case() {
  auto p = build_case(CaseKind::Tension, 11);
  BandCholesky f;
  CHECK(BandCholesky::factor(p.matrix, f), "");
  auto x = f.solve(p.rhs);
  double res = difference_norm(p.matrix.multiply(x), p.rhs) / vector_norm(p.rhs);
  CHECK(res < 1e-12, res);
}
void cases_assembled_matrices_are_symmetric() {
  for (auto k : {CaseKind::Tension, CaseKind::Slack, CaseKind::Dynamic}) {
    auto p = build_case(k, 9);
    CHECK(p.matrix.asymmetry() < 1e-12, int(k));
  }
}
void cases_uniform_prestretch_has_no_interior_force() {
  Mesh mesh = Mesh::grid(7, 7, 0.5, 0.5);
  Material m = Material::knit_baseline();
  std::vector<Vec3> x;
  for (auto& p : mesh.rest) x.push_back({1.03 * p[0], 1.08 * p[1], 0.0});
  std::vector<Vec3> force(mesh.rest.size(), Vec3{0, 0, 0});
  for (auto& t : mesh.triangles) {
    auto g = MembraneElement::make(t, mesh.rest).gradient(x, m);
    for (int k = 0; k < 3; ++k)
      for (int d = 0; d < 3; ++d) force[t[k]][d] += g[k][d];
  }
  for (int v = 0; v < int(mesh.rest.size()); ++v)
    if (!mesh.is_boundary(v))
      for (double f : force[v]) CHECK(std::fabs(f) < 1e-12, f);
}
void cases_material_is_convex() { CHECK(Material::knit_baseline().is_convex(), ""); }

// ---------------------------------------------------------------- newton (restated on the pinned drape)
void newton_regularization_schedule_rises_tenfold_from_start_and_relaxes_to_zero() {
  CHECK(raise_mu(0.0) == MU_START, "");
  CHECK(raise_mu(MU_START) == 10.0 * MU_START, "");
  CHECK(raise_mu(500.0) == MU_CAP, "");
  CHECK(std::fabs(relax_mu(0.1) - 0.01) < 1e-18, "");
  CHECK(relax_mu(MU_START) == 0.0, "");
  CHECK(relax_mu(0.0) == 0.0, "");
}
void newton_armijo_backtracks_an_overlong_newton_step() {
  Drape d(pinned_scene(9), TangentKind::Projected);
  std::vector<Vec3> v(d.start.size(), Vec3{0, 0, 0});
  DrapeStep step{&d, d.start};
  for (int i : d.free_) step.x_hat[i][2] += d.time_step * d.time_step * -9.81;
  auto x = d.start;
  auto g = step.residual(x);
  BandCholesky f;
  CHECK(BandCholesky::factor(step.tangent(x), f), "");
  std::vector<double> neg(g.size());
  for (size_t i = 0; i < g.size(); ++i) neg[i] = -4.0 * g[i];
  auto dir = step.scatter(f.solve(neg));
  NewtonSettings set{1e-12, 30, 1e-4, 30};
  double len = 0;
  int halvings = line_search(step, x, g, dir, set, &len);
  CHECK(halvings >= 1, halvings);
  double slope = 0;
  auto rows = step.gather(dir);
  for (size_t i = 0; i < g.size(); ++i) slope += g[i] * rows[i];
  CHECK(step.energy_change(x, dir, len) <= 1e-4 * len * slope, len);
}
void newton_assembled_derivatives_match_finite_differences() {
  Drape d(pinned_scene(9), TangentKind::Exact);
  Lcg rng(97);
  auto x = bent_state(d, rng);
  DrapeStep step{&d, d.start};
  auto g = step.residual(x);
  Bsr K = step.tangent(x);
  Lcg r2(5);
  std::vector<Vec3> v(x.size(), Vec3{0, 0, 0});
  for (int i : d.free_) v[i] = {r2.uniform(), r2.uniform(), r2.uniform()};
  double h = 1e-7;
  auto shifted = [&](double s) {
    auto y = x;
    for (size_t i = 0; i < y.size(); ++i) y[i] = add(y[i], scale(v[i], s));
    return y;
  };
  double fd = (step.value(shifted(h)) - step.value(shifted(-h))) / (2 * h);
  auto rows = step.gather(v);
  double exact = 0;
  for (size_t i = 0; i < g.size(); ++i) exact += g[i] * rows[i];
  CHECK(std::fabs(fd - exact) / std::fabs(exact) < 1e-6, fd << " vs " << exact);
  auto gp = step.residual(shifted(h)), gm = step.residual(shifted(-h));
  auto kv = K.multiply(rows);
  double num = 0, den = 0;
  for (size_t i = 0; i < g.size(); ++i) {
    double c = (gp[i] - gm[i]) / (2 * h);
    num += (c - kv[i]) * (c - kv[i]);
    den += kv[i] * kv[i];
  }
  CHECK(std::sqrt(num / den) < 1e-5, std::sqrt(num / den));
  double alpha = 0.7;
  double change = step.energy_change(x, v, 1e-4 * alpha), direct = step.value(shifted(1e-4 * alpha)) - step.value(x);
  CHECK(std::fabs(change - direct) <= 1e-9 * std::fabs(direct) + 1e-18, change << " vs " << direct);
}

// ---------------------------------------------------------------- drape
// newton.rs:128-149 plain Newton with band Cholesky, the dynamic drape's time step (drape.rs:410-439).
std::vector<Vec3> plain_step(const DrapeStep& s, std::vector<Vec3> x, double scale_, const NewtonSettings& set) {
  for (int it = 0;; ++it) {
    auto g = s.residual(x);
    if (vector_norm(g) / scale_ <= set.tolerance || it == set.max_iterations) return x;
    BandCholesky f;
    if (!BandCholesky::factor(s.tangent(x), f)) throw Failure("not positive definite");
    std::vector<double> neg(g.size());
    for (size_t i = 0; i < g.size(); ++i) neg[i] = -g[i];
    auto dir = s.scatter(f.solve(neg));
    double len = 0;
    if (line_search(s, x, g, dir, set, &len) < 0) return x;
    for (size_t i = 0; i < x.size(); ++i) x[i] = add(x[i], scale(dir[i], len));
  }
}
void drape_residual_is_the_gradient_of_the_incremental_potential() {
  Drape d(pinned_scene(7), TangentKind::Exact);
  auto x = d.start;
  std::vector<Vec3> v;
  for (size_t i = 0; i < x.size(); ++i) v.push_back({0.1 * double(i % 3), -0.05, 0.2});
  DrapeStep step{&d, x};
  double h = d.time_step;
  for (int i : d.free_)
    for (int k = 0; k < 3; ++k) step.x_hat[i][k] = x[i][k] + h * v[i][k] + h * h * d.gravity[k];
  auto y = x;
  for (size_t k = 0; k < d.free_.size(); ++k) y[d.free_[k]][2] += 1e-3 * (double(k % 5) - 2.0);
  auto r = step.residual(y);
  for (size_t row = 0; row < d.free_.size(); row += 4)
    for (int c = 0; c < 3; ++c) {
      double fd = central(y, d.free_[row], c, 1e-7, [&](const std::vector<Vec3>& z) { return step.value(z); });
      double ex = r[3 * row + c];
      CHECK(std::fabs(fd - ex) <= 1e-6 * (1.0 + std::fabs(ex)), row << c << ": " << fd << " vs " << ex);
    }
}
void drape_feasible_start_keeps_a_tenth_of_every_collider_distance() {
  Drape d(reference_scene(9, "e5"), TangentKind::Exact);
  std::vector<Vec3> x;
  for (auto& p : d.start) x.push_back({p[0], p[1], 0.2501});
  DrapeStep step{&d, x};
  double h = d.time_step;
  for (int i : d.free_) step.x_hat[i] = {x[i][0], x[i][1], x[i][2] + h * -2.0 + h * h * -9.81};
  auto s = feasible_start(step, x);
  double kept = INFINITY;
  for (int i : d.free_) kept = std::min(kept, d.contact.min_distance(s[i]) / d.contact.min_distance(x[i]));
  CHECK(std::fabs(kept - 0.1) < 1e-9, kept);
}
void drape_first_step_falls_by_h_squared_g_and_energy_decreases() {
  Drape d(pinned_scene(9), TangentKind::Projected);
  double h = d.time_step;
  std::vector<std::vector<Vec3>> xs{d.start}, vs{std::vector<Vec3>(d.start.size(), Vec3{0, 0, 0})};
  NewtonSettings set{1e-10, 30, 1e-4, 30};
  for (int n = 0; n < 3; ++n) {
    DrapeStep step{&d, xs.back()};
    for (int i : d.free_)
      for (int k = 0; k < 3; ++k) step.x_hat[i][k] = xs.back()[i][k] + h * vs.back()[i][k] + h * h * d.gravity[k];
    double sc = vector_norm(step.residual(xs.back()));
    auto next = plain_step(step, step.x_hat, sc, set);
    std::vector<Vec3> vel;
    for (size_t i = 0; i < next.size(); ++i) vel.push_back(scale(sub(next[i], xs.back()[i]), 1.0 / h));
    xs.push_back(next);
    vs.push_back(vel);
  }
  int centre = int(d.mesh.rest.size()) / 2;
  double drop = xs[1][centre][2];
  CHECK(std::fabs(drop + h * h * 9.81) < 1e-6, drop);
  std::vector<double> e;
  for (int n = 0; n < 4; ++n) {
    double kin = 0, grav = 0;
    for (size_t i = 0; i < xs[n].size(); ++i) {
      kin += 0.5 * d.mass[i] * dot(vs[n][i], vs[n][i]);
      grav += d.mass[i] * 9.81 * xs[n][i][2];
    }
    e.push_back(kin + grav + d.potential(xs[n]));
  }
  for (int n = 0; n < 3; ++n) CHECK(e[n + 1] <= e[n], e[n + 1] << " > " << e[n]);
}

// ---------------------------------------------------------------- PTC
void ptc_step_size_doubles_below_the_inner_cap_halves_at_it_and_is_clamped() {
  PtcRules r = PtcRules::reference();
  CHECK(next_step_size(r, 0.01, 3) == 0.02, "");
  CHECK(next_step_size(r, 0.01, r.inner_max) == 0.005, "");
  CHECK(next_step_size(r, 0.9, 1) == r.h_max, "");
  CHECK(next_step_size(r, r.h0 * r.h_min_factor, r.inner_max) == r.h0 * r.h_min_factor, "");
}
void ptc_the_start_of_a_step_residual_is_the_static_residual() {
  Drape d(reference_scene(9, "e5"), TangentKind::Exact);
  std::vector<Vec3> x;
  for (auto& p : d.start) x.push_back({p[0], p[1], p[2] + 0.002 * std::sin(p[0] * 31.0)});
  d.time_step = 0.05;
  DrapeStep sys{&d, ptc_prediction(d, x, 0.05)};
  auto dyn = sys.residual(x);
  auto st = static_gradient(d, x);
  for (size_t i = 0; i < dyn.size(); ++i) CHECK(std::fabs(dyn[i] - st[i]) <= 1e-12 * (1.0 + std::fabs(st[i])), i);
}
void ptc_a_ptc_step_never_raises_the_static_energy() {
  Drape d(reference_scene(9, "e5"), TangentKind::Exact);
  PtcRules r = PtcRules::reference();
  DirectionSolver dir;
  std::vector<std::vector<Vec3>> states{d.start};
  double h = r.h0;
  for (int n = 0; n < 6; ++n) {
    auto x = states.back();
    double res = vector_norm(static_gradient(d, x));
    std::vector<Vec3> next;
    PtcStep step{};
    CHECK(take_step(d, x, h, res, r, dir, next, step), "a step can be taken");
    h = next_step_size(r, step.h, step.inner_iterations);
    states.push_back(next);
  }
  for (size_t n = 0; n + 1 < states.size(); ++n)
    CHECK(static_energy(d, states[n + 1]) <= static_energy(d, states[n]) + 1e-15, n);
}
void ptc_a_failed_attempt_is_a_regularisation_failure_before_any_update_or_a_non_finite_state() {
  std::vector<Vec3> finite{{0, 0, 0}};
  CHECK(attempt_failed(StepStatus::RegularizationCap, 0, finite), "");
  CHECK(!attempt_failed(StepStatus::RegularizationCap, 2, finite), "");
  CHECK(!attempt_failed(StepStatus::Converged, 0, finite), "");
  CHECK(attempt_failed(StepStatus::Converged, 3, {{NAN, 0, 0}}), "");
}

// ---------------------------------------------------------------- e4 rules
std::vector<double> forcing_sequence(const std::vector<double>& norms) {
  std::vector<double> etas;
  double eta = 1e-2;
  for (size_t k = 0; k < norms.size(); ++k) {
    if (k > 0) eta = next_forcing(eta, norms[k] / norms[k - 1]);
    etas.push_back(eta);
  }
  return etas;
}
void e4_forcing_starts_at_its_maximum_and_follows_the_squared_residual_ratio() {
  auto e = forcing_sequence({1.0, 1e-1, 1e-3, 1e-6});
  CHECK(e[0] == 1e-2, e[0]);
  CHECK(std::fabs(e[1] - 9e-3) < 1e-15, e[1]);
  CHECK(std::fabs(e[2] - 9e-5) < 1e-17, e[2]);
  CHECK(std::fabs(e[3] - 9e-7) < 1e-19, e[3]);
}
void e4_forcing_is_clamped_to_its_interval() {
  CHECK(next_forcing(1e-2, 0.9) == 1e-2, "");
  CHECK(next_forcing(1e-2, 1e-6) == 1e-7, "");
}
void e4_update_rule_compares_with_the_step_taken() {
  CHECK(update_is_small(1e-9, 1e-4, 0.0), "");
  CHECK(!update_is_small(2e-8, 1e-4, 0.0), "");
  CHECK(update_is_small(1e-7, 1e-4, f32_spacing(0.5)), "");
}
void e4_f32_spacing_reads_the_binade() {
  CHECK(f32_spacing(0.5) == std::ldexp(1.0, -24), "");
  CHECK(f32_spacing(0.49999997) == std::ldexp(1.0, -25), "");
  CHECK(f32_spacing(1.0) == std::ldexp(1.0, -23), "");
}

// ---------------------------------------------------------------- e5 checks
void e5_contact_state_puts_every_vertex_inside_the_barrier_on_both_colliders() {
  Drape d(reference_scene(9, "e5"), TangentKind::Exact);
  auto x = contact_state(d);
  double dhat = d.contact.barrier.dhat;
  int sphere = 0, floor = 0;
  for (int i : d.free_) {
    double m = d.contact.min_distance(x[i]);
    CHECK(m >= 0.05 * dhat * 0.999 && m < dhat, m);
    sphere += d.contact.colliders[1].distance(x[i]) < dhat;
    floor += d.contact.colliders[0].distance(x[i]) < dhat;
  }
  CHECK(sphere > 0 && floor > 0, sphere << " " << floor);
}
void e5_active_barrier_derivatives_match_finite_differences() {
  Drape d(reference_scene(9, "e5"), TangentKind::Exact);
  auto x = contact_state(d);
  DrapeStep step{&d, x};
  // Errors are taken relative to the largest gradient / Hessian diagonal over the checked vertices, the analogue
  // of the reference's directional check over a patch: near d = d_hat b' vanishes quadratically while the FD
  // truncation term does not, so a per-vertex relative error there measures the FD step, not the derivative.
  double worst_g = 0, worst_h = 0, gmax = 0, hmax = 0;
  for (size_t row = 0; row < d.free_.size(); row += 3) {
    auto g = d.contact.gradient(x[d.free_[row]]);
    auto H = d.contact.hessian(x[d.free_[row]]);
    gmax = std::max(gmax, norm(g));
    for (int k = 0; k < 3; ++k) hmax = std::max(hmax, std::fabs(H[k][k]));
  }
  for (size_t row = 0; row < d.free_.size(); row += 3) {
    int i = d.free_[row];
    double h = 1e-3 * d.contact.min_distance(x[i]);
    auto g = d.contact.gradient(x[i]);
    auto H = d.contact.hessian(x[i]);
    for (int k = 0; k < 3; ++k) {
      Vec3 p = x[i], m = x[i];
      p[k] += h;
      m[k] -= h;
      double fd = (d.contact.energy(p) - d.contact.energy(m)) / (2 * h);
      worst_g = std::max(worst_g, std::fabs(fd - g[k]) / gmax);
      for (int r = 0; r < 3; ++r) {
        double col = (d.contact.gradient(p)[r] - d.contact.gradient(m)[r]) / (2 * h);
        worst_h = std::max(worst_h, std::fabs(col - H[r][k]) / hmax);
      }
    }
  }
  CHECK(worst_g <= 1e-6, worst_g);
  CHECK(worst_h <= 1e-5, worst_h);
}

// ---------------------------------------------------------------- prolong / jsonscan
void e7_prolongation_copies_coarse_vertices_and_averages_the_rest() {
  std::vector<Vec3> coarse;
  for (int v = 0; v < 9; ++v) coarse.push_back({double(v % 3), double(v / 3), double((v % 3) * (v / 3))});
  auto fine = prolong(coarse, 3);
  CHECK(fine.size() == 25, fine.size());
  CHECK(fine[0] == coarse[0], "");
  CHECK(fine[2] == coarse[1], "");
  CHECK((fine[1] == Vec3{0.5, 0.0, 0.0}), "");
  CHECK((fine[6] == Vec3{0.5, 0.5, 0.25}), "");
  CHECK((fine[18] == Vec3{1.5, 1.5, 2.25}), "");
}
void jsonscan_reads_nested_and_spaced_values() {
  std::string t = "{\"a\": {\"iterations\": 7}, \"b\": {\"iterations\": 9, \"gpu_ms\": null, \"name\": \"x, y\"}, \"ok\": true}";
  CHECK(json_number(t, "b", "iterations") == 9.0, "");
  CHECK(json_number(t, "", "iterations") == 7.0, "");
  CHECK(std::isnan(json_number(t, "", "gpu_ms")), "");
  CHECK(json_string(t, "", "name") == "x, y", "");
  CHECK(json_flag(t, "", "ok"), "");
}

const std::vector<std::pair<const char*, void (*)()>>& registry() {
  static const std::vector<std::pair<const char*, void (*)()>> r = {
#define T(f) {#f, &f}
      T(membrane_rest_state_is_stress_free),
      T(membrane_gradient_matches_energy_finite_difference),
      T(membrane_hessian_matches_gradient_finite_difference_in_tension),
      T(membrane_exact_tangent_matches_gradient_finite_difference_in_compression),
      T(membrane_energy_change_equals_energy_difference),
      T(membrane_rigid_rotation_is_stress_free),
      T(hinge_flat_hinge_has_zero_angle),
      T(hinge_angle_gradient_matches_finite_difference),
      T(hinge_generic_angle_gradient_matches_the_f64_one),
      T(hinge_exact_tangent_matches_gradient_finite_difference_when_bent),
      T(hinge_angle_hessian_is_symmetric),
      T(hinge_energy_change_equals_energy_difference),
      T(hinge_gauss_newton_hessian_is_exact_at_flat_state),
      T(dual_derivatives_match_calculus),
      T(contact_barrier_derivatives_match_finite_differences),
      T(contact_resting_kappa_balances_gravity_at_half_dhat),
      T(contact_gradient_and_hessian_match_finite_differences),
      T(contact_max_step_keeps_a_tenth_of_the_distance),
      T(pcg_f64_pcg_matches_cholesky_on_tension_case),
      T(pcg_residual_replacement_keeps_f32_pcg_on_the_true_residual),
      T(pcg_inverse_times_matrix_is_identity),
      T(band_cholesky_solves_tension_case),
      T(cases_assembled_matrices_are_symmetric),
      T(cases_uniform_prestretch_has_no_interior_force),
      T(cases_material_is_convex),
      T(newton_regularization_schedule_rises_tenfold_from_start_and_relaxes_to_zero),
      T(newton_armijo_backtracks_an_overlong_newton_step),
      T(newton_assembled_derivatives_match_finite_differences),
      T(drape_residual_is_the_gradient_of_the_incremental_potential),
      T(drape_feasible_start_keeps_a_tenth_of_every_collider_distance),
      T(drape_first_step_falls_by_h_squared_g_and_energy_decreases),
      T(ptc_step_size_doubles_below_the_inner_cap_halves_at_it_and_is_clamped),
      T(ptc_the_start_of_a_step_residual_is_the_static_residual),
      T(ptc_a_ptc_step_never_raises_the_static_energy),
      T(ptc_a_failed_attempt_is_a_regularisation_failure_before_any_update_or_a_non_finite_state),
      T(e4_forcing_starts_at_its_maximum_and_follows_the_squared_residual_ratio),
      T(e4_forcing_is_clamped_to_its_interval),
      T(e4_update_rule_compares_with_the_step_taken),
      T(e4_f32_spacing_reads_the_binade),
      T(e5_contact_state_puts_every_vertex_inside_the_barrier_on_both_colliders),
      T(e5_active_barrier_derivatives_match_finite_differences),
      T(e7_prolongation_copies_coarse_vertices_and_averages_the_rest),
      T(jsonscan_reads_nested_and_spaced_values),
#undef T
  };
  return r;
}

thread_local std::string g_message;

}  // namespace
}  // namespace oracle

extern "C" {
int oracle_unit_test_count() { return int(oracle::registry().size()); }
const char* oracle_unit_test_name(int i) { return oracle::registry().at(size_t(i)).first; }
// 0 = pass, 1 = fail (message from oracle_unit_test_message), -1 = unknown name.
int oracle_unit_test_run(const char* name) {
  for (auto& [n, f] : oracle::registry())
    if (std::string(n) == name) {
      try {
        f();
        oracle::g_message.clear();
        return 0;
      } catch (const std::exception& e) {
        oracle::g_message = e.what();
        return 1;
      }
    }
  return -1;
}
const char* oracle_unit_test_message() { return oracle::g_message.c_str(); }
}
