// Test infrastructure only (see core.h). The drape model, Newton and pseudo-transient continuation of the
// reference oracle crate, generalised over the scene (gravity vector, collider set, fixed or resting barrier
// stiffness, start state) so that the reference's sphere-on-floor scene and the 1 m y-up sheet over a sphere
// (and optional ground plane) are two scene specs of one model.
//   drape.rs:34-439, newton.rs:113-258, e4_rules.rs:15-44, e7_ptc.rs:9-189, e7_run.rs:18-26.
#pragma once
#include "core.h"

namespace oracle {

enum class TangentKind { Exact, Projected };

struct Scene {
  std::string name = "custom";
  Mesh mesh;
  Material material{};
  std::vector<int> fixed;
  Contact contact;
  Vec3 gravity{0.0, 0.0, -9.81};
  std::vector<Vec3> start;  // cold-start positions, one per vertex
};

// drape.rs:53-84 + e7_run.rs:18-26: the reference's E5/E7 sphere-on-floor scene (0.5 m knit sheet, z up).
// edit: "base" | "w1" | "w2" | "w3" (placed), "e5" (released 0.02 L above the sphere).
Scene reference_scene(int columns, const std::string& edit);
// drape.rs:145-155 with Scene::PinnedCorners: hung from the two top corners, no contact, flat at z = 0.
Scene pinned_scene(int columns);
// The 1.0 x 1.0 m sheet of n x n vertices in the xz-plane at y = 0.35 over a sphere at the origin (y up), with
// an optional ground plane; isotropic StVK (E, nu = 0.3, t = 5e-4 m), k_b = 1e-5 N m, density 0.15 kg/m^2,
// d_hat = 2e-3 m, kappa = 1e3, initial y jittered by Lcg(seed).uniform() * 1e-5 per vertex in index order.
Scene sheet_scene(int columns, uint64_t seed, double radius, double young, bool with_plane, double plane_y = -0.25);

struct Drape {
  Mesh mesh;
  Material material{};
  std::vector<MembraneElement> membranes;
  std::vector<HingeElement> hinges;
  std::vector<int> fixed, free_;
  std::vector<int> row_of;  // -1 for fixed vertices
  Bsr pattern;
  std::vector<double> mass;
  TangentKind tangent_kind = TangentKind::Exact;
  Contact contact;
  Vec3 gravity{0, 0, -9.81};
  std::vector<Vec3> start;
  mutable double time_step = 1.0 / 240.0;
  mutable bool barrier_curvature = true;

  explicit Drape(const Scene& s, TangentKind kind = TangentKind::Exact);
  int rows() const { return int(free_.size()); }
  bool has_contact() const { return !contact.colliders.empty(); }
  double g_norm() const { return norm(gravity); }
  double mass_over_h2(int v) const { return mass[v] / (time_step * time_step); }
  double potential(const std::vector<Vec3>& x) const;
  double barrier_energy(const std::vector<Vec3>& x) const;
  std::vector<Vec3> potential_gradient(const std::vector<Vec3>& x) const;
  // Scatter-add an element's blocks into a BSR with this pattern (drape.rs:238-246).
  template <size_t N>
  void add_blocks(Bsr& m, const std::array<int, N>& v, const std::array<std::array<Mat3, N>, N>& b) const {
    for (size_t k = 0; k < N; ++k)
      for (size_t l = 0; l < N; ++l) {
        int r = row_of[v[k]], c = row_of[v[l]];
        if (r >= 0 && c >= 0) m.add(r, c, b[k][l]);
      }
  }
};

// One backward-Euler / PTC step as an energy: Phi(x) = 1/(2h^2)(x - x_hat)^T M (x - x_hat) + Pi(x) (drape.rs:255-386).
struct DrapeStep {
  const Drape* drape;
  std::vector<Vec3> x_hat;

  double value(const std::vector<Vec3>& x) const;
  std::vector<double> residual(const std::vector<Vec3>& x) const;
  Bsr tangent(const std::vector<Vec3>& x) const;
  Bsr regularized_tangent(const std::vector<Vec3>& x, double mu) const;
  double energy_change(const std::vector<Vec3>& x, const std::vector<Vec3>& d, double alpha) const;
  double barrier_change(const std::vector<Vec3>& x, const std::vector<Vec3>& d, double alpha) const;
  std::vector<Vec3> scatter(const std::vector<double>& rows) const;
  std::vector<double> gather(const std::vector<Vec3>& v) const;
  double max_step(const std::vector<Vec3>& x, const std::vector<Vec3>& d) const;
  std::vector<double> absolute_contributions(const std::vector<Vec3>& x) const;
};

std::vector<Vec3> feasible_start(const DrapeStep& step, const std::vector<Vec3>& x);

// ---------------------------------------------------------------- Newton (newton.rs:113-258)
constexpr double MU_START = 1e-3;
constexpr double MU_CAP = 1e3;
inline double raise_mu(double mu) { return std::min(std::max(10.0 * mu, MU_START), MU_CAP); }
inline double relax_mu(double mu) {
  double n = mu / 10.0;
  return n < MU_START ? 0.0 : n;
}

enum class StepStatus { Converged, IterationLimit, LineSearchFailed, RegularizationCap, ConvergedAtFloor };
const char* status_name(StepStatus s);

struct NewtonSettings {
  double tolerance = 0.1;
  int max_iterations = 10;
  double armijo = 1e-4;
  int max_halvings = 30;
};

// How the Newton direction is solved: the reference's f64 band Cholesky, or f64 block-Jacobi PCG from x = 0
// with a fixed relative tolerance (a breakdown or a non-descent direction raises mu like a failed factorisation).
struct DirectionSolver {
  bool pcg = false;
  double rtol = 1e-6;
  int max_iterations = 2000;
};

struct Regularization {
  double max_mu = 0;
  int retries = 0;
  bool cap_hit = false;
};

struct StepSolution {
  std::vector<Vec3> positions;
  std::vector<double> residuals;
  std::vector<int> halvings;
  std::vector<double> step_lengths;
  std::vector<int> pcg_iterations;
  StepStatus status = StepStatus::IterationLimit;
  Regularization regularization;
};

// Backtracking from the CCD bound: accept when dPhi <= c alpha g^T d (newton.rs:158-167). Returns -1 when d is
// not a descent direction or halving runs out; else the halvings, with the accepted length in `length`.
int line_search(const DrapeStep& s, const std::vector<Vec3>& x, const std::vector<double>& g,
                const std::vector<Vec3>& d, const NewtonSettings& set, double* length);

StepSolution solve_step_regularized(const DrapeStep& s, std::vector<Vec3> start, double scale,
                                    const NewtonSettings& set, const DirectionSolver& dir);

// One backward-Euler step from (x, v) (drape.rs:403-417): x_hat = x + h v + h^2 g on the free vertices, Newton on
// Phi from x_hat, or with colliders from its feasible cut x + alpha_max (x_hat - x) (drape.rs:397-401), the residual
// scaled by |grad Phi(x)|; velocity (x_new - x) / h.
struct TimeStepResult {
  StepSolution solution;
  double scale = 0;
  std::vector<Vec3> velocity;
};
std::vector<Vec3> dynamic_prediction(const Drape& d, const std::vector<Vec3>& x, const std::vector<Vec3>& v, double h);
TimeStepResult time_step(const Drape& d, const std::vector<Vec3>& x, const std::vector<Vec3>& v, double h,
                         const NewtonSettings& set, const DirectionSolver& dir);

// e4_rules.rs:15-44
double next_forcing(double previous, double ratio);
double f32_spacing(double max_abs);
bool update_is_small(double update_inf, double step_inf, double resolution);

// ---------------------------------------------------------------- PTC (e7_ptc.rs:9-189)
enum class Controller { InnerCount, Doubling };

struct PtcRules {
  double h0 = 1.0 / 240.0, h_max = 1.0, h_min_factor = 0.1, growth = 2.0, shrink = 0.5;
  double inner_tolerance = 0.1;
  int inner_max = 10, max_rejections = 12, max_steps = 1000;
  double equilibrium = 1e-8;   // stop at r/L <= this ...
  double absolute = 0.0;       // ... or at r <= this (N), when positive
  double floor_factor = 2.0, floor_guard = 1e-6;
  bool floor_rule = true;
  Controller controller = Controller::InnerCount;
  // Inner Newton start: the reference's prediction x_k + h^2 g cut back by the CCD bound (e7_ptc.rs:129-133),
  // or the current state x_k (feasible, and grad Phi(x_k) = grad E_s(x_k)).
  bool predicted_start = true;
  double time_budget_s = 0.0;  // > 0: stop ("time_budget") once a step ends past this wall time
  static PtcRules reference() { return PtcRules{}; }
  // The sheet-over-sphere solve: dt0 = 1e-3 s, doubled after each accepted step, ||grad E_s|| <= 1e-6 N.
  static PtcRules doubling(double h0, double absolute) {
    PtcRules r;
    r.h0 = h0;
    r.controller = Controller::Doubling;
    r.absolute = absolute;
    r.equilibrium = 0.0;
    r.floor_rule = false;
    return r;
  }
};

struct PtcStep {
  double h, residual;
  int inner_iterations, rejected_attempts, pcg_iterations;
  double max_mu;
  bool mu_cap, curvature_dropped;
};

struct PtcRun {
  std::vector<std::vector<Vec3>> states;  // all states when keep_states, else first and last
  std::vector<PtcStep> steps;
  double final_residual = NAN, final_h = 0;
  std::string reason = "cap";
  bool converged() const { return reason == "tolerance" || reason == "floor"; }
};

double next_step_size(const PtcRules& r, double h, int inner);
double gravity_load(const Drape& d);
std::vector<double> static_gradient(const Drape& d, const std::vector<Vec3>& x);
double static_energy(const Drape& d, const std::vector<Vec3>& x);
std::vector<Vec3> ptc_prediction(const Drape& d, const std::vector<Vec3>& x, double h);
double static_floor(const Drape& d, const std::vector<Vec3>& x);
PtcRun ptc_solve(const Drape& d, std::vector<Vec3> start, double h_start, const PtcRules& rules,
                 const DirectionSolver& dir, bool keep_states, bool progress);
bool attempt_failed(StepStatus status, int iterations, const std::vector<Vec3>& positions);
// One accepted PTC step from x (attempts at h, h/2, ...); false when every attempt failed.
bool take_step(const Drape& d, const std::vector<Vec3>& x, double h, double residual, const PtcRules& rules,
               const DirectionSolver& dir, std::vector<Vec3>& next, PtcStep& step);

// e3_checks.rs:40-44 and e5_checks.rs:60-78: the kernel-check states.
std::vector<Vec3> bent_state(const Drape& d, Lcg& rng);
std::vector<Vec3> contact_state(const Drape& d);

// e7_prolong.rs:9-47
std::vector<Vec3> prolong(const std::vector<Vec3>& coarse, int coarse_columns);
int project_out(const Drape& d, std::vector<Vec3>& positions);

}  // namespace oracle
