// Host-side problem description of one drape: the mesh, material and scene types the GPU stage needs, laid
// out as flat arrays (what the reference's problem.bin carries: e3_generate.rs:84-104, e5_checks.rs:80-86,
// e7_run.rs:46), plus the two scene builders the product ships:
//   * the 1.0 m sheet over a sphere (and optional ground plane), y up, isotropic StVK;
//   * the reference's 0.5 m knit sheet over a sphere resting on a floor, z up (drape.rs:53-84).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace drape {

struct HostProblem {
  int columns = 0;
  int V = 0, T = 0, H = 0, R = 0, B = 0;
  std::vector<double> start;         // 3V cold-start positions
  std::vector<int32_t> tri;          // 3T vertex ids
  std::vector<double> tri_geom;      // 7T: dN0/dX, dN0/dY, dN1/dX, dN1/dY, dN2/dX, dN2/dY, rest area
  std::vector<int32_t> hinge;        // 4H: [left opposite, right opposite, edge a, edge b]
  std::vector<double> hinge_k;       // H: k_b(e) 3|e|^2/(A1 + A2)
  std::vector<int32_t> row_vertex;   // R: vertex of each unknown row (free vertices in order)
  std::vector<double> unit_mass;     // R: lumped mass of the row's vertex
  std::vector<int32_t> row_ptr;      // R+1: BSR(3x3) pattern over rows
  std::vector<int32_t> col_idx;      // B
  double wale = 0, course = 0, coupling = 0, shear = 0;  // membrane law (N/m)
  double gravity[3] = {0, 0, -9.81};
  std::vector<double> colliders;     // 8 per collider: kind (1 plane, 2 sphere), a, b, c, w, 0, 0, 0
  double dhat = 0, kappa = 0;

  int collider_count() const { return int(colliders.size() / 8); }
};

// Deterministic 64-bit LCG with uniform values in [-1, 1) (the scene jitter's generator, rng.rs:2-13).
struct Lcg64 {
  uint64_t state;
  explicit Lcg64(uint64_t seed);
  double uniform();
};

// The sheet over a sphere of radius `radius` at the origin (y up, gravity -9.81 y), optional ground plane at
// y = plane_y: n x n vertices on [-0.5, 0.5]^2 in the xz-plane at y = 0.35, y jittered by 1e-5 * Lcg(seed);
// E = young, nu = 0.3, t = 5e-4 m, k_b = 1e-5 N m, density 0.15 kg/m^2, d_hat = 2e-3 m, kappa = 1e3.
HostProblem sheet_problem(int columns, uint64_t seed, double radius, double young, bool with_plane,
                          double plane_y = -0.25, double poisson = 0.3, double kb = 1e-5);

// The reference's E7 scene: edit base|w1|w2|w3 (placed at 2 d_hat above the sphere top).
HostProblem reference_problem(int columns, const std::string& edit);

// Reads a problem.json / problem.bin pair written by the reference's `oracle e7-generate` (or the oracle
// restatement); f64 copies of the geometry arrays are used when present. Throws std::runtime_error.
HostProblem read_problem_files(const std::string& dir);
// One named array of a problem.bin as f64 (empty when the manifest has no such array): the check states
// kernel_state and contact_state and the per-row row_mass of the reference's files (e3_generate.rs:93-98).
std::vector<double> read_problem_array(const std::string& dir, const std::string& name);
// The same from any manifest / binary pair in that layout (the oracle's probes.json / probes.bin, io.rs:5-55).
std::vector<double> read_named_array(const std::string& json_path, const std::string& bin_path,
                                     const std::string& name);
// The whole file as text (throws if it cannot be read).
std::string read_text_file(const std::string& path);
// The number at the first "key": after the first "anchor" of a JSON text (NaN if absent): the flat key scan the
// reference reads problem.json with (jsonscan.rs:3-26).
double json_number(const std::string& text, const std::string& anchor, const std::string& key);

// Writes the same pair (the subset this GPU stage reads, plus f64 geometry).
void write_problem_files(const HostProblem& p, const std::string& dir);

// Coarse-to-fine start state for the prolong mode (the reference's e7_prolong.rs:7-64): the (2n - 1)^2 grid from the
// n^2 one, every fine vertex the average of its four (possibly repeated) coarse corners; then every vertex closer
// than d_hat to a collider moves along that collider's normal to d = d_hat, one pass over the colliders in order.
// Returns the number of vertices moved; `infeasible` (may be null) receives the vertices at or inside a collider
// afterwards. Throws std::invalid_argument when the prolonged grid is not `fine`'s.
int prolong_state(const HostProblem& fine, const std::vector<double>& coarse, int coarse_columns,
                  std::vector<double>* out, std::vector<int>* infeasible);

// Checks sizes and index ranges of every array; returns an empty string when consistent.
std::string validate(const HostProblem& p);

}  // namespace drape
