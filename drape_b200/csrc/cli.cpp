// `drape`: the GPU stage of the run-e*.sh pipeline as one command, in place of `node src/node/run-e7.ts` (its
// flags: engine/gpu/src/node/run-e7.ts:37-43; its outputs: run-e7.ts:93-107, state-files.ts).
//
//   drape --case <dir> [--mode cold|warm|prolong] [--start <state prefix>]
//         [--preconditioner jacobi|multilevel|learned] [--network <weights file>] [--device <n>] [--checks]
//   drape prolong --coarse <state prefix> --coarse-n <n> --fine-dir <case dir> --out <state prefix>
//   environment: E7_BUDGET_S (time budget of the solve, s), E7_PROGRESS (one stderr line per accepted step)
//
// Reads <dir>/problem.json + problem.bin (`oracle e7-generate`), solves to equilibrium with the rules of the
// problem's "ptc", "newton", "pcg" and "robust" blocks (the reference's start x_k + alpha (x_hat - x_k), its
// inner-count controller, Eisenstat-Walker forcing), and writes <dir>/gpu-<mode>/:
//   gpu-result.json               schema e7-gpu/1: the run-e7.ts fields this solver records
//   gpu-ptc.bin                   f64 [accepted steps][7]: step, h, residual, inner, rejected, pcgIterations, minDistance
//   gpu-equilibrium.{json,bin}    the equilibrium as an f32 state file with its final_h
//   gpu-states.bin                f32: the start state, then every accepted state (grids of <= 65 columns) or
//                                 the equilibrium alone
//   gpu-iterations.bin            f64 [Newton iterates][9]: the reference's RECORD_FIELDS (outputs.ts:8)
//   gpu-robust.bin                f64 [Newton iterates][16]: EXTRA_FIELDS (outputs.ts:9-10), NaN where this solver
//                                 has no counterpart (update/step norms, resolution, limiting vertex, noise tests)
//   gpu-attempts.bin              f64 [attempts][6]: step, attempt, h, reason, recordStart, recordEnd
// and with --checks, before the solve (run-e7.ts:81-91, 140-152):
//   gpu-kernel.bin                f32: exact element gradient [9T + 12H] and Hessian [81T + 144H], the projected
//                                 ones, then the row terms [3R + 9R] at kernel_state, x_hat = rest, mu = kernel_mu
//   gpu-contact-kernel.bin        f32 [3R + 9R]: the barrier row terms alone at contact_state
//   gpu-inertia-h.bin             f32: the inertia row terms at kernel_state for h = 1/240, 0.1, 1 s
//   gpu-probe-{iterations,robust}.bin, gpu-probe-iterates.bin, gpu-probe-directions.bin, gpu-probe-search.bin:
//                                 the PTC probes of the case's probes.json / probes.bin, when it has them
// Exit status: 0 when the solve ran to a stop rule, 1 on an error, 2 on a usage error.
#include <sys/stat.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/drape_b200.h"
#include "problem.h"

namespace {

const char* kUsage =
    "usage: drape --case <case dir> [--mode cold|warm|prolong] [--start <state prefix>]\n"
    "             [--preconditioner jacobi|multilevel|learned] [--network <weights>] [--device <n>] [--checks]\n";

struct Args {
  std::string dir, mode = "cold", start, preconditioner = "jacobi", network;
  int device = 0;
  bool checks = false;
};

bool parse(int argc, char** argv, Args* a, std::string* err) {
  for (int i = 1; i < argc; ++i) {
    const std::string k = argv[i];
    auto value = [&](std::string* out) {
      if (i + 1 >= argc) return false;
      *out = argv[++i];
      return true;
    };
    std::string dev;
    bool ok = k == "--case" ? value(&a->dir)
              : k == "--mode" ? value(&a->mode)
              : k == "--start" ? value(&a->start)
              : k == "--preconditioner" ? value(&a->preconditioner)
              : k == "--network" ? value(&a->network)
              : k == "--device" ? (value(&dev) && (a->device = std::atoi(dev.c_str()), true))
              : k == "--checks" ? (a->checks = true, true)
                                : false;
    if (!ok) {
      *err = "unknown or incomplete option " + k;
      return false;
    }
  }
  if (a->dir.empty()) *err = "--case is required";
  else if (a->mode != "cold" && a->mode != "warm" && a->mode != "prolong") *err = "unknown mode " + a->mode;
  else if (a->mode != "cold" && a->start.empty()) *err = "mode " + a->mode + " needs --start <state prefix>";
  else if (a->preconditioner != "jacobi" && a->preconditioner != "multilevel" && a->preconditioner != "learned")
    *err = "unknown preconditioner " + a->preconditioner;
  return err->empty();
}

// An f32 or f64 state file pair (e7_state.rs:9-40): positions and final_h.
bool read_state(const std::string& prefix, std::vector<double>* xyz, double* final_h, std::string* err) {
  std::string text;
  try {
    text = drape::read_text_file(prefix + ".json");
  } catch (const std::exception& e) {
    *err = e.what();
    return false;
  }
  const bool single = text.find("\"f32\"") != std::string::npos;
  *final_h = drape::json_number(text, "", "final_h");
  std::ifstream f(prefix + ".bin", std::ios::binary);
  std::vector<char> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  const size_t width = single ? 4 : 8;
  if (!f.good() && !f.eof()) {
    *err = prefix + ".bin: cannot read";
    return false;
  }
  xyz->resize(bytes.size() / width);
  for (size_t i = 0; i < xyz->size(); ++i) {
    if (single) {
      float v;
      std::memcpy(&v, bytes.data() + 4 * i, 4);
      (*xyz)[i] = v;
    } else {
      std::memcpy(&(*xyz)[i], bytes.data() + 8 * i, 8);
    }
  }
  return true;
}

bool write_bytes(const std::string& path, const void* data, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(static_cast<const char*>(data), std::streamsize(n));
  return bool(f);
}

// gpu-<prefix>iterations.bin (RECORD_FIELDS) and gpu-<prefix>robust.bin (EXTRA_FIELDS) of the context's Newton records
// (writeRun, outputs.ts:24-28): f64 rows, NaN where the reference's field has no counterpart in this solver or no
// value on the iterate (the last iterate of an attempt takes no solve).
bool write_run_tables(drape_ctx* ctx, const std::string& out, const std::string& prefix, int32_t* count) {
  const double nan = std::nan("");
  int32_t n = 0;
  drape_newton_records(ctx, nullptr, 0, &n);
  std::vector<drape_newton_record> rec(size_t(n > 0 ? n : 1));
  drape_newton_records(ctx, rec.data(), n, &n);
  std::vector<double> iterations, robust;
  for (int i = 0; i < n; ++i) {
    const drape_newton_record& r = rec[size_t(i)];
    const bool solved = r.pcg_iterations >= 0;
    const double it_row[9] = {double(r.step), double(r.iteration), r.relative_residual,
                              solved ? double(r.pcg_iterations) : nan, solved ? double(r.pcg_status) : nan,
                              solved ? r.linear_residual : nan, r.step_length,
                              r.halvings >= 0 ? double(r.halvings) : nan, double(r.status)};
    iterations.insert(iterations.end(), it_row, it_row + 9);
    // eta, mu, updateInf, stepInf, retries, resolution, alphaMax, limitingVertex, minDistance, deltaSum, deltaAbs,
    // noiseOnly, slope, slopeExact, normSquared, normSquaredExact
    const double rb_row[16] = {r.eta, r.mu, nan, nan, solved ? double(r.retries) : nan, r.resolution, r.alpha_max,
                               nan, nan, r.delta_sum, nan, nan, r.slope, nan, r.norm_squared, nan};
    robust.insert(robust.end(), rb_row, rb_row + 16);
  }
  *count = n;
  const std::string base = out + "/gpu-" + prefix;
  return write_bytes(base + "iterations.bin", iterations.data(), iterations.size() * sizeof(double)) &&
         write_bytes(base + "robust.bin", robust.data(), robust.size() * sizeof(double));
}

double rule(const std::string& text, const char* block, const char* key, double fallback) {
  const double v = drape::json_number(text, block, key);
  return std::isfinite(v) ? v : fallback;
}

// run-e7.ts --checks (runChecks, run-e7.ts:140-145; writeChecks, 81-91): the element and row terms at the problem's
// check states, in the reference's layouts. Needs kernel_state, rest_positions, row_mass (and contact_state for the
// contact file) in problem.bin, and the robust block's kernel_mu.
bool write_checks(drape_ctx* ctx, const std::string& dir, const std::string& text, const std::string& out,
                  const int64_t sizes[6], std::string* err) {
  const size_t V = size_t(sizes[0]), T = size_t(sizes[1]), H = size_t(sizes[2]), R = size_t(sizes[3]);
  std::vector<double> kernel_state, contact_state, rest, row_mass, unit_mass, colliders;
  try {
    kernel_state = drape::read_problem_array(dir, "kernel_state");
    contact_state = drape::read_problem_array(dir, "contact_state");
    rest = drape::read_problem_array(dir, "rest_positions");
    row_mass = drape::read_problem_array(dir, "row_mass");
    unit_mass = drape::read_problem_array(dir, "row_unit_mass_f64");
    if (unit_mass.empty()) unit_mass = drape::read_problem_array(dir, "row_unit_mass");
    colliders = drape::read_problem_array(dir, "colliders");
  } catch (const std::exception& e) {
    *err = e.what();
    return false;
  }
  const double kernel_mu = drape::json_number(text, "robust", "kernel_mu");
  if (kernel_state.size() != 3 * V || rest.size() != 3 * V || row_mass.size() != R || unit_mass.size() != R ||
      !std::isfinite(kernel_mu)) {
    *err = "--checks needs kernel_state, rest_positions, row_mass and row_unit_mass in problem.bin and "
           "robust.kernel_mu in problem.json";
    return false;
  }
  auto fail = [&](const char* what) {
    *err = std::string(what) + ": " + drape_last_error(ctx);
    return false;
  };
  std::vector<float> kernel, g(9 * T + 12 * H), h(81 * T + 144 * H), rg(3 * R), rh(9 * R);
  for (int exact = 1; exact >= 0; --exact) {
    if (drape_element_terms(ctx, kernel_state.data(), exact, g.data(), h.data()) != DRAPE_OK)
      return fail("element terms");
    kernel.insert(kernel.end(), g.begin(), g.end());
    kernel.insert(kernel.end(), h.begin(), h.end());
  }
  if (drape_row_terms(ctx, kernel_state.data(), rest.data(), row_mass.data(), kernel_mu, 0, 1, rg.data(),
                      rh.data()) != DRAPE_OK)
    return fail("row terms");
  kernel.insert(kernel.end(), rg.begin(), rg.end());
  kernel.insert(kernel.end(), rh.begin(), rh.end());
  bool ok = write_bytes(out + "/gpu-kernel.bin", kernel.data(), kernel.size() * sizeof(float));
  if (contact_state.size() == 3 * V) {
    // header word 3 of the collider array switches the barrier's curvature term off (contact-host.ts:92-97)
    const int curvature = colliders.size() > 3 && colliders[3] != 0.0 ? 0 : 1;
    if (drape_row_terms(ctx, contact_state.data(), contact_state.data(), nullptr, 0.0, 1, curvature, rg.data(),
                        rh.data()) != DRAPE_OK)
      return fail("contact terms");
    std::vector<float> contact(rg.begin(), rg.end());
    contact.insert(contact.end(), rh.begin(), rh.end());
    ok = ok && write_bytes(out + "/gpu-contact-kernel.bin", contact.data(), contact.size() * sizeof(float));
  }
  std::vector<float> inertia;
  for (double size : {1.0 / 240.0, 0.1, 1.0}) {
    std::vector<double> mass(R);
    for (size_t r = 0; r < R; ++r) mass[r] = double(float(unit_mass[r] / (size * size)));
    if (drape_row_terms(ctx, kernel_state.data(), rest.data(), mass.data(), 0.0, 0, 1, rg.data(), rh.data()) !=
        DRAPE_OK)
      return fail("inertia terms");
    inertia.insert(inertia.end(), rg.begin(), rg.end());
    inertia.insert(inertia.end(), rh.begin(), rh.end());
  }
  ok = ok && write_bytes(out + "/gpu-inertia-h.bin", inertia.data(), inertia.size() * sizeof(float));
  if (!ok) {
    *err = "cannot write the check files in " + out;
    return false;
  }
  // PTC probes when the case has them (probes.json / probes.bin of the oracle's cold base solves; run-e7.ts:65-79,
  // 146-152): one logged Newton attempt from each probed f32 state with its h
  std::ifstream probes_json(dir + "/probes.json");
  if (!probes_json) return true;
  std::vector<double> steps, hs, positions;
  try {
    steps = drape::read_named_array(dir + "/probes.json", dir + "/probes.bin", "probe_steps");
    hs = drape::read_named_array(dir + "/probes.json", dir + "/probes.bin", "probe_h");
    positions = drape::read_named_array(dir + "/probes.json", dir + "/probes.bin", "probe_positions");
  } catch (const std::exception& e) {
    *err = e.what();
    return false;
  }
  if (hs.size() != steps.size() || positions.size() != 3 * V * steps.size()) {
    *err = "probes.bin: probe_steps, probe_h and probe_positions disagree";
    return false;
  }
  if (drape_probe_begin(ctx) != DRAPE_OK) return fail("probes");
  for (size_t k = 0; k < steps.size(); ++k)
    if (drape_probe_step(ctx, positions.data() + 3 * V * k, hs[k], int32_t(steps[k])) != DRAPE_OK)
      return fail("probe");
  int64_t ni = 0, nd = 0, nt = 0;
  drape_probe_logs(ctx, nullptr, 0, &ni, nullptr, 0, &nd, nullptr, 0, &nt);
  std::vector<float> iterates(static_cast<size_t>(ni)), directions(static_cast<size_t>(nd));
  std::vector<double> trials(static_cast<size_t>(nt));
  drape_probe_logs(ctx, iterates.data(), ni, &ni, directions.data(), nd, &nd, trials.data(), nt, &nt);
  int32_t n_rec = 0;
  ok = write_run_tables(ctx, out, "probe-", &n_rec) &&
       write_bytes(out + "/gpu-probe-iterates.bin", iterates.data(), iterates.size() * sizeof(float)) &&
       write_bytes(out + "/gpu-probe-directions.bin", directions.data(), directions.size() * sizeof(float)) &&
       write_bytes(out + "/gpu-probe-search.bin", trials.data(), trials.size() * sizeof(double));
  if (!ok) *err = "cannot write the probe files in " + out;
  return ok;
}

}  // namespace

// `drape prolong --coarse <state prefix> --coarse-n <n> --fine-dir <case dir> --out <state prefix>`: the start state
// of the prolong mode from a coarse equilibrium, in place of `oracle e7-prolong` (e7_prolong.rs:52-64): host
// arithmetic only (drape::prolong_state), written in the coarse state's dtype with its final_h.
int prolong_main(int argc, char** argv) {
  std::string coarse, fine_dir, out, n_text;
  for (int i = 1; i < argc; ++i) {
    const std::string k = argv[i];
    std::string* dst = k == "--coarse" ? &coarse : k == "--coarse-n" ? &n_text : k == "--fine-dir" ? &fine_dir
                     : k == "--out" ? &out : nullptr;
    if (!dst || i + 1 >= argc) {
      std::fprintf(stderr, "drape prolong: unknown or incomplete option %s\n", k.c_str());
      return 2;
    }
    *dst = argv[++i];
  }
  if (coarse.empty() || fine_dir.empty() || out.empty() || n_text.empty()) {
    std::fprintf(stderr, "usage: drape prolong --coarse <state prefix> --coarse-n <n> --fine-dir <case dir> --out <state prefix>\n");
    return 2;
  }
  try {
    const drape::HostProblem fine = drape::read_problem_files(fine_dir);
    std::vector<double> xc;
    double h = 0.0;
    std::string err;
    if (!read_state(coarse, &xc, &h, &err)) throw std::runtime_error(err);
    const bool single = drape::read_text_file(coarse + ".json").find("\"f32\"") != std::string::npos;
    std::vector<double> xf;
    std::vector<int> bad;
    const int moved = drape::prolong_state(fine, xc, std::atoi(n_text.c_str()), &xf, &bad);
    std::printf("prolongation: %d vertices projected to d = d_hat, %zu infeasible\n", moved, bad.size());
    if (!bad.empty()) throw std::runtime_error("infeasible start after projection");
    bool ok;
    if (single) {
      std::vector<float> f(xf.begin(), xf.end());
      ok = write_bytes(out + ".bin", f.data(), f.size() * sizeof(float));
    } else {
      ok = write_bytes(out + ".bin", xf.data(), xf.size() * sizeof(double));
    }
    std::ofstream j(out + ".json");
    char buf[256];
    std::snprintf(buf, sizeof buf, "{\"vertices\":%d,\"final_h\":%.17g,\"dtype\":\"%s\"}\n", fine.V, h,
                  single ? "f32" : "f64");
    j << buf;
    if (!ok || !j) throw std::runtime_error("cannot write " + out);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "drape prolong: %s\n", e.what());
    return 1;
  }
  return 0;
}

int main(int argc, char** argv) {
  if (argc > 1 && std::string(argv[1]) == "prolong") return prolong_main(argc - 1, argv + 1);
  Args a;
  std::string err;
  if (!parse(argc, argv, &a, &err)) {
    std::fprintf(stderr, "drape: %s\n%s", err.c_str(), kUsage);
    return 2;
  }
  std::string text;
  try {
    text = drape::read_text_file(a.dir + "/problem.json");
  } catch (const std::exception& e) {
    std::fprintf(stderr, "drape: %s\n", e.what());
    return 1;
  }
  drape_options o;
  drape_default_options(&o);
  o.h0 = rule(text, "ptc", "h0", o.h0);
  o.h_max = rule(text, "ptc", "h_max", o.h_max);
  o.h_min_factor = rule(text, "ptc", "h_min_factor", o.h_min_factor);
  o.growth = rule(text, "ptc", "growth", o.growth);
  o.shrink = rule(text, "ptc", "shrink", o.shrink);
  o.max_rejections = int(rule(text, "ptc", "max_rejections", o.max_rejections));
  o.inner_tolerance = rule(text, "ptc", "inner_tolerance", o.inner_tolerance);
  o.inner_max = int(rule(text, "ptc", "inner_max_iterations", o.inner_max));
  o.max_steps = int(rule(text, "ptc", "max_steps", o.max_steps));
  o.equilibrium_relative = rule(text, "ptc", "equilibrium_f64", 1e-8);
  o.equilibrium_absolute = 0.0;
  o.armijo = rule(text, "newton", "armijo", o.armijo);
  o.max_halvings = int(rule(text, "newton", "max_halvings", o.max_halvings));
  o.pcg_max_iterations = int(rule(text, "pcg", "max_iterations", o.pcg_max_iterations));
  o.replace_every = int(rule(text, "pcg", "replace_every", 0));
  o.replace_above = rule(text, "pcg", "replace_above", o.replace_above);
  o.forcing = 1;
  o.newton_start = 1;
  o.controller = 0;
  o.preconditioner = a.preconditioner == "jacobi" ? 0 : a.preconditioner == "multilevel" ? 1 : 2;
  if (const char* b = std::getenv("E7_BUDGET_S")) o.time_budget_s = std::atof(b);
  o.progress = std::getenv("E7_PROGRESS") != nullptr;

  std::vector<double> start;
  double h0 = o.h0;
  if (!a.start.empty()) {
    if (!read_state(a.start, &start, &h0, &err)) {
      std::fprintf(stderr, "drape: %s\n", err.c_str());
      return 1;
    }
  }
  drape_ctx* ctx = nullptr;
  if (drape_create_from_files(a.dir.c_str(), &o, a.device, &ctx) != DRAPE_OK) {
    std::fprintf(stderr, "drape: %s\n", drape_last_error(nullptr));
    return 1;
  }
  int64_t sizes[6];
  drape_sizes(ctx, sizes);
  const size_t V = size_t(sizes[0]);
  if (!start.empty() && start.size() != 3 * V) {
    std::fprintf(stderr, "drape: %s has %zu values, the problem %zu vertices\n", a.start.c_str(), start.size(), V);
    drape_destroy(ctx);
    return 1;
  }
  drape_network* net = nullptr;
  if (o.preconditioner == 2) {
    std::string path = a.network;
    if (path.empty()) {  // the shipped weights beside the executable
      char self[4096];
      const ssize_t n = readlink("/proc/self/exe", self, sizeof self - 1);
      path = n > 0 ? std::string(self, size_t(n)) : std::string(argv[0]);
      path = path.substr(0, path.rfind('/') + 1) + "preconditioner_network.bin";
    }
    if (drape_network_create(a.device, 0, &net) != DRAPE_OK || drape_network_load(net, path.c_str()) != DRAPE_OK ||
        drape_set_network(ctx, net) != DRAPE_OK) {
      std::fprintf(stderr, "drape: preconditioner network %s: %s\n", path.c_str(), drape_last_error(nullptr));
      drape_destroy(ctx);
      drape_network_destroy(net);
      return 1;
    }
  }
  // every accepted state is kept for grids of at most 65 columns (run-e7.ts:29,133)
  const bool keep_states = drape::json_number(text, "", "grid_columns") <= 65;
  drape_keep_states(ctx, keep_states ? 1 : 0);
  const std::string out = a.dir + "/gpu-" + a.mode;
  ::mkdir(out.c_str(), 0755);
  // the solve's start, taken before the checks: the probe runs move the context's state
  std::vector<double> x0(3 * V);
  drape_get_state(ctx, x0.data(), nullptr);
  if (!start.empty()) x0 = start;
  if (a.checks && !write_checks(ctx, a.dir, text, out, sizes, &err)) {
    std::fprintf(stderr, "drape: %s\n", err.c_str());
    drape_destroy(ctx);
    drape_network_destroy(net);
    return 1;
  }
  drape_run_log log{};
  const drape_status st = drape_solve_equilibrium(ctx, x0.data(), h0, &log);
  if (st != DRAPE_OK && st != DRAPE_E_DIVERGED && st != DRAPE_E_TIMEOUT) {
    std::fprintf(stderr, "drape: %s\n", drape_last_error(ctx));
    drape_destroy(ctx);
    drape_network_destroy(net);
    return 1;
  }
  std::vector<double> x(3 * V);
  double final_h = 0.0;
  drape_get_state(ctx, x.data(), &final_h);
  int32_t count = 0;
  drape_step_records(ctx, nullptr, 0, &count);
  std::vector<drape_step_record> recs(size_t(count > 0 ? count : 1));
  drape_step_records(ctx, recs.data(), count, &count);

  std::vector<double> ptc;
  for (int i = 0; i < count; ++i) {
    const drape_step_record& r = recs[size_t(i)];
    const double row[7] = {double(r.step), r.h, r.residual, double(r.inner), double(r.rejected),
                           double(r.pcg_iterations), r.min_distance};
    ptc.insert(ptc.end(), row, row + 7);
  }
  // per-attempt table (run-e7.ts:98); the per-Newton tables are written with the others below
  int32_t n_att = 0;
  drape_attempt_records(ctx, nullptr, 0, &n_att);
  std::vector<drape_attempt_record> arec(size_t(n_att > 0 ? n_att : 1));
  drape_attempt_records(ctx, arec.data(), n_att, &n_att);
  std::vector<double> attempts;
  for (int i = 0; i < n_att; ++i) {
    const drape_attempt_record& r = arec[size_t(i)];
    const double row[6] = {double(r.step), double(r.attempt), r.h, double(r.reason), double(r.record_start),
                           double(r.record_end)};
    attempts.insert(attempts.end(), row, row + 6);
  }
  // the start state, then every accepted state (small grids) or the equilibrium alone (drape-e7.ts:159,175-178)
  std::vector<float> eq(x.begin(), x.end()), states(x0.begin(), x0.end());
  if (keep_states) {
    int64_t n_states = 0;
    drape_step_states(ctx, nullptr, 0, &n_states);
    std::vector<float> kept(size_t(n_states > 0 ? n_states : 1));
    drape_step_states(ctx, kept.data(), n_states, &n_states);
    states.insert(states.end(), kept.begin(), kept.begin() + n_states);
  } else {
    states.insert(states.end(), eq.begin(), eq.end());
  }
  bool ok = write_bytes(out + "/gpu-ptc.bin", ptc.data(), ptc.size() * sizeof(double)) &&
            write_bytes(out + "/gpu-equilibrium.bin", eq.data(), eq.size() * sizeof(float)) &&
            write_bytes(out + "/gpu-states.bin", states.data(), states.size() * sizeof(float)) &&
            write_bytes(out + "/gpu-attempts.bin", attempts.data(), attempts.size() * sizeof(double));
  int32_t n_rec = 0;
  ok = ok && write_run_tables(ctx, out, "", &n_rec);
  {
    std::ofstream f(out + "/gpu-equilibrium.json");
    char buf[256];
    std::snprintf(buf, sizeof buf, "{\"vertices\":%zu,\"final_h\":%.17g,\"dtype\":\"f32\"}\n", V, final_h);
    f << buf;
    ok = ok && bool(f);
  }
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, a.device);
  static const char* kStop[] = {"tolerance", "cap", "stalled", "time_budget"};
  const char* stop = log.reason >= 0 && log.reason < 4 ? kStop[log.reason] : "error";
  const int steps = log.ptc_steps > 0 ? log.ptc_steps : 1;
  {
    std::ofstream f(out + "/gpu-result.json");
    char buf[8192];
    std::snprintf(
        buf, sizeof buf,
        "{\n  \"schema\": \"e7-gpu/1\",\n  \"backend\": \"drape_b200-cuda\",\n  \"adapter\": \"%s\",\n  \"mode\": \"%s\",\n"
        "  \"preconditioner\": \"%s\",\n  \"grid_columns\": %d,\n  \"stop\": \"%s\",\n  \"cap\": %d,\n"
        "  \"accepted_steps\": %d,\n  \"rejected_attempts\": %d,\n  \"newton_iterations_total\": %d,\n"
        "  \"pcg_iterations_total\": %d,\n  \"final_h\": %.17g,\n  \"final_residual\": %.17g,\n"
        "  \"final_relative_residual\": %.17g,\n  \"trajectory_ms\": %.6f,\n  \"ms_per_step\": %.6f,\n"
        "  \"device_ms\": %.6f,\n  \"phase_ms_per_step\": {\"assembly\": %.6f, \"pcg\": %.6f, \"line_search\": %.6f, "
        "\"ccd\": %.6f, \"other\": %.6f},\n  \"kernel_launches\": %d,\n  \"fallbacks_to_jacobi\": %d,\n"
        "  \"newton_records\": %d,\n  \"attempt_records\": %d,\n"
        // the column names of gpu-iterations.bin and gpu-robust.bin (outputs.ts:8-10; e4_compare.rs:61-70 reads the
        // robust table by these names)
        "  \"record_fields\": [\"step\", \"iteration\", \"relativeResidual\", \"pcgIterations\", \"pcgStatus\", "
        "\"linearResidual\", \"stepLength\", \"halvings\", \"status\"],\n"
        "  \"robust_fields\": [\"eta\", \"mu\", \"updateInf\", \"stepInf\", \"retries\", \"resolution\", \"alphaMax\", "
        "\"limitingVertex\", \"minDistance\", \"deltaSum\", \"deltaAbs\", \"noiseOnly\", \"slope\", \"slopeExact\", "
        "\"normSquared\", \"normSquaredExact\"]\n}\n",
        prop.name, a.mode.c_str(), a.preconditioner.c_str(), int(drape::json_number(text, "", "grid_columns")), stop,
        o.max_steps, log.ptc_steps, log.rejected_attempts, log.newton_iterations, log.pcg_iterations, log.final_h,
        log.final_residual, log.final_relative_residual, 1e3 * log.seconds, 1e3 * log.seconds / steps,
        1e3 * log.device_seconds, log.ms_assembly / steps, log.ms_pcg / steps, log.ms_line_search / steps,
        log.ms_ccd / steps, log.ms_other / steps, log.kernel_launches, log.fallbacks, n_rec, n_att);
    f << buf;
    ok = ok && bool(f);
  }
  std::printf("%s %s: %d steps (+%d rejected), stop %s, r/L %.2e, %.2f s, h next %.2e\n",
              a.dir.substr(a.dir.rfind('/') + 1).c_str(), a.mode.c_str(), log.ptc_steps, log.rejected_attempts, stop,
              log.final_relative_residual, log.seconds, final_h);
  drape_destroy(ctx);
  drape_network_destroy(net);
  if (!ok) {
    std::fprintf(stderr, "drape: cannot write the outputs in %s\n", out.c_str());
    return 1;
  }
  return 0;
}
