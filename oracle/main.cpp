// Test infrastructure only (see core.h). The oracle command line (main.rs:55-156, e7-* subset):
//   oracle e7-generate --n N --edit base|w1|w2|w3 --out DIR      problem.json + problem.bin (e7_run.rs:41-50)
//   oracle e7-solve --dir DIR --mode cold|warm|prolong [--start P] reference-<mode>.json, equilibrium-<mode>.*
//   oracle e7-prolong --coarse P --coarse-n N --fine-dir DIR --out P
//   oracle sheet-solve --n N [--seed S --radius R --young E --plane 0|1 --direction cholesky|pcg --out P]
// The problem files follow e3_generate.rs:84-229 (arrays, scatter maps, rule blocks).
#include <chrono>
#include <cstdio>
#include <map>
#include <sys/stat.h>

#include "drape.h"
#include "io.h"

using namespace oracle;

namespace {

std::vector<float> f32(const std::vector<double>& v) { return std::vector<float>(v.begin(), v.end()); }
std::vector<double> flat(const std::vector<Vec3>& x) {
  std::vector<double> o;
  for (auto& p : x) o.insert(o.end(), p.begin(), p.end());
  return o;
}

// e3_generate.rs:119-161: ordered contribution lists per BSR block and per row.
void push_contributions(BinaryArrays& a, const std::string& name, const std::vector<std::vector<uint32_t>>& lists) {
  std::vector<uint32_t> ptr{0}, idx;
  for (auto& l : lists) {
    idx.insert(idx.end(), l.begin(), l.end());
    ptr.push_back(uint32_t(idx.size()));
  }
  a.push_u32(name + "_contrib_ptr", ptr);
  a.push_u32(name + "_contrib_idx", idx);
}

BinaryArrays problem_arrays(const Drape& d) {
  BinaryArrays a;
  size_t T = d.membranes.size(), H = d.hinges.size();
  a.push_f32("rest_positions", f32(flat(d.start)));
  std::vector<uint32_t> ev, hv, rv, dm, rp, ci, di, fx;
  std::vector<double> geom, hs, rm;
  for (auto& e : d.membranes) {
    for (int v : e.vertices) ev.push_back(uint32_t(v));
    for (auto& g : e.grad_n) geom.insert(geom.end(), g.begin(), g.end());
    geom.push_back(e.area);
  }
  for (auto& h : d.hinges) {
    for (int v : h.vertices) hv.push_back(uint32_t(v));
    hs.push_back(h.stiffness);
  }
  for (int v : d.free_) {
    rv.push_back(uint32_t(v));
    dm.push_back(7);
    rm.push_back(d.mass_over_h2(v));
  }
  a.push_u32("elem_vertices", ev);
  a.push_f32("elem_geom", f32(geom));
  a.push_u32("hinge_vertices", hv);
  a.push_f32("hinge_stiffness", f32(hs));
  a.push_u32("row_vertex", rv);
  a.push_u32("dof_mask", dm);
  a.push_f32("row_mass", f32(rm));
  for (int v : d.pattern.row_ptr) rp.push_back(uint32_t(v));
  for (int v : d.pattern.col_idx) ci.push_back(uint32_t(v));
  for (int v : d.pattern.diagonal_positions()) di.push_back(uint32_t(v));
  a.push_u32("row_ptr", rp);
  a.push_u32("col_idx", ci);
  a.push_u32("diag_idx", di);
  std::vector<std::vector<uint32_t>> blocks(size_t(d.pattern.blocks()));
  for (int row = 0; row < d.rows(); ++row) blocks[size_t(d.pattern.position(row, row))].push_back(uint32_t(9 * T + 16 * H + row));
  auto pairs = [&](const int* vs, int n, auto index) {
    for (int k = 0; k < n; ++k)
      for (int l = 0; l < n; ++l) {
        int r = d.row_of[vs[k]], c = d.row_of[vs[l]];
        if (r >= 0 && c >= 0) blocks[size_t(d.pattern.position(r, c))].push_back(uint32_t(index(k, l)));
      }
  };
  for (size_t e = 0; e < T; ++e) pairs(d.membranes[e].vertices.data(), 3, [&](int k, int l) { return 9 * e + 3 * k + l; });
  for (size_t h = 0; h < H; ++h) pairs(d.hinges[h].vertices.data(), 4, [&](int k, int l) { return 9 * T + 16 * h + 4 * k + l; });
  push_contributions(a, "block", blocks);
  std::vector<std::vector<uint32_t>> force(size_t(d.rows()));
  for (int row = 0; row < d.rows(); ++row) force[size_t(row)].push_back(uint32_t(3 * T + 4 * H + row));
  for (size_t e = 0; e < T; ++e)
    for (int k = 0; k < 3; ++k)
      if (d.row_of[d.membranes[e].vertices[k]] >= 0) force[size_t(d.row_of[d.membranes[e].vertices[k]])].push_back(uint32_t(3 * e + k));
  for (size_t h = 0; h < H; ++h)
    for (int k = 0; k < 4; ++k)
      if (d.row_of[d.hinges[h].vertices[k]] >= 0) force[size_t(d.row_of[d.hinges[h].vertices[k]])].push_back(uint32_t(3 * T + 4 * h + k));
  push_contributions(a, "force", force);
  for (int v : d.fixed) fx.push_back(uint32_t(v));
  a.push_u32("fixed_vertex", fx);
  Lcg rng(97);
  a.push_f32("kernel_state", f32(flat(bent_state(d, rng))));
  a.push_u32("probe_steps", {});
  a.push_f32("probe_positions", {});
  a.push_f32("probe_velocities", {});
  std::vector<double> col{double(d.contact.colliders.size()), d.contact.barrier.dhat, d.contact.barrier.kappa, 0.0};
  for (auto& c : d.contact.colliders)
    for (double v : c.packed()) col.push_back(v);
  a.push_f32("colliders", f32(col));
  a.push_f32("contact_state", f32(flat(contact_state(d))));
  std::vector<double> um;
  for (int v : d.free_) um.push_back(d.mass[v]);
  a.push_f32("row_unit_mass", f32(um));
  // f64 copies of what the f32 arrays round (start state, element geometry, stiffness, masses).
  a.push_f64("rest_positions_f64", flat(d.start));
  a.push_f64("elem_geom_f64", geom);
  a.push_f64("hinge_stiffness_f64", hs);
  a.push_f64("row_unit_mass_f64", um);
  return a;
}

std::string problem_json(const Drape& d, const std::string& edit, const std::string& manifest, const PtcRules& r) {
  const Material& m = d.material;
  Json mat, newton, pcg, robust, contact, ptc, params;
  mat.number("wale_N_per_m", m.wale).number("course_N_per_m", m.course).number("coupling_N_per_m", m.coupling).number("shear_N_per_m", m.shear);
  newton.number("tolerance", 1e-6).integer("max_iterations", 30).number("armijo", 1e-4).integer("max_halvings", 30);
  pcg.number("tolerance", 1e-7).integer("max_iterations", 20000).integer("replace_every", 50).number("replace_above", 1e-2);
  robust.number("eta_start", 1e-2).number("eta_min", 1e-7).number("eta_max", 1e-2).number("eta_gamma", 0.9).number("eta_safeguard", 0.1)
      .number("update_stop", 1e-4).number("resolution_factor", 2.0).number("mu_start", MU_START).number("mu_cap", MU_CAP).number("kernel_mu", 0.37);
  contact.integer("colliders", (long long)d.contact.colliders.size()).number("dhat_m", d.contact.barrier.dhat)
      .number("kappa", d.contact.barrier.kappa).number("keep_fraction", KEEP_FRACTION);
  ptc.number("h0", r.h0).number("h_max", r.h_max).number("h_min_factor", r.h_min_factor).number("growth", r.growth)
      .number("shrink", r.shrink).integer("max_rejections", r.max_rejections).number("floor_guard", r.floor_guard)
      .number("inner_tolerance", r.inner_tolerance).integer("inner_max_iterations", r.inner_max).integer("max_steps", r.max_steps)
      .number("equilibrium_f64", r.equilibrium).number("equilibrium_f32", 1e-3).integer("stagnation_window", 10)
      .number("stagnation_factor", 0.95).number("gravity_load", gravity_load(d));
  Json j;
  j.text("schema", "e7-problem/1").text("case", "drape-n" + std::to_string(d.mesh.columns)).integer("grid_columns", d.mesh.columns)
      .integer("vertices", (long long)d.mesh.rest.size()).integer("triangles", (long long)d.membranes.size())
      .integer("hinges", (long long)d.hinges.size()).integer("rows", d.rows()).integer("unknowns", 3 * d.rows())
      .integer("blocks", d.pattern.blocks()).integer("steps", 240).number("time_step_s", 1.0 / 240.0)
      .number("gravity_m_per_s2", d.g_norm()).text("tangent", "exact").flag("regularized", true).text("scene", "sphere_on_floor")
      .flag("reference", false).integer("probes", 0).raw("material", mat.render()).raw("newton", newton.render())
      .raw("pcg", pcg.render()).raw("robust", robust.render()).raw("contact", contact.render()).text("edit", edit)
      .raw("gravity_vector", "[" + render_number(d.gravity[0]) + "," + render_number(d.gravity[1]) + "," + render_number(d.gravity[2]) + "]")
      .raw("ptc", ptc.render()).raw("arrays", manifest);
  return j.render();
}

std::map<std::string, std::string> flags(int argc, char** argv) {
  std::map<std::string, std::string> f;
  for (int i = 2; i + 1 < argc; i += 2) {
    std::string k = argv[i];
    if (k.rfind("--", 0) != 0) throw std::runtime_error("expected '--flag value', got " + k);
    f[k.substr(2)] = argv[i + 1];
  }
  return f;
}
std::string need(const std::map<std::string, std::string>& f, const std::string& k) {
  auto it = f.find(k);
  if (it == f.end()) throw std::runtime_error("missing --" + k);
  return it->second;
}
std::string opt(const std::map<std::string, std::string>& f, const std::string& k, const std::string& d) {
  auto it = f.find(k);
  return it == f.end() ? d : it->second;
}

Json run_json(const Drape& d, const PtcRun& run, const std::string& mode, double secs) {
  double load = gravity_load(d);
  int newton = 0, rejected = 0, pcg = 0;
  for (auto& s : run.steps) {
    newton += s.inner_iterations;
    rejected += s.rejected_attempts;
    pcg += s.pcg_iterations;
  }
  Json j;
  j.text("schema", "e7-reference/1").text("mode", mode).flag("converged", run.converged()).text("reason", run.reason)
      .integer("ptc_steps", (long long)run.steps.size()).integer("rejected_attempts", rejected).integer("newton_iterations", newton)
      .integer("pcg_iterations", pcg).number("final_relative_residual", run.final_residual / load)
      .number("final_residual", run.final_residual).number("final_h", run.final_h).number("gravity_load", load)
      .number("static_energy", static_energy(d, run.states.back())).number("seconds", secs);
  return j;
}

int dispatch(int argc, char** argv) {
  if (argc < 2) throw std::runtime_error("missing command");
  std::string cmd = argv[1];
  auto f = flags(argc, argv);
  if (cmd == "e7-generate") {
    std::string dir = need(f, "out"), edit = need(f, "edit");
    mkdir(dir.c_str(), 0755);
    Drape d(reference_scene(std::stoi(opt(f, "n", "33")), edit));
    auto a = problem_arrays(d);
    a.write(dir + "/problem.bin");
    write_text(dir + "/problem.json", problem_json(d, edit, a.manifest(), PtcRules::reference()));
    return 0;
  }
  if (cmd == "sheet-generate") {
    std::string dir = need(f, "out");
    mkdir(dir.c_str(), 0755);
    Drape d(sheet_scene(std::stoi(opt(f, "n", "33")), std::stoull(opt(f, "seed", "0")), std::stod(opt(f, "radius", "0.25")),
                        std::stod(opt(f, "young", "5e5")), opt(f, "plane", "0") == "1"));
    auto a = problem_arrays(d);
    a.write(dir + "/problem.bin");
    write_text(dir + "/problem.json", problem_json(d, "sheet", a.manifest(), PtcRules::doubling(1e-3, 1e-6)));
    return 0;
  }
  if (cmd == "e7-solve" || cmd == "sheet-solve") {
    bool sheet = cmd == "sheet-solve";
    std::string mode = opt(f, "mode", "cold");
    Scene sc = sheet ? sheet_scene(std::stoi(opt(f, "n", "33")), std::stoull(opt(f, "seed", "0")), std::stod(opt(f, "radius", "0.25")),
                                   std::stod(opt(f, "young", "5e5")), opt(f, "plane", "0") == "1")
                     : reference_scene(std::stoi(json_string(read_text(need(f, "dir") + "/problem.json"), "", "case").substr(7)),
                                       json_string(read_text(need(f, "dir") + "/problem.json"), "", "edit"));
    Drape d(sc);
    PtcRules r = sheet ? PtcRules::doubling(1e-3, std::stod(opt(f, "tolerance", "1e-6"))) : PtcRules::reference();
    DirectionSolver dir{opt(f, "direction", sheet ? "pcg" : "cholesky") == "pcg", std::stod(opt(f, "rtol", "1e-6")),
                        std::stoi(opt(f, "maxit", "2000"))};
    double h = r.h0;
    auto x0 = d.start;
    if (f.count("start")) x0 = read_state(f["start"], &h);
    auto t0 = std::chrono::steady_clock::now();
    PtcRun run = ptc_solve(d, x0, h, r, dir, false, opt(f, "progress", "0") == "1");
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::string out = sheet ? need(f, "out") : need(f, "dir") + "/equilibrium-" + mode;
    write_state(out, run.states.back(), run.final_h, false);
    std::string js = run_json(d, run, mode, secs).render();
    if (!sheet) write_text(need(f, "dir") + "/reference-" + mode + ".json", js);
    std::printf("%s\n", js.c_str());
    return run.converged() ? 0 : 1;
  }
  if (cmd == "e7-prolong") {
    std::string text = read_text(need(f, "fine-dir") + "/problem.json");
    Drape d(reference_scene(std::stoi(json_string(text, "", "case").substr(7)), json_string(text, "", "edit")));
    double h = 0;
    auto coarse = read_state(need(f, "coarse"), &h);
    auto fine = prolong(coarse, std::stoi(need(f, "coarse-n")));
    if (fine.size() != d.mesh.rest.size()) throw std::runtime_error("prolonged vertex count does not match the fine mesh");
    int moved = project_out(d, fine);
    std::printf("prolongation: %d vertices projected to d = d_hat\n", moved);
    write_state(need(f, "out"), fine, h, false);
    return 0;
  }
  throw std::runtime_error("unknown command '" + cmd + "'");
}

}  // namespace

int main(int argc, char** argv) {
  try {
    return dispatch(argc, argv);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
