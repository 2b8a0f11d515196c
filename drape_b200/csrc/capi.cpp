// extern "C" boundary of libdrape_b200.so (declarations and reference citations: include/drape_b200.h).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>
#include <memory>
#include <string>
#include <thread>

#include "../../include/drape_b200.h"
#include "context.h"

struct drape_ctx {
  std::unique_ptr<drape::Context> impl;
};

struct drape_network {
  std::unique_ptr<drape::Network> impl;
};

namespace {

thread_local std::string g_create_error;

drape_status fail(drape_ctx* ctx, const std::string& msg, drape_status code) {
  if (ctx && ctx->impl) ctx->impl->last_error = msg;
  else g_create_error = msg;
  return code;
}

template <class F> drape_status guarded(drape_ctx* ctx, F&& fn) {
  if (!ctx || !ctx->impl) return fail(nullptr, "null or destroyed context", DRAPE_E_STATE);
  try {
    return fn(*ctx->impl);
  } catch (const drape::CudaError& e) {
    return fail(ctx, e.what(), e.code == cudaErrorLaunchTimeout ? DRAPE_E_TIMEOUT : DRAPE_E_CUDA);
  } catch (const std::invalid_argument& e) {
    return fail(ctx, e.what(), DRAPE_E_ARG);
  } catch (const std::exception& e) {
    return fail(ctx, e.what(), DRAPE_E_ARG);
  }
}

drape_status create(const drape::HostProblem& p, const drape_options* options, int32_t device, drape_ctx** out) {
  if (!out) return fail(nullptr, "out is null", DRAPE_E_ARG);
  *out = nullptr;
  drape_options opt;
  if (options) opt = *options;
  else drape_default_options(&opt);
  try {
    auto ctx = std::make_unique<drape_ctx>();
    ctx->impl = std::make_unique<drape::Context>(p, opt, device);
    *out = ctx.release();
    return DRAPE_OK;
  } catch (const drape::CudaError& e) {
    return fail(nullptr, e.what(), DRAPE_E_CUDA);
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_ARG);
  }
}

}  // namespace

namespace drape {
void set_global_error(const std::string& message) { g_create_error = message; }
}  // namespace drape

extern "C" {

const char* drape_version(void) { return "drape_b200 0.1 (sm_100a)"; }

void drape_default_options(drape_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->controller = 0;
  o->newton_start = 0;
  o->h0 = 1e-3;
  o->h_max = 1.0;
  o->h_min_factor = 0.1;
  o->growth = 2.0;
  o->shrink = 0.5;
  o->inner_tolerance = 0.1;
  o->inner_max = 10;
  o->max_rejections = 12;
  o->max_steps = 1000;
  o->equilibrium_relative = 0.0;
  o->equilibrium_absolute = 1e-6;
  o->pcg_rtol = 1e-6;
  o->pcg_max_iterations = 2000;
  o->forcing = 0;
  o->replace_every = 0;
  o->replace_above = 1e-2;
  o->refine = 1;
  o->refine_rtol = 0.1;
  o->curvature = 1;
  o->tangent = 0;
  o->preconditioner = 0;
  o->armijo = 1e-4;
  o->max_halvings = 30;
  o->time_budget_s = 0.0;
  o->prolongation = 0;
  o->pcg_single_reduction = 1;
}

drape_status drape_create(const drape_problem_view* v, const drape_options* options, int32_t device, drape_ctx** out) {
  if (!v) return fail(nullptr, "problem view is null", DRAPE_E_ARG);
  if (v->vertices <= 0 || v->rows <= 0 || v->triangles < 0 || v->hinges < 0 || v->blocks <= 0 || v->colliders < 0)
    return fail(nullptr, "negative or empty problem sizes", DRAPE_E_ARG);
  if (!v->start_xyz || !v->row_vertex || !v->row_unit_mass || !v->row_ptr || !v->col_idx ||
      (v->triangles && (!v->elem_vertices || !v->elem_geom)) ||
      (v->hinges && (!v->hinge_vertices || !v->hinge_stiffness)) || (v->colliders && !v->collider_data))
    return fail(nullptr, "a required problem array is null", DRAPE_E_ARG);
  drape::HostProblem p;
  p.columns = v->columns;
  p.V = v->vertices;
  p.T = v->triangles;
  p.H = v->hinges;
  p.R = v->rows;
  p.B = v->blocks;
  p.start.assign(v->start_xyz, v->start_xyz + 3 * size_t(p.V));
  p.tri.assign(v->elem_vertices, v->elem_vertices + 3 * size_t(p.T));
  p.tri_geom.assign(v->elem_geom, v->elem_geom + 7 * size_t(p.T));
  p.hinge.assign(v->hinge_vertices, v->hinge_vertices + 4 * size_t(p.H));
  p.hinge_k.assign(v->hinge_stiffness, v->hinge_stiffness + p.H);
  p.row_vertex.assign(v->row_vertex, v->row_vertex + p.R);
  p.unit_mass.assign(v->row_unit_mass, v->row_unit_mass + p.R);
  p.row_ptr.assign(v->row_ptr, v->row_ptr + p.R + 1);
  p.col_idx.assign(v->col_idx, v->col_idx + p.B);
  p.wale = v->wale;
  p.course = v->course;
  p.coupling = v->coupling;
  p.shear = v->shear;
  for (int k = 0; k < 3; ++k) p.gravity[k] = v->gravity[k];
  p.colliders.assign(v->collider_data, v->collider_data + 8 * size_t(v->colliders));
  p.dhat = v->dhat;
  p.kappa = v->kappa;
  std::string err = drape::validate(p);
  if (!err.empty()) return fail(nullptr, "inconsistent problem: " + err, DRAPE_E_ARG);
  return create(p, options, device, out);
}

drape_status drape_create_from_files(const char* dir, const drape_options* options, int32_t device, drape_ctx** out) {
  if (!dir) return fail(nullptr, "dir is null", DRAPE_E_ARG);
  try {
    return create(drape::read_problem_files(dir), options, device, out);
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_IO);
  }
}

drape_status drape_create_sheet(int32_t columns, uint64_t seed, double radius, double young, int32_t plane,
                                const drape_options* options, int32_t device, drape_ctx** out) {
  if (columns < 3 || !(radius > 0) || !(young > 0)) return fail(nullptr, "invalid sheet parameters", DRAPE_E_ARG);
  try {
    return create(drape::sheet_problem(columns, seed, radius, young, plane != 0), options, device, out);
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_ARG);
  }
}

drape_status drape_create_reference(int32_t columns, const char* edit, const drape_options* options, int32_t device,
                                    drape_ctx** out) {
  if (columns < 3) return fail(nullptr, "invalid column count", DRAPE_E_ARG);
  try {
    return create(drape::reference_problem(columns, edit ? edit : "base"), options, device, out);
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_ARG);
  }
}

drape_status drape_write_sheet_problem(int32_t columns, uint64_t seed, double radius, double young, int32_t plane,
                                       const char* dir) {
  if (!dir || columns < 3 || !(radius > 0) || !(young > 0)) return fail(nullptr, "invalid arguments", DRAPE_E_ARG);
  try {
    drape::write_problem_files(drape::sheet_problem(columns, seed, radius, young, plane != 0), dir);
    return DRAPE_OK;
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_IO);
  }
}

drape_status drape_write_reference_problem(int32_t columns, const char* edit, const char* dir) {
  if (!dir || columns < 3) return fail(nullptr, "invalid arguments", DRAPE_E_ARG);
  try {
    drape::write_problem_files(drape::reference_problem(columns, edit ? edit : "base"), dir);
    return DRAPE_OK;
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_IO);
  }
}

drape_status drape_inspect_problem(const char* dir, int64_t* out) {
  if (!dir || !out) return fail(nullptr, "invalid arguments", DRAPE_E_ARG);
  try {
    drape::HostProblem p = drape::read_problem_files(dir);
    out[0] = p.V;
    out[1] = p.T;
    out[2] = p.H;
    out[3] = p.R;
    out[4] = p.B;
    out[5] = p.collider_count();
    return DRAPE_OK;
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_IO);
  }
}

void drape_destroy(drape_ctx* ctx) { delete ctx; }

const char* drape_last_error(const drape_ctx* ctx) {
  if (ctx && ctx->impl) return ctx->impl->last_error.c_str();
  return g_create_error.c_str();
}

drape_status drape_sizes(const drape_ctx* ctx, int64_t* out) {
  if (!ctx || !ctx->impl || !out) return DRAPE_E_ARG;
  const auto& p = ctx->impl->problem();
  out[0] = p.V;
  out[1] = p.T;
  out[2] = p.H;
  out[3] = p.R;
  out[4] = p.B;
  out[5] = p.collider_count();
  return DRAPE_OK;
}

drape_status drape_set_options(drape_ctx* ctx, const drape_options* options) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!options) return fail(ctx, "options is null", DRAPE_E_ARG);
    if (options->preconditioner != 0 && c.mg_levels() == 0)
      return fail(ctx, "the multilevel preconditioner needs every vertex free on an n x n grid with n - 1 even",
                  DRAPE_E_ARG);
    c.options() = *options;
    c.options_changed();
    return DRAPE_OK;
  });
}

drape_status drape_set_state(drape_ctx* ctx, const double* xyz) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!xyz) return fail(ctx, "xyz is null", DRAPE_E_ARG);
    c.set_positions(xyz);
    return DRAPE_OK;
  });
}

drape_status drape_get_state(const drape_ctx* cctx, double* xyz, double* final_h) {
  auto* ctx = const_cast<drape_ctx*>(cctx);
  return guarded(ctx, [&](drape::Context& c) {
    if (xyz) c.get_positions(xyz);
    if (final_h) *final_h = c.final_h();
    return DRAPE_OK;
  });
}

drape_status drape_solve_equilibrium(drape_ctx* ctx, const double* start, double h0, drape_run_log* log) {
  return guarded(ctx, [&](drape::Context& c) {
    int reason = c.solve_equilibrium(start, h0, log);
    if (reason == 2) return fail(ctx, "the solve stalled: no PTC step could be taken", DRAPE_E_DIVERGED);
    if (reason == 3) return fail(ctx, "time budget exhausted", DRAPE_E_TIMEOUT);
    return DRAPE_OK;
  });
}

drape_status drape_time_step(drape_ctx* ctx, double h, const double* v, double tolerance, int32_t max_iterations,
                             double* v_out, drape_time_step_log* log) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!(h > 0) || !(tolerance > 0) || max_iterations < 1)
      return fail(ctx, "drape_time_step: h and tolerance must be positive and max_iterations at least 1",
                  DRAPE_E_ARG);
    c.time_step(h, v, tolerance, max_iterations, v_out, log);
    return DRAPE_OK;
  });
}

drape_status drape_prolong_state(const drape_ctx* cctx, const double* coarse, int32_t coarse_columns, double* fine_out,
                                 int32_t* moved, int32_t* infeasible) {
  drape_ctx* ctx = const_cast<drape_ctx*>(cctx);
  return guarded(ctx, [&](drape::Context& c) {
    if (!coarse || !fine_out || coarse_columns < 2) return fail(ctx, "drape_prolong_state: invalid arguments", DRAPE_E_ARG);
    const drape::HostProblem& p = c.problem();
    std::vector<double> in(coarse, coarse + 3 * size_t(coarse_columns) * coarse_columns), out;
    std::vector<int> bad;
    int m = 0;
    try {
      m = drape::prolong_state(p, in, coarse_columns, &out, &bad);
    } catch (const std::invalid_argument& e) {
      return fail(ctx, e.what(), DRAPE_E_ARG);
    }
    std::copy(out.begin(), out.end(), fine_out);
    if (moved) *moved = m;
    if (infeasible) *infeasible = int32_t(bad.size());
    return DRAPE_OK;
  });
}

drape_status drape_solve_batch(drape_ctx* const* ctxs, int32_t count, int32_t workers, drape_run_log* logs,
                               drape_status* statuses, double* solve_seconds, double* total_seconds) {
  if (!ctxs || count < 1 || workers < 1)
    return fail(nullptr, "drape_solve_batch: contexts is null, or count or workers is below 1", DRAPE_E_ARG);
  std::vector<drape_ctx*> sorted(ctxs, ctxs + count);
  for (int i = 0; i < count; ++i)
    if (!ctxs[i] || !ctxs[i]->impl)
      return fail(nullptr, "drape_solve_batch: context " + std::to_string(i) + " is null or destroyed", DRAPE_E_STATE);
  std::sort(sorted.begin(), sorted.end());
  if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
    return fail(nullptr, "drape_solve_batch: a context appears twice (one context solves on one thread)", DRAPE_E_ARG);
  std::vector<drape_status> status(count, DRAPE_OK);
  std::vector<double> seconds(count, 0.0);
  std::atomic<int> next{0};
  auto work = [&] {
    for (int i = next++; i < count; i = next++) {
      drape::Context& c = *ctxs[i]->impl;
      drape_run_log local{};
      const auto t0 = std::chrono::steady_clock::now();
      try {
        drape::check(cudaSetDevice(c.device()), "cudaSetDevice");
        c.set_blocking_sync(true);
        status[i] = drape_solve_equilibrium(ctxs[i], nullptr, 0.0, logs ? logs + i : &local);
        c.set_blocking_sync(false);
      } catch (const std::exception& e) {
        c.last_error = e.what();
        status[i] = DRAPE_E_CUDA;
      }
      seconds[i] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
  };
  const auto t_start = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  const int threads = std::min(workers, count);
  for (int t = 0; t < threads; ++t) pool.emplace_back(work);
  for (auto& t : pool) t.join();
  if (total_seconds) *total_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  if (statuses) std::copy(status.begin(), status.end(), statuses);
  if (solve_seconds) std::copy(seconds.begin(), seconds.end(), solve_seconds);
  for (int i = 0; i < count; ++i)
    if (status[i] != DRAPE_OK)
      return fail(nullptr, "drape_solve_batch: drape " + std::to_string(i) + ": " + ctxs[i]->impl->last_error, status[i]);
  return DRAPE_OK;
}

drape_status drape_step_records(const drape_ctx* cctx, drape_step_record* out, int32_t capacity, int32_t* count) {
  auto* ctx = const_cast<drape_ctx*>(cctx);
  return guarded(ctx, [&](drape::Context& c) {
    const auto& s = c.steps();
    if (count) *count = int32_t(s.size());
    for (int32_t i = 0; out && i < capacity && i < int32_t(s.size()); ++i) out[i] = s[size_t(i)];
    return DRAPE_OK;
  });
}

drape_status drape_newton_records(const drape_ctx* cctx, drape_newton_record* out, int32_t capacity, int32_t* count) {
  auto* ctx = const_cast<drape_ctx*>(cctx);
  return guarded(ctx, [&](drape::Context& c) {
    const auto& s = c.newton_records();
    if (count) *count = int32_t(s.size());
    for (int32_t i = 0; out && i < capacity && i < int32_t(s.size()); ++i) out[i] = s[size_t(i)];
    return DRAPE_OK;
  });
}

drape_status drape_probe_begin(drape_ctx* ctx) {
  return guarded(ctx, [&](drape::Context& c) {
    c.probe_begin();
    return DRAPE_OK;
  });
}

drape_status drape_probe_step(drape_ctx* ctx, const double* xyz, double h, int32_t step) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!xyz || !(h > 0)) return fail(ctx, "drape_probe_step needs positions and h > 0", DRAPE_E_ARG);
    c.probe_step(xyz, h, step);
    return DRAPE_OK;
  });
}

drape_status drape_probe_logs(const drape_ctx* cctx, float* iterates, int64_t iterates_capacity,
                              int64_t* iterates_count, float* directions, int64_t directions_capacity,
                              int64_t* directions_count, double* trials, int64_t trials_capacity,
                              int64_t* trials_count) {
  auto* ctx = const_cast<drape_ctx*>(cctx);
  return guarded(ctx, [&](drape::Context& c) {
    auto copy = [](const auto& v, auto* out, int64_t cap, int64_t* count) {
      if (count) *count = int64_t(v.size());
      if (out && cap > 0) std::copy(v.begin(), v.begin() + std::min<int64_t>(cap, int64_t(v.size())), out);
    };
    copy(c.probe_iterates(), iterates, iterates_capacity, iterates_count);
    copy(c.probe_directions(), directions, directions_capacity, directions_count);
    copy(c.probe_trials(), trials, trials_capacity, trials_count);
    return DRAPE_OK;
  });
}

drape_status drape_keep_states(drape_ctx* ctx, int32_t keep) {
  return guarded(ctx, [&](drape::Context& c) {
    c.set_keep_states(keep != 0);
    return DRAPE_OK;
  });
}

drape_status drape_step_states(const drape_ctx* cctx, float* out, int64_t capacity, int64_t* count) {
  auto* ctx = const_cast<drape_ctx*>(cctx);
  return guarded(ctx, [&](drape::Context& c) {
    const auto& s = c.step_states();
    if (count) *count = int64_t(s.size());
    if (out && capacity > 0) std::copy(s.begin(), s.begin() + std::min<int64_t>(capacity, int64_t(s.size())), out);
    return DRAPE_OK;
  });
}

drape_status drape_attempt_records(const drape_ctx* cctx, drape_attempt_record* out, int32_t capacity,
                                   int32_t* count) {
  auto* ctx = const_cast<drape_ctx*>(cctx);
  return guarded(ctx, [&](drape::Context& c) {
    const auto& s = c.attempt_records();
    if (count) *count = int32_t(s.size());
    for (int32_t i = 0; out && i < capacity && i < int32_t(s.size()); ++i) out[i] = s[size_t(i)];
    return DRAPE_OK;
  });
}

drape_status drape_assemble(drape_ctx* ctx, const double* x, const double* x_hat, double h, double mu, int32_t mode,
                            int32_t curvature, double* grad, float* blocks) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!x || (mode == 0 && (!x_hat || !(h > 0))) || (mode != 0 && mode != 1))
      return fail(ctx, "assemble needs x, and x_hat with h > 0 in mode 0", DRAPE_E_ARG);
    c.assemble_host(x, x_hat, h, mu, mode, curvature, grad, blocks);
    return DRAPE_OK;
  });
}

drape_status drape_pcg(drape_ctx* ctx, const float* blocks, const double* rhs, double rtol, int32_t max_iterations,
                       double* solution, int32_t* info, double* relative) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!rhs || !solution || !(rtol > 0) || max_iterations < 1) return fail(ctx, "invalid PCG arguments", DRAPE_E_ARG);
    drape::PcgResult r = c.pcg_host(blocks, rhs, rtol, max_iterations, solution);
    if (info) {
      info[0] = r.iterations;
      info[1] = r.status;
      info[2] = r.replacements;
    }
    if (relative) *relative = r.relative;
    return DRAPE_OK;
  });
}

drape_status drape_network_create(int32_t device, uint64_t seed, drape_network** out) {
  if (!out) return fail(nullptr, "out is null", DRAPE_E_ARG);
  *out = nullptr;
  try {
    auto n = std::make_unique<drape_network>();
    n->impl = std::make_unique<drape::Network>(device, seed);
    *out = n.release();
    return DRAPE_OK;
  } catch (const drape::CudaError& e) {
    return fail(nullptr, e.what(), DRAPE_E_CUDA);
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_ARG);
  }
}

void drape_network_destroy(drape_network* net) { delete net; }

drape_status drape_network_parameters(drape_network* net, float* get, const float* set) {
  if (!net || !net->impl) return fail(nullptr, "null network", DRAPE_E_STATE);
  try {
    if (get) net->impl->get(get);
    if (set) net->impl->set(set);
    return DRAPE_OK;
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_CUDA);
  }
}

drape_status drape_network_save(drape_network* net, const char* path) {
  if (!net || !net->impl || !path) return fail(nullptr, "null network or path", DRAPE_E_ARG);
  std::vector<float> p(drape::kNnParams);
  if (drape_status st = drape_network_parameters(net, p.data(), nullptr)) return st;
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(nullptr, std::string("cannot write ") + path, DRAPE_E_IO);
  const int32_t count = drape::kNnParams;
  bool ok = std::fwrite("DRAPENN1", 1, 8, f) == 8 && std::fwrite(&count, 4, 1, f) == 1 &&
            std::fwrite(p.data(), 4, p.size(), f) == p.size();
  ok = std::fclose(f) == 0 && ok;
  return ok ? DRAPE_OK : fail(nullptr, std::string("short write to ") + path, DRAPE_E_IO);
}

drape_status drape_network_load(drape_network* net, const char* path) {
  if (!net || !net->impl || !path) return fail(nullptr, "null network or path", DRAPE_E_ARG);
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(nullptr, std::string("cannot read ") + path, DRAPE_E_IO);
  char magic[8];
  int32_t count = 0;
  std::vector<float> p(drape::kNnParams);
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "DRAPENN1", 8) == 0 &&
            std::fread(&count, 4, 1, f) == 1 && count == drape::kNnParams &&
            std::fread(p.data(), 4, p.size(), f) == p.size();
  std::fclose(f);
  if (!ok) return fail(nullptr, std::string("not a drape network file of this layout: ") + path, DRAPE_E_IO);
  return drape_network_parameters(net, nullptr, p.data());
}

drape_status drape_set_network(drape_ctx* ctx, drape_network* net) {
  return guarded(ctx, [&](drape::Context& c) {
    c.attach_network(net ? net->impl.get() : nullptr);
    return DRAPE_OK;
  });
}

drape_status drape_network_gradient(drape_ctx* ctx, drape_network* net, const float* blocks, const double* rhs,
                                    const double* solution, double* loss, float* grad, float* factors) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!net || !net->impl || !blocks || !rhs || !solution) return fail(ctx, "invalid arguments", DRAPE_E_ARG);
    const double l = c.network_gradient_host(*net->impl, blocks, rhs, solution, grad, factors);
    if (loss) *loss = l;
    return DRAPE_OK;
  });
}

drape_status drape_network_train(drape_ctx* ctx, drape_network* net, int32_t tuples, const float* const* blocks,
                                 const double* const* rhs, const double* const* solutions, int32_t steps, double lr,
                                 double* losses) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!net || !net->impl || tuples < 1 || steps < 0 || !blocks || !rhs || !solutions || !(lr > 0))
      return fail(ctx, "invalid arguments", DRAPE_E_ARG);
    c.network_train_host(*net->impl, tuples, blocks, rhs, solutions, steps, lr, losses);
    return DRAPE_OK;
  });
}

drape_status drape_spmv_benchmark(int32_t device, int32_t rows, int64_t blocks, const int32_t* row_ptr,
                                  const int32_t* col_idx, const float* values, const float* x, int32_t launches,
                                  int32_t lanes_per_row, int32_t threads, float* y, float* ms) {
  if (rows < 1 || blocks < 1 || !row_ptr || !col_idx || !values || !x || !ms || launches < 1 ||
      (lanes_per_row != 4 && lanes_per_row != 8 && lanes_per_row != 16 && lanes_per_row != 32) ||
      threads < lanes_per_row || threads > 256 || threads % 32)
    return fail(nullptr, "invalid SpMV benchmark arguments", DRAPE_E_ARG);
  if (row_ptr[0] != 0 || row_ptr[rows] != blocks) return fail(nullptr, "row_ptr does not span the blocks", DRAPE_E_ARG);
  for (int64_t k = 0; k < blocks; ++k)
    if (col_idx[k] < 0 || col_idx[k] >= rows) return fail(nullptr, "column index out of range", DRAPE_E_ARG);
  try {
    drape::check(cudaSetDevice(device), "cudaSetDevice");
    std::vector<float4> h0(blocks), h1(blocks), hx(rows);
    std::vector<float> h2(blocks);
    for (int64_t k = 0; k < blocks; ++k) {
      const float* v = values + 9 * k;
      h0[k] = make_float4(v[0], v[1], v[2], v[3]);
      h1[k] = make_float4(v[4], v[5], v[6], v[7]);
      h2[k] = v[8];
    }
    for (int r = 0; r < rows; ++r) hx[r] = make_float4(x[3 * r], x[3 * r + 1], x[3 * r + 2], 0.0f);
    drape::DeviceArray<int> d_rp, d_ci;
    drape::DeviceArray<float4> d_a0, d_a1, d_x, d_y;
    drape::DeviceArray<float> d_a2;
    d_rp.alloc(rows + 1);
    d_ci.alloc(blocks);
    d_a0.alloc(blocks);
    d_a1.alloc(blocks);
    d_a2.alloc(blocks);
    d_x.alloc(rows);
    d_y.alloc(rows);
    d_rp.upload(row_ptr, rows + 1, nullptr);
    d_ci.upload(col_idx, blocks, nullptr);
    d_a0.upload(h0.data(), blocks, nullptr);
    d_a1.upload(h1.data(), blocks, nullptr);
    d_a2.upload(h2.data(), blocks, nullptr);
    d_x.upload(hx.data(), rows, nullptr);
    const drape::DevBsr A{d_a0.ptr, d_a1.ptr, d_a2.ptr};
    cudaEvent_t e0, e1;
    drape::check(cudaEventCreate(&e0), "event");
    drape::check(cudaEventCreate(&e1), "event");
    for (int k = 0; k < 3; ++k)
      drape::check(drape::launch_spmv(rows, d_rp.ptr, d_ci.ptr, A, d_x.ptr, d_y.ptr, lanes_per_row, threads, nullptr),
                   "spmv");
    drape::check(cudaEventRecord(e0), "event");
    for (int k = 0; k < launches; ++k)
      drape::check(drape::launch_spmv(rows, d_rp.ptr, d_ci.ptr, A, d_x.ptr, d_y.ptr, lanes_per_row, threads, nullptr),
                   "spmv");
    drape::check(cudaEventRecord(e1), "event");
    drape::check(cudaEventSynchronize(e1), "synchronize");
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / launches;
    if (y) {
      d_y.download(hx.data(), rows, nullptr);
      drape::check(cudaDeviceSynchronize(), "synchronize");
      for (int r = 0; r < rows; ++r) {
        y[3 * r] = hx[r].x;
        y[3 * r + 1] = hx[r].y;
        y[3 * r + 2] = hx[r].z;
      }
    }
    return DRAPE_OK;
  } catch (const drape::CudaError& e) {
    return fail(nullptr, e.what(), DRAPE_E_CUDA);
  } catch (const std::exception& e) {
    return fail(nullptr, e.what(), DRAPE_E_ARG);
  }
}

drape_status drape_precondition(drape_ctx* ctx, const float* blocks, const double* r, double* z) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!r || !z) return fail(ctx, "invalid arguments", DRAPE_E_ARG);
    if (c.mg_levels() == 0) return fail(ctx, "no multilevel hierarchy for this problem", DRAPE_E_ARG);
    c.precondition_host(blocks, r, z);
    return DRAPE_OK;
  });
}

drape_status drape_multilevel_view(drape_ctx* ctx, int32_t level, int32_t* columns, int32_t* width, double* op,
                                   float* smoother) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!columns) return fail(ctx, "columns is null", DRAPE_E_ARG);
    int w = 0;
    const int n = c.multilevel_view(level, &w, op, smoother);
    if (width) *width = w;
    if (n < 0) return fail(ctx, "no such multilevel level", DRAPE_E_ARG);
    *columns = n;
    return DRAPE_OK;
  });
}

drape_status drape_energy_change(drape_ctx* ctx, const double* x, const double* x_hat, double h, const double* d,
                                 double alpha, int32_t mode, double* out) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!x || !d || !out || (mode == 0 && (!x_hat || !(h > 0)))) return fail(ctx, "invalid arguments", DRAPE_E_ARG);
    *out = c.energy_change_host(x, x_hat, h, d, alpha, mode);
    return DRAPE_OK;
  });
}

drape_status drape_max_step(drape_ctx* ctx, const double* x, const double* d, double* out) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!x || !d || !out) return fail(ctx, "invalid arguments", DRAPE_E_ARG);
    *out = c.max_step_host(x, d);
    return DRAPE_OK;
  });
}

drape_status drape_static_residual(drape_ctx* ctx, const double* x, double* out) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!out) return fail(ctx, "out is null", DRAPE_E_ARG);
    if (x) c.set_positions(x);
    *out = c.static_residual();
    return DRAPE_OK;
  });
}

drape_status drape_static_energy(drape_ctx* ctx, const double* x, double* out) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!out) return fail(ctx, "out is null", DRAPE_E_ARG);
    *out = x ? c.static_energy_host(x) : c.static_energy();
    return DRAPE_OK;
  });
}

drape_status drape_element_terms(drape_ctx* ctx, const double* x, int32_t exact, float* grad, float* hess) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!x) return fail(ctx, "x is null", DRAPE_E_ARG);
    c.element_terms_host(x, exact, grad, hess);
    return DRAPE_OK;
  });
}

drape_status drape_row_terms(drape_ctx* ctx, const double* x, const double* x_hat, const double* row_mass, double mu,
                             int32_t contact, int32_t curvature, float* grad, float* hess) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!x || !x_hat) return fail(ctx, "x and x_hat are required", DRAPE_E_ARG);
    c.row_terms_host(x, x_hat, row_mass, mu, contact, curvature, grad, hess);
    return DRAPE_OK;
  });
}

drape_status drape_time_spmv(drape_ctx* ctx, int32_t launches, int32_t lanes_per_row, int32_t threads, float* ms) {
  return guarded(ctx, [&](drape::Context& c) {
    if (launches < 1 || !ms || threads < 32 || threads % 32 || threads > 1024) return fail(ctx, "invalid arguments", DRAPE_E_ARG);
    *ms = c.time_spmv(launches, lanes_per_row, threads);
    return DRAPE_OK;
  });
}

drape_status drape_time_assembly(drape_ctx* ctx, int32_t launches, float* ms) {
  return guarded(ctx, [&](drape::Context& c) {
    if (launches < 1 || !ms) return fail(ctx, "invalid arguments", DRAPE_E_ARG);
    *ms = c.time_assembly(launches);
    return DRAPE_OK;
  });
}

drape_status drape_time_multilevel(drape_ctx* ctx, int32_t iterations, float* out6) {
  return guarded(ctx, [&](drape::Context& c) {
    if (iterations < 2 || !out6) return fail(ctx, "invalid arguments", DRAPE_E_ARG);
    if (c.mg_levels() == 0) return fail(ctx, "no multilevel hierarchy for this problem", DRAPE_E_ARG);
    c.time_multilevel(iterations, out6, out6 + 3, out6 + 4);
    return DRAPE_OK;
  });
}

drape_status drape_pcg_profile(drape_ctx* ctx, int64_t* out, int32_t clear) {
  return guarded(ctx, [&](drape::Context& c) {
    if (!out) return fail(ctx, "out is null", DRAPE_E_ARG);
    long long t[8];
    c.pcg_profile(t, clear != 0);
    for (int k = 0; k < 7; ++k) out[k] = t[k];
    return DRAPE_OK;
  });
}

}  // extern "C"
