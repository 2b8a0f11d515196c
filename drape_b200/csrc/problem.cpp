// Scene builders and problem-file I/O of the GPU stage. Grid, checkerboard split and hinge orientation follow
// mesh.rs:14-107; element geometry membrane.rs:15-23; hinge stiffness hinge.rs:113-120 with the directional
// bending law material.rs:53-55; lumped masses mesh.rs:30-39; the BSR pattern bsr.rs:12-29 over the coupling
// groups of drape.rs:126-134; the problem files io.rs:5-55 and e3_generate.rs:84-229.
#include "problem.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <sys/stat.h>

namespace drape {

Lcg64::Lcg64(uint64_t seed) : state(seed * 6364136223846793005ULL + 1442695040888963407ULL) {}
double Lcg64::uniform() {
  state = state * 6364136223846793005ULL + 1442695040888963407ULL;
  return double(state >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

namespace {

struct Grid {
  int n;
  std::vector<double> rx, ry;   // rest coordinates
  std::vector<int32_t> tri;     // 3T
  std::vector<int32_t> hinge;   // 4H
};

Grid make_grid(int n, double size) {
  Grid g;
  g.n = n;
  double d = size / (n - 1);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      g.rx.push_back(i * d);
      g.ry.push_back(j * d);
    }
  for (int j = 0; j + 1 < n; ++j)
    for (int i = 0; i + 1 < n; ++i) {
      int a = j * n + i, b = a + 1, c = a + n, e = c + 1;
      // Checkerboard diagonal: even cells split along (i,j)-(i+1,j+1), odd ones along (i+1,j)-(i,j+1).
      int t[6] = {a, b, e, a, e, c};
      int u[6] = {a, b, c, b, e, c};
      const int* s = ((i + j) & 1) ? u : t;
      g.tri.insert(g.tri.end(), s, s + 6);
    }
  // Interior edges: each edge record carries its opposite vertex; edges seen twice become hinges.
  struct EdgeRec {
    int lo, hi, opp;
  };
  std::vector<EdgeRec> recs;
  size_t T = g.tri.size() / 3;
  for (size_t t = 0; t < T; ++t)
    for (int k = 0; k < 3; ++k) {
      int a = g.tri[3 * t + k], b = g.tri[3 * t + (k + 1) % 3], o = g.tri[3 * t + (k + 2) % 3];
      recs.push_back({std::min(a, b), std::max(a, b), o});
    }
  std::stable_sort(recs.begin(), recs.end(), [](const EdgeRec& p, const EdgeRec& q) {
    return p.lo != q.lo ? p.lo < q.lo : p.hi < q.hi;
  });
  std::vector<std::array<int32_t, 4>> hs;
  for (size_t k = 0; k + 1 < recs.size(); ++k) {
    if (recs[k].lo != recs[k + 1].lo || recs[k].hi != recs[k + 1].hi) continue;
    int a = recs[k].lo, b = recs[k].hi, p = recs[k].opp, q = recs[k + 1].opp;
    double cr = (g.rx[b] - g.rx[a]) * (g.ry[p] - g.ry[a]) - (g.ry[b] - g.ry[a]) * (g.rx[p] - g.rx[a]);
    hs.push_back(cr > 0.0 ? std::array<int32_t, 4>{p, q, a, b} : std::array<int32_t, 4>{q, p, a, b});
    ++k;
  }
  std::sort(hs.begin(), hs.end());
  for (auto& h : hs) g.hinge.insert(g.hinge.end(), h.begin(), h.end());
  return g;
}

// Element geometry, masses, hinge stiffness and the BSR pattern of a grid whose every vertex is free.
void fill(HostProblem& p, const Grid& g, double density, double bend_x_dir, double bend_y_dir) {
  p.columns = g.n;
  p.V = int(g.rx.size());
  p.T = int(g.tri.size() / 3);
  p.H = int(g.hinge.size() / 4);
  p.R = p.V;
  p.tri = g.tri;
  p.hinge = g.hinge;
  std::vector<double> area(p.V, 0.0);
  p.tri_geom.resize(7 * size_t(p.T));
  for (int t = 0; t < p.T; ++t) {
    int v0 = g.tri[3 * t], v1 = g.tri[3 * t + 1], v2 = g.tri[3 * t + 2];
    double a = g.rx[v1] - g.rx[v0], b = g.rx[v2] - g.rx[v0], c = g.ry[v1] - g.ry[v0], d = g.ry[v2] - g.ry[v0];
    double det = a * d - b * c;
    double g1x = d / det, g1y = -b / det, g2x = -c / det, g2y = a / det;
    double* o = &p.tri_geom[7 * size_t(t)];
    o[0] = -g1x - g2x;
    o[1] = -g1y - g2y;
    o[2] = g1x;
    o[3] = g1y;
    o[4] = g2x;
    o[5] = g2y;
    o[6] = 0.5 * std::fabs(det);
    for (int k = 0; k < 3; ++k) area[g.tri[3 * t + k]] += o[6] / 3.0;
  }
  p.hinge_k.resize(p.H);
  for (int h = 0; h < p.H; ++h) {
    const int32_t* v = &g.hinge[4 * size_t(h)];
    double ex = g.rx[v[3]] - g.rx[v[2]], ey = g.ry[v[3]] - g.ry[v[2]];
    double len2 = ex * ex + ey * ey, len = std::hypot(ex, ey);
    double dx = ex / len, dy = ey / len;
    double bending = bend_x_dir * dy * dy + bend_y_dir * dx * dx;
    auto tri_area = [&](int w) {
      return 0.5 * std::fabs((g.rx[v[2]] - g.rx[w]) * (g.ry[v[3]] - g.ry[w]) - (g.ry[v[2]] - g.ry[w]) * (g.rx[v[3]] - g.rx[w]));
    };
    p.hinge_k[h] = bending * 3.0 * len2 / (tri_area(v[0]) + tri_area(v[1]));
  }
  p.row_vertex.resize(p.R);
  p.unit_mass.resize(p.R);
  for (int r = 0; r < p.R; ++r) {
    p.row_vertex[r] = r;
    p.unit_mass[r] = density * area[r];
  }
  std::vector<std::vector<int32_t>> cols(p.R);
  for (int r = 0; r < p.R; ++r) cols[r].push_back(r);
  auto couple = [&](const int32_t* v, int k) {
    for (int a = 0; a < k; ++a)
      for (int b = 0; b < k; ++b) cols[v[a]].push_back(v[b]);
  };
  for (int t = 0; t < p.T; ++t) couple(&g.tri[3 * size_t(t)], 3);
  for (int h = 0; h < p.H; ++h) couple(&g.hinge[4 * size_t(h)], 4);
  p.row_ptr.assign(1, 0);
  p.col_idx.clear();
  for (auto& c : cols) {
    std::sort(c.begin(), c.end());
    c.erase(std::unique(c.begin(), c.end()), c.end());
    p.col_idx.insert(p.col_idx.end(), c.begin(), c.end());
    p.row_ptr.push_back(int32_t(p.col_idx.size()));
  }
  p.B = int(p.col_idx.size());
}

void push_collider(HostProblem& p, int kind, double a, double b, double c, double w) {
  double v[8] = {double(kind), a, b, c, w, 0, 0, 0};
  p.colliders.insert(p.colliders.end(), v, v + 8);
}

}  // namespace

HostProblem sheet_problem(int columns, uint64_t seed, double radius, double young, bool with_plane, double plane_y,
                          double poisson, double kb) {
  if (columns < 3) throw std::runtime_error("a sheet needs at least 3 columns");
  HostProblem p;
  Grid g = make_grid(columns, 1.0);
  const double thickness = 5e-4, density = 0.15;
  double c = thickness * young / (1.0 - poisson * poisson);
  p.wale = p.course = c;
  p.coupling = poisson * c;
  p.shear = thickness * young / (2.0 * (1.0 + poisson));
  fill(p, g, density, kb, kb);
  p.gravity[0] = 0;
  p.gravity[1] = -9.81;
  p.gravity[2] = 0;
  push_collider(p, 2, 0, 0, 0, radius);
  if (with_plane) push_collider(p, 1, 0, 1, 0, plane_y);
  p.dhat = 2e-3;
  p.kappa = 1e3;
  Lcg64 rng(seed);
  p.start.resize(3 * size_t(p.V));
  for (int v = 0; v < p.V; ++v) {
    p.start[3 * v] = g.rx[v] - 0.5;
    p.start[3 * v + 1] = 0.35 + 1e-5 * rng.uniform();
    p.start[3 * v + 2] = g.ry[v] - 0.5;
  }
  return p;
}

HostProblem reference_problem(int columns, const std::string& edit) {
  double mat = 1.0, radius_f = 1.0, rest_f = 1.0;
  if (edit == "w1") mat = 1.25;
  else if (edit == "w2") radius_f = 0.96;
  else if (edit == "w3") rest_f = 1.03;
  else if (edit != "base") throw std::runtime_error("unknown edit '" + edit + "' (base|w1|w2|w3)");
  const double sheet = 0.5, density = 0.13;
  Grid g = make_grid(columns, sheet);
  if (rest_f != 1.0)
    for (size_t v = 0; v < g.rx.size(); ++v) {
      g.rx[v] = 0.25 + rest_f * (g.rx[v] - 0.25);
      g.ry[v] = 0.25 + rest_f * (g.ry[v] - 0.25);
    }
  HostProblem p;
  p.wale = 1000.0 * mat;
  p.course = 300.0 * mat;
  p.coupling = 100.0 * mat;
  p.shear = 50.0 * mat;
  fill(p, g, density, 2.0e-6 * mat, 1.0e-6 * mat);
  double radius = 0.125 * radius_f, dhat = 5e-4;
  push_collider(p, 1, 0, 0, 1, 0.0);
  push_collider(p, 2, 0.25, 0.25, radius, radius);
  double heaviest = *std::max_element(p.unit_mass.begin(), p.unit_mass.end());
  // kappa that balances the heaviest vertex's weight at d = d_hat/2: m g / |b'(d_hat/2)| with kappa = 1.
  double d = 0.5 * dhat, t = d - dhat;
  double unit_slope = std::fabs(2.0 * t * std::log(d / dhat) + t * t / d);
  p.dhat = dhat;
  p.kappa = heaviest * 9.81 / unit_slope;
  p.gravity[0] = p.gravity[1] = 0;
  p.gravity[2] = -9.81;
  double lift = 2.0 * radius + 2.0 * dhat;
  p.start.resize(3 * size_t(p.V));
  for (int v = 0; v < p.V; ++v) {
    p.start[3 * v] = g.rx[v];
    p.start[3 * v + 1] = g.ry[v];
    p.start[3 * v + 2] = lift;
  }
  return p;
}

std::string validate(const HostProblem& p) {
  auto bad = [](const std::string& m) { return m; };
  if (p.V <= 0 || p.R <= 0 || p.R > p.V) return bad("vertex/row counts");
  if (p.start.size() != 3 * size_t(p.V)) return bad("start size");
  if (p.tri.size() != 3 * size_t(p.T) || p.tri_geom.size() != 7 * size_t(p.T)) return bad("triangle arrays");
  if (p.hinge.size() != 4 * size_t(p.H) || p.hinge_k.size() != size_t(p.H)) return bad("hinge arrays");
  if (p.row_vertex.size() != size_t(p.R) || p.unit_mass.size() != size_t(p.R)) return bad("row arrays");
  if (p.row_ptr.size() != size_t(p.R) + 1 || p.row_ptr[0] != 0 || p.row_ptr[p.R] != p.B ||
      p.col_idx.size() != size_t(p.B))
    return bad("BSR pattern sizes");
  for (int v : p.tri)
    if (v < 0 || v >= p.V) return bad("triangle vertex out of range");
  for (int v : p.hinge)
    if (v < 0 || v >= p.V) return bad("hinge vertex out of range");
  for (int v : p.row_vertex)
    if (v < 0 || v >= p.V) return bad("row vertex out of range");
  for (int r = 0; r < p.R; ++r) {
    if (p.row_ptr[r + 1] < p.row_ptr[r]) return bad("row_ptr not monotone");
    bool diag = false;
    for (int k = p.row_ptr[r]; k < p.row_ptr[r + 1]; ++k) {
      if (p.col_idx[k] < 0 || p.col_idx[k] >= p.R) return bad("column out of range");
      if (k > p.row_ptr[r] && p.col_idx[k] <= p.col_idx[k - 1]) return bad("columns not sorted");
      diag |= p.col_idx[k] == r;
    }
    if (!diag) return bad("row without a diagonal block");
  }
  for (int k = 0; k < p.collider_count(); ++k) {
    int kind = int(p.colliders[8 * k]);
    if (kind != 1 && kind != 2) return bad("unknown collider kind");
  }
  if (p.collider_count() > 0 && !(p.dhat > 0 && p.kappa > 0)) return bad("barrier parameters");
  return {};
}

// ---------------------------------------------------------------- problem files
namespace {

std::string read_all(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error(path + ": cannot read");
  std::stringstream s;
  s << f.rdbuf();
  return s.str();
}

// The first "key": after the first "anchor" (the reference's flat key scanner, jsonscan.rs:3-26).
std::string scan(const std::string& text, const std::string& anchor, const std::string& key) {
  size_t start = 0;
  if (!anchor.empty()) {
    start = text.find("\"" + anchor + "\"");
    if (start == std::string::npos) return {};
  }
  std::string m = "\"" + key + "\":";
  size_t at = text.find(m, start);
  if (at == std::string::npos) return {};
  at += m.size();
  while (at < text.size() && std::isspace(static_cast<unsigned char>(text[at]))) ++at;
  if (at < text.size() && text[at] == '"') return text.substr(at + 1, text.find('"', at + 1) - at - 1);
  if (at < text.size() && text[at] == '[') return text.substr(at, text.find(']', at) - at + 1);
  size_t end = text.find_first_of(",}\n", at);
  return text.substr(at, end - at);
}
double number(const std::string& t, const std::string& a, const std::string& k) {
  std::string v = scan(t, a, k);
  if (v.empty() || v == "null") return NAN;
  return std::strtod(v.c_str(), nullptr);
}

struct Manifest {
  std::string text, bytes;
  bool find(const std::string& name, std::string& dtype, size_t& offset, size_t& length) const {
    std::string key = "\"name\":\"" + name + "\"";
    size_t at = text.find(key);
    if (at == std::string::npos) return false;
    size_t end = text.find('}', at);
    std::string entry = text.substr(at, end - at);
    dtype = scan(entry, "", "dtype");
    offset = size_t(std::strtoull(scan("{" + entry, "", "offset").c_str(), nullptr, 10));
    length = size_t(std::strtoull(scan("{" + entry, "", "length").c_str(), nullptr, 10));
    size_t width = dtype == "f64" ? 8 : 4;
    if (offset + width * length > bytes.size()) throw std::runtime_error("array '" + name + "' runs past problem.bin");
    return true;
  }
  template <class T> std::vector<T> get(const std::string& name, bool required = true) const {
    std::string dtype;
    size_t off = 0, len = 0;
    if (!find(name, dtype, off, len)) {
      if (required) throw std::runtime_error("array '" + name + "' missing from the manifest");
      return {};
    }
    std::vector<T> out(len);
    const char* src = bytes.data() + off;
    for (size_t i = 0; i < len; ++i) {
      if (dtype == "f64") {
        double d;
        std::memcpy(&d, src + 8 * i, 8);
        out[i] = T(d);
      } else if (dtype == "f32") {
        float f;
        std::memcpy(&f, src + 4 * i, 4);
        out[i] = T(f);
      } else {
        uint32_t u;
        std::memcpy(&u, src + 4 * i, 4);
        out[i] = T(u);
      }
    }
    return out;
  }
  template <class T> std::vector<T> prefer(const std::string& wide, const std::string& narrow) const {
    auto w = get<T>(wide, false);
    return w.empty() ? get<T>(narrow) : w;
  }
};

}  // namespace

HostProblem read_problem_files(const std::string& dir) {
  std::string text = read_all(dir + "/problem.json");
  Manifest m{text.substr(text.find("\"arrays\"")), read_all(dir + "/problem.bin")};
  HostProblem p;
  p.columns = int(number(text, "", "grid_columns"));
  p.V = int(number(text, "", "vertices"));
  p.T = int(number(text, "", "triangles"));
  p.H = int(number(text, "", "hinges"));
  p.R = int(number(text, "", "rows"));
  p.B = int(number(text, "", "blocks"));
  p.wale = number(text, "material", "wale_N_per_m");
  p.course = number(text, "material", "course_N_per_m");
  p.coupling = number(text, "material", "coupling_N_per_m");
  p.shear = number(text, "material", "shear_N_per_m");
  std::string gv = scan(text, "", "gravity_vector");
  if (!gv.empty()) {
    std::sscanf(gv.c_str(), "[%lf,%lf,%lf]", &p.gravity[0], &p.gravity[1], &p.gravity[2]);
  } else {
    p.gravity[0] = p.gravity[1] = 0;
    p.gravity[2] = -number(text, "", "gravity_m_per_s2");
  }
  p.start = m.prefer<double>("rest_positions_f64", "rest_positions");
  p.tri = m.get<int32_t>("elem_vertices");
  p.tri_geom = m.prefer<double>("elem_geom_f64", "elem_geom");
  p.hinge = m.get<int32_t>("hinge_vertices");
  p.hinge_k = m.prefer<double>("hinge_stiffness_f64", "hinge_stiffness");
  p.row_vertex = m.get<int32_t>("row_vertex");
  p.unit_mass = m.prefer<double>("row_unit_mass_f64", "row_unit_mass");
  p.row_ptr = m.get<int32_t>("row_ptr");
  p.col_idx = m.get<int32_t>("col_idx");
  auto col = m.get<double>("colliders", false);
  if (col.size() >= 4) {
    int count = int(col[0]);
    p.dhat = col[1];
    p.kappa = col[2];
    if (col.size() < 4 + 8 * size_t(count)) throw std::runtime_error("colliders array too short");
    p.colliders.assign(col.begin() + 4, col.begin() + 4 + 8 * count);
    // The packed f32 colliders carry sphere centres and radii rounded; the JSON's d_hat and kappa are f64.
    double dh = number(text, "contact", "dhat_m"), ka = number(text, "contact", "kappa");
    if (std::isfinite(dh)) p.dhat = dh;
    if (std::isfinite(ka)) p.kappa = ka;
  }
  std::string err = validate(p);
  if (!err.empty()) throw std::runtime_error(dir + ": inconsistent problem (" + err + ")");
  return p;
}

std::vector<double> read_named_array(const std::string& json_path, const std::string& bin_path,
                                     const std::string& name) {
  std::string text = read_all(json_path);
  const size_t at = text.find("\"arrays\"");
  if (at == std::string::npos) return {};
  Manifest m{text.substr(at), read_all(bin_path)};
  return m.get<double>(name, false);
}

std::vector<double> read_problem_array(const std::string& dir, const std::string& name) {
  return read_named_array(dir + "/problem.json", dir + "/problem.bin", name);
}

void write_problem_files(const HostProblem& p, const std::string& dir) {
  mkdir(dir.c_str(), 0755);
  std::string bytes, manifest = "[";
  auto push = [&](const std::string& name, const char* dtype, const void* data, size_t count, size_t width) {
    while (bytes.size() % 8) bytes.push_back('\0');
    size_t off = bytes.size();
    bytes.append(static_cast<const char*>(data), count * width);
    if (manifest.size() > 1) manifest += ",";
    manifest += "{\"name\":\"" + name + "\",\"dtype\":\"" + dtype + "\",\"length\":" + std::to_string(count) +
                ",\"offset\":" + std::to_string(off) + "}";
  };
  auto f32 = [](const std::vector<double>& v) { return std::vector<float>(v.begin(), v.end()); };
  auto u32 = [](const std::vector<int32_t>& v) { return std::vector<uint32_t>(v.begin(), v.end()); };
  auto rp = f32(p.start), geom = f32(p.tri_geom), hk = f32(p.hinge_k), um = f32(p.unit_mass);
  auto tv = u32(p.tri), hv = u32(p.hinge), rv = u32(p.row_vertex), rptr = u32(p.row_ptr), ci = u32(p.col_idx);
  std::vector<float> col{float(p.collider_count()), float(p.dhat), float(p.kappa), 0.0f};
  for (double c : p.colliders) col.push_back(float(c));
  push("rest_positions", "f32", rp.data(), rp.size(), 4);
  push("elem_vertices", "u32", tv.data(), tv.size(), 4);
  push("elem_geom", "f32", geom.data(), geom.size(), 4);
  push("hinge_vertices", "u32", hv.data(), hv.size(), 4);
  push("hinge_stiffness", "f32", hk.data(), hk.size(), 4);
  push("row_vertex", "u32", rv.data(), rv.size(), 4);
  push("row_ptr", "u32", rptr.data(), rptr.size(), 4);
  push("col_idx", "u32", ci.data(), ci.size(), 4);
  push("colliders", "f32", col.data(), col.size(), 4);
  push("row_unit_mass", "f32", um.data(), um.size(), 4);
  push("rest_positions_f64", "f64", p.start.data(), p.start.size(), 8);
  push("elem_geom_f64", "f64", p.tri_geom.data(), p.tri_geom.size(), 8);
  push("hinge_stiffness_f64", "f64", p.hinge_k.data(), p.hinge_k.size(), 8);
  push("row_unit_mass_f64", "f64", p.unit_mass.data(), p.unit_mass.size(), 8);
  manifest += "]";
  char g[160];
  std::snprintf(g, sizeof g, "[%.17g,%.17g,%.17g]", p.gravity[0], p.gravity[1], p.gravity[2]);
  double gn = std::sqrt(p.gravity[0] * p.gravity[0] + p.gravity[1] * p.gravity[1] + p.gravity[2] * p.gravity[2]);
  char head[1024];
  std::snprintf(head, sizeof head,
                "{\"schema\":\"e7-problem/1\",\"case\":\"drape-n%d\",\"grid_columns\":%d,\"vertices\":%d,\"triangles\":%d,"
                "\"hinges\":%d,\"rows\":%d,\"unknowns\":%d,\"blocks\":%d,\"gravity_m_per_s2\":%.17g,\"gravity_vector\":%s,"
                "\"material\":{\"wale_N_per_m\":%.17g,\"course_N_per_m\":%.17g,\"coupling_N_per_m\":%.17g,"
                "\"shear_N_per_m\":%.17g},\"contact\":{\"colliders\":%d,\"dhat_m\":%.17g,\"kappa\":%.17g},",
                p.columns, p.columns, p.V, p.T, p.H, p.R, 3 * p.R, p.B, gn, g, p.wale, p.course, p.coupling, p.shear,
                p.collider_count(), p.dhat, p.kappa);
  std::ofstream(dir + "/problem.bin", std::ios::binary) << bytes;
  std::ofstream(dir + "/problem.json") << head << "\"arrays\":" << manifest << "}";
}

std::string read_text_file(const std::string& path) { return read_all(path); }

double json_number(const std::string& text, const std::string& anchor, const std::string& key) {
  return number(text, anchor, key);
}

namespace {

// Distance to collider `c` (8 doubles: kind 1 plane n.x = w, 2 sphere |x - c| = w) and its gradient.
double collider_distance(const double* c, const double x[3], double n[3]) {
  if (c[0] == 1.0) {
    for (int k = 0; k < 3; ++k) n[k] = c[1 + k];
    return c[1] * x[0] + c[2] * x[1] + c[3] * x[2] - c[4];
  }
  double q[3] = {x[0] - c[1], x[1] - c[2], x[2] - c[3]};
  const double len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  for (int k = 0; k < 3; ++k) n[k] = q[k] / len;
  return len - c[4];
}

}  // namespace

int prolong_state(const HostProblem& fine, const std::vector<double>& coarse, int coarse_columns,
                  std::vector<double>* out, std::vector<int>* infeasible) {
  const int nc = coarse_columns, nf = 2 * (coarse_columns - 1) + 1;
  if (nc < 2 || coarse.size() != size_t(3) * nc * nc)
    throw std::invalid_argument("prolong: the coarse state does not hold " + std::to_string(nc) + "^2 vertices");
  if (size_t(nf) * nf != size_t(fine.V))
    throw std::invalid_argument("prolong: prolonged " + std::to_string(nf * nf) + " vertices, the fine mesh has " +
                                std::to_string(fine.V));
  out->assign(3 * size_t(fine.V), 0.0);
  for (int v = 0; v < fine.V; ++v) {
    const int i = v % nf, j = v / nf;
    const int i0 = i / 2, i1 = (i + 1) / 2, j0 = j / 2, j1 = (j + 1) / 2;
    const int corners[4] = {j0 * nc + i0, j0 * nc + i1, j1 * nc + i0, j1 * nc + i1};
    for (int k = 0; k < 3; ++k) {
      double sum = 0.0;
      for (int c : corners) sum += coarse[3 * size_t(c) + k];
      (*out)[3 * size_t(v) + k] = sum / 4.0;
    }
  }
  int moved = 0;
  for (int v = 0; v < fine.V; ++v) {
    double* x = out->data() + 3 * size_t(v);
    const double before[3] = {x[0], x[1], x[2]};
    for (int c = 0; c < fine.collider_count(); ++c) {
      double n[3];
      const double d = collider_distance(fine.colliders.data() + 8 * size_t(c), x, n);
      if (d < fine.dhat)
        for (int k = 0; k < 3; ++k) x[k] += (fine.dhat - d) * n[k];
    }
    moved += (x[0] != before[0] || x[1] != before[1] || x[2] != before[2]) ? 1 : 0;
  }
  if (infeasible) {
    infeasible->clear();
    for (int v = 0; v < fine.V; ++v) {
      double dmin = INFINITY;
      for (int c = 0; c < fine.collider_count(); ++c) {
        double n[3];
        dmin = std::min(dmin, collider_distance(fine.colliders.data() + 8 * size_t(c), out->data() + 3 * size_t(v), n));
      }
      if (dmin <= 0.0) infeasible->push_back(v);
    }
  }
  return moved;
}

}  // namespace drape
