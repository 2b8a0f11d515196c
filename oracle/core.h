// Test infrastructure only: the f64 oracle of the quasi-static drape path. Nothing in the product
// (drape_b200/) links or calls this code; tests/, the smoke check and bench.py's CPU-baseline leg do.
//
// core.h: the element-level math of the reference oracle crate (engine/oracle/src), restated in C++17.
//   linalg.rs:1-60, rng.rs:2-13, mesh.rs:14-107, material.rs:4-56, membrane.rs:15-140, dual.rs:6-90,
//   hinge.rs:13-120, contact.rs:5-177, bsr.rs:4-93, band.rs:4-103, pcg.rs:37-281.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace oracle {

using Vec3 = std::array<double, 3>;
using Mat3 = std::array<std::array<double, 3>, 3>;
using Vec2 = std::array<double, 2>;

// ---------------------------------------------------------------- linalg (linalg.rs:1-60)
inline Vec3 add(Vec3 a, Vec3 b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline Vec3 sub(Vec3 a, Vec3 b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline Vec3 scale(Vec3 a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
inline double dot(Vec3 a, Vec3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline Vec3 cross(Vec3 a, Vec3 b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline double norm(Vec3 a) { return std::sqrt(dot(a, a)); }
inline Mat3 outer(Vec3 a, Vec3 b) {
  Mat3 m{};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m[r][c] = a[r] * b[c];
  return m;
}
inline void mat_add_scaled(Mat3& t, const Mat3& s, double f) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) t[r][c] += s[r][c] * f;
}
inline Mat3 identity_scaled(double s) { return Mat3{{{s, 0, 0}, {0, s, 0}, {0, 0, s}}}; }
inline double vector_norm(const std::vector<double>& v) {
  double s = 0;
  for (double x : v) s += x * x;
  return std::sqrt(s);
}
inline double difference_norm(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
  for (size_t i = 0; i < a.size(); ++i) s += (a[i] - b[i]) * (a[i] - b[i]);
  return std::sqrt(s);
}

// ---------------------------------------------------------------- rng (rng.rs:2-13)
// 64-bit LCG, uniform in [-1, 1); the multiplier/increment are Knuth's MMIX constants the reference uses.
struct Lcg {
  uint64_t s;
  explicit Lcg(uint64_t seed) : s(seed * 6364136223846793005ULL + 1442695040888963407ULL) {}
  double uniform() {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    return double(s >> 11) / double(1ULL << 53) * 2.0 - 1.0;
  }
};

// ---------------------------------------------------------------- mesh (mesh.rs:14-107)
struct Mesh {
  int columns = 0, rows = 0;
  double width = 0, height = 0;
  std::vector<Vec2> rest;
  std::vector<std::array<int, 3>> triangles;
  std::vector<std::array<int, 4>> hinges;  // [left opposite, right opposite, edge a, edge b]

  static Mesh grid(int columns, int rows, double width, double height);
  bool is_boundary(int v) const {
    int i = v % columns, j = v / columns;
    return i == 0 || j == 0 || i == columns - 1 || j == rows - 1;
  }
  std::vector<double> vertex_areas() const;
};

inline double cross2(Vec2 a, Vec2 b) { return a[0] * b[1] - a[1] * b[0]; }
inline Vec2 sub2(Vec2 a, Vec2 b) { return {a[0] - b[0], a[1] - b[1]}; }
inline double rest_area(const std::vector<Vec2>& rest, const std::array<int, 3>& t) {
  return 0.5 * std::fabs(cross2(sub2(rest[t[1]], rest[t[0]]), sub2(rest[t[2]], rest[t[0]])));
}

// mesh.rs:57-67: checkerboard diagonal.
inline std::array<std::array<int, 3>, 2> cell_triangles(int columns, int i, int j) {
  int v00 = j * columns + i, v10 = v00 + 1, v01 = v00 + columns, v11 = v01 + 1;
  if ((i + j) % 2 == 0) return {{{v00, v10, v11}, {v00, v11, v01}}};
  return {{{v00, v10, v01}, {v10, v11, v01}}};
}

inline std::vector<std::array<int, 4>> interior_hinges(const std::vector<Vec2>& rest,
                                                       const std::vector<std::array<int, 3>>& tris) {
  std::map<std::pair<int, int>, std::vector<int>> edges;
  for (auto& t : tris)
    for (int k = 0; k < 3; ++k) {
      int a = t[k], b = t[(k + 1) % 3], o = t[(k + 2) % 3];
      edges[{std::min(a, b), std::max(a, b)}].push_back(o);
    }
  std::vector<std::array<int, 4>> hinges;
  for (auto& [key, opp] : edges) {
    if (opp.size() != 2) continue;
    int a = key.first, b = key.second;
    bool left = cross2(sub2(rest[b], rest[a]), sub2(rest[opp[0]], rest[a])) > 0.0;
    hinges.push_back(left ? std::array<int, 4>{opp[0], opp[1], a, b} : std::array<int, 4>{opp[1], opp[0], a, b});
  }
  std::sort(hinges.begin(), hinges.end());
  return hinges;
}

inline Mesh Mesh::grid(int columns, int rows, double width, double height) {
  Mesh m;
  m.columns = columns;
  m.rows = rows;
  m.width = width;
  m.height = height;
  double dx = width / (columns - 1), dy = height / (rows - 1);
  for (int j = 0; j < rows; ++j)
    for (int i = 0; i < columns; ++i) m.rest.push_back({i * dx, j * dy});
  for (int j = 0; j < rows - 1; ++j)
    for (int i = 0; i < columns - 1; ++i)
      for (auto& t : cell_triangles(columns, i, j)) m.triangles.push_back(t);
  m.hinges = interior_hinges(m.rest, m.triangles);
  return m;
}

inline std::vector<double> Mesh::vertex_areas() const {
  std::vector<double> areas(rest.size(), 0.0);
  for (auto& t : triangles) {
    double a = rest_area(rest, t);
    for (int v : t) areas[v] += a / 3.0;
  }
  return areas;
}

// ---------------------------------------------------------------- material (material.rs:4-56)
struct Material {
  double wale, course, coupling, shear, bend_wale, bend_course, density;
  static Material knit_baseline() { return {1000.0, 300.0, 100.0, 50.0, 2.0e-6, 1.0e-6, 0.13}; }
  // Isotropic plane-stress St. Venant–Kirchhoff sheet mapped onto the orthotropic law:
  // wale = course = tE/(1-nu^2), coupling = nu*wale, shear = tE/(2(1+nu)), bend = k_b.
  static Material isotropic(double young, double poisson, double thickness, double kb, double density) {
    double c = thickness * young / (1.0 - poisson * poisson);
    return {c, c, poisson * c, thickness * young / (2.0 * (1.0 + poisson)), kb, kb, density};
  }
  std::array<double, 3> stress(std::array<double, 3> e) const {
    return {wale * e[0] + coupling * e[1], course * e[1] + coupling * e[0], 2.0 * shear * e[2]};
  }
  double energy_density(std::array<double, 3> e) const {
    return 0.5 * wale * e[0] * e[0] + 0.5 * course * e[1] * e[1] + coupling * e[0] * e[1] + 2.0 * shear * e[2] * e[2];
  }
  bool is_convex() const { return coupling * coupling < wale * course && shear > 0.0; }
  double hinge_bending(Vec2 d) const { return bend_wale * d[1] * d[1] + bend_course * d[0] * d[0]; }
};

// ---------------------------------------------------------------- membrane (membrane.rs:15-140)
using ElementHessian3 = std::array<std::array<Mat3, 3>, 3>;

inline std::array<double, 2> principal_direction(double a, double b, double c, double eig) {
  Vec2 first{b, eig - a}, second{eig - c, b};
  Vec2 pick = std::hypot(first[0], first[1]) >= std::hypot(second[0], second[1]) ? first : second;
  double len = std::hypot(pick[0], pick[1]);
  if (len == 0.0) return a >= c ? Vec2{1.0, 0.0} : Vec2{0.0, 1.0};
  return {pick[0] / len, pick[1] / len};
}

// membrane.rs:116-129: positive part of the 2x2 stress so the geometric block stays PSD.
inline std::array<double, 3> clamp_negative_stress(std::array<double, 3> s) {
  double a = s[0], c = s[1], b = s[2];
  double mean = 0.5 * (a + c), radius = std::sqrt(0.25 * (a - c) * (a - c) + b * b);
  double high = mean + radius, low = mean - radius;
  if (low >= 0.0) return s;
  if (high <= 0.0) return {0.0, 0.0, 0.0};
  Vec2 v = principal_direction(a, b, c, high);
  return {high * v[0] * v[0], high * v[1] * v[1], high * v[0] * v[1]};
}

struct MembraneElement {
  std::array<int, 3> vertices;
  std::array<Vec2, 3> grad_n;
  double area;

  static MembraneElement make(std::array<int, 3> v, const std::vector<Vec2>& rest) {
    Vec2 p0 = rest[v[0]], p1 = rest[v[1]], p2 = rest[v[2]];
    double dm[2][2] = {{p1[0] - p0[0], p2[0] - p0[0]}, {p1[1] - p0[1], p2[1] - p0[1]}};
    double det = dm[0][0] * dm[1][1] - dm[0][1] * dm[1][0];
    Vec2 g1{dm[1][1] / det, -dm[0][1] / det}, g2{-dm[1][0] / det, dm[0][0] / det};
    Vec2 g0{-g1[0] - g2[0], -g1[1] - g2[1]};
    return {v, {g0, g1, g2}, 0.5 * std::fabs(det)};
  }
  std::pair<Vec3, Vec3> columns(const std::vector<Vec3>& x) const {
    Vec3 e1 = sub(x[vertices[1]], x[vertices[0]]), e2 = sub(x[vertices[2]], x[vertices[0]]);
    Vec2 g1 = grad_n[1], g2 = grad_n[2];
    return {add(scale(e1, g1[0]), scale(e2, g2[0])), add(scale(e1, g1[1]), scale(e2, g2[1]))};
  }
  std::array<double, 3> strain(const std::vector<Vec3>& x) const {
    auto [fw, fc] = columns(x);
    return {0.5 * (dot(fw, fw) - 1.0), 0.5 * (dot(fc, fc) - 1.0), 0.5 * dot(fw, fc)};
  }
  double energy(const std::vector<Vec3>& x, const Material& m) const { return area * m.energy_density(strain(x)); }
  std::array<Vec3, 3> gradient(const std::vector<Vec3>& x, const Material& m) const {
    auto [fw, fc] = columns(x);
    auto s = m.stress(strain(x));
    Vec3 pw = add(scale(fw, s[0]), scale(fc, s[2])), pc = add(scale(fw, s[2]), scale(fc, s[1]));
    std::array<Vec3, 3> g;
    for (int k = 0; k < 3; ++k) g[k] = scale(add(scale(pw, grad_n[k][0]), scale(pc, grad_n[k][1])), area);
    return g;
  }
  ElementHessian3 hessian(const std::vector<Vec3>& x, const Material& m) const {
    return hessian_with_stress(x, m, clamp_negative_stress(m.stress(strain(x))));
  }
  ElementHessian3 tangent(const std::vector<Vec3>& x, const Material& m) const {
    return hessian_with_stress(x, m, m.stress(strain(x)));
  }
  // membrane.rs:66-78: S(E):dE + W(dE), exact for StVK and free of cancellation.
  double energy_change(const std::vector<Vec3>& x, const std::vector<Vec3>& d, double alpha, const Material& m) const {
    auto [fw, fc] = columns(x);
    auto [dw0, dc0] = columns(d);
    Vec3 dw = scale(dw0, alpha), dc = scale(dc0, alpha);
    std::array<double, 3> ch{dot(fw, dw) + 0.5 * dot(dw, dw), dot(fc, dc) + 0.5 * dot(dc, dc),
                             0.5 * (dot(fw, dc) + dot(dw, fc) + dot(dw, dc))};
    auto s = m.stress(strain(x));
    double first = s[0] * ch[0] + s[1] * ch[1] + 2.0 * s[2] * ch[2];
    return area * (first + m.energy_density(ch));
  }
  ElementHessian3 hessian_with_stress(const std::vector<Vec3>& x, const Material& m, std::array<double, 3> s) const {
    auto [fw, fc] = columns(x);
    std::array<std::array<Vec3, 3>, 3> rows;
    for (int k = 0; k < 3; ++k) {
      Vec2 g = grad_n[k];
      rows[k] = {scale(fw, g[0]), scale(fc, g[1]), scale(add(scale(fw, g[1]), scale(fc, g[0])), 0.5)};
    }
    ElementHessian3 h;
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 3; ++l) {
        Vec2 gk = grad_n[k], gl = grad_n[l];
        double geo = gk[0] * (s[0] * gl[0] + s[2] * gl[1]) + gk[1] * (s[2] * gl[0] + s[1] * gl[1]);
        Mat3 b = identity_scaled(geo);
        mat_add_scaled(b, outer(rows[k][0], rows[l][0]), m.wale);
        mat_add_scaled(b, outer(rows[k][1], rows[l][1]), m.course);
        mat_add_scaled(b, outer(rows[k][0], rows[l][1]), m.coupling);
        mat_add_scaled(b, outer(rows[k][1], rows[l][0]), m.coupling);
        mat_add_scaled(b, outer(rows[k][2], rows[l][2]), 4.0 * m.shear);
        for (auto& r : b)
          for (auto& v : r) v *= area;
        h[k][l] = b;
      }
    return h;
  }
};

// ---------------------------------------------------------------- dual numbers (dual.rs:6-90)
struct Dual {
  double v, t;
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.t + b.t}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.t - b.t}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.t * b.v + a.v * b.t}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.t * b.v - a.v * b.t) / (b.v * b.v)}; }
inline Dual operator-(Dual a) { return {-a.v, -a.t}; }
inline Dual dsqrt(Dual a) {
  double s = std::sqrt(a.v);
  return {s, a.t / (2.0 * s)};
}
inline double dsqrt(double a) { return std::sqrt(a); }
template <class T> inline T constant(double v);
template <> inline double constant<double>(double v) { return v; }
template <> inline Dual constant<Dual>(double v) { return {v, 0.0}; }

template <class T> using V3 = std::array<T, 3>;
template <class T> inline V3<T> sub3(V3<T> a, V3<T> b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
template <class T> inline V3<T> add3(V3<T> a, V3<T> b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
template <class T> inline V3<T> scale3(V3<T> a, T s) { return {a[0] * s, a[1] * s, a[2] * s}; }
template <class T> inline T dot3(V3<T> a, V3<T> b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
template <class T> inline V3<T> cross3(V3<T> a, V3<T> b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}

// hinge.rs:94-106: Bridson's dtheta/dx for any scalar type, one operation order.
template <class T> std::array<V3<T>, 4> angle_gradient_of(std::array<V3<T>, 4> p) {
  auto x1 = p[0], x2 = p[1], x3 = p[2], x4 = p[3];
  V3<T> edge = sub3(x4, x3);
  T length = dsqrt(dot3(edge, edge));
  V3<T> n1 = cross3(sub3(x1, x3), sub3(x1, x4)), n2 = cross3(sub3(x2, x4), sub3(x2, x3));
  V3<T> a1 = scale3(n1, constant<T>(1.0) / dot3(n1, n1)), a2 = scale3(n2, constant<T>(1.0) / dot3(n2, n2));
  V3<T> u1 = scale3(a1, length), u2 = scale3(a2, length);
  V3<T> u3 = add3(scale3(a1, dot3(sub3(x1, x4), edge) / length), scale3(a2, dot3(sub3(x2, x4), edge) / length));
  V3<T> u4 = add3(scale3(a1, -dot3(sub3(x1, x3), edge) / length), scale3(a2, -dot3(sub3(x2, x3), edge) / length));
  T m1 = constant<T>(-1.0);
  return {scale3(u1, m1), scale3(u2, m1), scale3(u3, m1), scale3(u4, m1)};
}

// ---------------------------------------------------------------- hinge (hinge.rs:13-120)
using ElementHessian4 = std::array<std::array<Mat3, 4>, 4>;

struct HingeElement {
  std::array<int, 4> vertices;
  double stiffness;

  std::array<Vec3, 4> points(const std::vector<Vec3>& x) const {
    return {x[vertices[0]], x[vertices[1]], x[vertices[2]], x[vertices[3]]};
  }
  double angle(const std::vector<Vec3>& x) const { return angle_of(points(x)); }
  static double angle_of(std::array<Vec3, 4> p) {
    Vec3 x1 = p[0], x2 = p[1], x3 = p[2], x4 = p[3];
    Vec3 edge = sub(x4, x3);
    Vec3 n1 = cross(sub(x1, x3), sub(x1, x4)), n2 = cross(sub(x2, x4), sub(x2, x3));
    Vec3 u1 = scale(n1, 1.0 / norm(n1)), u2 = scale(n2, 1.0 / norm(n2));
    double sine = dot(cross(u1, u2), scale(edge, 1.0 / norm(edge)));
    return std::atan2(sine, dot(u1, u2));
  }
  std::array<Vec3, 4> angle_gradient(const std::vector<Vec3>& x) const {
    return angle_gradient_of<double>(points(x));
  }
  double energy(const std::vector<Vec3>& x) const {
    double t = angle(x);
    return stiffness * t * t;
  }
  std::array<Vec3, 4> gradient(const std::vector<Vec3>& x) const {
    double f = 2.0 * stiffness * angle(x);
    auto g = angle_gradient(x);
    for (auto& v : g) v = scale(v, f);
    return g;
  }
  // Gauss–Newton 2k grad(theta) grad(theta)^T: PSD and exact at theta = 0.
  ElementHessian4 hessian(const std::vector<Vec3>& x) const {
    auto g = angle_gradient(x);
    double f = 2.0 * stiffness;
    ElementHessian4 b;
    for (int k = 0; k < 4; ++k)
      for (int l = 0; l < 4; ++l) {
        b[k][l] = outer(g[k], g[l]);
        for (auto& r : b[k][l])
          for (auto& v : r) v *= f;
      }
    return b;
  }
  // hinge.rs:66-75: exact d2theta by forward-mode duals over the analytic gradient.
  ElementHessian4 angle_hessian(const std::vector<Vec3>& x) const {
    auto p = points(x);
    ElementHessian4 b{};
    for (int l = 0; l < 4; ++l)
      for (int c = 0; c < 3; ++c) {
        std::array<V3<Dual>, 4> seeded;
        for (int k = 0; k < 4; ++k)
          for (int d = 0; d < 3; ++d) seeded[k][d] = Dual{p[k][d], (k == l && d == c) ? 1.0 : 0.0};
        auto col = angle_gradient_of<Dual>(seeded);
        for (int k = 0; k < 4; ++k)
          for (int r = 0; r < 3; ++r) b[k][l][r][c] = col[k][r].t;
      }
    return b;
  }
  ElementHessian4 tangent(const std::vector<Vec3>& x) const {
    double theta = angle(x);
    auto g = angle_gradient(x);
    auto h = angle_hessian(x);
    double f = 2.0 * stiffness;
    ElementHessian4 t;
    for (int k = 0; k < 4; ++k)
      for (int l = 0; l < 4; ++l)
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) t[k][l][r][c] = f * (g[k][r] * g[l][c] + theta * h[k][l][r][c]);
    return t;
  }
  double energy_change(const std::vector<Vec3>& x, const std::vector<Vec3>& d, double alpha) const {
    std::array<Vec3, 4> moved;
    for (int k = 0; k < 4; ++k) moved[k] = add(x[vertices[k]], scale(d[vertices[k]], alpha));
    double before = angle(x), after = angle_of(moved);
    return stiffness * (after - before) * (after + before);
  }
};

// hinge.rs:113-120: c_h = k_b(e) * 3|e|^2 / (A1 + A2).
inline double hinge_stiffness(const std::vector<Vec2>& rest, std::array<int, 4> v, double bending) {
  Vec2 p1 = rest[v[0]], p2 = rest[v[1]], p3 = rest[v[2]], p4 = rest[v[3]];
  Vec2 e{p4[0] - p3[0], p4[1] - p3[1]};
  double len2 = e[0] * e[0] + e[1] * e[1];
  auto area = [&](Vec2 p) { return 0.5 * std::fabs((p3[0] - p[0]) * (p4[1] - p[1]) - (p3[1] - p[1]) * (p4[0] - p[0])); };
  return bending * 3.0 * len2 / (area(p1) + area(p2));
}

// cases.rs:94-105
inline std::vector<HingeElement> hinge_elements(const Mesh& mesh, const Material& m) {
  std::vector<HingeElement> out;
  for (auto& v : mesh.hinges) {
    Vec2 a = mesh.rest[v[2]], b = mesh.rest[v[3]];
    double len = std::hypot(b[0] - a[0], b[1] - a[1]);
    Vec2 dir{(b[0] - a[0]) / len, (b[1] - a[1]) / len};
    out.push_back({v, hinge_stiffness(mesh.rest, v, m.hinge_bending(dir))});
  }
  return out;
}

// ---------------------------------------------------------------- contact (contact.rs:5-177)
constexpr double KEEP_FRACTION = 0.1;

struct Collider {
  int kind;  // 1 plane (normal, offset), 2 sphere (centre, radius)
  Vec3 a;    // normal or centre
  double w;  // offset or radius
  static Collider plane(Vec3 n, double offset) { return {1, n, offset}; }
  static Collider sphere(Vec3 c, double r) { return {2, c, r}; }
  double distance(Vec3 x) const { return kind == 1 ? dot(a, x) - w : norm(sub(x, a)) - w; }
  Vec3 normal(Vec3 x) const {
    if (kind == 1) return a;
    Vec3 q = sub(x, a);
    double l = norm(q);
    return {q[0] / l, q[1] / l, q[2] / l};
  }
  double curvature(Vec3 x) const { return kind == 1 ? 0.0 : 1.0 / norm(sub(x, a)); }
  double max_step(Vec3 x, Vec3 p) const {
    double d0 = distance(x);
    if (kind == 1) {
      double rate = dot(a, p);
      return std::min(rate >= 0.0 ? 1.0 : (1.0 - KEEP_FRACTION) * d0 / -rate, 1.0);
    }
    Vec3 q = sub(x, a);
    double A = dot(p, p), B = 2.0 * dot(q, p);
    double target = w + KEEP_FRACTION * d0;
    double C = (1.0 - KEEP_FRACTION) * d0 * (norm(q) + target);
    double disc = B * B - 4.0 * A * C;
    if (B >= 0.0 || disc < 0.0) return 1.0;
    return std::min(2.0 * C / (-B + std::sqrt(disc)), 1.0);
  }
  std::array<double, 8> packed() const { return {double(kind), a[0], a[1], a[2], w, 0, 0, 0}; }
};

struct Barrier {
  double dhat = 0, kappa = 0;
  double value(double d) const {
    if (d >= dhat) return 0.0;
    if (d <= 0.0) return std::numeric_limits<double>::infinity();
    return -kappa * (d - dhat) * (d - dhat) * std::log(d / dhat);
  }
  double first(double d) const {
    if (d >= dhat) return 0.0;
    double t = d - dhat;
    return -kappa * (2.0 * t * std::log(d / dhat) + t * t / d);
  }
  double second(double d) const {
    if (d >= dhat) return 0.0;
    double t = d - dhat;
    return -kappa * (2.0 * std::log(d / dhat) + 4.0 * t / d - t * t / (d * d));
  }
  static double resting_kappa(double dhat, double mass, double gravity) {
    Barrier unit{dhat, 1.0};
    return mass * gravity / std::fabs(unit.first(0.5 * dhat));
  }
};

struct Contact {
  std::vector<Collider> colliders;
  Barrier barrier;
  double energy(Vec3 x) const {
    double s = 0;
    for (auto& c : colliders) s += barrier.value(c.distance(x));
    return s;
  }
  Vec3 gradient(Vec3 x) const {
    Vec3 s{0, 0, 0};
    for (auto& c : colliders) {
      double slope = barrier.first(c.distance(x));
      Vec3 n = c.normal(x);
      for (int k = 0; k < 3; ++k) s[k] += slope * n[k];
    }
    return s;
  }
  // sum b'' n n^T + b' (I - n n^T)/|x - c|; `curvature_term` false drops the second part.
  Mat3 hessian_with(Vec3 x, bool curvature_term) const {
    Mat3 s{};
    for (auto& c : colliders) {
      double d = c.distance(x);
      double f = barrier.first(d), se = barrier.second(d), cu = curvature_term ? c.curvature(x) : 0.0;
      Vec3 n = c.normal(x);
      Mat3 nn = outer(n, n);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s[i][j] = s[i][j] + se * nn[i][j] + f * cu * ((i == j ? 1.0 : 0.0) - nn[i][j]);
    }
    return s;
  }
  Mat3 hessian(Vec3 x) const { return hessian_with(x, true); }
  double max_step(Vec3 x, Vec3 p) const {
    double a = 1.0;
    for (auto& c : colliders) a = std::min(a, c.max_step(x, p));
    return a;
  }
  double min_distance(Vec3 x) const {
    double m = std::numeric_limits<double>::infinity();
    for (auto& c : colliders) m = std::min(m, c.distance(x));
    return m;
  }
};

// ---------------------------------------------------------------- BSR (bsr.rs:4-93)
struct Bsr {
  std::vector<int> row_ptr, col_idx;
  std::vector<double> vals;

  static Bsr with_pattern(int rows, const std::vector<std::vector<int>>& groups) {
    std::vector<std::vector<int>> cols(rows);
    for (int r = 0; r < rows; ++r) cols[r].push_back(r);
    for (auto& g : groups)
      for (int r : g) cols[r].insert(cols[r].end(), g.begin(), g.end());
    Bsr m;
    m.row_ptr.push_back(0);
    for (auto& row : cols) {
      std::sort(row.begin(), row.end());
      row.erase(std::unique(row.begin(), row.end()), row.end());
      m.col_idx.insert(m.col_idx.end(), row.begin(), row.end());
      m.row_ptr.push_back(int(m.col_idx.size()));
    }
    m.vals.assign(9 * m.col_idx.size(), 0.0);
    return m;
  }
  int rows() const { return int(row_ptr.size()) - 1; }
  int blocks() const { return int(col_idx.size()); }
  int position(int row, int col) const {
    auto b = col_idx.begin() + row_ptr[row], e = col_idx.begin() + row_ptr[row + 1];
    auto it = std::lower_bound(b, e, col);
    if (it == e || *it != col) throw std::runtime_error("block outside sparsity pattern");
    return int(it - col_idx.begin());
  }
  void add(int row, int col, const Mat3& blk) {
    size_t base = 9 * size_t(position(row, col));
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) vals[base + 3 * r + c] += blk[r][c];
  }
  std::vector<double> multiply(const std::vector<double>& x) const {
    std::vector<double> y(x.size(), 0.0);
    for (int row = 0; row < rows(); ++row)
      for (int k = row_ptr[row]; k < row_ptr[row + 1]; ++k) {
        int c = col_idx[k];
        for (int r = 0; r < 3; ++r) {
          const double* v = &vals[9 * size_t(k) + 3 * r];
          y[3 * row + r] += v[0] * x[3 * c] + v[1] * x[3 * c + 1] + v[2] * x[3 * c + 2];
        }
      }
    return y;
  }
  std::vector<int> diagonal_positions() const {
    std::vector<int> d(rows());
    for (int r = 0; r < rows(); ++r) d[r] = position(r, r);
    return d;
  }
  double asymmetry() const {
    double largest = 0, worst = 0;
    for (double v : vals) largest = std::max(largest, std::fabs(v));
    for (int row = 0; row < rows(); ++row)
      for (int k = row_ptr[row]; k < row_ptr[row + 1]; ++k) {
        int mirror = position(col_idx[k], row);
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c)
            worst = std::max(worst, std::fabs(vals[9 * size_t(k) + 3 * r + c] - vals[9 * size_t(mirror) + 3 * c + r]));
      }
    return worst / largest;
  }
};

// ---------------------------------------------------------------- band Cholesky (band.rs:4-103)
struct BandCholesky {
  int size = 0, bandwidth = 0;
  std::vector<double> lower;

  size_t index(int i, int j) const { return size_t(i) * (bandwidth + 1) + (j + bandwidth - i); }
  int first(int i) const { return std::max(0, i - bandwidth); }

  // Returns false (with `error`) on a non-positive pivot.
  static bool factor(const Bsr& m, BandCholesky& out, std::string* error = nullptr) {
    BandCholesky b;
    b.size = 3 * m.rows();
    int widest = 0;
    for (int row = 0; row < m.rows(); ++row)
      for (int k = m.row_ptr[row]; k < m.row_ptr[row + 1]; ++k)
        if (m.col_idx[k] <= row) widest = std::max(widest, 3 * (row - m.col_idx[k]) + 2);
    b.bandwidth = widest;
    b.lower.assign(size_t(b.size) * (widest + 1), 0.0);
    for (int row = 0; row < m.rows(); ++row)
      for (int k = m.row_ptr[row]; k < m.row_ptr[row + 1]; ++k)
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) {
            int i = 3 * row + r, j = 3 * m.col_idx[k] + c;
            if (j <= i) b.lower[b.index(i, j)] = m.vals[9 * size_t(k) + 3 * r + c];
          }
    for (int i = 0; i < b.size; ++i)
      for (int j = b.first(i); j <= i; ++j) {
        int start = std::max(b.first(i), b.first(j));
        size_t ri = b.index(i, start), rj = b.index(j, start);
        int overlap = j - start;
        double product = 0;
        for (int k = 0; k < overlap; ++k) product += b.lower[ri + k] * b.lower[rj + k];
        double value = b.lower[b.index(i, j)] - product;
        if (i == j) {
          if (!(value > 0.0)) {
            if (error) *error = "matrix not positive definite at row " + std::to_string(i);
            return false;
          }
          b.lower[b.index(i, j)] = std::sqrt(value);
        } else {
          b.lower[b.index(i, j)] = value / b.lower[b.index(j, j)];
        }
      }
    out = std::move(b);
    return true;
  }
  std::vector<double> solve(const std::vector<double>& rhs) const {
    std::vector<double> y = rhs;
    for (int i = 0; i < size; ++i) {
      double s = 0;
      for (int k = first(i); k < i; ++k) s += lower[index(i, k)] * y[k];
      y[i] = (y[i] - s) / lower[index(i, i)];
    }
    for (int i = size - 1; i >= 0; --i) {
      int end = std::min(i + bandwidth + 1, size);
      double s = 0;
      for (int k = i + 1; k < end; ++k) s += lower[index(k, i)] * y[k];
      y[i] = (y[i] - s) / lower[index(i, i)];
    }
    return y;
  }
};

// ---------------------------------------------------------------- block-Jacobi PCG (pcg.rs:37-281)
constexpr int WORKGROUP = 256;

struct PcgSettings {
  double tolerance = 1e-7;
  int max_iterations = 20000;
  int history_stride = 16;
  int replace_every = 0;
  double replace_above = 0.0;
  // Stop with `breakdown` when p^T q <= 0 or non-finite (the GPU's reduce.wgsl status); the E1 oracle runs without it.
  bool detect_breakdown = false;
};

struct PcgReport {
  int iterations = 0;
  bool converged = false;
  bool breakdown = false;
  double recursive_relative_residual = 1.0;
  std::vector<double> solution;
  std::vector<std::pair<int, double>> history;
};

// pcg.rs:447-476: 256-wide workgroup trees, then one strided 256-lane pass and a final tree.
template <class T, class F> T reduce_rows(int rows, F value) {
  int groups = (rows + WORKGROUP - 1) / WORKGROUP;
  std::vector<T> partials(groups);
  T lane[WORKGROUP];
  auto tree = [&](T* l) {
    for (int stride = WORKGROUP / 2; stride > 0; stride /= 2)
      for (int t = 0; t < stride; ++t) l[t] = l[t] + l[t + stride];
    return l[0];
  };
  for (int g = 0; g < groups; ++g) {
    for (int t = 0; t < WORKGROUP; ++t) {
      int row = g * WORKGROUP + t;
      lane[t] = row < rows ? value(row) : T(0);
    }
    partials[g] = tree(lane);
  }
  for (int t = 0; t < WORKGROUP; ++t) {
    T s = T(0);
    for (int k = t; k < groups; k += WORKGROUP) s = s + partials[k];
    lane[t] = s;
  }
  return tree(lane);
}

// pcg.rs:479-492: adjugate inverse in the WGSL operation order.
template <class T> std::array<T, 9> invert3(const T* m) {
  T a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
  T c00 = e * i - f * h, c01 = c * h - b * i, c02 = b * f - c * e;
  T c10 = f * g - d * i, c11 = a * i - c * g, c12 = c * d - a * f;
  T c20 = d * h - e * g, c21 = b * g - a * h, c22 = a * e - b * d;
  T det = a * c00 + b * c10 + c * c20;
  return {c00 / det, c01 / det, c02 / det, c10 / det, c11 / det, c12 / det, c20 / det, c21 / det, c22 / det};
}

// Block-Jacobi PCG from x = 0 reproducing the WGSL arithmetic order (T = float emulates the GPU).
template <class T> PcgReport pcg_solve(const Bsr& A, const std::vector<double>& rhs, const PcgSettings& s) {
  int R = A.rows();
  size_t n = rhs.size();
  std::vector<T> vals(A.vals.size()), dinv(9 * size_t(R)), b(n);
  for (size_t k = 0; k < vals.size(); ++k) vals[k] = T(A.vals[k]);
  auto diag = A.diagonal_positions();
  for (int r = 0; r < R; ++r) {
    auto inv = invert3<T>(&vals[9 * size_t(diag[r])]);
    for (int k = 0; k < 9; ++k) dinv[9 * size_t(r) + k] = inv[k];
  }
  for (size_t i = 0; i < n; ++i) b[i] = T(rhs[i]);
  auto multiply_row = [&](int row, const std::vector<T>& p) {
    std::array<T, 3> acc{T(0), T(0), T(0)};
    for (int k = A.row_ptr[row]; k < A.row_ptr[row + 1]; ++k) {
      size_t c = 3 * size_t(A.col_idx[k]);
      const T* v = &vals[9 * size_t(k)];
      for (int r = 0; r < 3; ++r) acc[r] = acc[r] + (v[3 * r] * p[c] + v[3 * r + 1] * p[c + 1] + v[3 * r + 2] * p[c + 2]);
    }
    return acc;
  };
  auto precondition = [&](const std::vector<T>& r, std::vector<T>& z) {
    for (int row = 0; row < R; ++row) {
      const T* d = &dinv[9 * size_t(row)];
      T a = r[3 * row], bb = r[3 * row + 1], c = r[3 * row + 2];
      z[3 * row] = d[0] * a + d[1] * bb + d[2] * c;
      z[3 * row + 1] = d[3] * a + d[4] * bb + d[5] * c;
      z[3 * row + 2] = d[6] * a + d[7] * bb + d[8] * c;
    }
  };
  auto row_dot = [](const std::vector<T>& a, const std::vector<T>& bb, int row) {
    size_t i = 3 * size_t(row);
    return a[i] * bb[i] + a[i + 1] * bb[i + 1] + a[i + 2] * bb[i + 2];
  };
  std::vector<T> x(n, T(0)), r = b, z(n), p, q(n);
  precondition(r, z);
  T rz = reduce_rows<T>(R, [&](int row) { return row_dot(r, z, row); });
  T rr = reduce_rows<T>(R, [&](int row) { return row_dot(r, r, row); });
  T rr0 = rr;
  p = z;
  PcgReport rep;
  T tol2 = T(s.tolerance * s.tolerance);
  bool converged = rr <= T(0);
  auto relative = [&]() { return std::sqrt(double(rr) / double(rr0)); };
  while (!converged && rep.iterations < s.max_iterations) {
    for (int row = 0; row < R; ++row) {
      auto a = multiply_row(row, p);
      q[3 * row] = a[0];
      q[3 * row + 1] = a[1];
      q[3 * row + 2] = a[2];
    }
    T pq = reduce_rows<T>(R, [&](int row) { return row_dot(p, q, row); });
    if (s.detect_breakdown && (!(pq > T(0)) || !std::isfinite(double(pq)))) {
      rep.breakdown = true;
      break;
    }
    T alpha = rz / pq;
    for (size_t i = 0; i < n; ++i) {
      x[i] = x[i] + alpha * p[i];
      r[i] = r[i] - alpha * q[i];
    }
    precondition(r, z);
    T rz_new = reduce_rows<T>(R, [&](int row) { return row_dot(r, z, row); });
    rr = reduce_rows<T>(R, [&](int row) { return row_dot(r, r, row); });
    T beta = rz_new / rz;
    rz = rz_new;
    rep.iterations++;
    if (s.history_stride > 0 && rep.iterations % s.history_stride == 0) rep.history.push_back({rep.iterations, relative()});
    converged = rr <= tol2 * rr0;
    if (!converged)
      for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    bool due = s.replace_every > 0 && rep.iterations % s.replace_every == 0;
    if (!converged && due && rr > T(s.replace_above * s.replace_above) * rr0) {
      for (int row = 0; row < R; ++row) {
        auto ax = multiply_row(row, x);
        for (int d = 0; d < 3; ++d) r[3 * row + d] = b[3 * row + d] - ax[d];
      }
      precondition(r, z);
      rz = reduce_rows<T>(R, [&](int row) { return row_dot(r, z, row); });
      rr = reduce_rows<T>(R, [&](int row) { return row_dot(r, r, row); });
    }
  }
  rep.converged = converged;
  rep.recursive_relative_residual = relative();
  rep.history.push_back({rep.iterations, rep.recursive_relative_residual});
  rep.solution.resize(n);
  for (size_t i = 0; i < n; ++i) rep.solution[i] = double(x[i]);
  return rep;
}

}  // namespace oracle
