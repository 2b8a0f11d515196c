// Test infrastructure only (see core.h). The E1 linear cases of the reference (cases.rs:64-161): the
// quasi-static or dynamic Newton matrix of a clamped 0.5 m knit sheet and its load vector. They pin the PCG
// restatement against the iteration counts the reference stored for them (experiments/cases/*/reference.json).
#pragma once
#include "core.h"

namespace oracle {

enum class CaseKind { Tension, Slack, Dynamic };

struct LinearCase {
  Mesh mesh;
  Bsr matrix;
  std::vector<double> rhs;
};

inline LinearCase build_case(CaseKind kind, int columns) {
  const double sheet = 0.5, time_step = 1.0 / 240.0, gravity = 9.81, in_plane = 2.0;
  LinearCase c;
  c.mesh = Mesh::grid(columns, columns, sheet, sheet);
  Material m = Material::knit_baseline();
  std::vector<int> row_of(c.mesh.rest.size(), -1), free_;
  for (int v = 0; v < int(c.mesh.rest.size()); ++v)
    if (!c.mesh.is_boundary(v)) {
      row_of[v] = int(free_.size());
      free_.push_back(v);
    }
  double sw = kind == CaseKind::Tension ? 1.03 : 1.0, sc = kind == CaseKind::Tension ? 1.08 : 1.0;
  std::vector<Vec3> x;
  for (auto& p : c.mesh.rest) x.push_back({sw * p[0], sc * p[1], 0.0});
  std::vector<MembraneElement> membranes;
  for (auto& t : c.mesh.triangles) membranes.push_back(MembraneElement::make(t, c.mesh.rest));
  auto hinges = hinge_elements(c.mesh, m);
  std::vector<std::vector<int>> groups;
  auto to_rows = [&](const int* vs, int n) {
    std::vector<int> g;
    for (int k = 0; k < n; ++k)
      if (row_of[vs[k]] >= 0) g.push_back(row_of[vs[k]]);
    return g;
  };
  for (auto& t : c.mesh.triangles) groups.push_back(to_rows(t.data(), 3));
  for (auto& h : c.mesh.hinges) groups.push_back(to_rows(h.data(), 4));
  c.matrix = Bsr::with_pattern(int(free_.size()), groups);
  for (auto& e : membranes) {
    auto h = e.hessian(x, m);
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 3; ++l) {
        int r = row_of[e.vertices[k]], cc = row_of[e.vertices[l]];
        if (r >= 0 && cc >= 0) c.matrix.add(r, cc, h[k][l]);
      }
  }
  for (auto& e : hinges) {
    auto h = e.hessian(x);
    for (int k = 0; k < 4; ++k)
      for (int l = 0; l < 4; ++l) {
        int r = row_of[e.vertices[k]], cc = row_of[e.vertices[l]];
        if (r >= 0 && cc >= 0) c.matrix.add(r, cc, h[k][l]);
      }
  }
  auto areas = c.mesh.vertex_areas();
  if (kind == CaseKind::Dynamic)
    for (size_t row = 0; row < free_.size(); ++row)
      c.matrix.add(int(row), int(row), identity_scaled(m.density * areas[free_[row]] / (time_step * time_step)));
  for (int v : free_) {
    double px = c.mesh.rest[v][0], py = c.mesh.rest[v][1], w = c.mesh.width, h = c.mesh.height;
    double shape = std::sin(M_PI * px / w) * std::sin(M_PI * py / h);
    double skew = std::sin(2.0 * M_PI * px / w) * std::sin(M_PI * py / h);
    double a = areas[v];
    c.rhs.push_back(a * in_plane * shape);
    c.rhs.push_back(0.5 * a * in_plane * skew);
    c.rhs.push_back(-m.density * a * gravity);
  }
  return c;
}

}  // namespace oracle
