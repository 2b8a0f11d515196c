// The device view of one drape problem, passed by value to every kernel. All arrays live in HBM; the context
// (context.cpp) owns them. Layouts:
//   x, x_hat, d           f64 [3V]  vertex positions / prediction / direction (fixed vertices carry d = 0)
//   geom                  f64 [7T]  dN_k/dX per triangle vertex and the rest area
//   tri, hinge            i32 [3T], [4H]
//   row_vertex, unit_mass i32/f64 [R]
//   rt_ptr/rt_ent/rt_pos  row -> incident triangles: entry = (t << 2) | k (k the row's local index in t);
//                         rt_pos[3e + l] = block slot of vertex l within the row (-1: vertex l is fixed)
//   rh_ptr/rh_ent/rh_pos  the same for hinges with 4 slots per entry
//   BSR(3x3) f32 values   three planes, one 16-byte and one 4-byte element per block:
//                         a0[k] = (m00, m01, m02, m10), a1[k] = (m11, m12, m20, m21), a2[k] = m22
#pragma once
#include <cuda_runtime.h>

namespace drape {

struct DevProblem {
  int V, T, H, R, B, ncol, max_row_blocks, max_row_entries;
  const double* geom;
  const int* tri;
  const int* hinge;
  const double* hinge_k;
  const int* row_vertex;
  const double* unit_mass;
  const int* row_ptr;
  const int* col_idx;
  const int* diag_slot;  // slot of the diagonal block within its row
  const int* rt_ptr;
  const int* rt_ent;
  const int* rt_pos;
  const int* rh_ptr;
  const int* rh_ent;
  const int* rh_pos;
  const double* colliders;  // 8 per collider
  double wale, course, coupling, shear;
  double gravity[3];
  double dhat, kappa;
};

struct DevBsr {
  float4* a0;
  float4* a1;
  float* a2;
};

}  // namespace drape
