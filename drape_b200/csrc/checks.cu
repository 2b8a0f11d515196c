// Kernel checks of the drape GPU stage: the element and row terms in the reference's per-element layout, the
// arrays run-e7.ts --checks writes (run-e7.ts:140-145) and e4_compare.rs / e7_compare.rs score against the f64
// oracle. The solve never needs them: its assembly gathers element rows straight into BSR rows (elem.cu).
//   element_terms  one thread per membrane or hinge at positions x:
//                    gradient  [9T + 12H]: triangle e at 9e + 3k + i, hinge h at 9T + 12h + 3k + i
//                    Hessian   [81T + 144H]: triangle block (k, l) at 81e + 9(3k + l), hinge block (k, l) at
//                              81T + 144h + 9(4k + l), each 3x3 row-major
//                  (membrane_element.wgsl:38-76, hinge_element.wgsl:20-53); `exact` selects the exact tangent
//                  (StVK stress, hinge 2c(grad grad^T + theta d2 theta)) or the projected one (positive-part
//                  stress in the geometric term, Gauss-Newton hinge); the gradients are the same in both.
//   row_terms      one thread per unknown row: gradient [3R] = m_r (x - x_hat) + sum b'(d) n and block [9R] =
//                  m_r (1 + mu) I + sum b''(d) n n^T + b'(d) kappa (I - n n^T) over active colliders
//                  (inertia.wgsl:14-52), m_r the caller's per-row mass over h^2.
// Both evaluate in f64 and round each entry to f32 once.
#include <cuda_runtime.h>

#include "device_math.cuh"
#include "device_problem.h"
#include "kernels.h"

namespace drape {
using namespace dev;

namespace {

__global__ void element_terms_kernel(DevProblem p, const double* x, int exact, float* grad, float* hess) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < p.T) {
    const int* v = p.tri + 3 * e;
    const V3 x0 = load3(x, v[0]), x1 = load3(x, v[1]), x2 = load3(x, v[2]);
    const TriGeom G = load_geom(p.geom, e);
    V3 fw, fc;
    columns(G, x0, x1, x2, fw, fc);
    const Membrane m{p.wale, p.course, p.coupling, p.shear};
    for (int k = 0; k < 3; ++k) {
      const V3 g = membrane_gradient_row(m, G, fw, fc, k);
      float* o = grad + 9 * (size_t)e + 3 * k;
      o[0] = float(g.x);
      o[1] = float(g.y);
      o[2] = float(g.z);
      double blk[3][9];
      membrane_hessian_row(m, G, fw, fc, k, blk, !exact);
      for (int l = 0; l < 3; ++l)
        for (int i = 0; i < 9; ++i) hess[81 * (size_t)e + 9 * (3 * k + l) + i] = float(blk[l][i]);
    }
    return;
  }
  const int h = e - p.T;
  if (h >= p.H) return;
  const int* v = p.hinge + 4 * h;
  const V3 xs[4] = {load3(x, v[0]), load3(x, v[1]), load3(x, v[2]), load3(x, v[3])};
  V3 dg[4];
  hinge_angle_gradient(xs[0], xs[1], xs[2], xs[3], dg);
  const double theta = hinge_angle(xs[0], xs[1], xs[2], xs[3]);
  const double c2 = 2.0 * p.hinge_k[h];
  const size_t go = 9 * (size_t)p.T + 12 * (size_t)h, ho = 81 * (size_t)p.T + 144 * (size_t)h;
  for (int k = 0; k < 4; ++k) {
    const V3 g = dg[k] * (c2 * theta);
    grad[go + 3 * k] = float(g.x);
    grad[go + 3 * k + 1] = float(g.y);
    grad[go + 3 * k + 2] = float(g.z);
    double blk[4][9];
    if (exact) {
      hinge_exact_hessian_row(xs, dg, theta, c2, k, blk);
    } else {
      for (int l = 0; l < 4; ++l)
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) blk[l][3 * r + c] = c2 * comp(dg[k], r) * comp(dg[l], c);
    }
    for (int l = 0; l < 4; ++l)
      for (int i = 0; i < 9; ++i) hess[ho + 9 * (4 * k + l) + i] = float(blk[l][i]);
  }
}

__global__ void row_terms_kernel(DevProblem p, const double* x, const double* x_hat, const double* row_mass,
                                 double mu, int contact, int curvature, float* grad, float* hess) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= p.R) return;
  const int v = p.row_vertex[row];
  const V3 xv = load3(x, v);
  const double m = row_mass ? row_mass[row] : 0.0;
  V3 g = (xv - load3(x_hat, v)) * m;
  double blk[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  blk[0] = blk[4] = blk[8] = m * (1.0 + mu);
  if (contact) {
    const Barrier bar{p.dhat, p.kappa};
    for (int c = 0; c < p.ncol; ++c) {
      const Proximity q = proximity(p.colliders + 8 * c, xv);
      if (q.distance >= p.dhat) continue;
      const double b1 = bar.first(q.distance), b2 = bar.second(q.distance);
      g = g + q.normal * b1;
      const double curv = curvature ? b1 * q.curvature : 0.0;
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) {
          const double nn = comp(q.normal, r) * comp(q.normal, cc);
          blk[3 * r + cc] += b2 * nn + curv * ((r == cc ? 1.0 : 0.0) - nn);
        }
    }
  }
  grad[3 * (size_t)row] = float(g.x);
  grad[3 * (size_t)row + 1] = float(g.y);
  grad[3 * (size_t)row + 2] = float(g.z);
  for (int i = 0; i < 9; ++i) hess[9 * (size_t)row + i] = float(blk[i]);
}

}  // namespace

cudaError_t launch_element_terms(const DevProblem& p, const double* x, int exact, float* grad, float* hess,
                                 cudaStream_t s) {
  const int n = p.T + p.H;
  if (n > 0) element_terms_kernel<<<(n + 127) / 128, 128, 0, s>>>(p, x, exact, grad, hess);
  return cudaGetLastError();
}

cudaError_t launch_row_terms(const DevProblem& p, const double* x, const double* x_hat, const double* row_mass,
                             double mu, int contact, int curvature, float* grad, float* hess, cudaStream_t s) {
  if (p.R > 0)
    row_terms_kernel<<<(p.R + 255) / 256, 256, 0, s>>>(p, x, x_hat, row_mass, mu, contact, curvature, grad, hess);
  return cudaGetLastError();
}

}  // namespace drape
