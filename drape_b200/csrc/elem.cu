// Element kernels of the drape Newton step (sm_100a):
//   assemble_rows   one warp per BSR row: the row's incident triangles and hinges are evaluated by the warp's
//                   lanes (f64), their gradient rows are tree-reduced into the row's f64 residual, and their
//                   Hessian rows (stress-clamped membrane, Gauss-Newton hinge) are summed per block slot in a
//                   fixed order and rounded to f32 once, together with the row's inertia and barrier terms.
//                   No element Hessian is written to HBM and no atomics are used: every block is written by
//                   exactly one lane, so the assembly is deterministic.
//   energy_change   the cancellation-free per-element / per-row change of Phi along x + alpha d, summed in f64
//   max_step        the CCD bound: largest alpha <= 1 keeping every vertex at >= 0.1 of its collider distance
// Reference semantics: drape.rs:199-335 (gradient, tangent, energy change), membrane.rs:46-101, hinge.rs:45-90,
// contact.rs:126-162, inertia.wgsl:34-52, assemble_matrix.wgsl:15-34, ccd.wgsl:39-56.
#include <cuda_runtime.h>

#include "device_math.cuh"
#include "device_problem.h"
#include "kernels.h"

namespace drape {
using namespace dev;

namespace {

constexpr int WARPS_PER_CTA = 4;
// Four resident CTAs per SM for assemble_rows (16 warps; 156 KB of its shared staging): the register cap this
// sets (128 per thread, a few spilled) hides more of the f64 latency than 192 registers at 8 warps. Measured at
// n129: 0.293 ms per assembly against 0.372 ms (two CTAs, no cap), 0.311 ms (three) and 0.343 ms (five, heavier
// spills); register allocation does not change the arithmetic, so the blocks are bitwise the same.
constexpr int kAssembleMinCtas = 4;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void cta_partial(double s, double* partial, bool minimum) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double t = __shfl_xor_sync(0xffffffffu, s, o);
    s = minimum ? fmin(s, t) : s + t;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = minimum ? INFINITY : 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = minimum ? fmin(t, red[w]) : t + red[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(32 * WARPS_PER_CTA, kAssembleMinCtas) assemble_rows(AssembleArgs a) {
  __shared__ double contrib[WARPS_PER_CTA][kMaxRowEntries][4][9];
  __shared__ int slots[WARPS_PER_CTA][kMaxRowEntries][4];
  __shared__ double norms[WARPS_PER_CTA];
  const DevProblem& p = a.p;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * WARPS_PER_CTA + warp;
  const bool hess = a.bsr.a0 != nullptr;
  double row_norm = 0.0;
  if (row < p.R) {
    const Membrane mat{p.wale, p.course, p.coupling, p.shear};
    const int t0 = p.rt_ptr[row], nt = p.rt_ptr[row + 1] - t0;
    const int h0 = p.rh_ptr[row], nh = p.rh_ptr[row + 1] - h0;
    const int ne = nt + nh;  // <= kMaxRowEntries (checked when the context is created)
    const int b0 = p.row_ptr[row], nb = p.row_ptr[row + 1] - b0;
    V3 g = v3(0, 0, 0);
    if (lane < ne) {
      double blk[4][9];
      int nslot;
      if (lane < nt) {
        const int ent = p.rt_ent[t0 + lane], t = ent >> 2, k = ent & 3;
        const TriGeom G = load_geom(p.geom, t);
        const int* tv = p.tri + 3 * (size_t)t;
        V3 fw, fc;
        columns(G, load3(a.x, tv[0]), load3(a.x, tv[1]), load3(a.x, tv[2]), fw, fc);
        g = membrane_gradient_row(mat, G, fw, fc, k);
        if (hess) membrane_hessian_row(mat, G, fw, fc, k, blk, !a.exact);
        nslot = 3;
        if (hess)
          for (int l = 0; l < 3; ++l) slots[warp][lane][l] = p.rt_pos[3 * (size_t)(t0 + lane) + l];
      } else {
        const int eh = lane - nt;
        const int ent = p.rh_ent[h0 + eh], h = ent >> 2, k = ent & 3;
        const int* hv = p.hinge + 4 * (size_t)h;
        const V3 x1 = load3(a.x, hv[0]), x2 = load3(a.x, hv[1]), x3 = load3(a.x, hv[2]), x4 = load3(a.x, hv[3]);
        V3 dg[4];
        hinge_angle_gradient(x1, x2, x3, x4, dg);
        const double c2 = 2.0 * p.hinge_k[h];
        const double theta = hinge_angle(x1, x2, x3, x4);
        g = dg[k] * (c2 * theta);
        if (hess && a.exact) {
          const V3 xs[4] = {x1, x2, x3, x4};
          hinge_exact_hessian_row(xs, dg, theta, c2, k, blk);
        } else if (hess) {
          for (int l = 0; l < 4; ++l)
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) blk[l][3 * r + c] = c2 * comp(dg[k], r) * comp(dg[l], c);
        }
        nslot = 4;
        if (hess)
          for (int l = 0; l < 4; ++l) slots[warp][lane][l] = p.rh_pos[4 * (size_t)(h0 + eh) + l];
      }
      if (hess) {
        for (int l = 0; l < nslot; ++l)
          for (int i = 0; i < 9; ++i) contrib[warp][lane][l][i] = blk[l][i];
        if (nslot == 3) slots[warp][lane][3] = -1;
      }
    }
    // Gradient rows: fixed xor tree over the lanes.
    g = v3(warp_sum(g.x), warp_sum(g.y), warp_sum(g.z));
    // The row's own vertex: inertia (or gravity) and barrier terms, and its diagonal block.
    const int v = p.row_vertex[row];
    const V3 xv = load3(a.x, v);
    const double m = p.unit_mass[row];
    double diag[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) diag[i] = 0.0;
    if (a.mode == 0) {
      const double mh = m * a.inv_h2;
      g = g + (xv - load3(a.x_hat, v)) * mh;
      diag[0] = diag[4] = diag[8] = mh * (1.0 + a.mu);
    } else {
      g = g - v3(p.gravity[0], p.gravity[1], p.gravity[2]) * m;
    }
    const Barrier bar{p.dhat, p.kappa};
    for (int c = 0; c < p.ncol; ++c) {
      const Proximity q = proximity(p.colliders + 8 * c, xv);
      if (q.distance >= p.dhat) continue;
      const double b1 = bar.first(q.distance), b2 = bar.second(q.distance);
      g = g + q.normal * b1;
      const double curv = a.curvature ? b1 * q.curvature : 0.0;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const double nn = comp(q.normal, r) * comp(q.normal, cc);
          diag[3 * r + cc] += b2 * nn + curv * ((r == cc ? 1.0 : 0.0) - nn);
        }
    }
    if (lane == 0) {
      a.grad[3 * (size_t)row] = g.x;
      a.grad[3 * (size_t)row + 1] = g.y;
      a.grad[3 * (size_t)row + 2] = g.z;
    }
    row_norm = dot(g, g);
    if (hess) {
      __syncwarp();
      // Lane j owns block slot j of the row and sums its contributions in entry order.
      if (lane < nb) {
        double acc[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) acc[i] = 0.0;
        for (int q = 0; q < ne; ++q)
#pragma unroll
          for (int l = 0; l < 4; ++l)
            if (slots[warp][q][l] == lane)
#pragma unroll
              for (int i = 0; i < 9; ++i) acc[i] += contrib[warp][q][l][i];
        if (lane == p.diag_slot[row])
#pragma unroll
          for (int i = 0; i < 9; ++i) acc[i] += diag[i];
        const size_t k = (size_t)(b0 + lane);
        a.bsr.a0[k] = make_float4(float(acc[0]), float(acc[1]), float(acc[2]), float(acc[3]));
        a.bsr.a1[k] = make_float4(float(acc[4]), float(acc[5]), float(acc[6]), float(acc[7]));
        a.bsr.a2[k] = float(acc[8]);
      }
    }
  }
  if (lane == 0) norms[warp] = row_norm;
  __syncthreads();
  if (threadIdx.x == 0 && a.partial) {
    double s = 0.0;
    for (int w = 0; w < WARPS_PER_CTA; ++w) s += norms[w];
    a.partial[blockIdx.x] = s;
  }
}

// Per-CTA partial sums of the change of Phi (mode 0) or E_s (mode 1) along x + alpha d:
//   triangles S(E):dE + W(dE); hinges k (theta' - theta)(theta' + theta);
//   rows m/h^2 ((x - x_hat).(alpha d) + |alpha d|^2 / 2) or -m g.(alpha d), plus barrier changes.
__global__ void __launch_bounds__(256) energy_change_kernel(EnergyArgs a) {
  const DevProblem& p = a.p;
  const Membrane mat{p.wale, p.course, p.coupling, p.shear};
  const Barrier bar{p.dhat, p.kappa};
  const int total = p.T + p.H + p.R;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if (i < p.T) {
      const int* tv = p.tri + 3 * (size_t)i;
      const TriGeom G = load_geom(p.geom, i);
      V3 fw, fc, dw, dc;
      columns(G, load3(a.x, tv[0]), load3(a.x, tv[1]), load3(a.x, tv[2]), fw, fc);
      columns(G, load3(a.d, tv[0]), load3(a.d, tv[1]), load3(a.d, tv[2]), dw, dc);
      s += membrane_energy_change(mat, G, fw, fc, dw * a.alpha, dc * a.alpha);
    } else if (i < p.T + p.H) {
      const int h = i - p.T;
      const int* hv = p.hinge + 4 * (size_t)h;
      const V3 x1 = load3(a.x, hv[0]), x2 = load3(a.x, hv[1]), x3 = load3(a.x, hv[2]), x4 = load3(a.x, hv[3]);
      const double before = hinge_angle(x1, x2, x3, x4);
      const double after = hinge_angle(x1 + load3(a.d, hv[0]) * a.alpha, x2 + load3(a.d, hv[1]) * a.alpha,
                                       x3 + load3(a.d, hv[2]) * a.alpha, x4 + load3(a.d, hv[3]) * a.alpha);
      s += p.hinge_k[h] * (after - before) * (after + before);
    } else {
      const int row = i - p.T - p.H, v = p.row_vertex[row];
      const V3 xv = load3(a.x, v), st = load3(a.d, v) * a.alpha;
      const double m = p.unit_mass[row];
      if (a.mode == 0)
        s += m * a.inv_h2 * (dot(xv - load3(a.x_hat, v), st) + 0.5 * dot(st, st));
      else
        s -= m * dot(v3(p.gravity[0], p.gravity[1], p.gravity[2]), st);
      const V3 moved = xv + st;
      for (int c = 0; c < p.ncol; ++c) {
        const double* col = p.colliders + 8 * c;
        s += bar.value(proximity(col, moved).distance) - bar.value(proximity(col, xv).distance);
      }
    }
  }
  cta_partial(s, a.partial, false);
}

// Per-CTA minima of the CCD bound over the rows' vertices (1 when no collider limits the step).
__global__ void __launch_bounds__(256) max_step_kernel(DevProblem p, const double* x, const double* d, double* partial) {
  double m = 1.0;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < p.R; row += gridDim.x * blockDim.x) {
    const int v = p.row_vertex[row];
    const V3 xv = load3(x, v), dv = load3(d, v);
    for (int c = 0; c < p.ncol; ++c) m = fmin(m, collider_max_step(p.colliders + 8 * c, xv, dv));
  }
  cta_partial(m, partial, true);
}

// Per-CTA partial of sum_rows g_row . d_vertex (the Newton slope).
__global__ void __launch_bounds__(256) slope_kernel(DevProblem p, const double* g, const double* d, double* partial) {
  double s = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < p.R; r += gridDim.x * blockDim.x) {
    const int v = p.row_vertex[r];
    s += g[3 * r] * d[3 * v] + g[3 * r + 1] * d[3 * v + 1] + g[3 * r + 2] * d[3 * v + 2];
  }
  cta_partial(s, partial, false);
}

// Per-CTA partial of max over rows of |d| (the update's infinity norm).
__global__ void __launch_bounds__(256) inf_norm_kernel(DevProblem p, const double* d, double* partial) {
  double m = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < p.R; r += gridDim.x * blockDim.x) {
    const int v = p.row_vertex[r];
    m = fmax(m, fmax(fabs(d[3 * v]), fmax(fabs(d[3 * v + 1]), fabs(d[3 * v + 2]))));
  }
  // max via -min(-x)
  cta_partial(-m, partial, true);
}

// out[slot] = sum (op 0) or min (op 1) of n partials, in a fixed order (one CTA of 256 threads).
__global__ void __launch_bounds__(256) reduce_partials(const double* partial, int n, int op, double* out, int slot) {
  __shared__ double red[256];
  double s = op == 0 ? 0.0 : INFINITY;
  for (int i = threadIdx.x; i < n; i += 256) s = op == 0 ? s + partial[i] : fmin(s, partial[i]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      red[threadIdx.x] = op == 0 ? red[threadIdx.x] + red[threadIdx.x + w] : fmin(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[slot] = red[0];
}

// x_hat = x + h^2 g on the rows' vertices (x_hat starts as a copy of x).
// x_hat = x + h v + h^2 g on the free vertices (rows); v null: x + h^2 g (the PTC prediction, e7_ptc.rs:54-58);
// with v: the backward-Euler prediction (drape.rs:177-185, drape-step.ts:26-38).
__global__ void predict_rows_kernel(DevProblem p, const double* x, const double* vel, double h, double* x_hat) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.R) return;
  const int v = p.row_vertex[r];
  for (int k = 0; k < 3; ++k)
    x_hat[3 * v + k] = x[3 * v + k] + (vel ? h * vel[3 * v + k] : 0.0) + h * h * p.gravity[k];
}

__global__ void axpy_kernel(int n, const double* x, double alpha, const double* d, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = x[i] + alpha * d[i];
}

__global__ void sub_kernel(int n, const double* a, const double* b, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] - b[i];
}

// Vertex-layout f64 direction from the row-layout f32 PCG solution (float4 per row).
__global__ void scatter_direction_kernel(DevProblem p, const float4* sol, double* d) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.R) return;
  const int v = p.row_vertex[r];
  const float4 s = sol[r];
  d[3 * v] = double(s.x);
  d[3 * v + 1] = double(s.y);
  d[3 * v + 2] = double(s.z);
}

// b = -g as the f32 PCG right-hand side (float4 per row, w = 0).
__global__ void rhs_kernel(int R, const double* g, float4* b) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) b[r] = make_float4(float(-g[3 * r]), float(-g[3 * r + 1]), float(-g[3 * r + 2]), 0.0f);
}

// Per-CTA partial sums of E_s = membrane + hinge energy + barrier - m g.x (f64; e7_ptc.rs:48-51).
__global__ void __launch_bounds__(256) static_energy_kernel(DevProblem p, const double* x, double* partial) {
  const Membrane mat{p.wale, p.course, p.coupling, p.shear};
  const Barrier bar{p.dhat, p.kappa};
  const int total = p.T + p.H + p.R;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if (i < p.T) {
      const int* tv = p.tri + 3 * (size_t)i;
      const TriGeom G = load_geom(p.geom, i);
      V3 fw, fc;
      columns(G, load3(x, tv[0]), load3(x, tv[1]), load3(x, tv[2]), fw, fc);
      s += membrane_energy(mat, G, fw, fc);
    } else if (i < p.T + p.H) {
      const int h = i - p.T;
      const int* hv = p.hinge + 4 * (size_t)h;
      const double th = hinge_angle(load3(x, hv[0]), load3(x, hv[1]), load3(x, hv[2]), load3(x, hv[3]));
      s += p.hinge_k[h] * th * th;
    } else {
      const int row = i - p.T - p.H, v = p.row_vertex[row];
      const V3 xv = load3(x, v);
      s -= p.unit_mass[row] * dot(v3(p.gravity[0], p.gravity[1], p.gravity[2]), xv);
      for (int c = 0; c < p.ncol; ++c) s += bar.value(proximity(p.colliders + 8 * c, xv).distance);
    }
  }
  cta_partial(s, partial, false);
}

// Per-CTA minima of the smallest collider distance over the rows' vertices.
__global__ void __launch_bounds__(256) min_distance_kernel(DevProblem p, const double* x, double* partial) {
  double m = INFINITY;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < p.R; row += gridDim.x * blockDim.x) {
    const V3 xv = load3(x, p.row_vertex[row]);
    for (int c = 0; c < p.ncol; ++c) m = fmin(m, proximity(p.colliders + 8 * c, xv).distance);
  }
  cta_partial(m, partial, true);
}

int blocks_for(int n, int t) { return (n + t - 1) / t; }

}  // namespace

cudaError_t launch_static_energy(const DevProblem& p, const double* x, double* partial, int grid, cudaStream_t s) {
  static_energy_kernel<<<grid, 256, 0, s>>>(p, x, partial);
  return cudaGetLastError();
}

cudaError_t launch_min_distance(const DevProblem& p, const double* x, double* partial, int grid, cudaStream_t s) {
  min_distance_kernel<<<grid, 256, 0, s>>>(p, x, partial);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- launchers
int assemble_grid(int R) { return blocks_for(R, WARPS_PER_CTA); }

cudaError_t launch_assemble(const AssembleArgs& a, cudaStream_t s) {
  assemble_rows<<<assemble_grid(a.p.R), 32 * WARPS_PER_CTA, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_energy_change(const EnergyArgs& a, int grid, cudaStream_t s) {
  energy_change_kernel<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_max_step(const DevProblem& p, const double* x, const double* d, double* partial, int grid,
                            cudaStream_t s) {
  max_step_kernel<<<grid, 256, 0, s>>>(p, x, d, partial);
  return cudaGetLastError();
}

cudaError_t launch_slope(const DevProblem& p, const double* g, const double* d, double* partial, int grid,
                         cudaStream_t s) {
  slope_kernel<<<grid, 256, 0, s>>>(p, g, d, partial);
  return cudaGetLastError();
}

cudaError_t launch_inf_norm(const DevProblem& p, const double* d, double* partial, int grid, cudaStream_t s) {
  inf_norm_kernel<<<grid, 256, 0, s>>>(p, d, partial);
  return cudaGetLastError();
}

cudaError_t launch_reduce(const double* partial, int n, int op, double* out, int slot, cudaStream_t s) {
  reduce_partials<<<1, 256, 0, s>>>(partial, n, op, out, slot);
  return cudaGetLastError();
}

cudaError_t launch_predict(const DevProblem& p, const double* x, const double* vel, double h, double* x_hat,
                           cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(x_hat, x, 3 * sizeof(double) * (size_t)p.V, cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return e;
  predict_rows_kernel<<<blocks_for(p.R, 256), 256, 0, s>>>(p, x, vel, h, x_hat);
  return cudaGetLastError();
}

// v = (x - x_prev) / h on every vertex (fixed vertices: zero).
__global__ void velocity_kernel(int n, const double* x, const double* x_prev, double inv_h, double* v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (x[i] - x_prev[i]) * inv_h;
}

cudaError_t launch_velocity(int n, const double* x, const double* x_prev, double h, double* v, cudaStream_t s) {
  velocity_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, x, x_prev, 1.0 / h, v);
  return cudaGetLastError();
}

cudaError_t launch_axpy(int n, const double* x, double alpha, const double* d, double* out, cudaStream_t s) {
  axpy_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, x, alpha, d, out);
  return cudaGetLastError();
}

cudaError_t launch_sub(int n, const double* a, const double* b, double* out, cudaStream_t s) {
  sub_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, a, b, out);
  return cudaGetLastError();
}

cudaError_t launch_scatter_direction(const DevProblem& p, const float4* sol, double* d, cudaStream_t s) {
  scatter_direction_kernel<<<blocks_for(p.R, 256), 256, 0, s>>>(p, sol, d);
  return cudaGetLastError();
}

cudaError_t launch_rhs(int R, const double* g, float4* b, cudaStream_t s) {
  rhs_kernel<<<blocks_for(R, 256), 256, 0, s>>>(R, g, b);
  return cudaGetLastError();
}

}  // namespace drape
