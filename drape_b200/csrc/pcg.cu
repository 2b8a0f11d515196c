// Block-Jacobi PCG on the f32 BSR(3x3) Newton matrix as ONE persistent cooperative kernel (sm_100a).
//
// Each CTA owns a contiguous range of block rows for the whole solve. One iteration is two phases separated by
// grid barriers:
//   A  q = A p and p.q, where the direction update p = z + beta p_old is fused into the SpMV's column gathers
//      (p is double-buffered: the owner writes p for its rows into the other buffer while every CTA forms the
//      gathered columns from z and the previous buffer, which nobody writes in this phase);
//   B  alpha = rz / pq, x += alpha p, r -= alpha q, z = D^-1 r, and the partial sums of r.z and r.r.
// The CTA partials of each dot product are summed by every CTA in the same fixed order, so all CTAs take the
// same alpha, beta and stop decision, and the solve is deterministic. Residual replacement (r = b - A x every
// `replace_every` iterations while rr > replace_above^2 rr0, keeping p) follows pcg.rs:213-223.
// Block rows are processed by groups of `LPR` lanes; a group's lanes stride over the row's blocks and reduce
// with xor shuffles. Blocks are read as one 16-byte load from each of two planes plus one 4-byte load.
// Every grid barrier gives up after `spin_limit` cycles, sets `state->error` and the kernel returns (status
// kPcgTimeout), so a stalled launch cannot hang the GPU.
// Reference semantics: pcg.rs:271-296 (solve), 389-439 (State), 479-492 (invert3); WGSL cg_init, spmv_dot,
// update_dot, direction, reduce, residual.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "kernels.h"

namespace drape {
namespace {

__device__ __forceinline__ float4 f4(float a, float b, float c) { return make_float4(a, b, c, 0.0f); }
__device__ __forceinline__ float dot3(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Sense-free generation barrier over all CTAs of the cooperative grid, bounded by `limit` cycles.
__device__ __forceinline__ bool grid_barrier(PcgState* st, unsigned ctas, long long limit) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &st->barrier_gen;
    const unsigned g0 = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(&st->barrier_count, 1u);
    if (arrived == ctas - 1) {
      atomicExch(&st->barrier_count, 0u);
      __threadfence();
      atomicAdd(&st->barrier_gen, 1u);
    } else {
      const long long t0 = clock64();
      while (*gen == g0) {
        if (clock64() - t0 > limit) {
          atomicExch(&st->error, 1);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    ok = *(volatile int*)&st->error == 0;
  }
  __syncthreads();
  return ok;
}

// Sum of two per-thread floats over the CTA, written to partial[slot_a * grid + cta], partial[slot_b * ...].
__device__ __forceinline__ void cta_sum2(float a, float b, float* partial, int slot_a, int slot_b) {
  __shared__ float ra[32], rb[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    ra[threadIdx.x >> 5] = a;
    rb[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float sa = 0.0f, sb = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      sa += ra[w];
      sb += rb[w];
    }
    partial[slot_a * gridDim.x + blockIdx.x] = sa;
    if (slot_b >= 0) partial[slot_b * gridDim.x + blockIdx.x] = sb;
  }
}

// The grid-wide sum of one partial slot, computed identically (same order) by every CTA.
__device__ __forceinline__ float grid_total(const float* partial, int slot) {
  __shared__ float total;
  if (threadIdx.x < 32) {
    float s = 0.0f;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) s += __ldcg(partial + slot * gridDim.x + i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) total = s;
  }
  __syncthreads();
  float t = total;
  __syncthreads();
  return t;
}

// Row r of block k applied to v.
__device__ __forceinline__ void block_apply(const DevBsr& A, int k, float px, float py, float pz, float& y0, float& y1,
                                            float& y2) {
  const float4 m0 = __ldg(A.a0 + k), m1 = __ldg(A.a1 + k);
  const float m8 = __ldg(A.a2 + k);
  y0 += m0.x * px + m0.y * py + m0.z * pz;
  y1 += m0.w * px + m1.x * py + m1.y * pz;
  y2 += m1.z * px + m1.w * py + m8 * pz;
}

template <int LPR>
__device__ __forceinline__ void group_reduce(float& y0, float& y1, float& y2) {
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) {
    y0 += __shfl_xor_sync(0xffffffffu, y0, o, LPR);
    y1 += __shfl_xor_sync(0xffffffffu, y1, o, LPR);
    y2 += __shfl_xor_sync(0xffffffffu, y2, o, LPR);
  }
}

template <int LPR>
__global__ void __launch_bounds__(256) pcg_kernel(PcgArgs a) {
  const unsigned G = gridDim.x;
  const int cta = blockIdx.x;
  const int r_begin = (int)((long long)a.R * cta / G), r_end = (int)((long long)a.R * (cta + 1) / G);
  const int groups = blockDim.x / LPR, group = threadIdx.x / LPR, gl = threadIdx.x % LPR;
  PcgState* st = a.state;

  // ---- setup: D^-1, x = 0, r = b, z = D^-1 r, p = z; partial r.z, r.r
  float rz_l = 0.0f, rr_l = 0.0f;
  for (int row = r_begin + threadIdx.x; row < r_end; row += blockDim.x) {
    const int k = a.diag_pos[row];
    const float4 m0 = a.A.a0[k], m1 = a.A.a1[k];
    const float m8 = a.A.a2[k];
    // Adjugate inverse in the reference's operation order (pcg.rs:479-492).
    const float A_ = m0.x, B_ = m0.y, C_ = m0.z, D_ = m0.w, E_ = m1.x, F_ = m1.y, G_ = m1.z, H_ = m1.w, I_ = m8;
    const float c00 = E_ * I_ - F_ * H_, c01 = C_ * H_ - B_ * I_, c02 = B_ * F_ - C_ * E_;
    const float c10 = F_ * G_ - D_ * I_, c11 = A_ * I_ - C_ * G_, c12 = C_ * D_ - A_ * F_;
    const float c20 = D_ * H_ - E_ * G_, c21 = B_ * G_ - A_ * H_, c22 = A_ * E_ - B_ * D_;
    const float det = A_ * c00 + B_ * c10 + C_ * c20;
    const float4 d0 = f4(c00 / det, c01 / det, c02 / det), d1 = f4(c10 / det, c11 / det, c12 / det),
                 d2 = f4(c20 / det, c21 / det, c22 / det);
    a.dinv[3 * row] = d0;
    a.dinv[3 * row + 1] = d1;
    a.dinv[3 * row + 2] = d2;
    const float4 b = a.b[row];
    const float4 z = f4(dot3(d0, b), dot3(d1, b), dot3(d2, b));
    a.x[row] = f4(0.f, 0.f, 0.f);
    a.r[row] = b;
    a.z[row] = z;
    a.p0[row] = z;
    rz_l += dot3(b, z);
    rr_l += dot3(b, b);
  }
  cta_sum2(rz_l, rr_l, a.partial, 1, 2);
  if (!grid_barrier(st, G, a.spin_limit)) return;
  float rz = grid_total(a.partial, 1), rr = grid_total(a.partial, 2);
  const float rr0 = rr;
  int status = rr <= 0.0f ? kPcgConverged : kPcgRunning;
  int it = 0, cur = 0, replacements = 0;
  bool fused = false;
  float beta = 0.0f, alpha = 0.0f, pq = 0.0f;

  while (status == kPcgRunning) {
    // ---- phase A: p (fused update), q = A p, partial p.q
    float4* pold = cur ? a.p1 : a.p0;
    float4* pnew = cur ? a.p0 : a.p1;
    float pq_l = 0.0f;
    // Uniform trip count across the CTA: every lane reaches the group shuffles in every pass.
    for (int row0 = r_begin; row0 < r_end; row0 += groups) {
      const int row = row0 + group;
      const bool active = row < r_end;
      float y0 = 0.f, y1 = 0.f, y2 = 0.f;
      const int kb = active ? a.row_ptr[row] : 0, ke = active ? a.row_ptr[row + 1] : 0;
      for (int k = kb + gl; k < ke; k += LPR) {
        const int c = __ldg(a.col_idx + k);
        float4 pc = __ldcg(pold + c);
        if (fused) {
          const float4 zc = __ldcg(a.z + c);
          pc = f4(zc.x + beta * pc.x, zc.y + beta * pc.y, zc.z + beta * pc.z);
        }
        block_apply(a.A, k, pc.x, pc.y, pc.z, y0, y1, y2);
      }
      group_reduce<LPR>(y0, y1, y2);
      if (active && gl == 0) {
        float4 p = pold[row];
        if (fused) {
          const float4 z = a.z[row];
          p = f4(z.x + beta * p.x, z.y + beta * p.y, z.z + beta * p.z);
          pnew[row] = p;
        }
        const float4 q = f4(y0, y1, y2);
        a.q[row] = q;
        pq_l += dot3(p, q);
      }
    }
    cta_sum2(pq_l, 0.0f, a.partial, 0, -1);
    if (!grid_barrier(st, G, a.spin_limit)) return;
    pq = grid_total(a.partial, 0);
    if (!(pq > 0.0f) || !isfinite(pq)) {
      status = kPcgBreakdown;
      break;
    }
    const float4* p_it = fused ? pnew : pold;
    if (fused) cur ^= 1;
    alpha = rz / pq;
    // ---- phase B: x, r, z; partial r.z, r.r
    rz_l = rr_l = 0.0f;
    for (int row = r_begin + threadIdx.x; row < r_end; row += blockDim.x) {
      const float4 p = p_it[row], q = a.q[row];
      float4 x = a.x[row], r = a.r[row];
      x = f4(x.x + alpha * p.x, x.y + alpha * p.y, x.z + alpha * p.z);
      r = f4(r.x - alpha * q.x, r.y - alpha * q.y, r.z - alpha * q.z);
      const float4 z = f4(dot3(a.dinv[3 * row], r), dot3(a.dinv[3 * row + 1], r), dot3(a.dinv[3 * row + 2], r));
      a.x[row] = x;
      a.r[row] = r;
      a.z[row] = z;
      rz_l += dot3(r, z);
      rr_l += dot3(r, r);
    }
    cta_sum2(rz_l, rr_l, a.partial, 1, 2);
    if (!grid_barrier(st, G, a.spin_limit)) return;
    const float rz_new = grid_total(a.partial, 1);
    rr = grid_total(a.partial, 2);
    beta = rz_new / rz;
    rz = rz_new;
    ++it;
    fused = true;
    if (rr <= a.tol2 * rr0) {
      status = kPcgConverged;
      break;
    }
    if (it >= a.max_iterations) {
      status = kPcgIterationLimit;
      break;
    }
    if (a.replace_every > 0 && it % a.replace_every == 0 && rr > a.replace_above2 * rr0) {
      // Keep the direction: p = z + beta p_old for the own rows now, then r = b - A x, z = D^-1 r.
      float4* po = cur ? a.p1 : a.p0;
      float4* pn = cur ? a.p0 : a.p1;
      for (int row = r_begin + threadIdx.x; row < r_end; row += blockDim.x) {
        const float4 z = a.z[row], p = po[row];
        pn[row] = f4(z.x + beta * p.x, z.y + beta * p.y, z.z + beta * p.z);
      }
      cur ^= 1;
      fused = false;
      // A grid barrier, not just a CTA one: every CTA must have read the phase-B totals of slots 1 and 2
      // (grid_total above) before any CTA rewrites them below.
      if (!grid_barrier(st, G, a.spin_limit)) return;
      rz_l = rr_l = 0.0f;
      for (int row0 = r_begin; row0 < r_end; row0 += groups) {
        const int row = row0 + group;
        const bool active = row < r_end;
        float y0 = 0.f, y1 = 0.f, y2 = 0.f;
        const int kb = active ? a.row_ptr[row] : 0, ke = active ? a.row_ptr[row + 1] : 0;
        for (int k = kb + gl; k < ke; k += LPR) {
          const float4 xc = __ldcg(a.x + __ldg(a.col_idx + k));
          block_apply(a.A, k, xc.x, xc.y, xc.z, y0, y1, y2);
        }
        group_reduce<LPR>(y0, y1, y2);
        if (active && gl == 0) {
          const float4 b = a.b[row];
          const float4 r = f4(b.x - y0, b.y - y1, b.z - y2);
          const float4 z = f4(dot3(a.dinv[3 * row], r), dot3(a.dinv[3 * row + 1], r), dot3(a.dinv[3 * row + 2], r));
          a.r[row] = r;
          a.z[row] = z;
          rz_l += dot3(r, z);
          rr_l += dot3(r, r);
        }
      }
      cta_sum2(rz_l, rr_l, a.partial, 1, 2);
      if (!grid_barrier(st, G, a.spin_limit)) return;
      rz = grid_total(a.partial, 1);
      rr = grid_total(a.partial, 2);
      ++replacements;
    }
  }
  if (cta == 0 && threadIdx.x == 0) {
    st->rz = rz;
    st->rr = rr;
    st->rr0 = rr0;
    st->pq = pq;
    st->alpha = alpha;
    st->beta = beta;
    st->iterations = it;
    st->status = status;
    st->replacements = replacements;
  }
}

template <int LPR>
__global__ void __launch_bounds__(256) spmv_kernel(int R, const int* __restrict__ row_ptr, const int* __restrict__ col_idx,
                                                   DevBsr A, const float4* __restrict__ p, float4* __restrict__ y) {
  const int groups = blockDim.x / LPR;
  const int gl = threadIdx.x % LPR;
  // Uniform trip count across the grid so every lane reaches the group shuffles.
  for (int row0 = blockIdx.x * groups; row0 < R; row0 += gridDim.x * groups) {
    const int row = row0 + threadIdx.x / LPR;
    const bool active = row < R;
    float y0 = 0.f, y1 = 0.f, y2 = 0.f;
    const int kb = active ? row_ptr[row] : 0, ke = active ? row_ptr[row + 1] : 0;
    for (int k = kb + gl; k < ke; k += LPR) {
      const float4 pc = __ldg(p + __ldg(col_idx + k));
      block_apply(A, k, pc.x, pc.y, pc.z, y0, y1, y2);
    }
    group_reduce<LPR>(y0, y1, y2);
    if (active && gl == 0) y[row] = f4(y0, y1, y2);
  }
}

// r = b64 - A d computed in f64 from the f32 blocks; one 8-lane group per row.
__global__ void __launch_bounds__(256) refine_residual_kernel(int R, const int* row_ptr, const int* col_idx, DevBsr A,
                                                              const double* neg_g, const float4* d, float4* r_out,
                                                              double* partial) {
  __shared__ double red[32];
  const int gl = threadIdx.x & 7;
  double s = 0.0;
  const int groups = blockDim.x >> 3;
  // Uniform trip count across the grid so every lane reaches the group shuffles.
  for (int row0 = blockIdx.x * groups; row0 < R; row0 += gridDim.x * groups) {
    const int row = row0 + (threadIdx.x >> 3);
    const bool active = row < R;
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    const int kb = active ? row_ptr[row] : 0, ke = active ? row_ptr[row + 1] : 0;
    for (int k = kb + gl; k < ke; k += 8) {
      const float4 dc = d[col_idx[k]];
      const float4 m0 = A.a0[k], m1 = A.a1[k];
      const float m8 = A.a2[k];
      y0 += double(m0.x) * dc.x + double(m0.y) * dc.y + double(m0.z) * dc.z;
      y1 += double(m0.w) * dc.x + double(m1.x) * dc.y + double(m1.y) * dc.z;
      y2 += double(m1.z) * dc.x + double(m1.w) * dc.y + double(m8) * dc.z;
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      y0 += __shfl_xor_sync(0xffffffffu, y0, o, 8);
      y1 += __shfl_xor_sync(0xffffffffu, y1, o, 8);
      y2 += __shfl_xor_sync(0xffffffffu, y2, o, 8);
    }
    if (active && gl == 0) {
      // neg_g holds the f64 gradient g; the right-hand side is -g.
      const double r0 = -neg_g[3 * row] - y0, r1 = -neg_g[3 * row + 1] - y1, r2 = -neg_g[3 * row + 2] - y2;
      r_out[row] = f4(float(r0), float(r1), float(r2));
      s += r0 * r0 + r1 * r1 + r2 * r2;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void add_rows_kernel(int R, float4* d, const float4* e) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) {
    const float4 a = d[r], b = e[r];
    d[r] = f4(a.x + b.x, a.y + b.y, a.z + b.z);
  }
}

template <int LPR> const void* pcg_entry() { return reinterpret_cast<const void*>(&pcg_kernel<LPR>); }

const void* pcg_fn(int lpr) {
  switch (lpr) {
    case 4: return pcg_entry<4>();
    case 8: return pcg_entry<8>();
    case 16: return pcg_entry<16>();
    case 32: return pcg_entry<32>();
  }
  return nullptr;
}

}  // namespace

int pcg_max_grid(int threads, int lanes_per_row) {
  const void* fn = pcg_fn(lanes_per_row);
  if (!fn) return 0;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0) != cudaSuccess) return 0;
  return sms * per_sm;
}

cudaError_t launch_pcg(const PcgArgs& a, const PcgLaunch& cfg, cudaStream_t s) {
  const void* fn = pcg_fn(cfg.lanes_per_row);
  if (!fn || cfg.threads % 32 != 0 || cfg.threads > 256 || cfg.grid < 1) return cudaErrorInvalidValue;
  PcgArgs args = a;
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel(fn, dim3(cfg.grid), dim3(cfg.threads), params, 0, s);
}

cudaError_t launch_spmv(int R, const int* row_ptr, const int* col_idx, DevBsr A, const float4* p, float4* y,
                        int lanes_per_row, int threads, cudaStream_t s) {
  const int groups = threads / lanes_per_row;
  const int grid = (R + groups - 1) / groups;
  switch (lanes_per_row) {
    case 4: spmv_kernel<4><<<grid, threads, 0, s>>>(R, row_ptr, col_idx, A, p, y); break;
    case 8: spmv_kernel<8><<<grid, threads, 0, s>>>(R, row_ptr, col_idx, A, p, y); break;
    case 16: spmv_kernel<16><<<grid, threads, 0, s>>>(R, row_ptr, col_idx, A, p, y); break;
    case 32: spmv_kernel<32><<<grid, threads, 0, s>>>(R, row_ptr, col_idx, A, p, y); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_refine_residual(int R, const int* row_ptr, const int* col_idx, DevBsr A, const double* g,
                                   const float4* d, float4* r_out, double* partial, int grid, cudaStream_t s) {
  refine_residual_kernel<<<grid, 256, 0, s>>>(R, row_ptr, col_idx, A, g, d, r_out, partial);
  return cudaGetLastError();
}

cudaError_t launch_add_rows(int R, float4* d, const float4* e, cudaStream_t s) {
  add_rows_kernel<<<(R + 255) / 256, 256, 0, s>>>(R, d, e);
  return cudaGetLastError();
}

}  // namespace drape
