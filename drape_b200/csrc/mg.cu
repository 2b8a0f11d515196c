// Multilevel V-cycle preconditioner and flexible PCG (see mg.h for the hierarchy, layouts and the cycle).
//
// Every PCG iteration is a fixed sequence of small kernels (the kernel boundaries are the grid-wide syncs):
//   restrict 0->1 (+ convergence test), restrict l->l+1 ..., coarse solve, prolong+post-smooth ... l+1->l,
//   prolong+post-smooth 1->0 (partials z.r, z.r_prev), direction + SpMV (partial p.q), update (partial r.r, next
//   pre-smoothing).
// Dot products are per-CTA partials summed by every CTA of the next kernel in one fixed order, so all CTAs take
// the same decisions and a solve is bit-for-bit repeatable. After convergence, breakdown or the iteration limit
// (state->done) every kernel returns at once, so a launch sequence longer than needed costs only launch latency.
#include <cuda_runtime.h>

#include <cooperative_groups.h>

#include "bulk.cuh"
#include "mg.h"

namespace drape {
namespace {

constexpr int kLanes = 8;               // lanes per row in level row kernels
constexpr int kRowThreads = 256;        // 32 rows per CTA
constexpr int kRestrictRows = 8;        // coarse rows per restriction CTA (one warp each)
constexpr int kRestrictThreads = 32 * kRestrictRows;
constexpr int kUpdateThreads = 256;     // one thread per row

enum { kPartZr = 0, kPartZrPrev = 1, kPartPq = 2, kPartRr = 3 };

// Programmatic dependent launch. Each kernel of the cycle first waits for the previous grid (griddepcontrol.wait
// returns once it has completed and its writes are visible) and only then lets the next kernel launch. So when a
// kernel starts, the kernel before its predecessor has completed: the code before its own wait may read anything
// written two or more kernels back (the static matrix, the row structure, vectors of earlier phases) and so
// overlaps those loads with the predecessor's tail; what the predecessor writes is read only after the wait. Both
// instructions are no-ops for a kernel launched without the attribute (then every earlier kernel has completed).
__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Pulls the cache line of p into L1 ahead of its use.
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// A 36-byte f32 block of the fine BSR planes (a0, a1 16 bytes, a2 4 bytes) into L1.
__device__ __forceinline__ void prefetch_block(const DevBsr& A, int k) {
  prefetch_l1(A.a0 + k);
  prefetch_l1(A.a1 + k);
  prefetch_l1(A.a2 + k);
}

// A 48-byte coarse stencil block into L1 (it may straddle two 128-byte lines).
__device__ __forceinline__ void prefetch_stencil(const float4* A, int w2, int I, int o) {
  const float4* b = A + (size_t(I) * w2 + o) * 3;
  prefetch_l1(b);
  prefetch_l1(b + 2);
}

template <typename... Params, typename... Args>
cudaError_t launch(void (*kernel)(Params...), int grid, int block, cudaStream_t s, bool pdl, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}
// The same with dynamic shared memory (the kernel's ceiling raised to it first).
template <typename... Params, typename... Args>
cudaError_t launch_smem(void (*kernel)(Params...), int grid, int block, size_t smem, cudaStream_t s, bool pdl,
                        Args... args) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}
enum { kStatusRunning = 0, kStatusConverged = 1, kStatusLimit = 2, kStatusBreakdown = 3, kStatusStalled = 4 };

__device__ __forceinline__ void load_block(const DevBsr& A, int k, float m[9]) {
  float4 u = A.a0[k], v = A.a1[k];
  m[0] = u.x; m[1] = u.y; m[2] = u.z; m[3] = u.w;
  m[4] = v.x; m[5] = v.y; m[6] = v.z; m[7] = v.w;
  m[8] = A.a2[k];
}

__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 scale3(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float4 pack(float3 a) { return make_float4(a.x, a.y, a.z, 0.0f); }

__device__ __forceinline__ float3 mul(const float m[9], float3 v) {
  return make_float3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
                     m[6] * v.x + m[7] * v.y + m[8] * v.z);
}
// S r with S stored as [9][rows]; transposed: S^T r.
__device__ __forceinline__ float3 smooth(const float* S, int rows, int i, float3 r, bool transpose) {
  float m[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) m[e] = S[e * rows + i];
  if (!transpose) return mul(m, r);
  return make_float3(m[0] * r.x + m[3] * r.y + m[6] * r.z, m[1] * r.x + m[4] * r.y + m[7] * r.z,
                     m[2] * r.x + m[5] * r.y + m[8] * r.z);
}

// Column vertex J of offset o in a stencil of width w around (X, Y) on an n x n grid (false outside the grid).
__device__ __forceinline__ bool stencil_neighbour(int n, int w, int X, int Y, int o, int* J) {
  const int h = w >> 1;
  int dx = o % w - h, dy = o / w - h, x = X + dx, y = Y + dy;
  if (x < 0 || y < 0 || x >= n || y >= n) return false;
  *J = y * n + x;
  return true;
}

// Block (I, o) of a coarse level's f32 stencil (w2 = w * w offsets per row) times v.
__device__ __forceinline__ float3 stencil_apply(const float4* A, int w2, int I, int o, float3 v) {
  const float4* b = A + (size_t(I) * w2 + o) * 3;
  const float4 u = b[0], w = b[1], t = b[2];
  const float m[9] = {u.x, u.y, u.z, u.w, w.x, w.y, w.z, w.w, t.x};
  return mul(m, v);
}

// 1D bilinear weight of fine index f for coarse index C (fine position 2C).
__device__ __forceinline__ double w1d(int f, int C) {
  int d = f - 2 * C;
  return d == 0 ? 1.0 : (d == 1 || d == -1) ? 0.5 : 0.0;
}

// (P e)(fine vertex x, y): the bilinear interpolation of the coarse correction.
__device__ __forceinline__ float3 interpolate(const float4* e, int nc, int x, int y) {
  int X0 = x >> 1, Y0 = y >> 1;
  int nx = (x & 1) ? 2 : 1, ny = (y & 1) ? 2 : 1;
  float wx = (x & 1) ? 0.5f : 1.0f, wy = (y & 1) ? 0.5f : 1.0f;
  float3 s = make_float3(0.f, 0.f, 0.f);
  for (int b = 0; b < ny; ++b)
    for (int a = 0; a < nx; ++a) s = add3(s, scale3(wx * wy, f3(e[(Y0 + b) * nc + X0 + a])));
  return s;
}

// Sum of n per-CTA partials, the same value in every thread and every CTA (fixed order).
__device__ float sum_partials(const float* p, int n) {
  __shared__ float warp_sums[32];
  float s = 0.0f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += p[i];
#pragma unroll
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = s;
  __syncthreads();
  float t = 0.0f;
  const int nw = (blockDim.x + 31) >> 5;
  for (int w = 0; w < nw; ++w) t += warp_sums[w];
  __syncthreads();
  return t;
}

// Per-CTA sum of one value per thread (fixed order); the result is valid in thread 0.
__device__ float cta_sum(float v) {
  __shared__ float warp_sums[32];
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = v;
  __syncthreads();
  float t = 0.0f;
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) t += warp_sums[w];
  }
  __syncthreads();
  return t;
}

__device__ __forceinline__ float3 group_sum(float3 v) {
#pragma unroll
  for (int o = kLanes / 2; o; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    v.z += __shfl_xor_sync(0xffffffffu, v.z, o);
  }
  return v;
}

int row_grid(int rows) { return (rows + kRowThreads / kLanes - 1) / (kRowThreads / kLanes); }
int update_grid(int rows) { return (rows + kUpdateThreads - 1) / kUpdateThreads; }
int restrict_grid(int coarse_rows) { return (coarse_rows + kRestrictRows - 1) / kRestrictRows; }

// ---------------------------------------------------------------------------------------------- set-up

// A_{l+1}[I][o] = sum_{i in supp I} sum_{j} w(i, I) A_l(i, j) w(j, J), J = I + offset(o); f64 sums.
// One warp per coarse row: the warp first stages the nine fine support rows' entries (column, weight, block) in
// shared memory, then lane o < 25 sums the entries landing on offset o, in entry order (deterministic).
// kSrcW: 0 for the fine BSR level (<= 25 blocks per row), else the source stencil width (5 or 7). The staged
// entries of one warp take 9 x 25 x 88 B (2 warps per CTA) or 9 x 49 x 88 B (7 x 7 source: 1 warp per CTA).
struct GalerkinEntry {
  double m[9];
  double w;
  int jx, jy;  // the fine column's grid coordinates (jx < 0: outside the grid)
};

template <int kSrcW>
struct GalerkinShape {
  static constexpr int kEntries = 9 * (kSrcW == 7 ? kMgStencilWide : kMgStencil);
  static constexpr int kWarps = kSrcW == 7 ? 1 : 2;
};

template <int kSrcW>
__global__ void __launch_bounds__(32 * GalerkinShape<kSrcW>::kWarps) galerkin_kernel(MgFine fine, MgLevel src,
                                                                                       MgLevel dst, int* error) {
  constexpr bool kSrcBsr = kSrcW == 0;
  constexpr int kGalerkinWarps = GalerkinShape<kSrcW>::kWarps;
  constexpr int kGalerkinEntries = GalerkinShape<kSrcW>::kEntries;
  constexpr int kSrcW2 = kSrcW * kSrcW;
  __shared__ GalerkinEntry list[kGalerkinWarps][kGalerkinEntries];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int I = blockIdx.x * kGalerkinWarps + warp;
  if (I >= dst.rows) return;  // whole warps leave together
  const int nc = dst.n, nf = src.n, X = I % nc, Y = I / nc;
  GalerkinEntry* L = list[warp];
  // fine support row s = lane (lanes 0..8): its first entry and count
  // (a stencil source reserves its w^2 slots for every support row, inside the grid or not, so row s's entries start
  // at s w^2)
  int i = -1, first = 0, len = 0;
  if (lane < 9) {
    const int fx = 2 * X + lane % 3 - 1, fy = 2 * Y + lane / 3 - 1;
    if (!kSrcBsr) len = kSrcW2;
    if (fx >= 0 && fy >= 0 && fx < nf && fy < nf) {
      i = fy * nf + fx;
      if (kSrcBsr) {
        first = fine.row_ptr[i];
        len = fine.row_ptr[i + 1] - first;
      }
    }
  }
  int offset = len;  // exclusive prefix over lanes 0..8
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, offset, o);
    if (lane >= o) offset += v;
  }
  const int total = __shfl_sync(0xffffffffu, offset, 8);
  offset -= len;
  if (total > kGalerkinEntries) {  // a pattern wider than the 5 x 5 stencil layout: report, write nothing
    if (lane == 0) *error = 2;
    return;
  }
  for (int s = 0; s < 9; ++s) {
    const int si = __shfl_sync(0xffffffffu, i, s), sf = __shfl_sync(0xffffffffu, first, s);
    const int sl = __shfl_sync(0xffffffffu, len, s), so = __shfl_sync(0xffffffffu, offset, s);
    if (si < 0) continue;
    const double wi = (s % 3 != 1 ? 0.5 : 1.0) * (s / 3 != 1 ? 0.5 : 1.0);
    for (int t = lane; t < sl; t += 32) {
      GalerkinEntry& E = L[so + t];
      E.w = wi;
      if (kSrcBsr) {
        const int k = sf + t;
        const int j = fine.col_idx[k];
        E.jx = j % nf;
        E.jy = j / nf;
        float m[9];
        load_block(fine.A, k, m);
#pragma unroll
        for (int e = 0; e < 9; ++e) E.m[e] = m[e];
      } else {
        int j;
        const bool in = stencil_neighbour(nf, kSrcW, si % nf, si / nf, t, &j);
        E.jx = in ? j % nf : -1;
        E.jy = in ? j / nf : -1;
#pragma unroll
        for (int e = 0; e < 9; ++e) E.m[e] = in ? src.A64[(t * 9 + e) * src.rows + si] : 0.0;
      }
    }
  }
  __syncwarp();
  const unsigned staged = __ballot_sync(0xffffffffu, lane < 9 && i >= 0);  // support rows inside the fine grid
  if (lane < kMgStencil) {
    double acc[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) acc[e] = 0.0;
    int J;
    if (stencil_neighbour(nc, 5, X, Y, lane, &J)) {
      if (kSrcBsr) {  // the fine row's entries are its BSR blocks: find the ones whose column J interpolates
        const int JX = J % nc, JY = J / nc;
        for (int t = 0; t < total; ++t) {
          const GalerkinEntry& E = L[t];
          if (E.jx < 0) continue;
          const double wj = w1d(E.jx, JX) * w1d(E.jy, JY);
          if (wj == 0.0) continue;
          const double w = E.w * wj;
#pragma unroll
          for (int e = 0; e < 9; ++e) acc[e] += w * E.m[e];
        }
      } else {
        // A stencil source's entry for fine support row i = 2I + a and column j = 2J + c sits at offset
        // b = j - i = 2 (J - I) + c - a of row a's staged stencil: the (a, c) pairs enumerate the terms directly.
        constexpr int h = kSrcW / 2;
        const int dX = lane % 5 - 2, dY = lane / 5 - 2;
        for (int sa = 0; sa < 9; ++sa) {
          if (!((staged >> sa) & 1u)) continue;
          const int ax = sa % 3 - 1, ay = sa / 3 - 1;
          const double wa = (ax ? 0.5 : 1.0) * (ay ? 0.5 : 1.0);
#pragma unroll
          for (int sc = 0; sc < 9; ++sc) {
            const int cx = sc % 3 - 1, cy = sc / 3 - 1;
            const int bx = 2 * dX + cx - ax, by = 2 * dY + cy - ay;
            if (bx < -h || bx > h || by < -h || by > h) continue;
            const GalerkinEntry& E = L[sa * kSrcW2 + (by + h) * kSrcW + bx + h];
            if (E.jx < 0) continue;  // column outside the fine grid
            const double w = wa * (cx ? 0.5 : 1.0) * (cy ? 0.5 : 1.0);
#pragma unroll
            for (int e = 0; e < 9; ++e) acc[e] += w * E.m[e];
          }
        }
      }
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) dst.A64[(lane * 9 + e) * dst.rows + I] = acc[e];
    float4* b = dst.A + (size_t(I) * kMgStencil + lane) * 3;
    b[0] = make_float4(float(acc[0]), float(acc[1]), float(acc[2]), float(acc[3]));
    b[1] = make_float4(float(acc[4]), float(acc[5]), float(acc[6]), float(acc[7]));
    b[2] = make_float4(float(acc[8]), 0.0f, 0.0f, 0.0f);
  }
}

__device__ void inverse3(const double m[9], double omega, float out[9]) {
  double c[9];
  c[0] = m[4] * m[8] - m[5] * m[7];
  c[1] = m[2] * m[7] - m[1] * m[8];
  c[2] = m[1] * m[5] - m[2] * m[4];
  c[3] = m[5] * m[6] - m[3] * m[8];
  c[4] = m[0] * m[8] - m[2] * m[6];
  c[5] = m[2] * m[3] - m[0] * m[5];
  c[6] = m[3] * m[7] - m[4] * m[6];
  c[7] = m[1] * m[6] - m[0] * m[7];
  c[8] = m[0] * m[4] - m[1] * m[3];
  const double det = m[0] * c[0] + m[1] * c[3] + m[2] * c[6];
  const bool ok = det != 0.0 && isfinite(det);
#pragma unroll
  for (int e = 0; e < 9; ++e) out[e] = ok ? float(omega * c[e] / det) : 0.0f;
}

// S = omega D^{-1} per row (D the diagonal block).
template <bool kBsr>
__global__ void jacobi_smoother_kernel(MgFine fine, MgLevel lv, double omega) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= lv.rows) return;
  double m[9];
  if (kBsr) {
    float f[9];
    load_block(fine.A, fine.diag_pos[i], f);
#pragma unroll
    for (int e = 0; e < 9; ++e) m[e] = f[e];
  } else {
    const int centre = (lv.w * lv.w - 1) / 2;
#pragma unroll
    for (int e = 0; e < 9; ++e) m[e] = lv.A64[(centre * 9 + e) * lv.rows + i];
  }
  float s[9];
  inverse3(m, omega, s);
#pragma unroll
  for (int e = 0; e < 9; ++e) lv.S[e * lv.rows + i] = s[e];
}

// Sp = omega_P D^{-1} for the smoothed prolongation. S0 holds `scale` D^{-1} when this runs (scale 1 before the
// power method scales the smoothers; a fixed damping omega otherwise). omega_P = kMgProlongC / lambda with
// lambda = 2 / (1.1 omega_0 (1 + 1/30)), the power-method estimate of lambda_max(D^{-1} A) behind the level-0
// damping omega_0 (the fixed omega when `fixed`): Sp = kMgProlongC * 1.1 * (1 + 1/30) / 2 * omega_0 / scale * S0.
__global__ void sp_kernel(int count, const float* S0, const float* omega, int fixed, float* Sp) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const float c = kMgProlongC * 1.1f * (1.0f + 1.0f / 30.0f) * 0.5f;
  Sp[t] = (fixed ? c : c * omega[0]) * S0[t];
}

// Level 1 under the smoothed prolongation P_0 = (I - Sp A) P (mg.h), for coarse row I at fine vertex c = 2I:
//   B_i = P_0[i, I] = P(i, I) Id - Sp_i sum_k A_ik P(k, I)     fine rows i within 3 of c (P(k, I) != 0 within 1)
//   W_j = sum_i A_ji B_i                                      within 5
//   Z_k = sum_j A_kj Sp_j W_j,  V_k = W_k - Z_k                within 7
//   A_1[I, J] = sum_k P(k, J) V_k^T                           J within 3 of I (7 x 7)
// which is P_0^T A P_0 for a symmetric A (A_ij = A_ji^T) and symmetric Sp blocks: sum_i P_0[i,I]^T A_ij = W_j^T and
// sum_j W_j^T P_0[j, J] = sum_k P(k, J) (W_k - Z_k)^T. The ring J - I = 4, the only part dropped, holds products of
// the weak axial hinge couplings (~1e-12 of the largest entry). One CTA per coarse row, the three windows in shared
// memory in f64 (37 KB), 8 lanes per fine row and 4 rows per warp; sums in a fixed order (deterministic).
constexpr int kGsWarps = 8;
__device__ __forceinline__ void reduce8(double v[9]) {
#pragma unroll
  for (int o = 4; o; o >>= 1)
#pragma unroll
    for (int e = 0; e < 9; ++e) v[e] += __shfl_xor_sync(0xffffffffu, v[e], o);
}

__global__ void __launch_bounds__(32 * kGsWarps, 3) galerkin_smoothed_kernel(MgFine fine, const float* Sp, MgLevel dst) {
  __shared__ double sB[49][9], sW[121][9], sY[121][9], sV[225][9];
  const int I = blockIdx.x;
  const int nc = dst.n, nf = fine.n, R = fine.R;
  const int X = I % nc, Y = I / nc, cx = 2 * X, cy = 2 * Y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, sub = lane >> 3, l8 = lane & 7;
  // fine row of window index w (width ww, radius ww / 2) around c; -1 outside the grid
  auto window_row = [&](int w, int ww) {
    const int h = ww >> 1, fx = cx + w % ww - h, fy = cy + w / ww - h;
    return (fx >= 0 && fy >= 0 && fx < nf && fy < nf) ? fy * nf + fx : -1;
  };
  // window index of fine column j in the window of width ww around c; -1 outside it
  auto window_of = [&](int j, int ww) {
    const int h = ww >> 1, dx = j % nf - cx + h, dy = j / nf - cy + h;
    return (dx >= 0 && dy >= 0 && dx < ww && dy < ww) ? dy * ww + dx : -1;
  };
  auto sp_block = [&](int i, double m[9]) {
#pragma unroll
    for (int e = 0; e < 9; ++e) m[e] = Sp[e * R + i];
  };
  // Stage 1: B over the 7 x 7 window.
  for (int base = warp * 4; base < 49; base += kGsWarps * 4) {
    const int w = base + sub;
    const int i = w < 49 ? window_row(w, 7) : -1;
    double acc[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) acc[e] = 0.0;
    if (i >= 0) {
      for (int k = fine.row_ptr[i] + l8; k < fine.row_ptr[i + 1]; k += 8) {
        const int j = fine.col_idx[k];
        const double p = w1d(j % nf, X) * w1d(j / nf, Y);
        if (p == 0.0) continue;
        float m[9];
        load_block(fine.A, k, m);
#pragma unroll
        for (int e = 0; e < 9; ++e) acc[e] += p * m[e];
      }
    }
    reduce8(acc);
    if (w < 49 && l8 == 0) {
      if (i < 0) {
#pragma unroll
        for (int e = 0; e < 9; ++e) sB[w][e] = 0.0;
      } else {
        double sp[9];
        sp_block(i, sp);
        const double p = w1d(i % nf, X) * w1d(i / nf, Y);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b)
            sB[w][3 * a + b] = (a == b ? p : 0.0) -
                               (sp[3 * a] * acc[b] + sp[3 * a + 1] * acc[3 + b] + sp[3 * a + 2] * acc[6 + b]);
      }
    }
  }
  __syncthreads();
  // Stage 2: W = A B over the 11 x 11 window, Y = Sp W.
  for (int base = warp * 4; base < 121; base += kGsWarps * 4) {
    const int w = base + sub;
    const int j = w < 121 ? window_row(w, 11) : -1;
    double acc[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) acc[e] = 0.0;
    if (j >= 0) {
      for (int k = fine.row_ptr[j] + l8; k < fine.row_ptr[j + 1]; k += 8) {
        const int wb = window_of(fine.col_idx[k], 7);
        if (wb < 0) continue;
        float m[9];
        load_block(fine.A, k, m);
        const double* b = sB[wb];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c)
            acc[3 * a + c] += m[3 * a] * b[c] + m[3 * a + 1] * b[3 + c] + m[3 * a + 2] * b[6 + c];
      }
    }
    reduce8(acc);
    if (w < 121 && l8 == 0) {
      double sp[9];
      if (j >= 0) sp_block(j, sp);
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          sW[w][3 * a + c] = j >= 0 ? acc[3 * a + c] : 0.0;
          sY[w][3 * a + c] = j >= 0 ? sp[3 * a] * acc[c] + sp[3 * a + 1] * acc[3 + c] + sp[3 * a + 2] * acc[6 + c] : 0.0;
        }
    }
  }
  __syncthreads();
  // Stage 3: V = W - A Y over the 15 x 15 window.
  for (int base = warp * 4; base < 225; base += kGsWarps * 4) {
    const int w = base + sub;
    const int r = w < 225 ? window_row(w, 15) : -1;
    double acc[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) acc[e] = 0.0;
    if (r >= 0) {
      for (int k = fine.row_ptr[r] + l8; k < fine.row_ptr[r + 1]; k += 8) {
        const int wy = window_of(fine.col_idx[k], 11);
        if (wy < 0) continue;
        float m[9];
        load_block(fine.A, k, m);
        const double* b = sY[wy];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c)
            acc[3 * a + c] += m[3 * a] * b[c] + m[3 * a + 1] * b[3 + c] + m[3 * a + 2] * b[6 + c];
      }
    }
    reduce8(acc);
    if (w < 225 && l8 == 0) {
      const int ww = r >= 0 ? window_of(r, 11) : -1;
#pragma unroll
      for (int e = 0; e < 9; ++e) sV[w][e] = r < 0 ? 0.0 : (ww >= 0 ? sW[ww][e] : 0.0) - acc[e];
    }
  }
  __syncthreads();
  // A_1[I, J] = sum_k P(k, J) V_k^T, k the 3 x 3 fine vertices around 2J (all inside the 15 x 15 window).
  for (int t = threadIdx.x; t < kMgStencilWide * 9; t += blockDim.x) {
    const int o = t / 9, e = t % 9, a = e / 3, b = e % 3;
    const int JX = X + o % 7 - 3, JY = Y + o / 7 - 3;
    double v = 0.0;
    if (JX >= 0 && JY >= 0 && JX < nc && JY < nc) {
      for (int q = 0; q < 9; ++q) {
        const int kx = 2 * JX + q % 3 - 1, ky = 2 * JY + q / 3 - 1;
        if (kx < 0 || ky < 0 || kx >= nf || ky >= nf) continue;
        const double p = (q % 3 != 1 ? 0.5 : 1.0) * (q / 3 != 1 ? 0.5 : 1.0);
        v += p * sV[(ky - cy + 7) * 15 + (kx - cx + 7)][3 * b + a];
      }
    }
    dst.A64[(o * 9 + e) * dst.rows + I] = v;
    float* b32 = reinterpret_cast<float*>(dst.A + (size_t(I) * kMgStencilWide + o) * 3);
    b32[e] = float(v);
    if (e < 3) b32[9 + e] = 0.0f;
  }
}

// Dense inverse of the coarsest operator by block Gauss-Jordan elimination over its 3x3 vertex blocks, f64 in shared
// memory, one CTA. The operator is a Galerkin product of a symmetric positive definite matrix, so every pivot block
// (a Schur complement's diagonal block) is symmetric positive definite and no pivoting is needed: step k inverts
// the pivot block P = M[k][k] by its adjugate, scales block row k by P^{-1} and subtracts M[i][k] (block row k) from
// every other block row i. Afterwards the right half holds the inverse. A pivot block whose determinant is not
// positive and finite (the operator is not positive definite) sets *error, which hands the system to block-Jacobi
// PCG. Two CTA barriers per block step (25 steps for the 75 x 75 operator of n = 5).
__global__ void __launch_bounds__(1024) coarse_inverse_kernel(MgLevel lv, float* inv, int* error) {
  extern __shared__ double M[];  // [m][2m]
  __shared__ double s_row[3][6 * kMgCoarsestRowsMax];
  __shared__ double s_fac[3 * kMgCoarsestRowsMax][3];
  const int m = 3 * lv.rows, w = 2 * m, n = lv.n;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  for (int t = threadIdx.x; t < m * w; t += blockDim.x) M[t] = 0.0;
  __syncthreads();
  const int w2 = lv.w * lv.w;
  for (int t = threadIdx.x; t < lv.rows * w2; t += blockDim.x) {
    const int I = t / w2, o = t % w2;
    int J;
    if (!stencil_neighbour(n, lv.w, I % n, I / n, o, &J)) continue;
    for (int e = 0; e < 9; ++e) M[(3 * I + e / 3) * w + 3 * J + e % 3] = lv.A64[(o * 9 + e) * lv.rows + I];
  }
  for (int t = threadIdx.x; t < m; t += blockDim.x) M[t * w + m + t] = 1.0;
  __syncthreads();
  for (int k = 0; k < lv.rows; ++k) {
    const int kb = 3 * k;
    // Columns left of kb are eliminated (unit columns) and right-half columns past m + kb + 2 are still unit
    // columns with zeros in block row k, so the step touches columns kb .. m + kb + 2 only.
    const int c_end = m + kb + 3;
    // P^{-1} by the adjugate, in every thread (nine broadcast reads)
    const double a = M[kb * w + kb], b = M[kb * w + kb + 1], c = M[kb * w + kb + 2];
    const double d = M[(kb + 1) * w + kb], e = M[(kb + 1) * w + kb + 1], f = M[(kb + 1) * w + kb + 2];
    const double g = M[(kb + 2) * w + kb], h = M[(kb + 2) * w + kb + 1], i9 = M[(kb + 2) * w + kb + 2];
    const double c00 = e * i9 - f * h, c01 = c * h - b * i9, c02 = b * f - c * e;
    const double c10 = f * g - d * i9, c11 = a * i9 - c * g, c12 = c * d - a * f;
    const double c20 = d * h - e * g, c21 = b * g - a * h, c22 = a * e - b * d;
    const double det = a * c00 + b * c10 + c * c20;
    const bool ok = det > 0.0 && isfinite(det);
    if (!ok && threadIdx.x == 0) *error = 1;
    const double rd = ok ? 1.0 / det : 0.0;
    for (int t = threadIdx.x; t < 3 * (c_end - kb); t += blockDim.x) {
      const int r = t / (c_end - kb), col = kb + t % (c_end - kb);
      const double p0 = r == 0 ? c00 : r == 1 ? c10 : c20;  // row r of P^{-1} (times det)
      const double p1 = r == 0 ? c01 : r == 1 ? c11 : c21;
      const double p2 = r == 0 ? c02 : r == 1 ? c12 : c22;
      s_row[r][col] = rd * (p0 * M[kb * w + col] + p1 * M[(kb + 1) * w + col] + p2 * M[(kb + 2) * w + col]);
    }
    for (int t = threadIdx.x; t < 3 * m; t += blockDim.x) {
      const int r = t / 3, q = t % 3;
      s_fac[r][q] = r >= kb && r < kb + 3 ? 0.0 : M[r * w + kb + q];
    }
    __syncthreads();
    for (int r = warp; r < m; r += warps) {
      double* row = M + r * w;
      const bool pivot_row = r >= kb && r < kb + 3;
      const double f0 = s_fac[r][0], f1 = s_fac[r][1], f2 = s_fac[r][2];
      for (int col = kb + lane; col < c_end; col += 32)
        row[col] = pivot_row ? s_row[r - kb][col] : row[col] - (f0 * s_row[0][col] + f1 * s_row[1][col] + f2 * s_row[2][col]);
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) inv[t] = float(M[(t / m) * w + m + t % m]);
}

// ---------------------------------------------------------------------------------------------- the cycle

struct RestrictArgs {
  MgFine fine;        // level-0 operator (kSrcBsr)
  MgLevel src, dst;   // src.r / src.z: the level's right-hand side and pre-smoothed correction
  bool coarsest;      // dst is the coarsest level: no pre-smoothing there
  // convergence test (level-0 restriction of a PCG iteration)
  MgState* state;
  const float* rr_partial;
  int rr_count;
};

__device__ __forceinline__ float3 warp_sum3(float3 v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    v.z += __shfl_xor_sync(0xffffffffu, v.z, o);
  }
  return v;
}

// The flexible PCG's stopping test at the start of an iteration (the first kernel of its V-cycle): the residual
// norm from the update kernel's per-CTA partials against the tolerance, non-finite values, the iteration limit
// and, at the end of each stall window, a residual that fell by less than 10 %. Every CTA computes the same sums
// and takes the same decision; CTA 0 records it. Returns true when the solve has ended.
__device__ bool pcg_stop(MgState* st, const float* rr_partial, int rr_count) {
  if (st->done) return true;
  const float rr = sum_partials(rr_partial, rr_count);
  const int it = st->iterations;
  const float rr0 = it == 0 ? rr : st->rr0;
  const bool window_end = it > 0 && st->stall_window > 0 && it % st->stall_window == 0;
  const int window = st->stall_window > 0 ? it / st->stall_window : 0;
  int status = kStatusRunning;
  if (rr <= rr0 * st->tol2) status = kStatusConverged;
  else if (!isfinite(rr)) status = kStatusBreakdown;
  else if (it >= st->max_iterations) status = kStatusLimit;
  else if (window_end && !(rr <= 0.81f * st->stall_rr[(window - 1) & 1])) status = kStatusStalled;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->rr = rr;
    if (it == 0) st->rr0 = rr;
    if (it == 0 || window_end) st->stall_rr[window & 1] = rr;
    if (status != kStatusRunning) {
      st->status = status;
      st->done = 1;
    }
  }
  return status != kStatusRunning;
}

// r_{l+1} = P^T (r_l - A_l z_l), z_{l+1} = S_{l+1} r_{l+1}: one warp per coarse row; lanes 3s .. 3s + 2 take
// the 9 fine support rows s (their blocks or stencil offsets interleaved), lanes 27..31 idle. kSrcW: 0 for the fine
// level (BSR), else the source level's stencil width. Under the smoothed prolongation the fine restriction runs
// with src.r = t and src.z = Sp t (P_0^T t = P^T (t - A Sp t)).
// The level-0 restriction of a flexible PCG iteration first tests convergence, the limit and a stall (kCheck).
template <int kSrcW, bool kCheck>
__global__ void __launch_bounds__(kRestrictThreads) restrict_kernel(RestrictArgs a) {
  constexpr bool kSrcBsr = kSrcW == 0;
  constexpr int kSrcW2 = kSrcW * kSrcW;
  constexpr int kPer = kSrcBsr ? 9 : (kSrcW2 + 2) / 3;  // entries per lane (<= 25 blocks per fine row)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int I = blockIdx.x * kRestrictRows + warp;
  const int s = lane / 3, k3 = lane % 3;
  const int nc = a.dst.n, nf = a.src.n;
  const int X = I % nc, Y = I / nc, ax = s % 3 - 1, by = s / 3 - 1;
  const int fx = 2 * X + ax, fy = 2 * Y + by;
  const bool has_row = I < a.dst.rows && lane < 27 && fx >= 0 && fy >= 0 && fx < nf && fy < nf;
  const int i = has_row ? fy * nf + fx : 0;
  // Before the wait (mg.h's ordering): the row structure, the operator's blocks and the coarse smoother, which no
  // kernel of the solve writes; src.r and src.z come from the previous kernel and are read after it.
  int jj[kPer];
  int k0 = 0;
  if (kSrcBsr) {
    int k1 = 0;
    if (has_row) {
      k0 = a.fine.row_ptr[i] + k3;
      k1 = a.fine.row_ptr[i + 1];
    }
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      jj[t] = has_row && k0 + 3 * t < k1 ? a.fine.col_idx[k0 + 3 * t] : -1;
      if (jj[t] >= 0) prefetch_block(a.fine.A, k0 + 3 * t);
    }
  } else {
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const int o = k3 + 3 * t;
      int j = -1;
      jj[t] = has_row && o < kSrcW2 && stencil_neighbour(nf, kSrcW, fx, fy, o, &j) ? j : -1;
      if (jj[t] >= 0) prefetch_stencil(a.src.A, kSrcW2, i, o);
    }
  }
  float sm[9];
  const bool writer = lane == 0 && I < a.dst.rows && !a.coarsest;
#pragma unroll
  for (int e = 0; e < 9; ++e) sm[e] = writer ? a.dst.S[e * a.dst.rows + I] : 0.0f;
  pdl_wait();
  if (kCheck) {
    if (pcg_stop(a.state, a.rr_partial, a.rr_count)) return;
  } else if (a.state && a.state->done) {
    return;
  }
  float3 t = make_float3(0.f, 0.f, 0.f);
  if (has_row) {
    float3 acc = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      if (jj[q] < 0) continue;
      if (kSrcBsr) {
        float m[9];
        load_block(a.fine.A, k0 + 3 * q, m);
        acc = add3(acc, mul(m, f3(a.src.z[jj[q]])));
      } else {
        acc = add3(acc, stencil_apply(a.src.A, kSrcW2, i, k3 + 3 * q, f3(a.src.z[jj[q]])));
      }
    }
    const float w = (ax ? 0.5f : 1.0f) * (by ? 0.5f : 1.0f);
    t = scale3(w, k3 == 0 ? sub3(f3(a.src.r[i]), acc) : scale3(-1.0f, acc));
  }
  t = warp_sum3(t);
  if (lane == 0 && I < a.dst.rows) {
    a.dst.r[I] = pack(t);
    if (!a.coarsest) a.dst.z[I] = pack(mul(sm, t));
  }
}

struct SmoothedArgs {
  MgFine fine;
  const float4* r;      // residual: fine right-hand side
  const float4* z;      // pre-smoothed z_0
  const float* Sp;      // omega_P D^{-1}
  float4* t;            // out: r - A z_0
  float4* u;            // out: Sp t
  const float4* e1;     // level-1 correction (interp_smoothed_kernel)
  int nc;               // level-1 columns
  float4* y;            // out: z_0 + P_0 e_1
  MgState* state;       // flexible PCG state (null: stand-alone V-cycle)
  const float* rr_partial;
  int rr_count;
  float* rr_init;       // residual_smoothed_kernel at the start of flexible PCG: per-CTA |r|^2 (else null)
};

// Fine step before the smoothed restriction: t = r - A z_0, u = Sp t; inside flexible PCG it first takes the
// iteration's stopping test (kCheck), which restrict_kernel takes without the smoothed prolongation.
// The row structure of fine row i for 8 lanes: each lane's <= 4 column indices (-1 past the row's end) and its
// first block index; the blocks are prefetched into L1.
__device__ __forceinline__ int fine_row(const MgFine& f, int i, bool active, int lane, int jj[4]) {
  int k0 = 0, k1 = 0;
  if (active) {
    k0 = f.row_ptr[i] + lane;
    k1 = f.row_ptr[i + 1];
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    jj[t] = active && k0 + kLanes * t < k1 ? f.col_idx[k0 + kLanes * t] : -1;
    if (jj[t] >= 0) prefetch_block(f.A, k0 + kLanes * t);
  }
  return k0;
}

template <bool kCheck>
__global__ void __launch_bounds__(kRowThreads) residual_smoothed_kernel(SmoothedArgs a) {
  const int lane = threadIdx.x % kLanes;
  const int i = blockIdx.x * (kRowThreads / kLanes) + threadIdx.x / kLanes;
  const bool active = i < a.fine.R;
  // Before the wait: the row structure and blocks, Sp; r and z_0 are the previous kernel's (the update).
  int jj[4];
  const int k0 = fine_row(a.fine, i, active, lane, jj);
  float sp[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) sp[e] = active && lane == 0 ? a.Sp[e * a.fine.R + i] : 0.0f;
  pdl_wait();
  if (kCheck) {
    if (pcg_stop(a.state, a.rr_partial, a.rr_count)) return;
  } else if (a.state && a.state->done) {
    return;
  }
  float3 acc = make_float3(0.f, 0.f, 0.f);
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    if (jj[t] < 0) continue;
    float m[9];
    load_block(a.fine.A, k0 + kLanes * t, m);
    acc = add3(acc, mul(m, f3(a.z[jj[t]])));
  }
  acc = group_sum(acc);
  float rr = 0.0f;
  if (active && lane == 0) {
    const float3 r = f3(a.r[i]);
    const float3 t = sub3(r, acc);
    a.t[i] = pack(t);
    a.u[i] = pack(mul(sp, t));
    rr = dot3(r, r);
  }
  if (a.rr_init) {  // the first stopping test reads these slots (update_residual_kernel's layout)
    rr = cta_sum(rr);
    if (threadIdx.x == 0) a.rr_init[blockIdx.x] = rr;
  }
}

// Smoothed prolongation of the level-1 correction: v = P e_1 (bilinear), y = z_0 + v - Sp A v.
__global__ void __launch_bounds__(kRowThreads) interp_smoothed_kernel(SmoothedArgs a) {
  const int lane = threadIdx.x % kLanes;
  const int i = blockIdx.x * (kRowThreads / kLanes) + threadIdx.x / kLanes;
  const int n = a.fine.n;
  const bool active = i < a.fine.R;
  // Before the wait: the row structure and blocks, Sp and z_0 (the update's, many kernels back); e_1 is the
  // previous kernel's.
  int jj[4];
  const int k0 = fine_row(a.fine, i, active, lane, jj);
  const bool writer = active && lane == 0;
  float sp[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) sp[e] = writer ? a.Sp[e * a.fine.R + i] : 0.0f;
  const float3 zi = writer ? f3(a.z[i]) : make_float3(0.f, 0.f, 0.f);
  pdl_wait();
  if (a.state && a.state->done) return;
  float3 acc = make_float3(0.f, 0.f, 0.f);
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    if (jj[t] < 0) continue;
    const int j = jj[t];
    float m[9];
    load_block(a.fine.A, k0 + kLanes * t, m);
    acc = add3(acc, mul(m, interpolate(a.e1, a.nc, j % n, j / n)));
  }
  acc = group_sum(acc);
  if (writer) {
    const float3 v = interpolate(a.e1, a.nc, i % n, i / n);
    a.y[i] = pack(sub3(add3(zi, v), mul(sp, acc)));
  }
}

// e_L = A_L^{-1} r_L (dense f32 inverse), one CTA: r staged in shared memory, one warp per output entry.
__global__ void __launch_bounds__(1024) coarse_solve_kernel(MgLevel lv, const float* inv, const MgState* state) {
  const int m3 = 3 * lv.rows;
  for (int l = threadIdx.x; l * 32 < m3 * m3; l += blockDim.x) prefetch_l1(inv + 32 * l);  // static inverse
  pdl_wait();
  if (state && state->done) return;
  __shared__ float rs[3 * kMgCoarsestRowsMax];
  const int m = 3 * lv.rows;
  const float* r = reinterpret_cast<const float*>(lv.r);
  float* e = reinterpret_cast<float*>(lv.e);
  for (int j = threadIdx.x; j < m; j += blockDim.x) rs[j] = r[4 * (j / 3) + j % 3];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  for (int k = warp; k < m; k += warps) {
    float s = 0.0f;
    for (int j = lane; j < m; j += 32) s += inv[k * m + j] * rs[j];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) e[4 * (k / 3) + k % 3] = s;
  }
  for (int k = threadIdx.x; k < lv.rows; k += blockDim.x) e[4 * k + 3] = 0.0f;
}

// The last two levels in one CTA (T = L - 2, n_T <= 9, and the coarsest C): t = r_T - A_T z_T; r_C = P^T t;
// e_C = A_C^{-1} r_C; y = z_T + P e_C; e_T = y + S_T^T (r_T - A_T y). Replaces a restriction, the coarse solve
// and a prolongation (three launches) with one; the vectors stay in shared memory, one warp per row product.
constexpr int kTailRows = 81;  // n_T <= 9
__global__ void __launch_bounds__(1024) tail_kernel(MgLevel T, MgLevel C, const float* inv, const MgState* state) {
  {  // before the wait: the level's stencil, smoother and the coarsest inverse into L1 (static within a solve)
    const int mc = 3 * C.rows, a_lines = (T.rows * T.w * T.w * 48 + 127) / 128, s_lines = (9 * T.rows + 31) / 32;
    for (int l = threadIdx.x; l < a_lines; l += blockDim.x) prefetch_l1(reinterpret_cast<const char*>(T.A) + 128 * l);
    for (int l = threadIdx.x; l < s_lines; l += blockDim.x) prefetch_l1(T.S + 32 * l);
    for (int l = threadIdx.x; l * 32 < mc * mc; l += blockDim.x) prefetch_l1(inv + 32 * l);
  }
  pdl_wait();
  if (state && state->done) return;
  __shared__ float3 t_s[kTailRows], y_s[kTailRows];
  __shared__ float rc_s[3 * kMgCoarsestRowsMax], ec_s[3 * kMgCoarsestRowsMax];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  const int n = T.n, nc = C.n, m = 3 * C.rows;
  const int w2 = T.w * T.w;
  for (int i = warp; i < T.rows; i += warps) {
    float3 acc = make_float3(0.f, 0.f, 0.f);
    int j;
    for (int o = lane; o < w2; o += 32)
      if (stencil_neighbour(n, T.w, i % n, i / n, o, &j)) acc = add3(acc, stencil_apply(T.A, w2, i, o, f3(T.z[j])));
    acc = warp_sum3(acc);
    if (lane == 0) t_s[i] = sub3(f3(T.r[i]), acc);
  }
  __syncthreads();
  for (int I = threadIdx.x; I < C.rows; I += blockDim.x) {
    const int X = I % nc, Y = I / nc;
    float3 r = make_float3(0.f, 0.f, 0.f);
    for (int s = 0; s < 9; ++s) {
      const int ax = s % 3 - 1, by = s / 3 - 1, fx = 2 * X + ax, fy = 2 * Y + by;
      if (fx < 0 || fy < 0 || fx >= n || fy >= n) continue;
      r = add3(r, scale3((ax ? 0.5f : 1.0f) * (by ? 0.5f : 1.0f), t_s[fy * n + fx]));
    }
    rc_s[3 * I] = r.x;
    rc_s[3 * I + 1] = r.y;
    rc_s[3 * I + 2] = r.z;
  }
  __syncthreads();
  for (int k = warp; k < m; k += warps) {
    float s = 0.0f;
    for (int j = lane; j < m; j += 32) s += inv[k * m + j] * rc_s[j];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) ec_s[k] = s;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < T.rows; i += blockDim.x) {
    const int x = i % n, y = i / n, X0 = x >> 1, Y0 = y >> 1;
    const int nx = (x & 1) ? 2 : 1, ny = (y & 1) ? 2 : 1;
    const float w = ((x & 1) ? 0.5f : 1.0f) * ((y & 1) ? 0.5f : 1.0f);
    float3 v = f3(T.z[i]);
    for (int b = 0; b < ny; ++b)
      for (int a = 0; a < nx; ++a) {
        const int J = (Y0 + b) * nc + X0 + a;
        v = add3(v, scale3(w, make_float3(ec_s[3 * J], ec_s[3 * J + 1], ec_s[3 * J + 2])));
      }
    y_s[i] = v;
  }
  __syncthreads();
  for (int i = warp; i < T.rows; i += warps) {
    float3 acc = make_float3(0.f, 0.f, 0.f);
    int j;
    for (int o = lane; o < w2; o += 32)
      if (stencil_neighbour(n, T.w, i % n, i / n, o, &j)) acc = add3(acc, stencil_apply(T.A, w2, i, o, y_s[j]));
    acc = warp_sum3(acc);
    if (lane == 0) T.e[i] = pack(add3(y_s[i], smooth(T.S, T.rows, i, sub3(f3(T.r[i]), acc), true)));
  }
}

// The last three levels (n = 17, 9, 5: every hierarchy of five or more levels ends with them) in ONE launch of an
// 8-CTA thread-block cluster, replacing the restriction 17 -> 9, tail_kernel and the prolongation 9 -> 17. Each
// CTA owns a contiguous slice of the n17 rows (<= 37) and of the n9 rows (<= 11); before the programmatic wait it
// stages its slice of both stencils into shared memory with bulk copies (the stencils are static within a solve)
// and the coarsest inverse and smoother blocks with plain loads, so the cycle's products read shared memory. The
// CTAs exchange the vectors that cross slices (t_17, z_9, t_9, e_9) through distributed shared memory, five
// cluster barriers in all:
//   t_17 = r_17 - A_17 z_17 (own rows)                                   | sync
//   r_9 = P^T t_17, z_9 = S_9 r_9 (own rows)                             | sync
//   t_9 = r_9 - A_9 z_9 (own rows)                                       | sync
//   r_5 = P^T t_9, e_5 = A_5^{-1} r_5 (every CTA, all 25 rows); y_9 = z_9 + P e_5 on the fly;
//   e_9 = y_9 + S_9^T (r_9 - A_9 y_9) (own rows)                         | sync
//   every CTA copies all of e_9                                          | sync
//   y_17 = z_17 + P e_9 on the fly; e_17 = y_17 + S_17^T (r_17 - A_17 y_17) (own rows, to global memory).
// The same operations as restrict_kernel, tail_kernel and prolong_kernel on these levels, summed in another order.
constexpr int kT3Ranks = 8;
constexpr int kT3Threads = 512;
constexpr int kT3N3 = 17, kT3N4 = 9, kT3N5 = 5;
constexpr int kT3Rows3 = kT3N3 * kT3N3, kT3Rows4 = kT3N4 * kT3N4, kT3Rows5 = kT3N5 * kT3N5;
constexpr int kT3Per3 = (kT3Rows3 + kT3Ranks - 1) / kT3Ranks;  // 37 n17 rows per CTA
constexpr int kT3Per4 = (kT3Rows4 + kT3Ranks - 1) / kT3Ranks;  // 11 n9 rows per CTA
constexpr int kT3M5 = 3 * kT3Rows5;                              // 75 unknowns on the coarsest level
constexpr size_t kT3Smem = size_t(kT3Per3 + kT3Per4) * kMgStencil * 3 * sizeof(float4) + kT3M5 * kT3M5 * sizeof(float);
constexpr long long kT3Spin = 2000000000LL;  // ~1 s of SM clock for the staging copies

struct Tail3Args {
  MgLevel L3, L4, L5;   // n = 17, 9, 5
  const float* inv;     // the coarsest inverse, [75][75]
  const MgState* state;
  int* error;           // set to 3 if the staging copies did not land
};

// Block o of row `row` of a stencil slice in shared memory times v.
__device__ __forceinline__ float3 slice_apply(const float4* A, int row, int o, float3 v) {
  const float4* b = A + (row * kMgStencil + o) * 3;
  const float4 u = b[0], w = b[1], t = b[2];
  const float m[9] = {u.x, u.y, u.z, u.w, w.x, w.y, w.z, w.w, t.x};
  return mul(m, v);
}

// (P e)(fine vertex x, y) from a coarse correction stored as 3 floats per row (nc columns).
__device__ __forceinline__ float3 interpolate_flat(const float* e, int nc, int x, int y) {
  const int X0 = x >> 1, Y0 = y >> 1, nx = (x & 1) ? 2 : 1, ny = (y & 1) ? 2 : 1;
  const float w = ((x & 1) ? 0.5f : 1.0f) * ((y & 1) ? 0.5f : 1.0f);
  float3 s = make_float3(0.f, 0.f, 0.f);
  for (int b = 0; b < ny; ++b)
    for (int a = 0; a < nx; ++a) {
      const int J = (Y0 + b) * nc + X0 + a;
      s = add3(s, scale3(w, make_float3(e[3 * J], e[3 * J + 1], e[3 * J + 2])));
    }
  return s;
}

// S^T d for the smoother block of local row k of a shared-memory slice [9][P].
template <int P>
__device__ __forceinline__ float3 smooth_local(const float (&S)[9][P], int k, float3 d) {
  return make_float3(S[0][k] * d.x + S[3][k] * d.y + S[6][k] * d.z, S[1][k] * d.x + S[4][k] * d.y + S[7][k] * d.z,
                     S[2][k] * d.x + S[5][k] * d.y + S[8][k] * d.z);
}

__global__ void __cluster_dims__(kT3Ranks, 1, 1) __launch_bounds__(kT3Threads) tail3_kernel(Tail3Args a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = int(cluster.block_rank());
  extern __shared__ __align__(16) unsigned char t3_smem[];
  float4* A3s = reinterpret_cast<float4*>(t3_smem);       // [kT3Per3][25][3]
  float4* A4s = A3s + kT3Per3 * kMgStencil * 3;            // [kT3Per4][25][3]
  float* invs = reinterpret_cast<float*>(A4s + kT3Per4 * kMgStencil * 3);  // [75][75]
  __shared__ float S3s[9][kT3Per3], S4s[9][kT3Per4];
  __shared__ float4 t3s[kT3Per3], r4s[kT3Per4], z4s[kT3Per4], t4s[kT3Per4], e4s[kT3Per4];
  __shared__ float4 t4_all[kT3Rows4], e4_all[kT3Rows4];
  __shared__ float r5s[kT3M5], e5s[kT3M5];
  __shared__ __align__(8) unsigned long long stage_bar;
  const int i0 = rank * kT3Per3, n3 = min(kT3Rows3, i0 + kT3Per3) - i0;
  const int I0 = rank * kT3Per4, n4 = max(0, min(kT3Rows4, I0 + kT3Per4) - I0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = kT3Threads / 32;
  // Before the wait: the static operands (stencil slices by bulk copy, the inverse and the smoother blocks).
  const unsigned bar = smem_addr(&stage_bar);
  const unsigned bytes3 = unsigned(n3) * kMgStencil * 3 * 16u, bytes4 = unsigned(n4) * kMgStencil * 3 * 16u;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_proxy_async_shared();
    mbar_arrive_expect_tx(bar, bytes3 + bytes4);
    bulk_copy_g2s(smem_addr(A3s), a.L3.A + size_t(i0) * kMgStencil * 3, bytes3, bar);
    if (n4 > 0) bulk_copy_g2s(smem_addr(A4s), a.L4.A + size_t(I0) * kMgStencil * 3, bytes4, bar);
  }
  for (int t = threadIdx.x; t < kT3M5 * kT3M5; t += kT3Threads) invs[t] = a.inv[t];
  for (int t = threadIdx.x; t < 9 * kT3Per3; t += kT3Threads) {
    const int e = t / kT3Per3, k = t % kT3Per3;
    S3s[e][k] = k < n3 ? a.L3.S[e * kT3Rows3 + i0 + k] : 0.0f;
  }
  for (int t = threadIdx.x; t < 9 * kT3Per4; t += kT3Threads) {
    const int e = t / kT3Per4, k = t % kT3Per4;
    S4s[e][k] = k < n4 ? a.L4.S[e * kT3Rows4 + I0 + k] : 0.0f;
  }
  __syncthreads();  // the barrier's initialisation before any thread waits on it
  pdl_wait();
  // The copies write this CTA's shared memory: wait for them before anything else, a return included.
  const bool landed = __syncthreads_and(mbar_wait_parity(bar, 0, kT3Spin));
  if (!landed) {
    if (threadIdx.x == 0) atomicExch(a.error, 3);
    mbar_wait_parity(bar, 0, kT3Spin);
  }
  if (a.state && a.state->done) return;  // the same word in every CTA: all leave before the first cluster barrier

  // t_17 = r_17 - A_17 z_17 on the own rows: 8 lanes per row, 64 rows per pass (every lane reaches the shuffles)
  {
    const int g = threadIdx.x & (kLanes - 1), k = threadIdx.x / kLanes;
    const bool active = k < n3;
    const int i = i0 + k, X = i % kT3N3, Y = i / kT3N3;
    float3 acc = make_float3(0.f, 0.f, 0.f);
    if (active)
      for (int o = g; o < kMgStencil; o += kLanes) {
        int j;
        if (stencil_neighbour(kT3N3, 5, X, Y, o, &j)) acc = add3(acc, slice_apply(A3s, k, o, f3(a.L3.z[j])));
      }
    acc = group_sum(acc);
    if (active && g == 0) t3s[k] = pack(sub3(f3(a.L3.r[i]), acc));
  }
  cluster.sync();
  // r_9 = P^T t_17, z_9 = S_9 r_9 on the own n9 rows: one warp per row, lanes 0..8 the support rows
  if (warp < n4) {
    const int I = I0 + warp, X = I % kT3N4, Y = I / kT3N4;
    float3 t = make_float3(0.f, 0.f, 0.f);
    if (lane < 9) {
      const int ax = lane % 3 - 1, by = lane / 3 - 1, fx = 2 * X + ax, fy = 2 * Y + by;
      if (fx >= 0 && fy >= 0 && fx < kT3N3 && fy < kT3N3) {
        const int j = fy * kT3N3 + fx;
        const float4* src = cluster.map_shared_rank(t3s, j / kT3Per3);
        t = scale3((ax ? 0.5f : 1.0f) * (by ? 0.5f : 1.0f), f3(src[j % kT3Per3]));
      }
    }
    t = warp_sum3(t);
    if (lane == 0) {
      float sm[9];
#pragma unroll
      for (int e = 0; e < 9; ++e) sm[e] = S4s[e][warp];
      r4s[warp] = pack(t);
      z4s[warp] = pack(mul(sm, t));
    }
  }
  cluster.sync();
  // t_9 = r_9 - A_9 z_9 on the own n9 rows: one warp per row, lane o < 25 the stencil offset
  if (warp < n4) {
    const int I = I0 + warp, X = I % kT3N4, Y = I / kT3N4;
    float3 acc = make_float3(0.f, 0.f, 0.f);
    int J;
    if (lane < kMgStencil && stencil_neighbour(kT3N4, 5, X, Y, lane, &J)) {
      const float4* zr = cluster.map_shared_rank(z4s, J / kT3Per4);
      acc = slice_apply(A4s, warp, lane, f3(zr[J % kT3Per4]));
    }
    acc = warp_sum3(acc);
    if (lane == 0) t4s[warp] = pack(sub3(f3(r4s[warp]), acc));
  }
  cluster.sync();
  // every CTA: all of t_9, r_5 = P^T t_9, e_5 = A_5^{-1} r_5
  for (int J = threadIdx.x; J < kT3Rows4; J += kT3Threads) t4_all[J] = cluster.map_shared_rank(t4s, J / kT3Per4)[J % kT3Per4];
  __syncthreads();
  for (int K = warp; K < kT3Rows5; K += warps) {
    const int X = K % kT3N5, Y = K / kT3N5;
    float3 r = make_float3(0.f, 0.f, 0.f);
    if (lane < 9) {
      const int ax = lane % 3 - 1, by = lane / 3 - 1, fx = 2 * X + ax, fy = 2 * Y + by;
      if (fx >= 0 && fy >= 0 && fx < kT3N4 && fy < kT3N4)
        r = scale3((ax ? 0.5f : 1.0f) * (by ? 0.5f : 1.0f), f3(t4_all[fy * kT3N4 + fx]));
    }
    r = warp_sum3(r);
    if (lane == 0) {
      r5s[3 * K] = r.x;
      r5s[3 * K + 1] = r.y;
      r5s[3 * K + 2] = r.z;
    }
  }
  __syncthreads();
  for (int k = warp; k < kT3M5; k += warps) {
    float v = 0.0f;
    for (int j = lane; j < kT3M5; j += 32) v += invs[k * kT3M5 + j] * r5s[j];
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) e5s[k] = v;
  }
  __syncthreads();
  // e_9 = y_9 + S_9^T (r_9 - A_9 y_9), y_9 = z_9 + P e_5 formed at each neighbour
  if (warp < n4) {
    const int I = I0 + warp, X = I % kT3N4, Y = I / kT3N4;
    float3 acc = make_float3(0.f, 0.f, 0.f);
    int J;
    if (lane < kMgStencil && stencil_neighbour(kT3N4, 5, X, Y, lane, &J)) {
      const float4* zr = cluster.map_shared_rank(z4s, J / kT3Per4);
      const float3 y = add3(f3(zr[J % kT3Per4]), interpolate_flat(e5s, kT3N5, J % kT3N4, J / kT3N4));
      acc = slice_apply(A4s, warp, lane, y);
    }
    acc = warp_sum3(acc);
    if (lane == 0) {
      const float3 y = add3(f3(z4s[warp]), interpolate_flat(e5s, kT3N5, X, Y));
      e4s[warp] = pack(add3(y, smooth_local(S4s, warp, sub3(f3(r4s[warp]), acc))));
    }
  }
  cluster.sync();
  for (int J = threadIdx.x; J < kT3Rows4; J += kT3Threads) e4_all[J] = cluster.map_shared_rank(e4s, J / kT3Per4)[J % kT3Per4];
  cluster.sync();  // no CTA leaves while another still reads its shared memory
  // e_17 = y_17 + S_17^T (r_17 - A_17 y_17), y_17 = z_17 + P e_9 formed at each neighbour
  {
    const int g = threadIdx.x & (kLanes - 1), k = threadIdx.x / kLanes;
    const bool active = k < n3;
    const int i = i0 + k, X = i % kT3N3, Y = i / kT3N3;
    float3 acc = make_float3(0.f, 0.f, 0.f);
    if (active)
      for (int o = g; o < kMgStencil; o += kLanes) {
        int j;
        if (stencil_neighbour(kT3N3, 5, X, Y, o, &j)) {
          const float3 y = add3(f3(a.L3.z[j]), interpolate(e4_all, kT3N4, j % kT3N3, j / kT3N3));
          acc = add3(acc, slice_apply(A3s, k, o, y));
        }
      }
    acc = group_sum(acc);
    if (active && g == 0) {
      const float3 y = add3(f3(a.L3.z[i]), interpolate(e4_all, kT3N4, X, Y));
      a.L3.e[i] = pack(add3(y, smooth_local(S3s, k, sub3(f3(a.L3.r[i]), acc))));
    }
  }
}

struct ProlongArgs {
  MgFine fine;       // level-0 operator (kFine)
  MgLevel lv;        // level l: r, z (pre-smoothed), S, A; writes e
  MgLevel coarse;    // level l + 1: e
  const float4* y;   // kY: z_0 + P_0 e_1 at every fine row
  const MgState* state;
  // level 0 only: partial dots of the new z with the current and previous residuals
  const float4* r_prev;
  float* zr_partial;
  float* zrp_partial;
};

// y = z_l + P e_{l+1};  e_l = y + S^T (r_l - A_l y), y at the neighbours interpolated on the fly. kW: 0 for the
// fine level (BSR), else the level's stencil width. kY (fine level under the smoothed prolongation): y was formed
// by interp_smoothed_kernel and is read from a.y.
template <int kW, bool kY>
__global__ void __launch_bounds__(kRowThreads) prolong_kernel(ProlongArgs a) {
  constexpr bool kFine = kW == 0;
  constexpr int kW2 = kW * kW;
  constexpr int kPer = kFine ? 4 : (kW2 + kLanes - 1) / kLanes;  // <= 25 blocks per fine row: <= 4 per lane
  const int lane = threadIdx.x % kLanes;
  const int i = blockIdx.x * (kRowThreads / kLanes) + threadIdx.x / kLanes;
  const int n = a.lv.n, nc = a.coarse.n;
  const bool active = i < a.lv.rows;
  // Before the wait: the row structure and blocks, and this level's r and z (written by its restriction, or on the
  // fine level by the update, two or more kernels back), S and r_prev. The coarse correction e (the previous
  // kernel's) and y (kY: the previous kernel's) are read after it.
  int jj[kPer];
  int k0 = 0;
  if (kFine) {
    int k1 = 0;
    if (active) {
      k0 = a.fine.row_ptr[i] + lane;
      k1 = a.fine.row_ptr[i + 1];
    }
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      jj[t] = active && k0 + kLanes * t < k1 ? a.fine.col_idx[k0 + kLanes * t] : -1;
      if (jj[t] >= 0) prefetch_block(a.fine.A, k0 + kLanes * t);
    }
  } else {
    const int X = i % n, Y = i / n;
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const int o = lane + kLanes * t;
      int j = -1;
      jj[t] = active && o < kW2 && stencil_neighbour(n, kW, X, Y, o, &j) ? j : -1;
      if (jj[t] >= 0) prefetch_stencil(a.lv.A, kW2, i, o);
    }
  }
  float3 zj[kPer];
#pragma unroll
  for (int t = 0; t < kPer; ++t) zj[t] = !kY && jj[t] >= 0 ? f3(a.lv.z[jj[t]]) : make_float3(0.f, 0.f, 0.f);
  const bool writer = active && lane == 0;
  const bool dots = kFine && a.zr_partial;  // inside flexible PCG only (a stand-alone cycle has no r_prev)
  float sm[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) sm[e] = writer ? a.lv.S[e * a.lv.rows + i] : 0.0f;
  const float3 r = writer ? f3(a.lv.r[i]) : make_float3(0.f, 0.f, 0.f);
  const float3 zi = writer && !kY ? f3(a.lv.z[i]) : make_float3(0.f, 0.f, 0.f);
  const float3 rp = writer && dots ? f3(a.r_prev[i]) : make_float3(0.f, 0.f, 0.f);
  pdl_wait();
  if (a.state && a.state->done) return;
  float3 acc = make_float3(0.f, 0.f, 0.f);
#pragma unroll
  for (int t = 0; t < kPer; ++t) {
    const int j = jj[t];
    if (j < 0) continue;
    const float3 y = kY ? f3(a.y[j]) : add3(zj[t], interpolate(a.coarse.e, nc, j % n, j / n));
    if (kFine) {
      float m[9];
      load_block(a.fine.A, k0 + kLanes * t, m);
      acc = add3(acc, mul(m, y));
    } else {
      acc = add3(acc, stencil_apply(a.lv.A, kW2, i, lane + kLanes * t, y));
    }
  }
  acc = group_sum(acc);
  float zr = 0.0f, zrp = 0.0f;
  if (writer) {
    const float3 y = kY ? f3(a.y[i]) : add3(zi, interpolate(a.coarse.e, nc, i % n, i / n));
    const float3 d = sub3(r, acc);
    // e = y + S^T (r - A y)
    const float3 e = add3(y, make_float3(sm[0] * d.x + sm[3] * d.y + sm[6] * d.z, sm[1] * d.x + sm[4] * d.y + sm[7] * d.z,
                                         sm[2] * d.x + sm[5] * d.y + sm[8] * d.z));
    a.lv.e[i] = pack(e);
    if (dots) {
      zr = dot3(e, r);
      zrp = dot3(e, rp);
    }
  }
  if (dots) {
    zr = cta_sum(zr);
    zrp = cta_sum(zrp);
    if (threadIdx.x == 0) {
      a.zr_partial[blockIdx.x] = zr;
      a.zrp_partial[blockIdx.x] = zrp;
    }
  }
}

struct DirectionArgs {
  MgFine fine;
  const float4* z;      // preconditioned residual (level-0 e)
  const float4* p_old;
  float4* p_new;
  float4* q;
  MgState* state;
  const float* zr_partial;
  const float* zrp_partial;
  int zr_count;
  float* pq_partial;
  cudaGraphConditionalHandle cond;  // the solve graph's WHILE condition (fused update: this kernel ends the body)
  int set_cond;                     // clear the condition once the solve is done
};

// beta (Polak-Ribiere form of flexible CG) = z.(r - r_prev) / rz_old;  p = z + beta p_old;  q = A p.
__global__ void __launch_bounds__(kRowThreads) direction_kernel(DirectionArgs a) {
  MgState* st = a.state;
  const int lane = threadIdx.x % kLanes;
  const int i = blockIdx.x * (kRowThreads / kLanes) + threadIdx.x / kLanes;
  const bool active = i < a.fine.R;
  // Before the wait: the row structure and blocks, the previous direction p_old (this kernel's own output one
  // iteration back) and the update's scalars; z and the partial dot products are the previous kernel's.
  int jj[4];
  int k0 = 0, k1 = 0;
  if (active) {
    k0 = a.fine.row_ptr[i] + lane;
    k1 = a.fine.row_ptr[i + 1];
  }
  float3 po[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    jj[t] = active && k0 + kLanes * t < k1 ? a.fine.col_idx[k0 + kLanes * t] : -1;
    if (jj[t] >= 0) prefetch_block(a.fine.A, k0 + kLanes * t);
    po[t] = jj[t] >= 0 ? f3(a.p_old[jj[t]]) : make_float3(0.f, 0.f, 0.f);
  }
  const float3 po_i = active && lane == 0 ? f3(a.p_old[i]) : make_float3(0.f, 0.f, 0.f);
  const int iterations = st->iterations;
  const float rz_old = st->rz_old;
  pdl_wait();
  if (st->done) {
    if (a.set_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0);
    return;
  }
  const float zr = sum_partials(a.zr_partial, a.zr_count);
  const float zrp = sum_partials(a.zrp_partial, a.zr_count);
  const bool first = iterations == 0;
  const float beta = first ? 0.0f : (zr - zrp) / rz_old;
  float3 acc = make_float3(0.f, 0.f, 0.f);
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    if (jj[t] < 0) continue;
    const float3 z = f3(a.z[jj[t]]);
    const float3 p = first ? z : add3(z, scale3(beta, po[t]));
    float m[9];
    load_block(a.fine.A, k0 + kLanes * t, m);
    acc = add3(acc, mul(m, p));
  }
  acc = group_sum(acc);
  float pq = 0.0f;
  if (active && lane == 0) {
    const float3 z = f3(a.z[i]);
    const float3 p = first ? z : add3(z, scale3(beta, po_i));
    a.p_new[i] = pack(p);
    a.q[i] = pack(acc);
    pq = dot3(p, acc);
  }
  pq = cta_sum(pq);
  if (threadIdx.x == 0) a.pq_partial[blockIdx.x] = pq;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->zr = zr;
    st->beta = beta;
    st->has_direction = 1;  // update_restrict_kernel applies it
  }
}

struct UpdateArgs {
  int R;
  const float4* p;
  const float4* q;
  const float4* r_cur;
  float4* r_next;
  float4* x;
  const float* S0;       // level-0 smoother
  float4* z_pre;         // next pre-smoothing S0 r
  MgState* state;
  const float* pq_partial;
  int pq_count;
  float* rr_partial;
  cudaGraphConditionalHandle cond;  // the solve graph's WHILE condition
  int set_cond;                     // this launch ends the graph body: clear the condition once done
};

// alpha = z.r / p.q;  x += alpha p;  r_next = r - alpha q;  z_pre = S0 r_next.
__global__ void __launch_bounds__(kUpdateThreads) update_kernel(UpdateArgs a) {
  MgState* st = a.state;
  const int i = blockIdx.x * kUpdateThreads + threadIdx.x;
  const bool active = i < a.R;
  // Before the wait: x, the current residual (the previous iteration's update wrote them) and the fine smoother;
  // p, q, z.r and the partial p.q are the previous kernel's.
  const float3 x = active ? f3(a.x[i]) : make_float3(0.f, 0.f, 0.f);
  const float3 rc = active ? f3(a.r_cur[i]) : make_float3(0.f, 0.f, 0.f);
  float sm[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) sm[e] = active ? a.S0[e * a.R + i] : 0.0f;
  pdl_wait();
  if (st->done) {
    if (a.set_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0);
    return;
  }
  const float pq = sum_partials(a.pq_partial, a.pq_count);
  const float zr = st->zr;
  const float alpha = zr / pq;
  if (!(pq > 0.0f) || !isfinite(alpha)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->pq = pq;
      st->status = kStatusBreakdown;
      st->done = 1;
      if (a.set_cond) cudaGraphSetConditional(a.cond, 0);
    }
    return;
  }
  float rr = 0.0f;
  if (active) {
    const float3 p = f3(a.p[i]);
    a.x[i] = pack(add3(x, scale3(alpha, p)));
    const float3 r = sub3(rc, scale3(alpha, f3(a.q[i])));
    a.r_next[i] = pack(r);
    a.z_pre[i] = pack(mul(sm, r));
    rr = dot3(r, r);
  }
  rr = cta_sum(rr);
  if (threadIdx.x == 0) a.rr_partial[blockIdx.x] = rr;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->pq = pq;
    st->alpha = alpha;
    st->rz_old = zr;
    st->iterations = st->iterations + 1;
  }
}

// The update fused with the smoothed path's fine residual (one kernel instead of two): alpha = z.r / p.q;
// x += alpha p; r' = r - alpha q; z_0 = S0 r'; t = r' - A z_0; u = Sp t. r' and z_0 at the row's neighbours are
// recomputed from r, q and S0 (local once alpha is known), so no CTA waits for another's update; the partial
// |r'|^2 goes to the rows' CTA slot (row_grid(R) slots) for the next iteration's stopping test (restrict_kernel
// <0, true> on t and u).
__global__ void __launch_bounds__(kRowThreads) update_residual_kernel(UpdateArgs a, SmoothedArgs s) {
  MgState* st = a.state;
  const int lane = threadIdx.x % kLanes;
  const int i = blockIdx.x * (kRowThreads / kLanes) + threadIdx.x / kLanes;
  const bool active = i < a.R;
  // Before the wait: the row structure and blocks, r and S0 at the neighbours and the row, x and Sp at the row
  // (all written one iteration back or static); p, q and the partial p.q are the previous kernel's.
  int jj[4];
  const int k0 = fine_row(s.fine, i, active, lane, jj);
  float3 rj[4];
  float sj[4][9];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    rj[t] = jj[t] >= 0 ? f3(a.r_cur[jj[t]]) : make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int e = 0; e < 9; ++e) sj[t][e] = jj[t] >= 0 ? a.S0[e * a.R + jj[t]] : 0.0f;
  }
  const bool writer = active && lane == 0;
  float si[9], spi[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) {
    si[e] = writer ? a.S0[e * a.R + i] : 0.0f;
    spi[e] = writer ? s.Sp[e * a.R + i] : 0.0f;
  }
  const float3 xi = writer ? f3(a.x[i]) : make_float3(0.f, 0.f, 0.f);
  const float3 ri = writer ? f3(a.r_cur[i]) : make_float3(0.f, 0.f, 0.f);
  pdl_wait();
  if (st->done) {
    if (a.set_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0);
    return;
  }
  const float pq = sum_partials(a.pq_partial, a.pq_count);
  const float zr = st->zr;
  const float alpha = zr / pq;
  if (!(pq > 0.0f) || !isfinite(alpha)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->pq = pq;
      st->status = kStatusBreakdown;
      st->done = 1;
      if (a.set_cond) cudaGraphSetConditional(a.cond, 0);
    }
    return;
  }
  float3 acc = make_float3(0.f, 0.f, 0.f);
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    if (jj[t] < 0) continue;
    const float3 rn = sub3(rj[t], scale3(alpha, f3(a.q[jj[t]])));
    float m[9];
    load_block(s.fine.A, k0 + kLanes * t, m);
    acc = add3(acc, mul(m, mul(sj[t], rn)));
  }
  acc = group_sum(acc);
  float rr = 0.0f;
  if (writer) {
    a.x[i] = pack(add3(xi, scale3(alpha, f3(a.p[i]))));
    const float3 rn = sub3(ri, scale3(alpha, f3(a.q[i])));
    a.r_next[i] = pack(rn);
    a.z_pre[i] = pack(mul(si, rn));
    const float3 t = sub3(rn, acc);
    s.t[i] = pack(t);
    s.u[i] = pack(mul(spi, t));
    rr = dot3(rn, rn);
  }
  rr = cta_sum(rr);
  if (threadIdx.x == 0) a.rr_partial[blockIdx.x] = rr;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->pq = pq;
    st->alpha = alpha;
    st->rz_old = zr;
    st->iterations = st->iterations + 1;
  }
}

// The update fused with the first restriction (bilinear prolongation, three or more restricted levels): at the start
// of iteration k it applies iteration k-1's update and then restricts, one warp per coarse row I as restrict_kernel.
// The warp stages the 7 x 7 fine window around 2I (the nine support rows and their columns): r' = r - alpha q (no
// update at k = 0) and z_0 = S0 r' at every window vertex, recomputed by each coarse row that needs them (local
// once alpha is known), so no CTA waits for another's update. The coarse row owns the fine rows 2I + (0|1, 0|1):
// it writes their r', z_0 and x += alpha p and their |r'|^2 partial, which the next kernel (restrict_kernel<5,
// true>) turns into the stopping test. Buffers: u.r_cur the residual of iteration k-1 (r at k = 0), u.r_next the
// residual of iteration k, u.p the direction of iteration k-1 (at k = 0 the start leaves b in both residual buffers).
__global__ void __launch_bounds__(kRestrictThreads) update_restrict_kernel(UpdateArgs u, RestrictArgs a) {
  __shared__ float3 rn_s[kRestrictRows][49], z0_s[kRestrictRows][49];
  MgState* st = u.state;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int I = blockIdx.x * kRestrictRows + warp;
  const bool row_ok = I < a.dst.rows;
  const int nc = a.dst.n, nf = a.src.n;
  const int X = I % nc, Y = I / nc, cx = 2 * X, cy = 2 * Y;
  const int s = lane / 3, k3 = lane % 3, ax = s % 3 - 1, by = s / 3 - 1;
  const int fx = cx + ax, fy = cy + by;
  const bool has_row = row_ok && lane < 27 && fx >= 0 && fy >= 0 && fx < nf && fy < nf;
  const int i = has_row ? fy * nf + fx : 0;
  const int it = st->iterations;  // updates so far (the previous fused kernel's, many kernels back)
  // Before the wait: the support rows' structure and blocks, the window's r and S0, the owned rows' x, the coarse
  // smoother; q, p and the partial p.q are the previous kernel's (the direction).
  int jj[9];
  int k0 = 0, k1 = 0;
  if (has_row) {
    k0 = a.fine.row_ptr[i] + k3;
    k1 = a.fine.row_ptr[i + 1];
  }
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    jj[t] = has_row && k0 + 3 * t < k1 ? a.fine.col_idx[k0 + 3 * t] : -1;
    if (jj[t] >= 0) prefetch_block(a.fine.A, k0 + 3 * t);
  }
  int wv[2];
  float3 rc[2], xo[2];
  float sm0[2][9];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int w = lane + 32 * q, vx = cx + w % 7 - 3, vy = cy + w / 7 - 3;
    wv[q] = row_ok && w < 49 && vx >= 0 && vy >= 0 && vx < nf && vy < nf ? vy * nf + vx : -1;
    rc[q] = wv[q] >= 0 ? f3(u.r_cur[wv[q]]) : make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int e = 0; e < 9; ++e) sm0[q][e] = wv[q] >= 0 ? u.S0[e * u.R + wv[q]] : 0.0f;
    const bool owned = wv[q] >= 0 && (w % 7 == 3 || w % 7 == 4) && (w / 7 == 3 || w / 7 == 4);
    xo[q] = owned ? f3(u.x[wv[q]]) : make_float3(0.f, 0.f, 0.f);
  }
  float smd[9];
  const bool writer = lane == 0 && row_ok && !a.coarsest;
#pragma unroll
  for (int e = 0; e < 9; ++e) smd[e] = writer ? a.dst.S[e * a.dst.rows + I] : 0.0f;
  pdl_wait();
  if (st->done) return;
  // a direction exists once the first iteration's direction kernel has run
  const bool update = st->has_direction != 0;
  float alpha = 0.0f, pq = 0.0f, zr = 0.0f;
  if (update) {
    pq = sum_partials(u.pq_partial, u.pq_count);
    zr = st->zr;
    alpha = zr / pq;
    if (!(pq > 0.0f) || !isfinite(alpha)) {
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->pq = pq;
        st->status = kStatusBreakdown;
        st->done = 1;
      }
      return;
    }
  }
  float rr = 0.0f;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int w = lane + 32 * q;
    if (wv[q] < 0) continue;
    const float3 rn = update ? sub3(rc[q], scale3(alpha, f3(u.q[wv[q]]))) : rc[q];
    const float3 z0 = mul(sm0[q], rn);
    rn_s[warp][w] = rn;
    z0_s[warp][w] = z0;
    if ((w % 7 == 3 || w % 7 == 4) && (w / 7 == 3 || w / 7 == 4)) {  // an owned fine row
      if (update) {
        u.r_next[wv[q]] = pack(rn);
        u.x[wv[q]] = pack(add3(xo[q], scale3(alpha, f3(u.p[wv[q]]))));
      }
      u.z_pre[wv[q]] = pack(z0);
      rr += dot3(rn, rn);
    }
  }
  __syncwarp();
  float3 t = make_float3(0.f, 0.f, 0.f);
  if (has_row) {
    float3 acc = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const int j = jj[q];
      if (j < 0) continue;
      const int w = (j / nf - cy + 3) * 7 + (j % nf - cx + 3);
      float m[9];
      load_block(a.fine.A, k0 + 3 * q, m);
      acc = add3(acc, mul(m, z0_s[warp][w]));
    }
    const float wgt = (ax ? 0.5f : 1.0f) * (by ? 0.5f : 1.0f);
    t = scale3(wgt, k3 == 0 ? sub3(rn_s[warp][(by + 3) * 7 + ax + 3], acc) : scale3(-1.0f, acc));
  }
  t = warp_sum3(t);
  if (lane == 0 && row_ok) {
    a.dst.r[I] = pack(t);
    if (!a.coarsest) a.dst.z[I] = pack(mul(smd, t));
  }
  rr = cta_sum(rr);
  if (threadIdx.x == 0) u.rr_partial[blockIdx.x] = rr;
  if (update && blockIdx.x == 0 && threadIdx.x == 0) {
    st->pq = pq;
    st->alpha = alpha;
    st->rz_old = zr;
    st->iterations = it + 1;
  }
}

struct InitArgs {
  int R;
  const float4* b;
  float4* x;
  float4* r0;
  float4* r1;
  float4* p0;
  float4* p1;
  const float* S0;
  float4* z_pre;
  float* rr_partial;
  MgState* state;
  float tol2;
  int max_iterations;
  int stall_window;
};

__global__ void __launch_bounds__(kUpdateThreads) init_kernel(InitArgs a) {
  const int i = blockIdx.x * kUpdateThreads + threadIdx.x;
  float rr = 0.0f;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  if (i < a.R) {
    const float3 b = f3(a.b[i]);
    a.x[i] = zero;
    a.r0[i] = pack(b);
    a.r1[i] = pack(b);  // the fused update-restriction reads the previous residual from here at the start
    a.p0[i] = zero;
    a.p1[i] = zero;
    a.z_pre[i] = pack(smooth(a.S0, a.R, i, b, false));
    rr = dot3(b, b);
  }
  rr = cta_sum(rr);
  if (threadIdx.x == 0) a.rr_partial[blockIdx.x] = rr;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    MgState s{};
    s.tol2 = a.tol2;
    s.max_iterations = a.max_iterations;
    s.stall_window = a.stall_window;
    *a.state = s;
  }
}

// z_pre = S0 r (the pre-smoothing of a stand-alone V-cycle).
__global__ void presmooth_kernel(int R, const float* S0, const float4* r, float4* z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < R) z[i] = pack(smooth(S0, R, i, f3(r[i]), false));
}

MgLevel level0(const MgDevice& d, int parity) {
  MgLevel l = d.lv[0];
  l.r = d.r[parity];
  return l;
}

// The V-cycle on level-0 right-hand side r[parity] with z_pre already in lv[0].z; result in lv[0].e.
// Inside flexible PCG with the bilinear prolongation and at least two restricted levels, `fused` (non-null) carries
// the update of the previous iteration, which update_restrict_kernel applies with the first restriction; the
// stopping test then moves to the second restriction.
// tail3_kernel applies when the hierarchy ends with the 5 x 5-stencil levels n = 17, 9, 5 below at least two more
// levels (the restriction 1 -> 2, which holds the flexible PCG's stopping test, stays a kernel of its own).
bool use_tail3(const MgDevice& d) {
  const int L = d.levels;
  return L >= 5 && d.lv[L - 3].n == kT3N3 && d.lv[L - 2].n == kT3N4 && d.lv[L - 1].n == kT3N5 &&
         d.lv[L - 3].w == 5 && d.lv[L - 2].w == 5;
}

cudaError_t launch_cycle(const MgDevice& d, int parity, bool in_pcg, bool pdl, cudaStream_t s, int* launches,
                         const UpdateArgs* fused = nullptr) {
  const int L = d.levels;
  MgState* st = in_pcg ? d.state : nullptr;
  const bool smoothed = d.smoothed != 0;
  SmoothedArgs sa{};
  sa.fine = d.fine;
  sa.r = d.r[parity];
  sa.z = d.lv[0].z;
  sa.Sp = d.Sp;
  sa.t = d.t;
  sa.u = d.u;
  sa.e1 = d.lv[1].e;
  sa.nc = d.lv[1].n;
  sa.y = d.y;
  sa.state = st;
  sa.rr_partial = d.partial + kPartRr * kMgPartials;
  sa.rr_count = update_grid(d.fine.R);
  cudaError_t e;
  // t = r - A z_0, u = Sp t: inside flexible PCG the previous iteration's update_residual_kernel (or the start,
  // mg_pcg_init) formed them; a stand-alone V-cycle forms them here.
  if (smoothed && !in_pcg) {
    if ((e = launch(residual_smoothed_kernel<false>, row_grid(d.fine.R), kRowThreads, s, pdl, sa)) != cudaSuccess)
      return e;
    ++*launches;
  }
  // with five or more levels the last three (n = 17, 9, 5) run in one 8-CTA cluster (tail3_kernel); otherwise, with
  // three or more, the last two run in one CTA (tail_kernel: level L - 2 is a stencil level, n <= 9)
  const bool tail3 = use_tail3(d);
  const bool tail = !tail3 && L >= 3;
  const int last_restricted = tail3 ? L - 3 : tail ? L - 2 : L - 1;
  for (int l = 0; l < last_restricted; ++l) {
    RestrictArgs a{};
    a.fine = d.fine;
    a.src = l == 0 ? level0(d, parity) : d.lv[l];
    if (l == 0 && smoothed) {
      a.src.r = d.t;
      a.src.z = d.u;
    }
    a.dst = d.lv[l + 1];
    a.coarsest = l + 2 == L;
    a.state = st;
    a.rr_partial = d.partial + kPartRr * kMgPartials;
    // the update's CTA count (the fused update-restriction writes one slot per CTA of the first restriction)
    a.rr_count = fused ? restrict_grid(d.lv[1].rows) : smoothed ? row_grid(d.fine.R) : update_grid(d.fine.R);
    const int grid = restrict_grid(a.dst.rows);
    if (l == 0 && fused) e = launch(update_restrict_kernel, grid, kRestrictThreads, s, pdl, *fused, a);
    else if (l == 1 && fused) e = launch(restrict_kernel<5, true>, grid, kRestrictThreads, s, pdl, a);
    else if (l == 0 && in_pcg) e = launch(restrict_kernel<0, true>, grid, kRestrictThreads, s, pdl, a);
    else if (l == 0) e = launch(restrict_kernel<0, false>, grid, kRestrictThreads, s, pdl, a);
    else if (a.src.w == 7) e = launch(restrict_kernel<7, false>, grid, kRestrictThreads, s, pdl, a);
    else e = launch(restrict_kernel<5, false>, grid, kRestrictThreads, s, pdl, a);
    if (e != cudaSuccess) return e;
    ++*launches;
  }
  if (tail3) {
    Tail3Args ta{};
    ta.L3 = d.lv[L - 3];
    ta.L4 = d.lv[L - 2];
    ta.L5 = d.lv[L - 1];
    ta.inv = d.coarse_inv;
    ta.state = st;
    ta.error = d.error;
    e = launch_smem(tail3_kernel, kT3Ranks, kT3Threads, kT3Smem, s, pdl, ta);
  } else {
    e = tail ? launch(tail_kernel, 1, 1024, s, pdl, d.lv[L - 2], d.lv[L - 1], (const float*)d.coarse_inv,
                      (const MgState*)st)
             : launch(coarse_solve_kernel, 1, 1024, s, pdl, d.lv[L - 1], (const float*)d.coarse_inv,
                      (const MgState*)st);
  }
  if (e != cudaSuccess) return e;
  ++*launches;
  for (int l = last_restricted - 1; l >= 0; --l) {
    ProlongArgs a{};
    a.fine = d.fine;
    a.lv = l == 0 ? level0(d, parity) : d.lv[l];
    a.coarse = d.lv[l + 1];
    a.y = d.y;
    a.state = st;
    if (l == 0 && in_pcg) {
      a.r_prev = d.r[1 - parity];
      a.zr_partial = d.partial + kPartZr * kMgPartials;
      a.zrp_partial = d.partial + kPartZrPrev * kMgPartials;
    }
    const int grid = row_grid(a.lv.rows);
    if (l == 0 && smoothed) {  // y = z_0 + P_0 e_1, then the post-smoothing on y
      if ((e = launch(interp_smoothed_kernel, grid, kRowThreads, s, pdl, sa)) != cudaSuccess) return e;
      ++*launches;
      e = launch(prolong_kernel<0, true>, grid, kRowThreads, s, pdl, a);
    } else if (l == 0) {
      e = launch(prolong_kernel<0, false>, grid, kRowThreads, s, pdl, a);
    } else if (a.lv.w == 7) {
      e = launch(prolong_kernel<7, false>, grid, kRowThreads, s, pdl, a);
    } else {
      e = launch(prolong_kernel<5, false>, grid, kRowThreads, s, pdl, a);
    }
    if (e != cudaSuccess) return e;
    ++*launches;
  }
  return cudaGetLastError();
}

}  // namespace

int mg_level_count(int n) {
  int levels = 1;
  while (n > kMgCoarsestMax && (n - 1) % 2 == 0 && levels < kMgMaxLevels) {
    n = (n - 1) / 2 + 1;
    ++levels;
  }
  return n <= kMgCoarsestMax ? levels : 1;
}

namespace {

// Reproducible start vector of the power method: components uniform in [-1, 1) from a hash of the index.
__device__ __forceinline__ float hash_unit(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return float(x & 0xffffffu) * (2.0f / 16777216.0f) - 1.0f;
}

struct PowerArgs {
  MgFine fine;
  MgLevel lv[kMgMaxLevels];
  int cta_start[kMgMaxLevels + 1];  // first CTA of each level (indexed from level `first`)
  int first, end;                   // levels [first, end)
  int parity;                       // reads z (0) or e (1) of each level, writes the other; partial region
  int start;                        // first step: the hashed start vector instead of the read buffer
  float* partial;                   // two regions of kMgPartials per-CTA |w|^2
};

// One power-method step on every level at once: w = D^{-1} A (v / |v|), |v| from the previous step's partials.
// S holds D^{-1} during the set-up.
__global__ void __launch_bounds__(kRowThreads) power_kernel(PowerArgs a) {
  int l = a.first;
  while (l + 1 < a.end && int(blockIdx.x) >= a.cta_start[l + 1]) ++l;
  const MgLevel lv = a.lv[l];
  const int c0 = a.cta_start[l], c1 = a.cta_start[l + 1];
  float scale = 1.0f;
  if (!a.start) {
    const float ss = sum_partials(a.partial + (1 - a.parity) * kMgPartials + c0, c1 - c0);
    scale = ss > 0.0f ? rsqrtf(ss) : 0.0f;
  }
  const float4* v = a.parity ? lv.e : lv.z;
  float4* w = a.parity ? lv.z : lv.e;
  const int lane = threadIdx.x % kLanes;
  const int i = (blockIdx.x - c0) * (kRowThreads / kLanes) + threadIdx.x / kLanes;
  const bool active = i < lv.rows;
  auto value = [&](int j) -> float3 {
    if (a.start) {
      const unsigned h = 3u * unsigned(j) + 7919u * unsigned(l);
      return make_float3(hash_unit(h), hash_unit(h + 1), hash_unit(h + 2));
    }
    return scale3(scale, f3(v[j]));
  };
  float3 acc = make_float3(0.f, 0.f, 0.f);
  if (active) {
    if (l == 0) {
      for (int k = a.fine.row_ptr[i] + lane; k < a.fine.row_ptr[i + 1]; k += kLanes) {
        float m[9];
        load_block(a.fine.A, k, m);
        acc = add3(acc, mul(m, value(a.fine.col_idx[k])));
      }
    } else {
      const int n = lv.n, X = i % n, Y = i / n, w2 = lv.w * lv.w;
      for (int o = lane; o < w2; o += kLanes) {
        int j;
        if (stencil_neighbour(n, lv.w, X, Y, o, &j)) acc = add3(acc, stencil_apply(lv.A, w2, i, o, value(j)));
      }
    }
  }
  acc = group_sum(acc);
  float ww = 0.0f;
  if (active && lane == 0) {
    const float3 r = smooth(lv.S, lv.rows, i, acc, false);
    w[i] = pack(r);
    ww = dot3(r, r);
  }
  ww = cta_sum(ww);
  if (threadIdx.x == 0) a.partial[a.parity * kMgPartials + blockIdx.x] = ww;
}

// lambda_l = |D^{-1} A v| for the unit v of the last step; omega_l from it (one warp).
__global__ void power_finish_kernel(PowerArgs a, float* omega) {
  const int lane = threadIdx.x;
  const float* p = a.partial + a.parity * kMgPartials;
  for (int l = a.first; l < a.end; ++l) {
    float s = 0.0f;
    for (int c = a.cta_start[l] + lane; c < a.cta_start[l + 1]; c += 32) s += p[c];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      const float lambda = sqrtf(s);
      omega[l] = lambda > 0.0f && isfinite(lambda) ? 2.0f / (1.1f * lambda * (1.0f + 1.0f / 30.0f)) : 0.3f;
    }
  }
}

__global__ void scale_smoother_kernel(float* S, int count, const float* omega) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < count) S[t] *= *omega;
}

}  // namespace

namespace {

// The power method on levels [first, end) (S holds D^{-1} there), its omega_l into d.omega.
cudaError_t power_method(const MgDevice& d, int first, int end, cudaStream_t s) {
  PowerArgs pa{};
  pa.fine = d.fine;
  for (int l = 0; l < d.levels; ++l) pa.lv[l] = d.lv[l];
  pa.first = first;
  pa.end = end;
  pa.cta_start[first] = 0;
  for (int l = first; l < end; ++l) pa.cta_start[l + 1] = pa.cta_start[l] + row_grid(d.lv[l].rows);
  pa.partial = d.partial;
  const int grid = pa.cta_start[end];
  if (grid > kMgPartials) return cudaErrorInvalidValue;
  for (int k = 0; k < kMgPowerSteps; ++k) {
    pa.parity = k & 1;
    pa.start = k == 0;
    power_kernel<<<grid, kRowThreads, 0, s>>>(pa);
  }
  pa.parity = (kMgPowerSteps - 1) & 1;
  power_finish_kernel<<<1, 32, 0, s>>>(pa, d.omega);
  return cudaGetLastError();
}

}  // namespace

cudaError_t mg_setup(const MgDevice& d, float omega, bool fine_smoother, bool reuse_omega, cudaStream_t s,
                     cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, cudaEvent_t fine_ready,
                     bool* fine_ready_recorded) {
  if (d.levels < 2) return cudaErrorInvalidValue;
  cudaError_t e;
  const int first = fine_smoother ? 0 : 1, end = d.levels - 1;  // smoothed levels
  const double fixed = omega > 0.0f ? omega : 1.0;              // D^{-1} alone before the power method
  const bool spectral = omega <= 0.0f && first < end;
  if (fine_smoother) jacobi_smoother_kernel<true><<<(d.fine.R + 255) / 256, 256, 0, s>>>(d.fine, d.lv[0], fixed);
  // Reusing the spectral estimates, the fine smoother is final right away: scale it now and mark the point, so that
  // whatever needs only the fine level (the network) can run beside the Galerkin products.
  const bool early_fine = fine_ready && spectral && reuse_omega && first == 0 && !d.smoothed;
  if (fine_ready_recorded) *fine_ready_recorded = early_fine;
  if (early_fine) {
    const int count = 9 * d.lv[0].rows;
    scale_smoother_kernel<<<(count + 255) / 256, 256, 0, s>>>(d.lv[0].S, count, d.omega);
    if ((e = cudaEventRecord(fine_ready, s)) != cudaSuccess) return e;
  }
  int l0 = 0;  // first level whose Galerkin product the bilinear loop below forms
  if (d.smoothed) {
    // The smoothed prolongation needs the level-0 spectral estimate before level 1 exists: power method on the
    // fine level first, Sp from it, then the 7 x 7 level-1 product.
    if (spectral && !reuse_omega && first == 0 && (e = power_method(d, 0, 1, s)) != cudaSuccess) return e;
    const int count = 9 * d.fine.R;
    sp_kernel<<<(count + 255) / 256, 256, 0, s>>>(count, d.lv[0].S, d.omega, omega > 0.0f ? 1 : 0, d.Sp);
    galerkin_smoothed_kernel<<<d.lv[1].rows, 32 * kGsWarps, 0, s>>>(d.fine, d.Sp, d.lv[1]);
    if (2 < d.levels) jacobi_smoother_kernel<false><<<(d.lv[1].rows + 255) / 256, 256, 0, s>>>(d.fine, d.lv[1], fixed);
    l0 = 1;
  }
  for (int l = l0; l + 1 < d.levels; ++l) {
    if (l == 0) {
      const int grid = (d.lv[1].rows + GalerkinShape<0>::kWarps - 1) / GalerkinShape<0>::kWarps;
      galerkin_kernel<0><<<grid, 32 * GalerkinShape<0>::kWarps, 0, s>>>(d.fine, d.lv[0], d.lv[1], d.error);
    } else if (d.lv[l].w == 7) {
      const int grid = (d.lv[l + 1].rows + GalerkinShape<7>::kWarps - 1) / GalerkinShape<7>::kWarps;
      galerkin_kernel<7><<<grid, 32 * GalerkinShape<7>::kWarps, 0, s>>>(d.fine, d.lv[l], d.lv[l + 1], d.error);
    } else {
      const int grid = (d.lv[l + 1].rows + GalerkinShape<5>::kWarps - 1) / GalerkinShape<5>::kWarps;
      galerkin_kernel<5><<<grid, 32 * GalerkinShape<5>::kWarps, 0, s>>>(d.fine, d.lv[l], d.lv[l + 1], d.error);
    }
    if (l + 2 < d.levels) {
      const MgLevel& c = d.lv[l + 1];
      jacobi_smoother_kernel<false><<<(c.rows + 255) / 256, 256, 0, s>>>(d.fine, c, fixed);
    }
  }
  {  // the coarsest inverse needs only the last Galerkin product
    const MgLevel& top = d.lv[d.levels - 1];
    const int m = 3 * top.rows;
    const size_t smem = size_t(m) * 2 * m * sizeof(double);
    // The ceiling is one process-wide setting: the largest coarsest level's size for every call, so that
    // concurrent set-ups of different hierarchies never lower it under another's launch.
    constexpr int kCoarseSmemMax = 3 * kMgCoarsestRowsMax * 2 * 3 * kMgCoarsestRowsMax * int(sizeof(double));
    if ((e = cudaFuncSetAttribute(coarse_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kCoarseSmemMax)) != cudaSuccess)
      return e;
    cudaStream_t inv_stream = s;
    if (side) {
      if ((e = cudaEventRecord(fork, s)) != cudaSuccess || (e = cudaStreamWaitEvent(side, fork, 0)) != cudaSuccess)
        return e;
      inv_stream = side;
    }
    coarse_inverse_kernel<<<1, 1024, smem, inv_stream>>>(top, d.coarse_inv, d.error);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (side && (e = cudaEventRecord(join, side)) != cudaSuccess) return e;
  }
  if (spectral) {
    // without the smoothed prolongation every smoothed level in one power method; with it, the rest
    const int from = d.smoothed && first == 0 ? 1 : first;
    if (!reuse_omega && from < end && (e = power_method(d, from, end, s)) != cudaSuccess) return e;
    for (int l = early_fine ? 1 : first; l < end; ++l) {
      const int count = 9 * d.lv[l].rows;
      scale_smoother_kernel<<<(count + 255) / 256, 256, 0, s>>>(d.lv[l].S, count, d.omega + l);
    }
  }
  return cudaGetLastError();
}

cudaError_t mg_pcg_init(const MgDevice& d, float tol2, int max_iterations, int stall_window, cudaStream_t s) {
  InitArgs a{};
  a.R = d.fine.R;
  a.b = d.b;
  a.x = d.x;
  a.r0 = d.r[0];
  a.r1 = d.r[1];
  a.p0 = d.p[0];
  a.p1 = d.p[1];
  a.S0 = d.lv[0].S;
  a.z_pre = d.lv[0].z;
  a.rr_partial = d.partial + kPartRr * kMgPartials;
  a.state = d.state;
  a.tol2 = tol2;
  a.max_iterations = max_iterations;
  a.stall_window = stall_window;
  init_kernel<<<update_grid(a.R), kUpdateThreads, 0, s>>>(a);
  if (d.smoothed) {  // the first iteration's t, u and |r0|^2 slots, as update_residual_kernel leaves them
    SmoothedArgs sa{};
    sa.fine = d.fine;
    sa.r = d.r[0];
    sa.z = d.lv[0].z;
    sa.Sp = d.Sp;
    sa.t = d.t;
    sa.u = d.u;
    sa.rr_init = d.partial + kPartRr * kMgPartials;
    residual_smoothed_kernel<false><<<row_grid(a.R), kRowThreads, 0, s>>>(sa);
  }
  return cudaGetLastError();
}

namespace {

// Iterations of parity 0 and 1 (one graph body); the second update kernel owns the WHILE condition.
cudaError_t launch_body(const MgDevice& d, cudaGraphConditionalHandle cond, bool graph, bool pdl, cudaStream_t s,
                        int* launches) {
  const int R = d.fine.R;
  // bilinear prolongation with two or more restricted levels: each iteration's update runs fused with the next
  // iteration's first restriction (update_restrict_kernel), and the direction kernel ends the graph body
  const bool fused = !d.smoothed && d.levels >= 4;
  for (int par = 0; par < 2; ++par) {
    UpdateArgs fa{};
    fa.R = R;
    fa.p = d.p[1 - par];
    fa.q = d.q;
    fa.r_cur = d.r[1 - par];
    fa.r_next = d.r[par];
    fa.x = d.x;
    fa.S0 = d.lv[0].S;
    fa.z_pre = d.lv[0].z;
    fa.state = d.state;
    fa.pq_partial = d.partial + kPartPq * kMgPartials;
    fa.pq_count = row_grid(R);
    fa.rr_partial = d.partial + kPartRr * kMgPartials;
    cudaError_t e = launch_cycle(d, par, true, pdl, s, launches, fused ? &fa : nullptr);
    if (e != cudaSuccess) return e;
    DirectionArgs da{};
    da.fine = d.fine;
    da.z = d.lv[0].e;
    da.p_old = d.p[1 - par];
    da.p_new = d.p[par];
    da.q = d.q;
    da.state = d.state;
    da.zr_partial = d.partial + kPartZr * kMgPartials;
    da.zrp_partial = d.partial + kPartZrPrev * kMgPartials;
    da.zr_count = row_grid(R);
    da.pq_partial = d.partial + kPartPq * kMgPartials;
    da.cond = cond;
    da.set_cond = fused && graph && par == 1;
    if ((e = launch(direction_kernel, row_grid(R), kRowThreads, s, pdl, da)) != cudaSuccess) return e;
    if (fused) {
      *launches += 1;
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      continue;
    }
    UpdateArgs ua{};
    ua.R = R;
    ua.p = d.p[par];
    ua.q = d.q;
    ua.r_cur = d.r[par];
    ua.r_next = d.r[1 - par];
    ua.x = d.x;
    ua.S0 = d.lv[0].S;
    ua.z_pre = d.lv[0].z;
    ua.state = d.state;
    ua.pq_partial = d.partial + kPartPq * kMgPartials;
    ua.pq_count = row_grid(R);
    ua.rr_partial = d.partial + kPartRr * kMgPartials;
    ua.cond = cond;
    ua.set_cond = graph && par == 1;
    if (d.smoothed) {
      SmoothedArgs sa{};
      sa.fine = d.fine;
      sa.Sp = d.Sp;
      sa.t = d.t;
      sa.u = d.u;
      if ((e = launch(update_residual_kernel, row_grid(R), kRowThreads, s, pdl, ua, sa)) != cudaSuccess) return e;
    } else if ((e = launch(update_kernel, update_grid(R), kUpdateThreads, s, pdl, ua)) != cudaSuccess) {
      return e;
    }
    *launches += 2;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

cudaError_t mg_build_solve_graph(const MgDevice& d, cudaStream_t s, cudaGraphExec_t* exec, int* launches_per_body,
                                 bool pdl) {
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaGraphCreate(&graph, 0);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle cond;
  cudaGraphNodeParams p{};
  cudaGraphNode_t node;
  if ((e = cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess) goto done;
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = cond;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  if ((e = cudaGraphAddNode(&node, graph, nullptr, 0, &p)) != cudaSuccess) goto done;
  {
    cudaGraph_t body = p.conditional.phGraph_out[0];
    if ((e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
      goto done;
    *launches_per_body = 0;
    cudaError_t le = launch_body(d, cond, true, pdl, s, launches_per_body);
    e = cudaStreamEndCapture(s, &body);
    if (le != cudaSuccess) e = le;
    if (e != cudaSuccess) goto done;
  }
  e = cudaGraphInstantiate(exec, graph, 0);
done:
  cudaGraphDestroy(graph);
  return e;
}

cudaError_t mg_launch_iterations(const MgDevice& d, int pairs, cudaStream_t s) {
  int launches = 0;
  for (int k = 0; k < pairs; ++k) {
    cudaError_t e = launch_body(d, cudaGraphConditionalHandle{}, false, true, s, &launches);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t mg_apply(const MgDevice& d, cudaStream_t s) {
  const int R = d.fine.R;
  presmooth_kernel<<<(R + 255) / 256, 256, 0, s>>>(R, d.lv[0].S, d.r[0], d.lv[0].z);
  int launches = 0;
  return launch_cycle(d, 0, false, false, s, &launches);
}

}  // namespace drape
