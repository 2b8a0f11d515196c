// Preconditioner network kernels (see nn.h): features, bf16 tensor-core forward layers, f32 backward, Adam.
// Every reduction over rows goes through per-CTA partials summed in a fixed order (deterministic training).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "nn.h"

namespace drape {
namespace {

constexpr int kH = kNnHidden;
constexpr int kBackThreads = 256;

__device__ __forceinline__ void load_block(const DevBsr& A, int k, float m[9]) {
  const float4 u = A.a0[k], v = A.a1[k];
  m[0] = u.x; m[1] = u.y; m[2] = u.z; m[3] = u.w;
  m[4] = v.x; m[5] = v.y; m[6] = v.z; m[7] = v.w;
  m[8] = A.a2[k];
}

__device__ __forceinline__ float frob(const float m[9]) {
  float s = 0.0f;
#pragma unroll
  for (int e = 0; e < 9; ++e) s += m[e] * m[e];
  return sqrtf(s);
}

__device__ __forceinline__ float sigmoid(float o) { return 1.0f / (1.0f + expf(-o)); }

// 16 scale-free features of row i and the aggregation weights w_ij of its off-diagonal blocks.
//   0..5  diagonal block entries (00, 11, 22, 01, 02, 12) / trace
//   6, 7  sum and max of off-diagonal |A_ij|_F over |D_i|_F
//   8     blocks in the row / 25
//   9     the fine level's spectral damping omega_0
//   10    sum_j |D_i^{-1} A_ij|_F / 10 (a local bound on the row's spectral radius)
//   11    1
__global__ void features_kernel(NnBuffers b, const float* omega0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.R) return;
  const int k0 = b.row_ptr[i], k1 = b.row_ptr[i + 1], kd = b.diag_pos[i];
  float D[9];
  load_block(b.A, kd, D);
  const float tr = D[0] + D[4] + D[8];
  const float dn = frob(D);
  // D^{-1} by the adjugate (zero if singular)
  float c[9];
  c[0] = D[4] * D[8] - D[5] * D[7];
  c[1] = D[2] * D[7] - D[1] * D[8];
  c[2] = D[1] * D[5] - D[2] * D[4];
  c[3] = D[5] * D[6] - D[3] * D[8];
  c[4] = D[0] * D[8] - D[2] * D[6];
  c[5] = D[2] * D[3] - D[0] * D[5];
  c[6] = D[3] * D[7] - D[4] * D[6];
  c[7] = D[1] * D[6] - D[0] * D[7];
  c[8] = D[0] * D[4] - D[1] * D[3];
  const float det = D[0] * c[0] + D[1] * c[3] + D[2] * c[6];
  const float rdet = det != 0.0f && isfinite(det) ? 1.0f / det : 0.0f;
  float off_sum = 0.0f, off_max = 0.0f, local = 0.0f;
  for (int k = k0; k < k1; ++k) {
    if (k == kd) continue;
    float m[9];
    load_block(b.A, k, m);
    const float f = frob(m);
    off_sum += f;
    off_max = fmaxf(off_max, f);
    float p[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        p[3 * r + q] = rdet * (c[3 * r] * m[q] + c[3 * r + 1] * m[3 + q] + c[3 * r + 2] * m[6 + q]);
    local += frob(p);
  }
  const float inv_off = off_sum > 0.0f ? 1.0f / off_sum : 0.0f;
  for (int k = k0; k < k1; ++k) {
    if (k == kd) {
      b.w[k] = 0.0f;
      continue;
    }
    float m[9];
    load_block(b.A, k, m);
    b.w[k] = frob(m) * inv_off;
  }
  const float rt = tr != 0.0f && isfinite(tr) ? 1.0f / tr : 0.0f;
  const float rn = dn > 0.0f ? 1.0f / dn : 0.0f;
  float* f = b.feat + size_t(i) * kNnIn;
  f[0] = D[0] * rt;
  f[1] = D[4] * rt;
  f[2] = D[8] * rt;
  f[3] = 0.5f * (D[1] + D[3]) * rt;
  f[4] = 0.5f * (D[2] + D[6]) * rt;
  f[5] = 0.5f * (D[5] + D[7]) * rt;
  f[6] = off_sum * rn;
  f[7] = off_max * rn;
  f[8] = float(k1 - k0) * (1.0f / 25.0f);
  f[9] = *omega0;
  f[10] = 0.1f * local;
  f[11] = 1.0f;
#pragma unroll
  for (int q = 12; q < kNnIn; ++q) f[q] = 0.0f;
}

__device__ __forceinline__ void mma_bf16(float c[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// out = relu(X W + bias) for 64 rows per CTA, X = in rows (K = 16) or [h_i, sum_j w_ij h_j] (K = 128), bf16
// operands in shared memory, one warp per 16 rows x 64 outputs (8 n-tiles of m16n8k16).
template <int K, bool kAgg>
__global__ void __launch_bounds__(128) layer_kernel(NnBuffers b, const float* in, const __nv_bfloat16* Wt,
                                                    const float* bias, float* out) {
  constexpr int KP = K + 8;  // padded row (bank spread), even: 32-bit fragment loads stay aligned
  __shared__ __align__(16) __nv_bfloat16 Xs[kNnRowsPerCta * KP];
  __shared__ __align__(16) __nv_bfloat16 Ws[kH * KP];
  const int row0 = blockIdx.x * kNnRowsPerCta;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int t = threadIdx.x; t < kH * K; t += blockDim.x) Ws[(t / K) * KP + t % K] = Wt[t];
  if (!kAgg) {
    for (int t = threadIdx.x; t < kNnRowsPerCta * K; t += blockDim.x) {
      const int r = t / K, k = t % K, i = row0 + r;
      Xs[r * KP + k] = __float2bfloat16(i < b.R ? in[size_t(i) * K + k] : 0.0f);
    }
  } else {
    for (int rr = 0; rr < 16; ++rr) {
      const int r = warp * 16 + rr, i = row0 + r;
      float self[2] = {0.0f, 0.0f}, agg[2] = {0.0f, 0.0f};
      if (i < b.R) {
        self[0] = in[size_t(i) * kH + lane];
        self[1] = in[size_t(i) * kH + lane + 32];
        for (int k = b.row_ptr[i]; k < b.row_ptr[i + 1]; ++k) {
          const float wk = b.w[k];
          if (wk == 0.0f) continue;
          const float* hj = in + size_t(b.col_idx[k]) * kH;
          agg[0] += wk * hj[lane];
          agg[1] += wk * hj[lane + 32];
        }
      }
      Xs[r * KP + lane] = __float2bfloat16(self[0]);
      Xs[r * KP + lane + 32] = __float2bfloat16(self[1]);
      Xs[r * KP + kH + lane] = __float2bfloat16(agg[0]);
      Xs[r * KP + kH + lane + 32] = __float2bfloat16(agg[1]);
    }
  }
  __syncthreads();
  const int gid = lane >> 2, tig = lane & 3;
  float c[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.0f;
#pragma unroll
  for (int kb = 0; kb < K; kb += 16) {
    const __nv_bfloat16* xa = Xs + (warp * 16 + gid) * KP + kb + tig * 2;
    const uint32_t a0 = *reinterpret_cast<const uint32_t*>(xa);
    const uint32_t a1 = *reinterpret_cast<const uint32_t*>(xa + 8 * KP);
    const uint32_t a2 = *reinterpret_cast<const uint32_t*>(xa + 8);
    const uint32_t a3 = *reinterpret_cast<const uint32_t*>(xa + 8 * KP + 8);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const __nv_bfloat16* wb = Ws + (nt * 8 + gid) * KP + kb + tig * 2;
      mma_bf16(c[nt], a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(wb),
               *reinterpret_cast<const uint32_t*>(wb + 8));
    }
  }
  const int i0 = row0 + warp * 16 + gid, i1 = i0 + 8;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int n = nt * 8 + tig * 2;
    if (i0 < b.R) {
      out[size_t(i0) * kH + n] = fmaxf(c[nt][0] + bias[n], 0.0f);
      out[size_t(i0) * kH + n + 1] = fmaxf(c[nt][1] + bias[n + 1], 0.0f);
    }
    if (i1 < b.R) {
      out[size_t(i1) * kH + n] = fmaxf(c[nt][2] + bias[n], 0.0f);
      out[size_t(i1) * kH + n + 1] = fmaxf(c[nt][3] + bias[n + 1], 0.0f);
    }
  }
}

// o_i = w_o . h4_i + b_o; f_i = kNnFactorLow + kNnFactorSpan sigmoid(o_i + kNnFactorShift) scales row i of the
// smoother S [9][R] (if given).
__global__ void head_kernel(NnBuffers b, const float* params, float* S) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.R) return;
  const float* h4 = b.h + (size_t(kNnLayers) * b.R + i) * kH;
  float o = params[kNnOffBo];
  for (int n = 0; n < kH; ++n) o += params[kNnOffWo + n] * h4[n];
  b.o[i] = o;
  if (S) {
    const float f = kNnFactorLow + kNnFactorSpan * sigmoid(o + kNnFactorShift);
#pragma unroll
    for (int e = 0; e < 9; ++e) S[e * b.R + i] *= f;
  }
}

// ------------------------------------------------------------------------------------------------ backward

// do_i = dL/df_i * sigmoid'(o_i); dh4 = do w_o; partials of w_o and b_o.
__global__ void __launch_bounds__(kBackThreads) head_backward_kernel(NnBuffers b, const float* params,
                                                                     const float* dfactor, float* dh4) {
  __shared__ float do_s[kNnBackRows];
  const int row0 = blockIdx.x * kNnBackRows;
  if (threadIdx.x < kNnBackRows) {
    const int i = row0 + threadIdx.x;
    float d = 0.0f;
    if (i < b.R) {
      const float s = sigmoid(b.o[i] + kNnFactorShift);
      d = dfactor[i] * kNnFactorSpan * s * (1.0f - s);
    }
    do_s[threadIdx.x] = d;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kNnBackRows * kH; t += blockDim.x) {
    const int r = t / kH, n = t % kH, i = row0 + r;
    if (i < b.R) dh4[size_t(i) * kH + n] = do_s[r] * params[kNnOffWo + n];
  }
  float* part = b.partial + size_t(blockIdx.x) * kNnParams;
  const float* h4 = b.h + size_t(kNnLayers) * b.R * kH;
  if (threadIdx.x < kH) {
    float s = 0.0f;
    for (int r = 0; r < kNnBackRows; ++r) {
      const int i = row0 + r;
      if (i < b.R) s += do_s[r] * h4[size_t(i) * kH + threadIdx.x];
    }
    part[kNnOffWo + threadIdx.x] = s;
  } else if (threadIdx.x == kH) {
    float s = 0.0f;
    for (int r = 0; r < kNnBackRows; ++r) s += do_s[r];
    part[kNnOffBo] = s;
  }
}

// One dense layer backward on 32 rows: dpre = dh_out * [h_out > 0]; partials of W (X^T dpre) and b; dx = dpre W^T
// (K = 128 only). X is rebuilt in f32 (the forward rounded it to bf16).
template <int K, bool kAgg>
__global__ void __launch_bounds__(kBackThreads) layer_backward_kernel(NnBuffers b, const float* params, int off_w,
                                                                      int off_b, const float* in, const float* h_out,
                                                                      const float* dh_out) {
  extern __shared__ float smem[];
  float* Ws = smem;                    // [K][64]
  float* Xs = Ws + K * kH;             // [32][K]
  float* Ds = Xs + kNnBackRows * K;    // [32][64]
  const int row0 = blockIdx.x * kNnBackRows;
  for (int t = threadIdx.x; t < K * kH; t += blockDim.x) Ws[t] = params[off_w + t];
  for (int t = threadIdx.x; t < kNnBackRows * kH; t += blockDim.x) {
    const int r = t / kH, n = t % kH, i = row0 + r;
    float d = 0.0f;
    if (i < b.R && h_out[size_t(i) * kH + n] > 0.0f) d = dh_out[size_t(i) * kH + n];
    Ds[t] = d;
  }
  if (!kAgg) {
    for (int t = threadIdx.x; t < kNnBackRows * K; t += blockDim.x) {
      const int r = t / K, k = t % K, i = row0 + r;
      Xs[t] = i < b.R ? in[size_t(i) * K + k] : 0.0f;
    }
  } else {
    for (int t = threadIdx.x; t < kNnBackRows * kH; t += blockDim.x) {
      const int r = t / kH, f = t % kH, i = row0 + r;
      float self = 0.0f, agg = 0.0f;
      if (i < b.R) {
        self = in[size_t(i) * kH + f];
        for (int k = b.row_ptr[i]; k < b.row_ptr[i + 1]; ++k) {
          const float wk = b.w[k];
          if (wk != 0.0f) agg += wk * in[size_t(b.col_idx[k]) * kH + f];
        }
      }
      Xs[r * K + f] = self;
      Xs[r * K + kH + f] = agg;
    }
  }
  __syncthreads();
  float* part = b.partial + size_t(blockIdx.x) * kNnParams;
  for (int p = threadIdx.x; p < K * kH; p += blockDim.x) {
    const int k = p / kH, n = p % kH;
    float s = 0.0f;
    for (int r = 0; r < kNnBackRows; ++r) s += Xs[r * K + k] * Ds[r * kH + n];
    part[off_w + p] = s;
  }
  if (threadIdx.x < kH) {
    float s = 0.0f;
    for (int r = 0; r < kNnBackRows; ++r) s += Ds[r * kH + threadIdx.x];
    part[off_b + threadIdx.x] = s;
  }
  if (kAgg) {
    for (int t = threadIdx.x; t < kNnBackRows * K; t += blockDim.x) {
      const int r = t / K, k = t % K, i = row0 + r;
      if (i >= b.R) continue;
      float s = 0.0f;
      for (int n = 0; n < kH; ++n) s += Ws[k * kH + n] * Ds[r * kH + n];
      b.dx[size_t(i) * 2 * kH + k] = s;
    }
  }
}

// dh_prev_j = dx_j[0:64] + sum_{i : j in N(i)} w_ij dx_i[64:128] (the transpose of the aggregation).
__global__ void scatter_backward_kernel(NnBuffers b, float* dh_prev) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = t / kH, f = t % kH;
  if (j >= b.R) return;
  float s = b.dx[size_t(j) * 2 * kH + f];
  for (int k = b.row_ptr[j]; k < b.row_ptr[j + 1]; ++k) {
    const float wk = b.w[b.transpose[k]];  // w_ij of row i = col_idx[k]
    if (wk != 0.0f) s += wk * b.dx[size_t(b.col_idx[k]) * 2 * kH + kH + f];
  }
  dh_prev[size_t(j) * kH + f] = s;
}

__global__ void reduce_grad_kernel(const float* partial, int ctas, float* grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNnParams) return;
  float s = 0.0f;
  for (int c = 0; c < ctas; ++c) s += partial[size_t(c) * kNnParams + p];
  grad[p] = s;
}

__global__ void adam_kernel(NnWeights w, const float* grad, float lr, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNnParams) return;
  const float g = grad[p];
  const float m = 0.9f * w.adam_m[p] + 0.1f * g;
  const float v = 0.999f * w.adam_v[p] + 0.001f * g * g;
  w.adam_m[p] = m;
  w.adam_v[p] = v;
  w.master[p] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
}

// Transposed bf16 copies: Wt_in[n][k] = W_in[k][n] (k < 16), Wt_l[n][k] = W_l[k][n] (k < 128).
__global__ void bf16_kernel(NnWeights w) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kNnBf16) return;
  if (t < kNnIn * kH) {
    const int n = t / kNnIn, k = t % kNnIn;
    w.bf16[t] = __float2bfloat16(w.master[kNnOffWin + k * kH + n]);
    return;
  }
  const int u = t - kNnIn * kH, l = u / (2 * kH * kH), v = u % (2 * kH * kH);
  const int n = v / (2 * kH), k = v % (2 * kH);
  w.bf16[t] = __float2bfloat16(w.master[kNnOffLayer0 + l * kNnLayerSize + k * kH + n]);
}

int back_smem(int K) { return (K * kH + kNnBackRows * K + kNnBackRows * kH) * int(sizeof(float)); }

// ------------------------------------------------------------------------------------- training vector operations

__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }

__device__ __forceinline__ float3 block_mul(const float* S, int R, int i, float3 v) {
  float m[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) m[e] = S[e * R + i];
  return make_float3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
                     m[6] * v.x + m[7] * v.y + m[8] * v.z);
}

__global__ void vec_kernel(int R, const float4* x, const float4* y, float4* out, float a, float bb, const float* scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R) return;
  const float s = scale ? *scale : 1.0f;
  const float4 u = x[i];
  const float4 v = y ? y[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  out[i] = make_float4(s * (a * u.x + bb * v.x), s * (a * u.y + bb * v.y), s * (a * u.z + bb * v.z), 0.0f);
}

__global__ void block_apply_kernel(int R, const float* S, const float4* v, float4* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R) return;
  const float3 r = block_mul(S, R, i, f3(v[i]));
  out[i] = make_float4(r.x, r.y, r.z, 0.0f);
}

constexpr int kDotThreads = 256, kDotGrid = 148;

__global__ void __launch_bounds__(kDotThreads) dot_kernel(int R, const float4* x, const float4* y, double* partial) {
  __shared__ double ws[kDotThreads / 32];
  double s = 0.0;
  for (int i = blockIdx.x * kDotThreads + threadIdx.x; i < R; i += kDotGrid * kDotThreads) {
    const float4 u = x[i], v = y[i];
    s += double(u.x) * v.x + double(u.y) * v.y + double(u.z) * v.z;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kDotThreads / 32; ++w) t += ws[w];
    partial[blockIdx.x] = t;
  }
}

// scalars[slot] = sum of the partials; mode 1 also writes scalars[slot + 1] = -2 / that sum (as f32 in fscale).
__global__ void dot_finish_kernel(const double* partial, double* scalars, int slot, float* fscale) {
  if (threadIdx.x != 0) return;
  double t = 0.0;
  for (int c = 0; c < kDotGrid; ++c) t += partial[c];
  scalars[slot] = t;
  if (fscale) *fscale = t != 0.0 ? float(-2.0 / t) : 0.0f;
}

// dL/df_i = g_post_i . (S0_i u_i) + g_pre_i . (S0_i b_i)  (S_i = f_i S0_i in both smoothing steps).
__global__ void dfactor_kernel(int R, const float* S0, const float4* g_post, const float4* u, const float4* g_pre,
                               const float4* b, float* dfac) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R) return;
  const float3 su = block_mul(S0, R, i, f3(u[i])), sb = block_mul(S0, R, i, f3(b[i]));
  const float3 gp = f3(g_post[i]), gq = f3(g_pre[i]);
  dfac[i] = gp.x * su.x + gp.y * su.y + gp.z * su.z + gq.x * sb.x + gq.y * sb.y + gq.z * sb.z;
}

}  // namespace

cudaError_t nn_vec(int R, const float4* x, const float4* y, float4* out, float a, float b, const float* scale,
                   cudaStream_t s) {
  vec_kernel<<<(R + 255) / 256, 256, 0, s>>>(R, x, y, out, a, b, scale);
  return cudaGetLastError();
}

cudaError_t nn_block_apply(int R, const float* S, const float4* v, float4* out, cudaStream_t s) {
  block_apply_kernel<<<(R + 255) / 256, 256, 0, s>>>(R, S, v, out);
  return cudaGetLastError();
}

cudaError_t nn_dot(int R, const float4* x, const float4* y, double* partial, double* scalars, int slot, float* fscale,
                   cudaStream_t s) {
  dot_kernel<<<kDotGrid, kDotThreads, 0, s>>>(R, x, y, partial);
  dot_finish_kernel<<<1, 32, 0, s>>>(partial, scalars, slot, fscale);
  return cudaGetLastError();
}

cudaError_t nn_dfactor(int R, const float* S0, const float4* g_post, const float4* u, const float4* g_pre,
                       const float4* b, float* dfac, cudaStream_t s) {
  dfactor_kernel<<<(R + 255) / 256, 256, 0, s>>>(R, S0, g_post, u, g_pre, b, dfac);
  return cudaGetLastError();
}

int nn_back_ctas(int R) { return (R + kNnBackRows - 1) / kNnBackRows; }

cudaError_t nn_forward(const NnBuffers& b, const NnWeights& w, const float* omega0, float* S, cudaStream_t s) {
  const int R = b.R;
  features_kernel<<<(R + 255) / 256, 256, 0, s>>>(b, omega0);
  const int grid = (R + kNnRowsPerCta - 1) / kNnRowsPerCta;
  layer_kernel<kNnIn, false><<<grid, 128, 0, s>>>(b, b.feat, w.bf16, w.master + kNnOffBin, b.h);
  for (int l = 0; l < kNnLayers; ++l) {
    const __nv_bfloat16* Wt = w.bf16 + kNnIn * kH + l * 2 * kH * kH;
    const float* bias = w.master + kNnOffLayer0 + l * kNnLayerSize + 2 * kH * kH;
    layer_kernel<2 * kNnHidden, true><<<grid, 128, 0, s>>>(b, b.h + size_t(l) * R * kH, Wt, bias,
                                                           b.h + size_t(l + 1) * R * kH);
  }
  head_kernel<<<(R + 255) / 256, 256, 0, s>>>(b, w.master, S);
  return cudaGetLastError();
}

cudaError_t nn_backward(const NnBuffers& b, const NnWeights& w, const float* dfactor, cudaStream_t s) {
  const int R = b.R, ctas = nn_back_ctas(R);
  cudaError_t e;
  float* dh[2] = {b.dh, b.dh + size_t(R) * kH};
  head_backward_kernel<<<ctas, kBackThreads, 0, s>>>(b, w.master, dfactor, dh[0]);
  const int sm128 = back_smem(2 * kH), sm16 = back_smem(kNnIn);
  if ((e = cudaFuncSetAttribute(layer_backward_kernel<2 * kNnHidden, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, sm128)) != cudaSuccess)
    return e;
  int cur = 0;
  for (int l = kNnLayers - 1; l >= 0; --l) {
    const int off_w = kNnOffLayer0 + l * kNnLayerSize, off_b = off_w + 2 * kH * kH;
    const float* in = b.h + size_t(l) * R * kH;
    const float* out = b.h + size_t(l + 1) * R * kH;
    layer_backward_kernel<2 * kNnHidden, true><<<ctas, kBackThreads, sm128, s>>>(b, w.master, off_w, off_b, in, out,
                                                                                dh[cur]);
    scatter_backward_kernel<<<(R * kH + 255) / 256, 256, 0, s>>>(b, dh[1 - cur]);
    cur = 1 - cur;
  }
  layer_backward_kernel<kNnIn, false><<<ctas, kBackThreads, sm16, s>>>(b, w.master, kNnOffWin, kNnOffBin, b.feat, b.h,
                                                                      dh[cur]);
  reduce_grad_kernel<<<(kNnParams + 255) / 256, 256, 0, s>>>(b.partial, ctas, b.grad);
  return cudaGetLastError();
}

cudaError_t nn_adam(const NnWeights& w, const float* grad, float lr, int t, cudaStream_t s) {
  const float c1 = 1.0f - powf(0.9f, float(t)), c2 = 1.0f - powf(0.999f, float(t));
  adam_kernel<<<(kNnParams + 255) / 256, 256, 0, s>>>(w, grad, lr, c1, c2);
  return nn_refresh_bf16(w, s);
}

cudaError_t nn_refresh_bf16(const NnWeights& w, cudaStream_t s) {
  bf16_kernel<<<(kNnBf16 + 255) / 256, 256, 0, s>>>(w);
  return cudaGetLastError();
}

}  // namespace drape
