// Block-Jacobi PCG on the f32 BSR(3x3) Newton matrix as ONE persistent cooperative kernel (sm_100a).
//
// Each CTA owns a contiguous range of block rows for the whole solve and keeps, in shared memory, the rows'
// BSR blocks and column indices (when they fit), the inverted diagonal blocks and the row vectors x, r, z, p, q
// and b. Only the vectors other CTAs gather (p and z) are published to global memory (L2). One iteration:
//   A  q = A p and the partial p.q. The direction update p = z + beta p_old is fused into the column gathers
//      (every CTA forms the gathered p from the published z and previous p; the owner publishes its new p into
//      the other of two buffers, which nobody reads in this phase);
//   B  alpha = rz / pq, x += alpha p, r -= alpha q, z = D^-1 r (all from shared memory), publish z, and the
//      partials of r.z and r.r.
// Each phase ends in a reduce-and-broadcast barrier: every CTA publishes its partials as 64-bit words
// (generation << 32 | float bits); a master warp in CTA 0 waits for all words of the generation, sums them in a
// fixed order and publishes (generation, total) words that every CTA waits for. No atomics, so every CTA takes
// the same alpha, beta and stop decision and the solve is deterministic; every wait gives up after `spin_limit`
// cycles, sets `*error` and the kernel returns, so a stalled launch cannot hang the GPU.
// That is the reference's two-reduction iteration; the default form (SINGLE, see pcg_kernel) takes one phase and one
// reduce barrier per iteration through the Chronopoulos-Gear recurrences.
// Residual replacement (r = b - A x every `replace_every` iterations while rr > replace_above^2 rr0, keeping p)
// follows pcg.rs:213-223 (two-reduction form only). Block rows are processed by groups of LPR lanes with xor-shuffle reductions; every row
// loop has a CTA-uniform trip count so all lanes reach the shuffles.
// Reference semantics: pcg.rs:271-296 (solve), 389-439 (State), 479-492 (invert3); WGSL cg_init, spmv_dot,
// update_dot, direction, reduce, residual.
#include <cuda_runtime.h>

#include <cstdint>

#include "bulk.cuh"
#include "kernels.h"

namespace drape {
namespace {

__device__ __forceinline__ float4 f4(float a, float b, float c) { return make_float4(a, b, c, 0.0f); }
__device__ __forceinline__ float dot3(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// s a + b per component, rounded once (the same bits wherever it is evaluated)
__device__ __forceinline__ float4 fma4(float s, float4 a, float4 b) {
  return f4(__fmaf_rn(s, a.x, b.x), __fmaf_rn(s, a.y, b.y), __fmaf_rn(s, a.z, b.z));
}
__device__ __forceinline__ unsigned long long pack(unsigned gen, float v) {
  return (static_cast<unsigned long long>(gen) << 32) | __float_as_uint(v);
}
// CTA sum of NV per-thread floats into out[] (valid in thread 0 after the call).
template <int NV> __device__ __forceinline__ void cta_sum(float (&v)[NV], float* out) {
  __shared__ float red[NV][32];
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) red[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x < 32) {
    const int warps = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      float s = threadIdx.x < warps ? red[k][threadIdx.x] : 0.0f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (threadIdx.x == 0) out[k] = s;
    }
  }
}

__device__ __forceinline__ void store_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long load_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Publishes this CTA's NV partials for generation `gen` and returns (in vals, all threads) the grid totals.
// All-to-all: thread 0 release-stores the CTA's (gen, partial) words after a CTA barrier (so they order every
// thread's earlier stores of published vectors); thread t of every CTA acquire-polls CTA t's words (all words in
// parallel, blockDim.x >= gridDim.x, host-checked); every CTA then sums the words in the same fixed order.
// Words alternate between two buffers by generation parity: a CTA can only rewrite a buffer after every CTA has
// published the next generation, i.e. after every CTA has read this one. Each parity holds STRIDE values per CTA
// (2 for the two-reduction iteration, 3 for the single-reduction one).
template <int NV, int STRIDE = 2>
__device__ __forceinline__ bool reduce_barrier(const PcgArgs& a, unsigned gen, float* vals) {
  static_assert(NV <= STRIDE, "more values than slots");
  __shared__ float words[NV][1024];
  __shared__ float totals[NV];
  __shared__ int bad;
  const unsigned G = gridDim.x;
  unsigned long long* slots = a.slots + (gen & 1u) * unsigned(STRIDE) * G;
  if (threadIdx.x == 0) {
    bad = 0;
#pragma unroll
    for (int k = 0; k < NV; ++k) store_release(slots + k * G + blockIdx.x, pack(gen, vals[k]));
  }
  __syncthreads();
  if (threadIdx.x < G) {
    const long long t0 = clock64();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      unsigned long long w = load_acquire(slots + k * G + threadIdx.x);
      while (static_cast<unsigned>(w >> 32) != gen) {
        if (clock64() - t0 > a.spin_limit) {
          bad = 1;
          break;
        }
        w = load_acquire(slots + k * G + threadIdx.x);
      }
      words[k][threadIdx.x] = __uint_as_float(static_cast<unsigned>(w));
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      float s = 0.0f;
      for (unsigned i = threadIdx.x; i < G; i += 32) s += words[k][i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (threadIdx.x == 0) totals[k] = s;
    }
    if (threadIdx.x == 0 && bad) atomicExch(a.error, 1);
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) vals[k] = totals[k];
  return !bad;
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

__device__ __forceinline__ void apply(float4 m0, float4 m1, float m8, float4 p, float& y0, float& y1, float& y2) {
  y0 += m0.x * p.x + m0.y * p.y + m0.z * p.z;
  y1 += m0.w * p.x + m1.x * p.y + m1.y * p.z;
  y2 += m1.z * p.x + m1.w * p.y + m8 * p.z;
}

// The single-reduction iteration (SINGLE, Chronopoulos-Gear PCG: A. T. Chronopoulos and C. W. Gear, J. Comput.
// Appl. Math. 25 (1989) 153-168) carries w = A u and s = A p (a recurrence), so that one grid reduction per
// iteration gives every dot product the next step needs:
//   s = w + beta s, p = u + beta p, x += alpha p, r -= alpha s, u = M r,
//   w = A u;  gamma = r.u, delta = w.u, rho = r.r, u.s + p.w, p.s  (one reduce barrier);
//   beta = gamma / gamma_old, p.A p = delta + beta (u.s + p.w) + beta^2 p.s, alpha = gamma / p.A p.
// (Chronopoulos and Gear take p.A p = delta - beta gamma / alpha_old, which assumes exact orthogonality and broke
// down in f32 on the reference's tension system after ~100 iterations; the expansion over the current vectors does
// not.)
// The SpMV runs in the same phase that forms u, so a CTA forms the u of each gathered column itself, from what
// the column's owner published in the previous iteration: u_old = M r_old, M w_old and M s_older, as
// u_old - alpha (M w_old + beta M s_older) (= M r in exact arithmetic; one step's rounding away from the owner's
// M r, which the owner recomputes directly every iteration, so the difference never accumulates: carrying u itself
// as a recurrence stagnated at a relative residual of ~4e-6 on the reference's tension system). The published
// vectors are double-buffered by iteration parity. Residual replacement is not available in this form.
template <int LPR, bool MSMEM, bool SINGLE>
__global__ void __launch_bounds__(1024) pcg_kernel(PcgArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int G = gridDim.x, cta = blockIdx.x;
  const int r0 = (int)((long long)a.R * cta / G), r1 = (int)((long long)a.R * (cta + 1) / G), n = r1 - r0;
  const int kb0 = a.row_ptr[r0], nb = a.row_ptr[r1] - kb0;
  const int groups = blockDim.x / LPR, group = threadIdx.x / LPR, gl = threadIdx.x % LPR;
  const int cap = a.cap_rows;
  float4* xs = reinterpret_cast<float4*>(smem);
  float4* rs = xs + cap;
  float4* zs = rs + cap;
  float4* ps = zs + cap;
  float4* qs = ps + cap;
  float4* bs = qs + cap;
  float4* dv = bs + cap;  // 3 per row
  float4* ss = dv + 3 * cap;                  // SINGLE: s = A p
  float4* mss = ss + (SINGLE ? cap : 0);      // SINGLE: M s (published for the gathers)
  // The 4-byte planes (a2, column indices) hold cap_blocks + 4 words rounded up to 16 bytes: block kb0 + k sits at
  // word (kb0 & 3) + k, so that a bulk copy starting at the 16-byte boundary below kb0 lands on a 16-byte boundary.
  const int cw = MSMEM ? pcg_word_plane(a.cap_blocks) : 0, sh = kb0 & 3;
  float4* m0s = mss + (SINGLE ? cap : 0);
  float4* m1s = m0s + (MSMEM ? a.cap_blocks : 0);
  float* m8b = reinterpret_cast<float*>(m1s + (MSMEM ? a.cap_blocks : 0));
  int* colb = reinterpret_cast<int*>(m8b + cw);
  int* rp = colb + cw;  // n + 1 local row offsets
  float* m8s = m8b + sh;
  int* cols = colb + sh;

  // ---- stage the CTA's rows: one bulk copy (TMA, cp.async.bulk) per plane, completing on an mbarrier. The a0/a1
  // planes are 16-byte blocks; the 4-byte planes copy whole 16-byte words from the boundary at or below kb0 and
  // load the last (s + nb) % 4 words plainly. Without 16-byte aligned planes the rows are loaded plainly.
  __shared__ __align__(8) unsigned long long stage_bar;
  const bool bulk = MSMEM && a.bulk && nb > 0;
  const unsigned bar = smem_addr(&stage_bar);
  const int words = (sh + nb) & ~3;  // words of each 4-byte plane the bulk copy moves
  if (bulk && threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_proxy_async_shared();
    mbar_arrive_expect_tx(bar, 32u * unsigned(nb) + 8u * unsigned(words));
    bulk_copy_g2s(smem_addr(m0s), a.A.a0 + kb0, 16u * unsigned(nb), bar);
    bulk_copy_g2s(smem_addr(m1s), a.A.a1 + kb0, 16u * unsigned(nb), bar);
    if (words > 0) {
      bulk_copy_g2s(smem_addr(m8b), a.A.a2 + (kb0 - sh), 4u * unsigned(words), bar);
      bulk_copy_g2s(smem_addr(colb), a.col_idx + (kb0 - sh), 4u * unsigned(words), bar);
    }
  }
  for (int i = threadIdx.x; i <= n; i += blockDim.x) rp[i] = a.row_ptr[r0 + i] - kb0;
  if (bulk) {
    for (int j = words + threadIdx.x; j < sh + nb; j += blockDim.x) {
      m8b[j] = a.A.a2[kb0 - sh + j];
      colb[j] = a.col_idx[kb0 - sh + j];
    }
  } else if (MSMEM) {
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
      m0s[k] = a.A.a0[kb0 + k];
      m1s[k] = a.A.a1[kb0 + k];
      m8s[k] = a.A.a2[kb0 + k];
      cols[k] = a.col_idx[kb0 + k];
    }
  }
  __syncthreads();
  if (bulk) {
    // Every thread waits for the copies' bytes (phase 0 of the barrier), at most spin_limit cycles. A CTA whose
    // copies did not land sets the error flag, waits once more for them to drain and returns; the other CTAs then
    // give up at their first reduce barrier.
    const bool landed = mbar_wait_parity(bar, 0, a.spin_limit);
    if (__syncthreads_or(!landed)) {
      if (threadIdx.x == 0) atomicExch(a.error, 1);
      mbar_wait_parity(bar, 0, a.spin_limit);
      return;
    }
  }
  // ---- setup: D^-1 (adjugate, pcg.rs:479-492), x = 0, r = b, z = D^-1 r, p = z; partial r.z, r.r
  float acc[2] = {0.0f, 0.0f};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int k = a.diag_pos[r0 + i];
    const float4 m0 = a.A.a0[k], m1 = a.A.a1[k];
    const float m8 = a.A.a2[k];
    const float A_ = m0.x, B_ = m0.y, C_ = m0.z, D_ = m0.w, E_ = m1.x, F_ = m1.y, G_ = m1.z, H_ = m1.w, I_ = m8;
    const float c00 = E_ * I_ - F_ * H_, c01 = C_ * H_ - B_ * I_, c02 = B_ * F_ - C_ * E_;
    const float c10 = F_ * G_ - D_ * I_, c11 = A_ * I_ - C_ * G_, c12 = C_ * D_ - A_ * F_;
    const float c20 = D_ * H_ - E_ * G_, c21 = B_ * G_ - A_ * H_, c22 = A_ * E_ - B_ * D_;
    const float det = A_ * c00 + B_ * c10 + C_ * c20;
    const float4 d0 = f4(c00 / det, c01 / det, c02 / det), d1 = f4(c10 / det, c11 / det, c12 / det),
                 d2 = f4(c20 / det, c21 / det, c22 / det);
    dv[3 * i] = d0;
    dv[3 * i + 1] = d1;
    dv[3 * i + 2] = d2;
    const float4 b = a.b[r0 + i];
    const float4 z = f4(dot3(d0, b), dot3(d1, b), dot3(d2, b));
    bs[i] = b;
    xs[i] = f4(0.f, 0.f, 0.f);
    rs[i] = b;
    zs[i] = z;
    ps[i] = SINGLE ? f4(0.f, 0.f, 0.f) : z;  // SINGLE: p, s, ms of iteration -1 are zero (beta_0 = 0)
    if (SINGLE) ss[i] = mss[i] = f4(0.f, 0.f, 0.f);
    a.p0[r0 + i] = z;                         // SINGLE: u_0, read by iteration 0's gathers
    acc[0] += dot3(b, z);
    acc[1] += dot3(b, b);
  }
  float tot[2];
  cta_sum<2>(acc, tot);
  unsigned gen = 1;
  if (!reduce_barrier<2>(a, gen++, tot)) return;
  float rz = tot[0], rr = tot[1];
  const float rr0 = rr;
  int status = rr <= 0.0f ? kPcgConverged : kPcgRunning;
  int it = 0, cur = 0, replacements = 0;
  bool fused = false;
  float beta = 0.0f, alpha = 0.0f, pq = 0.0f;
  const int passes = (n + groups - 1) / groups;
  long long tm[7] = {0, 0, 0, 0, 0, 0, 0};

  if constexpr (SINGLE) {
    float gamma = rz;  // gamma of the previous iteration
    for (int k = 0; status == kPcgRunning; ++k) {
      const long long t_a0 = clock64();
      const int rd = k & 1;  // read the buffers of parity k & 1, write the other
      // own rows to iteration k (alpha, beta of iteration k - 1)
      if (k > 0)
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
          const float4 sv = fma4(beta, ss[i], qs[i]), pv = fma4(beta, ps[i], zs[i]);
          const float4 r = fma4(-alpha, sv, rs[i]);
          ss[i] = sv;
          ps[i] = pv;
          xs[i] = fma4(alpha, pv, xs[i]);
          rs[i] = r;
          zs[i] = f4(dot3(dv[3 * i], r), dot3(dv[3 * i + 1], r), dot3(dv[3 * i + 2], r));
          mss[i] = f4(dot3(dv[3 * i], sv), dot3(dv[3 * i + 1], sv), dot3(dv[3 * i + 2], sv));
        }
      __syncthreads();
      // w = A u; u of each gathered column from its published u, mw, ms (iteration k - 1)
      const float4* Ur = rd ? a.p1 : a.p0;
      const float4* MWr = rd ? a.mw[1] : a.mw[0];
      const float4* MSr = rd ? a.ms[1] : a.ms[0];
      float4* Uw = rd ? a.p0 : a.p1;
      float4* MWw = rd ? a.mw[0] : a.mw[1];
      float4* MSw = rd ? a.ms[0] : a.ms[1];
      float part[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
      for (int pass = 0; pass < passes; ++pass) {
        const int i = pass * groups + group;
        const bool active = i < n;
        float y0 = 0.f, y1 = 0.f, y2 = 0.f;
        const int kb = active ? rp[i] : 0, ke = active ? rp[i + 1] : 0;
        for (int kk = kb + gl; kk < ke; kk += LPR) {
          const int c = MSMEM ? cols[kk] : __ldg(a.col_idx + kb0 + kk);
          float4 uc = __ldcg(Ur + c);
          if (k > 0) uc = fma4(-alpha, fma4(beta, __ldcg(MSr + c), __ldcg(MWr + c)), uc);
          if (MSMEM)
            apply(m0s[kk], m1s[kk], m8s[kk], uc, y0, y1, y2);
          else
            apply(__ldg(a.A.a0 + kb0 + kk), __ldg(a.A.a1 + kb0 + kk), __ldg(a.A.a2 + kb0 + kk), uc, y0, y1, y2);
        }
        group_reduce<LPR>(y0, y1, y2);
        if (active && gl == 0) {
          const float4 w = f4(y0, y1, y2), u = zs[i], r = rs[i];
          const float4 mw = f4(dot3(dv[3 * i], w), dot3(dv[3 * i + 1], w), dot3(dv[3 * i + 2], w));
          qs[i] = w;
          Uw[r0 + i] = u;
          MWw[r0 + i] = mw;
          MSw[r0 + i] = mss[i];
          const float4 pv = ps[i], sv = ss[i];  // p, s of iteration k - 1 (zero at k = 0)
          part[0] += dot3(r, u);
          part[1] += dot3(w, u);
          part[2] += dot3(r, r);
          part[3] += dot3(u, sv) + dot3(pv, w);
          part[4] += dot3(pv, sv);
        }
      }
      float t3[5];
      const long long t_a1 = clock64();
      cta_sum<5>(part, t3);
      const long long t_a2 = clock64();
      if (!reduce_barrier<5, 5>(a, gen++, t3)) return;
      if (a.timing && cta == 0 && threadIdx.x == 0) {
        tm[0] += t_a1 - t_a0;
        tm[1] += t_a2 - t_a1;
        tm[2] += clock64() - t_a2;
        tm[6] += 1;
      }
      const float g = t3[0], d = t3[1];
      rr = t3[2];
      it = k;
      if (k > 0 && rr <= a.tol2 * rr0) {
        status = kPcgConverged;
        break;
      }
      if (k >= a.max_iterations) {
        status = kPcgIterationLimit;
        break;
      }
      beta = k == 0 ? 0.0f : g / gamma;
      // p.A p of the coming direction p = u + beta p_old, expanded over the dots of this phase (no conjugacy or
      // orthogonality assumed, unlike the textbook delta - beta gamma / alpha, which loses p.A p in f32)
      pq = d + beta * t3[3] + beta * beta * t3[4];
      if (!(pq > 0.0f) || !isfinite(pq) || !isfinite(beta)) {
        status = kPcgBreakdown;
        break;
      }
      alpha = g / pq;
      gamma = g;
      rz = g;
    }
  } else
  while (status == kPcgRunning) {
    // ---- phase A: p (fused update), q = A p, partial p.q
    long long t_a0 = clock64();
    const float4* pold = cur ? a.p1 : a.p0;
    float4* pnew = cur ? a.p0 : a.p1;
    float pq_l[1] = {0.0f};
    for (int pass = 0; pass < passes; ++pass) {
      const int i = pass * groups + group;
      const bool active = i < n;
      float y0 = 0.f, y1 = 0.f, y2 = 0.f;
      const int kb = active ? rp[i] : 0, ke = active ? rp[i + 1] : 0;
      // The lane's first two blocks: both column gathers are issued before either is used (one L2 round trip).
      const int k0 = kb + gl, k1 = k0 + LPR;
      const int c0 = k0 < ke ? (MSMEM ? cols[k0] : __ldg(a.col_idx + kb0 + k0)) : -1;
      const int c1 = k1 < ke ? (MSMEM ? cols[k1] : __ldg(a.col_idx + kb0 + k1)) : -1;
      float4 p0c = make_float4(0.f, 0.f, 0.f, 0.f), p1c = p0c, z0c = p0c, z1c = p0c;
      if (c0 >= 0) p0c = __ldcg(pold + c0);
      if (c1 >= 0) p1c = __ldcg(pold + c1);
      if (fused && c0 >= 0) z0c = __ldcg(a.z + c0);
      if (fused && c1 >= 0) z1c = __ldcg(a.z + c1);
      if (fused) {
        p0c = f4(z0c.x + beta * p0c.x, z0c.y + beta * p0c.y, z0c.z + beta * p0c.z);
        p1c = f4(z1c.x + beta * p1c.x, z1c.y + beta * p1c.y, z1c.z + beta * p1c.z);
      }
      if (c0 >= 0) {
        if (MSMEM)
          apply(m0s[k0], m1s[k0], m8s[k0], p0c, y0, y1, y2);
        else
          apply(__ldg(a.A.a0 + kb0 + k0), __ldg(a.A.a1 + kb0 + k0), __ldg(a.A.a2 + kb0 + k0), p0c, y0, y1, y2);
      }
      if (c1 >= 0) {
        if (MSMEM)
          apply(m0s[k1], m1s[k1], m8s[k1], p1c, y0, y1, y2);
        else
          apply(__ldg(a.A.a0 + kb0 + k1), __ldg(a.A.a1 + kb0 + k1), __ldg(a.A.a2 + kb0 + k1), p1c, y0, y1, y2);
      }
      for (int k = k1 + LPR; k < ke; k += LPR) {
        const int c = MSMEM ? cols[k] : __ldg(a.col_idx + kb0 + k);
        float4 pc = __ldcg(pold + c);
        if (fused) {
          const float4 zc = __ldcg(a.z + c);
          pc = f4(zc.x + beta * pc.x, zc.y + beta * pc.y, zc.z + beta * pc.z);
        }
        if (MSMEM)
          apply(m0s[k], m1s[k], m8s[k], pc, y0, y1, y2);
        else
          apply(__ldg(a.A.a0 + kb0 + k), __ldg(a.A.a1 + kb0 + k), __ldg(a.A.a2 + kb0 + k), pc, y0, y1, y2);
      }
      group_reduce<LPR>(y0, y1, y2);
      if (active && gl == 0) {
        float4 p = ps[i];
        if (fused) {
          const float4 z = zs[i];
          p = f4(z.x + beta * p.x, z.y + beta * p.y, z.z + beta * p.z);
          ps[i] = p;
          pnew[r0 + i] = p;
        }
        const float4 q = f4(y0, y1, y2);
        qs[i] = q;
        pq_l[0] += dot3(p, q);
      }
    }
    float t1[1];
    const long long t_a1 = clock64();
    cta_sum<1>(pq_l, t1);
    const long long t_a2 = clock64();
    if (!reduce_barrier<1>(a, gen++, t1)) return;
    const long long t_a3 = clock64();
    pq = t1[0];
    if (!(pq > 0.0f) || !isfinite(pq)) {
      status = kPcgBreakdown;
      break;
    }
    if (fused) cur ^= 1;
    alpha = rz / pq;
    // ---- phase B: x, r, z in shared memory; publish z; partial r.z, r.r
    acc[0] = acc[1] = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const float4 p = ps[i], q = qs[i];
      float4 x = xs[i], r = rs[i];
      x = f4(x.x + alpha * p.x, x.y + alpha * p.y, x.z + alpha * p.z);
      r = f4(r.x - alpha * q.x, r.y - alpha * q.y, r.z - alpha * q.z);
      const float4 z = f4(dot3(dv[3 * i], r), dot3(dv[3 * i + 1], r), dot3(dv[3 * i + 2], r));
      xs[i] = x;
      rs[i] = r;
      zs[i] = z;
      a.z[r0 + i] = z;
      acc[0] += dot3(r, z);
      acc[1] += dot3(r, r);
    }
    const long long t_b1 = clock64();
    cta_sum<2>(acc, tot);
    const long long t_b2 = clock64();
    if (!reduce_barrier<2>(a, gen++, tot)) return;
    if (a.timing && cta == 0 && threadIdx.x == 0) {
      const long long t_b3 = clock64();
      tm[0] += t_a1 - t_a0;
      tm[1] += t_a2 - t_a1;
      tm[2] += t_a3 - t_a2;
      tm[3] += t_b1 - t_a3;
      tm[4] += t_b2 - t_b1;
      tm[5] += t_b3 - t_b2;
      tm[6] += 1;
    }
    const float rz_new = tot[0];
    rr = tot[1];
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
      // Keep the direction (p = z + beta p_old, published), publish x, then r = b - A x and z = D^-1 r.
      float4* pn = cur ? a.p0 : a.p1;
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 z = zs[i], p = ps[i];
        const float4 np = f4(z.x + beta * p.x, z.y + beta * p.y, z.z + beta * p.z);
        ps[i] = np;
        pn[r0 + i] = np;
        a.x[r0 + i] = xs[i];
      }
      cur ^= 1;
      fused = false;
      float none[1] = {0.0f};
      __syncthreads();
      if (!reduce_barrier<1>(a, gen++, none)) return;
      acc[0] = acc[1] = 0.0f;
      for (int pass = 0; pass < passes; ++pass) {
        const int i = pass * groups + group;
        const bool active = i < n;
        float y0 = 0.f, y1 = 0.f, y2 = 0.f;
        const int kb = active ? rp[i] : 0, ke = active ? rp[i + 1] : 0;
        for (int k = kb + gl; k < ke; k += LPR) {
          const int c = MSMEM ? cols[k] : __ldg(a.col_idx + kb0 + k);
          const float4 xc = __ldcg(a.x + c);
          if (MSMEM)
            apply(m0s[k], m1s[k], m8s[k], xc, y0, y1, y2);
          else
            apply(__ldg(a.A.a0 + kb0 + k), __ldg(a.A.a1 + kb0 + k), __ldg(a.A.a2 + kb0 + k), xc, y0, y1, y2);
        }
        group_reduce<LPR>(y0, y1, y2);
        if (active && gl == 0) {
          const float4 b = bs[i];
          const float4 r = f4(b.x - y0, b.y - y1, b.z - y2);
          const float4 z = f4(dot3(dv[3 * i], r), dot3(dv[3 * i + 1], r), dot3(dv[3 * i + 2], r));
          rs[i] = r;
          zs[i] = z;
          a.z[r0 + i] = z;
          acc[0] += dot3(r, z);
          acc[1] += dot3(r, r);
        }
      }
      cta_sum<2>(acc, tot);
      if (!reduce_barrier<2>(a, gen++, tot)) return;
      rz = tot[0];
      rr = tot[1];
      ++replacements;
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) a.x[r0 + i] = xs[i];
  if (a.timing && cta == 0 && threadIdx.x == 0)
    for (int k = 0; k < 7; ++k) a.timing[k] += tm[k];
  if (cta == 0 && threadIdx.x == 0) {
    PcgState* st = a.state;
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

__device__ __forceinline__ void block_apply(const DevBsr& A, int k, float4 p, float& y0, float& y1, float& y2) {
  apply(__ldg(A.a0 + k), __ldg(A.a1 + k), __ldg(A.a2 + k), p, y0, y1, y2);
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
    for (int k = kb + gl; k < ke; k += LPR) block_apply(A, k, __ldg(p + __ldg(col_idx + k)), y0, y1, y2);
    group_reduce<LPR>(y0, y1, y2);
    if (active && gl == 0) y[row] = f4(y0, y1, y2);
  }
}

// r = b64 - A d computed in f64 from the f32 blocks; one 8-lane group per row.
__global__ void __launch_bounds__(256) refine_residual_kernel(int R, const int* row_ptr, const int* col_idx, DevBsr A,
                                                              const double* g, const float4* d, float4* r_out,
                                                              double* partial) {
  __shared__ double red[32];
  const int gl = threadIdx.x & 7;
  double s = 0.0;
  const int groups = blockDim.x >> 3;
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
      // g is the f64 gradient; the right-hand side is -g.
      const double r0 = -g[3 * row] - y0, r1 = -g[3 * row + 1] - y1, r2 = -g[3 * row + 2] - y2;
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

const void* pcg_fn(int lpr, bool msmem, bool single) {
#define DRAPE_PCG_FN(L, M, S) \
  if (lpr == L && msmem == M && single == S) return reinterpret_cast<const void*>(&pcg_kernel<L, M, S>);
  DRAPE_PCG_FN(4, true, false) DRAPE_PCG_FN(8, true, false) DRAPE_PCG_FN(16, true, false)
  DRAPE_PCG_FN(4, false, false) DRAPE_PCG_FN(8, false, false) DRAPE_PCG_FN(16, false, false)
  DRAPE_PCG_FN(4, true, true) DRAPE_PCG_FN(8, true, true) DRAPE_PCG_FN(16, true, true)
  DRAPE_PCG_FN(4, false, true) DRAPE_PCG_FN(8, false, true) DRAPE_PCG_FN(16, false, true)
#undef DRAPE_PCG_FN
  return nullptr;
}

// Raises the kernel's dynamic shared-memory ceiling to all that the device allows beside the kernel's static shared
// memory. The ceiling is one setting per kernel for the whole process: setting it to this fixed value, rather than
// to each launch's own size, keeps host threads that launch the kernel concurrently for drapes of different sizes
// from lowering it between another thread's set and launch.
cudaError_t allow_dynamic_smem(const void* fn) {
  int dev = 0, optin = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
  cudaFuncAttributes fa{};
  if ((e = cudaFuncGetAttributes(&fa, fn)) != cudaSuccess) return e;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - int(fa.sharedSizeBytes));
}

}  // namespace

size_t pcg_smem_bytes(int cap_rows, int cap_blocks, bool msmem, bool single) {
  return size_t(cap_rows) * ((single ? 8 : 6) * 16 + 3 * 16) +
         (msmem ? size_t(cap_blocks) * (16 + 16) + size_t(pcg_word_plane(cap_blocks)) * (4 + 4) : 0) +
         size_t(cap_rows + 1) * 4;
}

int pcg_max_grid(int threads, int lanes_per_row, size_t smem, bool msmem, bool single) {
  const void* fn = pcg_fn(lanes_per_row, msmem, single);
  if (!fn) return 0;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (allow_dynamic_smem(fn) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) return 0;
  return sms * per_sm;
}

cudaError_t launch_pcg(const PcgArgs& a, const PcgLaunch& cfg, cudaStream_t s) {
  const void* fn = pcg_fn(cfg.lanes_per_row, cfg.matrix_in_smem, cfg.single_reduction);
  if (cfg.single_reduction && (a.replace_every > 0 || !a.mw[0] || !a.mw[1] || !a.ms[0] || !a.ms[1]))
    return cudaErrorInvalidValue;
  if (!fn || cfg.threads % 32 != 0 || cfg.threads > 1024 || cfg.grid < 1) return cudaErrorInvalidValue;
  cudaError_t e = allow_dynamic_smem(fn);
  if (e != cudaSuccess) return e;
  PcgArgs args = a;
  const auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  args.bulk = cfg.matrix_in_smem && aligned(a.A.a0) && aligned(a.A.a1) && aligned(a.A.a2) && aligned(a.col_idx);
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel(fn, dim3(cfg.grid), dim3(cfg.threads), params, cfg.smem, s);
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
