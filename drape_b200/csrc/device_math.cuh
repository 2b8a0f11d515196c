// Device-side element math of the drape energy (f64 unless stated):
//   membrane CST with StVK stress (membrane.rs:26-101; its stress-clamped PSD Hessian, membrane.rs:116-140),
//   dihedral hinge with Bridson's gradient and the Gauss-Newton Hessian (hinge.rs:13-61, 94-106),
//   IPC log barrier against planes and spheres (contact.rs:14-101) and the CCD step bound (contact.rs:40-77).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace drape {
namespace dev {

struct V3 {
  double x, y, z;
};
__device__ __forceinline__ V3 v3(double a, double b, double c) { return {a, b, c}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3 load3(const double* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ double comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// Membrane constants (N/m): wale, course, coupling, shear.
struct Membrane {
  double wale, course, coupling, shear;
};

struct TriGeom {
  double g[3][2];  // dN_k/dX_(wale, course)
  double area;
};
__device__ __forceinline__ TriGeom load_geom(const double* geom, int t) {
  const double* o = geom + 7 * (size_t)t;
  TriGeom g;
  g.g[0][0] = o[0];
  g.g[0][1] = o[1];
  g.g[1][0] = o[2];
  g.g[1][1] = o[3];
  g.g[2][0] = o[4];
  g.g[2][1] = o[5];
  g.area = o[6];
  return g;
}

// Deformation columns F_w, F_c of the triangle x0, x1, x2.
__device__ __forceinline__ void columns(const TriGeom& G, V3 x0, V3 x1, V3 x2, V3& fw, V3& fc) {
  V3 e1 = x1 - x0, e2 = x2 - x0;
  fw = e1 * G.g[1][0] + e2 * G.g[2][0];
  fc = e1 * G.g[1][1] + e2 * G.g[2][1];
}

__device__ __forceinline__ void stress_of(const Membrane& m, V3 fw, V3 fc, double s[3]) {
  double eww = 0.5 * (dot(fw, fw) - 1.0), ecc = 0.5 * (dot(fc, fc) - 1.0), ewc = 0.5 * dot(fw, fc);
  s[0] = m.wale * eww + m.coupling * ecc;
  s[1] = m.course * ecc + m.coupling * eww;
  s[2] = 2.0 * m.shear * ewc;
}

// Positive part of the 2x2 stress [[a, b], [b, c]]: keeps the geometric stiffness PSD.
__device__ __forceinline__ void clamp_stress(double s[3]) {
  double a = s[0], c = s[1], b = s[2];
  double mean = 0.5 * (a + c), radius = sqrt(0.25 * (a - c) * (a - c) + b * b);
  double hi = mean + radius, lo = mean - radius;
  if (lo >= 0.0) return;
  if (hi <= 0.0) {
    s[0] = s[1] = s[2] = 0.0;
    return;
  }
  double p0 = b, p1 = hi - a, q0 = hi - c, q1 = b;
  double lp = hypot(p0, p1), lq = hypot(q0, q1);
  double v0, v1;
  if (lp >= lq) {
    v0 = p0;
    v1 = p1;
  } else {
    v0 = q0;
    v1 = q1;
  }
  double len = lp >= lq ? lp : lq;
  if (len == 0.0) {
    v0 = a >= c ? 1.0 : 0.0;
    v1 = a >= c ? 0.0 : 1.0;
  } else {
    v0 /= len;
    v1 /= len;
  }
  s[0] = hi * v0 * v0;
  s[1] = hi * v1 * v1;
  s[2] = hi * v0 * v1;
}

// Gradient of the membrane energy at local vertex k.
__device__ __forceinline__ V3 membrane_gradient_row(const Membrane& m, const TriGeom& G, V3 fw, V3 fc, int k) {
  double s[3];
  stress_of(m, fw, fc, s);
  V3 pw = fw * s[0] + fc * s[2], pc = fw * s[2] + fc * s[1];
  return (pw * G.g[k][0] + pc * G.g[k][1]) * G.area;
}

// Row k of the membrane Hessian: blocks (k, l) for l = 0..2, row-major 3x3 each. `clamp` projects the stress
// onto its positive part (PSD, membrane.rs:54-57); otherwise this is the exact tangent (membrane.rs:59-62).
__device__ __forceinline__ void membrane_hessian_row(const Membrane& m, const TriGeom& G, V3 fw, V3 fc, int k,
                                                     double out[3][9], bool clamp) {
  double s[3];
  stress_of(m, fw, fc, s);
  if (clamp) clamp_stress(s);
  V3 bw[3], bc[3], bs[3];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    bw[l] = fw * G.g[l][0];
    bc[l] = fc * G.g[l][1];
    bs[l] = (fw * G.g[l][1] + fc * G.g[l][0]) * 0.5;
  }
  const double gkx = G.g[k][0], gky = G.g[k][1];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    double geo = gkx * (s[0] * G.g[l][0] + s[2] * G.g[l][1]) + gky * (s[2] * G.g[l][0] + s[1] * G.g[l][1]);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double wk = comp(bw[k], r), ck = comp(bc[k], r), sk = comp(bs[k], r);
        double wl = comp(bw[l], c), cl = comp(bc[l], c), sl = comp(bs[l], c);
        double v = m.wale * wk * wl + m.course * ck * cl + m.coupling * (wk * cl + ck * wl) + 4.0 * m.shear * sk * sl;
        if (r == c) v += geo;
        out[l][3 * r + c] = v * G.area;
      }
  }
}

// W(x + a d) - W(x) = S:dE + W(dE), exact for StVK (membrane.rs:66-78).
__device__ __forceinline__ double membrane_energy_change(const Membrane& m, const TriGeom& G, V3 fw, V3 fc, V3 dw,
                                                         V3 dc) {
  double ch0 = dot(fw, dw) + 0.5 * dot(dw, dw), ch1 = dot(fc, dc) + 0.5 * dot(dc, dc);
  double ch2 = 0.5 * (dot(fw, dc) + dot(dw, fc) + dot(dw, dc));
  double s[3];
  stress_of(m, fw, fc, s);
  double first = s[0] * ch0 + s[1] * ch1 + 2.0 * s[2] * ch2;
  double w = 0.5 * m.wale * ch0 * ch0 + 0.5 * m.course * ch1 * ch1 + m.coupling * ch0 * ch1 + 2.0 * m.shear * ch2 * ch2;
  return G.area * (first + w);
}

__device__ __forceinline__ double membrane_energy(const Membrane& m, const TriGeom& G, V3 fw, V3 fc) {
  double e0 = 0.5 * (dot(fw, fw) - 1.0), e1 = 0.5 * (dot(fc, fc) - 1.0), e2 = 0.5 * dot(fw, fc);
  return G.area * (0.5 * m.wale * e0 * e0 + 0.5 * m.course * e1 * e1 + m.coupling * e0 * e1 + 2.0 * m.shear * e2 * e2);
}

// Dihedral angle of the hinge [x1 left opposite, x2 right opposite, x3 edge start, x4 edge end].
__device__ __forceinline__ double hinge_angle(V3 x1, V3 x2, V3 x3, V3 x4) {
  V3 e = x4 - x3;
  V3 n1 = cross(x1 - x3, x1 - x4), n2 = cross(x2 - x4, x2 - x3);
  V3 u1 = n1 * (1.0 / sqrt(dot(n1, n1))), u2 = n2 * (1.0 / sqrt(dot(n2, n2)));
  double sine = dot(cross(u1, u2), e * (1.0 / sqrt(dot(e, e))));
  return atan2(sine, dot(u1, u2));
}

// d theta / d x_k for k = 0..3 (Bridson et al. bending modes).
__device__ __forceinline__ void hinge_angle_gradient(V3 x1, V3 x2, V3 x3, V3 x4, V3 g[4]) {
  V3 e = x4 - x3;
  double len = sqrt(dot(e, e));
  V3 n1 = cross(x1 - x3, x1 - x4), n2 = cross(x2 - x4, x2 - x3);
  V3 a1 = n1 * (1.0 / dot(n1, n1)), a2 = n2 * (1.0 / dot(n2, n2));
  g[0] = a1 * (-len);
  g[1] = a2 * (-len);
  g[2] = (a1 * (dot(x1 - x4, e) / len) + a2 * (dot(x2 - x4, e) / len)) * -1.0;
  g[3] = (a1 * (dot(x1 - x3, e) / len) + a2 * (dot(x2 - x3, e) / len));
}

// Forward-mode dual numbers (value, derivative along one seed direction): differentiating the analytic
// gradient with them gives the exact Hessian column without new formulas (dual.rs:6-90, hinge.rs:66-82).
struct Dual {
  double v, t;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.t + b.t}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.t - b.t}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.t * b.v + a.v * b.t}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.t * b.v - a.v * b.t) / (b.v * b.v)}; }
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const double s = sqrt(a.v);
  return {s, a.t / (2.0 * s)};
}
struct DV3 {
  Dual x, y, z;
};
__device__ __forceinline__ DV3 operator-(DV3 a, DV3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ DV3 operator+(DV3 a, DV3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ DV3 operator*(DV3 a, Dual s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ Dual ddot(DV3 a, DV3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ DV3 dcross(DV3 a, DV3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Component k of d theta / dx in dual arithmetic (the same formula as hinge_angle_gradient).
__device__ __forceinline__ DV3 hinge_angle_gradient_dual(DV3 x1, DV3 x2, DV3 x3, DV3 x4, int k) {
  const DV3 e = x4 - x3;
  const Dual len = dsqrt(ddot(e, e));
  const DV3 n1 = dcross(x1 - x3, x1 - x4), n2 = dcross(x2 - x4, x2 - x3);
  const Dual one{1.0, 0.0}, mone{-1.0, 0.0};
  const DV3 a1 = n1 * (one / ddot(n1, n1)), a2 = n2 * (one / ddot(n2, n2));
  if (k == 0) return a1 * (mone * len);
  if (k == 1) return a2 * (mone * len);
  if (k == 2) return (a1 * (ddot(x1 - x4, e) / len) + a2 * (ddot(x2 - x4, e) / len)) * mone;
  return a1 * (ddot(x1 - x3, e) / len) + a2 * (ddot(x2 - x3, e) / len);
}

// Row k of the exact hinge Hessian 2c (grad theta grad theta^T + theta d2 theta): blocks (k, l), l = 0..3.
__device__ __forceinline__ void hinge_exact_hessian_row(const V3 x[4], const V3 dg[4], double theta, double c2, int k,
                                                        double out[4][9]) {
#pragma unroll 1
  for (int l = 0; l < 4; ++l)
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      DV3 p[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const double sx = (m == l && c == 0) ? 1.0 : 0.0, sy = (m == l && c == 1) ? 1.0 : 0.0,
                     sz = (m == l && c == 2) ? 1.0 : 0.0;
        p[m] = {{x[m].x, sx}, {x[m].y, sy}, {x[m].z, sz}};
      }
      const DV3 col = hinge_angle_gradient_dual(p[0], p[1], p[2], p[3], k);
      const double h[3] = {col.x.t, col.y.t, col.z.t};
#pragma unroll
      for (int r = 0; r < 3; ++r) out[l][3 * r + c] = c2 * (comp(dg[k], r) * comp(dg[l], c) + theta * h[r]);
    }
}

// Barrier b(d) = -kappa (d - dhat)^2 ln(d / dhat) on 0 < d < dhat, and its first two derivatives.
struct Barrier {
  double dhat, kappa;
  __device__ __forceinline__ double value(double d) const {
    if (d >= dhat) return 0.0;
    if (d <= 0.0) return INFINITY;
    double t = d - dhat;
    return -kappa * t * t * log(d / dhat);
  }
  __device__ __forceinline__ double first(double d) const {
    if (d >= dhat) return 0.0;
    double t = d - dhat;
    return -kappa * (2.0 * t * log(d / dhat) + t * t / d);
  }
  __device__ __forceinline__ double second(double d) const {
    if (d >= dhat) return 0.0;
    double t = d - dhat;
    return -kappa * (2.0 * log(d / dhat) + 4.0 * t / d - t * t / (d * d));
  }
};

// Colliders packed 8 doubles each: kind (1 plane n.x = w, 2 sphere |x - c| = w), a, b, c, w, 0, 0, 0.
struct Proximity {
  double distance;
  V3 normal;
  double curvature;
};
__device__ __forceinline__ Proximity proximity(const double* col, V3 x) {
  V3 a = v3(col[1], col[2], col[3]);
  if (col[0] == 1.0) return {dot(a, x) - col[4], a, 0.0};
  V3 q = x - a;
  double len = sqrt(dot(q, q));
  return {len - col[4], q * (1.0 / len), 1.0 / len};
}

// Largest alpha in (0, 1] with d(x + alpha p) >= 0.1 d(x) (contact.rs:40-77).
__device__ __forceinline__ double collider_max_step(const double* col, V3 x, V3 p) {
  const double keep = 0.1;
  V3 a = v3(col[1], col[2], col[3]);
  if (col[0] == 1.0) {
    double d0 = dot(a, x) - col[4], rate = dot(a, p);
    double s = rate >= 0.0 ? 1.0 : (1.0 - keep) * d0 / -rate;
    return s < 1.0 ? s : 1.0;
  }
  V3 q = x - a;
  double lq = sqrt(dot(q, q)), d0 = lq - col[4];
  double A = dot(p, p), B = 2.0 * dot(q, p), target = col[4] + keep * d0;
  double C = (1.0 - keep) * d0 * (lq + target);
  double disc = B * B - 4.0 * A * C;
  if (B >= 0.0 || disc < 0.0) return 1.0;
  double s = 2.0 * C / (-B + sqrt(disc));
  return s < 1.0 ? s : 1.0;
}

}  // namespace dev
}  // namespace drape
