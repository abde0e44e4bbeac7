// Device-side math of the cloth solver: float3 helpers, 3x3 blocks, the energy terms (row-wise derivatives in FP32,
// energies in FP64), the collision field and the post-solve push-out.
//
// The term formulas restate the reference's double-precision math (libs/sim/src/energies.cpp:11-110, stretch.hpp:15-49,
// bending.hpp:29-51), organised for the assembly: a term's derivative record once, then any vertex's gradient and
// Hessian blocks. The collision-field sampling uses explicitly rounded IEEE operations in the reference's FP32 order
// (libs/sim/kernels/term_math.h:203-243 restating collision_field.cpp:8-41) so that the contact-candidate decisions
// (phi < r + reach, |grad| < 1e-4) are bit-identical to the reference's 32-bit path on identical inputs.
#pragma once

#include <cstdint>

namespace dcu {

// ---------------------------------------------------------------------------------------------------------------
// float3 / 3x3.

__device__ __forceinline__ float3 mk(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float4 f4(float3 a, float w = 0.0f) { return make_float4(a.x, a.y, a.z, w); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3& operator+=(float3& a, float3 b) {
  a = a + b;
  return a;
}
__device__ __forceinline__ float3& operator-=(float3& a, float3 b) {
  a = a - b;
  return a;
}
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 div(float3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }

// Row-major 3x3.
struct M3 {
  float m[9];
};
__device__ __forceinline__ void zero(M3& a) {
#pragma unroll
  for (int k = 0; k < 9; ++k) a.m[k] = 0.0f;
}
// a += s * u v^T
__device__ __forceinline__ void addOuter(M3& a, float s, float3 u, float3 v) {
  const float su[3] = {s * u.x, s * u.y, s * u.z};
  const float vv[3] = {v.x, v.y, v.z};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) a.m[3 * i + j] += su[i] * vv[j];
}
// a += s * (I - n n^T)
__device__ __forceinline__ void addProjector(M3& a, float s, float3 n) {
  const float nn[3] = {n.x, n.y, n.z};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) a.m[3 * i + j] += s * ((i == j ? 1.0f : 0.0f) - nn[i] * nn[j]);
}
__device__ __forceinline__ float3 mul(const M3& a, float3 v) {
  return mk(a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z, a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
            a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z);
}

// Inverse of a symmetric positive-definite block by an unpivoted LDL^T factorisation of its lower triangle; ok is
// false (and the identity returned) when a pivot is not positive. The reference's block-Jacobi preconditioner
// inverts each diagonal block (cpu_solver.cpp:171-178; 32-bit path term_math.h:285-312) with the identity as fallback.
__device__ inline M3 invertSpd(const M3& A, bool& ok) {
  M3 out;
  zero(out);
  out.m[0] = out.m[4] = out.m[8] = 1.0f;
  ok = false;
  const float a00 = A.m[0], a10 = A.m[3], a20 = A.m[6], a11 = A.m[4], a21 = A.m[7], a22 = A.m[8];
  const float d0 = a00;
  if (!(d0 > 0.0f)) return out;
  const float l10 = a10 / d0, l20 = a20 / d0;
  const float d1 = a11 - l10 * l10 * d0;
  if (!(d1 > 0.0f)) return out;
  const float l21 = (a21 - l20 * l10 * d0) / d1;
  const float d2 = a22 - l20 * l20 * d0 - l21 * l21 * d1;
  if (!(d2 > 0.0f)) return out;
  ok = true;
  const float i0 = 1.0f / d0, i1 = 1.0f / d1, i2 = 1.0f / d2;
  // A^{-1} = L^{-T} D^{-1} L^{-1}; L^{-1} is unit lower triangular with entries m10, m20, m21.
  const float m10 = -l10, m21 = -l21, m20 = l10 * l21 - l20;
  // column k of A^{-1} = L^{-T} (D^{-1} (L^{-1} e_k))
  const float y[3][3] = {{1.0f, m10, m20}, {0.0f, 1.0f, m21}, {0.0f, 0.0f, 1.0f}};  // y[k] = L^{-1} e_k
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float z0 = y[k][0] * i0, z1 = y[k][1] * i1, z2 = y[k][2] * i2;
    const float x2 = z2;
    const float x1 = z1 - l21 * x2;
    const float x0 = z0 - l10 * x1 - l20 * x2;
    out.m[0 * 3 + k] = x0;
    out.m[1 * 3 + k] = x1;
    out.m[2 * 3 + k] = x2;
  }
  return out;
}

// ---------------------------------------------------------------------------------------------------------------
// Terms, FP32 derivatives for one vertex (row a).

struct StretchIn {
  float4 d;  // dmInv (0,0), (1,0), (0,1), (1,1)
  float area;
  float k[3];      // warp, weft, bias
  float limit[2];  // strain limits warp, weft
  float limitScale;
};

// Coefficient of vertex `k` in f_u (column 0) or f_v (column 1): f = sum_k c_k x_k (energies.cpp:13-18).
__device__ __forceinline__ float coef(float4 d, int column, int k) {
  const float c0 = column == 0 ? d.x : d.z;
  const float c1 = column == 0 ? d.y : d.w;
  return k == 1 ? c0 : (k == 2 ? c1 : -(c0 + c1));
}

// Stretch term (warp |f_u| - 1, weft |f_v| - 1, bias n_u . n_v, each 1/2 K C^2 with K = k area; tension stiffness
// for C > 0 and the one-sided strain limit at limitScale K; energies.cpp:27-62, stretch.hpp:15-49) at x[0..2]
// (relative to vertex 0), in two parts: stretchDerivs evaluates the term once and keeps what every vertex's row needs
// (per direction the unit vector n = f / |f| and the gradient, Gauss-Newton and tension scales; for the bias the
// derivatives of n_u . n_v with respect to f_u and f_v and its scales), and stretchBlockFrom forms any block (a, b)
// of its Hessian and the gradient of vertex a from that record and the term's dmInv coefficients.
struct StretchDer {
  float4 w[6];  // warp: (n, gs), (hs, ts, flags, -); weft: (n, gs), (hs, ts, -, -); bias: (dfu, K c), (dfv, K)
};
constexpr uint32_t kStretchWarp = 1u, kStretchWeft = 2u, kStretchBias = 4u;  // flags: parts that contribute

__device__ inline void stretchDerivs(const StretchIn& t, const float3 x[3], StretchDer& o) {
  const float3 e1 = x[1] - x[0], e2 = x[2] - x[0];
  const float3 fu = e1 * t.d.x + e2 * t.d.y;
  const float3 fv = e1 * t.d.z + e2 * t.d.w;
  const float lu = len(fu), lv = len(fv);
  const float tiny = 1e-12f;
  uint32_t flags = 0;
#pragma unroll
  for (int which = 0; which < 2; ++which) {
    o.w[2 * which] = make_float4(0, 0, 0, 0);
    o.w[2 * which + 1] = make_float4(0, 0, 0, 0);
    if (!(t.k[which] > 0.0f)) continue;
    const float3 f = which == 0 ? fu : fv;
    const float l = which == 0 ? lu : lv;
    if (!(l > tiny)) continue;  // C = 0 and a zero gradient: nothing to add
    const float3 n = div(f, l);
    const float C = l - 1.0f;
    const float K = t.k[which] * t.area;
    float gs = K * C, hs = K;                // gradient and Gauss-Newton scales
    float ts = C > 0.0f ? K * C / l : 0.0f;  // tension scale (addTension with |f| >= 1e-12)
    if (t.limit[which] > 0.0f && C > t.limit[which]) {
      const float KL = t.limitScale * K, ex = C - t.limit[which];
      gs += KL * ex;
      hs += KL;
      if (ex > 0.0f) ts += KL * ex / l;
    }
    o.w[2 * which] = f4(n, gs);
    o.w[2 * which + 1] = make_float4(hs, ts, 0.0f, 0.0f);
    flags |= which == 0 ? kStretchWarp : kStretchWeft;
  }
  o.w[4] = make_float4(0, 0, 0, 0);
  o.w[5] = make_float4(0, 0, 0, 0);
  if (t.k[2] > 0.0f && lu > tiny && lv > tiny) {
    const float3 nu = div(fu, lu), nv = div(fv, lv);
    const float c = dot(nu, nv);
    const float3 dfu = div(nv - nu * c, lu);
    const float3 dfv = div(nu - nv * c, lv);
    const float K = t.k[2] * t.area;
    o.w[4] = f4(dfu, K * c);
    o.w[5] = f4(dfv, K);
    flags |= kStretchBias;
  }
  o.w[1].z = __uint_as_float(flags);
}

// Block (a, b) of a stretch term's Hessian and, with Grad, the gradient of vertex a, read from the term's record in
// global memory: per direction K (grad_a C)(grad_b C)^T plus the tension projector, then the bias part.
template <bool Grad>
__device__ inline void stretchBlockFrom(float4 d, const float4* __restrict__ rec, int a, int b, float3& g, M3& H) {
  zero(H);
  g = mk(0, 0, 0);
  // The whole record in one round of loads (the flags in word 1 then select what is used).
  float4 r[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) r[k] = rec[k];
  const float4 w1 = r[1];
  const uint32_t flags = __float_as_uint(w1.z);
#pragma unroll
  for (int which = 0; which < 2; ++which) {
    if (!(flags & (which == 0 ? kStretchWarp : kStretchWeft))) continue;
    const float4 wn = r[2 * which];
    const float4 ws = which == 0 ? w1 : r[3];
    const float3 n = xyz(wn);
    const float gs = wn.w, hs = ws.x, ts = ws.y;
    const float ca = coef(d, which, a), cb = coef(d, which, b);
    const float3 gra = n * ca, grb = n * cb;
    if (Grad) g += gra * gs;
    addOuter(H, hs, gra, grb);
    if (ts != 0.0f) addProjector(H, ts * ca * cb, n);
  }
  if (flags & kStretchBias) {
    const float4 w4 = r[4], w5 = r[5];
    const float3 dfu = xyz(w4), dfv = xyz(w5);
    const float3 gra = dfu * coef(d, 0, a) + dfv * coef(d, 1, a);
    const float3 grb = dfu * coef(d, 0, b) + dfv * coef(d, 1, b);
    if (Grad) g += gra * w4.w;
    addOuter(H, w5.w, gra, grb);
  }
}

// Dihedral angle theta = atan2((n1 x n2) . e, n1 . n2) and its gradient (Bridson, Marino & Fedkiw 2003, sign as in
// bending.hpp:29-51).
__device__ inline float dihedral(const float3 x[4], float3 g[4]) {
  const float3 n1 = cross(x[0] - x[2], x[0] - x[3]);
  const float3 n2 = cross(x[1] - x[3], x[1] - x[2]);
  const float3 E = x[3] - x[2];
  const float n1sq = dot(n1, n1), n2sq = dot(n2, n2), el = len(E);
  if (n1sq < 1e-24f || n2sq < 1e-24f || el < 1e-12f) {
#pragma unroll
    for (int k = 0; k < 4; ++k) g[k] = mk(0, 0, 0);
    return 0.0f;
  }
  const float3 e = div(E, el);
  const float3 m1 = n1 * rsqrtf(n1sq), m2 = n2 * rsqrtf(n2sq);
  const float theta = atan2f(dot(cross(m1, m2), e), dot(m1, m2));
  const float3 A = div(n1, n1sq), B = div(n2, n2sq);
  g[0] = A * -el;
  g[1] = B * -el;
  g[2] = -(A * (dot(x[0] - x[3], E) / el) + B * (dot(x[1] - x[3], E) / el));
  g[3] = A * (dot(x[0] - x[2], E) / el) + B * (dot(x[1] - x[2], E) / el);
  return theta;
}

// Hinge term 1/2 K (theta - theta0)^2 with a Gauss-Newton Hessian (energies.cpp:64-69), in two parts: hingeDerivs
// evaluates theta and its gradient once per term, hingeBlockFrom forms vertex a's gradient and any Hessian block.
struct HingeDer {
  float4 w[4];  // gradient of theta at vertex k (xyz); w[0].w = K (theta - rest), w[1].w = K
};

__device__ inline void hingeDerivs(float K, float rest, const float3 x[4], HingeDer& o) {
  float3 gr[4];
  const float theta = dihedral(x, gr);
  const float C = theta - rest;
  o.w[0] = f4(gr[0], K * C);
  o.w[1] = f4(gr[1], K);
  o.w[2] = f4(gr[2]);
  o.w[3] = f4(gr[3]);
}

// Block (a, b) of a hinge term's Hessian, K (grad_a theta)(grad_b theta)^T, and with Grad the gradient of vertex a,
// K (theta - rest) grad_a theta, from its record.
template <bool Grad>
__device__ inline void hingeBlockFrom(const float4* __restrict__ rec, int a, int b, float3& g, M3& H) {
  const float4 wa = rec[a], wb = rec[b];
  const float K = rec[1].w;
  if (Grad) g = xyz(wa) * rec[0].w;
  zero(H);
  addOuter(H, K, xyz(wa), xyz(wb));
}

// One-sided seam spring 1/2 K (d - target)^2 for d > target (energies.cpp:71-91): row a of the 2 x 2 block system.
__device__ inline void seamRow(float K, float target, float3 x0, float3 x1, int a, float3& g, M3 H[2]) {
  zero(H[0]);
  zero(H[1]);
  g = mk(0, 0, 0);
  const float3 diff = x0 - x1;
  const float d = len(diff);
  if (d <= target) return;
  M3 B;
  zero(B);
  if (d < 1e-12f) {
    B.m[0] = B.m[4] = B.m[8] = K;
  } else {
    const float3 n = div(diff, d);
    const float ext = d - target;
    g = n * (a == 0 ? K * ext : -K * ext);
    addOuter(B, K, n, n);
    addProjector(B, K * (ext / d), n);
  }
  const float s0 = a == 0 ? 1.0f : -1.0f;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    H[0].m[k] = s0 * B.m[k];
    H[1].m[k] = -s0 * B.m[k];
  }
}

// IPC smoothed Coulomb friction muLambda f0(|P dx|) with slip length eps (energies.cpp:93-110); dx = x - x0.
__device__ inline void frictionRow(float3 dx, float3 n, float muLambda, float eps, float3& g, M3& H) {
  if (!(muLambda > 0.0f) || !(eps > 0.0f)) return;
  const float3 u = dx - n * dot(n, dx);
  const float s = len(u);
  if (s < eps) {
    const float f1OverS = 2.0f / eps - s / (eps * eps);
    g += u * (muLambda * f1OverS);
    addProjector(H, muLambda * f1OverS, n);
    if (s > 0.0f) addOuter(H, -muLambda / (eps * eps * s), u, u);
  } else {
    const float3 dir = div(u, s);
    g += dir * muLambda;
    addProjector(H, muLambda / s, n);
    addOuter(H, -muLambda / s, dir, dir);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Term energies in FP64 (the line-search and Newton-energy precision).

struct d3 {
  double x, y, z;
};
__device__ __forceinline__ d3 toD(float3 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator*(double s, d3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dotd(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 crossd(d3 a, d3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double lend(d3 a) { return sqrt(dotd(a, a)); }

__device__ inline double stretchEnergy(const StretchIn& t, const d3 x[3]) {
  const d3 e1 = x[1] - x[0], e2 = x[2] - x[0];
  const d3 fu = (double)t.d.x * e1 + (double)t.d.y * e2;
  const d3 fv = (double)t.d.z * e1 + (double)t.d.w * e2;
  const double lu = lend(fu), lv = lend(fv), tiny = 1e-12;
  double e = 0;
  for (int which = 0; which < 2; ++which) {
    if (!(t.k[which] > 0.0f)) continue;
    const double l = which == 0 ? lu : lv;
    const double C = l > tiny ? l - 1.0 : 0.0;
    const double K = (double)t.k[which] * (double)t.area;
    e += 0.5 * K * C * C;
    if (t.limit[which] > 0.0f && C > t.limit[which]) {
      const double ex = C - t.limit[which];
      e += 0.5 * (double)t.limitScale * K * ex * ex;
    }
  }
  if (t.k[2] > 0.0f && lu > tiny && lv > tiny) {
    const double c = dotd(fu, fv) / (lu * lv);
    e += 0.5 * (double)t.k[2] * (double)t.area * c * c;
  }
  return e;
}

__device__ inline double hingeEnergy(double K, double rest, const d3 x[4]) {
  const d3 n1 = crossd(x[0] - x[2], x[0] - x[3]);
  const d3 n2 = crossd(x[1] - x[3], x[1] - x[2]);
  const d3 E = x[3] - x[2];
  const double n1sq = dotd(n1, n1), n2sq = dotd(n2, n2), el = lend(E);
  double theta = 0;
  if (!(n1sq < 1e-24 || n2sq < 1e-24 || el < 1e-12)) {
    const d3 m1 = (1.0 / sqrt(n1sq)) * n1, m2 = (1.0 / sqrt(n2sq)) * n2;
    theta = atan2(dotd(crossd(m1, m2), (1.0 / el) * E), dotd(m1, m2));
  }
  const double C = theta - rest;
  return 0.5 * K * C * C;
}

__device__ inline double seamEnergy(double K, double target, d3 x0, d3 x1) {
  const double d = lend(x0 - x1);
  if (d <= target || d < 1e-12) return 0.0;
  const double ext = d - target;
  return 0.5 * K * ext * ext;
}

__device__ inline double frictionEnergy(d3 dx, d3 n, double muLambda, double eps) {
  if (!(muLambda > 0) || !(eps > 0)) return 0.0;
  const d3 u = dx - dotd(n, dx) * n;
  const double s = lend(u);
  if (s < eps) return muLambda * (-s * s * s / (3 * eps * eps) + s * s / eps + eps / 3);
  return muLambda * s;
}

// ---------------------------------------------------------------------------------------------------------------
// Collision field.

struct FieldInfo {
  float ox, oy, oz, cell, band;
  int dims[3];
  int present;  // 0: no samples (every query returns band)
};

// Trilinear signed distance, any point outside the sampled box (or NaN) -> +band. Every operation is an explicitly
// rounded IEEE float op in the reference's order, so the result is bit-identical to the reference's 32-bit sample.
__device__ inline float fieldSample(const float* __restrict__ values, const FieldInfo& f, float3 p) {
  if (!f.present) return f.band;
  const float l[3] = {__fdiv_rn(__fsub_rn(p.x, f.ox), f.cell), __fdiv_rn(__fsub_rn(p.y, f.oy), f.cell),
                      __fdiv_rn(__fsub_rn(p.z, f.oz), f.cell)};
  int i[3];
  float t[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float maxCoord = __fsub_rn(static_cast<float>(f.dims[a]), 1.0f);
    if (!(l[a] >= 0.0f && l[a] <= maxCoord)) return f.band;
    const int fl = static_cast<int>(floorf(l[a]));
    const int top = f.dims[a] - 2;
    i[a] = fl < top ? fl : top;
    t[a] = __fsub_rn(l[a], static_cast<float>(i[a]));
  }
  float result = 0.0f;
#pragma unroll
  for (int dz = 0; dz < 2; ++dz)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const float wx = dx ? t[0] : __fsub_rn(1.0f, t[0]);
        const float wy = dy ? t[1] : __fsub_rn(1.0f, t[1]);
        const float wz = dz ? t[2] : __fsub_rn(1.0f, t[2]);
        const float w = __fmul_rn(__fmul_rn(wx, wy), wz);
        const uint32_t idx = (static_cast<uint32_t>(i[2] + dz) * static_cast<uint32_t>(f.dims[1]) +
                              static_cast<uint32_t>(i[1] + dy)) * static_cast<uint32_t>(f.dims[0]) +
                             static_cast<uint32_t>(i[0] + dx);
        result = __fadd_rn(result, __fmul_rn(w, __ldg(values + idx)));
      }
  return result;
}

// Central differences with step cell, normalised; zero where |g| < 1e-4 (the 32-bit flat threshold,
// term_math.h:228-231). Explicitly rounded like fieldSample.
__device__ inline float3 fieldGradient(const float* __restrict__ values, const FieldInfo& f, float3 p) {
  const float h = f.cell;
  const float h2 = __fmul_rn(2.0f, h);
  const float gx = __fdiv_rn(__fsub_rn(fieldSample(values, f, mk(__fadd_rn(p.x, h), p.y, p.z)),
                                       fieldSample(values, f, mk(__fsub_rn(p.x, h), p.y, p.z))), h2);
  const float gy = __fdiv_rn(__fsub_rn(fieldSample(values, f, mk(p.x, __fadd_rn(p.y, h), p.z)),
                                       fieldSample(values, f, mk(p.x, __fsub_rn(p.y, h), p.z))), h2);
  const float gz = __fdiv_rn(__fsub_rn(fieldSample(values, f, mk(p.x, p.y, __fadd_rn(p.z, h))),
                                       fieldSample(values, f, mk(p.x, p.y, __fsub_rn(p.z, h)))), h2);
  const float n = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz)));
  if (n < 1e-4f) return mk(0, 0, 0);
  return mk(__fdiv_rn(gx, n), __fdiv_rn(gy, n), __fdiv_rn(gz, n));
}

__device__ __forceinline__ bool isZero(float3 v) { return v.x == 0.0f && v.y == 0.0f && v.z == 0.0f; }

// Double-precision sample for the FP64 statistics (the reference computes penetration with the double field,
// sim_model.cpp:237-239).
__device__ inline double fieldSampleD(const float* __restrict__ values, const FieldInfo& f, double px, double py,
                                      double pz, double ox, double oy, double oz, double cell) {
  if (!f.present) return f.band;
  const double l[3] = {(px - ox) / cell, (py - oy) / cell, (pz - oz) / cell};
  int i[3];
  double t[3];
  for (int a = 0; a < 3; ++a) {
    const double maxCoord = f.dims[a] - 1;
    if (!(l[a] >= 0.0 && l[a] <= maxCoord)) return f.band;
    const int fl = static_cast<int>(floor(l[a]));
    i[a] = fl < f.dims[a] - 2 ? fl : f.dims[a] - 2;
    t[a] = l[a] - i[a];
  }
  double result = 0;
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        const double w = (dx ? t[0] : 1 - t[0]) * (dy ? t[1] : 1 - t[1]) * (dz ? t[2] : 1 - t[2]);
        const size_t idx = (static_cast<size_t>(i[2] + dz) * f.dims[1] + (i[1] + dy)) * f.dims[0] + (i[0] + dx);
        result += w * static_cast<double>(values[idx]);
      }
  return result;
}

// Push out to `radius` along the field gradient, then positional Coulomb friction against this substep's tangential
// motion (collision.cpp:5-22, in float as the reference's 32-bit path).
__device__ inline void collideBody(const float* __restrict__ values, const FieldInfo& f, float radius, float friction,
                                   float3 xPrev, float3& x) {
  const float phi = fieldSample(values, f, x);
  if (phi >= radius) return;
  const float3 n = fieldGradient(values, f, x);
  if (isZero(n)) return;
  const float depth = radius - phi;
  x += n * depth;
  const float3 delta = x - xPrev;
  const float3 tangential = delta - n * dot(delta, n);
  const float t = len(tangential);
  if (t <= friction * depth) {
    x -= tangential;
  } else if (t > 0.0f) {
    x -= tangential * (friction * depth / t);
  }
}

// Last point on from -> to at least `radius` from the body (40 bisections), or `from` if it is already closer
// (collision.cpp:24-34).
__device__ inline float3 landOnBody(const float* __restrict__ values, const FieldInfo& f, float radius, float3 from,
                                    float3 to) {
  if (!(fieldSample(values, f, from) >= radius)) return from;
  float lo = 0.0f, hi = 1.0f;
  const float3 d = to - from;
  for (int i = 0; i < 40; ++i) {
    const float mid = 0.5f * (lo + hi);
    if (fieldSample(values, f, from + d * mid) >= radius) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  return from + d * lo;
}

}  // namespace dcu
