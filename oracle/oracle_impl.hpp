// ORACLE — test infrastructure only (see oracle_api.h). CPU restatement of the reference solver:
//   model build, block-CSR structure and slot maps  <- libs/sim/src/sim_model.cpp:12-274
//   fixed-order gather lists                        <- libs/sim/src/gpu/gpu_solver_core.cpp:184-224
//   term math                                       <- libs/sim/src/energies.cpp:11-110, stretch.hpp:15-49,
//                                                      bending.hpp:29-51, bending.cpp:7-18
//   collision field and push-out                    <- libs/core/src/collision_field.cpp:8-41,
//                                                      libs/sim/src/collision.cpp:5-34
//   Newton / PCG / line search / finish             <- libs/sim/src/cpu_solver.cpp:34-338
// No Eigen: small fixed-size vector and matrix types below.
#pragma once
#include "oracle_api.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace oracle {

// Loops over fewer items than this run on the calling thread (a parallel region costs more than they do).
constexpr std::ptrdiff_t kParallelMin = 4096;

// ---------------------------------------------------------------------------------------------------------------
// Fixed-size math.

template <class T>
struct V3 {
  T x = 0, y = 0, z = 0;
  T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class T> V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> V3<T>& operator+=(V3<T>& a, V3<T> b) { return a = a + b; }
template <class T> V3<T>& operator-=(V3<T>& a, V3<T> b) { return a = a - b; }
template <class T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> T sqnorm(V3<T> a) { return dot(a, a); }
template <class T> T norm(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> bool isZero(V3<T> a) { return a.x == 0 && a.y == 0 && a.z == 0; }
template <class T> bool finite(V3<T> a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }

using V3d = V3<double>;
using V3f = V3<float>;
inline V3f tof(V3d a) { return {static_cast<float>(a.x), static_cast<float>(a.y), static_cast<float>(a.z)}; }
inline V3d tod(V3f a) { return {a.x, a.y, a.z}; }

struct M3 {
  double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  static M3 identity() {
    M3 r;
    r.m[0][0] = r.m[1][1] = r.m[2][2] = 1;
    return r;
  }
  static M3 outer(V3d a, V3d b) {
    M3 r;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) r.m[i][j] = a[i] * b[j];
    return r;
  }
  M3& operator+=(const M3& o) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) m[i][j] += o.m[i][j];
    return *this;
  }
  M3& operator-=(const M3& o) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) m[i][j] -= o.m[i][j];
    return *this;
  }
};
inline M3 operator*(double s, const M3& a) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = s * a.m[i][j];
  return r;
}
inline M3 operator+(M3 a, const M3& b) { return a += b; }
inline M3 operator-(M3 a, const M3& b) { return a -= b; }
inline V3d operator*(const M3& a, V3d v) {
  return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z, a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
          a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}

// Inverse of a symmetric 3x3 matrix by an LDL^T factorisation with symmetric diagonal pivoting (the largest remaining
// diagonal entry first), the method of the Eigen::LDLT the reference uses for its preconditioner blocks
// (cpu_solver.cpp:176-177). ok is false when a pivot is zero or not finite.
inline M3 invertSymmetric(const M3& A, bool& ok) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = A.m[i][j];
  int perm[3] = {0, 1, 2};
  double L[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, D[3] = {0, 0, 0};
  ok = true;
  for (int k = 0; k < 3; ++k) {
    int best = k;
    for (int i = k + 1; i < 3; ++i)
      if (std::abs(a[i][i]) > std::abs(a[best][best])) best = i;
    if (best != k) {
      std::swap(perm[k], perm[best]);
      for (int j = 0; j < 3; ++j) std::swap(a[k][j], a[best][j]);
      for (int i = 0; i < 3; ++i) std::swap(a[i][k], a[i][best]);
      for (int j = 0; j < k; ++j) std::swap(L[k][j], L[best][j]);
    }
    D[k] = a[k][k];
    if (!(D[k] != 0) || !std::isfinite(D[k])) {
      ok = false;
      return M3::identity();
    }
    for (int i = k + 1; i < 3; ++i) L[i][k] = a[i][k] / D[k];
    for (int i = k + 1; i < 3; ++i)
      for (int j = k + 1; j < 3; ++j) a[i][j] -= L[i][k] * D[k] * L[j][k];
  }
  // P A P^T = L D L^T  =>  A^{-1} = P^T L^{-T} D^{-1} L^{-1} P.
  M3 inv;
  for (int c = 0; c < 3; ++c) {
    double e[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i) e[i] = perm[i] == c ? 1.0 : 0.0;  // P e_c
    double y[3];
    for (int i = 0; i < 3; ++i) {
      y[i] = e[i];
      for (int j = 0; j < i; ++j) y[i] -= L[i][j] * y[j];
    }
    for (int i = 0; i < 3; ++i) y[i] /= D[i];
    double xs[3];
    for (int i = 2; i >= 0; --i) {
      xs[i] = y[i];
      for (int j = i + 1; j < 3; ++j) xs[i] -= L[j][i] * xs[j];
    }
    for (int i = 0; i < 3; ++i) inv.m[perm[i]][c] = xs[i];
  }
  return inv;
}

// ---------------------------------------------------------------------------------------------------------------
// Collision field (collision_field.cpp:8-41).

struct Field {
  V3d origin;
  double cellSize = 0.004;
  int dims[3] = {0, 0, 0};
  double band = 0.02;
  std::vector<float> values;

  double sample(V3d p) const {
    if (values.empty()) return band;
    const V3d local = {(p.x - origin.x) / cellSize, (p.y - origin.y) / cellSize, (p.z - origin.z) / cellSize};
    int i[3];
    double t[3];
    for (int a = 0; a < 3; ++a) {
      const double maxCoord = dims[a] - 1;
      if (!(local[a] >= 0.0 && local[a] <= maxCoord)) return band;
      i[a] = std::min(static_cast<int>(std::floor(local[a])), dims[a] - 2);
      t[a] = local[a] - i[a];
    }
    double result = 0;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const double w = (dx ? t[0] : 1 - t[0]) * (dy ? t[1] : 1 - t[1]) * (dz ? t[2] : 1 - t[2]);
          const std::size_t idx =
              (static_cast<std::size_t>(i[2] + dz) * dims[1] + (i[1] + dy)) * dims[0] + (i[0] + dx);
          result += w * static_cast<double>(values[idx]);
        }
    return result;
  }

  V3d gradient(V3d p) const {
    V3d g;
    for (int a = 0; a < 3; ++a) {
      V3d d;
      d[a] = cellSize;
      g[a] = (sample(p + d) - sample(p - d)) / (2 * cellSize);
    }
    const double n = norm(g);
    return n < 1e-9 ? V3d{} : g / n;
  }
};

Field fieldFrom(const drape_field_desc* f) {
  Field out;
  if (!f) return out;
  out.origin = {f->origin[0], f->origin[1], f->origin[2]};
  out.cellSize = f->cell_size;
  for (int a = 0; a < 3; ++a) out.dims[a] = f->dims[a];
  out.band = f->band;
  const std::size_t count = static_cast<std::size_t>(std::max(0, f->dims[0])) * std::max(0, f->dims[1]) *
                            std::max(0, f->dims[2]);
  if (f->values && count > 0) out.values.assign(f->values, f->values + count);
  return out;
}

// collision.cpp:5-22, in float as the reference does (Eigen::Vector3f arithmetic, double field queries).
void collideBodyF(const Field& body, float radius, float friction, V3f xPrev, V3f& x) {
  const V3d p = tod(x);
  const double phi = body.sample(p);
  if (phi >= radius) return;
  const V3f n = tof(body.gradient(p));
  if (isZero(n)) return;
  const float depth = static_cast<float>(radius - phi);
  x += depth * n;
  const V3f delta = x - xPrev;
  const V3f tangential = delta - dot(delta, n) * n;
  const float t = norm(tangential);
  if (t <= friction * depth) {
    x -= tangential;
  } else if (t > 0) {
    x -= tangential * (friction * depth / t);
  }
}

// collision.cpp:24-34.
V3f landOnBodyF(const Field& body, float radius, V3f from, V3f to) {
  auto clear = [&](float t) { return body.sample(tod(from + t * (to - from))) >= radius; };
  if (!clear(0)) return from;
  float lo = 0, hi = 1;
  for (int i = 0; i < 40; ++i) {
    const float mid = 0.5f * (lo + hi);
    (clear(mid) ? lo : hi) = mid;
  }
  return from + lo * (to - from);
}

// The same two helpers with double particle state (full FP64 mode).
void collideBodyD(const Field& body, double radius, double friction, V3d xPrev, V3d& x) {
  const double phi = body.sample(x);
  if (phi >= radius) return;
  const V3d n = body.gradient(x);
  if (isZero(n)) return;
  const double depth = radius - phi;
  x += depth * n;
  const V3d delta = x - xPrev;
  const V3d tangential = delta - dot(delta, n) * n;
  const double t = norm(tangential);
  if (t <= friction * depth) {
    x -= tangential;
  } else if (t > 0) {
    x -= tangential * (friction * depth / t);
  }
}

V3d landOnBodyD(const Field& body, double radius, V3d from, V3d to) {
  auto clear = [&](double t) { return body.sample(from + t * (to - from)) >= radius; };
  if (!clear(0)) return from;
  double lo = 0, hi = 1;
  for (int i = 0; i < 40; ++i) {
    const double mid = 0.5 * (lo + hi);
    (clear(mid) ? lo : hi) = mid;
  }
  return from + lo * (to - from);
}

// ---------------------------------------------------------------------------------------------------------------
// Term math (energies.hpp:16-56, energies.cpp, stretch.hpp, bending.hpp, bending.cpp).

template <int N>
struct TermEval {
  double energy = 0;
  V3d grad[N];
  M3 hess[N][N];
};

struct Dm {  // Eigen::Matrix2d dmInv: d[r][c]
  double d[2][2] = {{1, 0}, {0, 1}};
};

double vertexCoefficient(const Dm& dm, int column, int local) {
  if (local == 1) return dm.d[0][column];
  if (local == 2) return dm.d[1][column];
  return -(dm.d[0][column] + dm.d[1][column]);
}

template <int N>
void addQuadratic(TermEval<N>& out, double K, double C, const V3d* g) {
  out.energy += 0.5 * K * C * C;
  for (int i = 0; i < N; ++i) {
    out.grad[i] += K * C * g[i];
    for (int j = 0; j < N; ++j) out.hess[i][j] += M3::outer(K * g[i], g[j]);
  }
}

void addTension(TermEval<3>& out, double K, double C, const Dm& dm, int column, V3d f) {
  if (C <= 0) return;
  const double len = norm(f);
  if (len < 1e-12) return;
  const V3d n = f / len;
  const M3 P = (K * C / len) * (M3::identity() - M3::outer(n, n));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out.hess[i][j] += (vertexCoefficient(dm, column, i) * vertexCoefficient(dm, column, j)) * P;
}

void evalStretch(const V3d* x, const Dm& dm, int which, double& C, V3d* grad) {
  const V3d e1 = x[1] - x[0];
  const V3d e2 = x[2] - x[0];
  const V3d fu = e1 * dm.d[0][0] + e2 * dm.d[1][0];
  const V3d fv = e1 * dm.d[0][1] + e2 * dm.d[1][1];
  const double lu = norm(fu), lv = norm(fv);
  const double tiny = 1e-12;
  V3d dfu, dfv;
  C = 0;
  if (which == 0) {
    if (lu > tiny) {
      C = lu - 1;
      dfu = fu / lu;
    }
  } else if (which == 1) {
    if (lv > tiny) {
      C = lv - 1;
      dfv = fv / lv;
    }
  } else if (lu > tiny && lv > tiny) {
    const V3d nu = fu / lu, nv = fv / lv;
    const double c = dot(nu, nv);
    C = c;
    dfu = (nv - c * nu) / lu;
    dfv = (nu - c * nv) / lv;
  }
  grad[1] = dfu * dm.d[0][0] + dfv * dm.d[0][1];
  grad[2] = dfu * dm.d[1][0] + dfv * dm.d[1][1];
  grad[0] = -(grad[1] + grad[2]);
}

struct Fabric {
  double stretchWarp = 0, stretchWeft = 0, stretchBias = 0, strainLimitWarp = 0, strainLimitWeft = 0;
  double bendWarp = 0, bendWeft = 0, weight = 0, thickness = 0, friction = 0, damping = 0;
};

Fabric fabricFrom(const drape_fabric& f) {
  return {f.stretch_warp, f.stretch_weft, f.stretch_bias, f.strain_limit_warp, f.strain_limit_weft, f.bend_warp,
          f.bend_weft, f.weight, f.thickness, f.friction, f.damping};
}

void evalStretchTerm(const Dm& dm, double area, const V3d* x, const Fabric& f, double limitScale, TermEval<3>& out) {
  const double k[3] = {f.stretchWarp, f.stretchWeft, f.stretchBias};
  const double limit[2] = {f.strainLimitWarp, f.strainLimitWeft};
  const V3d e1 = x[1] - x[0], e2 = x[2] - x[0];
  const V3d fcol[2] = {e1 * dm.d[0][0] + e2 * dm.d[1][0], e1 * dm.d[0][1] + e2 * dm.d[1][1]};
  V3d g[3];
  double C = 0;
  for (int which = 0; which < 3; ++which) {
    if (k[which] <= 0) continue;
    evalStretch(x, dm, which, C, g);
    const double K = k[which] * area;
    addQuadratic<3>(out, K, C, g);
    if (which == 2) continue;
    addTension(out, K, C, dm, which, fcol[which]);
    if (limit[which] > 0 && C > limit[which]) {
      const double KL = limitScale * K;
      const double excess = C - limit[which];
      addQuadratic<3>(out, KL, excess, g);
      addTension(out, KL, excess, dm, which, fcol[which]);
    }
  }
}

void evalDihedral(const V3d* x, double& theta, V3d* grad) {
  const V3d n1 = cross(x[0] - x[2], x[0] - x[3]);
  const V3d n2 = cross(x[1] - x[3], x[1] - x[2]);
  const V3d E = x[3] - x[2];
  const double n1sq = sqnorm(n1), n2sq = sqnorm(n2), elen = norm(E);
  if (n1sq < 1e-24 || n2sq < 1e-24 || elen < 1e-12) {
    theta = 0;
    for (int i = 0; i < 4; ++i) grad[i] = V3d{};
    return;
  }
  const V3d e = E / elen;
  const V3d m1 = n1 / std::sqrt(n1sq), m2 = n2 / std::sqrt(n2sq);
  theta = std::atan2(dot(cross(m1, m2), e), dot(m1, m2));
  const V3d a = n1 / n1sq, b = n2 / n2sq;
  grad[0] = -elen * a;
  grad[1] = -elen * b;
  grad[2] = -((dot(x[0] - x[3], E) / elen) * a + (dot(x[1] - x[3], E) / elen) * b);
  grad[3] = (dot(x[0] - x[2], E) / elen) * a + (dot(x[1] - x[2], E) / elen) * b;
}

void evalHingeTerm(double K, double restAngle, const V3d* x, TermEval<4>& out) {
  double theta = 0;
  V3d g[4];
  evalDihedral(x, theta, g);
  addQuadratic<4>(out, K, theta - restAngle, g);
}

void evalSeamTerm(const V3d* x, double target, double K, TermEval<2>& out) {
  const V3d diff = x[0] - x[1];
  const double d = norm(diff);
  if (d <= target) return;
  M3 block;
  if (d < 1e-12) {
    block = K * M3::identity();
  } else {
    const V3d n = diff / d;
    const double ext = d - target;
    out.energy += 0.5 * K * ext * ext;
    out.grad[0] += K * ext * n;
    out.grad[1] -= K * ext * n;
    const M3 nn = M3::outer(n, n);
    block = K * (nn + (ext / d) * (M3::identity() - nn));
  }
  out.hess[0][0] += block;
  out.hess[1][1] += block;
  out.hess[0][1] -= block;
  out.hess[1][0] -= block;
}

void evalFrictionTerm(V3d x, V3d x0, V3d n, double muLambda, double eps, TermEval<1>& out) {
  if (muLambda <= 0 || eps <= 0) return;
  const M3 P = M3::identity() - M3::outer(n, n);
  const V3d u = P * (x - x0);
  const double s = norm(u);
  if (s < eps) {
    out.energy += muLambda * (-s * s * s / (3 * eps * eps) + s * s / eps + eps / 3);
    const double f1OverS = 2 / eps - s / (eps * eps);
    out.grad[0] += muLambda * f1OverS * u;
    out.hess[0][0] += (muLambda * f1OverS) * P;
    if (s > 0) out.hess[0][0] -= (muLambda / (eps * eps * s)) * M3::outer(u, u);
  } else {
    const V3d dir = u / s;
    out.energy += muLambda * s;
    out.grad[0] += muLambda * dir;
    out.hess[0][0] += (muLambda / s) * (P - M3::outer(dir, dir));
  }
}

struct BendCoefficients {
  double p = 0, q = 0;
};
BendCoefficients bendingCoefficients(double bendWarp, double bendWeft) {
  const double floor = 0.05 * std::min(bendWarp, bendWeft);
  return {std::max((3.0 * bendWarp - bendWeft) / 2.0, floor), std::max(bendWeft, floor)};
}
double edgeBendStiffness(const BendCoefficients& c, const double restEdgeDir[2], const double grain[2]) {
  const double dn = std::sqrt(restEdgeDir[0] * restEdgeDir[0] + restEdgeDir[1] * restEdgeDir[1]);
  const double un = std::sqrt(grain[0] * grain[0] + grain[1] * grain[1]);
  const double d[2] = {restEdgeDir[0] / dn, restEdgeDir[1] / dn};
  const double u[2] = {grain[0] / un, grain[1] / un};
  const double cosPhi = d[0] * u[0] + d[1] * u[1];
  const double sinPhi = d[0] * u[1] - d[1] * u[0];
  return c.p * sinPhi * sinPhi + c.q * cosPhi * cosPhi;
}

// ---------------------------------------------------------------------------------------------------------------
// Model (sim_model.hpp:20-83, sim_model.cpp).

constexpr double kContactReach = 0.01;   // sim_model.hpp:14
constexpr double kContactSnap = 0.0005;  // sim_model.hpp:15

enum Phase { Assembling = 0, Settling = 1 };

struct Settings {
  V3d gravity{0, -9.81, 0};
  double collisionOffset = 0.003, assemblyClosingSpeed = 0.25, assemblyExtraDamping = 10.0, dampingScale = 5.0;
  double strainLimitStiffnessScale = 100.0, seamStiffness = 1e4, frictionSlipSpeed = 3e-4;
  int maxCgIterations = 50;
  double cgTolerance = 1e-2;
};

struct Model {
  struct Garment {
    std::string id;
    uint32_t offset = 0, count = 0;
    Phase phase = Settling;
    double assemblyTime = 0;
    uint32_t fabricOffset = 0, pieceCount = 0;
  };
  struct HingeSide {
    uint32_t fabric = 0;
    double edgeDir[2] = {1, 0}, grain[2] = {0, 1};
  };
  struct Stretch {
    std::array<uint32_t, 3> v{};
    Dm dmInv;
    double area = 0;
    uint32_t fabric = 0;
  };
  struct Hinge {
    std::array<uint32_t, 4> v{};
    double K = 0, restAngle = 0;
  };
  struct Seam {
    uint32_t a = 0, b = 0, garment = 0;
    float startGap = 0;
  };

  bool fp64 = false;  // particle state precision: float (faithful) or double
  Settings settings;
  bool hasBody = false;
  Field body;
  std::vector<Garment> garments;
  std::vector<Fabric> fabrics;
  std::vector<V3d> x, v;  // exactly float-representable in faithful mode
  std::vector<double> mass, vertexArea;
  std::vector<V3d> fExt;
  std::vector<uint32_t> pFabric, pGarment;
  std::vector<uint8_t> pinned;
  std::vector<std::pair<uint32_t, V3d>> pins;
  std::vector<Stretch> stretch;
  std::vector<Hinge> hinges;
  std::vector<std::array<HingeSide, 2>> hingeSides;
  std::vector<double> hingeGeom;
  std::vector<Seam> seams;
  std::vector<uint32_t> rowStart, colIndex, diagSlot;
  std::vector<std::array<uint32_t, 9>> stretchSlots;
  std::vector<std::array<uint32_t, 16>> hingeSlots;
  std::vector<std::array<uint32_t, 4>> seamSlots;
  std::vector<double> contactForce;

  V3d state(V3d a) const { return fp64 ? a : tod(tof(a)); }

  std::size_t garmentIndex(const std::string& id) const {
    for (std::size_t i = 0; i < garments.size(); ++i)
      if (garments[i].id == id) return i;
    throw std::out_of_range("unknown garment '" + id + "'");
  }
  double contactRadius(std::size_t i) const { return settings.collisionOffset + 0.5 * fabrics[pFabric[i]].thickness; }
  double seamTarget(const Seam& sp) const {
    const auto& g = garments[sp.garment];
    if (g.phase != Assembling) return 0.0;
    return std::max(0.0, static_cast<double>(sp.startGap) - settings.assemblyClosingSpeed * g.assemblyTime);
  }
  double hingeStiffness(std::size_t hgi) const {
    double B = 0;
    for (const auto& side : hingeSides[hgi]) {
      const auto& f = fabrics[side.fabric];
      B += 0.5 * edgeBendStiffness(bendingCoefficients(f.bendWarp, f.bendWeft), side.edgeDir, side.grain);
    }
    return B * hingeGeom[hgi];
  }
  void updateMass(uint32_t i) { mass[i] = std::max(vertexArea[i] * fabrics[pFabric[i]].weight, 1e-12); }
  uint32_t slot(uint32_t row, uint32_t col) const {
    const auto begin = colIndex.begin() + rowStart[row];
    const auto end = colIndex.begin() + rowStart[row + 1];
    return static_cast<uint32_t>(std::lower_bound(begin, end, col) - colIndex.begin());
  }
  // |x_a - x_b| as the reference computes it on Vec3f in faithful mode.
  double gap(uint32_t a, uint32_t b) const {
    if (fp64) return norm(x[a] - x[b]);
    return static_cast<double>(norm(tof(x[a]) - tof(x[b])));
  }

  void buildStructure() {
    const std::size_t n = x.size();
    std::vector<std::vector<uint32_t>> cols(n);
    auto couple = [&](const uint32_t* vs, int m) {
      for (int a = 0; a < m; ++a)
        for (int b = 0; b < m; ++b) cols[vs[a]].push_back(vs[b]);
    };
    for (std::size_t i = 0; i < n; ++i) cols[i].push_back(static_cast<uint32_t>(i));
    for (const auto& t : stretch) couple(t.v.data(), 3);
    for (const auto& h : hinges) couple(h.v.data(), 4);
    for (const auto& s : seams) {
      const uint32_t ab[2] = {s.a, s.b};
      couple(ab, 2);
    }
    rowStart.assign(n + 1, 0);
    colIndex.clear();
    for (std::size_t i = 0; i < n; ++i) {
      std::sort(cols[i].begin(), cols[i].end());
      cols[i].erase(std::unique(cols[i].begin(), cols[i].end()), cols[i].end());
      colIndex.insert(colIndex.end(), cols[i].begin(), cols[i].end());
      rowStart[i + 1] = static_cast<uint32_t>(colIndex.size());
    }
    diagSlot.resize(n);
    for (uint32_t i = 0; i < n; ++i) diagSlot[i] = slot(i, i);
    auto slotsFor = [&](const uint32_t* vs, int m, uint32_t* out) {
      for (int a = 0; a < m; ++a)
        for (int b = 0; b < m; ++b) out[a * m + b] = slot(vs[a], vs[b]);
    };
    stretchSlots.resize(stretch.size());
    for (std::size_t k = 0; k < stretch.size(); ++k) slotsFor(stretch[k].v.data(), 3, stretchSlots[k].data());
    hingeSlots.resize(hinges.size());
    for (std::size_t k = 0; k < hinges.size(); ++k) slotsFor(hinges[k].v.data(), 4, hingeSlots[k].data());
    seamSlots.resize(seams.size());
    for (std::size_t k = 0; k < seams.size(); ++k) {
      const uint32_t ab[2] = {seams[k].a, seams[k].b};
      slotsFor(ab, 2, seamSlots[k].data());
    }
    contactForce.assign(n, 0.0);
  }

  static Model build(const drape_scene_desc& scene, bool fp64) {
    Model next;
    next.fp64 = fp64;
    const auto& s = scene.settings;
    next.settings.gravity = {s.gravity[0], s.gravity[1], s.gravity[2]};
    next.settings.collisionOffset = s.collision_offset;
    next.settings.assemblyClosingSpeed = s.assembly_closing_speed;
    next.settings.assemblyExtraDamping = s.assembly_extra_damping;
    next.settings.dampingScale = s.damping_scale;
    next.settings.strainLimitStiffnessScale = s.strain_limit_stiffness_scale;
    next.settings.seamStiffness = s.seam_stiffness;
    next.settings.frictionSlipSpeed = s.friction_slip_speed;
    next.settings.maxCgIterations = s.max_cg_iterations;
    next.settings.cgTolerance = s.cg_tolerance;
    next.hasBody = scene.body != nullptr;
    if (scene.body) next.body = fieldFrom(scene.body);
    for (uint32_t gi0 = 0; gi0 < scene.garment_count; ++gi0) {
      const drape_garment_desc& sg = scene.garments[gi0];
      const std::string id = sg.id ? sg.id : "";
      // One initial position per mesh vertex and one fabric per piece are structural in this flattened form (the
      // counts are shared); the reference's two size checks (sim_model.cpp:81-86) reduce to null checks here.
      if (sg.vertex_count > 0 && !sg.initial_positions)
        throw std::invalid_argument("garment '" + id + "': one initial position per mesh vertex required");
      if (sg.piece_count > 0 && !sg.piece_fabric)
        throw std::invalid_argument("garment '" + id + "': one fabric per pattern piece required");
      Garment g;
      g.id = id;
      g.offset = static_cast<uint32_t>(next.x.size());
      g.count = sg.vertex_count;
      g.fabricOffset = static_cast<uint32_t>(next.fabrics.size());
      g.pieceCount = sg.piece_count;
      const auto gi = static_cast<uint32_t>(next.garments.size());
      const uint32_t off = g.offset;
      for (uint32_t p = 0; p < sg.piece_count; ++p) next.fabrics.push_back(fabricFrom(sg.piece_fabric[p]));
      auto rest = [&](uint32_t vtx) { return std::array<double, 2>{sg.rest[2 * vtx], sg.rest[2 * vtx + 1]}; };
      for (uint32_t vtx = 0; vtx < sg.vertex_count; ++vtx) {
        const V3d p0{sg.initial_positions[3 * vtx], sg.initial_positions[3 * vtx + 1], sg.initial_positions[3 * vtx + 2]};
        next.x.push_back(next.state(p0));
        next.vertexArea.push_back(sg.vertex_area[vtx]);
        next.pFabric.push_back(g.fabricOffset + sg.vertex_piece[vtx]);
        next.pGarment.push_back(gi);
      }
      auto tri = [&](uint32_t t) {
        return std::array<uint32_t, 3>{sg.triangles[3 * t], sg.triangles[3 * t + 1], sg.triangles[3 * t + 2]};
      };
      auto triArea = [&](uint32_t t) {
        const auto tr = tri(t);
        const auto r0 = rest(tr[0]), r1 = rest(tr[1]), r2 = rest(tr[2]);
        const double a[2] = {r1[0] - r0[0], r1[1] - r0[1]}, b[2] = {r2[0] - r0[0], r2[1] - r0[1]};
        return 0.5 * std::abs(a[0] * b[1] - a[1] * b[0]);
      };
      auto grain = [&](uint32_t piece) { return std::array<double, 2>{sg.piece_grain[2 * piece], sg.piece_grain[2 * piece + 1]}; };
      // Stretch terms in each piece's grain frame (sim_model.cpp:107-123).
      for (uint32_t t = 0; t < sg.triangle_count; ++t) {
        const auto tr = tri(t);
        const uint32_t piece = sg.triangle_piece[t];
        const auto u = grain(piece);
        const double vdir[2] = {-u[1], u[0]};
        double rr[3][2];
        for (int k = 0; k < 3; ++k) {
          const auto r = rest(tr[k]);
          rr[k][0] = r[0] * u[0] + r[1] * u[1];
          rr[k][1] = r[0] * vdir[0] + r[1] * vdir[1];
        }
        const double m00 = rr[1][0] - rr[0][0], m01 = rr[2][0] - rr[0][0];
        const double m10 = rr[1][1] - rr[0][1], m11 = rr[2][1] - rr[0][1];
        const double det = m00 * m11 - m10 * m01;
        Stretch st;
        for (int k = 0; k < 3; ++k) st.v[k] = off + tr[k];
        // Closed-form 2x2 inverse: the adjugate times 1 / det, the order of operations of Eigen's Matrix2d::inverse.
        const double invdet = 1.0 / det;
        st.dmInv.d[0][0] = m11 * invdet;
        st.dmInv.d[0][1] = -m01 * invdet;
        st.dmInv.d[1][0] = -m10 * invdet;
        st.dmInv.d[1][1] = m00 * invdet;
        st.area = 0.5 * std::abs(det);
        st.fabric = g.fabricOffset + piece;
        next.stretch.push_back(st);
      }
      // Hinges: one per interior edge shared by two triangles of the same piece, in std::map edge order
      // (sim_model.cpp:124-146).
      std::map<std::pair<uint32_t, uint32_t>, std::vector<uint32_t>> edgeTris;
      for (uint32_t t = 0; t < sg.triangle_count; ++t) {
        const auto tr = tri(t);
        for (int k = 0; k < 3; ++k) edgeTris[std::minmax(tr[k], tr[(k + 1) % 3])].push_back(t);
      }
      auto opposite = [&](uint32_t t, uint32_t e0, uint32_t e1) {
        for (auto vtx : tri(t))
          if (vtx != e0 && vtx != e1) return vtx;
        return e0;
      };
      for (const auto& [edge, tris] : edgeTris) {
        if (tris.size() != 2 || sg.triangle_piece[tris[0]] != sg.triangle_piece[tris[1]]) continue;
        const uint32_t piece = sg.triangle_piece[tris[0]];
        const auto r0 = rest(edge.first), r1 = rest(edge.second);
        const double d[2] = {r1[0] - r0[0], r1[1] - r0[1]};
        Hinge hg;
        hg.v = {off + opposite(tris[0], edge.first, edge.second), off + opposite(tris[1], edge.first, edge.second),
                off + edge.first, off + edge.second};
        next.hinges.push_back(hg);
        HingeSide side;
        side.fabric = g.fabricOffset + piece;
        side.edgeDir[0] = d[0];
        side.edgeDir[1] = d[1];
        const auto gr = grain(piece);
        side.grain[0] = gr[0];
        side.grain[1] = gr[1];
        next.hingeSides.push_back({side, side});
        next.hingeGeom.push_back((d[0] * d[0] + d[1] * d[1]) / (triArea(tris[0]) + triArea(tris[1])));
      }
      // Seam springs, plus seam hinges across consecutive pairs (sim_model.cpp:147-175).
      auto triangleWithEdge = [&](uint32_t e0, uint32_t e1) -> int64_t {
        auto it = edgeTris.find(std::minmax(e0, e1));
        return (it == edgeTris.end() || it->second.size() != 1) ? -1 : it->second[0];
      };
      auto pair = [&](uint32_t k) {
        return std::array<uint32_t, 3>{sg.seam_pairs[4 * k], sg.seam_pairs[4 * k + 1], sg.seam_pairs[4 * k + 2]};
      };
      auto init = [&](uint32_t vtx) {
        return V3d{sg.initial_positions[3 * vtx], sg.initial_positions[3 * vtx + 1], sg.initial_positions[3 * vtx + 2]};
      };
      for (uint32_t k = 0; k < sg.seam_pair_count; ++k) {
        const auto sp = pair(k);
        Seam spring;
        spring.a = off + sp[0];
        spring.b = off + sp[1];
        spring.garment = gi;
        spring.startGap = static_cast<float>(norm(init(sp[0]) - init(sp[1])));
        next.seams.push_back(spring);
        if (k + 1 >= sg.seam_pair_count || pair(k + 1)[2] != sp[2]) continue;
        const auto nx = pair(k + 1);
        const int64_t tA = triangleWithEdge(sp[0], nx[0]);
        const int64_t tB = triangleWithEdge(sp[1], nx[1]);
        if (tA < 0 || tB < 0) continue;
        const auto ta = static_cast<uint32_t>(tA), tb = static_cast<uint32_t>(tB);
        const uint32_t pieceA = sg.triangle_piece[ta], pieceB = sg.triangle_piece[tb];
        const auto ra0 = rest(sp[0]), ra1 = rest(nx[0]), rb0 = rest(sp[1]), rb1 = rest(nx[1]);
        const double dA[2] = {ra1[0] - ra0[0], ra1[1] - ra0[1]};
        const double dB[2] = {rb1[0] - rb0[0], rb1[1] - rb0[1]};
        Hinge hg;
        hg.v = {off + opposite(ta, sp[0], nx[0]), off + opposite(tb, sp[1], nx[1]), off + sp[0], off + nx[0]};
        next.hinges.push_back(hg);
        HingeSide sa, sb;
        sa.fabric = g.fabricOffset + pieceA;
        sa.edgeDir[0] = dA[0];
        sa.edgeDir[1] = dA[1];
        sa.grain[0] = grain(pieceA)[0];
        sa.grain[1] = grain(pieceA)[1];
        sb.fabric = g.fabricOffset + pieceB;
        sb.edgeDir[0] = dB[0];
        sb.edgeDir[1] = dB[1];
        sb.grain[0] = grain(pieceB)[0];
        sb.grain[1] = grain(pieceB)[1];
        next.hingeSides.push_back({sa, sb});
        next.hingeGeom.push_back((dA[0] * dA[0] + dA[1] * dA[1]) / (triArea(ta) + triArea(tb)));
      }
      next.garments.push_back(g);
    }
    const std::size_t n = next.x.size();
    next.v.assign(n, V3d{});
    next.fExt.assign(n, V3d{});
    next.pinned.assign(n, 0);
    next.mass.assign(n, 0.0);
    for (uint32_t k = 0; k < scene.pin_count; ++k) {
      const uint32_t p = scene.pin_particles[k];
      if (p >= n) throw std::out_of_range("pin particle out of range");
      const V3d pos = next.state({scene.pin_positions[3 * k], scene.pin_positions[3 * k + 1], scene.pin_positions[3 * k + 2]});
      next.pinned[p] = 1;
      next.pins.push_back({p, pos});
      next.x[p] = pos;
    }
    for (uint32_t k = 0; k < scene.force_count; ++k) {
      const uint32_t p = scene.force_particles[k];
      if (p >= n) throw std::out_of_range("force particle out of range");
      next.fExt[p] += V3d{scene.forces[3 * k], scene.forces[3 * k + 1], scene.forces[3 * k + 2]};
    }
    for (uint32_t i = 0; i < n; ++i) next.updateMass(i);
    for (std::size_t hgi = 0; hgi < next.hinges.size(); ++hgi) next.hinges[hgi].K = next.hingeStiffness(hgi);
    next.buildStructure();
    return next;
  }

  void updateFabric(const std::string& id, const drape_fabric* pieceFabric, uint32_t count) {
    auto& g = garments[garmentIndex(id)];
    if (count != g.pieceCount) throw std::invalid_argument("one fabric per pattern piece required");
    for (uint32_t p = 0; p < count; ++p) fabrics[g.fabricOffset + p] = fabricFrom(pieceFabric[p]);
    for (uint32_t i = g.offset; i < g.offset + g.count; ++i) updateMass(i);
    for (std::size_t hgi = 0; hgi < hinges.size(); ++hgi) {
      const auto fi = hingeSides[hgi][0].fabric;
      if (fi >= g.fabricOffset && fi < g.fabricOffset + g.pieceCount) hinges[hgi].K = hingeStiffness(hgi);
    }
  }

  void setPhase(const std::string& id, Phase phase) {
    const auto gi = garmentIndex(id);
    auto& g = garments[gi];
    g.phase = phase;
    if (phase == Assembling) {
      g.assemblyTime = 0;
      for (auto& sp : seams)
        if (sp.garment == gi) sp.startGap = static_cast<float>(gap(sp.a, sp.b));
    }
  }

  drape_stats stats() const {
    drape_stats st{};
    double sumV2 = 0;
    std::size_t moving = 0;
    for (std::size_t i = 0; i < x.size(); ++i) {
      if (!finite(x[i]) || !finite(v[i])) st.has_non_finite = 1;
      if (pinned[i]) continue;
      const double v2 = sqnorm(v[i]);
      st.kinetic_energy += 0.5 * mass[i] * v2;
      sumV2 += v2;
      ++moving;
    }
    st.rms_speed = moving ? std::sqrt(sumV2 / static_cast<double>(moving)) : 0.0;
    for (const auto& sp : seams) st.max_seam_gap = std::max(st.max_seam_gap, gap(sp.a, sp.b));
    if (hasBody) {
      for (const auto& p : x) st.max_body_penetration = std::max(st.max_body_penetration, -body.sample(p));
    }
    return st;
  }
};

// ---------------------------------------------------------------------------------------------------------------
// Solver (cpu_solver.cpp:34-338).

struct Solver {
  Model m;
  std::vector<V3d> contactNormal;
  std::vector<double> contactOffset, frictionLambda;
  double substepH = 1.0 / 60.0;
  std::vector<uint8_t> contactNear, contactActive;
  std::vector<V3d> xd, xStart, y, grad, step, r, z, p, ap, trial, apFull, resid;
  std::vector<M3> blocks, precond;
  drape_counters counters{};
  bool built = false;

  void allocate() {
    const std::size_t n = m.x.size();
    blocks.assign(m.colIndex.size(), M3{});
    precond.assign(n, M3::identity());
    for (auto* vec : {&xd, &xStart, &y, &grad, &step, &r, &z, &p, &ap, &trial, &apFull, &resid}) vec->assign(n, V3d{});
    contactNormal.assign(n, V3d{});
    contactOffset.assign(n, 0.0);
    frictionLambda.assign(n, 0.0);
    contactNear.assign(n, 0);
    contactActive.assign(n, 0);
    buildGatherLists();
  }

  double contactGap(std::size_t i, V3d pos) const { return contactOffset[i] - dot(contactNormal[i], pos - xStart[i]); }
  void filter(std::vector<V3d>& vec) const {
    for (std::size_t i = 0; i < vec.size(); ++i)
      if (contactActive[i]) vec[i] -= contactNormal[i] * dot(contactNormal[i], vec[i]);
  }

  // Parallel evaluation with the serial oracle's arithmetic, bit for bit. The reference CpuSolver scatters each term's
  // gradient and Hessian blocks into the shared arrays in term order (cpu_solver.cpp:76-90, :92-145) and sums the
  // energy and the dot products in index order (:161-165). Here every term is evaluated independently (in parallel)
  // into its own record; each block slot and each particle then adds its contributions in exactly the order the
  // serial scatter would (inertia first, then stretch, hinge and seam terms in term order, friction last), and every
  // energy and dot-product sum runs serially in index order over per-item values computed in parallel. The results
  // are therefore identical for any thread count, the single-threaded run included.
  std::vector<TermEval<3>> stretchEval;
  std::vector<TermEval<4>> hingeEval;
  std::vector<TermEval<2>> seamEval;
  std::vector<TermEval<1>> frictionEval;
  std::vector<double> eInertia, eStretch, eHinge, eSeam, eFriction, dotTmp;
  // Contribution lists: entry = kind (2 bits: 0 stretch, 1 hinge, 2 seam) << 30 | local (4 bits) << 26 | term.
  std::vector<uint32_t> slotListStart, slotList, gradListStart, gradList;
  std::vector<int32_t> slotDiag;  // the particle whose diagonal block a slot holds, or -1

  static uint32_t entry(uint32_t kind, uint32_t local, uint32_t term) { return kind << 30 | local << 26 | term; }

  template <class Fn>
  void forEachContribution(Fn&& fn) const {  // fn(kind, term, a, b, N, slot): in the serial scatter's order
    for (std::size_t k = 0; k < m.stretch.size(); ++k)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) fn(0u, k, a, b, 3, m.stretchSlots[k][a * 3 + b], m.stretch[k].v[a]);
    for (std::size_t k = 0; k < m.hinges.size(); ++k)
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) fn(1u, k, a, b, 4, m.hingeSlots[k][a * 4 + b], m.hinges[k].v[a]);
    for (std::size_t k = 0; k < m.seams.size(); ++k) {
      const uint32_t ab[2] = {m.seams[k].a, m.seams[k].b};
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) fn(2u, k, a, b, 2, m.seamSlots[k][a * 2 + b], ab[a]);
    }
  }

  void buildGatherLists() {
    const std::size_t n = m.x.size(), B = m.colIndex.size();
    if (m.stretch.size() >= (1u << 26) || m.hinges.size() >= (1u << 26) || m.seams.size() >= (1u << 26))
      throw std::invalid_argument("oracle: too many terms for the gather lists");
    slotListStart.assign(B + 1, 0);
    gradListStart.assign(n + 1, 0);
    forEachContribution([&](uint32_t, std::size_t, int, int b, int, uint32_t slot, uint32_t va) {
      ++slotListStart[slot + 1];
      if (b == 0) ++gradListStart[va + 1];
    });
    for (std::size_t s = 0; s < B; ++s) slotListStart[s + 1] += slotListStart[s];
    for (std::size_t i = 0; i < n; ++i) gradListStart[i + 1] += gradListStart[i];
    slotList.assign(slotListStart[B], 0);
    gradList.assign(gradListStart[n], 0);
    std::vector<uint32_t> sFill(slotListStart.begin(), slotListStart.end() - 1);
    std::vector<uint32_t> gFill(gradListStart.begin(), gradListStart.end() - 1);
    forEachContribution([&](uint32_t kind, std::size_t k, int a, int b, int N, uint32_t slot, uint32_t va) {
      slotList[sFill[slot]++] = entry(kind, static_cast<uint32_t>(a * N + b), static_cast<uint32_t>(k));
      if (b == 0) gradList[gFill[va]++] = entry(kind, static_cast<uint32_t>(a), static_cast<uint32_t>(k));
    });
    slotDiag.assign(B, -1);
    for (std::size_t i = 0; i < n; ++i) slotDiag[m.diagSlot[i]] = static_cast<int32_t>(i);
    stretchEval.resize(m.stretch.size());
    hingeEval.resize(m.hinges.size());
    seamEval.resize(m.seams.size());
    frictionEval.resize(n);
    eInertia.resize(n);
    eStretch.resize(m.stretch.size());
    eHinge.resize(m.hinges.size());
    eSeam.resize(m.seams.size());
    eFriction.resize(n);
    dotTmp.resize(n);
  }

  const M3& hessOf(uint32_t e) const {
    const uint32_t kind = e >> 30, local = (e >> 26) & 15u, k = e & ((1u << 26) - 1);
    if (kind == 0) return stretchEval[k].hess[local / 3][local % 3];
    if (kind == 1) return hingeEval[k].hess[local / 4][local % 4];
    return seamEval[k].hess[local / 2][local % 2];
  }
  const V3d& gradOf(uint32_t e) const {
    const uint32_t kind = e >> 30, local = (e >> 26) & 15u, k = e & ((1u << 26) - 1);
    if (kind == 0) return stretchEval[k].grad[local];
    if (kind == 1) return hingeEval[k].grad[local];
    return seamEval[k].grad[local];
  }

  template <int N>
  static void gatherTerm(const uint32_t* vs, const std::vector<V3d>& pos, V3d* xs) {
    for (int a = 0; a < N; ++a) xs[a] = pos[vs[a]];
  }

  double evaluate(const std::vector<V3d>& pos, double invH2, bool withDerivatives) {
    const std::ptrdiff_t n = static_cast<std::ptrdiff_t>(pos.size());
    const std::ptrdiff_t S = static_cast<std::ptrdiff_t>(m.stretch.size());
    const std::ptrdiff_t H = static_cast<std::ptrdiff_t>(m.hinges.size());
    const std::ptrdiff_t K = static_cast<std::ptrdiff_t>(m.seams.size());
    const double limitScale = m.settings.strainLimitStiffnessScale;
    const double slipEps = m.settings.frictionSlipSpeed * substepH;
#pragma omp parallel if (n + S + H >= kParallelMin)
    {
#pragma omp for schedule(static) nowait
      for (std::ptrdiff_t i = 0; i < n; ++i) {
        eInertia[i] = 0;
        if (m.pinned[i]) continue;
        const double k = m.mass[i] * invH2;
        const V3d d = pos[i] - y[i];
        eInertia[i] = 0.5 * k * sqnorm(d);
      }
#pragma omp for schedule(static) nowait
      for (std::ptrdiff_t k = 0; k < S; ++k) {
        const auto& t = m.stretch[k];
        V3d xs[3];
        gatherTerm<3>(t.v.data(), pos, xs);
        TermEval<3> local;
        TermEval<3>& te = withDerivatives ? (stretchEval[k] = TermEval<3>{}) : local;
        evalStretchTerm(t.dmInv, t.area, xs, m.fabrics[t.fabric], limitScale, te);
        eStretch[k] = te.energy;
      }
#pragma omp for schedule(static) nowait
      for (std::ptrdiff_t k = 0; k < H; ++k) {
        const auto& h = m.hinges[k];
        V3d xs[4];
        gatherTerm<4>(h.v.data(), pos, xs);
        TermEval<4> local;
        TermEval<4>& te = withDerivatives ? (hingeEval[k] = TermEval<4>{}) : local;
        evalHingeTerm(h.K, h.restAngle, xs, te);
        eHinge[k] = te.energy;
      }
#pragma omp for schedule(static) nowait
      for (std::ptrdiff_t k = 0; k < K; ++k) {
        const auto& s = m.seams[k];
        const uint32_t ab[2] = {s.a, s.b};
        V3d xs[2];
        gatherTerm<2>(ab, pos, xs);
        TermEval<2> local;
        TermEval<2>& te = withDerivatives ? (seamEval[k] = TermEval<2>{}) : local;
        evalSeamTerm(xs, m.seamTarget(s), m.settings.seamStiffness, te);
        eSeam[k] = te.energy;
      }
#pragma omp for schedule(static)
      for (std::ptrdiff_t i = 0; i < n; ++i) {
        eFriction[i] = 0;
        if (frictionLambda[i] <= 0) continue;
        TermEval<1> local;
        TermEval<1>& te = withDerivatives ? (frictionEval[i] = TermEval<1>{}) : local;
        evalFrictionTerm(pos[i], xStart[i], contactNormal[i], m.fabrics[m.pFabric[i]].friction * frictionLambda[i],
                         slipEps, te);
        eFriction[i] = te.energy;
      }
      if (withDerivatives) {
        const std::ptrdiff_t B = static_cast<std::ptrdiff_t>(blocks.size());
#pragma omp for schedule(static) nowait
        for (std::ptrdiff_t s = 0; s < B; ++s) {
          M3 acc{};
          const int32_t i = slotDiag[s];
          if (i >= 0 && !m.pinned[i]) acc += (m.mass[i] * invH2) * M3::identity();
          for (uint32_t e = slotListStart[s]; e < slotListStart[s + 1]; ++e) acc += hessOf(slotList[e]);
          if (i >= 0 && frictionLambda[i] > 0) acc += frictionEval[i].hess[0][0];
          blocks[s] = acc;
        }
#pragma omp for schedule(static)
        for (std::ptrdiff_t i = 0; i < n; ++i) {
          V3d acc{};
          if (!m.pinned[i]) acc += (m.mass[i] * invH2) * (pos[i] - y[i]);
          for (uint32_t e = gradListStart[i]; e < gradListStart[i + 1]; ++e) acc += gradOf(gradList[e]);
          if (frictionLambda[i] > 0) acc += frictionEval[i].grad[0];
          grad[i] = m.pinned[i] ? V3d{} : acc;
        }
      }
    }
    // The energy in the serial order: inertia (unpinned particles), stretch, hinge, seam terms, friction.
    double energy = 0;
    for (std::ptrdiff_t i = 0; i < n; ++i)
      if (!m.pinned[i]) energy += eInertia[i];
    for (std::ptrdiff_t k = 0; k < S; ++k) energy += eStretch[k];
    for (std::ptrdiff_t k = 0; k < H; ++k) energy += eHinge[k];
    for (std::ptrdiff_t k = 0; k < K; ++k) energy += eSeam[k];
    for (std::ptrdiff_t i = 0; i < n; ++i)
      if (frictionLambda[i] > 0) energy += eFriction[i];
    return energy;
  }

  void multiply(const std::vector<V3d>& in, std::vector<V3d>& out) const {
    const std::ptrdiff_t n = static_cast<std::ptrdiff_t>(in.size());
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
    for (std::ptrdiff_t i = 0; i < n; ++i) {
      V3d acc;
      if (!m.pinned[i]) {
        for (uint32_t s = m.rowStart[i]; s < m.rowStart[i + 1]; ++s) {
          const auto j = m.colIndex[s];
          if (!m.pinned[j]) acc += blocks[s] * in[j];
        }
      }
      out[i] = acc;
    }
  }

  // a . b summed in index order (the per-particle products in parallel, the sum serial).
  double vdot(const std::vector<V3d>& a, const std::vector<V3d>& b) {
    const std::ptrdiff_t n = static_cast<std::ptrdiff_t>(a.size());
    if (dotTmp.size() < a.size()) dotTmp.resize(a.size());
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
    for (std::ptrdiff_t i = 0; i < n; ++i) dotTmp[i] = dot(a[i], b[i]);
    double s = 0;
    for (std::ptrdiff_t i = 0; i < n; ++i) s += dotTmp[i];
    return s;
  }

  void filterRow(std::vector<V3d>& vec, std::ptrdiff_t i) const {
    if (contactActive[i]) vec[i] -= contactNormal[i] * dot(contactNormal[i], vec[i]);
  }

  void solveLinear() {
    const std::ptrdiff_t n = static_cast<std::ptrdiff_t>(grad.size());
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
    for (std::ptrdiff_t i = 0; i < n; ++i) {
      if (m.pinned[i]) {
        precond[i] = M3{};
      } else {
        bool ok = false;
        const M3 inv = invertSymmetric(blocks[m.diagSlot[i]], ok);
        precond[i] = ok ? inv : M3::identity();
      }
      step[i] = V3d{};
      resid[i] = -grad[i];
      r[i] = resid[i];
      filterRow(r, i);
      z[i] = precond[i] * r[i];
      filterRow(z, i);
      p[i] = z[i];
    }
    double rz = vdot(r, z);
    const double r0 = std::sqrt(vdot(r, r));
    for (int it = 0; r0 > 0 && it < m.settings.maxCgIterations; ++it) {
      multiply(p, apFull);
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
      for (std::ptrdiff_t i = 0; i < n; ++i) {
        ap[i] = apFull[i];
        filterRow(ap, i);
      }
      const double pAp = vdot(p, ap);
      if (!(pAp > 0)) break;
      const double alpha = rz / pAp;
      ++counters.cg_iterations;
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
      for (std::ptrdiff_t i = 0; i < n; ++i) {
        step[i] += alpha * p[i];
        r[i] -= alpha * ap[i];
        resid[i] -= alpha * apFull[i];
      }
      if (std::sqrt(vdot(r, r)) <= m.settings.cgTolerance * r0) break;
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
      for (std::ptrdiff_t i = 0; i < n; ++i) {
        z[i] = precond[i] * r[i];
        filterRow(z, i);
      }
      const double rzNew = vdot(r, z);
      const double beta = rzNew / rz;
      rz = rzNew;
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
      for (std::ptrdiff_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
    for (std::ptrdiff_t i = 0; i < n; ++i)
      m.contactForce[i] = contactActive[i] ? std::max(0.0, -dot(resid[i], contactNormal[i])) : 0.0;
  }

  double evaluateWithContact(double invH2) {
    const std::ptrdiff_t n = static_cast<std::ptrdiff_t>(xd.size());
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
    for (std::ptrdiff_t i = 0; i < n; ++i) {
      if (!contactNear[i]) continue;
      const double c = contactGap(i, xd[i]);
      if (c > -kContactSnap) contactActive[i] = 1;
      if (contactActive[i] && c > 0) xd[i] += c * contactNormal[i];
    }
    const double e = evaluate(xd, invH2, true);
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
    for (std::ptrdiff_t i = 0; i < n; ++i)
      if (contactActive[i] && dot(grad[i], contactNormal[i]) < 0) contactActive[i] = 0;
    return e;
  }

  // Predict and contact setup (cpu_solver.cpp:234-263).
  void beginSubstep(double h) {
    const V3d gravity = m.settings.gravity;
    const std::ptrdiff_t n = static_cast<std::ptrdiff_t>(m.x.size());
    substepH = h;
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
    for (std::ptrdiff_t i = 0; i < n; ++i) {
      xStart[i] = m.x[i];
      const V3d vel = m.v[i];
      if (m.pinned[i]) {
        y[i] = xStart[i];
        xd[i] = xStart[i];
      } else {
        const V3d g = m.garments[m.pGarment[i]].phase == Settling ? gravity : V3d{};
        y[i] = xStart[i] + h * vel + h * h * (g + m.fExt[i] / m.mass[i]);
        xd[i] = xStart[i] + h * vel;
      }
      contactNear[i] = 0;
      contactActive[i] = 0;
      frictionLambda[i] = 0;
      const double lastForce = m.contactForce[i];
      m.contactForce[i] = 0;
      if (!m.hasBody || m.pinned[i]) continue;
      const double radius = m.contactRadius(i);
      const double phi = m.body.sample(xStart[i]);
      if (phi >= radius + kContactReach) continue;
      const V3d normal = m.body.gradient(xStart[i]);
      if (isZero(normal)) continue;
      contactNear[i] = 1;
      contactNormal[i] = normal;
      contactOffset[i] = radius - phi;
      frictionLambda[i] = lastForce;
    }
  }

  void substep(double h, int newtonIterations) {
    const double invH2 = 1.0 / (h * h);
    const std::ptrdiff_t n = static_cast<std::ptrdiff_t>(m.x.size());
    ++counters.substeps;
    beginSubstep(h);
    for (int it = 0; it < newtonIterations; ++it) {
      ++counters.newton_iterations;
      const double e0 = evaluateWithContact(invH2);
      solveLinear();
      const double slope = vdot(grad, step);
      if (!(slope < 0)) break;
      double alpha = 1.0;
      for (int ls = 0; ls < 20; ++ls) {
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
        for (std::ptrdiff_t i = 0; i < n; ++i) trial[i] = xd[i] + alpha * step[i];
        if (evaluate(trial, invH2, false) <= e0 + 1e-4 * alpha * slope) break;
        alpha *= 0.5;
        ++counters.line_search_halvings;
      }
      double maxMove = 0;  // a maximum: the same for any grouping
#pragma omp parallel for schedule(static) reduction(max : maxMove) if (n >= kParallelMin)
      for (std::ptrdiff_t i = 0; i < n; ++i) {
        xd[i] += alpha * step[i];
        const V3d d = alpha * step[i];
        maxMove = std::max(maxMove, std::max(std::abs(d.x), std::max(std::abs(d.y), std::abs(d.z))));
      }
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
      for (std::ptrdiff_t i = 0; i < n; ++i) frictionLambda[i] = contactActive[i] ? m.contactForce[i] : 0.0;
      if (maxMove < 1e-9) break;
    }
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
    for (std::ptrdiff_t i = 0; i < n; ++i) {
      m.x[i] = m.state(xd[i]);
      if (!m.hasBody || m.pinned[i]) continue;
      const double radius = m.contactRadius(i);
      if (m.body.sample(m.x[i]) >= radius - kContactSnap) continue;
      const bool flat = isZero(m.body.gradient(m.x[i]));
      if (m.fp64) {
        if (flat) {
          m.x[i] = landOnBodyD(m.body, radius, xStart[i], m.x[i]);
        } else {
          collideBodyD(m.body, radius, m.fabrics[m.pFabric[i]].friction, xStart[i], m.x[i]);
        }
      } else {
        if (flat) {
          m.x[i] = tod(landOnBodyF(m.body, static_cast<float>(radius), tof(xStart[i]), tof(m.x[i])));
        } else {
          V3f xf = tof(m.x[i]);
          collideBodyF(m.body, static_cast<float>(radius), static_cast<float>(m.fabrics[m.pFabric[i]].friction),
                       tof(xStart[i]), xf);
          m.x[i] = tod(xf);
        }
      }
    }
    for (const auto& [i, pos] : m.pins) m.x[i] = pos;
#pragma omp parallel for schedule(static) if (n >= kParallelMin)
    for (std::ptrdiff_t i = 0; i < n; ++i) {
      double c = m.settings.dampingScale * m.fabrics[m.pFabric[i]].damping;
      if (m.garments[m.pGarment[i]].phase == Assembling) c += m.settings.assemblyExtraDamping;
      if (m.fp64) {
        m.v[i] = ((m.x[i] - xStart[i]) / h) * std::max(0.0, 1.0 - c * h);
      } else {
        const V3f vel = tof((m.x[i] - xStart[i]) / h);
        m.v[i] = tod(vel * static_cast<float>(std::max(0.0, 1.0 - c * h)));
      }
    }
    for (auto& g : m.garments)
      if (g.phase == Assembling) g.assemblyTime += h;
  }
  void advance(double dt, int substeps, int iterations) {
    const int s = std::max(1, substeps);
    const double h = dt / s;
    const int its = std::max(1, iterations);
    for (int k = 0; k < s; ++k) substep(h, its);
  }
};

}  // namespace oracle

