// ORACLE — test infrastructure only.
//
// CPU restatement of bakeCollisionField (libs/avatar/src/collision_bake.cpp:17-208) and isClosedManifold
// (libs/core/src/triangle_mesh.cpp:16-28), serial as the reference: triangles in order, each visiting the samples of
// its box grown by the band, keeping a sample's nearest triangle when strictly closer (the first reaching the
// minimum wins), the sign from the nearest feature's pseudonormal, a breadth-first flood fill from the grid boundary
// through samples farther than the band, and the per-component union by minimum. Plain doubles in the reference's
// operation order (Eigen's 3-vector dot and squared norm sum left to right; normalized() divides by the norm); the
// reference itself needs Eigen 3.4, absent here.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <deque>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace obake {

struct V3 {
  double x = 0, y = 0, z = 0;
};
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 normalized(V3 a) {
  const double z = dot(a, a);
  if (!(z > 0)) return a;
  const double n = std::sqrt(z);
  return {a.x / n, a.y / n, a.z / n};
}

struct Mesh {
  std::vector<V3> v;
  std::vector<std::array<uint32_t, 3>> t;
};

inline bool closedManifold(const Mesh& m) {
  if (m.t.empty()) return false;
  std::map<std::pair<uint32_t, uint32_t>, int> directed;
  for (const auto& t : m.t)
    for (int k = 0; k < 3; ++k) ++directed[{t[k], t[(k + 1) % 3]}];
  for (const auto& [e, count] : directed) {
    if (count != 1) return false;
    auto it = directed.find({e.second, e.first});
    if (it == directed.end() || it->second != 1) return false;
  }
  return true;
}

enum class Feature { VertexA, VertexB, VertexC, EdgeAB, EdgeBC, EdgeCA, Face };

inline V3 closestPoint(V3 p, V3 a, V3 b, V3 c, Feature& f) {
  const V3 ab = b - a, ac = c - a, ap = p - a;
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) {
    f = Feature::VertexA;
    return a;
  }
  const V3 bp = p - b;
  const double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) {
    f = Feature::VertexB;
    return b;
  }
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    f = Feature::EdgeAB;
    return a + (d1 / (d1 - d3)) * ab;
  }
  const V3 cp = p - c;
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) {
    f = Feature::VertexC;
    return c;
  }
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    f = Feature::EdgeCA;
    return a + (d2 / (d2 - d6)) * ac;
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    f = Feature::EdgeBC;
    return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
  }
  const double denom = 1.0 / (va + vb + vc);
  f = Feature::Face;
  return (a + (vb * denom) * ab) + (vc * denom) * ac;
}

struct Pseudonormals {
  std::vector<V3> face, vertex;
  std::map<std::pair<uint32_t, uint32_t>, V3> edge;
  explicit Pseudonormals(const Mesh& m) : face(m.t.size()), vertex(m.v.size()) {
    for (size_t t = 0; t < m.t.size(); ++t) {
      const auto& tri = m.t[t];
      const V3 a = m.v[tri[0]], b = m.v[tri[1]], c = m.v[tri[2]];
      face[t] = normalized(cross(b - a, c - a));
      for (int k = 0; k < 3; ++k) {
        const V3 p = m.v[tri[k]];
        const V3 e1 = normalized(m.v[tri[(k + 1) % 3]] - p);
        const V3 e2 = normalized(m.v[tri[(k + 2) % 3]] - p);
        vertex[tri[k]] = vertex[tri[k]] + std::acos(std::clamp(dot(e1, e2), -1.0, 1.0)) * face[t];
        auto key = std::minmax(tri[k], tri[(k + 1) % 3]);
        auto [it, inserted] = edge.try_emplace(key, V3{});
        it->second = it->second + face[t];
      }
    }
  }
  V3 of(const Mesh& m, size_t t, Feature f) const {
    const auto& tri = m.t[t];
    switch (f) {
      case Feature::VertexA: return vertex[tri[0]];
      case Feature::VertexB: return vertex[tri[1]];
      case Feature::VertexC: return vertex[tri[2]];
      case Feature::EdgeAB: return edge.at(std::minmax(tri[0], tri[1]));
      case Feature::EdgeBC: return edge.at(std::minmax(tri[1], tri[2]));
      case Feature::EdgeCA: return edge.at(std::minmax(tri[2], tri[0]));
      case Feature::Face: return face[t];
    }
    return face[t];
  }
};

struct Field {
  double origin[3];
  int dims[3];
  std::vector<float> values;
};

inline Field bake(const std::vector<Mesh>& components, double cell, double padding, double band) {
  const double inf = std::numeric_limits<double>::infinity();
  V3 lo{inf, inf, inf}, hi{-inf, -inf, -inf};
  for (size_t c = 0; c < components.size(); ++c) {
    if (!closedManifold(components[c]))
      throw std::invalid_argument("collision component " + std::to_string(c) + " is not a closed manifold");
    for (const auto& v : components[c].v) {
      lo = {std::min(lo.x, v.x), std::min(lo.y, v.y), std::min(lo.z, v.z)};
      hi = {std::max(hi.x, v.x), std::max(hi.y, v.y), std::max(hi.z, v.z)};
    }
  }
  Field f;
  f.origin[0] = lo.x - padding;
  f.origin[1] = lo.y - padding;
  f.origin[2] = lo.z - padding;
  const double ext[3] = {(hi.x - lo.x) + 2 * padding, (hi.y - lo.y) + 2 * padding, (hi.z - lo.z) + 2 * padding};
  for (int a = 0; a < 3; ++a) f.dims[a] = static_cast<int>(std::ceil(ext[a] / cell)) + 1;
  const size_t nx = f.dims[0], ny = f.dims[1], nz = f.dims[2], count = nx * ny * nz;
  f.values.assign(count, static_cast<float>(band));
  auto index = [&](size_t x, size_t y, size_t z) { return (z * ny + y) * nx + x; };
  auto position = [&](size_t x, size_t y, size_t z) {
    return V3{f.origin[0] + cell * static_cast<double>(x), f.origin[1] + cell * static_cast<double>(y),
              f.origin[2] + cell * static_cast<double>(z)};
  };
  auto cellRange = [&](double minV, double maxV, int axis, size_t& i0, size_t& i1) {
    const double o = f.origin[axis];
    i0 = static_cast<size_t>(std::max(0.0, std::ceil((minV - o) / cell)));
    i1 = static_cast<size_t>(std::min<double>(f.dims[axis] - 1, std::floor((maxV - o) / cell)));
  };
  std::vector<double> dist2(count);
  std::vector<int8_t> sign(count);
  std::vector<uint8_t> outside(count);
  for (const auto& mesh : components) {
    std::fill(dist2.begin(), dist2.end(), inf);
    std::fill(sign.begin(), sign.end(), 0);
    const Pseudonormals normals(mesh);
    for (size_t t = 0; t < mesh.t.size(); ++t) {
      const auto& tri = mesh.t[t];
      const V3 a = mesh.v[tri[0]], b = mesh.v[tri[1]], c = mesh.v[tri[2]];
      const V3 tmin{std::min(std::min(a.x, b.x), c.x), std::min(std::min(a.y, b.y), c.y),
                    std::min(std::min(a.z, b.z), c.z)};
      const V3 tmax{std::max(std::max(a.x, b.x), c.x), std::max(std::max(a.y, b.y), c.y),
                    std::max(std::max(a.z, b.z), c.z)};
      size_t r[3][2];
      cellRange(tmin.x - band, tmax.x + band, 0, r[0][0], r[0][1]);
      cellRange(tmin.y - band, tmax.y + band, 1, r[1][0], r[1][1]);
      cellRange(tmin.z - band, tmax.z + band, 2, r[2][0], r[2][1]);
      for (size_t z = r[2][0]; z <= r[2][1]; ++z)
        for (size_t y = r[1][0]; y <= r[1][1]; ++y)
          for (size_t x = r[0][0]; x <= r[0][1]; ++x) {
            const size_t i = index(x, y, z);
            const V3 p = position(x, y, z);
            const V3 gap{std::max(std::max(tmin.x - p.x, p.x - tmax.x), 0.0),
                         std::max(std::max(tmin.y - p.y, p.y - tmax.y), 0.0),
                         std::max(std::max(tmin.z - p.z, p.z - tmax.z), 0.0)};
            if (dot(gap, gap) >= dist2[i]) continue;
            Feature fe;
            const V3 q = closestPoint(p, a, b, c, fe);
            const double d2 = dot(p - q, p - q);
            if (d2 < dist2[i]) {
              dist2[i] = d2;
              sign[i] = dot(p - q, normals.of(mesh, t, fe)) >= 0 ? 1 : -1;
            }
          }
    }
    std::fill(outside.begin(), outside.end(), 0);
    std::deque<size_t> queue;
    auto seed = [&](size_t x, size_t y, size_t z) {
      const size_t i = index(x, y, z);
      if (!outside[i] && dist2[i] > band * band) {
        outside[i] = 1;
        queue.push_back(i);
      }
    };
    for (size_t z = 0; z < nz; ++z)
      for (size_t y = 0; y < ny; ++y)
        for (size_t x = 0; x < nx; ++x)
          if (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1) seed(x, y, z);
    while (!queue.empty()) {
      const size_t i = queue.front();
      queue.pop_front();
      const size_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
      if (x > 0) seed(x - 1, y, z);
      if (x + 1 < nx) seed(x + 1, y, z);
      if (y > 0) seed(x, y - 1, z);
      if (y + 1 < ny) seed(x, y + 1, z);
      if (z > 0) seed(x, y, z - 1);
      if (z + 1 < nz) seed(x, y, z + 1);
    }
    for (size_t i = 0; i < count; ++i) {
      double v;
      if (dist2[i] <= band * band) {
        v = sign[i] * std::sqrt(dist2[i]);
      } else {
        v = outside[i] ? band : -band;
      }
      f.values[i] = std::min(f.values[i], static_cast<float>(std::clamp(v, -band, band)));
    }
  }
  return f;
}

}  // namespace obake
