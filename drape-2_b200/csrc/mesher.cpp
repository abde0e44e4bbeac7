// Pattern -> simulation mesh (include/drape_mesh.h) on the host, for the reference's buildSimMesh contract
// (libs/garment/src/sim_mesh_builder.cpp:196-323; pattern rules libs/garment/src/validate.cpp:25-87).
//
// Per piece: validate the pattern; walk the outline once into boundary stations (each seam side one run with its
// seam's station count, the free stretches between seam sides split at the corners into runs of ceil(length / h)
// steps); fill the interior with a grain-aligned hexagonal lattice, row by row in the grain frame, keeping points
// inside the outline and at least h / 2 from it; triangulate stations and lattice with the outline as constraint and
// drop the outside; relax the interior vertices toward their incident triangles' centroids without letting any
// incident angle shrink; vertex areas are a third of the incident triangle areas; seam pairs join station k of the
// two sides.
//
// The constrained Delaunay triangulation is this file's own (the reference uses the CDT 1.4.5 library, absent here):
// Lawson incremental insertion (point location by walking, split of the containing triangle or edge, legalising flips
// with the in-circle test), constraint edges recovered by flipping the edges that cross them (Sloan 1993), then a
// flood fill from the enclosing triangle's corners that stops at constraint edges removes the outside. Vertex and
// triangle order are this file's.
#include "../../include/drape_mesh.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace dmesh {

struct V2 {
  double x = 0, y = 0;
};
inline V2 operator+(V2 a, V2 b) { return {a.x + b.x, a.y + b.y}; }
inline V2 operator-(V2 a, V2 b) { return {a.x - b.x, a.y - b.y}; }
inline V2 operator*(double s, V2 a) { return {s * a.x, s * a.y}; }
inline double dot(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
inline double norm(V2 a) { return std::sqrt(dot(a, a)); }
inline V2 unit(V2 a) {
  const double n = norm(a);
  return n > 0 ? V2{a.x / n, a.y / n} : a;
}

class MeshError : public std::invalid_argument {
 public:
  using std::invalid_argument::invalid_argument;
};

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------------------------------
// Cubic Bezier outline with arc-length positions (libs/core/src/bezier.cpp, outline.cpp): each segment's length
// table holds 256 intervals, each integrated with 5-point Gauss-Legendre quadrature of the speed.

struct Cubic {
  V2 p[4];
  V2 point(double t) const {
    const double u = 1 - t;
    return (u * u * u) * p[0] + (3 * u * u * t) * p[1] + (3 * u * t * t) * p[2] + (t * t * t) * p[3];
  }
  V2 derivative(double t) const {
    const double u = 1 - t;
    return (3 * u * u) * (p[1] - p[0]) + (6 * u * t) * (p[2] - p[1]) + (3 * t * t) * (p[3] - p[2]);
  }
};

class LengthTable {
 public:
  explicit LengthTable(const Cubic& c, int intervals = 256) : cum_(intervals + 1, 0.0) {
    static const double x[5] = {-0.9061798459386640, -0.5384693101056831, 0.0, 0.5384693101056831,
                                0.9061798459386640};
    static const double w[5] = {0.2369268850561891, 0.4786286704993665, 0.5688888888888889, 0.4786286704993665,
                                0.2369268850561891};
    for (int i = 0; i < intervals; ++i) {
      const double a = static_cast<double>(i) / intervals, b = static_cast<double>(i + 1) / intervals;
      const double half = 0.5 * (b - a), mid = 0.5 * (a + b);
      double s = 0;
      for (int k = 0; k < 5; ++k) s += w[k] * norm(c.derivative(mid + half * x[k]));
      cum_[i + 1] = cum_[i] + s * half;
    }
  }
  double length() const { return cum_.back(); }
  // Curve parameter at arc length s along the segment (linear inside an interval).
  double paramAt(double s) const {
    const double total = length();
    if (total <= 0) return 0;
    s = std::clamp(s, 0.0, total);
    const auto it = std::upper_bound(cum_.begin(), cum_.end(), s);
    if (it == cum_.end()) return 1.0;
    const std::size_t i = static_cast<std::size_t>(it - cum_.begin()) - 1;
    const double s0 = cum_[i], s1 = cum_[i + 1];
    const double f = s1 > s0 ? (s - s0) / (s1 - s0) : 0.0;
    return (static_cast<double>(i) + f) / static_cast<double>(cum_.size() - 1);
  }

 private:
  std::vector<double> cum_;
};

struct Outline {
  std::vector<Cubic> seg;
  std::vector<LengthTable> len;
  std::vector<double> start{0.0};  // start[i]: arc length at segment i; back(): perimeter

  void add(const Cubic& c) {
    seg.push_back(c);
    len.emplace_back(c);
    start.push_back(start.back() + len.back().length());
  }
  double perimeter() const { return start.back(); }
  bool closed(double tol = 1e-9) const {
    if (seg.empty()) return false;
    for (std::size_t i = 0; i < seg.size(); ++i)
      if (norm(seg[i].p[3] - seg[(i + 1) % seg.size()].p[0]) > tol) return false;
    return true;
  }
  V2 pointAt(double s) const {
    s = std::clamp(s, 0.0, perimeter());
    if (s >= perimeter()) return seg[0].point(0.0);
    const auto it = std::upper_bound(start.begin(), start.end(), s);
    const std::size_t i = static_cast<std::size_t>(it - start.begin()) - 1;
    return seg[i].point(len[i].paramAt(s - start[i]));
  }
  // Points every <= spacing along each segment (arc-length spaced), segment starts included.
  std::vector<V2> polyline(double spacing) const {
    std::vector<V2> out;
    for (std::size_t i = 0; i < seg.size(); ++i) {
      const double L = len[i].length();
      const int n = std::max(1, static_cast<int>(std::ceil(L / spacing)));
      for (int k = 0; k < n; ++k) out.push_back(seg[i].point(len[i].paramAt(L * k / n)));
    }
    return out;
  }
};

// ---------------------------------------------------------------------------------------------------------------
// Polygon predicates (libs/core/src/polygon.cpp).

double signedArea(const std::vector<V2>& poly) {
  double a = 0;
  for (std::size_t i = 0; i < poly.size(); ++i) {
    const V2 p = poly[i], q = poly[(i + 1) % poly.size()];
    a += p.x * q.y - q.x * p.y;
  }
  return 0.5 * a;
}

double cross3(V2 a, V2 b, V2 c) { return (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x); }

bool segmentsMeet(V2 a, V2 b, V2 c, V2 d) {
  auto sgn = [](double v) { return (v > 0) - (v < 0); };
  auto within = [](V2 p, V2 q, V2 r) {
    return std::min(p.x, q.x) <= r.x && r.x <= std::max(p.x, q.x) && std::min(p.y, q.y) <= r.y &&
           r.y <= std::max(p.y, q.y);
  };
  const int o1 = sgn(cross3(a, b, c)), o2 = sgn(cross3(a, b, d)), o3 = sgn(cross3(c, d, a)), o4 = sgn(cross3(c, d, b));
  if (o1 != o2 && o3 != o4) return true;
  return (o1 == 0 && within(a, b, c)) || (o2 == 0 && within(a, b, d)) || (o3 == 0 && within(c, d, a)) ||
         (o4 == 0 && within(c, d, b));
}

// No two non-adjacent edges meet; edges are tested only against those whose x-ranges overlap.
bool simplePolygon(const std::vector<V2>& poly) {
  const std::size_t n = poly.size();
  if (n < 4) return true;
  std::vector<std::size_t> order(n);
  std::vector<double> lo(n), hi(n);
  for (std::size_t i = 0; i < n; ++i) {
    lo[i] = std::min(poly[i].x, poly[(i + 1) % n].x);
    hi[i] = std::max(poly[i].x, poly[(i + 1) % n].x);
    order[i] = i;
  }
  std::sort(order.begin(), order.end(), [&](std::size_t a, std::size_t b) { return lo[a] < lo[b]; });
  for (std::size_t oi = 0; oi < n; ++oi) {
    const std::size_t i = order[oi];
    for (std::size_t oj = oi + 1; oj < n && lo[order[oj]] <= hi[i]; ++oj) {
      const std::size_t j = order[oj];
      const std::size_t d = i > j ? i - j : j - i;
      if (d == 1 || d == n - 1) continue;
      if (segmentsMeet(poly[i], poly[(i + 1) % n], poly[j], poly[(j + 1) % n])) return false;
    }
  }
  return true;
}

double pointSegmentDistance(V2 p, V2 a, V2 b) {
  const V2 ab = b - a;
  const double l2 = dot(ab, ab);
  if (l2 <= 0) return norm(p - a);
  const double t = std::clamp(dot(p - a, ab) / l2, 0.0, 1.0);
  return norm(p - (a + t * ab));
}

// ---------------------------------------------------------------------------------------------------------------
// Pattern and validation (validate.cpp:25-87).

struct Piece {
  std::string id;
  Outline outline;
  V2 grain;
  std::string fabricSlot;
};
struct EdgeRef {
  std::string piece;
  double start = 0, end = 0;
  bool reversed = false;
};
struct Seam {
  std::string id;
  EdgeRef a, b;
  double ease = 0;
};
struct Pattern {
  std::vector<Piece> pieces;
  std::vector<Seam> seams;
  int find(const std::string& id) const {
    for (std::size_t i = 0; i < pieces.size(); ++i)
      if (pieces[i].id == id) return static_cast<int>(i);
    return -1;
  }
};

std::vector<std::pair<std::string, std::string>> validate(const Pattern& pat) {
  constexpr double kEps = 1e-9, kSeamTolerance = 0.002;
  std::vector<std::pair<std::string, std::string>> issues;
  auto add = [&](const std::string& rule, const std::string& msg) { issues.emplace_back(rule, msg); };
  for (const auto& p : pat.pieces) {
    const std::string who = "piece '" + p.id + "'";
    if (!p.outline.closed()) {
      add("outline-closed", who + ": outline is not closed");
    } else {
      const auto poly = p.outline.polyline(0.002);
      if (!simplePolygon(poly))
        add("outline-simple", who + ": outline crosses itself");
      else if (signedArea(poly) <= 0)
        add("outline-ccw", who + ": outline must run counter-clockwise");
    }
    if (norm(p.grain) < kEps) add("grainline", who + ": grainline is zero");
    if (p.fabricSlot.empty()) add("fabric-slot", who + ": fabric slot is empty");
  }
  struct Span {
    double start, end;
    std::string seam;
  };
  std::map<std::string, std::vector<Span>> spans;
  for (const auto& s : pat.seams) {
    const std::string who = "seam '" + s.id + "'";
    bool ranges = true;
    for (const EdgeRef* e : {&s.a, &s.b}) {
      const int pi = pat.find(e->piece);
      if (pi < 0) {
        add("seam-piece", who + ": unknown piece '" + e->piece + "'");
        ranges = false;
        continue;
      }
      const double per = pat.pieces[pi].outline.perimeter();
      if (!(e->start >= 0 && e->start < e->end && e->end <= per + kEps)) {
        add("seam-range", who + ": edge on piece '" + e->piece + "' is outside [0, perimeter] or empty");
        ranges = false;
        continue;
      }
      spans[e->piece].push_back({e->start, e->end, s.id});
    }
    if (s.a.reversed == s.b.reversed)
      add("seam-twisted", who + ": edges must be joined with opposite traversal (one reversed)");
    if (ranges) {
      const double d = std::abs((s.a.end - s.a.start) - (s.b.end - s.b.start));
      const double allowed = kSeamTolerance + std::abs(s.ease);
      if (d > allowed)
        add("seam-length", who + ": edge lengths differ by " + std::to_string(d * 1000) + " mm (allowed " +
                               std::to_string(allowed * 1000) + " mm)");
    }
  }
  for (auto& [piece, list] : spans) {
    std::sort(list.begin(), list.end(), [](const Span& x, const Span& y) { return x.start < y.start; });
    for (std::size_t i = 1; i < list.size(); ++i)
      if (list[i].start < list[i - 1].end - kEps)
        add("seam-overlap", "piece '" + piece + "': seams '" + list[i - 1].seam + "' and '" + list[i].seam +
                                "' overlap");
  }
  return issues;
}

// ---------------------------------------------------------------------------------------------------------------
// Constrained Delaunay triangulation.

class Cdt {
 public:
  // Triangles: vertices counter-clockwise; nb[k] is the triangle across the edge opposite vertex k (-1: none).
  struct Tri {
    std::array<int, 3> v;
    std::array<int, 3> nb;
    std::array<bool, 3> fixed;  // the edge opposite vertex k is a constraint
    bool alive;
  };

  explicit Cdt(const std::vector<V2>& pts) : p_(pts) {
    double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
    for (const V2& q : pts) {
      x0 = std::min(x0, q.x);
      x1 = std::max(x1, q.x);
      y0 = std::min(y0, q.y);
      y1 = std::max(y1, q.y);
    }
    scale_ = std::max({x1 - x0, y1 - y0, 1e-9});
    const double cx = 0.5 * (x0 + x1), cy = 0.5 * (y0 + y1), r = 40 * scale_;
    n_ = static_cast<int>(pts.size());
    p_.push_back({cx - r, cy - r});
    p_.push_back({cx + r, cy - r});
    p_.push_back({cx, cy + r});
    vt_.assign(p_.size(), 0);
    newTri(n_, n_ + 1, n_ + 2);
    last_ = 0;
  }

  void insertAll() {
    for (int i = 0; i < n_; ++i) insert(i);
  }

  // Makes every (a, b) an edge and marks it as a constraint.
  void constrain(const std::vector<std::pair<int, int>>& edges) {
    for (const auto& [a, b] : edges) recover(a, b);
  }

  // Triangles of the region bounded by the constraint edges (the outside is flooded from the enclosing corners).
  std::vector<std::array<int, 3>> inside() const {
    std::vector<char> out(tris_.size(), 0);
    std::deque<int> q;
    for (int t = 0; t < static_cast<int>(tris_.size()); ++t)
      if (tris_[t].alive && (tris_[t].v[0] >= n_ || tris_[t].v[1] >= n_ || tris_[t].v[2] >= n_)) {
        out[t] = 1;
        q.push_back(t);
      }
    while (!q.empty()) {
      const int t = q.front();
      q.pop_front();
      for (int k = 0; k < 3; ++k) {
        const int u = tris_[t].nb[k];
        if (u < 0 || out[u] || tris_[t].fixed[k]) continue;
        out[u] = 1;
        q.push_back(u);
      }
    }
    std::vector<std::array<int, 3>> res;
    for (int t = 0; t < static_cast<int>(tris_.size()); ++t)
      if (tris_[t].alive && !out[t]) res.push_back(tris_[t].v);
    return res;
  }

 private:
  std::vector<V2> p_;
  std::vector<Tri> tris_;
  std::vector<int> vt_;  // a live triangle with vertex v
  int n_ = 0, last_ = 0;
  double scale_ = 1;

  double orient(int a, int b, int c) const { return cross3(p_[a], p_[b], p_[c]); }
  // > 0 when d lies inside the circumcircle of the counter-clockwise triangle (a, b, c).
  double incircle(int a, int b, int c, int d) const {
    const double adx = p_[a].x - p_[d].x, ady = p_[a].y - p_[d].y;
    const double bdx = p_[b].x - p_[d].x, bdy = p_[b].y - p_[d].y;
    const double cdx = p_[c].x - p_[d].x, cdy = p_[c].y - p_[d].y;
    const double ad = adx * adx + ady * ady, bd = bdx * bdx + bdy * bdy, cd = cdx * cdx + cdy * cdy;
    return adx * (bdy * cd - bd * cdy) - ady * (bdx * cd - bd * cdx) + ad * (bdx * cdy - bdy * cdx);
  }
  int edgeIndex(int t, int a, int b) const {  // k such that the edge opposite v[k] is {a, b}
    for (int k = 0; k < 3; ++k) {
      const int x = tris_[t].v[(k + 1) % 3], y = tris_[t].v[(k + 2) % 3];
      if ((x == a && y == b) || (x == b && y == a)) return k;
    }
    return -1;
  }
  void link(int t, int k, int u) {
    tris_[t].nb[k] = u;
    if (u < 0) return;
    const int ku = edgeIndex(u, tris_[t].v[(k + 1) % 3], tris_[t].v[(k + 2) % 3]);
    tris_[u].nb[ku] = t;
    tris_[u].fixed[ku] = tris_[t].fixed[k];
  }
  int newTri(int a, int b, int c) {
    tris_.push_back({{a, b, c}, {-1, -1, -1}, {false, false, false}, true});
    const int t = static_cast<int>(tris_.size()) - 1;
    vt_[a] = vt_[b] = vt_[c] = t;  // every operation replaces dead triangles by new ones over the same vertices
    return t;
  }

  // Walks from the last triangle towards p; returns the triangle containing p and the edge p lies on (-1: interior).
  int locate(int pi, int& onEdge) {
    int t = last_;
    if (!tris_[t].alive) {
      for (t = static_cast<int>(tris_.size()) - 1; t >= 0 && !tris_[t].alive; --t) {
      }
    }
    const double eps = 1e-13 * scale_ * scale_;
    for (std::size_t steps = 0; steps < 4 * tris_.size() + 16; ++steps) {
      int next = -1;
      onEdge = -1;
      for (int k = 0; k < 3; ++k) {
        const int a = tris_[t].v[(k + 1) % 3], b = tris_[t].v[(k + 2) % 3];
        const double o = orient(a, b, pi);
        if (o < -eps) {
          next = tris_[t].nb[k];
          break;
        }
        if (o <= eps) onEdge = k;
      }
      if (next < 0) return t;
      t = next;
    }
    throw std::runtime_error("mesher: point location did not converge");
  }

  void insert(int pi) {
    int e = -1;
    const int t = locate(pi, e);
    std::vector<std::pair<int, int>> check;  // (triangle, edge index) to legalise: the edge opposite pi
    if (e < 0) {
      const auto [a, b, c] = tris_[t].v;
      const auto nb = tris_[t].nb;
      const auto fx = tris_[t].fixed;
      tris_[t].alive = false;
      const int t0 = newTri(pi, b, c), t1 = newTri(pi, c, a), t2 = newTri(pi, a, b);
      tris_[t0].fixed[0] = fx[0];
      tris_[t1].fixed[0] = fx[1];
      tris_[t2].fixed[0] = fx[2];
      link(t0, 0, nb[0]);
      link(t1, 0, nb[1]);
      link(t2, 0, nb[2]);
      tris_[t0].nb[1] = t1;
      tris_[t1].nb[2] = t0;
      tris_[t1].nb[1] = t2;
      tris_[t2].nb[2] = t1;
      tris_[t2].nb[1] = t0;
      tris_[t0].nb[2] = t2;
      check = {{t0, 0}, {t1, 0}, {t2, 0}};
      last_ = t0;
    } else {
      // pi on the edge opposite v[e] of t: split t and its neighbour across that edge into four.
      const int a = tris_[t].v[e], b = tris_[t].v[(e + 1) % 3], c = tris_[t].v[(e + 2) % 3];
      const int u = tris_[t].nb[e];
      const bool fixedEdge = tris_[t].fixed[e];
      const int nbB = tris_[t].nb[(e + 1) % 3], nbC = tris_[t].nb[(e + 2) % 3];
      const bool fxB = tris_[t].fixed[(e + 1) % 3], fxC = tris_[t].fixed[(e + 2) % 3];
      tris_[t].alive = false;
      // t = (a, b, c), edge (b, c) split at pi: (a, b, pi) and (a, pi, c).
      const int t0 = newTri(a, b, pi), t1 = newTri(a, pi, c);
      tris_[t0].fixed[2] = fxC;  // edge (a, b) is opposite pi (index 2) and was opposite c in t
      tris_[t1].fixed[1] = fxB;  // edge (c, a) is opposite pi (index 1) and was opposite b in t
      link(t0, 2, nbC);
      link(t1, 1, nbB);
      tris_[t0].nb[1] = t1;  // edge (pi, a) of t0 is opposite b
      tris_[t1].nb[2] = t0;  // edge (a, pi) of t1 is opposite c
      check = {{t0, 2}, {t1, 1}};
      if (u >= 0) {
        const int ku = edgeIndex(u, b, c);
        const int d = tris_[u].v[ku];
        const int nbUb = tris_[u].nb[edgeIndex(u, c, d)], nbUc = tris_[u].nb[edgeIndex(u, d, b)];
        const bool fxUb = tris_[u].fixed[edgeIndex(u, c, d)], fxUc = tris_[u].fixed[edgeIndex(u, d, b)];
        tris_[u].alive = false;
        // u = (d, c, b) counter-clockwise: (d, c, pi) and (d, pi, b).
        const int t2 = newTri(d, c, pi), t3 = newTri(d, pi, b);
        tris_[t2].fixed[2] = fxUb;
        tris_[t3].fixed[1] = fxUc;
        link(t2, 2, nbUb);
        link(t3, 1, nbUc);
        tris_[t2].nb[1] = t3;
        tris_[t3].nb[2] = t2;
        // Across the split edge: t0 (b, pi) with t3, t1 (pi, c) with t2.
        tris_[t0].nb[0] = t3;
        tris_[t3].nb[0] = t0;
        tris_[t1].nb[0] = t2;
        tris_[t2].nb[0] = t1;
        tris_[t0].fixed[0] = tris_[t3].fixed[0] = fixedEdge;
        tris_[t1].fixed[0] = tris_[t2].fixed[0] = fixedEdge;
        check.push_back({t2, 2});
        check.push_back({t3, 1});
      } else {
        tris_[t0].fixed[0] = tris_[t1].fixed[0] = fixedEdge;
      }
      last_ = t0;
    }
    while (!check.empty()) {
      const auto [t0, k] = check.back();
      check.pop_back();
      if (!tris_[t0].alive || tris_[t0].fixed[k]) continue;
      const int u = tris_[t0].nb[k];
      if (u < 0) continue;
      const int a = tris_[t0].v[k], b = tris_[t0].v[(k + 1) % 3], c = tris_[t0].v[(k + 2) % 3];
      const int ku = edgeIndex(u, b, c);
      const int d = tris_[u].v[ku];
      if (incircle(a, b, c, d) > 0) {
        const auto [n0, n1] = flip(t0, k);
        // The edges of the new triangles that face away from a (the inserted point) are the ones to check.
        check.push_back({n0, edgeIndex(n0, b, d) >= 0 ? edgeIndex(n0, b, d) : edgeIndex(n0, c, d)});
        check.push_back({n1, edgeIndex(n1, c, d) >= 0 ? edgeIndex(n1, c, d) : edgeIndex(n1, b, d)});
      }
    }
  }

  // Flips the edge opposite v[k] of t (shared with its neighbour); returns the two new triangles, the first holding
  // t's vertex a = v[k].
  std::pair<int, int> flip(int t, int k) {
    const int u = tris_[t].nb[k];
    const int a = tris_[t].v[k], b = tris_[t].v[(k + 1) % 3], c = tris_[t].v[(k + 2) % 3];
    const int ku = edgeIndex(u, b, c);
    const int d = tris_[u].v[ku];
    // Outer neighbours: of t across (a, b) and (c, a); of u across (b, d) and (d, c).
    const int nAB = tris_[t].nb[(k + 2) % 3], nCA = tris_[t].nb[(k + 1) % 3];
    const bool fAB = tris_[t].fixed[(k + 2) % 3], fCA = tris_[t].fixed[(k + 1) % 3];
    const int iBD = edgeIndex(u, b, d), iDC = edgeIndex(u, d, c);
    const int nBD = tris_[u].nb[iBD], nDC = tris_[u].nb[iDC];
    const bool fBD = tris_[u].fixed[iBD], fDC = tris_[u].fixed[iDC];
    tris_[t].alive = tris_[u].alive = false;
    // New triangles (a, b, d) and (a, d, c), both counter-clockwise since the quad a-b-d-c is convex.
    const int n0 = newTri(a, b, d), n1 = newTri(a, d, c);
    tris_[n0].fixed[2] = fAB;  // (a, b) opposite d
    tris_[n0].fixed[0] = fBD;  // (b, d) opposite a
    tris_[n1].fixed[1] = fCA;  // (c, a) opposite d
    tris_[n1].fixed[0] = fDC;  // (d, c) opposite a
    link(n0, 2, nAB);
    link(n0, 0, nBD);
    link(n1, 1, nCA);
    link(n1, 0, nDC);
    tris_[n0].nb[1] = n1;  // (d, a) of n0 opposite b
    tris_[n1].nb[2] = n0;  // (a, d) of n1 opposite c
    last_ = n0;
    return {n0, n1};
  }

  // A live triangle with edge (a, b) and that edge's index, by turning around vertex a (its star is closed: the
  // enclosing triangle's corners are never queried); t = -1 when (a, b) is not an edge.
  void findEdge(int a, int b, int& t, int& k) const {
    const int start = vt_[a];
    int cur = start;
    for (std::size_t guard = 0; guard < tris_.size(); ++guard) {
      const auto& T = tris_[cur];
      const int ka = T.v[0] == a ? 0 : (T.v[1] == a ? 1 : 2);
      if (T.v[(ka + 1) % 3] == b) {
        t = cur;
        k = (ka + 2) % 3;
        return;
      }
      if (T.v[(ka + 2) % 3] == b) {
        t = cur;
        k = (ka + 1) % 3;
        return;
      }
      cur = T.nb[(ka + 2) % 3];  // across the edge (a, v[ka + 1])
      if (cur < 0 || cur == start) break;
    }
    t = k = -1;
  }

  bool markIfEdge(int a, int b) {
    int t, k;
    findEdge(a, b, t, k);
    if (t < 0) return false;
    tris_[t].fixed[k] = true;
    const int u = tris_[t].nb[k];
    if (u >= 0) tris_[u].fixed[edgeIndex(u, a, b)] = true;
    return true;
  }

  bool crosses(int a, int b, int c, int d) const {  // open segments (a, b) and (c, d) cross properly
    const double o1 = orient(a, b, c), o2 = orient(a, b, d), o3 = orient(c, d, a), o4 = orient(c, d, b);
    return ((o1 > 0 && o2 < 0) || (o1 < 0 && o2 > 0)) && ((o3 > 0 && o4 < 0) || (o3 < 0 && o4 > 0));
  }

  // Sloan's recovery: the edges crossing (a, b) are flipped (when their quad is convex) until none crosses it.
  void recover(int a, int b) {
    if (markIfEdge(a, b)) return;
    for (int round = 0; round < 64; ++round) {
      std::deque<std::pair<int, int>> crossing;  // edges (c, d) crossing (a, b)
      for (int t = 0; t < static_cast<int>(tris_.size()); ++t) {
        if (!tris_[t].alive) continue;
        for (int k = 0; k < 3; ++k) {
          const int c = tris_[t].v[(k + 1) % 3], d = tris_[t].v[(k + 2) % 3];
          if (c < d && crosses(a, b, c, d)) crossing.emplace_back(c, d);
        }
      }
      if (crossing.empty()) break;
      std::size_t stall = 0;
      while (!crossing.empty() && stall <= crossing.size()) {
        const auto [c, d] = crossing.front();
        crossing.pop_front();
        int t = -1, k = -1;
        findEdge(c, d, t, k);
        if (t < 0) continue;
        const int u = tris_[t].nb[k];
        const int x = tris_[t].v[k], y = tris_[u].v[edgeIndex(u, c, d)];
        // Convex quad x-c-y-d: the diagonals cross.
        if (tris_[t].fixed[k] || !crosses(x, y, c, d)) {
          crossing.emplace_back(c, d);
          ++stall;
          continue;
        }
        stall = 0;
        flip(t, k);
        if (crosses(a, b, x, y)) crossing.emplace_back(std::min(x, y), std::max(x, y));
      }
      if (markIfEdge(a, b)) return;
    }
    if (!markIfEdge(a, b)) throw MeshError("mesher: constraint edge could not be recovered");
  }
};

// ---------------------------------------------------------------------------------------------------------------
// The mesher. Per piece: the outline is walked into boundary stations (in outline order, from arc length 0), a
// grain-aligned hexagonal lattice fills the interior, the stations and the lattice are triangulated with the outline
// as constraint, and the interior vertices are relaxed. The output follows the reference's SimMesh contract
// (libs/garment/src/sim_mesh_builder.cpp:196-323): seam sides carry the same station count on both pieces so seam
// pairs match one to one, outline corners are vertices, lattice edges follow the grain's 60-degree directions,
// vertex areas are a third of the incident triangle areas.

struct Mesh {
  std::vector<V2> rest;
  std::vector<uint32_t> vertexPiece;
  std::vector<uint8_t> boundary;
  std::vector<double> vertexArea;
  std::vector<std::array<uint32_t, 3>> triangles;
  std::vector<uint32_t> trianglePiece;
  std::vector<V2> pieceGrain;
  std::vector<std::array<uint32_t, 4>> seamPairs;
};

constexpr double kArcEps = 1e-9;

// Stations on a run of outline: the fewest equal arc steps no longer than h (at least one).
int stationsFor(double length, double h) { return std::max(1, static_cast<int>(std::ceil(length / h - kArcEps))); }

// Arc positions of the segment joints where the outline's direction turns by more than 10 degrees (the reference's
// corner rule).
std::vector<double> turningPoints(const Outline& o) {
  std::vector<double> out;
  const std::size_t n = o.seg.size();
  for (std::size_t i = 0; i < n; ++i) {
    const Cubic& before = o.seg[(i + n - 1) % n];
    const Cubic& after = o.seg[i];
    V2 din = before.derivative(1.0), dout = after.derivative(0.0);
    if (norm(din) < 1e-14) din = before.p[3] - before.p[0];  // degenerate end tangents: use the chords
    if (norm(dout) < 1e-14) dout = after.p[3] - after.p[0];
    const double turn = std::acos(std::clamp(dot(unit(din), unit(dout)), -1.0, 1.0));
    if (turn > 10.0 * kPi / 180.0) out.push_back(o.start[i]);
  }
  return out;
}

// A stretch of outline sampled as one unit: [a, b] in arc length with `count` equal steps. A seam side is one run
// (seam >= 0, side 0 or 1) whatever corners it covers, so both of its pieces sample it at the same fractions.
struct Run {
  double a = 0, b = 0;
  int count = 1;
  int seam = -1, side = 0;
};

struct BoundaryWalk {
  std::vector<V2> points;  // stations in outline order; station 0 at arc length 0
  std::map<std::pair<int, int>, std::vector<uint32_t>> seamStations;  // (seam, side) -> stations 0..count
};

// Walks the outline once: the gaps between this piece's seam sides are split at the turning points into free runs of
// stationsFor(length, h) steps; every run emits its start and interior stations, so the stations come out in outline
// order, and each seam side records its station indices as it is emitted (the last one is the next run's first, or
// station 0 where the outline closes).
BoundaryWalk walkBoundary(const Outline& o, std::vector<Run> seamRuns, double h) {
  const double perimeter = o.perimeter();
  std::sort(seamRuns.begin(), seamRuns.end(), [](const Run& x, const Run& y) { return x.a < y.a; });
  const std::vector<double> turns = turningPoints(o);
  std::vector<Run> runs;
  auto addFree = [&](double a, double b) {
    if (b - a <= kArcEps) return;
    double from = a;
    for (double t : turns) {
      if (t <= from + kArcEps || t >= b - kArcEps) continue;
      runs.push_back({from, t, stationsFor(t - from, h)});
      from = t;
    }
    runs.push_back({from, b, stationsFor(b - from, h)});
  };
  double cursor = 0.0;
  for (const Run& s : seamRuns) {
    addFree(cursor, s.a);
    runs.push_back(s);
    cursor = std::max(cursor, s.b);
  }
  addFree(cursor, perimeter);
  BoundaryWalk w;
  std::vector<std::pair<const Run*, uint32_t>> pending;  // seam runs and their first station
  for (const Run& r : runs) {
    const uint32_t first = static_cast<uint32_t>(w.points.size());
    for (int k = 0; k < r.count; ++k) w.points.push_back(o.pointAt(r.a + (r.b - r.a) * k / r.count));
    if (r.seam >= 0) pending.emplace_back(&r, first);
  }
  const uint32_t total = static_cast<uint32_t>(w.points.size());
  for (const auto& [r, first] : pending) {
    std::vector<uint32_t>& v = w.seamStations[{r->seam, r->side}];
    for (int k = 0; k <= r->count; ++k) v.push_back((first + static_cast<uint32_t>(k)) % total);
  }
  return w;
}

// The hexagonal lattice aligned with `grain` (rows along the grain, h sqrt(3)/2 apart, every other row shifted by
// h/2), restricted to the points inside the closed polygon `poly` (nonzero winding) that keep at least h/2 from every
// polygon edge. Work happens in the grain frame, row by row: each polygon edge is listed under the rows its
// h/2-neighbourhood reaches, so a row sees exactly the edges that can cross it or come within h/2 of it; the winding
// of a lattice point is the signed count of those edges crossing the row beyond it.
std::vector<V2> grainLattice(const std::vector<V2>& poly, V2 grain, double h) {
  const V2 gu = unit(grain), gv{-gu.y, gu.x};
  const std::size_t n = poly.size();
  std::vector<V2> q(n);
  double vLo = 1e300, vHi = -1e300, uLo = 1e300, uHi = -1e300;
  for (std::size_t i = 0; i < n; ++i) {
    q[i] = {dot(poly[i], gu), dot(poly[i], gv)};
    uLo = std::min(uLo, q[i].x);
    uHi = std::max(uHi, q[i].x);
    vLo = std::min(vLo, q[i].y);
    vHi = std::max(vHi, q[i].y);
  }
  const double pitch = h * std::sqrt(0.75), clearance = 0.5 * h;
  const int jLo = static_cast<int>(std::floor(vLo / pitch)), jHi = static_cast<int>(std::ceil(vHi / pitch));
  std::vector<std::vector<uint32_t>> rowEdges(static_cast<std::size_t>(jHi - jLo + 1));
  for (std::size_t k = 0; k < n; ++k) {
    const V2 a = q[k], b = q[(k + 1) % n];
    const int r0 = std::max(jLo, static_cast<int>(std::ceil((std::min(a.y, b.y) - clearance) / pitch)));
    const int r1 = std::min(jHi, static_cast<int>(std::floor((std::max(a.y, b.y) + clearance) / pitch)));
    for (int j = r0; j <= r1; ++j) rowEdges[static_cast<std::size_t>(j - jLo)].push_back(static_cast<uint32_t>(k));
  }
  std::vector<V2> out;
  std::vector<std::pair<double, int>> hits;  // (u of the crossing, winding contribution)
  for (int j = jLo; j <= jHi; ++j) {
    const std::vector<uint32_t>& edges = rowEdges[static_cast<std::size_t>(j - jLo)];
    const double v = j * pitch;
    hits.clear();
    int winding = 0;
    for (uint32_t k : edges) {
      const V2 a = q[k], b = q[(k + 1) % n];
      if ((a.y <= v) == (b.y <= v)) continue;
      const int dir = b.y > a.y ? 1 : -1;
      hits.emplace_back(a.x + (v - a.y) * (b.x - a.x) / (b.y - a.y), dir);
      winding += dir;
    }
    if (hits.empty()) continue;
    std::sort(hits.begin(), hits.end());
    const double shift = (j % 2 != 0) ? 0.5 * h : 0.0;
    const int iLo = static_cast<int>(std::ceil((uLo - shift) / h)), iHi = static_cast<int>(std::floor((uHi - shift) / h));
    std::size_t next = 0;
    for (int i = iLo; i <= iHi; ++i) {
      const double u = i * h + shift;
      while (next < hits.size() && hits[next].first <= u) winding -= hits[next++].second;
      if (winding == 0) continue;
      const V2 p{u, v};
      bool clear = true;
      for (uint32_t k : edges)
        if (pointSegmentDistance(p, q[k], q[(k + 1) % n]) < clearance) {
          clear = false;
          break;
        }
      if (clear) out.push_back(u * gu + v * gv);
    }
  }
  return out;
}

double triArea(V2 a, V2 b, V2 c) { return 0.5 * cross3(a, b, c); }

// Largest corner cosine of a triangle: the smaller its smallest angle, the larger this is.
double largestCosine(V2 a, V2 b, V2 c) {
  auto cosAt = [](V2 p, V2 x, V2 y) {
    const V2 e = x - p, f = y - p;
    return dot(e, f) / std::max(1e-300, norm(e) * norm(f));
  };
  return std::max(cosAt(a, b, c), std::max(cosAt(b, c, a), cosAt(c, a, b)));
}

// Centroidal relaxation of the interior vertices [firstInterior, pts.size()), `sweeps` Gauss-Seidel passes: a vertex
// moves to the area-weighted mean of its incident triangles' centroids. The move is kept only if every incident
// triangle stays counter-clockwise (area > 1e-14) and the smallest angle among them does not shrink; otherwise half
// the move is tried, then none. A vertex inside an undistorted hexagonal patch is its own target and stays put.
void relaxInterior(std::vector<V2>& pts, const std::vector<std::array<uint32_t, 3>>& tris, std::size_t firstInterior,
                   int sweeps) {
  std::vector<uint32_t> start(pts.size() + 1, 0), list;
  for (const auto& t : tris)
    for (uint32_t v : t) ++start[v + 1];
  for (std::size_t i = 0; i < pts.size(); ++i) start[i + 1] += start[i];
  list.resize(start.back());
  std::vector<uint32_t> fill(start.begin(), start.end() - 1);
  for (uint32_t t = 0; t < tris.size(); ++t)
    for (uint32_t v : tris[t]) list[fill[v]++] = t;
  auto worst = [&](std::size_t i, double& minArea) {
    double c = -1.0;
    minArea = 1e300;
    for (uint32_t e = start[i]; e < start[i + 1]; ++e) {
      const auto& t = tris[list[e]];
      minArea = std::min(minArea, triArea(pts[t[0]], pts[t[1]], pts[t[2]]));
      c = std::max(c, largestCosine(pts[t[0]], pts[t[1]], pts[t[2]]));
    }
    return c;
  };
  for (int sweep = 0; sweep < sweeps; ++sweep) {
    for (std::size_t i = firstInterior; i < pts.size(); ++i) {
      if (start[i] == start[i + 1]) continue;
      double weight = 0;
      V2 target{0, 0};
      for (uint32_t e = start[i]; e < start[i + 1]; ++e) {
        const auto& t = tris[list[e]];
        const double a = std::abs(triArea(pts[t[0]], pts[t[1]], pts[t[2]]));
        target = target + (a / 3.0) * (pts[t[0]] + pts[t[1]] + pts[t[2]]);
        weight += a;
      }
      if (!(weight > 0)) continue;
      target = (1.0 / weight) * target;
      const V2 home = pts[i];
      double area = 0;
      const double before = worst(i, area);
      for (double step : {1.0, 0.5}) {
        pts[i] = home + step * (target - home);
        const double after = worst(i, area);
        if (area > 1e-14 && after <= before + 1e-12) break;
        pts[i] = home;
      }
    }
  }
}

Mesh build(const Pattern& pat, double h) {
  if (!(h > 0)) throw MeshError("particle distance must be positive");
  const auto issues = validate(pat);
  if (!issues.empty()) {
    std::string msg = "pattern is invalid:";
    for (const auto& [rule, text] : issues) msg += " [" + rule + "] " + text + ";";
    throw MeshError(msg);
  }
  // Every seam gets one station count (from its longer side) and places a run of it on each side's piece.
  std::vector<int> seamCount(pat.seams.size());
  std::vector<std::vector<Run>> pieceSeamRuns(pat.pieces.size());
  for (std::size_t s = 0; s < pat.seams.size(); ++s) {
    const Seam& sm = pat.seams[s];
    seamCount[s] = stationsFor(std::max(sm.a.end - sm.a.start, sm.b.end - sm.b.start), h);
    const EdgeRef* sides[2] = {&sm.a, &sm.b};
    for (int side = 0; side < 2; ++side)
      pieceSeamRuns[static_cast<std::size_t>(pat.find(sides[side]->piece))].push_back(
          {sides[side]->start, sides[side]->end, seamCount[s], static_cast<int>(s), side});
  }
  Mesh mesh;
  std::map<std::pair<int, int>, std::vector<uint32_t>> seamVertices;  // (seam, side) -> mesh vertices
  for (std::size_t pi = 0; pi < pat.pieces.size(); ++pi) {
    const Piece& piece = pat.pieces[pi];
    const BoundaryWalk walk = walkBoundary(piece.outline, pieceSeamRuns[pi], h);
    std::vector<V2> pts = walk.points;
    const std::size_t boundaryCount = pts.size();
    const V2 grain = unit(piece.grain);
    const std::vector<V2> inner = grainLattice(walk.points, grain, h);
    pts.insert(pts.end(), inner.begin(), inner.end());
    {
      std::vector<V2> sorted = pts;
      std::sort(sorted.begin(), sorted.end(), [](V2 a, V2 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
      for (std::size_t i = 1; i < sorted.size(); ++i)
        if (sorted[i].x == sorted[i - 1].x && sorted[i].y == sorted[i - 1].y)
          throw MeshError("piece '" + piece.id + "': duplicate mesh vertices");
    }
    Cdt cdt(pts);
    cdt.insertAll();
    std::vector<std::pair<int, int>> loop(boundaryCount);
    for (std::size_t i = 0; i < boundaryCount; ++i)
      loop[i] = {static_cast<int>(i), static_cast<int>((i + 1) % boundaryCount)};
    cdt.constrain(loop);
    std::vector<std::array<uint32_t, 3>> tris;
    for (const auto& t : cdt.inside()) {
      std::array<uint32_t, 3> tri{static_cast<uint32_t>(t[0]), static_cast<uint32_t>(t[1]), static_cast<uint32_t>(t[2])};
      if (triArea(pts[tri[0]], pts[tri[1]], pts[tri[2]]) < 0) std::swap(tri[1], tri[2]);
      tris.push_back(tri);
    }
    relaxInterior(pts, tris, boundaryCount, 3);

    const uint32_t base = static_cast<uint32_t>(mesh.rest.size());
    for (std::size_t i = 0; i < pts.size(); ++i) {
      mesh.rest.push_back(pts[i]);
      mesh.vertexPiece.push_back(static_cast<uint32_t>(pi));
      mesh.boundary.push_back(i < boundaryCount ? 1 : 0);
      mesh.vertexArea.push_back(0.0);
    }
    for (const auto& t : tris) {
      const double area = triArea(pts[t[0]], pts[t[1]], pts[t[2]]);
      if (!(area > 1e-12)) throw MeshError("piece '" + piece.id + "': degenerate triangle");
      mesh.triangles.push_back({t[0] + base, t[1] + base, t[2] + base});
      mesh.trianglePiece.push_back(static_cast<uint32_t>(pi));
      for (uint32_t v : t) mesh.vertexArea[base + v] += area / 3.0;
    }
    mesh.pieceGrain.push_back(grain);
    for (const auto& [key, stations] : walk.seamStations) {
      std::vector<uint32_t>& dst = seamVertices[key];
      for (uint32_t v : stations) dst.push_back(base + v);
    }
  }
  // Seam pairs: station k of each side, counted from the side's far end when the side is reversed.
  for (std::size_t s = 0; s < pat.seams.size(); ++s) {
    const int n = seamCount[s];
    const std::vector<uint32_t>& a = seamVertices.at({static_cast<int>(s), 0});
    const std::vector<uint32_t>& b = seamVertices.at({static_cast<int>(s), 1});
    const bool ra = pat.seams[s].a.reversed, rb = pat.seams[s].b.reversed;
    for (int k = 0; k <= n; ++k)
      mesh.seamPairs.push_back({a[static_cast<std::size_t>(ra ? n - k : k)], b[static_cast<std::size_t>(rb ? n - k : k)],
                                static_cast<uint32_t>(s), static_cast<uint32_t>(k)});
  }
  return mesh;
}

}  // namespace dmesh

struct drape_mesh {
  dmesh::Mesh m;
};

namespace {
thread_local std::string g_meshError;

template <class F>
int meshGuarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::invalid_argument& e) {
    g_meshError = e.what();
    return -1;
  } catch (const std::exception& e) {
    g_meshError = e.what();
    return -3;
  }
}
}  // namespace

extern "C" {

double drape_mesh_particle_distance(int quality) {
  switch (quality) {
    case 0: return 0.020;
    case 1: return 0.010;
    case 2: return 0.005;
    default: return 0.010;
  }
}

int drape_mesh_build(const drape_pattern_desc* pattern, double particle_distance, drape_mesh** out) {
  return meshGuarded([&] {
    if (!pattern || !out) throw std::invalid_argument("null pattern or output");
    *out = nullptr;
    dmesh::Pattern pat;
    for (uint32_t i = 0; i < pattern->piece_count; ++i) {
      const drape_piece_desc& d = pattern->pieces[i];
      if (d.segment_count > 0 && !d.segments) throw std::invalid_argument("piece without segment data");
      dmesh::Piece p;
      p.id = d.id ? d.id : "";
      p.fabricSlot = d.fabric_slot ? d.fabric_slot : "";
      p.grain = {d.grain[0], d.grain[1]};
      for (uint32_t k = 0; k < d.segment_count; ++k) {
        dmesh::Cubic c;
        for (int q = 0; q < 4; ++q) c.p[q] = {d.segments[k].p[2 * q], d.segments[k].p[2 * q + 1]};
        p.outline.add(c);
      }
      pat.pieces.push_back(std::move(p));
    }
    for (uint32_t i = 0; i < pattern->seam_count; ++i) {
      const drape_seam_desc& d = pattern->seams[i];
      dmesh::Seam s;
      s.id = d.id ? d.id : "";
      s.a = {d.piece_a ? d.piece_a : "", d.start_a, d.end_a, d.reversed_a != 0};
      s.b = {d.piece_b ? d.piece_b : "", d.start_b, d.end_b, d.reversed_b != 0};
      s.ease = d.ease;
      pat.seams.push_back(std::move(s));
    }
    auto m = std::make_unique<drape_mesh>();
    m->m = dmesh::build(pat, particle_distance);
    *out = m.release();
  });
}

void drape_mesh_destroy(drape_mesh* m) { delete m; }

const char* drape_mesh_last_error(void) { return g_meshError.c_str(); }

int drape_mesh_sizes(const drape_mesh* m, uint32_t sizes[4]) {
  return meshGuarded([&] {
    if (!m || !sizes) throw std::invalid_argument("null mesh or sizes");
    sizes[0] = static_cast<uint32_t>(m->m.rest.size());
    sizes[1] = static_cast<uint32_t>(m->m.triangles.size());
    sizes[2] = static_cast<uint32_t>(m->m.pieceGrain.size());
    sizes[3] = static_cast<uint32_t>(m->m.seamPairs.size());
  });
}

int drape_mesh_read(const drape_mesh* m, double* rest, uint32_t* vertex_piece, uint8_t* boundary, double* vertex_area,
                    uint32_t* triangles, uint32_t* triangle_piece, double* piece_grain, uint32_t* seam_pairs) {
  return meshGuarded([&] {
    if (!m) throw std::invalid_argument("null mesh");
    const dmesh::Mesh& x = m->m;
    for (std::size_t i = 0; i < x.rest.size(); ++i) {
      if (rest) {
        rest[2 * i] = x.rest[i].x;
        rest[2 * i + 1] = x.rest[i].y;
      }
      if (vertex_piece) vertex_piece[i] = x.vertexPiece[i];
      if (boundary) boundary[i] = x.boundary[i];
      if (vertex_area) vertex_area[i] = x.vertexArea[i];
    }
    for (std::size_t t = 0; t < x.triangles.size(); ++t) {
      if (triangles)
        for (int k = 0; k < 3; ++k) triangles[3 * t + k] = x.triangles[t][k];
      if (triangle_piece) triangle_piece[t] = x.trianglePiece[t];
    }
    for (std::size_t p = 0; p < x.pieceGrain.size(); ++p)
      if (piece_grain) {
        piece_grain[2 * p] = x.pieceGrain[p].x;
        piece_grain[2 * p + 1] = x.pieceGrain[p].y;
      }
    for (std::size_t k = 0; k < x.seamPairs.size(); ++k)
      if (seam_pairs)
        for (int q = 0; q < 4; ++q) seam_pairs[4 * k + q] = x.seamPairs[k][q];
  });
}

}  // extern "C"
