// Host-side scene model of the CUDA solver (see model.hpp).
#include "model.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <exception>
#include <stdexcept>
#include <thread>

namespace drape_b200 {

namespace {

double norm3(double x, double y, double z) { return std::sqrt(x * x + y * y + z * z); }

// FabricPhysical bending coefficients and edge stiffness (bending.cpp:7-18).
void bendCoefficients(double bendWarp, double bendWeft, double& p, double& q) {
  const double floor = 0.05 * std::min(bendWarp, bendWeft);
  p = std::max((3.0 * bendWarp - bendWeft) / 2.0, floor);
  q = std::max(bendWeft, floor);
}

double edgeStiffness(double p, double q, const double dir[2], const double grain[2]) {
  const double dn = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1]);
  const double gn = std::sqrt(grain[0] * grain[0] + grain[1] * grain[1]);
  const double d0 = dir[0] / dn, d1 = dir[1] / dn, u0 = grain[0] / gn, u1 = grain[1] / gn;
  const double c = d0 * u0 + d1 * u1;
  const double s = d0 * u1 - d1 * u0;
  return p * s * s + q * c * c;
}

inline uint64_t edgeKey(uint32_t a, uint32_t b) {
  const uint32_t lo = std::min(a, b), hi = std::max(a, b);
  return (static_cast<uint64_t>(lo) << 32) | hi;
}

// Runs f(c) for c in [0, chunks) on up to `chunks` threads (the calling thread takes chunk 0); the first exception a
// chunk throws is rethrown after all have finished.
template <class F>
void parallelChunks(std::size_t chunks, F&& f) {
  if (chunks <= 1) {
    if (chunks == 1) f(0);
    return;
  }
  std::vector<std::exception_ptr> errors(chunks);
  std::vector<std::thread> pool;
  for (std::size_t c = 1; c < chunks; ++c)
    pool.emplace_back([&, c] {
      try {
        f(c);
      } catch (...) {
        errors[c] = std::current_exception();
      }
    });
  try {
    f(0);
  } catch (...) {
    errors[0] = std::current_exception();
  }
  for (auto& t : pool) t.join();
  for (auto& e : errors)
    if (e) std::rethrow_exception(e);
}

// Host threads for the build's parallel loops, and the chunk count for `items` items of at least `grain` each.
std::size_t buildThreads() {
  return std::max<std::size_t>(1, std::min<std::size_t>(16, std::thread::hardware_concurrency()));
}
std::size_t chunksFor(std::size_t items, std::size_t grain) {
  return std::max<std::size_t>(1, std::min(buildThreads(), (items + grain - 1) / grain));
}

}  // namespace

std::size_t Model::garmentIndex(const std::string& id) const {
  for (std::size_t i = 0; i < garments.size(); ++i)
    if (garments[i].id == id) return i;
  throw std::out_of_range("unknown garment '" + id + "'");
}

double Model::hingeStiffness(std::size_t hgi) const {
  double B = 0;
  for (const auto& side : hingeSides[hgi]) {
    const auto& f = fabrics[side.fabric];
    double p, q;
    bendCoefficients(f.bend_warp, f.bend_weft, p, q);
    B += 0.5 * edgeStiffness(p, q, side.edgeDir, side.grain);
  }
  return B * hingeGeom[hgi];
}

void Model::updateMass(uint32_t i) { mass[i] = std::max(vertexArea[i] * fabrics[pFabric[i]].weight, 1e-12); }

uint32_t Model::slot(uint32_t row, uint32_t col) const {
  const auto begin = colIndex.begin() + rowStart[row];
  const auto end = colIndex.begin() + rowStart[row + 1];
  return static_cast<uint32_t>(std::lower_bound(begin, end, col) - colIndex.begin());
}

Model Model::build(const drape_scene_desc& scene, bool copyField) {
  Model next;
  next.settings = scene.settings;
  if (scene.body) {
    next.hasBody = true;
    next.field = *scene.body;
    const long long count = static_cast<long long>(std::max(0, scene.body->dims[0])) *
                            std::max(0, scene.body->dims[1]) * std::max(0, scene.body->dims[2]);
    if (scene.body->values && count > 0) {
      if (scene.body->dims[0] < 2 || scene.body->dims[1] < 2 || scene.body->dims[2] < 2)
        throw std::invalid_argument("collision field needs at least 2 samples per axis");
      next.fieldCount = static_cast<std::size_t>(count);
      if (copyField) {
        next.fieldValues.assign(scene.body->values, scene.body->values + count);
      } else {
        next.fieldSource = scene.body->values;
      }
    }
    next.field.values = nullptr;
  }
  for (uint32_t gi0 = 0; gi0 < scene.garment_count; ++gi0) {
    const drape_garment_desc& sg = scene.garments[gi0];
    const std::string id = sg.id ? sg.id : "";
    if (sg.vertex_count > 0 && (!sg.initial_positions || !sg.rest || !sg.vertex_area || !sg.vertex_piece))
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
    next.fabrics.insert(next.fabrics.end(), sg.piece_fabric, sg.piece_fabric + sg.piece_count);
    for (uint32_t v = 0; v < sg.vertex_count; ++v) {
      if (sg.vertex_piece[v] >= sg.piece_count)
        throw std::invalid_argument("garment '" + id + "': vertex piece out of range");
      next.x.push_back({static_cast<float>(sg.initial_positions[3 * v]), static_cast<float>(sg.initial_positions[3 * v + 1]),
                        static_cast<float>(sg.initial_positions[3 * v + 2])});
      next.vertexArea.push_back(sg.vertex_area[v]);
      next.pFabric.push_back(g.fabricOffset + sg.vertex_piece[v]);
      next.pGarment.push_back(gi);
    }
    const uint32_t* T = sg.triangles;
    for (uint32_t t = 0; t < sg.triangle_count; ++t)
      for (int k = 0; k < 3; ++k)
        if (T[3 * t + k] >= sg.vertex_count) throw std::invalid_argument("garment '" + id + "': triangle vertex out of range");
    auto rest = [&](uint32_t v, int c) { return sg.rest[2 * v + c]; };
    auto triArea = [&](uint32_t t) {
      const uint32_t a = T[3 * t], b = T[3 * t + 1], c = T[3 * t + 2];
      const double e0 = rest(b, 0) - rest(a, 0), e1 = rest(b, 1) - rest(a, 1);
      const double f0 = rest(c, 0) - rest(a, 0), f1 = rest(c, 1) - rest(a, 1);
      return 0.5 * std::abs(e0 * f1 - e1 * f0);
    };
    const std::size_t stretchBase = next.stretch.size();
    next.stretch.resize(stretchBase + sg.triangle_count);
    // Stretch terms: rest shape in the piece's grain frame, dmInv = Dm^-1, area = |det Dm| / 2 (sim_model.cpp:107-123);
    // every triangle on its own, in parallel chunks.
    const std::size_t triChunks = chunksFor(sg.triangle_count, 16384);
    parallelChunks(triChunks, [&](std::size_t ch) {
      for (uint32_t t = static_cast<uint32_t>(sg.triangle_count * ch / triChunks);
           t < static_cast<uint32_t>(sg.triangle_count * (ch + 1) / triChunks); ++t) {
        const uint32_t piece = sg.triangle_piece[t];
        const double u0 = sg.piece_grain[2 * piece], u1 = sg.piece_grain[2 * piece + 1];
        double r[3][2];
        for (int k = 0; k < 3; ++k) {
          const uint32_t v = T[3 * t + k];
          r[k][0] = rest(v, 0) * u0 + rest(v, 1) * u1;
          r[k][1] = rest(v, 0) * -u1 + rest(v, 1) * u0;
        }
        const double a = r[1][0] - r[0][0], b = r[2][0] - r[0][0], c = r[1][1] - r[0][1], d = r[2][1] - r[0][1];
        const double det = a * d - c * b;
        const double invdet = 1.0 / det;  // adjugate times 1 / det (the operation order of Eigen's 2x2 inverse)
        Stretch st;
        for (int k = 0; k < 3; ++k) st.v[k] = off + T[3 * t + k];
        st.dmInv[0][0] = d * invdet;
        st.dmInv[0][1] = -b * invdet;
        st.dmInv[1][0] = -c * invdet;
        st.dmInv[1][1] = a * invdet;
        st.area = 0.5 * std::abs(det);
        st.fabric = g.fabricOffset + piece;
        next.stretch[stretchBase + t] = st;
      }
    });
    // Edge occurrences in insertion order (triangle t, then k = 0, 1, 2), stably sorted by (min, max): the same
    // sequence a std::map<pair<min,max>, vector<tri>> iterates. Counting sort by the smaller vertex (stable), then a
    // stable insertion sort of each vertex's few edges by the larger one.
    std::vector<std::pair<uint64_t, uint32_t>> occ(3 * static_cast<std::size_t>(sg.triangle_count));
    {
      std::vector<uint32_t> start(sg.vertex_count + 1, 0);
      for (uint32_t t = 0; t < sg.triangle_count; ++t)
        for (int k = 0; k < 3; ++k) ++start[std::min(T[3 * t + k], T[3 * t + (k + 1) % 3]) + 1];
      for (uint32_t v = 0; v < sg.vertex_count; ++v) start[v + 1] += start[v];
      std::vector<uint32_t> fill(start.begin(), start.end() - 1);
      for (uint32_t t = 0; t < sg.triangle_count; ++t)
        for (int k = 0; k < 3; ++k) {
          const uint64_t key = edgeKey(T[3 * t + k], T[3 * t + (k + 1) % 3]);
          occ[fill[key >> 32]++] = {key, t};
        }
      for (uint32_t v = 0; v < sg.vertex_count; ++v)
        for (uint32_t i = start[v] + 1; i < start[v + 1]; ++i) {
          const auto item = occ[i];
          uint32_t j = i;
          for (; j > start[v] && occ[j - 1].first > item.first; --j) occ[j] = occ[j - 1];
          occ[j] = item;
        }
    }
    // Interior edges in occurrence order (the map order): the first occurrence of every edge shared by exactly two
    // triangles of one piece, found by a serial scan; their hinges are then formed in parallel chunks.
    std::vector<std::size_t> interior;
    interior.reserve(occ.size() / 2);
    for (std::size_t i = 0; i < occ.size();) {
      std::size_t j = i;
      while (j < occ.size() && occ[j].first == occ[i].first) ++j;
      if (j - i == 2 && sg.triangle_piece[occ[i].second] == sg.triangle_piece[occ[i + 1].second]) interior.push_back(i);
      i = j;
    }
    const std::size_t hingeBase = next.hinges.size();
    {
      const std::size_t more = interior.size() + sg.seam_pair_count;
      next.hinges.reserve(hingeBase + more);
      next.hingeSides.reserve(hingeBase + more);
      next.hingeGeom.reserve(hingeBase + more);
      next.hinges.resize(hingeBase + interior.size());
      next.hingeSides.resize(hingeBase + interior.size());
      next.hingeGeom.resize(hingeBase + interior.size());
    }
    auto opposite = [&](uint32_t t, uint32_t e0, uint32_t e1) {
      for (int k = 0; k < 3; ++k) {
        const uint32_t v = T[3 * t + k];
        if (v != e0 && v != e1) return v;
      }
      return e0;
    };
    const std::size_t hingeChunks = chunksFor(interior.size(), 16384);
    parallelChunks(hingeChunks, [&](std::size_t ch) {
      for (std::size_t h = interior.size() * ch / hingeChunks; h < interior.size() * (ch + 1) / hingeChunks; ++h) {
        const std::size_t i = interior[h];
        const uint32_t e0 = static_cast<uint32_t>(occ[i].first >> 32), e1 = static_cast<uint32_t>(occ[i].first);
        const uint32_t t0 = occ[i].second, t1 = occ[i + 1].second;
        const uint32_t piece = sg.triangle_piece[t0];
        Hinge hg;
        hg.v = {off + opposite(t0, e0, e1), off + opposite(t1, e0, e1), off + e0, off + e1};
        next.hinges[hingeBase + h] = hg;
        HingeSide side;
        side.fabric = g.fabricOffset + piece;
        side.edgeDir[0] = rest(e1, 0) - rest(e0, 0);
        side.edgeDir[1] = rest(e1, 1) - rest(e0, 1);
        side.grain[0] = sg.piece_grain[2 * piece];
        side.grain[1] = sg.piece_grain[2 * piece + 1];
        next.hingeSides[hingeBase + h] = {side, side};
        next.hingeGeom[hingeBase + h] = (side.edgeDir[0] * side.edgeDir[0] + side.edgeDir[1] * side.edgeDir[1]) /
                                        (triArea(t0) + triArea(t1));
      }
    });
    // The triangle of a boundary edge (an edge with exactly one triangle), or -1.
    auto triangleWithEdge = [&](uint32_t a, uint32_t b) -> int64_t {
      const uint64_t key = edgeKey(a, b);
      auto lo = std::lower_bound(occ.begin(), occ.end(), key,
                                 [](const std::pair<uint64_t, uint32_t>& p, uint64_t k) { return p.first < k; });
      if (lo == occ.end() || lo->first != key) return -1;
      if (lo + 1 != occ.end() && (lo + 1)->first == key) return -1;
      return lo->second;
    };
    const uint32_t* SP = sg.seam_pairs;
    for (uint32_t k = 0; k < sg.seam_pair_count; ++k) {
      const uint32_t a = SP[4 * k], b = SP[4 * k + 1], seam = SP[4 * k + 2];
      if (a >= sg.vertex_count || b >= sg.vertex_count)
        throw std::invalid_argument("garment '" + id + "': seam pair vertex out of range");
      Seam spring;
      spring.a = off + a;
      spring.b = off + b;
      spring.garment = gi;
      const double* pa = sg.initial_positions + 3 * a;
      const double* pb = sg.initial_positions + 3 * b;
      spring.startGap = static_cast<float>(norm3(pa[0] - pb[0], pa[1] - pb[1], pa[2] - pb[2]));
      next.seams.push_back(spring);
      if (k + 1 >= sg.seam_pair_count || SP[4 * (k + 1) + 2] != seam) continue;
      const uint32_t na = SP[4 * (k + 1)], nb = SP[4 * (k + 1) + 1];
      const int64_t tA = triangleWithEdge(a, na), tB = triangleWithEdge(b, nb);
      if (tA < 0 || tB < 0) continue;
      const auto ta = static_cast<uint32_t>(tA), tb = static_cast<uint32_t>(tB);
      const uint32_t pieceA = sg.triangle_piece[ta], pieceB = sg.triangle_piece[tb];
      Hinge hg;
      hg.v = {off + opposite(ta, a, na), off + opposite(tb, b, nb), off + a, off + na};
      next.hinges.push_back(hg);
      HingeSide sa, sb;
      sa.fabric = g.fabricOffset + pieceA;
      sa.edgeDir[0] = rest(na, 0) - rest(a, 0);
      sa.edgeDir[1] = rest(na, 1) - rest(a, 1);
      sa.grain[0] = sg.piece_grain[2 * pieceA];
      sa.grain[1] = sg.piece_grain[2 * pieceA + 1];
      sb.fabric = g.fabricOffset + pieceB;
      sb.edgeDir[0] = rest(nb, 0) - rest(b, 0);
      sb.edgeDir[1] = rest(nb, 1) - rest(b, 1);
      sb.grain[0] = sg.piece_grain[2 * pieceB];
      sb.grain[1] = sg.piece_grain[2 * pieceB + 1];
      next.hingeSides.push_back({sa, sb});
      next.hingeGeom.push_back((sa.edgeDir[0] * sa.edgeDir[0] + sa.edgeDir[1] * sa.edgeDir[1]) / (triArea(ta) + triArea(tb)));
    }
    next.garments.push_back(g);
  }
  const std::size_t n = next.x.size();
  next.v.assign(n, Vec3f{});
  next.fExt.assign(n, Vec3d{});
  next.pinned.assign(n, 0);
  next.mass.assign(n, 0.0);
  for (uint32_t k = 0; k < scene.pin_count; ++k) {
    const uint32_t p = scene.pin_particles[k];
    if (p >= n) throw std::out_of_range("pin particle out of range");
    const Vec3f pos{static_cast<float>(scene.pin_positions[3 * k]), static_cast<float>(scene.pin_positions[3 * k + 1]),
                    static_cast<float>(scene.pin_positions[3 * k + 2])};
    next.pinned[p] = 1;
    next.pins.push_back({p, pos});
    next.x[p] = pos;
  }
  for (uint32_t k = 0; k < scene.force_count; ++k) {
    const uint32_t p = scene.force_particles[k];
    if (p >= n) throw std::out_of_range("force particle out of range");
    next.fExt[p].x += scene.forces[3 * k];
    next.fExt[p].y += scene.forces[3 * k + 1];
    next.fExt[p].z += scene.forces[3 * k + 2];
  }
  for (uint32_t i = 0; i < n; ++i) next.updateMass(i);
  const std::size_t kChunks = chunksFor(next.hinges.size(), 16384);
  parallelChunks(kChunks, [&](std::size_t ch) {
    for (std::size_t h = next.hinges.size() * ch / kChunks; h < next.hinges.size() * (ch + 1) / kChunks; ++h)
      next.hinges[h].K = next.hingeStiffness(h);
  });
  next.buildIncidence();
  next.buildStructure();
  return next;
}

// Calls f(vertices, count) for every term's vertex set: stretch terms, hinges, then seam springs.
template <class F>
void Model::forEachTerm(F&& f) const {
  for (const auto& t : stretch) f(t.v.data(), 3);
  for (const auto& h : hinges) f(h.v.data(), 4);
  for (const auto& s : seams) {
    const uint32_t ab[2] = {s.a, s.b};
    f(ab, 2);
  }
}

// Vertex count of the term an incidence entry names (3 stretch, 4 hinge, 2 seam).
int Model::entryArity(uint32_t code) {
  const uint32_t kind = code >> 30;
  return kind == 0 ? 3 : (kind == 1 ? 4 : 2);
}

// Vertex set of the term an incidence entry names; returns its size.
int Model::termVertices(uint32_t code, uint32_t ab[4]) const {
  const uint32_t kind = code >> 30, term = (code >> 2) & 0x0FFFFFFFu;
  if (kind == 0) {
    std::copy(stretch[term].v.begin(), stretch[term].v.end(), ab);
    return 3;
  }
  if (kind == 1) {
    std::copy(hinges[term].v.begin(), hinges[term].v.end(), ab);
    return 4;
  }
  ab[0] = seams[term].a;
  ab[1] = seams[term].b;
  return 2;
}

void Model::buildIncidence() {
  const std::size_t n = x.size();
  if (stretch.size() >= (1u << 28) || hinges.size() >= (1u << 28) || seams.size() >= (1u << 28))
    throw std::invalid_argument("too many terms for the incidence encoding");
  incStart.assign(n + 1, 0);
  forEachTerm([&](const uint32_t* vs, int m) {
    for (int a = 0; a < m; ++a) ++incStart[vs[a] + 1];
  });
  for (std::size_t i = 0; i < n; ++i) incStart[i + 1] += incStart[i];
  incEntry.assign(incStart[n], 0);
  incLocal.assign(incStart[n], 0);
  // Entries in the reference's gather order (gpu_solver_core.cpp:184-224): stretch (t, a) in term order, then hinges,
  // then seams.
  std::vector<uint32_t> fill(incStart.begin(), incStart.end() - 1);
  auto add = [&](uint32_t kind, uint32_t term, const uint32_t* vs, int m) {
    for (int a = 0; a < m; ++a) incEntry[fill[vs[a]]++] = (kind << 30) | (term << 2) | static_cast<uint32_t>(a);
  };
  for (uint32_t t = 0; t < stretch.size(); ++t) add(0, t, stretch[t].v.data(), 3);
  for (uint32_t h = 0; h < hinges.size(); ++h) add(1, h, hinges[h].v.data(), 4);
  for (uint32_t k = 0; k < seams.size(); ++k) {
    const uint32_t ab[2] = {seams[k].a, seams[k].b};
    add(2, k, ab, 2);
  }
  maxRowEntries = 0;
  for (std::size_t i = 0; i < n; ++i) maxRowEntries = std::max(maxRowEntries, incStart[i + 1] - incStart[i]);
}

void Model::buildStructure() {
  const std::size_t n = x.size();
  // Row i's columns: i itself and every vertex of every term that contains i, deduplicated with a stamp array and
  // sorted -- the sorted unique coupled columns of the reference's per-row vectors (sim_model.cpp:41-74). Each term's
  // slots are the positions of its vertices' columns in their rows (the reference finds them by binary search,
  // sim_model.cpp:35-39; the slots are the same). Rows are built in chunks on several threads, each chunk into its
  // own buffers with row-local positions; a prefix sum over the row sizes then places every chunk.
  if (n >= (1u << 26)) throw std::invalid_argument("too many particles for the slot encoding");
  if (incStart[n] >= (1u << 29)) throw std::invalid_argument("too many term incidences for the contribution encoding");
  rowStart.assign(n + 1, 0);
  diagSlot.assign(n, 0);
  stretchSlots.resize(stretch.size());
  hingeSlots.resize(hinges.size());
  seamSlots.resize(seams.size());
  struct Chunk {
    uint32_t r0 = 0, r1 = 0;
    std::vector<uint32_t> cols, offSlot, offStart, offContrib;
    uint32_t maxL = 0;
  };
  const std::size_t chunkCount = chunksFor(n, 8192);
  std::vector<Chunk> chunks(chunkCount);
  for (std::size_t c = 0; c < chunkCount; ++c) {
    chunks[c].r0 = static_cast<uint32_t>(n * c / chunkCount);
    chunks[c].r1 = static_cast<uint32_t>(n * (c + 1) / chunkCount);
  }
  // Pass 1: per row, the sorted columns, the row-local slot positions of its incidence entries (incLocal), its
  // diagonal position (kept in diagSlot until pass 2) and its off-diagonal slots' contribution lists in slot order
  // (entry e's block b lands in row-local slot byte b of incLocal[e]; each list keeps the incidence order).
  parallelChunks(chunkCount, [&](std::size_t c) {
    Chunk& ch = chunks[c];
    std::vector<uint32_t> stamp(n, UINT32_MAX), where(n, 0);
    uint32_t vs[4];
    for (uint32_t i = ch.r0; i < ch.r1; ++i) {
      const std::size_t rs = ch.cols.size();
      stamp[i] = i;
      ch.cols.push_back(i);
      for (uint32_t e = incStart[i]; e < incStart[i + 1]; ++e) {
        const int m = termVertices(incEntry[e], vs);
        for (int b = 0; b < m; ++b)
          if (stamp[vs[b]] != i) {
            stamp[vs[b]] = i;
            ch.cols.push_back(vs[b]);
          }
      }
      std::sort(ch.cols.begin() + static_cast<std::ptrdiff_t>(rs), ch.cols.end());
      const uint32_t L = static_cast<uint32_t>(ch.cols.size() - rs);
      ch.maxL = std::max(ch.maxL, L);
      if (L > kMaxRowSlots)
        throw std::invalid_argument("a particle couples to " + std::to_string(L) + " particles; the CUDA solver supports " +
                                    std::to_string(kMaxRowSlots));
      rowStart[i + 1] = L;
      for (uint32_t t = 0; t < L; ++t) where[ch.cols[rs + t]] = t;
      const uint32_t dl = where[i];
      diagSlot[i] = dl;
      for (uint32_t t = 0; t < L; ++t)
        if (t != dl) ch.offSlot.push_back((i << 6) | t);
      uint32_t cnt[kMaxRowSlots] = {};
      for (uint32_t e = incStart[i]; e < incStart[i + 1]; ++e) {
        const int m = termVertices(incEntry[e], vs);
        uint32_t packed = 0;
        for (int b = 0; b < m; ++b) {
          const uint32_t t = where[vs[b]];
          packed |= t << (8 * b);
          ++cnt[t];
        }
        incLocal[e] = packed;
      }
      uint32_t pos[kMaxRowSlots];
      uint32_t next = static_cast<uint32_t>(ch.offContrib.size());
      for (uint32_t t = 0; t < L; ++t) {
        if (t == dl) continue;
        ch.offStart.push_back(next);
        pos[t] = next;
        next += cnt[t];
      }
      ch.offContrib.resize(next);
      for (uint32_t e = incStart[i]; e < incStart[i + 1]; ++e) {
        const int m = entryArity(incEntry[e]);
        for (int b = 0; b < m; ++b) {
          const uint32_t t = (incLocal[e] >> (8 * b)) & 0xFFu;
          if (t != dl) ch.offContrib[pos[t]++] = (e << 2) | static_cast<uint32_t>(b);
        }
      }
    }
  });
  maxRowSlots = 0;
  for (const Chunk& ch : chunks) maxRowSlots = std::max(maxRowSlots, ch.maxL);
  for (std::size_t i = 0; i < n; ++i) rowStart[i + 1] += rowStart[i];
  std::vector<std::size_t> offBase(chunkCount + 1, 0), contribBase(chunkCount + 1, 0);
  for (std::size_t c = 0; c < chunkCount; ++c) {
    offBase[c + 1] = offBase[c] + chunks[c].offSlot.size();
    contribBase[c + 1] = contribBase[c] + chunks[c].offContrib.size();
  }
  colIndex.assign(rowStart[n], 0);
  offSlot.assign(offBase[chunkCount], 0);
  offStart.assign(offBase[chunkCount] + 1, 0);
  offContrib.assign(contribBase[chunkCount], 0);
  offStart[offBase[chunkCount]] = static_cast<uint32_t>(contribBase[chunkCount]);
  // Pass 2: every chunk into place; global slots of the diagonal and of every term's blocks.
  parallelChunks(chunkCount, [&](std::size_t c) {
    const Chunk& ch = chunks[c];
    std::copy(ch.cols.begin(), ch.cols.end(), colIndex.begin() + rowStart[ch.r0]);
    std::copy(ch.offSlot.begin(), ch.offSlot.end(), offSlot.begin() + static_cast<std::ptrdiff_t>(offBase[c]));
    for (std::size_t k = 0; k < ch.offStart.size(); ++k)
      offStart[offBase[c] + k] = static_cast<uint32_t>(contribBase[c] + ch.offStart[k]);
    std::copy(ch.offContrib.begin(), ch.offContrib.end(),
              offContrib.begin() + static_cast<std::ptrdiff_t>(contribBase[c]));
    for (uint32_t i = ch.r0; i < ch.r1; ++i) {
      const uint32_t rs = rowStart[i];
      diagSlot[i] += rs;
      for (uint32_t e = incStart[i]; e < incStart[i + 1]; ++e) {
        const uint32_t code = incEntry[e], kind = code >> 30, term = (code >> 2) & 0x0FFFFFFFu, a = code & 3u;
        const int m = entryArity(code);
        uint32_t* out = kind == 0 ? stretchSlots[term].data() : (kind == 1 ? hingeSlots[term].data() : seamSlots[term].data());
        for (int b = 0; b < m; ++b) out[a * m + b] = rs + ((incLocal[e] >> (8 * b)) & 0xFFu);
      }
    }
  });
  const std::size_t terms = std::max(stretch.size(), std::max(hinges.size(), seams.size()));
  if (terms >= (1u << 26)) throw std::invalid_argument("too many terms for the contribution encoding");
  offCode.resize(offContrib.size());
  parallelChunks(chunkCount, [&](std::size_t c) {
    for (std::size_t k = contribBase[c]; k < contribBase[c + 1]; ++k) {
      const uint32_t v = offContrib[k], code = incEntry[v >> 2];
      offCode[k] = (code & 0xC0000000u) | (((code >> 2) & 0x03FFFFFFu) << 4) | ((code & 3u) << 2) | (v & 3u);
    }
  });
  contactForce.assign(n, 0.0);
}

void Model::updateFabric(const std::string& id, const drape_fabric* pieceFabric, uint32_t count) {
  auto& g = garments[garmentIndex(id)];
  if (count != g.pieceCount) throw std::invalid_argument("one fabric per pattern piece required");
  std::copy(pieceFabric, pieceFabric + count, fabrics.begin() + g.fabricOffset);
  for (uint32_t i = g.offset; i < g.offset + g.count; ++i) updateMass(i);
  for (std::size_t h = 0; h < hinges.size(); ++h) {
    const auto fi = hingeSides[h][0].fabric;
    if (fi >= g.fabricOffset && fi < g.fabricOffset + g.pieceCount) hinges[h].K = hingeStiffness(h);
  }
}

void Model::setPhase(const std::string& id, int phase) {
  const auto gi = garmentIndex(id);
  auto& g = garments[gi];
  g.phase = phase;
  if (phase == DRAPE_PHASE_ASSEMBLING) {
    g.assemblyTime = 0;
    for (auto& sp : seams) {
      if (sp.garment != gi) continue;
      // |x_a - x_b| on float positions, as the reference's Vec3f norm (sim_model.cpp:302).
      const float dx = x[sp.a].x - x[sp.b].x, dy = x[sp.a].y - x[sp.b].y, dz = x[sp.a].z - x[sp.b].z;
      sp.startGap = std::sqrt(dx * dx + dy * dy + dz * dz);
    }
  }
}

}  // namespace drape_b200
