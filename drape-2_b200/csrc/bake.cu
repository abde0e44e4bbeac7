// Collision-field bake (include/drape_bake.h): bakeCollisionField (libs/avatar/src/collision_bake.cpp:98-208) on the
// GPU. The reference walks triangles serially and keeps per sample the first triangle reaching the smallest squared
// distance; here every triangle is one block and the choice is made in two passes with 64-bit atomics (the exact
// FP64 minimum, then the lowest triangle index reaching it), which is the same triangle. All double arithmetic is
// explicitly rounded in the reference's order (Ericson's closest point, RTCD 5.1.5; dot products summed left to
// right), so the field equals the serial algorithm's in FP64 rounded to float. Pseudonormals (face, angle-weighted
// vertex, edge sums) are computed on the host in the same order as the reference. The outside of the band is found
// by line sweeps along the six axis directions, repeated until nothing changes: the same set as the reference's
// breadth-first flood fill from the grid boundary.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/drape_bake.h"
#include "../../include/drape_cuda.h"
#include "device_buffer.hpp"

using dbuf::check;
using dbuf::DBuf;
#define KCK(x) check((x), #x)

namespace bake {

struct D3 {
  double x, y, z;
};

// Explicitly rounded double operations (no contraction into fused multiply-adds).
__device__ __forceinline__ D3 sub(D3 a, D3 b) { return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)}; }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ double dot(D3 a, D3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
// a + s * v per component.
__device__ __forceinline__ D3 axpy(D3 a, double s, D3 v) {
  return {add(a.x, mul(s, v.x)), add(a.y, mul(s, v.y)), add(a.z, mul(s, v.z))};
}

enum Feature : int { kVertexA, kVertexB, kVertexC, kEdgeAB, kEdgeBC, kEdgeCA, kFace };

// Closest point on triangle abc to p and the feature it lies on (collision_bake.cpp:19-55).
__device__ inline D3 closestPoint(D3 p, D3 a, D3 b, D3 c, int& f) {
  const D3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) {
    f = kVertexA;
    return a;
  }
  const D3 bp = sub(p, b);
  const double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) {
    f = kVertexB;
    return b;
  }
  const double vc = dsub(mul(d1, d4), mul(d3, d2));
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    f = kEdgeAB;
    return axpy(a, ddiv(d1, dsub(d1, d3)), ab);
  }
  const D3 cp = sub(p, c);
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) {
    f = kVertexC;
    return c;
  }
  const double vb = dsub(mul(d5, d2), mul(d1, d6));
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    f = kEdgeCA;
    return axpy(a, ddiv(d2, dsub(d2, d6)), ac);
  }
  const double va = dsub(mul(d3, d6), mul(d5, d4));
  const double e43 = dsub(d4, d3), e56 = dsub(d5, d6);
  if (va <= 0 && e43 >= 0 && e56 >= 0) {
    f = kEdgeBC;
    return axpy(b, ddiv(e43, add(e43, e56)), sub(c, b));
  }
  const double denom = ddiv(1.0, add(add(va, vb), vc));
  f = kFace;
  return axpy(axpy(a, mul(vb, denom), ab), mul(vc, denom), ac);
}

struct Grid {
  double ox, oy, oz, cell, band, band2;
  int nx, ny, nz;
};

struct Mesh {
  const D3* v;
  const uint3* t;
  const double* tbox;  // per triangle: tmin xyz, tmax xyz
  const int* trange;   // per triangle: x0 x1 y0 y1 z0 z1 (sample box, inclusive)
  const D3* faceN;     // per triangle
  const D3* vertexN;   // per vertex
  const D3* edgeN;     // per triangle: AB, BC, CA
  uint32_t nt;
};

__device__ __forceinline__ D3 samplePos(const Grid& g, int x, int y, int z) {
  return {add(g.ox, mul(g.cell, static_cast<double>(x))), add(g.oy, mul(g.cell, static_cast<double>(y))),
          add(g.oz, mul(g.cell, static_cast<double>(z)))};
}

// Squared distance from p to the triangle's bounding box (the reference's cheap reject).
__device__ __forceinline__ double boxGap2(const double* tb, D3 p) {
  const double gx = fmax(fmax(dsub(tb[0], p.x), dsub(p.x, tb[3])), 0.0);
  const double gy = fmax(fmax(dsub(tb[1], p.y), dsub(p.y, tb[4])), 0.0);
  const double gz = fmax(fmax(dsub(tb[2], p.z), dsub(p.z, tb[5])), 0.0);
  return add(add(mul(gx, gx), mul(gy, gy)), mul(gz, gz));
}

__device__ __forceinline__ size_t sampleIndex(const Grid& g, int x, int y, int z) {
  return (static_cast<size_t>(z) * g.ny + y) * g.nx + x;
}

// Pass 1 (Owner = false): the smallest squared distance per sample (atomic minimum on the double's bits; non-negative
// doubles order like their bit patterns). Pass 2 (Owner = true): the lowest triangle index reaching that minimum.
template <bool Owner>
__global__ void k_bake_distance(Grid g, Mesh m, unsigned long long* dist2, uint32_t* owner) {
  for (uint32_t t = blockIdx.x; t < m.nt; t += gridDim.x) {
    const int* r = m.trange + 6 * static_cast<size_t>(t);
    const int bx = r[1] - r[0] + 1, by = r[3] - r[2] + 1, bz = r[5] - r[4] + 1;
    if (bx <= 0 || by <= 0 || bz <= 0) continue;
    const uint3 tri = m.t[t];
    const D3 a = m.v[tri.x], b = m.v[tri.y], c = m.v[tri.z];
    const double* tb = m.tbox + 6 * static_cast<size_t>(t);
    const int total = bx * by * bz;
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
      const int x = r[0] + k % bx, y = r[2] + (k / bx) % by, z = r[4] + k / (bx * by);
      const size_t i = sampleIndex(g, x, y, z);
      const D3 p = samplePos(g, x, y, z);
      const double best = __longlong_as_double(static_cast<long long>(
          Owner ? dist2[i] : *reinterpret_cast<volatile unsigned long long*>(dist2 + i)));
      const double gap = boxGap2(tb, p);
      // Pass 1: no improvement possible when the box is already as far as the best; pass 2: only an exact tie with
      // the final minimum counts, and d2 >= gap.
      if (Owner ? gap > best : gap >= best) continue;
      int f;
      const D3 q = closestPoint(p, a, b, c, f);
      const D3 d = sub(p, q);
      const double d2 = dot(d, d);
      if (!Owner) {
        if (d2 < best) atomicMin(dist2 + i, static_cast<unsigned long long>(__double_as_longlong(d2)));
      } else if (d2 == best) {
        atomicMin(owner + i, t);
      }
    }
  }
}

// Pass 3: the sign of every sample with an owner, from the pseudonormal of the nearest feature.
__global__ void k_bake_sign(Grid g, Mesh m, const uint32_t* owner, int8_t* sign, size_t count) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const uint32_t t = owner[i];
    if (t == 0xFFFFFFFFu) continue;
    const int x = static_cast<int>(i % g.nx), y = static_cast<int>((i / g.nx) % g.ny),
              z = static_cast<int>(i / (static_cast<size_t>(g.nx) * g.ny));
    const D3 p = samplePos(g, x, y, z);
    const uint3 tri = m.t[t];
    int f;
    const D3 q = closestPoint(p, m.v[tri.x], m.v[tri.y], m.v[tri.z], f);
    D3 n;
    switch (f) {
      case kVertexA: n = m.vertexN[tri.x]; break;
      case kVertexB: n = m.vertexN[tri.y]; break;
      case kVertexC: n = m.vertexN[tri.z]; break;
      case kEdgeAB: n = m.edgeN[3 * static_cast<size_t>(t)]; break;
      case kEdgeBC: n = m.edgeN[3 * static_cast<size_t>(t) + 1]; break;
      case kEdgeCA: n = m.edgeN[3 * static_cast<size_t>(t) + 2]; break;
      default: n = m.faceN[t]; break;
    }
    sign[i] = dot(sub(p, q), n) >= 0 ? 1 : -1;
  }
}

// Flood-fill state per sample: bit 0 far (farther than the band), bit 1 outside. Seeds: far samples on the grid
// boundary.
constexpr uint8_t kFar = 1, kOutside = 2;

__global__ void k_bake_seed(Grid g, const unsigned long long* dist2, uint8_t* state, size_t count) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int x = static_cast<int>(i % g.nx), y = static_cast<int>((i / g.nx) % g.ny),
              z = static_cast<int>(i / (static_cast<size_t>(g.nx) * g.ny));
    const bool boundary = x == 0 || y == 0 || z == 0 || x == g.nx - 1 || y == g.ny - 1 || z == g.nz - 1;
    const bool far = __longlong_as_double(static_cast<long long>(dist2[i])) > g.band2;
    state[i] = far ? (boundary ? kFar | kOutside : kFar) : 0;
  }
}

// One sweep along `axis` in direction `dir` (+1 / -1): every line carries "outside" through consecutive far samples.
// A thread takes its line 32 samples at a time (independent loads) as bit masks in walking order, F (far) and O
// (outside, a subset of F); with the carry c_in from the previous word, the sum F + O + c_in carries through exactly
// the far runs that hold a seed or continue the previous run, so the reached set is O | ((F + O + c_in) ^ F ^ O) & F
// and the carry out of bit 31 goes to the next word. Sets *changed when it marks a sample.
__global__ void k_bake_sweep(Grid g, uint8_t* state, int axis, int dir, int* changed) {
  const int n[3] = {g.nx, g.ny, g.nz};
  const int u = axis == 0 ? 1 : 0, w = axis == 2 ? 1 : 2;  // the two other axes
  const size_t lines = static_cast<size_t>(n[u]) * n[w];
  const size_t strides[3] = {1, static_cast<size_t>(g.nx), static_cast<size_t>(g.nx) * g.ny};
  const int len = n[axis];
  int marked = 0;
  for (size_t l = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; l < lines;
       l += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t base = (l % n[u]) * strides[u] + (l / n[u]) * strides[w];
    const long long step = dir > 0 ? static_cast<long long>(strides[axis]) : -static_cast<long long>(strides[axis]);
    const size_t first = dir > 0 ? base : base + static_cast<size_t>(len - 1) * strides[axis];
    uint32_t cin = 0;
    for (int s0 = 0; s0 < len; s0 += 32) {
      const int cnt = min(32, len - s0);
      uint8_t st[32];
#pragma unroll
      for (int e = 0; e < 32; ++e)
        st[e] = e < cnt ? state[static_cast<size_t>(static_cast<long long>(first) + (s0 + e) * step)] : 0;
      uint32_t F = 0, O = 0;
#pragma unroll
      for (int e = 0; e < 32; ++e) {
        F |= static_cast<uint32_t>(st[e] & kFar) << e;
        O |= static_cast<uint32_t>((st[e] & kOutside) >> 1) << e;
      }
      const unsigned long long sum = static_cast<unsigned long long>(F) + O + cin;
      const uint32_t reached = O | ((static_cast<uint32_t>(sum) ^ F ^ O) & F);
      cin = static_cast<uint32_t>(sum >> 32);
      const uint32_t fresh = reached & ~O;
      if (fresh) {
        marked = 1;
#pragma unroll
        for (int e = 0; e < 32; ++e)
          if (fresh >> e & 1u) state[static_cast<size_t>(static_cast<long long>(first) + (s0 + e) * step)] = kFar | kOutside;
      }
    }
  }
  if (marked) atomicExch(changed, 1);
}

// Combine this component into the field (collision_bake.cpp:196-204).
__global__ void k_bake_combine(Grid g, const unsigned long long* dist2, const int8_t* sign, const uint8_t* state,
                               float* values, size_t count) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const double d2 = __longlong_as_double(static_cast<long long>(dist2[i]));
    double v;
    if (d2 <= g.band2) {
      v = static_cast<double>(sign[i]) * __dsqrt_rn(d2);
    } else {
      v = (state[i] & kOutside) ? g.band : -g.band;
    }
    v = fmin(fmax(v, -g.band), g.band);
    values[i] = fminf(values[i], __double2float_rn(v));
  }
}

__global__ void k_fill(float* values, size_t count, float v) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    values[i] = v;
}

__global__ void k_reset(unsigned long long* dist2, uint32_t* owner, int8_t* sign, size_t count) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    dist2[i] = 0x7FF0000000000000ull;  // +inf
    owner[i] = 0xFFFFFFFFu;
    sign[i] = 0;
  }
}

}  // namespace bake

namespace {

thread_local std::string g_bakeError;
thread_local double g_bakeMs = 0.0;

using bake::D3;

D3 vtx(const drape_mesh_desc& m, uint32_t i) { return {m.vertices[3 * i], m.vertices[3 * i + 1], m.vertices[3 * i + 2]}; }
D3 hsub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
double hdot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
D3 hcross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
// Eigen's normalized(): divide by the norm when the squared norm is positive.
D3 hnormalized(D3 a) {
  const double z = hdot(a, a);
  if (!(z > 0)) return a;
  const double s = std::sqrt(z);
  return {a.x / s, a.y / s, a.z / s};
}

// isClosedManifold (libs/core/src/triangle_mesh.cpp:16-28): every directed edge once, and its reverse once.
bool closedManifold(const drape_mesh_desc& m) {
  if (m.triangle_count == 0) return false;
  std::vector<uint64_t> e;
  e.reserve(3ull * m.triangle_count);
  for (uint32_t t = 0; t < m.triangle_count; ++t)
    for (int k = 0; k < 3; ++k)
      e.push_back(static_cast<uint64_t>(m.triangles[3 * t + k]) << 32 | m.triangles[3 * t + (k + 1) % 3]);
  std::sort(e.begin(), e.end());
  for (size_t i = 1; i < e.size(); ++i)
    if (e[i] == e[i - 1]) return false;
  for (uint64_t x : e) {
    const uint64_t rev = (x << 32) | (x >> 32);
    if (!std::binary_search(e.begin(), e.end(), rev)) return false;
  }
  return true;
}

void validate(const drape_mesh_desc* components, uint32_t count, const drape_bake_options* o) {
  if (!components || count == 0) throw std::invalid_argument("no collision components");
  if (!o || !(o->cell_size > 0) || !(o->band > 0) || !(o->padding >= 0))
    throw std::invalid_argument("bake options need cell_size > 0, band > 0, padding >= 0");
  for (uint32_t c = 0; c < count; ++c) {
    const drape_mesh_desc& m = components[c];
    if (!m.vertices || !m.triangles) throw std::invalid_argument("null mesh arrays");
    for (size_t k = 0; k < 3ull * m.triangle_count; ++k)
      if (m.triangles[k] >= m.vertex_count) throw std::invalid_argument("triangle vertex index out of range");
    if (!closedManifold(m))
      throw std::invalid_argument("collision component " + std::to_string(c) + " is not a closed manifold");
  }
}

// Grid of the bake (collision_bake.cpp:99-117).
void gridOf(const drape_mesh_desc* components, uint32_t count, const drape_bake_options& o, double origin[3],
            int dims[3]) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t c = 0; c < count; ++c)
    for (uint32_t i = 0; i < components[c].vertex_count; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], components[c].vertices[3 * i + a]);
        hi[a] = std::max(hi[a], components[c].vertices[3 * i + a]);
      }
  for (int a = 0; a < 3; ++a) {
    origin[a] = lo[a] - o.padding;
    const double extent = (hi[a] - lo[a]) + 2 * o.padding;
    dims[a] = static_cast<int>(std::ceil(extent / o.cell_size)) + 1;
  }
}

}  // namespace

extern "C" {

int drape_bake_grid(const drape_mesh_desc* components, uint32_t count, const drape_bake_options* options,
                    double origin[3], int32_t dims[3]) {
  try {
    validate(components, count, options);
    if (!origin || !dims) throw std::invalid_argument("null argument");
    int d[3];
    gridOf(components, count, *options, origin, d);
    for (int a = 0; a < 3; ++a) dims[a] = d[a];
    return DRAPE_OK;
  } catch (const std::invalid_argument& e) {
    g_bakeError = e.what();
    return DRAPE_INVALID;
  } catch (const std::exception& e) {
    g_bakeError = e.what();
    return DRAPE_DEVICE_ERROR;
  }
}

int drape_bake_field(int device, const drape_mesh_desc* components, uint32_t count, const drape_bake_options* options,
                     float* values, size_t value_count) {
  try {
    validate(components, count, options);
    const drape_bake_options& o = *options;
    double origin[3];
    int dims[3];
    gridOf(components, count, o, origin, dims);
    const size_t total = static_cast<size_t>(dims[0]) * dims[1] * dims[2];
    if (!values || value_count != total) throw std::invalid_argument("values must hold dims[0] * dims[1] * dims[2]");
    int devices = 0;
    KCK(cudaGetDeviceCount(&devices));
    if (device < 0 || device >= devices) throw std::runtime_error("cuda: no device " + std::to_string(device));
    KCK(cudaSetDevice(device));
    cudaStream_t st;
    KCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaEvent_t e0, e1;
    KCK(cudaEventCreate(&e0));
    KCK(cudaEventCreate(&e1));
    struct Cleanup {
      cudaStream_t s;
      cudaEvent_t a, b;
      ~Cleanup() {
        cudaStreamSynchronize(s);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaStreamDestroy(s);
      }
    } cleanup{st, e0, e1};
    int sms = 0;
    KCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    bake::Grid g{origin[0], origin[1], origin[2], o.cell_size, o.band, o.band * o.band, dims[0], dims[1], dims[2]};
    DBuf<unsigned long long> dist2;
    DBuf<uint32_t> owner;
    DBuf<int8_t> sign;
    DBuf<uint8_t> state;  // flood-fill state per sample (far, outside)
    DBuf<float> field;
    DBuf<int> changed;
    dist2.alloc(total);
    owner.alloc(total);
    sign.alloc(total);
    state.alloc(total);
    field.alloc(total);
    changed.alloc(1);
    const int pointGrid = sms * 8;
    // Host preparation of every component first (boxes, sample ranges, pseudonormals), then the device work.
    struct Prepared {
      DBuf<D3> v, face, vert, edge;
      DBuf<uint3> t;
      DBuf<double> box;
      DBuf<int> range;
      uint32_t nt = 0;
    };
    std::vector<Prepared> prepared(count);
    for (uint32_t c = 0; c < count; ++c) {
      const drape_mesh_desc& m = components[c];
      // Host: vertices, triangles, boxes and sample ranges, pseudonormals (collision_bake.cpp:57-95).
      const uint32_t nv = m.vertex_count, nt = m.triangle_count;
      std::vector<D3> v(nv), faceN(nt), vertexN(nv, D3{0, 0, 0}), edgeN(3ull * nt);
      for (uint32_t i = 0; i < nv; ++i) v[i] = vtx(m, i);
      std::vector<uint3> tris(nt);
      std::vector<double> tbox(6ull * nt);
      std::vector<int> trange(6ull * nt);
      std::vector<std::pair<uint64_t, D3>> edgeSum;  // (min, max) vertex pair -> sum of face normals
      edgeSum.reserve(3ull * nt);
      auto edgeKey = [](uint32_t a, uint32_t b) {
        return static_cast<uint64_t>(std::min(a, b)) << 32 | std::max(a, b);
      };
      for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t* tr = m.triangles + 3ull * t;
        tris[t] = make_uint3(tr[0], tr[1], tr[2]);
        const D3 a = v[tr[0]], b = v[tr[1]], c3 = v[tr[2]];
        faceN[t] = hnormalized(hcross(hsub(b, a), hsub(c3, a)));
        for (int k = 0; k < 3; ++k) {
          const D3 p = v[tr[k]];
          const D3 e1 = hnormalized(hsub(v[tr[(k + 1) % 3]], p));
          const D3 e2 = hnormalized(hsub(v[tr[(k + 2) % 3]], p));
          const double ang = std::acos(std::clamp(hdot(e1, e2), -1.0, 1.0));
          D3& vn = vertexN[tr[k]];
          vn = {vn.x + ang * faceN[t].x, vn.y + ang * faceN[t].y, vn.z + ang * faceN[t].z};
          edgeSum.push_back({edgeKey(tr[k], tr[(k + 1) % 3]), faceN[t]});
        }
        const double mn[3] = {std::min(std::min(a.x, b.x), c3.x), std::min(std::min(a.y, b.y), c3.y),
                              std::min(std::min(a.z, b.z), c3.z)};
        const double mx[3] = {std::max(std::max(a.x, b.x), c3.x), std::max(std::max(a.y, b.y), c3.y),
                              std::max(std::max(a.z, b.z), c3.z)};
        for (int a3 = 0; a3 < 3; ++a3) {
          tbox[6ull * t + a3] = mn[a3];
          tbox[6ull * t + 3 + a3] = mx[a3];
          const double oa = origin[a3];
          const double i0 = std::max(0.0, std::ceil(((mn[a3] - o.band) - oa) / o.cell_size));
          const double i1 = std::min<double>(dims[a3] - 1, std::floor(((mx[a3] + o.band) - oa) / o.cell_size));
          trange[6ull * t + 2 * a3] = static_cast<int>(i0);
          trange[6ull * t + 2 * a3 + 1] = static_cast<int>(i1);
        }
      }
      // Edge pseudonormals: the two faces' normals summed in triangle order (the reference's map accumulation).
      std::stable_sort(edgeSum.begin(), edgeSum.end(),
                       [](const auto& x, const auto& y) { return x.first < y.first; });
      std::vector<uint64_t> keys(edgeSum.size());
      std::vector<D3> sums(edgeSum.size());
      size_t u = 0;
      for (size_t i = 0; i < edgeSum.size(); ++i) {
        if (i > 0 && edgeSum[i].first == edgeSum[i - 1].first) {
          D3& s = sums[u - 1];
          s = {s.x + edgeSum[i].second.x, s.y + edgeSum[i].second.y, s.z + edgeSum[i].second.z};
        } else {
          keys[u] = edgeSum[i].first;
          sums[u] = {0.0 + edgeSum[i].second.x, 0.0 + edgeSum[i].second.y, 0.0 + edgeSum[i].second.z};
          ++u;
        }
      }
      keys.resize(u);
      for (uint32_t t = 0; t < nt; ++t)
        for (int k = 0; k < 3; ++k) {  // edges AB, BC, CA
          const uint64_t key = edgeKey(m.triangles[3ull * t + k], m.triangles[3ull * t + (k + 1) % 3]);
          edgeN[3ull * t + k] = sums[std::lower_bound(keys.begin(), keys.end(), key) - keys.begin()];
        }
      Prepared& pr = prepared[c];
      pr.v.upload(v, st);
      pr.face.upload(faceN, st);
      pr.vert.upload(vertexN, st);
      pr.edge.upload(edgeN, st);
      pr.t.upload(tris, st);
      pr.box.upload(tbox, st);
      pr.range.upload(trange, st);
      pr.nt = nt;
      KCK(cudaStreamSynchronize(st));  // the host vectors go out of scope
    }
    KCK(cudaEventRecord(e0, st));
    bake::k_fill<<<pointGrid, 256, 0, st>>>(field.p, total, static_cast<float>(o.band));
    KCK(cudaGetLastError());
    for (uint32_t c = 0; c < count; ++c) {
      const Prepared& pr = prepared[c];
      const uint32_t nt = pr.nt;
      bake::Mesh dm{pr.v.p, pr.t.p, pr.box.p, pr.range.p, pr.face.p, pr.vert.p, pr.edge.p, nt};
      bake::k_reset<<<pointGrid, 256, 0, st>>>(dist2.p, owner.p, sign.p, total);
      const int triGrid = static_cast<int>(std::min<uint32_t>(nt, static_cast<uint32_t>(sms) * 16));
      bake::k_bake_distance<false><<<triGrid, 256, 0, st>>>(g, dm, dist2.p, owner.p);
      bake::k_bake_distance<true><<<triGrid, 256, 0, st>>>(g, dm, dist2.p, owner.p);
      bake::k_bake_sign<<<pointGrid, 256, 0, st>>>(g, dm, owner.p, sign.p, total);
      bake::k_bake_seed<<<pointGrid, 256, 0, st>>>(g, dist2.p, state.p, total);
      KCK(cudaGetLastError());
      // Sweeps until a full round of six marks nothing (bounded by the number of samples, which is never reached).
      for (size_t round = 0; round < total; ++round) {
        KCK(cudaMemsetAsync(changed.p, 0, sizeof(int), st));
        for (int axis = 0; axis < 3; ++axis)
          for (int dir : {1, -1}) {
            const size_t lines = static_cast<size_t>(axis == 0 ? dims[1] * dims[2]
                                                               : (axis == 1 ? dims[0] * dims[2] : dims[0] * dims[1]));
            const int grid = static_cast<int>(std::min<size_t>((lines + 255) / 256, static_cast<size_t>(sms) * 8));
            bake::k_bake_sweep<<<grid, 256, 0, st>>>(g, state.p, axis, dir, changed.p);
          }
        KCK(cudaGetLastError());
        int h = 0;
        KCK(cudaMemcpyAsync(&h, changed.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        KCK(cudaStreamSynchronize(st));
        if (!h) break;
      }
      bake::k_bake_combine<<<pointGrid, 256, 0, st>>>(g, dist2.p, sign.p, state.p, field.p, total);
      KCK(cudaGetLastError());
      KCK(cudaStreamSynchronize(st));
    }
    KCK(cudaEventRecord(e1, st));
    KCK(cudaMemcpyAsync(values, field.p, sizeof(float) * total, cudaMemcpyDeviceToHost, st));
    KCK(cudaStreamSynchronize(st));
    float ms = 0;
    KCK(cudaEventElapsedTime(&ms, e0, e1));
    g_bakeMs = ms;
    return DRAPE_OK;
  } catch (const std::invalid_argument& e) {
    g_bakeError = e.what();
    return DRAPE_INVALID;
  } catch (const std::exception& e) {
    g_bakeError = e.what();
    return DRAPE_DEVICE_ERROR;
  }
}

double drape_bake_last_ms(void) { return g_bakeMs; }

const char* drape_bake_last_error(void) { return g_bakeError.c_str(); }

}  // extern "C"
