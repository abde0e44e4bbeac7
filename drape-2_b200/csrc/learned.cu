// Learned preconditioner: network kernels (forward, loss, backward, Adam) and the host Network class.
//
// Tile kernels run 128 threads (4 warps). A tile is 128 rows of a GEMM: 128 nodes, 128 slots, or the slots of a
// "row tile" (consecutive rows of the block-CSR graph whose slots total at most 128, so every row's slots lie in one
// tile and per-row sums stay inside one CTA, in a fixed order). Operands are staged by the threads into shared memory
// in the K-major core-matrix layout (umma.cuh), one thread issues the tcgen05 MMAs, the accumulators live in TMEM and
// come back through tcgen05.ld (thread t of warp w owns row 32 w + t). Weight gradients accumulate in TMEM across a
// CTA's tiles and leave as per-CTA partials that a second kernel sums in CTA order: no floating-point atomics, so a
// training step is deterministic.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <stdexcept>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "device_math.cuh"
#include "learned.hpp"
#include "umma.cuh"

namespace net {

namespace {

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("cuda: ") + what + ": " + cudaGetErrorString(e));
}
#define NCK(x) ck((x), #x)

constexpr uint32_t kPinBit = 0x80000000u;
constexpr int kThreads = 128;

__device__ __forceinline__ bool pinnedRow(const Graph& g, uint32_t i) {
  return g.pinnedBase != nullptr && g.pinnedBase[static_cast<size_t>(i) * g.pinnedStride] != 0;
}
__device__ __forceinline__ bool activeRow(const Graph& g, uint32_t i) {
  return g.activeBase != nullptr && g.activeBase[static_cast<size_t>(i) * g.activeStride] != 0;
}
__device__ __forceinline__ uint32_t colOf(const Graph& g, uint32_t s) { return __ldg(g.colIndex + s) & ~kPinBit; }

__device__ __forceinline__ float blockAt(const Graph& g, uint32_t s, int k) { return __ldg(g.blocks + k * g.SP + s); }

__device__ __forceinline__ void st16(unsigned char* tile, uint32_t r, uint32_t c, uint32_t K, uint4 v) {
  *reinterpret_cast<uint4*>(tile + umma::kmajorOffset(r, c * 8u, K)) = v;
}
__device__ __forceinline__ void st1(unsigned char* tile, uint32_t r, uint32_t k, uint32_t K, __nv_bfloat16 v) {
  *reinterpret_cast<__nv_bfloat16*>(tile + umma::kmajorOffset(r, k, K)) = v;
}
__device__ __forceinline__ uint4 zero4() { return make_uint4(0u, 0u, 0u, 0u); }

__device__ __forceinline__ uint4 packBf16(const float* v) {
  uint4 out;
  uint32_t* w = reinterpret_cast<uint32_t*>(&out);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    w[i] = *reinterpret_cast<const uint32_t*>(&p);
  }
  return out;
}
__device__ __forceinline__ void unpackBf16(uint4 u, float* v) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 p = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
    v[2 * i] = __low2float(p);
    v[2 * i + 1] = __high2float(p);
  }
}
// Scatter a 16-byte chunk (8 BF16 of features 8c..8c+7 of row q) into the transposed tile (row = feature, k = q).
__device__ __forceinline__ void st16T(unsigned char* tile, uint32_t q, uint32_t c, uint32_t K, uint4 v) {
  const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&v);
#pragma unroll
  for (int i = 0; i < 8; ++i) st1(tile, c * 8u + i, q, K, e[i]);
}

// Shared state of a tile kernel: one mbarrier for MMA completion and a TMEM allocation held for the whole launch.
struct TileCtx {
  uint64_t* bar;
  uint32_t* slot;
  uint32_t tmem = 0, parity = 0, cols = 0;
  int* error;
  __device__ void init(uint64_t* b, uint32_t* s, uint32_t c, int* err) {
    bar = b;
    slot = s;
    cols = c;
    error = err;
    if (threadIdx.x == 0) umma::mbarInit(bar, 1);
    if (threadIdx.x < 32) umma::tmemAlloc(slot, cols);
    umma::fenceBeforeSync();
    __syncthreads();
    umma::fenceAfterSync();
    tmem = *slot;
  }
  // Publishes the staged operands, lets thread 0 issue the MMAs and one commit, waits for them. All threads get
  // the same verdict.
  template <class F>
  __device__ bool run(F&& issue) {
    umma::fenceSmemForMma();
    umma::fenceBeforeSync();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fenceAfterSync();
      issue();
      umma::commit(bar);
    }
    const bool good = umma::mbarWait(bar, parity, error);
    parity ^= 1u;
    umma::fenceAfterSync();
    return __syncthreads_and(good) != 0;
  }
  __device__ void done() {
    umma::fenceBeforeSync();
    __syncthreads();
    if (threadIdx.x < 32) umma::tmemFree(tmem, cols);
  }
  // Row (32 * warp + lane) of the accumulator at column `col`, 16 columns.
  __device__ void load(uint32_t col, float (&v)[16]) const {
    umma::load16(umma::tmemAt(tmem, (threadIdx.x / 32u) * 32u, col), v);
  }
};

__device__ __forceinline__ unsigned char* alignSmem(unsigned char* p) {
  return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 127u) & ~static_cast<uintptr_t>(127u));
}
extern __shared__ unsigned char netSmem[];

// ------------------------------------------------------------------------------------------------------------------
// Features

// C_i = chol(inv(A_ii)) (lower), identity when A_ii is not SPD, zero for a pinned row. One thread per row.
__global__ void k_scale(Graph g) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  float c[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (!pinnedRow(g, i)) {
    uint32_t d = __ldg(g.rowStart + i);
    const uint32_t end = __ldg(g.rowStart + i + 1);
    while (d < end && colOf(g, d) != i) ++d;
    dcu::M3 A;
    for (int k = 0; k < 9; ++k) A.m[k] = d < end ? blockAt(g, d, k) : (k % 4 == 0 ? 1.0f : 0.0f);
    bool ok = false;
    const dcu::M3 inv = dcu::invertSpd(A, ok);
    c[0] = c[4] = c[8] = 1.0f;
    if (ok) {
      const float l00s = inv.m[0];
      if (l00s > 0.0f) {
        const float l00 = sqrtf(l00s), l10 = inv.m[3] / l00, l20 = inv.m[6] / l00;
        const float l11s = inv.m[4] - l10 * l10;
        if (l11s > 0.0f) {
          const float l11 = sqrtf(l11s), l21 = (inv.m[7] - l20 * l10) / l11;
          const float l22s = inv.m[8] - l20 * l20 - l21 * l21;
          if (l22s > 0.0f) {
            c[0] = l00;
            c[1] = 0.0f;
            c[2] = 0.0f;
            c[3] = l10;
            c[4] = l11;
            c[5] = 0.0f;
            c[6] = l20;
            c[7] = l21;
            c[8] = sqrtf(l22s);
          }
        }
      }
    }
  }
  for (int k = 0; k < 9; ++k) g.C[9 * static_cast<size_t>(i) + k] = c[k];
}

// Ahat_s = C_i^T A_s C_j, slot features e_s and node features f_i. Sixteen lanes per row (two rows a warp).
__global__ void k_features(Graph g) {
  const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / 16u;
  const int lane = threadIdx.x & 15;
  const unsigned mask = 0xFFFFu << (threadIdx.x & 16);
  if (i >= g.n) return;
  const bool pi = pinnedRow(g, i);
  float Ci[9];
  for (int k = 0; k < 9; ++k) Ci[k] = g.C[9 * static_cast<size_t>(i) + k];
  float deg = 0.0f, sumFro = 0.0f, maxFro = 0.0f, rd0 = 0.0f, rd1 = 0.0f, rd2 = 0.0f;
  const uint32_t rs = __ldg(g.rowStart + i), re = __ldg(g.rowStart + i + 1);
  for (uint32_t s = rs + lane; s < re; s += 16) {
    const uint32_t j = colOf(g, s);
    const bool live = !pi && !pinnedRow(g, j);
    float ah[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (live) {
      float Cj[9], T[9];
      for (int k = 0; k < 9; ++k) Cj[k] = g.C[9 * static_cast<size_t>(j) + k];
      // T = A_s C_j; Ahat = C_i^T T.
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
          T[3 * r + c] = blockAt(g, s, 3 * r) * Cj[c] + blockAt(g, s, 3 * r + 1) * Cj[3 + c] +
                         blockAt(g, s, 3 * r + 2) * Cj[6 + c];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) ah[3 * r + c] = Ci[r] * T[c] + Ci[3 + r] * T[3 + c] + Ci[6 + r] * T[6 + c];
    }
    float fro = 0.0f;
    for (int k = 0; k < 9; ++k) fro += ah[k] * ah[k];
    fro = sqrtf(fro);
    if (g.Ahat)
      for (int k = 0; k < 9; ++k) g.Ahat[9 * static_cast<size_t>(s) + k] = ah[k];
    if (g.code) g.code[s] = j | (live ? 0u : kPinBit);
    float ev[16] = {0};
    for (int k = 0; k < 9; ++k) ev[k] = ah[k];
    ev[9] = fro;
    ev[10] = j == i ? 1.0f : 0.0f;
    ev[11] = j < i ? 1.0f : 0.0f;
    uint4* ep = reinterpret_cast<uint4*>(g.e + 16 * static_cast<size_t>(s));
    ep[0] = packBf16(ev);
    ep[1] = packBf16(ev + 8);
    if (live && j != i) {
      deg += 1.0f;
      sumFro += fro;
      maxFro = fmaxf(maxFro, fro);
      rd0 += ah[0];
      rd1 += ah[4];
      rd2 += ah[8];
    }
  }
  for (int o = 8; o > 0; o >>= 1) {
    deg += __shfl_xor_sync(mask, deg, o);
    sumFro += __shfl_xor_sync(mask, sumFro, o);
    maxFro = fmaxf(maxFro, __shfl_xor_sync(mask, maxFro, o));
    rd0 += __shfl_xor_sync(mask, rd0, o);
    rd1 += __shfl_xor_sync(mask, rd1, o);
    rd2 += __shfl_xor_sync(mask, rd2, o);
  }
  if (lane == 0) {
    float fv[16] = {0};
    fv[0] = 1.0f;
    fv[1] = (activeRow(g, i) && !pi) ? 1.0f : 0.0f;
    fv[2] = deg / 16.0f;
    fv[3] = sumFro / fmaxf(deg, 1.0f);
    fv[4] = maxFro;
    fv[5] = rd0;
    fv[6] = rd1;
    fv[7] = rd2;
    fv[8] = pi ? 1.0f : 0.0f;
    uint4* fp = reinterpret_cast<uint4*>(g.f + 16 * static_cast<size_t>(i));
    fp[0] = packBf16(fv);
    fp[1] = packBf16(fv + 8);
  }
}

// ------------------------------------------------------------------------------------------------------------------
// Encoder: out = relu(X W^T + b) for `rows` rows of 16 BF16 features; out 64 BF16 per row.

struct EncodeSmem {
  unsigned char x[128 * 16 * 2];
  unsigned char w[64 * 16 * 2];
  float b[64];
  uint64_t bar;
  uint32_t tmem;
};

__global__ void __launch_bounds__(kThreads) k_encode(uint32_t rows, const __nv_bfloat16* __restrict__ X,
                                                     const __nv_bfloat16* __restrict__ W, const float* __restrict__ b,
                                                     __nv_bfloat16* __restrict__ out, int* error) {
  EncodeSmem& S = *reinterpret_cast<EncodeSmem*>(alignSmem(netSmem));
  TileCtx T;
  T.init(&S.bar, &S.tmem, 64, error);
  const int t = threadIdx.x;
  for (int k = t; k < 64 * 2; k += kThreads)
    st16(S.w, k / 2, k % 2, 16, reinterpret_cast<const uint4*>(W)[k]);
  if (t < 64) S.b[t] = b[t];
  const uint32_t tiles = (rows + 127) / 128;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const uint32_t r0 = tile * 128;
    for (int k = t; k < 128 * 2; k += kThreads) {
      const uint32_t q = k / 2, c = k % 2, r = r0 + q;
      st16(S.x, q, c, 16, r < rows ? reinterpret_cast<const uint4*>(X + 16 * static_cast<size_t>(r))[c] : zero4());
    }
    if (!T.run([&] { umma::gemmIssue(T.tmem, S.x, S.w, 128, 64, 16, false); })) break;
    const uint32_t r = r0 + t;
    for (int c = 0; c < 4; ++c) {
      float v[16];
      T.load(16 * c, v);
      if (r < rows) {
        for (int k = 0; k < 16; ++k) v[k] = fmaxf(v[k] + S.b[16 * c + k], 0.0f);
        uint4* o = reinterpret_cast<uint4*>(out + 64 * static_cast<size_t>(r));
        o[2 * c] = packBf16(v);
        o[2 * c + 1] = packBf16(v + 8);
      }
    }
    umma::fenceBeforeSync();
    __syncthreads();
  }
  T.done();
}

// ------------------------------------------------------------------------------------------------------------------
// Message-passing layer over row tiles: m_s = relu(W_m [h_j; eps_s] + b_m) on message slots, a_i = sum m_s / 8 per
// row, h_i' = h_i + relu(W_u [h_i; a_i] + b_u).

struct TileRows {
  uint32_t r0, r1, s0, s1;
};

__device__ __forceinline__ TileRows tileRows(const Graph& g, uint32_t tile) {
  TileRows t;
  t.r0 = __ldg(g.tileRow + tile);
  t.r1 = __ldg(g.tileRow + tile + 1);
  t.s0 = __ldg(g.rowStart + t.r0);
  t.s1 = __ldg(g.rowStart + t.r1);
  return t;
}

struct LayerSmem {
  unsigned char x[128 * 128 * 2];
  unsigned char wm[64 * 128 * 2];
  unsigned char wu[64 * 128 * 2];
  float buf[128][65];
  float bm[64], bu[64];
  int slotRow[128];   // local row of slot q when it carries a message, else -1
  int rowFirst[129];  // first local slot of local row r
  uint64_t bar;
  uint32_t tmem;
};

__device__ __forceinline__ void stageWeights(unsigned char* tile, const __nv_bfloat16* W, int rows, int K) {
  const int chunks = K / 8;
  for (int k = threadIdx.x; k < rows * chunks; k += blockDim.x)
    st16(tile, k / chunks, k % chunks, K, reinterpret_cast<const uint4*>(W + static_cast<size_t>(k / chunks) * K)[k % chunks]);
}
// Transposed weights W^T (rows = K_in of W, K = rows of W) as a K-major operand.
__device__ __forceinline__ void stageWeightsT(unsigned char* tile, const __nv_bfloat16* W, int outRows, int inCols) {
  for (int k = threadIdx.x; k < outRows * inCols; k += blockDim.x) {
    const int o = k / inCols, i = k % inCols;
    st1(tile, i, o, outRows, W[static_cast<size_t>(o) * inCols + i]);
  }
}

__device__ __forceinline__ void tileSlotInfo(const Graph& g, const TileRows& tr, int* slotRow, int* rowFirst,
                                             bool messages) {
  const int t = threadIdx.x;
  for (uint32_t r = tr.r0 + t; r <= tr.r1 && r - tr.r0 <= 128; r += blockDim.x)
    rowFirst[r - tr.r0] = static_cast<int>(__ldg(g.rowStart + r) - tr.s0);
  __syncthreads();
  for (int q = t; q < 128; q += blockDim.x) {
    int row = -1;
    const uint32_t s = tr.s0 + q;
    if (s < tr.s1) {
      // Local row: the last r with rowFirst[r] <= q.
      int lo = 0, hi = static_cast<int>(tr.r1 - tr.r0) - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (rowFirst[mid] <= q) lo = mid; else hi = mid - 1;
      }
      const uint32_t i = tr.r0 + lo, j = colOf(g, s);
      const bool keep = messages ? (j != i && !pinnedRow(g, i) && !pinnedRow(g, j))
                                 : (j <= i && !pinnedRow(g, i) && !pinnedRow(g, j));
      row = keep ? lo : -(lo + 2);  // -(lo + 2): in the tile but not kept
    }
    slotRow[q] = row;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads) k_layer(Graph g, const __nv_bfloat16* __restrict__ Wm,
                                                    const __nv_bfloat16* __restrict__ Wu, const float* __restrict__ bm,
                                                    const float* __restrict__ bu, const __nv_bfloat16* __restrict__ hin,
                                                    __nv_bfloat16* __restrict__ hout, __nv_bfloat16* __restrict__ aggOut,
                                                    int* error) {
  LayerSmem& S = *reinterpret_cast<LayerSmem*>(alignSmem(netSmem));
  TileCtx T;
  T.init(&S.bar, &S.tmem, 128, error);
  const int t = threadIdx.x;
  stageWeights(S.wm, Wm, 64, 128);
  stageWeights(S.wu, Wu, 64, 128);
  if (t < 64) {
    S.bm[t] = bm[t];
    S.bu[t] = bu[t];
  }
  for (uint32_t tile = blockIdx.x; tile < g.nTiles; tile += gridDim.x) {
    const TileRows tr = tileRows(g, tile);
    tileSlotInfo(g, tr, S.slotRow, S.rowFirst, true);
    // X_msg: [h_j; eps_s] per message slot. Thread t owns 16-byte chunk c = t % 16 of slots q = t / 16 + 8 i; its 16
    // gathers are all issued before the first store into the tile, so they are in flight together.
    {
      const int c = t % 16;
      uint4 v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int q = t / 16 + 8 * i;
        v[i] = zero4();
        if (S.slotRow[q] >= 0) {
          const uint32_t s = tr.s0 + q;
          v[i] = c < 8 ? reinterpret_cast<const uint4*>(hin + 64 * static_cast<size_t>(colOf(g, s)))[c]
                       : reinterpret_cast<const uint4*>(g.eps + 64 * static_cast<size_t>(s))[c - 8];
        }
      }
#pragma unroll
      for (int i = 0; i < 16; ++i) st16(S.x, t / 16 + 8 * i, c, 128, v[i]);
    }
    if (!T.run([&] { umma::gemmIssue(T.tmem, S.x, S.wm, 128, 64, 128, false); })) break;
    {
      const bool keep = S.slotRow[t] >= 0;
      for (int c = 0; c < 4; ++c) {
        float v[16];
        T.load(16 * c, v);
        for (int k = 0; k < 16; ++k) S.buf[t][16 * c + k] = keep ? fmaxf(v[k] + S.bm[16 * c + k], 0.0f) : 0.0f;
      }
    }
    __syncthreads();
    // a_i = (1/8) sum over the row's slots, in slot order; X_upd = [h_i; a_i] (reuses the X_msg tile).
    const int R = static_cast<int>(tr.r1 - tr.r0);
    for (int k = t; k < 128 * 8; k += kThreads) {
      const int r = k / 8, c = k % 8;
      uint4 hv = zero4(), av = zero4();
      if (r < R) {
        hv = reinterpret_cast<const uint4*>(hin + 64 * static_cast<size_t>(tr.r0 + r))[c];
        float a[8];
        for (int e = 0; e < 8; ++e) {
          float sum = 0.0f;
          for (int q = S.rowFirst[r]; q < S.rowFirst[r + 1]; ++q) sum += S.buf[q][8 * c + e];
          a[e] = sum * kAggScale;
        }
        av = packBf16(a);
        if (aggOut) reinterpret_cast<uint4*>(aggOut + 64 * static_cast<size_t>(tr.r0 + r))[c] = av;
      }
      st16(S.x, r, c, 128, hv);
      st16(S.x, r, 8 + c, 128, av);
    }
    if (!T.run([&] { umma::gemmIssue(T.tmem + 64, S.x, S.wu, 128, 64, 128, false); })) break;
    for (int c = 0; c < 4; ++c) {
      float v[16];
      T.load(64 + 16 * c, v);
      if (t < R) {
        const size_t row = tr.r0 + t;
        float h[16];
        const uint4* hp = reinterpret_cast<const uint4*>(hin + 64 * row);
        unpackBf16(hp[2 * c], h);
        unpackBf16(hp[2 * c + 1], h + 8);
        for (int k = 0; k < 16; ++k) h[k] += fmaxf(v[k] + S.bu[16 * c + k], 0.0f);
        uint4* op = reinterpret_cast<uint4*>(hout + 64 * row);
        op[2 * c] = packBf16(h);
        op[2 * c + 1] = packBf16(h + 8);
      }
    }
    umma::fenceBeforeSync();
    __syncthreads();
  }
  T.done();
}

// ------------------------------------------------------------------------------------------------------------------
// Output: o_s = W_o [h_i; h_j; eps_s] + b_o on lower live slots; G_s and L_s = C_i G_s.

struct OutputSmem {
  unsigned char x[128 * 192 * 2];
  unsigned char w[16 * 192 * 2];
  float b[16];
  int slotRow[128];
  int rowFirst[129];
  uint64_t bar;
  uint32_t tmem;
};

__device__ __forceinline__ void outputToG(const float* o, bool diag, float* G) {
  if (diag) {
    G[0] = expf(fminf(fmaxf(o[0], -kDiagClamp), kDiagClamp));
    G[1] = 0.0f;
    G[2] = 0.0f;
    G[3] = o[3];
    G[4] = expf(fminf(fmaxf(o[1], -kDiagClamp), kDiagClamp));
    G[5] = 0.0f;
    G[6] = o[4];
    G[7] = o[5];
    G[8] = expf(fminf(fmaxf(o[2], -kDiagClamp), kDiagClamp));
  } else {
    for (int k = 0; k < 9; ++k) G[k] = o[k];
  }
}

__global__ void __launch_bounds__(kThreads) k_output(Graph g, const __nv_bfloat16* __restrict__ Wo,
                                                     const float* __restrict__ bo, const __nv_bfloat16* __restrict__ h,
                                                     int training, int* error) {
  OutputSmem& S = *reinterpret_cast<OutputSmem*>(alignSmem(netSmem));
  TileCtx T;
  T.init(&S.bar, &S.tmem, 32, error);
  const int t = threadIdx.x;
  stageWeights(S.w, Wo, 16, 192);
  if (t < 16) S.b[t] = bo[t];
  for (uint32_t tile = blockIdx.x; tile < g.nTiles; tile += gridDim.x) {
    const TileRows tr = tileRows(g, tile);
    tileSlotInfo(g, tr, S.slotRow, S.rowFirst, false);
    // [h_i; h_j; eps_s] per lower slot, in two rounds of 12 chunks a thread: each round's gathers are issued before
    // its first store into the tile (12 loads in flight at a moderate register count).
    for (int round = 0; round < 2; ++round) {
      uint4 v[12];
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const int k = t + kThreads * (12 * round + i), q = k / 24, c = k % 24;
        v[i] = zero4();
        const int sr = S.slotRow[q];
        if (sr >= 0) {
          const uint32_t s = tr.s0 + q;
          if (c < 8) v[i] = reinterpret_cast<const uint4*>(h + 64 * static_cast<size_t>(tr.r0 + sr))[c];
          else if (c < 16) v[i] = reinterpret_cast<const uint4*>(h + 64 * static_cast<size_t>(colOf(g, s)))[c - 8];
          else v[i] = reinterpret_cast<const uint4*>(g.eps + 64 * static_cast<size_t>(s))[c - 16];
        }
      }
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const int k = t + kThreads * (12 * round + i);
        st16(S.x, k / 24, k % 24, 192, v[i]);
      }
    }
    if (!T.run([&] { umma::gemmIssue(T.tmem, S.x, S.w, 128, 16, 192, false); })) break;
    float o[16];
    T.load(0, o);
    const int sr = S.slotRow[t];
    const uint32_t s = tr.s0 + t;
    if (s < tr.s1) {
      float G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int k = 0; k < 16; ++k) o[k] = sr >= 0 ? o[k] + S.b[k] : 0.0f;
      if (sr >= 0) {
        const uint32_t i = tr.r0 + sr;
        outputToG(o, colOf(g, s) == i, G);
        const float* C = g.C + 9 * static_cast<size_t>(i);
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) L[3 * r + c] = C[3 * r] * G[c] + C[3 * r + 1] * G[3 + c] + C[3 * r + 2] * G[6 + c];
      }
      for (int k = 0; k < 9; ++k) g.L[k * g.SP + s] = L[k];
      if (training) {
        for (int k = 0; k < 9; ++k) g.G[9 * static_cast<size_t>(s) + k] = G[k];
        for (int k = 0; k < 16; ++k) g.o[16 * static_cast<size_t>(s) + k] = o[k];
      }
    }
    umma::fenceBeforeSync();
    __syncthreads();
  }
  T.done();
}

// ------------------------------------------------------------------------------------------------------------------
// Inference path (the solver's forward; the same network as above, regrouped so that no tensor-core operand is
// gathered). The message GEMM splits by its input halves, W_m [h_j; eps_s] = W_mh h_j + W_me eps_s, and the output
// layer's likewise, W_o [h_i; h_j; eps_s] = W_oi h_i + W_oj h_j + W_oe eps_s:
//   k_slot_encode   per 128 consecutive slots (contiguous tiles): eps = relu(W_ee e + b_ee), then in one MMA the
//                   four layers' slot terms E^l = W_me^l eps + b_m^l (N = 256, stored BF16) and the output layer's
//                   F = W_oe eps + b_o (FP32); results leave through a swizzled shared-memory tile as coalesced rows;
//   k_node          per 2 x 128 consecutive rows: h' = relu(W_ne f + b_ne) (the node encoder) or h' = h + relu(W_u
//                   [h; a] + b_u) (a layer's update), then from the same tile the next layer's node term P = W_mh h'
//                   (BF16) or the output layer's Q = [W_oi h'; W_oj h'] (FP32);
//   k_message       eight lanes per row (four rows a warp): a_i = (1/8) sum over the row's message slots, in slot
//                   order, of relu(P_j + E^l_s), lane k holding features 8k..8k+7 (each slot's E and P_j are 128-byte
//                   coalesced rows);
//   k_output_slots  one thread per slot: o = F_s + Q_i + Q_j, G_s, L_s = C_i G_s.
// k_features writes each slot's code (column, bit 31 when the slot carries nothing: either row pinned), so the gathers
// need no pinned-flag lookups. The GEMMs stage only contiguous rows; every irregular access is a plain coalesced row
// gather on the CUDA cores. Against the fused tile kernels the results differ by FP32 summation order and by the BF16
// roundings of E and P.

// Loads every 16-byte chunk of rows [r0, r0 + ROWS) of a K-major operand tile of K columns, src(o, c) for row r0 + o
// chunk c (8 BF16), into registers before the first store into the tile (all in flight together), with THREADS threads.
template <int K, int ROWS, int THREADS, class Src>
__device__ __forceinline__ void stageRowsT(unsigned char* tile, int r0, Src&& src) {
  constexpr int kChunks = K / 8, kTotal = ROWS * kChunks, kPer = (kTotal + THREADS - 1) / THREADS;
  uint4 v[kPer];
#pragma unroll
  for (int m = 0; m < kPer; ++m) {
    const int k = threadIdx.x + THREADS * m;
    v[m] = k < kTotal ? src(k / kChunks, k % kChunks) : zero4();
  }
#pragma unroll
  for (int m = 0; m < kPer; ++m) {
    const int k = threadIdx.x + THREADS * m;
    if (k < kTotal) st16(tile, r0 + k / kChunks, k % kChunks, K, v[m]);
  }
}
template <int K, int ROWS, class Src>
__device__ __forceinline__ void stageRows(unsigned char* tile, int r0, Src&& src) {
  stageRowsT<K, ROWS, kThreads>(tile, r0, static_cast<Src&&>(src));
}
// Rows of W (row length ld) from column col0 as a K-major tile of K columns.
template <int K, int ROWS>
__device__ __forceinline__ void stageWeightRows(unsigned char* tile, int r0, const __nv_bfloat16* W, int ld, int col0) {
  stageRows<K, ROWS>(tile, r0, [&](int o, int c) {
    return *reinterpret_cast<const uint4*>(W + static_cast<size_t>(o) * ld + col0 + 8 * c);
  });
}

struct SlotEncSmem {
  unsigned char out[2][128 * 128];  // one layer's results (128 slots x 128 B, TMA 128-byte swizzle); 1024-B aligned
  unsigned char x[128 * 16 * 2];
  unsigned char wee[64 * 16 * 2];
  unsigned char eps[128 * 64 * 2];
  unsigned char wme[256 * 64 * 2];
  unsigned char woe[16 * 64 * 2];
  float bee[64], bm[256], bo[16];
  uint64_t bar;
  uint32_t tmem;
};

// TMA tensor stores (cp.async.bulk.tensor, bulk-group completion) from a shared-memory tile: E^l rows [s0, s0 + 128)
// of layer l through the 3-D map [layer][slot][64 BF16] (128-byte swizzle), F rows through the 2-D map [slot][16 FP32]
// (64-byte swizzle); rows past B are clipped by the maps. The writing threads fence their shared-memory stores for the
// async proxy and meet at a barrier before one thread issues.
__device__ __forceinline__ void tmaStoreE(const CUtensorMap* map, const void* tile, int slot, int layer) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(map),
               "r"(umma::smemAddr(tile)), "r"(0), "r"(slot), "r"(layer)
               : "memory");
}
__device__ __forceinline__ void tmaStoreF(const CUtensorMap* map, const void* tile, int slot) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(map),
               "r"(umma::smemAddr(tile)), "r"(0), "r"(slot)
               : "memory");
}
__device__ __forceinline__ void bulkCommit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until at most N of this thread's committed bulk groups still read their shared-memory source.
template <int N>
__device__ __forceinline__ void bulkWaitRead() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulkWaitAll() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ unsigned char* alignSmem1024(unsigned char* p) {
  return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 1023u) & ~static_cast<uintptr_t>(1023u));
}

__global__ void __launch_bounds__(kThreads) k_slot_encode(Graph g, const __grid_constant__ CUtensorMap tmE,
                                                          const __grid_constant__ CUtensorMap tmF,
                                                          const __nv_bfloat16* __restrict__ W,
                                                          const float* __restrict__ M, int* error) {
  SlotEncSmem& S = *reinterpret_cast<SlotEncSmem*>(alignSmem1024(netSmem));
  TileCtx T;
  T.init(&S.bar, &S.tmem, 256, error);
  const int t = threadIdx.x;
  stageWeightRows<16, 64>(S.wee, 0, W + Layout::kEe, 16, 0);
  for (int l = 0; l < kLayers; ++l) stageWeightRows<64, 64>(S.wme, 64 * l, W + Layout::m(l), 2 * kHidden, kHidden);
  stageWeightRows<64, kOutputs>(S.woe, 0, W + Layout::kO, 3 * kHidden, 2 * kHidden);
  for (int k = t; k < 64; k += kThreads) S.bee[k] = M[Layout::kEeB + k];
  for (int k = t; k < 256; k += kThreads) S.bm[k] = M[Layout::mB(k / 64) + k % 64];
  if (t < kOutputs) S.bo[t] = M[Layout::kOB + t];
  const uint32_t tiles = (g.B + 127) / 128;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const uint32_t s0 = tile * 128;
    // The previous tile's stores have read both staging tiles before this tile writes them (the next run's barrier
    // carries the wait to every thread).
    if (t == 0) bulkWaitRead<0>();
    stageRows<16, 128>(S.x, 0, [&](int q, int c) {
      const uint32_t s = s0 + q;
      return s < g.B ? reinterpret_cast<const uint4*>(g.e + 16 * static_cast<size_t>(s))[c] : zero4();
    });
    if (!T.run([&] { umma::gemmIssue(T.tmem, S.x, S.wee, 128, 64, 16, false); })) break;
    for (int c = 0; c < 4; ++c) {
      float v[16];
      T.load(16 * c, v);
      for (int k = 0; k < 16; ++k) v[k] = fmaxf(v[k] + S.bee[16 * c + k], 0.0f);
      st16(S.eps, t, 2 * c, 64, packBf16(v));
      st16(S.eps, t, 2 * c + 1, 64, packBf16(v + 8));
    }
    if (!T.run([&] { umma::gemmIssue(T.tmem, S.eps, S.wme, 128, 256, 64, false); })) break;
    // Layer l: thread t writes its slot's 8 chunks into row t of out[l & 1] (chunk c at c ^ (t & 7), the TMA's
    // 128-byte swizzle: the eight lanes of a store phase hit eight different bank groups); one thread stores the tile.
    for (int l = 0; l < kLayers; ++l) {
      unsigned char* buf = S.out[l & 1];
      if (l >= 2) {
        if (t == 0) bulkWaitRead<1>();  // layer l - 2's store has read buf
        __syncthreads();
      }
      for (int c = 0; c < 4; ++c) {
        float v[16];
        T.load(64 * l + 16 * c, v);
        for (int k = 0; k < 16; ++k) v[k] += S.bm[64 * l + 16 * c + k];
        *reinterpret_cast<uint4*>(buf + 128 * t + 16 * ((2 * c) ^ (t & 7))) = packBf16(v);
        *reinterpret_cast<uint4*>(buf + 128 * t + 16 * ((2 * c + 1) ^ (t & 7))) = packBf16(v + 8);
      }
      umma::fenceSmemForMma();  // fence.proxy.async.shared::cta: the stores, for the TMA's reads
      __syncthreads();
      if (t == 0) {
        tmaStoreE(&tmE, buf, static_cast<int>(s0), l);
        bulkCommit();
      }
    }
    if (!T.run([&] { umma::gemmIssue(T.tmem, S.eps, S.woe, 128, kOutputs, 64, false); })) break;
    {
      // F: 64 B a slot, rows of 4 chunks (chunk c at c ^ ((t >> 1) & 3), the TMA's 64-byte swizzle), in out[0] once
      // layer 2's store has read it.
      if (t == 0) bulkWaitRead<1>();
      __syncthreads();
      unsigned char* buf = S.out[0];
      float v[16];
      T.load(0, v);
      for (int c = 0; c < 4; ++c)
        *reinterpret_cast<float4*>(buf + 64 * t + 16 * (c ^ ((t >> 1) & 3))) =
            make_float4(v[4 * c] + S.bo[4 * c], v[4 * c + 1] + S.bo[4 * c + 1], v[4 * c + 2] + S.bo[4 * c + 2],
                        v[4 * c + 3] + S.bo[4 * c + 3]);
      umma::fenceSmemForMma();
      __syncthreads();
      if (t == 0) {
        tmaStoreF(&tmF, buf, static_cast<int>(s0));
        bulkCommit();
      }
    }
    umma::fenceBeforeSync();
    __syncthreads();
  }
  if (t == 0) bulkWaitAll();  // every store has landed before the block's shared memory goes
  T.done();
}

// Two row tiles per block (256 threads: warps 0-3 take tile 0, warps 4-7 tile 1; TMEM columns [128 u, 128 u + 128)
// hold tile u's accumulators), so that the n / 128 tiles of a graph run in one wave at two blocks per SM. Tile u's
// operand x[u] is [h; a] (K = 128) or f (K = 16); h' goes back into x[u] as a K = 64 operand: into the a columns
// (dead after the first MMA; start + 1024, 8-row groups 2048 B apart) for K = 128, behind the f tile (start + 16 KB,
// the plain K = 64 layout) for K = 16.
struct NodeSmem {
  unsigned char x[2][128 * 128 * 2];
  unsigned char w1[64 * 128 * 2];
  unsigned char w2[64 * 64 * 2];
  float b1[64];
  uint64_t bar;
  uint32_t tmem;
};
constexpr int kNodeThreads = 256;

// K1 = 16: h' = relu(W1 f + b1) (node encoder; X = f). K1 = 128: h' = h + relu(W1 [h; a] + b1) (a layer's update).
// Then Out = W2 h' (N2 rows of W2: rows 0..N2-1 of the tile from W2's columns col2a, or for N2 = 32 rows 0..15 from
// col2a and 16..31 from col2b): N2 = 64, BF16 (the next layer's P); N2 = 32, FP32 (the output layer's Q); either way
// 128 bytes a row. h' and Out leave through shared memory as coalesced 128-byte rows: h' read back from its operand
// layout, Out from a swizzled staging tile in x[u] (16-byte chunk c of row q at c ^ (q & 7)).
template <int K1, int N2>
__global__ void __launch_bounds__(kNodeThreads, 2) k_node(uint32_t n, const __nv_bfloat16* __restrict__ X,
                                                       const __nv_bfloat16* __restrict__ A,
                                                       const __nv_bfloat16* __restrict__ W1,
                                                       const float* __restrict__ b1,
                                                       const __nv_bfloat16* __restrict__ W2, int ld2, int col2a,
                                                       int col2b, __nv_bfloat16* __restrict__ hout,
                                                       void* __restrict__ out, int* error) {
  NodeSmem& S = *reinterpret_cast<NodeSmem*>(alignSmem(netSmem));
  TileCtx T;
  T.init(&S.bar, &S.tmem, 256, error);
  const int t = threadIdx.x, u = t / 128, q = t % 128;  // tile u, row q of it
  auto weights = [&](int o, int c, const __nv_bfloat16* W, int ld, int col0) {
    return *reinterpret_cast<const uint4*>(W + static_cast<size_t>(o) * ld + col0 + 8 * c);
  };
  stageRowsT<K1, 64, kNodeThreads>(S.w1, 0, [&](int o, int c) { return weights(o, c, W1, K1, 0); });
  if (N2 == 64) {
    stageRowsT<64, 64, kNodeThreads>(S.w2, 0, [&](int o, int c) { return weights(o, c, W2, ld2, col2a); });
  } else {
    stageRowsT<64, 16, kNodeThreads>(S.w2, 0, [&](int o, int c) { return weights(o, c, W2, ld2, col2a); });
    stageRowsT<64, 16, kNodeThreads>(S.w2, 16, [&](int o, int c) { return weights(o, c, W2, ld2, col2b); });
  }
  if (t < 64) S.b1[t] = b1[t];
  constexpr uint32_t kHbOffset = K1 == 128 ? 1024u : 16384u, kHbSbo = K1 == 128 ? 2048u : 1024u;
  const uint32_t tiles = (n + 127) / 128, pairs = (tiles + 1) / 2;
  // This thread's TMEM lane group (warp % 4) and tile u's columns.
  const uint32_t tm = umma::tmemAt(T.tmem, ((t / 32) % 4) * 32, 128 * u);
  for (uint32_t pair = blockIdx.x; pair < pairs; pair += gridDim.x) {
    const uint32_t rBase = pair * 256;  // tile u covers rows rBase + 128 u ...
    if (K1 == 16) {
      for (int v = 0; v < 2; ++v)
        stageRowsT<16, 128, kNodeThreads>(S.x[v], 0, [&](int rr, int c) {
          const uint32_t r = rBase + 128 * v + rr;
          return r < n ? reinterpret_cast<const uint4*>(X + 16 * static_cast<size_t>(r))[c] : zero4();
        });
    } else {
      // 256 rows x 16 chunks as one K = 128 operand of 256 rows: rows 128..255 land in x[1] (x[0] is exactly 128 rows).
      stageRowsT<128, 256, kNodeThreads>(S.x[0], 0, [&](int rr, int c) {
        const uint32_t r = rBase + rr;
        if (r >= n) return zero4();
        return c < 8 ? reinterpret_cast<const uint4*>(X + 64 * static_cast<size_t>(r))[c]
                     : reinterpret_cast<const uint4*>(A + 64 * static_cast<size_t>(r))[c - 8];
      });
    }
    if (!T.run([&] {
          for (int v = 0; v < 2; ++v) umma::gemmIssue(T.tmem + 128 * v, S.x[v], S.w1, 128, 64, K1, false);
        }))
      break;
    unsigned char* xu = S.x[u];
    for (int c = 0; c < 4; ++c) {
      float v[16];
      umma::load16(tm + 16 * c, v);
      for (int k = 0; k < 16; ++k) v[k] = fmaxf(v[k] + S.b1[16 * c + k], 0.0f);
      if (K1 == 128) {
        float h[16];
        unpackBf16(*reinterpret_cast<const uint4*>(xu + umma::kmajorOffset(q, 16 * c, 128)), h);
        unpackBf16(*reinterpret_cast<const uint4*>(xu + umma::kmajorOffset(q, 16 * c + 8, 128)), h + 8);
        for (int k = 0; k < 16; ++k) v[k] += h[k];
      }
      // h' chunks 2c, 2c + 1 of row q, in the operand layout described above.
      if (K1 == 128) {
        st16(xu, q, 8 + 2 * c, 128, packBf16(v));
        st16(xu, q, 9 + 2 * c, 128, packBf16(v + 8));
      } else {
        st16(xu + kHbOffset, q, 2 * c, 64, packBf16(v));
        st16(xu + kHbOffset, q, 2 * c + 1, 64, packBf16(v + 8));
      }
    }
    if (!T.run([&] {
          const uint64_t bDesc = umma::smemDesc(S.w2, 64);
          for (int v = 0; v < 2; ++v)
            umma::gemmIssueDesc(T.tmem + 128 * v + 64, umma::smemDescSbo(S.x[v] + kHbOffset, kHbSbo), bDesc, 128,
                                N2, 64, false);
        }))
      break;
    // h' out: chunk k of the pair's 2 x 128 rows x 8 chunks (tile k / 1024), read from its operand layout.
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int k = t + kNodeThreads * m, v = k >> 10, row = (k >> 3) & 127, c = k & 7;
      const uint32_t r = rBase + 128 * v + row;
      const unsigned char* src = K1 == 128 ? S.x[v] + umma::kmajorOffset(row, 64 + 8 * c, 128)
                                           : S.x[v] + kHbOffset + umma::kmajorOffset(row, 8 * c, 64);
      if (r < n) reinterpret_cast<uint4*>(hout + 64 * static_cast<size_t>(r))[c] = *reinterpret_cast<const uint4*>(src);
    }
    __syncthreads();  // x[u] is now free for the staging tile
    {
      uint4 w[8];
      if (N2 == 64) {
        for (int c = 0; c < 4; ++c) {
          float v[16];
          umma::load16(tm + 64 + 16 * c, v);
          w[2 * c] = packBf16(v);
          w[2 * c + 1] = packBf16(v + 8);
        }
      } else {
        for (int c = 0; c < 2; ++c) {
          float v[16];
          umma::load16(tm + 64 + 16 * c, v);
          for (int k = 0; k < 4; ++k) w[4 * c + k] = make_uint4(__float_as_uint(v[4 * k]), __float_as_uint(v[4 * k + 1]),
                                                                 __float_as_uint(v[4 * k + 2]), __float_as_uint(v[4 * k + 3]));
        }
      }
      for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(xu + 128 * q + 16 * (c ^ (q & 7))) = w[c];
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int k = t + kNodeThreads * m, v = k >> 10, row = (k >> 3) & 127, c = k & 7;
      const uint32_t r = rBase + 128 * v + row;
      if (r < n)
        reinterpret_cast<uint4*>(out)[8 * static_cast<size_t>(r) + c] =
            *reinterpret_cast<const uint4*>(S.x[v] + 128 * row + 16 * (c ^ (row & 7)));
    }
    umma::fenceBeforeSync();
    __syncthreads();
  }
  T.done();
}

// slotRow[s] = the row of slot s. One thread per row; run once per graph.
__global__ void k_slot_rows(Graph g) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  for (uint32_t s = __ldg(g.rowStart + i); s < __ldg(g.rowStart + i + 1); ++s) g.slotRow[s] = i;
}

// Eight lanes per row (four rows a warp): a_i = (1/8) sum of relu(P_j + E_s) over the row's message slots (code
// without bit 31, j != i) in slot order; lane k of the row's eight accumulates features 8k..8k+7. The row's codes are
// read eight at a time (one a lane) and shared by shuffles; four slots' E and P_j rows are loaded before the first add.
__global__ void k_message(Graph g, const __nv_bfloat16* __restrict__ P, const __nv_bfloat16* __restrict__ E,
                          __nv_bfloat16* __restrict__ aOut) {
  const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t i = gt / 8u;
  const int sub = threadIdx.x & 7;
  const unsigned mask = 0xFFu << (threadIdx.x & 24);
  const bool row = i < g.n;
  const uint32_t rs = row ? __ldg(g.rowStart + i) : 0u, re = row ? __ldg(g.rowStart + i + 1) : 0u;
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // Every lane of a row group loops the same number of times (the row's slot count).
  for (uint32_t base = rs; base < re; base += 8) {
    const uint32_t cnt = min(8u, re - base);
    const uint32_t myCode = sub < static_cast<int>(cnt) ? __ldg(g.code + base + sub) : kPinBit;
#pragma unroll
    for (int k0 = 0; k0 < 8; k0 += 4) {
      uint4 e[4], pv[4];
      bool kp[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t code = __shfl_sync(mask, myCode, k0 + u, 8);
        const uint32_t j = code & ~kPinBit;
        kp[u] = !(code & kPinBit) && j != i;
        e[u] = pv[u] = zero4();
        if (kp[u]) {
          e[u] = __ldg(reinterpret_cast<const uint4*>(E + 64 * static_cast<size_t>(base + k0 + u)) + sub);
          pv[u] = __ldg(reinterpret_cast<const uint4*>(P + 64 * static_cast<size_t>(j)) + sub);
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (!kp[u]) continue;
        float ev[8], pf[8];
        unpackBf16(e[u], ev);
        unpackBf16(pv[u], pf);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += fmaxf(pf[k] + ev[k], 0.0f);
      }
    }
  }
  if (row) {
    for (int k = 0; k < 8; ++k) acc[k] *= kAggScale;
    reinterpret_cast<uint4*>(aOut + 64 * static_cast<size_t>(i))[sub] = packBf16(acc);
  }
}

// One thread per slot: L_s = C_i G_s on lower live slots (o = F_s + Q_i[0..8] + Q_j[16..24]), zero on the others.
__global__ void k_output_slots(Graph g, const float* __restrict__ Q) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.B) return;
  const uint32_t code = __ldg(g.code + s), i = __ldg(g.slotRow + s), j = code & ~kPinBit;
  float L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (!(code & kPinBit) && j <= i) {
    const float4* f = reinterpret_cast<const float4*>(g.F + kOutputs * static_cast<size_t>(s));
    const float4* qi = reinterpret_cast<const float4*>(Q + 32 * static_cast<size_t>(i));
    const float4* qj = reinterpret_cast<const float4*>(Q + 32 * static_cast<size_t>(j) + 16);
    const float4 f0 = __ldg(f), f1 = __ldg(f + 1), f2 = __ldg(f + 2);
    const float4 a0 = __ldg(qi), a1 = __ldg(qi + 1), a2 = __ldg(qi + 2);
    const float4 b0 = __ldg(qj), b1 = __ldg(qj + 1), b2 = __ldg(qj + 2);
    float C[9];
    for (int k = 0; k < 9; ++k) C[k] = __ldg(g.C + 9 * static_cast<size_t>(i) + k);
    const float fv[9] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w, f2.x};
    const float av[9] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x};
    const float bv[9] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w, b2.x};
    float o[9], G[9];
    for (int k = 0; k < 9; ++k) o[k] = fv[k] + av[k] + bv[k];
    outputToG(o, j == i, G);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) L[3 * r + c] = C[3 * r] * G[c] + C[3 * r + 1] * G[3 + c] + C[3 * r + 2] * G[6 + c];
  }
  for (int k = 0; k < 9; ++k) g.L[k * g.SP + s] = L[k];
  if (g.LF != nullptr && j <= i) {
    // The block by rows at its own slot and, below the diagonal, at its transposed slot too (every upper slot has its
    // lower counterpart, so every slot of LF is written).
    const float4 r0 = make_float4(L[0], L[1], L[2], 0.0f), r1 = make_float4(L[3], L[4], L[5], 0.0f),
                 r2 = make_float4(L[6], L[7], L[8], 0.0f);
    float4* o = g.LF + 3 * static_cast<size_t>(s);
    o[0] = r0;
    o[1] = r1;
    o[2] = r2;
    if (j < i) {
      float4* u = g.LF + 3 * static_cast<size_t>(__ldg(g.tslot + s));
      u[0] = r0;
      u[1] = r1;
      u[2] = r2;
    }
  }
}

// ------------------------------------------------------------------------------------------------------------------
// Loss: rhat = S^T r, a = G^T rhat, b = G a, e = Ahat b - rhat; backward to d loss / d o. Vectors are float4 (xyz).

__device__ __forceinline__ float3 ld3(const float4* p, uint32_t i) {
  const float4 v = p[i];
  return make_float3(v.x, v.y, v.z);
}
__device__ __forceinline__ float3 mulM(const float* M, float3 x) {
  return make_float3(M[0] * x.x + M[1] * x.y + M[2] * x.z, M[3] * x.x + M[4] * x.y + M[5] * x.z,
                     M[6] * x.x + M[7] * x.y + M[8] * x.z);
}
__device__ __forceinline__ float3 mulMT(const float* M, float3 x) {
  return make_float3(M[0] * x.x + M[3] * x.y + M[6] * x.z, M[1] * x.x + M[4] * x.y + M[7] * x.z,
                     M[2] * x.x + M[5] * x.y + M[8] * x.z);
}

__device__ inline void blockSumD(double v, double* out) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < static_cast<int>((blockDim.x + 31) / 32); ++w) s += red[w];
    *out = s;
  }
}

// rhat_i = C_i^T r_i; partial |rhat|^2 per block.
__global__ void k_rhat(Graph g, const float* __restrict__ r, float4* rhat, double* partial) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < g.n) {
    const float3 x = make_float3(r[3 * i], r[3 * i + 1], r[3 * i + 2]);
    const float3 y = mulMT(g.C + 9 * static_cast<size_t>(i), x);
    rhat[i] = make_float4(y.x, y.y, y.z, 0.0f);
    v = static_cast<double>(y.x) * y.x + static_cast<double>(y.y) * y.y + static_cast<double>(y.z) * y.z;
  }
  blockSumD(v, partial + blockIdx.x);
}

// y_j = sum_{slots (j, i), i >= j} M_{(i, j)}^T x_i, M given per slot (B x 9, zero off the lower live slots).
__global__ void k_lower_t(Graph g, const float* __restrict__ M, const float4* __restrict__ x, float4* y) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= g.n) return;
  float3 acc = make_float3(0, 0, 0);
  for (uint32_t s = __ldg(g.rowStart + j); s < __ldg(g.rowStart + j + 1); ++s) {
    const uint32_t i = colOf(g, s);
    if (i < j) continue;
    const float3 v = mulMT(M + 9 * static_cast<size_t>(__ldg(g.tslot + s)), ld3(x, i));
    acc.x += v.x;
    acc.y += v.y;
    acc.z += v.z;
  }
  y[j] = make_float4(acc.x, acc.y, acc.z, 0.0f);
}

// y_i = sum_{j <= i} M_s x_j.
__global__ void k_lower(Graph g, const float* __restrict__ M, const float4* __restrict__ x, float4* y) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  float3 acc = make_float3(0, 0, 0);
  for (uint32_t s = __ldg(g.rowStart + i); s < __ldg(g.rowStart + i + 1); ++s) {
    const uint32_t j = colOf(g, s);
    if (j > i) continue;
    const float3 v = mulM(M + 9 * static_cast<size_t>(s), ld3(x, j));
    acc.x += v.x;
    acc.y += v.y;
    acc.z += v.z;
  }
  y[i] = make_float4(acc.x, acc.y, acc.z, 0.0f);
}

// y = Ahat x (- sub when given); partial |y|^2 per block.
__global__ void k_ahat(Graph g, const float4* __restrict__ x, const float4* __restrict__ sub, float4* y,
                       double* partial) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < g.n) {
    float3 acc = make_float3(0, 0, 0);
    for (uint32_t s = __ldg(g.rowStart + i); s < __ldg(g.rowStart + i + 1); ++s) {
      const float3 w = mulM(g.Ahat + 9 * static_cast<size_t>(s), ld3(x, colOf(g, s)));
      acc.x += w.x;
      acc.y += w.y;
      acc.z += w.z;
    }
    if (sub) {
      const float3 b = ld3(sub, i);
      acc.x -= b.x;
      acc.y -= b.y;
      acc.z -= b.z;
    }
    y[i] = make_float4(acc.x, acc.y, acc.z, 0.0f);
    v = static_cast<double>(acc.x) * acc.x + static_cast<double>(acc.y) * acc.y + static_cast<double>(acc.z) * acc.z;
  }
  blockSumD(v, partial + blockIdx.x);
}

// out[k] = sum of `count` partials (one block, fixed order).
__global__ void k_sum(const double* partial, int count, double* out) {
  __shared__ double s[256];
  double v = 0.0;
  for (int k = threadIdx.x; k < count; k += blockDim.x) v += partial[k];
  s[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < static_cast<int>(blockDim.x); ++k) t += s[k];
    *out = t;
  }
}

// ge = 2 e / |rhat|^2 (scalars[0] = |rhat|^2).
__global__ void k_ge(uint32_t n, const float4* e, const double* scalars, float4* ge) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float s = static_cast<float>(2.0 / scalars[0]);
  const float4 v = e[i];
  ge[i] = make_float4(v.x * s, v.y * s, v.z * s, 0.0f);
}

// d loss / d o per slot: gG = gb_i a_j^T + rhat_i ga_j^T on lower live slots, mapped through G(o). One warp per row.
__global__ void k_grad_o(Graph g, const float4* gb, const float4* a, const float4* rhat, const float4* ga,
                         float* go) {
  const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const int lane = threadIdx.x & 31;
  if (i >= g.n) return;
  const bool pi = pinnedRow(g, i);
  const float3 gbi = ld3(gb, i), ri = ld3(rhat, i);
  for (uint32_t s = __ldg(g.rowStart + i) + lane; s < __ldg(g.rowStart + i + 1); s += 32) {
    const uint32_t j = colOf(g, s);
    float out[16] = {0};
    if (!pi && !pinnedRow(g, j) && j <= i) {
      const float3 aj = ld3(a, j), gaj = ld3(ga, j);
      const float u[3] = {gbi.x, gbi.y, gbi.z}, v[3] = {aj.x, aj.y, aj.z};
      const float p[3] = {ri.x, ri.y, ri.z}, w[3] = {gaj.x, gaj.y, gaj.z};
      float gG[9];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) gG[3 * r + c] = u[r] * v[c] + p[r] * w[c];
      if (j == i) {
        const float* o = g.o + 16 * static_cast<size_t>(s);
        for (int k = 0; k < 3; ++k) {
          const float ok = o[k];
          out[k] = fabsf(ok) < kDiagClamp ? gG[4 * k] * expf(ok) : 0.0f;
        }
        out[3] = gG[3];
        out[4] = gG[6];
        out[5] = gG[7];
      } else {
        for (int k = 0; k < 9; ++k) out[k] = gG[k];
      }
    }
    float4* dst = reinterpret_cast<float4*>(go + 16 * static_cast<size_t>(s));
    for (int k = 0; k < 4; ++k) dst[k] = make_float4(out[4 * k], out[4 * k + 1], out[4 * k + 2], out[4 * k + 3]);
  }
}

// Kaporin objective on a probe w: b = G w, c = Ahat b, t = b.c (k_ahat_dot), logdet = sum of clamped o0..o2 over live
// diagonal slots (k_logdet); d/dG_(i,j) = (2 / t) c_i w_j^T, d/do_k (diagonal) -= 2 / N.
__global__ void k_ahat_dot(Graph g, const float4* __restrict__ x, float4* y, double* partial) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < g.n) {
    float3 acc = make_float3(0, 0, 0);
    for (uint32_t s = __ldg(g.rowStart + i); s < __ldg(g.rowStart + i + 1); ++s) {
      const float3 w = mulM(g.Ahat + 9 * static_cast<size_t>(s), ld3(x, colOf(g, s)));
      acc.x += w.x;
      acc.y += w.y;
      acc.z += w.z;
    }
    y[i] = make_float4(acc.x, acc.y, acc.z, 0.0f);
    const float3 xi = ld3(x, i);
    v = static_cast<double>(xi.x) * acc.x + static_cast<double>(xi.y) * acc.y + static_cast<double>(xi.z) * acc.z;
  }
  blockSumD(v, partial + blockIdx.x);
}

__global__ void k_logdet(Graph g, double* partial) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < g.n && !pinnedRow(g, i)) {
    uint32_t d = __ldg(g.rowStart + i);
    while (d < __ldg(g.rowStart + i + 1) && colOf(g, d) != i) ++d;
    const float* o = g.o + 16 * static_cast<size_t>(d);
    for (int k = 0; k < 3; ++k) v += fminf(fmaxf(o[k], -kDiagClamp), kDiagClamp);
  }
  blockSumD(v, partial + blockIdx.x);
}

// One warp per row. scalars[0] = t; invN = 1 / N.
__global__ void k_grad_o_kaporin(Graph g, const float4* c, const float4* w, const double* scalars, float invN,
                                 float* go) {
  const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const int lane = threadIdx.x & 31;
  if (i >= g.n) return;
  const bool pi = pinnedRow(g, i);
  const float scale = static_cast<float>(2.0 / scalars[0]);
  const float3 ci = ld3(c, i);
  for (uint32_t s = __ldg(g.rowStart + i) + lane; s < __ldg(g.rowStart + i + 1); s += 32) {
    const uint32_t j = colOf(g, s);
    float out[16] = {0};
    if (!pi && !pinnedRow(g, j) && j <= i) {
      const float3 wj = ld3(w, j);
      const float u[3] = {ci.x * scale, ci.y * scale, ci.z * scale}, v[3] = {wj.x, wj.y, wj.z};
      float gG[9];
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) gG[3 * r + k] = u[r] * v[k];
      if (j == i) {
        const float* o = g.o + 16 * static_cast<size_t>(s);
        for (int k = 0; k < 3; ++k) {
          const bool inside = fabsf(o[k]) < kDiagClamp;
          out[k] = inside ? gG[4 * k] * expf(o[k]) - 2.0f * invN : 0.0f;
        }
        out[3] = gG[3];
        out[4] = gG[6];
        out[5] = gG[7];
      } else {
        for (int k = 0; k < 9; ++k) out[k] = gG[k];
      }
    }
    float4* dst = reinterpret_cast<float4*>(go + 16 * static_cast<size_t>(s));
    for (int k = 0; k < 4; ++k) dst[k] = make_float4(out[4 * k], out[4 * k + 1], out[4 * k + 2], out[4 * k + 3]);
  }
}

// ------------------------------------------------------------------------------------------------------------------
// Backward, output layer (row tiles): gX = go W_o -> gh_i (row sums into GH), gh_j (GSLOT), geps (GEPS);
// dW_o^T += X^T go accumulated in TMEM; db_o.

struct BwOutSmem {
  unsigned char a[128 * 16 * 2];    // go tile (M = 128 slots, K = 16)
  unsigned char wt[192 * 16 * 2];   // W_o^T (N = 192, K = 16)
  unsigned char xt[256 * 128 * 2];  // X_out^T (M = 256 features (192 used), K = 128 slots)
  unsigned char gt[16 * 128 * 2];   // go^T (N = 16, K = 128)
  float buf[128][65];
  float gof[128][17];
  int slotRow[128];
  int rowFirst[129];
  uint64_t bar;
  uint32_t tmem;
};

__global__ void __launch_bounds__(kThreads) k_bw_output(Graph g, const __nv_bfloat16* __restrict__ Wo,
                                                        const __nv_bfloat16* __restrict__ h,
                                                        const float* __restrict__ go, float* GH, float* GSLOT,
                                                        float* GEPS, float* partials, int* error) {
  BwOutSmem& S = *reinterpret_cast<BwOutSmem*>(alignSmem(netSmem));
  TileCtx T;
  T.init(&S.bar, &S.tmem, 256, error);
  const int t = threadIdx.x;
  stageWeightsT(S.wt, Wo, 16, 192);
  for (int k = t; k < 64 * 128; k += kThreads) st1(S.xt, 192 + k / 128, k % 128, 128, __float2bfloat16_rn(0.0f));
  float dbAcc = 0.0f;
  bool first = true, good = true;
  for (uint32_t tile = blockIdx.x; tile < g.nTiles; tile += gridDim.x) {
    const TileRows tr = tileRows(g, tile);
    tileSlotInfo(g, tr, S.slotRow, S.rowFirst, false);
    const uint32_t nq = tr.s1 - tr.s0;
    {
      float v[16] = {0};
      if (t < static_cast<int>(nq)) {
        const float4* src = reinterpret_cast<const float4*>(go + 16 * static_cast<size_t>(tr.s0 + t));
        for (int k = 0; k < 4; ++k) {
          const float4 w = src[k];
          v[4 * k] = w.x;
          v[4 * k + 1] = w.y;
          v[4 * k + 2] = w.z;
          v[4 * k + 3] = w.w;
        }
      }
      float rv[16];
      const uint4 p0 = packBf16(v), p1 = packBf16(v + 8);
      unpackBf16(p0, rv);
      unpackBf16(p1, rv + 8);
      st16(S.a, t, 0, 16, p0);
      st16(S.a, t, 1, 16, p1);
      for (int k = 0; k < 16; ++k) {
        S.gof[t][k] = rv[k];
        st1(S.gt, k, t, 128, __float2bfloat16_rn(rv[k]));
      }
    }
    for (int k = t; k < 128 * 24; k += kThreads) {
      const int q = k / 24, c = k % 24;
      uint4 v = zero4();
      if (q < static_cast<int>(nq)) {
        const uint32_t s = tr.s0 + q;
        const int sr = S.slotRow[q] >= 0 ? S.slotRow[q] : -S.slotRow[q] - 2;
        if (c < 8) v = reinterpret_cast<const uint4*>(h + 64 * static_cast<size_t>(tr.r0 + sr))[c];
        else if (c < 16) v = reinterpret_cast<const uint4*>(h + 64 * static_cast<size_t>(colOf(g, s)))[c - 8];
        else v = reinterpret_cast<const uint4*>(g.eps + 64 * static_cast<size_t>(s))[c - 16];
      }
      st16T(S.xt, q, c, 128, v);
    }
    const bool acc = !first;
    good = T.run([&] {
      umma::gemmIssue(T.tmem, S.a, S.wt, 128, 192, 16, false);
      umma::gemmIssue(T.tmem + 192, S.xt, S.gt, 128, 16, 128, acc);
      umma::gemmIssue(T.tmem + 224, S.xt + 16 * (16 * 128), S.gt, 128, 16, 128, acc);
    });
    if (!good) break;
    first = false;
    for (int c = 0; c < 12; ++c) {
      float v[16];
      T.load(16 * c, v);
      if (t < static_cast<int>(nq)) {
        const size_t s = tr.s0 + t;
        if (c < 4) {
          for (int k = 0; k < 16; ++k) S.buf[t][16 * c + k] = v[k];
        } else if (c < 8) {
          float4* d = reinterpret_cast<float4*>(GSLOT + 64 * s + 16 * (c - 4));
          for (int k = 0; k < 4; ++k) d[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
        } else {
          float4* d = reinterpret_cast<float4*>(GEPS + 64 * s + 16 * (c - 8));
          for (int k = 0; k < 4; ++k) d[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
        }
      }
    }
    __syncthreads();
    const int R = static_cast<int>(tr.r1 - tr.r0);
    for (int k = t; k < R * 64; k += kThreads) {
      const int r = k / 64, f = k % 64;
      float sum = 0.0f;
      for (int q = S.rowFirst[r]; q < S.rowFirst[r + 1]; ++q) sum += S.buf[q][f];
      GH[64 * static_cast<size_t>(tr.r0 + r) + f] = sum;
    }
    if (t < 16)
      for (int q = 0; q < static_cast<int>(nq); ++q) dbAcc += S.gof[q][t];
    umma::fenceBeforeSync();
    __syncthreads();
  }
  float* P = partials + static_cast<size_t>(blockIdx.x) * (Layout::kOB - Layout::kO + kOutputs);
  if (good && !first) {
    for (int blk = 0; blk < 2; ++blk) {
      float v[16];
      T.load(192 + 32 * blk, v);
      const int m = 128 * blk + t;
      if (m < 192)
        for (int o = 0; o < 16; ++o) P[o * 192 + m] = v[o];
    }
  } else {
    for (int k = t; k < 16 * 192; k += kThreads) P[k] = 0.0f;
  }
  if (t < 16) P[16 * 192 + t] = dbAcc;
  T.done();
}

// GH[j] (+)= sum over slots (j, i) of GSLOT[(i, j)]: messages (i != j, both live) or lower slots (i >= j).
__global__ void k_gather(Graph g, const float* __restrict__ GSLOT, float* GH, int messages) {
  const uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const int lane = threadIdx.x & 31;
  if (j >= g.n) return;
  const bool pj = pinnedRow(g, j);
  float a0 = GH[64 * static_cast<size_t>(j) + lane], a1 = GH[64 * static_cast<size_t>(j) + 32 + lane];
  for (uint32_t s = __ldg(g.rowStart + j); s < __ldg(g.rowStart + j + 1); ++s) {
    const uint32_t i = colOf(g, s);
    const bool keep = messages ? (i != j && !pj && !pinnedRow(g, i)) : (i >= j);
    if (!keep) continue;
    const size_t ts = __ldg(g.tslot + s);
    a0 += GSLOT[64 * ts + lane];
    a1 += GSLOT[64 * ts + 32 + lane];
  }
  GH[64 * static_cast<size_t>(j) + lane] = a0;
  GH[64 * static_cast<size_t>(j) + 32 + lane] = a1;
}

// ------------------------------------------------------------------------------------------------------------------
// Backward, one message-passing layer (row tiles).

struct BwLayerSmem {
  unsigned char x[128 * 128 * 2];   // X_upd, then X_msg (M = 128, K = 128)
  unsigned char xt[128 * 128 * 2];  // transposed X (M = 128 features, K = 128 rows / slots)
  unsigned char ga[128 * 64 * 2];   // gu / gv (M = 128, K = 64)
  unsigned char gt[64 * 128 * 2];   // gu^T / gv^T (N = 64, K = 128)
  unsigned char wu[64 * 128 * 2];   // W_u (N = 64, K = 128)
  unsigned char wm[64 * 128 * 2];   // W_m
  unsigned char wut[128 * 64 * 2];  // W_u^T (N = 128, K = 64)
  unsigned char wmt[128 * 64 * 2];  // W_m^T
  float buf[128][65];
  float bu[64], bm[64];
  int slotRow[128];
  int rowFirst[129];
  uint64_t bar;
  uint32_t tmem;
};

__global__ void __launch_bounds__(kThreads) k_bw_layer(Graph g, const __nv_bfloat16* __restrict__ Wm,
                                                       const __nv_bfloat16* __restrict__ Wu,
                                                       const float* __restrict__ bm, const float* __restrict__ bu,
                                                       const __nv_bfloat16* __restrict__ hl,
                                                       const __nv_bfloat16* __restrict__ agg,
                                                       const float* __restrict__ GH, float* GHprev, float* GSLOT,
                                                       float* GEPS, float* partials, int* error) {
  BwLayerSmem& S = *reinterpret_cast<BwLayerSmem*>(alignSmem(netSmem));
  TileCtx T;
  T.init(&S.bar, &S.tmem, 512, error);
  const int t = threadIdx.x;
  stageWeights(S.wu, Wu, 64, 128);
  stageWeights(S.wm, Wm, 64, 128);
  stageWeightsT(S.wut, Wu, 64, 128);
  stageWeightsT(S.wmt, Wm, 64, 128);
  if (t < 64) {
    S.bu[t] = bu[t];
    S.bm[t] = bm[t];
  }
  float dbu = 0.0f, dbm = 0.0f;
  bool first = true, good = true;
  constexpr uint32_t kU = 0, kGX = 64, kDWU = 192, kDWM = 256;
  for (uint32_t tile = blockIdx.x; tile < g.nTiles; tile += gridDim.x) {
    const TileRows tr = tileRows(g, tile);
    tileSlotInfo(g, tr, S.slotRow, S.rowFirst, true);
    const int R = static_cast<int>(tr.r1 - tr.r0);
    const int nq = static_cast<int>(tr.s1 - tr.s0);
    const bool acc = !first;
    // --- node part: u = W_u [h; a] + b_u, gu = GH (u > 0).
    {  // thread t: chunk c = t % 16 of rows t / 16 + 8 i, all loads in flight before the stores
      const int c = t % 16;
      uint4 v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int r = t / 16 + 8 * i;
        v[i] = zero4();
        if (r < R)
          v[i] = c < 8 ? reinterpret_cast<const uint4*>(hl + 64 * static_cast<size_t>(tr.r0 + r))[c]
                       : reinterpret_cast<const uint4*>(agg + 64 * static_cast<size_t>(tr.r0 + r))[c - 8];
      }
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        st16(S.x, t / 16 + 8 * i, c, 128, v[i]);
        st16T(S.xt, t / 16 + 8 * i, c, 128, v[i]);
      }
    }
    if (!(good = T.run([&] { umma::gemmIssue(T.tmem + kU, S.x, S.wu, 128, 64, 128, false); }))) break;
    {
      float gu[64];
      for (int c = 0; c < 4; ++c) {
        float v[16];
        T.load(kU + 16 * c, v);
        for (int k = 0; k < 16; ++k) {
          const int f = 16 * c + k;
          const float u = v[k] + S.bu[f];
          gu[f] = (t < R && u > 0.0f) ? GH[64 * static_cast<size_t>(tr.r0 + t) + f] : 0.0f;
        }
      }
      for (int c = 0; c < 8; ++c) {
        const uint4 p = packBf16(gu + 8 * c);
        st16(S.ga, t, c, 64, p);
        float rv[8];
        unpackBf16(p, rv);
        for (int k = 0; k < 8; ++k) {
          S.buf[t][8 * c + k] = rv[k];
          st1(S.gt, 8 * c + k, t, 128, reinterpret_cast<const __nv_bfloat16*>(&p)[k]);
        }
      }
    }
    __syncthreads();
    if (t < 64)
      for (int q = 0; q < R; ++q) dbu += S.buf[q][t];
    if (!(good = T.run([&] {
          umma::gemmIssue(T.tmem + kGX, S.ga, S.wut, 128, 128, 64, false);
          umma::gemmIssue(T.tmem + kDWU, S.xt, S.gt, 128, 64, 128, acc);
        })))
      break;
    // gh_prev = GH + gX[0:64]; ga = gX[64:128] -> buf.
    for (int c = 0; c < 8; ++c) {
      float v[16];
      T.load(kGX + 16 * c, v);
      if (t < R) {
        const size_t row = tr.r0 + t;
        if (c < 4) {
          for (int k = 0; k < 16; ++k) GHprev[64 * row + 16 * c + k] = GH[64 * row + 16 * c + k] + v[k];
        } else {
          for (int k = 0; k < 16; ++k) S.buf[t][16 * (c - 4) + k] = v[k];
        }
      }
    }
    __syncthreads();
    // --- message part: v = W_m [h_j; eps_s] + b_m, gv = (ga_i / 8) (v > 0).
    {  // thread t: chunk c = t % 16 of slots t / 16 + 8 i, all 16 gathers in flight before the stores
      const int c = t % 16;
      uint4 v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int q = t / 16 + 8 * i;
        v[i] = zero4();
        if (S.slotRow[q] >= 0) {
          const uint32_t s = tr.s0 + q;
          v[i] = c < 8 ? reinterpret_cast<const uint4*>(hl + 64 * static_cast<size_t>(colOf(g, s)))[c]
                       : reinterpret_cast<const uint4*>(g.eps + 64 * static_cast<size_t>(s))[c - 8];
        }
      }
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        st16(S.x, t / 16 + 8 * i, c, 128, v[i]);
        st16T(S.xt, t / 16 + 8 * i, c, 128, v[i]);
      }
    }
    if (!(good = T.run([&] { umma::gemmIssue(T.tmem + kU, S.x, S.wm, 128, 64, 128, false); }))) break;
    float gv[64];
    {
      const int sr = S.slotRow[t];
      for (int c = 0; c < 4; ++c) {
        float v[16];
        T.load(kU + 16 * c, v);
        for (int k = 0; k < 16; ++k) {
          const int f = 16 * c + k;
          const float pre = v[k] + S.bm[f];
          gv[f] = (sr >= 0 && pre > 0.0f) ? S.buf[sr][f] * kAggScale : 0.0f;
        }
      }
    }
    __syncthreads();  // buf (ga) fully read
    for (int c = 0; c < 8; ++c) {
      const uint4 p = packBf16(gv + 8 * c);
      st16(S.ga, t, c, 64, p);
      float rv[8];
      unpackBf16(p, rv);
      for (int k = 0; k < 8; ++k) {
        S.buf[t][8 * c + k] = rv[k];
        st1(S.gt, 8 * c + k, t, 128, reinterpret_cast<const __nv_bfloat16*>(&p)[k]);
      }
    }
    __syncthreads();
    if (t < 64)
      for (int q = 0; q < nq; ++q) dbm += S.buf[q][t];
    if (!(good = T.run([&] {
          umma::gemmIssue(T.tmem + kGX, S.ga, S.wmt, 128, 128, 64, false);
          umma::gemmIssue(T.tmem + kDWM, S.xt, S.gt, 128, 64, 128, acc);
        })))
      break;
    first = false;
    for (int c = 0; c < 8; ++c) {
      float v[16];
      T.load(kGX + 16 * c, v);
      if (t < nq) {
        const size_t s = tr.s0 + t;
        if (c < 4) {
          float4* d = reinterpret_cast<float4*>(GSLOT + 64 * s + 16 * c);
          for (int k = 0; k < 4; ++k) d[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
        } else if (S.slotRow[t] >= 0) {
          float* d = GEPS + 64 * s + 16 * (c - 4);
          for (int k = 0; k < 16; ++k) d[k] += v[k];
        }
      }
    }
    umma::fenceBeforeSync();
    __syncthreads();
  }
  // Partials in the layer's parameter order: W_m, b_m, W_u, b_u.
  constexpr size_t W = kHidden * 2 * kHidden;
  float* P = partials + static_cast<size_t>(blockIdx.x) * Layout::kLayerSize;
  if (good && !first) {
    for (int c = 0; c < 4; ++c) {
      float vm[16], vu[16];
      T.load(kDWM + 16 * c, vm);
      T.load(kDWU + 16 * c, vu);
      for (int k = 0; k < 16; ++k) {
        P[(16 * c + k) * 128 + t] = vm[k];
        P[W + kHidden + (16 * c + k) * 128 + t] = vu[k];
      }
    }
  } else {
    for (size_t k = t; k < Layout::kLayerSize; k += kThreads) P[k] = 0.0f;
  }
  __syncthreads();
  if (t < 64) {
    P[W + t] = dbm;
    P[2 * W + kHidden + t] = dbu;
  }
  T.done();
}

// ------------------------------------------------------------------------------------------------------------------
// Backward of an encoder: q = X W^T + b, gq = G (q > 0); dW^T += X^T gq (X has 16 features, padded to 128 rows).

struct BwEncSmem {
  unsigned char x[128 * 16 * 2];
  unsigned char w[64 * 16 * 2];
  unsigned char xt[128 * 128 * 2];
  unsigned char gt[64 * 128 * 2];
  float buf[128][65];
  float b[64];
  uint64_t bar;
  uint32_t tmem;
};

__global__ void __launch_bounds__(kThreads) k_bw_encode(uint32_t rows, const __nv_bfloat16* __restrict__ X,
                                                        const __nv_bfloat16* __restrict__ W,
                                                        const float* __restrict__ b, const float* __restrict__ G,
                                                        float* partials, int* error) {
  BwEncSmem& S = *reinterpret_cast<BwEncSmem*>(alignSmem(netSmem));
  TileCtx T;
  T.init(&S.bar, &S.tmem, 128, error);
  const int t = threadIdx.x;
  for (int k = t; k < 64 * 2; k += kThreads) st16(S.w, k / 2, k % 2, 16, reinterpret_cast<const uint4*>(W)[k]);
  for (int k = t; k < 112 * 128; k += kThreads) st1(S.xt, 16 + k / 128, k % 128, 128, __float2bfloat16_rn(0.0f));
  if (t < 64) S.b[t] = b[t];
  float db = 0.0f;
  bool first = true, good = true;
  const uint32_t tiles = (rows + 127) / 128;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const uint32_t r0 = tile * 128;
    for (int k = t; k < 128 * 2; k += kThreads) {
      const uint32_t q = k / 2, c = k % 2, r = r0 + q;
      const uint4 v = r < rows ? reinterpret_cast<const uint4*>(X + 16 * static_cast<size_t>(r))[c] : zero4();
      st16(S.x, q, c, 16, v);
      st16T(S.xt, q, c, 128, v);
    }
    if (!(good = T.run([&] { umma::gemmIssue(T.tmem, S.x, S.w, 128, 64, 16, false); }))) break;
    const uint32_t r = r0 + t;
    for (int c = 0; c < 4; ++c) {
      float v[16];
      T.load(16 * c, v);
      float gq[16];
      for (int k = 0; k < 16; ++k) {
        const float q = v[k] + S.b[16 * c + k];
        gq[k] = (r < rows && q > 0.0f) ? G[64 * static_cast<size_t>(r) + 16 * c + k] : 0.0f;
      }
      const uint4 p0 = packBf16(gq), p1 = packBf16(gq + 8);
      float rv[16];
      unpackBf16(p0, rv);
      unpackBf16(p1, rv + 8);
      for (int k = 0; k < 16; ++k) {
        S.buf[t][16 * c + k] = rv[k];
        st1(S.gt, 16 * c + k, t, 128, __float2bfloat16_rn(rv[k]));
      }
    }
    __syncthreads();
    if (t < 64)
      for (int q = 0; q < 128; ++q) db += S.buf[q][t];
    const bool acc = !first;
    if (!(good = T.run([&] { umma::gemmIssue(T.tmem + 64, S.xt, S.gt, 128, 64, 128, acc); }))) break;
    first = false;
  }
  float* P = partials + static_cast<size_t>(blockIdx.x) * (64 * 16 + 64);
  if (good && !first) {
    for (int c = 0; c < 4; ++c) {
      float v[16];
      T.load(64 + 16 * c, v);
      if (t < 16)
        for (int k = 0; k < 16; ++k) P[(16 * c + k) * 16 + t] = v[k];
    }
  } else {
    for (int k = t; k < 64 * 16; k += kThreads) P[k] = 0.0f;
  }
  if (t < 64) P[64 * 16 + t] = db;
  T.done();
}

// Vector steps of the evaluation PCG (scaled system): y += a x, and partial dot products.
__global__ void k_axpy(uint32_t n, const double* coef, int index, float sign, const float4* x, float4* y) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float a = sign * static_cast<float>(coef[index]);
  const float4 u = x[i], v = y[i];
  y[i] = make_float4(v.x + a * u.x, v.y + a * u.y, v.z + a * u.z, 0.0f);
}
// p = z + beta p with beta = coef[0] / coef[1].
__global__ void k_xpby(uint32_t n, const double* coef, const float4* z, float4* p) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float b = static_cast<float>(coef[0] / coef[1]);
  const float4 u = z[i], v = p[i];
  p[i] = make_float4(u.x + b * v.x, u.y + b * v.y, u.z + b * v.z, 0.0f);
}
__global__ void k_dot(uint32_t n, const float4* x, const float4* y, double* partial) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < n) {
    const float4 a = x[i], b = y[i];
    v = static_cast<double>(a.x) * b.x + static_cast<double>(a.y) * b.y + static_cast<double>(a.z) * b.z;
  }
  blockSumD(v, partial + blockIdx.x);
}
// coef[dst] = coef[num] / coef[den].
__global__ void k_ratio(double* coef, int num, int den, int dst) { coef[dst] = coef[num] / coef[den]; }

// ------------------------------------------------------------------------------------------------------------------
// Gradient reduction and optimiser.

__global__ void k_reduce(const float* __restrict__ partials, int grid, uint32_t count, float* dst, float scale) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= count) return;
  float s = 0.0f;
  for (int c = 0; c < grid; ++c) s += partials[static_cast<size_t>(c) * count + p];
  dst[p] += scale * s;
}

__global__ void k_adam(float* master, float* grad, float* m, float* v, uint32_t count, float lr, float b1, float b2,
                       float eps, float c1, float c2, __nv_bfloat16* wb) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= count) return;
  const float gr = grad[p];
  const float mm = b1 * m[p] + (1.0f - b1) * gr;
  const float vv = b2 * v[p] + (1.0f - b2) * gr * gr;
  m[p] = mm;
  v[p] = vv;
  const float w = master[p] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  master[p] = w;
  wb[p] = __float2bfloat16_rn(w);
  grad[p] = 0.0f;
}

__global__ void k_to_bf16(const float* src, __nv_bfloat16* dst, uint32_t count) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < count) dst[p] = __float2bfloat16_rn(src[p]);
}

template <class T>
T* dalloc(size_t count) {
  T* p = nullptr;
  NCK(cudaMalloc(&p, sizeof(T) * std::max<size_t>(count, 1)));
  NCK(cudaMemset(p, 0, sizeof(T) * std::max<size_t>(count, 1)));
  // The zeroing is on the legacy default stream, unordered with the network's and the solver's non-blocking streams.
  NCK(cudaStreamSynchronize(nullptr));
  return p;
}

size_t smemFor(size_t bytes) { return bytes + 128; }
// k_slot_encode holds 256 TMEM columns: at most two of its blocks fit an SM's shared memory (3 x 91 KB > 228 KB), so a
// third never waits in tcgen05.alloc for a resident block's columns (the grid is also capped at two blocks per SM).
// Its tile needs 1024-byte alignment (the TMA swizzle), hence the extra 1 KB.
constexpr size_t kSlotEncodeSmem = sizeof(SlotEncSmem) + 1024 - 128;
static_assert(3 * (kSlotEncodeSmem + 128 + 1024) > 228 * 1024, "k_slot_encode: three blocks would share an SM's TMEM");

}  // namespace

// ------------------------------------------------------------------------------------------------------------------
// Host side.

std::vector<uint32_t> rowTiles(const std::vector<uint32_t>& rowStart) {
  std::vector<uint32_t> tiles{0};
  const uint32_t n = static_cast<uint32_t>(rowStart.size()) - 1;
  uint32_t first = 0;
  for (uint32_t r = 0; r < n; ++r) {
    if (rowStart[r + 1] - rowStart[first] > static_cast<uint32_t>(kTileSlots)) {
      tiles.push_back(r);
      first = r;
    }
    if (rowStart[r + 1] - rowStart[r] > static_cast<uint32_t>(kTileSlots))
      throw std::invalid_argument("a row has more than 128 slots");
  }
  tiles.push_back(n);
  return tiles;
}

std::vector<uint32_t> transposedSlots(const std::vector<uint32_t>& rowStart, const std::vector<uint32_t>& colIndex) {
  const uint32_t n = static_cast<uint32_t>(rowStart.size()) - 1;
  std::vector<uint32_t> t(colIndex.size());
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t s = rowStart[i]; s < rowStart[i + 1]; ++s) {
      const uint32_t j = colIndex[s] & ~kPinBit;
      const auto b = colIndex.begin() + rowStart[j], e = colIndex.begin() + rowStart[j + 1];
      auto it = std::lower_bound(b, e, i, [](uint32_t c, uint32_t v) { return (c & ~kPinBit) < v; });
      if (it == e || (*it & ~kPinBit) != i) throw std::invalid_argument("the block pattern is not symmetric");
      t[s] = static_cast<uint32_t>(it - colIndex.begin());
    }
  return t;
}

struct GraphStore {
  Graph g;
  std::vector<void*> owned;
  std::vector<float4> residuals;  // residualCount x n (host copies, staged on demand)
  uint32_t residualCount = 0;
  float4 *rhat = nullptr, *a = nullptr, *b = nullptr, *e = nullptr, *ge = nullptr, *gb = nullptr, *ga = nullptr;
  float *r = nullptr, *go = nullptr, *GH = nullptr, *GH2 = nullptr, *GSLOT = nullptr, *GEPS = nullptr;
  double* partial = nullptr;
  int partialCount = 0;
  uint32_t liveUnknowns = 0;  // 3 x unpinned rows
  bool inference = false;     // the inference workspace is allocated
  CUtensorMap maps[2];        // k_slot_encode's TMA store maps of E and F (inference)
  ~GraphStore() {
    for (void* p : owned) cudaFree(p);
  }
  template <class T>
  T* own(size_t count) {
    T* p = dalloc<T>(count);
    owned.push_back(p);
    return p;
  }
};

namespace {

// The driver's cuTensorMapEncodeTiled, looked up once through the runtime (the library links the static runtime only).
PFN_cuTensorMapEncodeTiled_v12000 tensorMapEncoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    NCK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p) throw std::runtime_error("cuda: cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

void allocInference(GraphStore& s, cudaStream_t st) {
  if (s.inference) return;
  Graph& g = s.g;
  g.code = s.own<uint32_t>(g.B);
  g.slotRow = s.own<uint32_t>(g.B);
  k_slot_rows<<<static_cast<int>((g.n + 255) / 256), 256, 0, st>>>(g);
  NCK(cudaGetLastError());
  g.E = s.own<__nv_bfloat16>(kLayers * 64 * static_cast<size_t>(g.B));
  g.F = s.own<float>(kOutputs * static_cast<size_t>(g.B));
  {
    // E: [layer][slot][64] BF16 as a 3-D tensor, boxes of 64 x 128 x 1 (one layer of one 128-slot tile), 128-byte
    // swizzle; F: [slot][16] FP32, boxes of 16 x 128, 64-byte swizzle. Every stride is a multiple of 16 bytes.
    auto encode = tensorMapEncoder();
    const cuuint64_t eDim[3] = {64, g.B, static_cast<cuuint64_t>(kLayers)};
    const cuuint64_t eStride[2] = {128, 128ull * g.B};
    const cuuint32_t eBox[3] = {64, 128, 1}, one[3] = {1, 1, 1};
    if (encode(&s.maps[0], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, g.E, eDim, eStride, eBox, one,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      throw std::runtime_error("cuda: cuTensorMapEncodeTiled failed for the slot terms");
    const cuuint64_t fDim[2] = {static_cast<cuuint64_t>(kOutputs), g.B};
    const cuuint64_t fStride[1] = {64};
    const cuuint32_t fBox[2] = {static_cast<cuuint32_t>(kOutputs), 128};
    if (encode(&s.maps[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, g.F, fDim, fStride, fBox, one,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      throw std::runtime_error("cuda: cuTensorMapEncodeTiled failed for the output terms");
    g.tmaps = s.maps;
  }
  g.P = s.own<__nv_bfloat16>(64 * static_cast<size_t>(g.n));
  g.Q = s.own<float>(32 * static_cast<size_t>(g.n));
  g.a = s.own<__nv_bfloat16>(64 * static_cast<size_t>(g.n));
  s.inference = true;
}

// training: every activation the backward pass reads (a training sample); otherwise the inference path's buffers
// (a solver's bound graph).
void allocWorkspace(GraphStore& s, bool training, cudaStream_t st) {
  Graph& g = s.g;
  g.C = s.own<float>(9 * static_cast<size_t>(g.n));
  g.f = s.own<__nv_bfloat16>(16 * static_cast<size_t>(g.n));
  g.e = s.own<__nv_bfloat16>(16 * static_cast<size_t>(g.B));
  const int hs = training ? kLayers + 1 : 2;
  for (int l = 0; l < hs; ++l) g.h[l] = s.own<__nv_bfloat16>(64 * static_cast<size_t>(g.n));
  g.L = s.own<float>(9 * static_cast<size_t>(g.SP));
  if (!training) allocInference(s, st);
  if (training) {
    g.Ahat = s.own<float>(9 * static_cast<size_t>(g.B));
    g.eps = s.own<__nv_bfloat16>(64 * static_cast<size_t>(g.B));
    for (int l = 0; l < kLayers; ++l) g.agg[l] = s.own<__nv_bfloat16>(64 * static_cast<size_t>(g.n));
    g.G = s.own<float>(9 * static_cast<size_t>(g.B));
    g.o = s.own<float>(16 * static_cast<size_t>(g.B));
    for (float4** v : {&s.rhat, &s.a, &s.b, &s.e, &s.ge, &s.gb, &s.ga}) *v = s.own<float4>(g.n);
    s.r = s.own<float>(3 * static_cast<size_t>(g.n));
    s.go = s.own<float>(16 * static_cast<size_t>(g.B));
    s.GH = s.own<float>(64 * static_cast<size_t>(g.n));
    s.GH2 = s.own<float>(64 * static_cast<size_t>(g.n));
    s.GSLOT = s.own<float>(64 * static_cast<size_t>(g.B));
    s.GEPS = s.own<float>(64 * static_cast<size_t>(g.B));
    s.partialCount = static_cast<int>((g.n + 255) / 256);
    s.partial = s.own<double>(s.partialCount + 4);
  }
}

int gridFor(uint32_t work, int cap) { return static_cast<int>(std::max<uint32_t>(1, std::min<uint32_t>(work, cap))); }

}  // namespace

Network::Network(int device) : device_(device) {
  NCK(cudaSetDevice(device));
  cudaDeviceProp prop{};
  NCK(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) throw std::runtime_error("cuda: the learned preconditioner needs an sm_100 device");
  numSMs_ = prop.multiProcessorCount;
  NCK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  master_ = dalloc<float>(Layout::kCount);
  wBf16_ = dalloc<__nv_bfloat16>(Layout::kCount);
  grad_ = dalloc<float>(Layout::kCount);
  adamM_ = dalloc<float>(Layout::kCount);
  adamV_ = dalloc<float>(Layout::kCount);
  partialsCount_ = static_cast<size_t>(numSMs_) * Layout::kLayerSize;
  partials_ = dalloc<float>(partialsCount_);
  error_ = dalloc<int>(1);
  scalars_ = dalloc<double>(8);
  const struct {
    const void* fn;
    size_t bytes;
  } kernels[] = {{reinterpret_cast<const void*>(k_encode), sizeof(EncodeSmem)},
                 {reinterpret_cast<const void*>(k_layer), sizeof(LayerSmem)},
                 {reinterpret_cast<const void*>(k_output), sizeof(OutputSmem)},
                 {reinterpret_cast<const void*>(k_bw_output), sizeof(BwOutSmem)},
                 {reinterpret_cast<const void*>(k_bw_layer), sizeof(BwLayerSmem)},
                 {reinterpret_cast<const void*>(k_bw_encode), sizeof(BwEncSmem)},
                 {reinterpret_cast<const void*>(k_slot_encode), kSlotEncodeSmem},
                 {reinterpret_cast<const void*>(k_node<16, 64>), sizeof(NodeSmem)},
                 {reinterpret_cast<const void*>(k_node<128, 64>), sizeof(NodeSmem)},
                 {reinterpret_cast<const void*>(k_node<128, 32>), sizeof(NodeSmem)}};
  for (const auto& k : kernels)
    NCK(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smemFor(k.bytes))));
}

Network::~Network() {
  samples_.clear();
  for (void* p : std::initializer_list<void*>{master_, wBf16_, grad_, adamM_, adamV_, partials_, error_, scalars_})
    if (p) cudaFree(p);
  if (stream_) cudaStreamDestroy(stream_);
}

void Network::setParams(const float* p, size_t count) {
  if (count != Layout::kCount) throw std::invalid_argument("expected " + std::to_string(Layout::kCount) + " parameters");
  NCK(cudaMemcpyAsync(master_, p, sizeof(float) * count, cudaMemcpyHostToDevice, stream_));
  k_to_bf16<<<(count + 255) / 256, 256, 0, stream_>>>(master_, wBf16_, static_cast<uint32_t>(count));
  NCK(cudaGetLastError());
  NCK(cudaMemsetAsync(adamM_, 0, sizeof(float) * count, stream_));
  NCK(cudaMemsetAsync(adamV_, 0, sizeof(float) * count, stream_));
  NCK(cudaMemsetAsync(grad_, 0, sizeof(float) * count, stream_));
  adamStep_ = 0;
  NCK(cudaStreamSynchronize(stream_));
}

void Network::getParams(float* p, size_t count) {
  if (count != Layout::kCount) throw std::invalid_argument("expected " + std::to_string(Layout::kCount) + " parameters");
  NCK(cudaMemcpyAsync(p, master_, sizeof(float) * count, cudaMemcpyDeviceToHost, stream_));
  NCK(cudaStreamSynchronize(stream_));
}

int Network::addSample(uint32_t n, const uint32_t* rowStart, const uint32_t* colIndex, const float* blocks,
                       const uint8_t* pinned, const uint8_t* active, const float* residuals, uint32_t residualCount) {
  if (!rowStart || !colIndex || !blocks || !pinned || !active || (residualCount && !residuals))
    throw std::invalid_argument("null argument");
  auto s = std::make_unique<GraphStore>();
  std::vector<uint32_t> rs(rowStart, rowStart + n + 1);
  const uint32_t B = rs[n];
  std::vector<uint32_t> ci(colIndex, colIndex + B);
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t k = rs[i]; k < rs[i + 1]; ++k) {
      if (ci[k] >= n) throw std::invalid_argument("column index out of range");
      if (k > rs[i] && ci[k] <= ci[k - 1]) throw std::invalid_argument("columns must increase along a row");
    }
  const auto tiles = rowTiles(rs);
  const auto ts = transposedSlots(rs, ci);
  Graph& g = s->g;
  g.n = n;
  g.B = B;
  g.SP = (B + 31u) & ~31u;
  g.nTiles = static_cast<uint32_t>(tiles.size() - 1);
  auto upload = [&](auto* dst, const auto* src, size_t count) {
    NCK(cudaMemcpyAsync(dst, src, sizeof(*src) * count, cudaMemcpyHostToDevice, stream_));
  };
  uint32_t* drs = s->own<uint32_t>(n + 1);
  uint32_t* dci = s->own<uint32_t>(B);
  uint32_t* dts = s->own<uint32_t>(B);
  uint32_t* dtiles = s->own<uint32_t>(tiles.size());
  float* dbl = s->own<float>(9 * static_cast<size_t>(g.SP));
  uint8_t* dpin = s->own<uint8_t>(n);
  uint8_t* dact = s->own<uint8_t>(n);
  std::vector<float> planes(9 * static_cast<size_t>(g.SP), 0.0f);
  for (size_t k = 0; k < B; ++k)
    for (int c = 0; c < 9; ++c) planes[c * g.SP + k] = blocks[9 * k + c];
  upload(drs, rs.data(), rs.size());
  upload(dci, ci.data(), ci.size());
  upload(dts, ts.data(), ts.size());
  upload(dtiles, tiles.data(), tiles.size());
  upload(dbl, planes.data(), planes.size());
  upload(dpin, pinned, n);
  upload(dact, active, n);
  g.rowStart = drs;
  g.colIndex = dci;
  g.tslot = dts;
  g.tileRow = dtiles;
  g.blocks = dbl;
  g.pinnedBase = dpin;
  g.activeBase = dact;
  allocWorkspace(*s, true, stream_);
  s->residualCount = residualCount;
  for (uint32_t i = 0; i < n; ++i) s->liveUnknowns += pinned[i] ? 0u : 3u;
  s->residuals.resize(static_cast<size_t>(residualCount) * n);
  for (size_t k = 0; k < static_cast<size_t>(residualCount) * n; ++k)
    s->residuals[k] = make_float4(residuals[3 * k], residuals[3 * k + 1], residuals[3 * k + 2], 0.0f);
  NCK(cudaStreamSynchronize(stream_));
  samples_.push_back(std::move(s));
  return static_cast<int>(samples_.size()) - 1;
}

void Network::clearSamples() { samples_.clear(); }
int Network::sampleCount() const { return static_cast<int>(samples_.size()); }

Graph& Network::graphOf(GraphStore& s) { return s.g; }

void GraphStoreDeleter::operator()(GraphStore* s) const { delete s; }

GraphHandle Network::bind(uint32_t n, uint32_t B, uint32_t SP, const uint32_t* hostRowStart,
                                          const uint32_t* hostColIndex, const uint32_t* dRowStart,
                                          const uint32_t* dColIndex, const float* dBlocks,
                                          const uint8_t* pinnedBase, uint32_t pinnedStride,
                                          const uint8_t* activeBase, uint32_t activeStride, cudaStream_t st,
                                          bool factorRows) {
  auto s = std::make_unique<GraphStore>();
  std::vector<uint32_t> rs(hostRowStart, hostRowStart + n + 1), ci(hostColIndex, hostColIndex + B);
  const auto tiles = rowTiles(rs);
  const auto ts = transposedSlots(rs, ci);
  Graph& g = s->g;
  g.n = n;
  g.B = B;
  g.SP = SP;
  g.nTiles = static_cast<uint32_t>(tiles.size() - 1);
  uint32_t* dts = s->own<uint32_t>(B);
  uint32_t* dtiles = s->own<uint32_t>(tiles.size());
  NCK(cudaMemcpyAsync(dts, ts.data(), sizeof(uint32_t) * B, cudaMemcpyHostToDevice, st));
  NCK(cudaMemcpyAsync(dtiles, tiles.data(), sizeof(uint32_t) * tiles.size(), cudaMemcpyHostToDevice, st));
  g.rowStart = dRowStart;
  g.colIndex = dColIndex;
  g.tslot = dts;
  g.tileRow = dtiles;
  g.blocks = dBlocks;
  g.pinnedBase = pinnedBase;
  g.pinnedStride = pinnedStride;
  g.activeBase = activeBase;
  g.activeStride = activeStride;
  allocWorkspace(*s, false, st);
  if (factorRows) g.LF = s->own<float4>(3 * static_cast<size_t>(SP));
  NCK(cudaStreamSynchronize(st));
  return GraphHandle(s.release());
}

void Network::forwardOn(Graph& g, cudaStream_t st, bool training, int* error) {
  int* error_ = error ? error : this->error_;
  const int rowBlocks = static_cast<int>((g.n + 127) / 128);
  k_scale<<<rowBlocks, 128, 0, st>>>(g);
  k_features<<<static_cast<int>((g.n + 15) / 16), 256, 0, st>>>(g);
  const int cap = 2 * numSMs_;
  const __nv_bfloat16* W = wBf16_;
  const float* M = master_;
  if (!training) {
    if (!g.E) throw std::logic_error("forwardOn: the graph has no inference workspace");
    const int rowGroups = static_cast<int>((g.n + 31) / 32);  // eight lanes a row
    const int nodeGrid = gridFor((g.n + 255) / 256, 2 * numSMs_);  // two row tiles a block
    const size_t nodeSmem = smemFor(sizeof(NodeSmem));
    const CUtensorMap* maps = static_cast<const CUtensorMap*>(g.tmaps);
    k_slot_encode<<<gridFor((g.B + 127) / 128, 2 * numSMs_), kThreads, smemFor(kSlotEncodeSmem), st>>>(
        g, maps[0], maps[1], W, M, error_);
    k_node<16, 64><<<nodeGrid, kNodeThreads, nodeSmem, st>>>(g.n, g.f, nullptr, W + Layout::kNe, M + Layout::kNeB,
                                                         W + Layout::m(0), 2 * kHidden, 0, 0, g.h[0], g.P, error_);
    for (int l = 0; l < kLayers; ++l) {
      k_message<<<rowGroups, 256, 0, st>>>(g, g.P, g.E + l * 64 * static_cast<size_t>(g.B), g.a);
      const __nv_bfloat16* hin = g.h[l & 1];
      __nv_bfloat16* hout = g.h[(l + 1) & 1];
      if (l + 1 < kLayers)
        k_node<128, 64><<<nodeGrid, kNodeThreads, nodeSmem, st>>>(g.n, hin, g.a, W + Layout::u(l), M + Layout::uB(l),
                                                              W + Layout::m(l + 1), 2 * kHidden, 0, 0, hout, g.P,
                                                              error_);
      else
        k_node<128, 32><<<nodeGrid, kNodeThreads, nodeSmem, st>>>(g.n, hin, g.a, W + Layout::u(l), M + Layout::uB(l),
                                                              W + Layout::kO, 3 * kHidden, 0, kHidden, hout, g.Q,
                                                              error_);
    }
    k_output_slots<<<static_cast<int>((g.B + 255) / 256), 256, 0, st>>>(g, g.Q);
    NCK(cudaGetLastError());
    return;
  }
  k_encode<<<gridFor((g.n + 127) / 128, 4 * numSMs_), kThreads, smemFor(sizeof(EncodeSmem)), st>>>(
      g.n, g.f, W + Layout::kNe, M + Layout::kNeB, g.h[0], error_);
  k_encode<<<gridFor((g.B + 127) / 128, 4 * numSMs_), kThreads, smemFor(sizeof(EncodeSmem)), st>>>(
      g.B, g.e, W + Layout::kEe, M + Layout::kEeB, g.eps, error_);
  for (int l = 0; l < kLayers; ++l) {
    const __nv_bfloat16* hin = training ? g.h[l] : g.h[l & 1];
    __nv_bfloat16* hout = training ? g.h[l + 1] : g.h[(l + 1) & 1];
    k_layer<<<gridFor(g.nTiles, cap), kThreads, smemFor(sizeof(LayerSmem)), st>>>(
        g, W + Layout::m(l), W + Layout::u(l), M + Layout::mB(l), M + Layout::uB(l), hin, hout,
        training ? g.agg[l] : nullptr, error_);
  }
  // k_output's 57 KB of shared memory fit three blocks on an SM (k_layer's 100 KB fit two: `cap`).
  k_output<<<gridFor(g.nTiles, 3 * numSMs_), kThreads, smemFor(sizeof(OutputSmem)), st>>>(
      g, W + Layout::kO, M + Layout::kOB, training ? g.h[kLayers] : g.h[kLayers & 1], training ? 1 : 0, error_);
  NCK(cudaGetLastError());
}

void Network::lossForward(GraphStore& s, int residual) {
  Graph& g = s.g;
  const int nb = static_cast<int>((g.n + 255) / 256);
  if (objective_ == 1) {
    std::vector<float4> w(s.residuals.begin() + static_cast<size_t>(residual) * g.n,
                          s.residuals.begin() + static_cast<size_t>(residual + 1) * g.n);
    NCK(cudaMemcpyAsync(s.rhat, w.data(), sizeof(float4) * g.n, cudaMemcpyHostToDevice, stream_));
    k_lower<<<nb, 256, 0, stream_>>>(g, g.G, s.rhat, s.b);
    k_ahat_dot<<<nb, 256, 0, stream_>>>(g, s.b, s.e, s.partial);
    k_sum<<<1, 256, 0, stream_>>>(s.partial, nb, scalars_ + 0);
    k_logdet<<<nb, 256, 0, stream_>>>(g, s.partial);
    k_sum<<<1, 256, 0, stream_>>>(s.partial, nb, scalars_ + 1);
    NCK(cudaStreamSynchronize(stream_));  // w must outlive the copy
    return;
  }
  std::vector<float> r(3 * static_cast<size_t>(g.n));
  for (uint32_t i = 0; i < g.n; ++i) {
    const float4 v = s.residuals[static_cast<size_t>(residual) * g.n + i];
    r[3 * i] = v.x;
    r[3 * i + 1] = v.y;
    r[3 * i + 2] = v.z;
  }
  NCK(cudaMemcpyAsync(s.r, r.data(), sizeof(float) * r.size(), cudaMemcpyHostToDevice, stream_));
  k_rhat<<<nb, 256, 0, stream_>>>(g, s.r, s.rhat, s.partial);
  k_sum<<<1, 256, 0, stream_>>>(s.partial, nb, scalars_ + 0);
  k_lower_t<<<nb, 256, 0, stream_>>>(g, g.G, s.rhat, s.a);
  k_lower<<<nb, 256, 0, stream_>>>(g, g.G, s.a, s.b);
  k_ahat<<<nb, 256, 0, stream_>>>(g, s.b, s.rhat, s.e, s.partial);
  k_sum<<<1, 256, 0, stream_>>>(s.partial, nb, scalars_ + 1);
  NCK(cudaStreamSynchronize(stream_));  // the host vector r must outlive the copy
}

void Network::reduceInto(const float* partials, int grid, size_t count, size_t offset, float scale) {
  k_reduce<<<static_cast<int>((count + 255) / 256), 256, 0, stream_>>>(partials, grid, static_cast<uint32_t>(count),
                                                                      grad_ + offset, scale);
  NCK(cudaGetLastError());
}

void Network::backward(GraphStore& s) {
  Graph& g = s.g;
  const int nb = static_cast<int>((g.n + 255) / 256);
  const int wb = static_cast<int>((g.n + 7) / 8);
  if (objective_ == 1) {
    k_grad_o_kaporin<<<wb, 256, 0, stream_>>>(g, s.e, s.rhat, scalars_, 1.0f / std::max(1u, s.liveUnknowns), s.go);
  } else {
    k_ge<<<nb, 256, 0, stream_>>>(g.n, s.e, scalars_, s.ge);
    k_ahat<<<nb, 256, 0, stream_>>>(g, s.ge, nullptr, s.gb, s.partial);
    k_lower_t<<<nb, 256, 0, stream_>>>(g, g.G, s.gb, s.ga);
    k_grad_o<<<wb, 256, 0, stream_>>>(g, s.gb, s.a, s.rhat, s.ga, s.go);
  }
  const __nv_bfloat16* W = wBf16_;
  const float* M = master_;
  const int grid = gridFor(g.nTiles, numSMs_);
  k_bw_output<<<grid, kThreads, smemFor(sizeof(BwOutSmem)), stream_>>>(g, W + Layout::kO, g.h[kLayers], s.go, s.GH,
                                                                         s.GSLOT, s.GEPS, partials_, error_);
  reduceInto(partials_, grid, Layout::kOB - Layout::kO + kOutputs, Layout::kO, 1.0f);
  k_gather<<<wb, 256, 0, stream_>>>(g, s.GSLOT, s.GH, 0);
  float* gh = s.GH;
  float* ghPrev = s.GH2;
  for (int l = kLayers - 1; l >= 0; --l) {
    k_bw_layer<<<grid, kThreads, smemFor(sizeof(BwLayerSmem)), stream_>>>(
        g, W + Layout::m(l), W + Layout::u(l), M + Layout::mB(l), M + Layout::uB(l), g.h[l], g.agg[l], gh, ghPrev,
        s.GSLOT, s.GEPS, partials_, error_);
    reduceInto(partials_, grid, Layout::kLayerSize, Layout::m(l), 1.0f);
    k_gather<<<wb, 256, 0, stream_>>>(g, s.GSLOT, ghPrev, 1);
    std::swap(gh, ghPrev);
  }
  const int encGridE = gridFor((g.B + 127) / 128, numSMs_);
  k_bw_encode<<<encGridE, kThreads, smemFor(sizeof(BwEncSmem)), stream_>>>(g.B, g.e, W + Layout::kEe,
                                                                            M + Layout::kEeB, s.GEPS, partials_,
                                                                            error_);
  reduceInto(partials_, encGridE, 64 * 16 + 64, Layout::kEe, 1.0f);
  const int encGridN = gridFor((g.n + 127) / 128, numSMs_);
  k_bw_encode<<<encGridN, kThreads, smemFor(sizeof(BwEncSmem)), stream_>>>(g.n, g.f, W + Layout::kNe,
                                                                            M + Layout::kNeB, gh, partials_, error_);
  reduceInto(partials_, encGridN, 64 * 16 + 64, Layout::kNe, 1.0f);
  NCK(cudaGetLastError());
}

namespace {
void checkError(int* err, cudaStream_t st) {
  int h = 0;
  NCK(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  NCK(cudaStreamSynchronize(st));
  if (h) {
    NCK(cudaMemsetAsync(err, 0, sizeof(int), st));
    throw std::runtime_error("cuda: a tensor-core wait in the network kernels timed out");
  }
}
}  // namespace

void Network::forward(int sample, float* Gout, float* Lout) {
  if (sample < 0 || sample >= sampleCount()) throw std::out_of_range("no such sample");
  GraphStore& s = *samples_[sample];
  forwardOn(s.g, stream_, true);
  checkError(error_, stream_);
  const Graph& g = s.g;
  if (Gout) NCK(cudaMemcpyAsync(Gout, g.G, sizeof(float) * 9 * g.B, cudaMemcpyDeviceToHost, stream_));
  if (Lout) {
    std::vector<float> planes(9 * static_cast<size_t>(g.SP));
    NCK(cudaMemcpyAsync(planes.data(), g.L, sizeof(float) * planes.size(), cudaMemcpyDeviceToHost, stream_));
    NCK(cudaStreamSynchronize(stream_));
    for (uint32_t k = 0; k < g.B; ++k)
      for (int c = 0; c < 9; ++c) Lout[9 * static_cast<size_t>(k) + c] = planes[c * g.SP + k];
  }
  NCK(cudaStreamSynchronize(stream_));
}

void Network::forwardInference(int sample, float* Lout) {
  if (sample < 0 || sample >= sampleCount()) throw std::out_of_range("no such sample");
  GraphStore& s = *samples_[sample];
  allocInference(s, stream_);
  forwardOn(s.g, stream_, false);
  checkError(error_, stream_);
  const Graph& g = s.g;
  if (Lout) {
    std::vector<float> planes(9 * static_cast<size_t>(g.SP));
    NCK(cudaMemcpyAsync(planes.data(), g.L, sizeof(float) * planes.size(), cudaMemcpyDeviceToHost, stream_));
    NCK(cudaStreamSynchronize(stream_));
    for (uint32_t k = 0; k < g.B; ++k)
      for (int c = 0; c < 9; ++c) Lout[9 * static_cast<size_t>(k) + c] = planes[c * g.SP + k];
  }
  NCK(cudaStreamSynchronize(stream_));
}

double Network::lossValue(const GraphStore& s, const double* sc) const {
  if (objective_ == 1) {
    const double N = std::max(1u, s.liveUnknowns);
    return std::log(sc[0] / N) - 2.0 * sc[1] / N;
  }
  return sc[0] > 0.0 ? sc[1] / sc[0] : 0.0;
}

double Network::lossGrad(int sample, int residual, float* grad, bool accumulate) {
  if (sample < 0 || sample >= sampleCount()) throw std::out_of_range("no such sample");
  GraphStore& s = *samples_[sample];
  if (residual < 0 || residual >= static_cast<int>(s.residualCount)) throw std::out_of_range("no such residual");
  if (!accumulate) NCK(cudaMemsetAsync(grad_, 0, sizeof(float) * Layout::kCount, stream_));
  forwardOn(s.g, stream_, true);
  lossForward(s, residual);
  backward(s);
  double sc[2] = {0, 0};
  NCK(cudaMemcpyAsync(sc, scalars_, sizeof(sc), cudaMemcpyDeviceToHost, stream_));
  if (grad) NCK(cudaMemcpyAsync(grad, grad_, sizeof(float) * Layout::kCount, cudaMemcpyDeviceToHost, stream_));
  checkError(error_, stream_);
  return lossValue(s, sc);
}

void Network::apply(int sample, const float* r, float* z) {
  if (sample < 0 || sample >= sampleCount()) throw std::out_of_range("no such sample");
  GraphStore& s = *samples_[sample];
  Graph& g = s.g;
  forwardOn(g, stream_, true);
  std::vector<float4> rv(g.n), zv(g.n);
  for (uint32_t i = 0; i < g.n; ++i) rv[i] = make_float4(r[3 * i], r[3 * i + 1], r[3 * i + 2], 0.0f);
  NCK(cudaMemcpyAsync(s.rhat, rv.data(), sizeof(float4) * g.n, cudaMemcpyHostToDevice, stream_));
  // L per slot (B x 9) from the planes, through the AoS lower-slot kernels.
  const int nb = static_cast<int>((g.n + 255) / 256);
  std::vector<float> planes(9 * static_cast<size_t>(g.SP)), aos(9 * static_cast<size_t>(g.B));
  NCK(cudaMemcpyAsync(planes.data(), g.L, sizeof(float) * planes.size(), cudaMemcpyDeviceToHost, stream_));
  NCK(cudaStreamSynchronize(stream_));
  for (uint32_t k = 0; k < g.B; ++k)
    for (int c = 0; c < 9; ++c) aos[9 * static_cast<size_t>(k) + c] = planes[c * g.SP + k];
  NCK(cudaMemcpyAsync(s.go, aos.data(), sizeof(float) * aos.size(), cudaMemcpyHostToDevice, stream_));
  k_lower_t<<<nb, 256, 0, stream_>>>(g, s.go, s.rhat, s.a);
  k_lower<<<nb, 256, 0, stream_>>>(g, s.go, s.a, s.b);
  NCK(cudaMemcpyAsync(zv.data(), s.b, sizeof(float4) * g.n, cudaMemcpyDeviceToHost, stream_));
  checkError(error_, stream_);
  for (uint32_t i = 0; i < g.n; ++i) {
    z[3 * i] = zv[i].x;
    z[3 * i + 1] = zv[i].y;
    z[3 * i + 2] = zv[i].z;
  }
}

int Network::pcg(int sample, int rhs, bool useLearned, int maxIterations, double tolerance, double* relres) {
  if (sample < 0 || sample >= sampleCount()) throw std::out_of_range("no such sample");
  GraphStore& s = *samples_[sample];
  if (rhs < 0 || rhs >= static_cast<int>(s.residualCount)) throw std::out_of_range("no such residual");
  Graph& g = s.g;
  forwardOn(g, stream_, true);
  const uint32_t n = g.n;
  const int nb = static_cast<int>((n + 255) / 256);
  // Scaled system Ahat x = rhat (rhat = S^T r); the preconditioner is G G^T, or the identity (block-Jacobi).
  std::vector<float> r(3 * static_cast<size_t>(n));
  for (uint32_t i = 0; i < n; ++i) {
    const float4 v = s.residuals[static_cast<size_t>(rhs) * n + i];
    r[3 * i] = v.x;
    r[3 * i + 1] = v.y;
    r[3 * i + 2] = v.z;
  }
  NCK(cudaMemcpyAsync(s.r, r.data(), sizeof(float) * r.size(), cudaMemcpyHostToDevice, stream_));
  float4 *R = s.rhat, *Z = s.a, *P = s.b, *Q = s.e, *X = s.ge, *T = s.gb;
  double* coef = scalars_;  // 0 rz, 1 rz_old, 2 pq, 3 alpha, 4 rr, 5 rr0
  k_rhat<<<nb, 256, 0, stream_>>>(g, s.r, R, s.partial);
  k_sum<<<1, 256, 0, stream_>>>(s.partial, nb, coef + 5);
  NCK(cudaMemsetAsync(X, 0, sizeof(float4) * n, stream_));
  auto precondition = [&] {
    if (useLearned) {
      k_lower_t<<<nb, 256, 0, stream_>>>(g, g.G, R, T);
      k_lower<<<nb, 256, 0, stream_>>>(g, g.G, T, Z);
    } else {
      NCK(cudaMemcpyAsync(Z, R, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream_));
    }
    k_dot<<<nb, 256, 0, stream_>>>(n, R, Z, s.partial);
    k_sum<<<1, 256, 0, stream_>>>(s.partial, nb, coef + 0);
  };
  precondition();
  NCK(cudaMemcpyAsync(P, Z, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream_));
  double host[6] = {0, 0, 0, 0, 0, 0};
  int it = 0;
  for (; it < maxIterations;) {
    k_ahat_dot<<<nb, 256, 0, stream_>>>(g, P, Q, s.partial);
    k_sum<<<1, 256, 0, stream_>>>(s.partial, nb, coef + 2);
    k_ratio<<<1, 1, 0, stream_>>>(coef, 0, 2, 3);
    k_axpy<<<nb, 256, 0, stream_>>>(n, coef, 3, 1.0f, P, X);
    k_axpy<<<nb, 256, 0, stream_>>>(n, coef, 3, -1.0f, Q, R);
    ++it;
    k_dot<<<nb, 256, 0, stream_>>>(n, R, R, s.partial);
    k_sum<<<1, 256, 0, stream_>>>(s.partial, nb, coef + 4);
    NCK(cudaMemcpyAsync(host, coef, sizeof(host), cudaMemcpyDeviceToHost, stream_));
    NCK(cudaStreamSynchronize(stream_));
    if (!(host[2] > 0.0) || std::sqrt(host[4]) <= tolerance * std::sqrt(host[5])) break;
    NCK(cudaMemcpyAsync(coef + 1, coef + 0, sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    precondition();
    k_xpby<<<nb, 256, 0, stream_>>>(n, coef, Z, P);
  }
  NCK(cudaGetLastError());
  NCK(cudaMemcpyAsync(host, coef, sizeof(host), cudaMemcpyDeviceToHost, stream_));
  NCK(cudaStreamSynchronize(stream_));
  if (relres) *relres = host[5] > 0.0 ? std::sqrt(host[4] / host[5]) : 0.0;
  checkError(error_, stream_);
  return it;
}

void Network::train(int steps, float lr, int batch, uint64_t seed, float* losses) {
  if (samples_.empty()) throw std::invalid_argument("no training samples");
  if (steps < 0 || batch < 1) throw std::invalid_argument("steps must be >= 0 and batch >= 1");
  std::mt19937_64 rng(seed);
  std::vector<std::pair<int, int>> pairs;
  for (int s = 0; s < sampleCount(); ++s)
    for (uint32_t r = 0; r < samples_[s]->residualCount; ++r) pairs.emplace_back(s, static_cast<int>(r));
  if (pairs.empty()) throw std::invalid_argument("the samples carry no residuals");
  NCK(cudaMemsetAsync(grad_, 0, sizeof(float) * Layout::kCount, stream_));
  for (int step = 0; step < steps; ++step) {
    double sum = 0.0;
    for (int b = 0; b < batch; ++b) {
      const auto& pr = pairs[rng() % pairs.size()];
      GraphStore& s = *samples_[pr.first];
      forwardOn(s.g, stream_, true);
      lossForward(s, pr.second);
      backward(s);
      double sc[2] = {0, 0};
      NCK(cudaMemcpyAsync(sc, scalars_, sizeof(sc), cudaMemcpyDeviceToHost, stream_));
      NCK(cudaStreamSynchronize(stream_));
      sum += lossValue(s, sc);
    }
    ++adamStep_;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(adamStep_));
    const float c2 = 1.0f - std::pow(b2, static_cast<float>(adamStep_));
    // The gradient accumulates over the batch; Adam is invariant to its scale, so no division is needed.
    k_adam<<<static_cast<int>((Layout::kCount + 255) / 256), 256, 0, stream_>>>(
        master_, grad_, adamM_, adamV_, static_cast<uint32_t>(Layout::kCount), lr, b1, b2, 1e-8f * batch, c1, c2,
        wBf16_);
    NCK(cudaGetLastError());
    if (losses) losses[step] = static_cast<float>(sum / batch);
  }
  checkError(error_, stream_);
}

}  // namespace net

// ------------------------------------------------------------------------------------------------------------------
// C ABI (include/drape_precond.h).

#include "../../include/drape_precond.h"

namespace {
thread_local std::string g_netError;

template <class F>
int netGuarded(drape_precond* p, F&& f) {
  try {
    f();
    return DRAPE_OK;
  } catch (const std::invalid_argument& e) {
    (p ? p->error : g_netError) = e.what();
    return DRAPE_INVALID;
  } catch (const std::out_of_range& e) {
    (p ? p->error : g_netError) = e.what();
    return DRAPE_OUT_OF_RANGE;
  } catch (const std::exception& e) {
    (p ? p->error : g_netError) = e.what();
    return DRAPE_DEVICE_ERROR;
  }
}
void needNet(drape_precond* p) {
  if (!p || !p->net) throw std::invalid_argument("null preconditioner handle");
}
}  // namespace

extern "C" {

uint32_t drape_precond_param_count(void) { return static_cast<uint32_t>(net::Layout::kCount); }

int drape_precond_create(int device, drape_precond** out) {
  return netGuarded(nullptr, [&] {
    if (!out) throw std::invalid_argument("null argument");
    auto p = std::make_unique<drape_precond>();
    p->net = std::make_unique<net::Network>(device);
    *out = p.release();
  });
}

void drape_precond_destroy(drape_precond* p) { delete p; }

const char* drape_precond_last_error(drape_precond* p) { return p ? p->error.c_str() : g_netError.c_str(); }

int drape_precond_set_params(drape_precond* p, const float* params, size_t count) {
  return netGuarded(p, [&] {
    needNet(p);
    if (!params) throw std::invalid_argument("null argument");
    p->net->setParams(params, count);
  });
}

int drape_precond_get_params(drape_precond* p, float* params, size_t count) {
  return netGuarded(p, [&] {
    needNet(p);
    if (!params) throw std::invalid_argument("null argument");
    p->net->getParams(params, count);
  });
}

int drape_precond_add_sample(drape_precond* p, uint32_t n, const uint32_t* row_start, const uint32_t* col_index,
                             const float* blocks, const uint8_t* pinned, const uint8_t* active,
                             const float* residuals, uint32_t residual_count, int* sample) {
  return netGuarded(p, [&] {
    needNet(p);
    if (n == 0) throw std::invalid_argument("empty system");
    for (uint32_t i = 0; row_start && col_index && i < n; ++i) {
      bool diag = false;
      for (uint32_t k = row_start[i]; k < row_start[i + 1]; ++k) diag = diag || col_index[k] == i;
      if (!diag) throw std::invalid_argument("row " + std::to_string(i) + " has no diagonal block");
    }
    const int id = p->net->addSample(n, row_start, col_index, blocks, pinned, active, residuals, residual_count);
    if (sample) *sample = id;
  });
}

int drape_precond_clear_samples(drape_precond* p) {
  return netGuarded(p, [&] {
    needNet(p);
    p->net->clearSamples();
  });
}

int drape_precond_forward(drape_precond* p, int sample, float* g_blocks, float* l_blocks) {
  return netGuarded(p, [&] {
    needNet(p);
    p->net->forward(sample, g_blocks, l_blocks);
  });
}

int drape_precond_forward_inference(drape_precond* p, int sample, float* l_blocks) {
  return netGuarded(p, [&] {
    needNet(p);
    p->net->forwardInference(sample, l_blocks);
  });
}

int drape_precond_loss_grad(drape_precond* p, int sample, int residual, double* loss, float* grad) {
  return netGuarded(p, [&] {
    needNet(p);
    const double v = p->net->lossGrad(sample, residual, grad, false);
    if (loss) *loss = v;
  });
}

int drape_precond_apply(drape_precond* p, int sample, const float* r, float* z) {
  return netGuarded(p, [&] {
    needNet(p);
    if (!r || !z) throw std::invalid_argument("null argument");
    p->net->apply(sample, r, z);
  });
}

int drape_precond_pcg(drape_precond* p, int sample, int rhs, int use_learned, int max_iterations, double tolerance,
                      int* iterations, double* relative_residual) {
  return netGuarded(p, [&] {
    needNet(p);
    if (!iterations || max_iterations < 1) throw std::invalid_argument("bad argument");
    *iterations = p->net->pcg(sample, rhs, use_learned != 0, max_iterations, tolerance, relative_residual);
  });
}

int drape_precond_set_objective(drape_precond* p, int objective) {
  return netGuarded(p, [&] {
    needNet(p);
    if (objective != DRAPE_PRECOND_DEFECT && objective != DRAPE_PRECOND_KAPORIN)
      throw std::invalid_argument("unknown objective");
    p->net->setObjective(objective);
  });
}

int drape_precond_train(drape_precond* p, int steps, float learning_rate, int batch, uint64_t seed, float* losses) {
  return netGuarded(p, [&] {
    needNet(p);
    if (!(learning_rate > 0.0f)) throw std::invalid_argument("learning rate must be positive");
    p->net->train(steps, learning_rate, batch, seed, losses);
  });
}

}  // extern "C"
