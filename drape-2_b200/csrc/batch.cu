// Batched drapes (include/drape_batch.h): independent garments, each on its own body, advanced together.
//
// Storage: every garment's model (model.hpp, built from its own one-garment scene, so all its indices are local) is
// concatenated into one set of device arrays; a garment's segment view (dcu::Dev) points at its slices, so the
// kernels of kernels.cuh run on it unchanged. Launches:
//   - point kernels (substep begin, contact activation, finish) and the assembly kernel cover all garments in one
//     launch each: block b belongs to the garment whose block range holds b (a prefix array per kernel);
//   - the solve is one cooperative launch per Newton iteration: each garment that is still advancing gets a group of
//     co-resident blocks, sized by its share of the work (block slots + 5 x particles, the SpMV's byte ratio); the
//     group runs that garment's PCG, FP64 reductions, convergence test and line search (solveGroup) with its own
//     grid barrier counter and partials;
//   - a frame (H2D per-garment control, snapshot actions, substeps, statistics, D2H) is captured once as a CUDA graph
//     and replayed; it is re-captured only when the frame's substep count or the solve variant changes.
// Garments advance independently: a garment's frame control gives its substep length and count (0 = frozen), so
// a garment that doubled its substeps after a retry, or that has settled, does not change the others' arithmetic.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/drape_batch.h"
#include "device_buffer.hpp"
#include "device_model.hpp"
#include "kernels.cuh"
#include "learned.hpp"
#include "model.hpp"

using drape_b200::Model;
using dbuf::check;
using dbuf::DBuf;
using dbuf::HostPinned;
#define BCK(x) check((x), #x)

namespace bcu {

// Per-garment frame control, written by the host before every frame.
struct SegRun {
  float h, invH2;
  double hD;
  int32_t substeps;   // substeps of this frame; 0: the garment does not advance
  int32_t action;     // kActRestore | kActSettle | kActAssemble | kActSave, applied before the substeps
  uint32_t smemSlots; // block slots a solve block of this garment keeps in shared memory
  uint32_t pad;
};
constexpr int32_t kActRestore = 1, kActSettle = 2, kActAssemble = 4, kActSave = 8;

using dcu::StatsOut;

struct View {
  const dcu::Dev* segs;         // G segment views
  const SegRun* run;            // G
  const uint32_t* solveStart;   // G + 1: solve blocks of garment g are [solveStart[g], solveStart[g + 1])
  const uint32_t* pointStart;   // G + 1: point-kernel blocks
  const uint32_t* asmStart;     // G + 1: assembly blocks
  const uint32_t* pBase;        // G: first particle of garment g in the batch arrays
  const uint32_t* kBase;        // G: first seam
  double* partials;             // 2 * kPartialStride doubles per solve block
  dcu::Seam* seams;             // all seams (writable: start gaps)
  float4 *snapX, *snapV;        // per-garment drape-runner snapshot
  dcu::Contact* snapC;
  dcu::Garment* snapG;
  float* snapGap;
  StatsOut* stats;              // G
  uint32_t G;
};

// The largest g with start[g] <= b (blocks of garments with an empty range are skipped).
__device__ __forceinline__ uint32_t segmentOf(const uint32_t* start, uint32_t G, uint32_t b) {
  uint32_t lo = 0, hi = G - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (__ldg(start + mid) <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Garment g's segment view into shared memory, with this frame's substep length and solve sizes.
__device__ inline void loadSegment(const View& V, uint32_t g, dcu::Dev& sD) {
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(V.segs + g);
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sD);
  for (uint32_t k = threadIdx.x; k < sizeof(dcu::Dev) / 8; k += blockDim.x) dst[k] = src[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    const SegRun r = V.run[g];
    sD.P.h = r.h;
    sD.P.invH2 = r.invH2;
    sD.P.hD = r.hD;
    sD.P.smemSlots = r.smemSlots;
  }
  __syncthreads();
}

static_assert(sizeof(dcu::Dev) % 8 == 0, "segment views are copied in 8-byte words");

// Snapshot actions on particle data (restore before save; a frame never asks for both).
__global__ void k_actions_particles(View V) {
  __shared__ uint32_t g, rank, size;
  __shared__ int32_t act;
  if (threadIdx.x == 0) {
    g = segmentOf(V.pointStart, V.G, blockIdx.x);
    rank = blockIdx.x - V.pointStart[g];
    size = V.pointStart[g + 1] - V.pointStart[g];
    act = V.run[g].action;
  }
  __syncthreads();
  if ((act & (kActRestore | kActSave)) == 0) return;
  const dcu::Dev& D = V.segs[g];
  const uint32_t n = D.P.n, base = V.pBase[g];
  for (uint32_t i = rank * blockDim.x + threadIdx.x; i < n; i += size * blockDim.x) {
    if (act & kActRestore) {
      D.x[i] = V.snapX[base + i];
      D.v[i] = V.snapV[base + i];
      D.contact[i] = V.snapC[base + i];
    } else {
      V.snapX[base + i] = D.x[i];
      V.snapV[base + i] = D.v[i];
      V.snapC[base + i] = D.contact[i];
    }
  }
}

// Garment-level actions, one block per garment: restore the garment record and seam gaps, phase changes (entering
// Assembling resets the clock and measures the seam gaps from the current positions, as Model::setPhase), save.
__global__ void k_actions_garment(View V) {
  const uint32_t g = blockIdx.x;
  const int32_t act = V.run[g].action;
  if (act == 0) return;
  const dcu::Dev& D = V.segs[g];
  dcu::Seam* seams = V.seams + V.kBase[g];
  const uint32_t K = D.P.nSeam;
  if (act & kActRestore) {
    if (threadIdx.x == 0) *D.garment = V.snapG[g];
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) seams[k].startGap = V.snapGap[V.kBase[g] + k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (act & kActSettle) D.garment->phase = 1;
    if (act & kActAssemble) {
      D.garment->phase = 0;
      D.garment->assemblyTime = 0.0;
    }
  }
  if (act & kActAssemble)
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) {
      const float4 a = D.x[seams[k].a], b = D.x[seams[k].b];
      const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
      seams[k].startGap = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
    }
  __syncthreads();
  if (act & kActSave) {
    if (threadIdx.x == 0) V.snapG[g] = *D.garment;
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) V.snapGap[V.kBase[g] + k] = seams[k].startGap;
  }
}

// The point kernels: block b works on its garment's share; a garment that does not take substep s is skipped (its
// Newton loop is marked done so its activation, assembly and solve blocks return at once).
template <int Kind>
__global__ void k_points(View V, int substep) {
  __shared__ dcu::Dev sD;
  __shared__ uint32_t g, rank, size;
  __shared__ int live;
  if (threadIdx.x == 0) {
    g = segmentOf(V.pointStart, V.G, blockIdx.x);
    rank = blockIdx.x - V.pointStart[g];
    size = V.pointStart[g + 1] - V.pointStart[g];
    live = substep < V.run[g].substeps;
  }
  __syncthreads();
  if (!live) {
    if (Kind == 0 && rank == 0 && threadIdx.x == 0) V.segs[g].ctl->newtonDone = 1;
    return;
  }
  loadSegment(V, g, sD);
  if (Kind == 0) dcu::beginRows(sD, rank, size);
  if (Kind == 1) {
    // The solve's grid barrier counts from zero for the group that the next solve launch gives this garment.
    if (rank == 0 && threadIdx.x == 0 && !sD.ctl->newtonDone) sD.ctl->barrierArrivals = 0;
    dcu::activateRows(sD, rank, size);
  }
  if (Kind == 2) dcu::finishRows(sD, rank, size);
}

// Per-term derivative records of every advancing garment (dcu::termsRows), on the assembly partition.
__global__ void __launch_bounds__(dcu::kAssembleThreads) k_terms_batch(View V) {
  __shared__ dcu::Dev sD;
  __shared__ uint32_t g, rank, size;
  if (threadIdx.x == 0) {
    g = segmentOf(V.asmStart, V.G, blockIdx.x);
    rank = blockIdx.x - V.asmStart[g];
    size = V.asmStart[g + 1] - V.asmStart[g];
  }
  __syncthreads();
  if (V.segs[g].ctl->newtonDone) return;
  loadSegment(V, g, sD);
  dcu::termsRows(sD, rank, size);
}

__global__ void __launch_bounds__(dcu::kAssembleThreads) k_assemble_batch(View V) {
  __shared__ dcu::Dev sD;
  __shared__ uint32_t g, rank, size;
  if (threadIdx.x == 0) {
    g = segmentOf(V.asmStart, V.G, blockIdx.x);
    rank = blockIdx.x - V.asmStart[g];
    size = V.asmStart[g + 1] - V.asmStart[g];
  }
  __syncthreads();
  if (V.segs[g].ctl->newtonDone) return;
  loadSegment(V, g, sD);
  dcu::assembleSlots(sD, rank, size);
}

// One Newton iteration's solve for every advancing garment: the blocks of garment g form its group.
template <bool Learned, int RL, int Threads>
__global__ void __launch_bounds__(Threads, 1024 / Threads) k_solve_batch(View V) {
  __shared__ dcu::Dev sD;
  __shared__ uint32_t g, rank, size;
  if (threadIdx.x == 0) {
    g = segmentOf(V.solveStart, V.G, blockIdx.x);
    rank = blockIdx.x - V.solveStart[g];
    size = V.solveStart[g + 1] - V.solveStart[g];
  }
  __syncthreads();
  if (V.segs[g].ctl->newtonDone) return;
  loadSegment(V, g, sD);
  if (threadIdx.x == 0) sD.partials = V.partials + 2ull * V.solveStart[g] * dcu::kPartialStride;
  __syncthreads();
  dcu::GridSync gs;
  gs.init(sD.ctl, sD.P.barrierLimitNs, rank, size);
  dcu::solveGroup<Learned, RL>(sD, gs);
}

// Assembly clocks of the garments that took substep s.
__global__ void k_clock_batch(View V, int substep) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.G || substep >= V.run[g].substeps) return;
  dcu::Garment* gr = V.segs[g].garment;
  if (gr->phase == 0) gr->assemblyTime += V.run[g].hD;
}

// Statistics of every garment (sim_model.cpp:222-241) in FP64 over the point-kernel partition: each block reduces
// its share of its garment's particles and seams into a row of `part`; the garment's last block to finish combines
// the garment's rows in block order (deterministic, no floating-point atomics) and resets the garment's counter.
__global__ void k_stats_batch(View V, double* part, unsigned int* done) {
  __shared__ uint32_t g, rank, size;
  if (threadIdx.x == 0) {
    g = segmentOf(V.pointStart, V.G, blockIdx.x);
    rank = blockIdx.x - V.pointStart[g];
    size = V.pointStart[g + 1] - V.pointStart[g];
  }
  __syncthreads();
  const dcu::Dev& D = V.segs[g];
  double ke = 0, v2s = 0, gap = 0, pen = 0;
  unsigned long long moving = 0;
  int bad = 0;
  const uint32_t stride = size * blockDim.x;
  for (uint32_t i = rank * blockDim.x + threadIdx.x; i < D.P.n; i += stride) {
    const float4 x4 = D.x[i], v4 = D.v[i];
    if (!isfinite(x4.x) || !isfinite(x4.y) || !isfinite(x4.z) || !isfinite(v4.x) || !isfinite(v4.y) ||
        !isfinite(v4.z))
      bad = 1;
    if (D.field.present) {
      const double phi = dcu::fieldSampleD(D.fieldValues, D.field, x4.x, x4.y, x4.z, D.fieldOrigin[0],
                                           D.fieldOrigin[1], D.fieldOrigin[2], D.fieldCell);
      pen = fmax(pen, -phi);
    }
    if (D.particle[i].pinned != 0u) continue;
    const double vv = static_cast<double>(v4.x) * v4.x + static_cast<double>(v4.y) * v4.y +
                      static_cast<double>(v4.z) * v4.z;
    ke += 0.5 * static_cast<double>(D.particle[i].mass) * vv;
    v2s += vv;
    ++moving;
  }
  for (uint32_t k = rank * blockDim.x + threadIdx.x; k < D.P.nSeam; k += stride) {
    const float4 a = D.x[D.seam[k].a], b = D.x[D.seam[k].b];
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    gap = fmax(gap, static_cast<double>(sqrtf(dx * dx + dy * dy + dz * dz)));
  }
  double sums[2] = {ke, v2s};
  __shared__ double tot[2];
  dcu::blockSum<2>(sums, tot);
  __shared__ double mx[2][32];
  __shared__ unsigned long long mv[32];
  __shared__ int bd[32];
  for (int o = 16; o > 0; o >>= 1) {
    gap = fmax(gap, __shfl_down_sync(0xffffffffu, gap, o));
    pen = fmax(pen, __shfl_down_sync(0xffffffffu, pen, o));
    moving += __shfl_down_sync(0xffffffffu, moving, o);
    bad |= __shfl_down_sync(0xffffffffu, bad, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0) {
    mx[0][w] = gap;
    mx[1][w] = pen;
    mv[w] = moving;
    bd[w] = bad;
  }
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x == 0) {
    double gp = 0, pn = 0;
    unsigned long long m = 0;
    int bb = 0;
    for (int k = 0; k < nw; ++k) {
      gp = fmax(gp, mx[0][k]);
      pn = fmax(pn, mx[1][k]);
      m += mv[k];
      bb |= bd[k];
    }
    double* row = part + blockIdx.x * 8ull;
    row[0] = tot[0];
    row[1] = tot[1];
    row[2] = gp;
    row[3] = pn;
    row[4] = static_cast<double>(m);
    row[5] = bb;
    __threadfence();
    last = atomicAdd(done + g, 1u) == size - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    StatsOut s{};
    for (uint32_t b = V.pointStart[g]; b < V.pointStart[g + 1]; ++b) {
      const double* row = part + b * 8ull;
      s.kineticEnergy += __ldcg(row + 0);
      s.sumV2 += __ldcg(row + 1);
      s.maxSeamGap = fmax(s.maxSeamGap, __ldcg(row + 2));
      s.maxPenetration = fmax(s.maxPenetration, __ldcg(row + 3));
      s.moving += static_cast<unsigned long long>(__ldcg(row + 4));
      s.nonFinite |= __ldcg(row + 5) != 0.0;
    }
    V.stats[g] = s;
    done[g] = 0;
  }
}

// Whole-batch copy of the advancing state (drape_batch_save / restore).
__global__ void k_copy_state(uint32_t n, const float4* x, const float4* v, const dcu::Contact* c, float4* xo,
                             float4* vo, dcu::Contact* co) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    xo[i] = x[i];
    vo[i] = v[i];
    co[i] = c[i];
  }
}

}  // namespace bcu

// ---------------------------------------------------------------------------------------------------------------
// Host side.

namespace {

thread_local std::string g_batchError;

constexpr int kPointThreads = 256;
constexpr int kPointRowsPerBlock = 1024;  // rows per point-kernel block (grid-stride within the garment's share)

using SolveKernel = void (*)(bcu::View);

struct Variant {
  int rowLanes, threads;
  SolveKernel jacobi, learned;
};

// Product scheme (0: slot-parallel, else lanes per row) x block size.
const Variant kVariants[] = {
    {0, 256, bcu::k_solve_batch<false, 0, 256>, bcu::k_solve_batch<true, 0, 256>},
    {2, 256, bcu::k_solve_batch<false, 2, 256>, bcu::k_solve_batch<true, 2, 256>},
    {4, 256, bcu::k_solve_batch<false, 4, 256>, bcu::k_solve_batch<true, 4, 256>},
    {8, 256, bcu::k_solve_batch<false, 8, 256>, bcu::k_solve_batch<true, 8, 256>},
    {0, 512, bcu::k_solve_batch<false, 0, 512>, bcu::k_solve_batch<true, 0, 512>},
    {2, 512, bcu::k_solve_batch<false, 2, 512>, bcu::k_solve_batch<true, 2, 512>},
    {4, 512, bcu::k_solve_batch<false, 4, 512>, bcu::k_solve_batch<true, 4, 512>},
    {8, 512, bcu::k_solve_batch<false, 8, 512>, bcu::k_solve_batch<true, 8, 512>},
    {0, 1024, bcu::k_solve_batch<false, 0, 1024>, bcu::k_solve_batch<true, 0, 1024>},
    {2, 1024, bcu::k_solve_batch<false, 2, 1024>, bcu::k_solve_batch<true, 2, 1024>},
    {4, 1024, bcu::k_solve_batch<false, 4, 1024>, bcu::k_solve_batch<true, 4, 1024>},
    {8, 1024, bcu::k_solve_batch<false, 8, 1024>, bcu::k_solve_batch<true, 8, 1024>},
};
constexpr int kVariantCount = sizeof(kVariants) / sizeof(kVariants[0]);

uint32_t maxRangeSlots(const std::vector<uint32_t>& rowStart, uint32_t n, uint32_t parts) {
  const uint32_t per = (n + parts - 1) / parts;
  uint32_t most = 0;
  for (uint32_t b = 0; b < parts; ++b) {
    const uint32_t r0 = std::min(n, b * per), r1 = std::min(n, r0 + per);
    most = std::max(most, rowStart[r1] - rowStart[r0]);
  }
  return most;
}

std::vector<uint32_t> prefix(const std::vector<uint32_t>& counts) {
  std::vector<uint32_t> out(counts.size() + 1, 0);
  for (size_t g = 0; g < counts.size(); ++g) out[g + 1] = out[g] + counts[g];
  return out;
}

// Splits `total` blocks among the weighted garments: every garment with a positive weight gets at least one block,
// the rest in proportion (largest remainders first). Throws when there are more such garments than blocks.
std::vector<uint32_t> apportion(const std::vector<double>& weight, uint32_t total) {
  const size_t G = weight.size();
  std::vector<uint32_t> out(G, 0);
  double W = 0;
  uint32_t live = 0;
  for (double w : weight)
    if (w > 0) {
      W += w;
      ++live;
    }
  if (live == 0) return out;
  if (live > total) throw std::invalid_argument("more advancing garments than solve blocks");
  std::vector<std::pair<double, size_t>> rem;
  uint32_t used = 0;
  for (size_t g = 0; g < G; ++g) {
    if (weight[g] <= 0) continue;
    const double share = (total - live) * weight[g] / W;
    out[g] = 1 + static_cast<uint32_t>(share);
    used += out[g];
    rem.push_back({share - std::floor(share), g});
  }
  std::sort(rem.begin(), rem.end(), [](const auto& a, const auto& b) {
    return a.first > b.first || (a.first == b.first && a.second < b.second);
  });
  for (size_t k = 0; used < total && k < rem.size(); ++k, ++used) ++out[rem[k].second];
  return out;
}

// One garment's drape runner (DrapeSession, libs/sim/src/drape_session.cpp:32-95, with the batch's frame split:
// decisions taken after a frame act at the start of the next one).
struct Session {
  int state = DRAPE_STATE_ASSEMBLING, phase = DRAPE_PHASE_ASSEMBLING;
  double time = 0, phaseTime = 0, lastEnergy = INFINITY;
  int substeps = 1, stillFrames = 0, riseFrames = 0, keptFrames = 0;
  double savedTime = 0, savedPhaseTime = 0;
  int savedPhase = DRAPE_PHASE_ASSEMBLING;
  drape_drape_result result{};
  double finishedAt = 0;  // wall seconds from the start of the drape
  bool finished() const {
    return state == DRAPE_STATE_SETTLED || state == DRAPE_STATE_FAILED || state == DRAPE_STATE_TIMED_OUT;
  }
};

}  // namespace

struct drape_batch {
  int device = 0, numSMs = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  std::vector<Model> models;
  bool built = false;
  uint32_t G = 0, N = 0, B = 0, SP = 0;
  unsigned long long barrierLimitNs = 2000000000ull;
  std::vector<uint32_t> pBase, sBase, kBase;
  std::vector<uint32_t> pointCount, asmCount;

  DBuf<dcu::Particle> particle;
  DBuf<dcu::Fabric> fabric;
  DBuf<dcu::Garment> garment, snapG, saveG;
  DBuf<dcu::Stretch> stretch;
  DBuf<dcu::Hinge> hinge;
  DBuf<dcu::Seam> seam, saveSeam;
  DBuf<uint32_t> rowStart, colIndex, diagSlot, incStart, incEntry, offSlot, offStart, offCode, tslot;
  DBuf<uint32_t> starts, bases;  // point and assembly prefixes; pBase and kBase
  DBuf<float> fieldValues, blocks, snapGap;
  DBuf<float4> x, v, xStart, yRel, u, grad, step, r, z, p0, p1, ap, apFull, resid, fExt, pinPos, precond;
  DBuf<float4> snapX, snapV, saveX, saveV;
  DBuf<float4> stretchDer, hingeDer;  // per-term derivative records (6 and 4 float4 per term)
  DBuf<dcu::Contact> contact, snapC, saveC;
  DBuf<double> partials;
  DBuf<dcu::Control> ctl;
  DBuf<dcu::Dev> segs;
  DBuf<bcu::StatsOut> stats;
  DBuf<double> statsPart;         // 8 doubles per point-kernel block
  DBuf<unsigned int> statsDone;   // per garment: blocks of k_stats_batch finished
  DBuf<unsigned char> control;  // frame control: G SegRun, then G + 1 solve-block starts
  HostPinned<unsigned char> hControl;
  HostPinned<bcu::StatsOut> hStats;
  HostPinned<dcu::Control> hCtl;
  bcu::View view{};

  // Learned preconditioner over the whole batch graph (global indices), the factor read per garment.
  std::unique_ptr<net::Network> net;
  net::GraphHandle netGraph;
  DBuf<uint32_t> gRowStart, gColIndex;
  bool learnedOn = false;

  int variant = 0;          // kVariants index: slot-parallel products, 256 threads
  int solveBlocks = 0;      // blocks of the solve launch for the variant
  uint32_t capSlots = 0;    // shared-memory slot capacity of one solve block for the variant
  size_t solveSmem = 0;
  std::vector<uint32_t> solveCount;  // current solve partition
  bool tunedByHand = false;

  cudaGraphExec_t graphExec = nullptr;
  int graphSubsteps = -1, graphIterations = -1, graphVariant = -1, graphLearned = -1;
  bool graphUsable = true;

  bool profiling = false;
  drape_batch_profile prof{};
  std::vector<cudaEvent_t> events;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> solveEvents, frameEvents;

  explicit drape_batch(int dev) : device(dev) {
    int count = 0;
    BCK(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) throw std::runtime_error("cuda: no device " + std::to_string(device));
    BCK(cudaSetDevice(device));
    cudaDeviceProp prop{};
    BCK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) throw std::runtime_error(std::string("cuda: device ") + prop.name + " is not sm_100");
    if (!prop.cooperativeLaunch) throw std::runtime_error("cuda: device does not support cooperative launch");
    numSMs = prop.multiProcessorCount;
    BCK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    hStats.alloc(1);
    hCtl.alloc(1);
  }

  ~drape_batch() {
    if (stream) {
      cudaSetDevice(device);
      cudaStreamSynchronize(stream);
      if (graphExec) cudaGraphExecDestroy(graphExec);
      for (auto e : events) cudaEventDestroy(e);
      for (auto& p : solveEvents) {
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
      }
      for (auto& p : frameEvents) {
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
      }
      cudaStreamDestroy(stream);
    }
  }

  void use() const { BCK(cudaSetDevice(device)); }
  void requireBuilt() const {
    if (!built) throw std::logic_error("not built");
  }

  bcu::SegRun* runs() { return reinterpret_cast<bcu::SegRun*>(hControl.p); }
  uint32_t* solveStartHost() { return reinterpret_cast<uint32_t*>(hControl.p + sizeof(bcu::SegRun) * G); }

  void add(const drape_scene_desc& scene) {
    if (built) throw std::logic_error("the batch is already built");
    if (scene.garment_count != 1) throw std::invalid_argument("a batch garment's scene must hold exactly one garment");
    models.push_back(Model::build(scene));
  }

  // ---- build ----

  void build() {
    if (built) throw std::logic_error("the batch is already built");
    if (models.empty()) throw std::invalid_argument("the batch has no garments");
    use();
    G = static_cast<uint32_t>(models.size());
    pBase.assign(G, 0);
    sBase.assign(G, 0);
    kBase.assign(G, 0);
    std::vector<uint32_t> tBase(G), hBase(G), eBase(G), fabBase(G), fieldBase(G), rBase(G), cBase(G);
    uint32_t n = 0, b = 0, t = 0, h = 0, k = 0, e = 0, fab = 0, fv = 0, cc = 0;
    for (uint32_t g = 0; g < G; ++g) {
      const Model& m = models[g];
      pBase[g] = n;
      sBase[g] = b;
      tBase[g] = t;
      hBase[g] = h;
      kBase[g] = k;
      eBase[g] = e;
      fabBase[g] = fab;
      fieldBase[g] = fv;
      rBase[g] = n + g;
      cBase[g] = cc;
      n += static_cast<uint32_t>(m.x.size());
      b += static_cast<uint32_t>(m.colIndex.size());
      t += static_cast<uint32_t>(m.stretch.size());
      h += static_cast<uint32_t>(m.hinges.size());
      k += static_cast<uint32_t>(m.seams.size());
      e += static_cast<uint32_t>(m.incEntry.size());
      cc += static_cast<uint32_t>(m.offContrib.size());
      fab += static_cast<uint32_t>(dmodel::fabrics(m).size());
      fv += static_cast<uint32_t>(std::max<size_t>(m.fieldValues.size(), 1));
    }
    N = n;
    B = b;
    SP = (B + 31u) & ~31u;
    // Host staging of the concatenated arrays.
    std::vector<dcu::Particle> hp;
    std::vector<dcu::Fabric> hf;
    std::vector<dcu::Garment> hg;
    std::vector<dcu::Stretch> hs;
    std::vector<dcu::Hinge> hh;
    std::vector<dcu::Seam> hk;
    std::vector<uint32_t> hrs, hci, hds, his, hie, hos, hoS, hoc, hts;
    std::vector<float> hfv;
    std::vector<float4> hx, hv, hfe, hpp;
    for (uint32_t g = 0; g < G; ++g) {
      const Model& m = models[g];
      auto append = [](auto& dst, const auto& src) { dst.insert(dst.end(), src.begin(), src.end()); };
      append(hp, dmodel::particles(m));
      append(hf, dmodel::fabrics(m));
      append(hg, dmodel::garments(m));
      append(hs, dmodel::stretches(m));
      append(hh, dmodel::hinges(m));
      append(hk, dmodel::seams(m));
      append(hrs, m.rowStart);
      const std::vector<uint32_t> cols = dmodel::columns(m);
      append(hci, cols);
      append(hds, m.diagSlot);
      append(his, m.incStart);
      append(hie, m.incEntry);
      append(hos, m.offSlot);
      append(hoS, m.offStart);
      append(hoc, m.offCode);
      append(hts, net::transposedSlots(m.rowStart, cols));
      if (m.fieldValues.empty()) hfv.push_back(0.0f); else append(hfv, m.fieldValues);
      std::vector<float4> xs, vs, fe, pp;
      dmodel::state(m, xs, vs, fe, pp);
      append(hx, xs);
      append(hv, vs);
      append(hfe, fe);
      append(hpp, pp);
    }
    cudaStream_t s = stream;
    particle.upload(hp, s);
    fabric.upload(hf, s);
    garment.upload(hg, s);
    stretch.upload(hs, s);
    hinge.upload(hh, s);
    seam.upload(hk, s);
    rowStart.upload(hrs, s);
    colIndex.upload(hci, s);
    diagSlot.upload(hds, s);
    incStart.upload(his, s);
    incEntry.upload(hie, s);
    offSlot.upload(hos, s);
    offStart.upload(hoS, s);
    offCode.upload(hoc, s);
    tslot.upload(hts, s);
    fieldValues.upload(hfv, s);
    blocks.alloc(static_cast<size_t>(SP) * 9);
    for (DBuf<float4>* buf : {&x, &v, &xStart, &yRel, &u, &grad, &step, &r, &z, &p0, &p1, &ap, &apFull, &resid,
                              &fExt, &pinPos, &snapX, &snapV, &saveX, &saveV})
      buf->alloc(N);
    precond.alloc(static_cast<size_t>(N) * 3);
    stretchDer.alloc(std::max<size_t>(1, 6ull * t));
    hingeDer.alloc(std::max<size_t>(1, 4ull * h));
    for (DBuf<dcu::Contact>* buf : {&contact, &snapC, &saveC}) buf->alloc(N);
    x.upload(hx, s);
    v.upload(hv, s);
    fExt.upload(hfe, s);
    pinPos.upload(hpp, s);
    snapG.alloc(G);
    saveG.alloc(G);
    saveSeam.alloc(std::max<uint32_t>(k, 1));
    snapGap.alloc(std::max<uint32_t>(k, 1));
    ctl.alloc(G);
    stats.alloc(G);
    hStats.alloc(G);
    hCtl.alloc(G);
    // Launch partitions of the point and assembly kernels (fixed): blocks in proportion to the garment's rows.
    pointCount.assign(G, 0);
    asmCount.assign(G, 0);
    for (uint32_t g = 0; g < G; ++g) {
      const uint32_t ng = static_cast<uint32_t>(models[g].x.size());
      pointCount[g] = std::max<uint32_t>(1, (ng + kPointRowsPerBlock - 1) / kPointRowsPerBlock);
      const uint32_t bg = static_cast<uint32_t>(models[g].colIndex.size());
      asmCount[g] = std::max<uint32_t>(1, (bg + dcu::kAssembleThreads - 1) / dcu::kAssembleThreads);
    }
    const auto pStart = prefix(pointCount), aStart = prefix(asmCount);
    statsPart.alloc(8ull * pStart[G]);
    statsDone.alloc(G);
    std::vector<uint32_t> st(pStart);
    st.insert(st.end(), aStart.begin(), aStart.end());
    starts.upload(st, s);
    std::vector<uint32_t> bs(pBase);
    bs.insert(bs.end(), kBase.begin(), kBase.end());
    bases.upload(bs, s);
    // Segment views.
    std::vector<dcu::Dev> views(G);
    for (uint32_t g = 0; g < G; ++g) {
      const Model& m = models[g];
      dcu::Dev& d = views[g];
      d = dcu::Dev{};
      dmodel::params(m, SP, barrierLimitNs, d);
      const uint32_t pb = pBase[g];
      d.fieldValues = fieldValues.p + fieldBase[g];
      d.particle = particle.p + pb;
      d.fabric = fabric.p + fabBase[g];
      d.garment = garment.p + g;
      d.stretch = stretch.p + tBase[g];
      d.hinge = hinge.p + hBase[g];
      d.stretchDer = stretchDer.p + 6ull * tBase[g];
      d.hingeDer = hingeDer.p + 4ull * hBase[g];
      d.seam = seam.p + kBase[g];
      d.rowStart = rowStart.p + rBase[g];
      d.colIndex = colIndex.p + sBase[g];
      d.diagSlot = diagSlot.p + pb;
      d.incStart = incStart.p + rBase[g];
      d.incEntry = incEntry.p + eBase[g];
      d.offSlot = offSlot.p + (sBase[g] - pBase[g]);
      d.offStart = offStart.p + (sBase[g] - pBase[g] + g);
      d.offCode = offCode.p + cBase[g];
      for (auto [dst, src] : {std::pair<float4**, float4*>{&d.x, x.p}, {&d.v, v.p}, {&d.xStart, xStart.p},
                              {&d.yRel, yRel.p}, {&d.u, u.p}, {&d.grad, grad.p}, {&d.step, step.p}, {&d.r, r.p},
                              {&d.z, z.p}, {&d.p0, p0.p}, {&d.p1, p1.p}, {&d.ap, ap.p}, {&d.apFull, apFull.p},
                              {&d.resid, resid.p}})
        *dst = src + pb;
      d.fExt = fExt.p + pb;
      d.pinPos = pinPos.p + pb;
      d.blocks = blocks.p + sBase[g];
      d.precond = precond.p + 3ull * pb;
      d.contact = contact.p + pb;
      d.ctl = ctl.p + g;
      d.tslot = tslot.p + sBase[g];
      d.cgLog = nullptr;
    }
    segs.upload(views, s);
    control.alloc(sizeof(bcu::SegRun) * G + sizeof(uint32_t) * (G + 1));
    hControl.alloc(sizeof(bcu::SegRun) * G + sizeof(uint32_t) * (G + 1));
    view.segs = segs.p;
    view.run = reinterpret_cast<const bcu::SegRun*>(control.p);
    view.solveStart = reinterpret_cast<const uint32_t*>(control.p + sizeof(bcu::SegRun) * G);
    view.pointStart = starts.p;
    view.asmStart = starts.p + (G + 1);
    view.pBase = bases.p;
    view.kBase = bases.p + G;
    view.seams = seam.p;
    view.snapX = snapX.p;
    view.snapV = snapV.p;
    view.snapC = snapC.p;
    view.snapG = snapG.p;
    view.snapGap = snapGap.p;
    view.stats = stats.p;
    view.G = G;
    BCK(cudaStreamSynchronize(s));
    built = true;
    setVariant(variant);
    if (learnedOn) bindNet();
  }

  // ---- solve variant and partition ----

  void setVariant(int vi) {
    const Variant& V = kVariants[vi];
    const int perSM = 1024 / V.threads;
    size_t dyn = 0;
    for (SolveKernel k : {V.jacobi, V.learned}) {
      size_t avail = 0;
      BCK(cudaOccupancyAvailableDynamicSMemPerBlock(&avail, reinterpret_cast<const void*>(k), perSM, V.threads));
      dyn = dyn == 0 ? avail : std::min(dyn, avail);
    }
    capSlots = static_cast<uint32_t>(dyn / dcu::kSmemSlotBytes);
    solveSmem = static_cast<size_t>(capSlots) * dcu::kSmemSlotBytes;
    for (SolveKernel k : {V.jacobi, V.learned}) {
      BCK(cudaFuncSetAttribute(reinterpret_cast<const void*>(k), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(solveSmem)));
      int blocksPerSM = 0;
      BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocksPerSM, reinterpret_cast<const void*>(k), V.threads,
                                                        solveSmem));
      if (blocksPerSM < perSM) throw std::runtime_error("cuda: the batch solve variant does not fit its blocks per SM");
    }
    variant = vi;
    solveBlocks = numSMs * perSM;
    partials.alloc(2ull * solveBlocks * dcu::kPartialStride);
    view.partials = partials.p;
    solveCount.clear();
  }

  // Solve blocks for the advancing garments (substeps > 0 this frame); writes the starts and smem slot caps into the
  // frame control.
  void partition(const std::vector<int>& substeps) {
    std::vector<double> w(G, 0.0);
    for (uint32_t g = 0; g < G; ++g)
      if (substeps[g] > 0) w[g] = static_cast<double>(models[g].colIndex.size()) + 5.0 * models[g].x.size();
    solveCount = apportion(w, static_cast<uint32_t>(solveBlocks));
    const std::vector<uint32_t>& count = solveCount;
    const auto start = prefix(count);
    uint32_t* hs = solveStartHost();
    for (uint32_t g = 0; g <= G; ++g) hs[g] = start[g];
    bcu::SegRun* rr = runs();
    for (uint32_t g = 0; g < G; ++g) {
      const uint32_t ng = static_cast<uint32_t>(models[g].x.size());
      rr[g].smemSlots = count[g] ? std::min(capSlots, maxRangeSlots(models[g].rowStart, ng, count[g])) : 0;
    }
  }

  // ---- learned preconditioner ----

  void bindNet() {
    std::vector<uint32_t> grs(N + 1), gci;
    grs[0] = 0;
    gci.reserve(B);
    for (uint32_t g = 0; g < G; ++g) {
      const Model& m = models[g];
      for (size_t i = 1; i < m.rowStart.size(); ++i) grs[pBase[g] + i] = sBase[g] + m.rowStart[i];
      for (uint32_t c : dmodel::columns(m)) gci.push_back(c + pBase[g]);  // the pinned bit (bit 31) is kept
    }
    gRowStart.upload(grs, stream);
    gColIndex.upload(gci, stream);
    netGraph = net->bind(N, B, SP, grs.data(), gci.data(), gRowStart.p, gColIndex.p, blocks.p,
                         reinterpret_cast<const uint8_t*>(particle.p) + offsetof(dcu::Particle, pinned),
                         sizeof(dcu::Particle),
                         reinterpret_cast<const uint8_t*>(contact.p) + offsetof(dcu::Contact, active),
                         sizeof(dcu::Contact), stream);
    const float* L = net->graphOf(*netGraph).L;
    std::vector<dcu::Dev> views(G);
    BCK(cudaMemcpyAsync(views.data(), segs.p, sizeof(dcu::Dev) * G, cudaMemcpyDeviceToHost, stream));
    BCK(cudaStreamSynchronize(stream));
    for (uint32_t g = 0; g < G; ++g) views[g].Lf = L + sBase[g];
    segs.upload(views, stream);
    BCK(cudaStreamSynchronize(stream));
    dropGraph();
  }

  void setPrecond(drape_precond* p) {
    if (!p) {
      learnedOn = false;
      netGraph.reset();
      dropGraph();
      return;
    }
    if (!p->net) throw std::invalid_argument("null preconditioner handle");
    std::vector<float> w(net::Layout::kCount);
    p->net->getParams(w.data(), w.size());
    if (!net) net = std::make_unique<net::Network>(device);
    net->setParams(w.data(), w.size());
    learnedOn = true;
    if (built) bindNet();
  }

  // ---- frames ----

  void dropGraph() {
    if (graphExec) {
      cudaGraphExecDestroy(graphExec);
      graphExec = nullptr;
    }
    graphSubsteps = graphIterations = graphVariant = graphLearned = -1;
  }

  cudaEvent_t takeEvent() {
    if (events.empty()) {
      cudaEvent_t e;
      BCK(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = events.back();
    events.pop_back();
    return e;
  }

  void launchSolve(bool timed) {
    const Variant& V = kVariants[variant];
    SolveKernel k = learnedOn && netGraph ? V.learned : V.jacobi;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(solveBlocks);
    cfg.blockDim = dim3(V.threads);
    cfg.dynamicSmemBytes = solveSmem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaEvent_t a = nullptr;
    if (timed) {
      a = takeEvent();
      BCK(cudaEventRecord(a, stream));
    }
    BCK(cudaLaunchKernelEx(&cfg, k, view));
    if (timed) {
      cudaEvent_t b = takeEvent();
      BCK(cudaEventRecord(b, stream));
      solveEvents.push_back({a, b});
    }
  }

  // Enqueues one frame: per-garment control upload, actions, substeps x (activation, assembly, [network], solve),
  // finish and clocks, statistics, control-block and statistics download. Returns the kernels it launched.
  int enqueueFrame(int maxSubsteps, int iterations, bool timed) {
    const size_t ctlBytes = sizeof(bcu::SegRun) * G + sizeof(uint32_t) * (G + 1);
    BCK(cudaMemcpyAsync(control.p, hControl.p, ctlBytes, cudaMemcpyHostToDevice, stream));
    int launches = 0;
    const uint32_t pointGrid = [&] { uint32_t t = 0; for (auto c : pointCount) t += c; return t; }();
    const uint32_t asmGrid = [&] { uint32_t t = 0; for (auto c : asmCount) t += c; return t; }();
    bcu::k_actions_particles<<<pointGrid, kPointThreads, 0, stream>>>(view);
    bcu::k_actions_garment<<<G, 128, 0, stream>>>(view);
    launches += 2;
    for (int s = 0; s < maxSubsteps; ++s) {
      bcu::k_points<0><<<pointGrid, kPointThreads, 0, stream>>>(view, s);
      ++launches;
      for (int it = 0; it < iterations; ++it) {
        bcu::k_points<1><<<pointGrid, kPointThreads, 0, stream>>>(view, s);
        bcu::k_terms_batch<<<asmGrid, dcu::kAssembleThreads, 0, stream>>>(view);
        bcu::k_assemble_batch<<<asmGrid, dcu::kAssembleThreads, 0, stream>>>(view);
        launches += 3;
        if (learnedOn && netGraph) {
          net->forwardOn(net->graphOf(*netGraph), stream, false, &ctl.p->error);
          launches += 8;
        }
        launchSolve(timed);
        ++launches;
      }
      bcu::k_points<2><<<pointGrid, kPointThreads, 0, stream>>>(view, s);
      bcu::k_clock_batch<<<(G + 127) / 128, 128, 0, stream>>>(view, s);
      launches += 2;
    }
    bcu::k_stats_batch<<<pointGrid, kPointThreads, 0, stream>>>(view, statsPart.p, statsDone.p);
    ++launches;
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(hStats.p, stats.p, sizeof(bcu::StatsOut) * G, cudaMemcpyDeviceToHost, stream));
    BCK(cudaMemcpyAsync(hCtl.p, ctl.p, sizeof(dcu::Control) * G, cudaMemcpyDeviceToHost, stream));
    return launches;
  }

  // Runs one frame with the frame control already in the pinned buffer (substeps, lengths, actions); the solve
  // partition follows the advancing garments. Reads back statistics and control blocks; throws on a device error.
  void runFrame(const std::vector<int>& substeps, int iterations) {
    partition(substeps);  // the partition lives in the frame control, which a graph replay reads at launch
    int maxSub = 0;
    for (int s : substeps) maxSub = std::max(maxSub, s);
    const bool learned = learnedOn && netGraph;
    if (profiling) {
      cudaEvent_t a = takeEvent(), b = takeEvent();
      BCK(cudaEventRecord(a, stream));
      prof.kernel_launches += enqueueFrame(maxSub, iterations, true);
      BCK(cudaEventRecord(b, stream));
      frameEvents.push_back({a, b});
      prof.solve_launches += maxSub * iterations;
    } else {
      if (graphUsable && (!graphExec || graphSubsteps != maxSub || graphIterations != iterations ||
                          graphVariant != variant || graphLearned != static_cast<int>(learned))) {
        dropGraph();
        capture(maxSub, iterations);
      }
      if (graphExec) {
        BCK(cudaGraphLaunch(graphExec, stream));
        ++prof.graph_launches;
      } else {
        prof.kernel_launches += enqueueFrame(maxSub, iterations, false);
      }
    }
    ++prof.frames;
    BCK(cudaStreamSynchronize(stream));
    if (profiling) collectEvents();
    for (uint32_t g = 0; g < G; ++g)
      if (hCtl.p[g].error != 0) {
        const int e = hCtl.p[g].error;
        resetErrors();
        throw std::runtime_error(e == 1 ? "cuda: a grid barrier timed out (the batch frame was abandoned)"
                                        : "cuda: device error status " + std::to_string(e));
      }
  }

  void capture(int maxSub, int iterations) {
    cudaGraph_t graph = nullptr;
    BCK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    int launches = 0;
    try {
      launches = enqueueFrame(maxSub, iterations, false);
    } catch (...) {
      cudaStreamEndCapture(stream, &graph);
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      graphUsable = false;
      return;
    }
    if (cudaStreamEndCapture(stream, &graph) != cudaSuccess || !graph) {
      cudaGetLastError();
      graphUsable = false;
      return;
    }
    const cudaError_t e = cudaGraphInstantiate(&graphExec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      cudaGetLastError();
      graphExec = nullptr;
      graphUsable = false;
      return;
    }
    graphSubsteps = maxSub;
    graphIterations = iterations;
    graphVariant = variant;
    graphLearned = learnedOn && netGraph ? 1 : 0;
    graphLaunchesPerFrame = launches;
  }
  int graphLaunchesPerFrame = 0;

  void collectEvents() {
    for (auto& p : solveEvents) {
      float ms = 0;
      BCK(cudaEventElapsedTime(&ms, p.first, p.second));
      prof.solve_ms += ms;
      events.push_back(p.first);
      events.push_back(p.second);
    }
    solveEvents.clear();
    for (auto& p : frameEvents) {
      float ms = 0;
      BCK(cudaEventElapsedTime(&ms, p.first, p.second));
      prof.frame_ms += ms;
      events.push_back(p.first);
      events.push_back(p.second);
    }
    frameEvents.clear();
  }

  void resetErrors() {
    std::vector<dcu::Control> c(G);
    BCK(cudaMemcpy(c.data(), ctl.p, sizeof(dcu::Control) * G, cudaMemcpyDeviceToHost));
    for (auto& x : c) {
      x.error = 0;
      x.barrierArrivals = 0;
    }
    BCK(cudaMemcpy(ctl.p, c.data(), sizeof(dcu::Control) * G, cudaMemcpyHostToDevice));
  }

  void setRun(uint32_t g, double dt, int substeps, int32_t action) {
    bcu::SegRun& r = runs()[g];
    const int sub = std::max(1, substeps);
    const double h = dt / sub;
    r.h = static_cast<float>(h);
    r.invH2 = static_cast<float>(1.0 / (h * h));
    r.hD = h;
    r.substeps = substeps;
    r.action = action;
  }

  // ---- public operations ----

  void advance(double dt, int substeps, int iterations) {
    requireBuilt();
    use();
    std::vector<int> subs(G, std::max(1, substeps));
    for (uint32_t g = 0; g < G; ++g) setRun(g, dt, subs[g], 0);
    runFrame(subs, std::max(1, iterations));
  }

  void setPhase(uint32_t g, int phase) {
    requireBuilt();
    if (g >= G) throw std::out_of_range("no such garment in the batch");
    if (phase != DRAPE_PHASE_ASSEMBLING && phase != DRAPE_PHASE_SETTLING) throw std::invalid_argument("unknown phase");
    use();
    for (uint32_t k = 0; k < G; ++k) setRun(k, 1.0, 0, 0);
    runs()[g].action = phase == DRAPE_PHASE_ASSEMBLING ? bcu::kActAssemble : bcu::kActSettle;
    runFrame(std::vector<int>(G, 0), 1);
  }

  drape_stats statsOf(uint32_t g) const {
    drape_stats st{};
    const bcu::StatsOut& s = hStats.p[g];
    st.has_non_finite = s.nonFinite;
    st.kinetic_energy = s.kineticEnergy;
    st.rms_speed = s.moving ? std::sqrt(s.sumV2 / static_cast<double>(s.moving)) : 0.0;
    st.max_seam_gap = s.maxSeamGap;
    st.max_body_penetration = models[g].hasBody ? s.maxPenetration : 0.0;
    return st;
  }

  // Statistics of the current state without advancing (a frame in which no garment takes a substep).
  void refreshStats() {
    for (uint32_t k = 0; k < G; ++k) setRun(k, 1.0, 0, 0);
    runFrame(std::vector<int>(G, 0), 1);
  }

  // drapeToRest for every garment (the loop of drape_session.cpp:32-95 per garment).
  void drapeToRest(const drape_drape_options& o, drape_drape_result* results, double* settleSeconds) {
    requireBuilt();
    use();
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<Session> ss(G);
    constexpr double kEps = 1e-9;
    // Start: every garment enters Assembling; the snapshot holds that state.
    for (uint32_t g = 0; g < G; ++g) {
      ss[g].substeps = o.substeps;
      setRun(g, o.frame_dt, 0, bcu::kActAssemble | bcu::kActSave);
    }
    runFrame(std::vector<int>(G, 0), o.iterations);
    std::vector<int> subs(G, 0);
    std::vector<int32_t> nextAction(G, 0);
    for (;;) {
      bool any = false;
      for (uint32_t g = 0; g < G; ++g) {
        Session& S = ss[g];
        subs[g] = 0;
        if (S.finished()) continue;
        if (S.time >= o.max_sim_seconds - kEps) {
          S.result.simulated_seconds = S.time;
          S.state = DRAPE_STATE_TIMED_OUT;
          S.finishedAt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
          continue;
        }
        subs[g] = std::max(1, S.substeps);
        any = true;
      }
      if (!any) break;
      for (uint32_t g = 0; g < G; ++g) setRun(g, o.frame_dt, subs[g], nextAction[g]);
      runFrame(subs, std::max(1, o.iterations));
      const double now = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      for (uint32_t g = 0; g < G; ++g) {
        nextAction[g] = 0;
        if (subs[g] == 0) continue;
        Session& S = ss[g];
        ++S.result.frames_run;
        ++S.keptFrames;
        S.time += o.frame_dt;
        S.phaseTime += o.frame_dt;
        const drape_stats st = statsOf(g);
        S.riseFrames = st.kinetic_energy > S.lastEnergy ? S.riseFrames + 1 : 0;
        S.lastEnergy = st.kinetic_energy;
        auto resetCounters = [&] {
          S.stillFrames = 0;
          S.riseFrames = 0;
          S.lastEnergy = INFINITY;
        };
        if (st.has_non_finite || S.riseFrames >= o.energy_rise_frames) {
          ++S.result.retries;
          if (S.result.retries > o.max_retries) {
            S.result.retries = o.max_retries;
            S.result.failed = 1;
            S.result.simulated_seconds = S.time;
            S.state = DRAPE_STATE_FAILED;
            S.finishedAt = now;
            continue;
          }
          nextAction[g] = bcu::kActRestore;
          S.time = S.savedTime;
          S.phase = S.savedPhase;
          S.phaseTime = S.savedPhaseTime;
          S.keptFrames = static_cast<int>(S.savedTime / o.frame_dt + 0.5);
          S.substeps *= 2;
          resetCounters();
          S.state = S.phase == DRAPE_PHASE_ASSEMBLING ? DRAPE_STATE_ASSEMBLING : DRAPE_STATE_SETTLING;
          continue;
        }
        if (S.phase == DRAPE_PHASE_ASSEMBLING) {
          if (st.max_seam_gap < o.seam_gap_done || S.phaseTime >= o.max_assembly_seconds - kEps) {
            S.result.assembly_end_seam_gap = st.max_seam_gap;
            S.result.assembly_seconds = S.time;
            S.phase = DRAPE_PHASE_SETTLING;
            nextAction[g] |= bcu::kActSettle;
            S.phaseTime = 0;
            resetCounters();
          }
        } else {
          S.stillFrames = st.rms_speed < o.settle_rms_speed ? S.stillFrames + 1 : 0;
          if (S.stillFrames >= o.settle_hold_frames) {
            S.result.settled = 1;
            S.result.simulated_seconds = S.time;
            S.state = DRAPE_STATE_SETTLED;
            S.finishedAt = now;
            continue;
          }
        }
        if (S.keptFrames % o.snapshot_every == 0) {
          nextAction[g] |= bcu::kActSave;
          S.savedTime = S.time;
          S.savedPhase = S.phase;
          S.savedPhaseTime = S.phaseTime;
        }
        if (S.time >= o.max_sim_seconds - kEps) {
          S.result.simulated_seconds = S.time;
          S.state = DRAPE_STATE_TIMED_OUT;
          S.finishedAt = now;
          continue;
        }
        S.state = S.phase == DRAPE_PHASE_ASSEMBLING ? DRAPE_STATE_ASSEMBLING : DRAPE_STATE_SETTLING;
      }
    }
    // Apply the phase changes still pending for finished garments, so the device state matches the sessions.
    bool pending = false;
    for (uint32_t g = 0; g < G; ++g) {
      setRun(g, o.frame_dt, 0, nextAction[g] & bcu::kActSettle);
      pending |= nextAction[g] != 0;
    }
    if (pending) runFrame(std::vector<int>(G, 0), 1);
    for (uint32_t g = 0; g < G; ++g) {
      results[g] = ss[g].result;
      if (settleSeconds) settleSeconds[g] = ss[g].finishedAt;
    }
  }

  void save() {
    requireBuilt();
    use();
    const int grid = numSMs * 4;
    bcu::k_copy_state<<<grid, 256, 0, stream>>>(N, x.p, v.p, contact.p, saveX.p, saveV.p, saveC.p);
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(saveG.p, garment.p, sizeof(dcu::Garment) * G, cudaMemcpyDeviceToDevice, stream));
    BCK(cudaMemcpyAsync(saveSeam.p, seam.p, sizeof(dcu::Seam) * seam.n, cudaMemcpyDeviceToDevice, stream));
    BCK(cudaStreamSynchronize(stream));
    saved = true;
  }
  bool saved = false;

  void restore() {
    requireBuilt();
    if (!saved) throw std::logic_error("no saved batch state");
    use();
    const int grid = numSMs * 4;
    bcu::k_copy_state<<<grid, 256, 0, stream>>>(N, saveX.p, saveV.p, saveC.p, x.p, v.p, contact.p);
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(garment.p, saveG.p, sizeof(dcu::Garment) * G, cudaMemcpyDeviceToDevice, stream));
    BCK(cudaMemcpyAsync(seam.p, saveSeam.p, sizeof(dcu::Seam) * seam.n, cudaMemcpyDeviceToDevice, stream));
    BCK(cudaStreamSynchronize(stream));
  }

  drape_batch_tuning tuning() const {
    drape_batch_tuning t{};
    t.row_lanes = kVariants[variant].rowLanes;
    t.block_threads = kVariants[variant].threads;
    t.blocks = solveBlocks;
    return t;
  }

  drape_batch_tuning autotune(int frames) {
    requireBuilt();
    use();
    if (frames < 1) throw std::invalid_argument("frames must be >= 1");
    // Keep the caller's saved state: tuning saves and restores its own.
    const bool wasSaved = saved;
    DBuf<float4> kx, kv;
    DBuf<dcu::Contact> kc;
    DBuf<dcu::Garment> kg;
    DBuf<dcu::Seam> ks;
    if (wasSaved) {
      kx.alloc(N);
      kv.alloc(N);
      kc.alloc(N);
      kg.alloc(G);
      ks.alloc(seam.n);
      BCK(cudaMemcpyAsync(kx.p, saveX.p, sizeof(float4) * N, cudaMemcpyDeviceToDevice, stream));
      BCK(cudaMemcpyAsync(kv.p, saveV.p, sizeof(float4) * N, cudaMemcpyDeviceToDevice, stream));
      BCK(cudaMemcpyAsync(kc.p, saveC.p, sizeof(dcu::Contact) * N, cudaMemcpyDeviceToDevice, stream));
      BCK(cudaMemcpyAsync(kg.p, saveG.p, sizeof(dcu::Garment) * G, cudaMemcpyDeviceToDevice, stream));
      BCK(cudaMemcpyAsync(ks.p, saveSeam.p, sizeof(dcu::Seam) * seam.n, cudaMemcpyDeviceToDevice, stream));
    }
    save();
    const bool wasProfiling = profiling;
    const drape_batch_profile keep = prof;
    int best = variant, timed = 0;
    double bestMs = INFINITY;
    for (int vi = 0; vi < kVariantCount; ++vi) {
      ++timed;
      setVariant(vi);
      restore();
      profiling = true;
      prof = drape_batch_profile{};
      for (int f = 0; f < frames; ++f) advance(1.0 / 60.0, 1, 2);
      const double ms = prof.solve_ms / std::max<int64_t>(1, prof.solve_launches);
      if (ms < bestMs) {
        bestMs = ms;
        best = vi;
      }
    }
    profiling = wasProfiling;
    prof = keep;
    setVariant(best);
    restore();
    dropGraph();
    if (wasSaved) {
      BCK(cudaMemcpyAsync(saveX.p, kx.p, sizeof(float4) * N, cudaMemcpyDeviceToDevice, stream));
      BCK(cudaMemcpyAsync(saveV.p, kv.p, sizeof(float4) * N, cudaMemcpyDeviceToDevice, stream));
      BCK(cudaMemcpyAsync(saveC.p, kc.p, sizeof(dcu::Contact) * N, cudaMemcpyDeviceToDevice, stream));
      BCK(cudaMemcpyAsync(saveG.p, kg.p, sizeof(dcu::Garment) * G, cudaMemcpyDeviceToDevice, stream));
      BCK(cudaMemcpyAsync(saveSeam.p, ks.p, sizeof(dcu::Seam) * seam.n, cudaMemcpyDeviceToDevice, stream));
      BCK(cudaStreamSynchronize(stream));
    }
    saved = wasSaved;
    resetCounters();
    drape_batch_tuning t = tuning();
    t.variants_timed = timed;
    t.ms_per_newton = bestMs;
    return t;
  }

  void setTuning(drape_batch_tuning& t) {
    int found = -1;
    for (int vi = 0; vi < kVariantCount; ++vi)
      if (kVariants[vi].rowLanes == t.row_lanes && kVariants[vi].threads == t.block_threads) found = vi;
    if (found < 0) throw std::invalid_argument("row_lanes must be 0, 2, 4 or 8 and block_threads 256, 512 or 1024");
    use();
    if (built) setVariant(found); else variant = found;
    dropGraph();
    t = tuning();
    t.variants_timed = 0;
    t.ms_per_newton = 0;
  }

  void resetCounters() {
    use();
    std::vector<dcu::Control> c(G);
    BCK(cudaMemcpyAsync(c.data(), ctl.p, sizeof(dcu::Control) * G, cudaMemcpyDeviceToHost, stream));
    BCK(cudaStreamSynchronize(stream));
    for (auto& x : c) {
      x.substeps = x.newtonIterations = x.cgIterations = x.lineSearchHalvings = x.energyEvaluations = 0;
      x.learnedSolves = x.precondFallbacks = x.pcgNs = 0;
    }
    BCK(cudaMemcpyAsync(ctl.p, c.data(), sizeof(dcu::Control) * G, cudaMemcpyHostToDevice, stream));
    BCK(cudaStreamSynchronize(stream));
  }

  drape_counters countersOf(uint32_t g) {
    use();
    dcu::Control c{};
    BCK(cudaMemcpyAsync(&c, ctl.p + g, sizeof(c), cudaMemcpyDeviceToHost, stream));
    BCK(cudaStreamSynchronize(stream));
    drape_counters out{};
    out.substeps = c.substeps;
    out.newton_iterations = c.newtonIterations;
    out.cg_iterations = c.cgIterations;
    out.line_search_halvings = c.lineSearchHalvings;
    out.precond_fallbacks = c.precondFallbacks;
    out.learned_solves = c.learnedSolves;
    out.pcg_nanoseconds = c.pcgNs;
    return out;
  }

  // Algorithmic bytes of the solve launches since the counters' last reset (the PCG and energy-pass figures).
  double pcgBytes(int64_t* cg) {
    use();
    std::vector<dcu::Control> c(G);
    BCK(cudaMemcpyAsync(c.data(), ctl.p, sizeof(dcu::Control) * G, cudaMemcpyDeviceToHost, stream));
    BCK(cudaStreamSynchronize(stream));
    double bytes = 0;
    int64_t total = 0;
    for (uint32_t g = 0; g < G; ++g) {
      const Model& m = models[g];
      const double n = static_cast<double>(m.x.size()), slots = static_cast<double>(m.colIndex.size());
      const double pcg = 40.0 * slots + 200.0 * n;
      const double energy = 48.0 * m.stretch.size() + 32.0 * m.hinges.size() + 16.0 * m.seams.size() + 96.0 * n;
      bytes += c[g].cgIterations * pcg + c[g].energyEvaluations * energy;
      total += c[g].cgIterations;
    }
    if (cg) *cg = total;
    return bytes;
  }
};

// ---------------------------------------------------------------------------------------------------------------
// C ABI

namespace {

template <class F>
int bguarded(const drape_batch* cb, F&& f) {
  auto* b = const_cast<drape_batch*>(cb);
  try {
    f();
    return DRAPE_OK;
  } catch (const std::invalid_argument& e) {
    (b ? b->error : g_batchError) = e.what();
    return DRAPE_INVALID;
  } catch (const std::out_of_range& e) {
    (b ? b->error : g_batchError) = e.what();
    return DRAPE_OUT_OF_RANGE;
  } catch (const std::logic_error& e) {
    (b ? b->error : g_batchError) = e.what();
    return DRAPE_NOT_BUILT;
  } catch (const std::exception& e) {
    (b ? b->error : g_batchError) = e.what();
    return DRAPE_DEVICE_ERROR;
  }
}

void needBatch(const drape_batch* b) {
  if (!b) throw std::invalid_argument("null batch handle");
}

}  // namespace

extern "C" {

int drape_batch_create(int device, drape_batch** out) {
  return bguarded(nullptr, [&] {
    if (!out) throw std::invalid_argument("null argument");
    *out = new drape_batch(device);
  });
}

void drape_batch_destroy(drape_batch* b) { delete b; }

const char* drape_batch_last_error(const drape_batch* b) { return b ? b->error.c_str() : g_batchError.c_str(); }

int drape_batch_add(drape_batch* b, const drape_scene_desc* scene, uint32_t* index) {
  return bguarded(b, [&] {
    needBatch(b);
    if (!scene) throw std::invalid_argument("null scene");
    b->add(*scene);
    if (index) *index = static_cast<uint32_t>(b->models.size() - 1);
  });
}

int drape_batch_build(drape_batch* b) {
  return bguarded(b, [&] {
    needBatch(b);
    b->build();
  });
}

int drape_batch_set_precond(drape_batch* b, drape_precond* p) {
  return bguarded(b, [&] {
    needBatch(b);
    b->use();
    b->setPrecond(p);
  });
}

int drape_batch_autotune(drape_batch* b, int frames, drape_batch_tuning* out) {
  return bguarded(b, [&] {
    needBatch(b);
    const drape_batch_tuning t = b->autotune(frames);
    if (out) *out = t;
  });
}

int drape_batch_set_tuning(drape_batch* b, drape_batch_tuning* tuning) {
  return bguarded(b, [&] {
    needBatch(b);
    if (!tuning) throw std::invalid_argument("null argument");
    b->setTuning(*tuning);
  });
}

int drape_batch_step(drape_batch* b, double dt, int substeps, int iterations) {
  return bguarded(b, [&] {
    needBatch(b);
    b->advance(dt, substeps, iterations);
  });
}

int drape_batch_set_phase(drape_batch* b, uint32_t index, int phase) {
  return bguarded(b, [&] {
    needBatch(b);
    b->setPhase(index, phase);
  });
}

int drape_batch_drape_to_rest(drape_batch* b, const drape_drape_options* options, drape_drape_result* results,
                              double* settle_seconds, uint32_t count) {
  return bguarded(b, [&] {
    needBatch(b);
    b->requireBuilt();
    if (!results || count != b->G) throw std::invalid_argument("results must hold one entry per garment");
    drape_drape_options o{};
    if (options) {
      o = *options;
    } else {
      o.substeps = 1;
      o.iterations = 2;
      o.frame_dt = 1.0 / 60.0;
      o.max_assembly_seconds = 3.0;
      o.seam_gap_done = 0.001;
      o.settle_rms_speed = 0.002;
      o.settle_hold_frames = 60;
      o.max_sim_seconds = 20.0;
      o.snapshot_every = 30;
      o.max_retries = 3;
      o.energy_rise_frames = 60;
      o.frames_per_wait = 1;
    }
    if (o.frame_dt <= 0 || o.snapshot_every < 1 || o.substeps < 1)
      throw std::invalid_argument("frame_dt, substeps and snapshot_every must be positive");
    b->drapeToRest(o, results, settle_seconds);
  });
}

int drape_batch_size(const drape_batch* b, uint32_t* garments, uint64_t* particles, uint64_t* block_slots) {
  return bguarded(b, [&] {
    needBatch(b);
    uint64_t n = 0, s = 0;
    for (const auto& m : b->models) {
      n += m.x.size();
      s += m.colIndex.size();
    }
    if (garments) *garments = static_cast<uint32_t>(b->models.size());
    if (particles) *particles = n;
    if (block_slots) *block_slots = s;
  });
}

int drape_batch_particle_count(const drape_batch* b, uint32_t index, uint32_t* count) {
  return bguarded(b, [&] {
    needBatch(b);
    if (index >= b->models.size()) throw std::out_of_range("no such garment in the batch");
    if (!count) throw std::invalid_argument("null argument");
    *count = static_cast<uint32_t>(b->models[index].x.size());
  });
}

int drape_batch_read_positions(const drape_batch* cb, uint32_t index, float* out, size_t count) {
  return bguarded(cb, [&] {
    needBatch(cb);
    auto* b = const_cast<drape_batch*>(cb);
    b->requireBuilt();
    if (index >= b->G) throw std::out_of_range("no such garment in the batch");
    const size_t n = b->models[index].x.size();
    if (count != n || !out) throw std::invalid_argument("readPositions: span size must equal the garment's particle count");
    b->use();
    std::vector<float4> tmp(n);
    if (n) {
      BCK(cudaMemcpyAsync(tmp.data(), b->x.p + b->pBase[index], sizeof(float4) * n, cudaMemcpyDeviceToHost,
                          b->stream));
      BCK(cudaStreamSynchronize(b->stream));
    }
    for (size_t i = 0; i < n; ++i) {
      out[3 * i] = tmp[i].x;
      out[3 * i + 1] = tmp[i].y;
      out[3 * i + 2] = tmp[i].z;
    }
  });
}

int drape_batch_stats(drape_batch* b, uint32_t index, drape_stats* out) {
  return bguarded(b, [&] {
    needBatch(b);
    b->requireBuilt();
    if (index >= b->G) throw std::out_of_range("no such garment in the batch");
    if (!out) throw std::invalid_argument("null argument");
    b->use();
    b->refreshStats();
    *out = b->statsOf(index);
  });
}

int drape_batch_counters(const drape_batch* cb, uint32_t index, drape_counters* out) {
  return bguarded(cb, [&] {
    needBatch(cb);
    auto* b = const_cast<drape_batch*>(cb);
    b->requireBuilt();
    if (index >= b->G) throw std::out_of_range("no such garment in the batch");
    if (!out) throw std::invalid_argument("null argument");
    *out = b->countersOf(index);
  });
}

int drape_batch_reset_counters(drape_batch* b) {
  return bguarded(b, [&] {
    needBatch(b);
    b->requireBuilt();
    b->resetCounters();
  });
}

int drape_batch_save(drape_batch* b) {
  return bguarded(b, [&] {
    needBatch(b);
    b->save();
  });
}

int drape_batch_restore(drape_batch* b) {
  return bguarded(b, [&] {
    needBatch(b);
    b->restore();
  });
}

int drape_batch_set_profiling(drape_batch* b, int enable) {
  return bguarded(b, [&] {
    needBatch(b);
    b->profiling = enable != 0;
    b->prof = drape_batch_profile{};
  });
}

int drape_batch_profile_read(const drape_batch* cb, drape_batch_profile* out) {
  return bguarded(cb, [&] {
    needBatch(cb);
    if (!out) throw std::invalid_argument("null argument");
    auto* b = const_cast<drape_batch*>(cb);
    *out = b->prof;
    out->kernel_launches += b->prof.graph_launches * b->graphLaunchesPerFrame;
    if (b->built) out->pcg_bytes = b->pcgBytes(&out->cg_iterations);
  });
}

int drape_batch_stream(const drape_batch* b, void** stream) {
  return bguarded(b, [&] {
    needBatch(b);
    if (!stream) throw std::invalid_argument("null argument");
    *stream = static_cast<void*>(b->stream);
  });
}

}  // extern "C"
