// Device data layout and kernels of one implicit-Euler substep (predict / contact setup, contact activation,
// term records and slot-parallel assembly, persistent PCG + line search, finish), plus statistics.
//
// Reference algorithm: CpuSolver::Impl::substep (libs/sim/src/cpu_solver.cpp:230-314) in the displacement form of the
// reference's 32-bit GPU path (u = x - xStart, term positions relative to the term's first vertex;
// libs/sim/kernels/kernels.h:30-448). Per Newton iteration this file runs four launches instead of the reference's
// ~40 + 13 per CG iteration dispatches with host round trips (gpu_solver_core.cpp:325-407):
//   k_activate   contact activation (kernels.h:85-99)
//   k_terms      every stretch and hinge term evaluated once into a derivative record (kernels.h:137-176)
//   k_assemble   each 3x3 Hessian block summed by the thread that owns its slot from the records of the row's incident
//                terms; the diagonal slot's thread adds the gradient, block-Jacobi inverse and contact release
//                (replaces the contribution buffers + gather, kernels.h:104-231)
//   k_solve      one cooperative persistent launch: PCG (kernels.h:237-347), contact force, FP64 Newton slope, FP64
//                line search and step application (cpu_solver.cpp:264-283) with device-side decisions.
#pragma once

#include <cuda/atomic>
#include <cstdint>

#include "device_math.cuh"

namespace dcu {

constexpr int kWarp = 32;
constexpr int kAssembleThreads = 256;  // k_assemble block size (one thread per block slot)
constexpr int kRowLanes = 2;        // lanes per block row in the single solver's SpMV
constexpr int kSolveThreads = 1024; // k_solve block size (one block per SM)
constexpr uint32_t kPinnedBit = 0x80000000u;
constexpr uint32_t kSmemSlotBytes = 40;      // one block slot in shared memory: 9 floats + a column index
constexpr int kPartialStride = 4;   // doubles per block in the partials array

struct Particle {
  float mass;
  uint32_t fabric, garment, pinned;
};

struct Fabric {
  float k[3];       // stretch warp, weft, bias
  float limit[2];   // strain limits
  float thickness, friction, damping;
};

struct Stretch {
  uint32_t v[3];
  uint32_t fabric;
  float4 d;  // dmInv (0,0), (1,0), (0,1), (1,1)
  float area;
  float pad[3];
};

struct Hinge {
  uint32_t v[4];
  float K, rest;
  float pad[2];
};

struct Seam {
  uint32_t a, b, garment;
  float startGap;
};

struct Contact {
  float4 normal;  // xyz: plane normal, w: offset = r - phi(xStart)
  float force, frictionLambda;
  uint32_t nearBody, active;
};

struct Garment {
  int32_t phase;  // 0 Assembling, 1 Settling
  int32_t pad;
  double assemblyTime;
};

// Device control block: the PCG / Newton scalars every block of k_solve recomputes identically, plus counters.
struct Control {
  int newtonDone;   // this substep's Newton loop has stopped (slope >= 0 or max move < 1e-9)
  int error;        // 1: a grid barrier gave up waiting; 2: a row exceeded the assembly capacity; 4: a block's sliced
                    // matrix exceeded its shared memory (k_solve_rows)
  unsigned long long barrierArrivals;
  long long cgIterations, newtonIterations, lineSearchHalvings, substeps, energyEvaluations;
  double lastAlpha, lastSlope, lastE0, lastMaxMove;
  int lastCg;
  int pad;
  long long learnedSolves, precondFallbacks;  // PCG solves with the learned preconditioner; of those, restarted
  long long pcgNs;  // %globaltimer nanoseconds inside the PCG solves (block 0's view: CG init to the last iteration)
  unsigned long long frameBeginNs;  // %globaltimer at the current frame's first kernel (0: not started)
};

constexpr unsigned int kCgLogCapacity = 1u << 16;  // PCG iterations per Newton iteration, ring buffer

struct Params {
  float h, invH2;
  float gravity[3];
  float limitScale, seamStiffness, closingSpeed, frictionSlip, collisionOffset, dampingScale, assemblyExtraDamping;
  float contactReach, contactSnap;
  double hD, cgTolerance;
  int maxCg;
  uint32_t n, nStretch, nHinge, nSeam, nBlocks, nGarments, slotsPadded;
  uint32_t smemSlots;   // k_solve: block slots a block keeps in shared memory
  int learnedSwitch;    // k_solve<true>: block-Jacobi iterations before the learned preconditioner takes over
  int pcgVariant;       // the block-Jacobi PCG form: 0 reference order (resident rows where the scene fits), 1 pipelined,
                        // 2 Chronopoulos-Gear, 3 reference order on the 1024-thread kernel (kept in the view so that
                        // captured frame graphs are recaptured when it changes)
  uint32_t slicedSlots; // k_solve_rows: padded slots of the sliced layout a block may hold in shared memory
  unsigned long long barrierLimitNs;
};

struct Dev {
  Params P;
  FieldInfo field;
  double fieldOrigin[3], fieldCell;
  const float* fieldValues;
  const Particle* particle;
  const Fabric* fabric;
  Garment* garment;
  const Stretch* stretch;
  const Hinge* hinge;
  const Seam* seam;
  const uint32_t* rowStart;
  const uint32_t* colIndex;  // bit 31: the column's particle is pinned
  const uint32_t* diagSlot;
  const uint32_t* incStart;
  const uint32_t* incEntry;
  const uint32_t* offSlot;   // the off-diagonal slots in slot order: row << 6 | row-local position
  const uint32_t* offStart;  // per off-diagonal slot: its contributions [offStart[k], offStart[k + 1]) of offCode
  const uint32_t* offCode;     // per contribution, in gather order: kind << 30 | term << 4 | vertex a << 2 | block b
  float4 *x, *v, *xStart, *yRel, *u, *grad, *step, *r, *z, *p0, *p1, *ap, *apFull, *resid;
  float4 *pm0, *pm1, *pz;  // pipelined PCG only: the two m = M w buffers and z = A q (null where not allocated)
  float4* stretchDer;      // per stretch term: its StretchDer record (6 float4), written by termsRows
  float4* hingeDer;        // per hinge term: its HingeDer record (4 float4)
  const float* Lf;         // learned factor L: 9 planes of slotsPadded floats on lower slots (k_solve<true>)
  const uint32_t* tslot;   // slot of (j, i) for slot (i, j)
  const float4* LfRows;    // the factor by rows, three float4 a slot: L_ij at lower slots, L_ji at upper (i, j)
  const float4* fExt;
  const float4* pinPos;
  float* blocks;   // 9 planes of slotsPadded floats, component 3*row+col
  float4* precond; // 3 float4 (rows) per particle
  Contact* contact;
  double* partials;
  Control* ctl;
  int* cgLog;  // kCgLogCapacity entries
};

// ---------------------------------------------------------------------------------------------------------------
// Synchronisation of a group of co-resident blocks for the cooperative persistent kernels (cooperative launch
// guarantees co-residency). A group is the whole grid for one solver, or the blocks a batched launch gives one
// garment: `rank` is the block's index in its group and `size` the group's block count.
//
// Arrivals only ever increase: a launch's k-th barrier completes when the counter reaches base + k * size, base
// being the counter at the launch's start rounded down to a multiple of size (no barrier can complete before
// every block has arrived, so a block that reads the counter late still rounds to the same base). Thread 0 adds its
// block's arrival with release semantics after publishing the block's partial sums and polls with acquire loads; a
// time limit turns a lost block into an error status and a return instead of a hang.
//
// Reductions alternate between two halves of the group's partials array, so a block that has already passed a
// barrier and publishes its next partial cannot overwrite values a slower block is still summing.

__device__ __forceinline__ unsigned long long globalTimerNs() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

struct GridSync {
  Control* ctl;
  unsigned long long target, limitNs;
  unsigned int parity;
  uint32_t rank, size;

  __device__ void init(Control* c, unsigned long long lim, uint32_t rank_, uint32_t size_) {
    __shared__ unsigned long long base;
    if (threadIdx.x == 0) {
      cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> a(c->barrierArrivals);
      const unsigned long long now = a.load(cuda::memory_order_relaxed);
      base = now - now % size_;
    }
    __syncthreads();
    ctl = c;
    target = base;
    limitNs = lim;
    parity = 0;
    rank = rank_;
    size = size_;
  }
  // The whole grid as one group.
  __device__ void init(Control* c, unsigned long long lim) { init(c, lim, blockIdx.x, gridDim.x); }

  // One thread's arrival for the whole block (release: the block's writes before it, ordered by the caller, become
  // visible) and its bounded wait for the group (acquire). The caller advances `target` first. Returns 0 when the
  // limit ran out or another block raised the error flag.
  __device__ int arriveAndWait() const {
    unsigned long long* counter = &ctl->barrierArrivals;
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(counter), "l"(1ull) : "memory");
    unsigned int spins = 0;
    const unsigned long long start = globalTimerNs();
    for (;;) {
      unsigned long long seen;
      asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(seen) : "l"(counter) : "memory");
      if (seen >= target) return 1;
      if ((++spins & 31u) == 0) {
        if (*reinterpret_cast<volatile int*>(&ctl->error) != 0) return 0;
        if (globalTimerNs() - start > limitNs) {
          atomicExch(&ctl->error, 1);
          return 0;
        }
      }
    }
  }

  // A barrier of the whole group (no data).
  __device__ bool sync() {
    __shared__ int ok;
    target += size;
    __syncthreads();
    if (threadIdx.x == 0) ok = arriveAndWait();
    __syncthreads();
    return ok != 0;
  }
};

// Block-wide FP64 sums (or maxima); thread 0 gets the result in out. Fixed tree shape, so deterministic.
template <int K, bool Max = false>
__device__ inline void blockReduce(double (&v)[K], double* out) {
  __shared__ double red[K][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, v[k], o);
      v[k] = Max ? fmax(v[k], y) : v[k] + y;
    }
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k][w] = v[k];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = lane < nw ? red[k][lane] : (Max ? -INFINITY : 0.0);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double y = __shfl_down_sync(0xffffffffu, s, o);
        s = Max ? fmax(s, y) : s + y;
      }
      if (lane == 0) out[k] = s;
    }
  }
}

template <int K>
__device__ inline void blockSum(double (&v)[K], double* out) {
  blockReduce<K, false>(v, out);
}

// a + b, or the larger of the two.
template <bool Max>
__device__ __forceinline__ double combine(double a, double b) {
  return Max ? fmax(a, b) : a + b;
}

// Grid-wide FP64 sums (or maxima). The warps' sums meet in shared memory; warp 0 combines them, publishes the block
// total, arrives at the group barrier and waits, then reads every block's total (lane l: blocks l, l + 32, ..., all
// loads issued before the first add) and combines them in a fixed order; the other warps wait at one block barrier
// meanwhile. Every block obtains bit-identical results and takes the same branches. Two block barriers per call: `red`
// is rewritten only after the closing barrier, by which warp 0 has read it, and `res` only after the next call's first
// barrier, by which every warp has read it; so every call shares one scratch. Returns false when the barrier gave up.
struct ReduceScratch {
  double red[3][32];  // per-warp sums (at most three values, 32 warps)
  double res[3];
  int ok;
};

__device__ __forceinline__ ReduceScratch& reduceScratch() {
  __shared__ ReduceScratch r;
  return r;
}

// The grid stage: the caller has put nw per-warp sums in red and passed a block barrier.
template <int K, bool Max>
__device__ inline bool gridCombine(const Dev& D, GridSync& gs, int nw, double (&out)[K]) {
  static_assert(K >= 1 && K <= 3, "gridReduce: one to three values");
  constexpr int kLoads = 5;  // partials a lane loads at a time (160 blocks per round: one round for one block per SM)
  constexpr double kIdentity = Max ? -INFINITY : 0.0;
  ReduceScratch& sc = reduceScratch();
  double* half = D.partials + static_cast<size_t>(gs.parity) * gs.size * kPartialStride;
  gs.parity ^= 1u;
  gs.target += gs.size;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (w == 0) {
    double s[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      s[k] = lane < nw ? sc.red[k][lane] : kIdentity;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s[k] = combine<Max>(s[k], __shfl_down_sync(0xffffffffu, s[k], o));
    }
    int good = 0;
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) half[gs.rank * kPartialStride + k] = s[k];
      good = gs.arriveAndWait();
    }
    good = __shfl_sync(0xffffffffu, good, 0);
    __syncwarp();  // the other lanes' reads below follow lane 0's acquire
    if (good) {
      double t[K];
#pragma unroll
      for (int k = 0; k < K; ++k) t[k] = kIdentity;
      for (unsigned int b0 = 0; b0 < gs.size; b0 += 32 * kLoads) {
        double x[kLoads][K];
#pragma unroll
        for (int j = 0; j < kLoads; ++j) {
          const unsigned int b = b0 + 32 * j + lane;
#pragma unroll
          for (int k = 0; k < K; ++k) x[j][k] = b < gs.size ? __ldcg(half + b * kPartialStride + k) : kIdentity;
        }
#pragma unroll
        for (int j = 0; j < kLoads; ++j)
#pragma unroll
          for (int k = 0; k < K; ++k) t[k] = combine<Max>(t[k], x[j][k]);
      }
#pragma unroll
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t[k] = combine<Max>(t[k], __shfl_down_sync(0xffffffffu, t[k], o));
      if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) sc.res[k] = t[k];
    }
    if (lane == 0) sc.ok = good;
  }
  __syncthreads();
  if (!sc.ok) return false;
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = sc.res[k];
  return true;
}

// HalfWarps (blocks of at most 512 threads): each half-warp is summed on its own (a 16-lane tree) into its own entry
// of `red`, so 16 rows per entry as in a 1024-thread block whose rows sit on even lanes (pcgReferenceOrder<2>'s p.Ap
// partials): that block's tree with zeros on its odd lanes adds the same values in the same order.
template <int K, bool Max = false, bool HalfWarps = false>
__device__ inline bool gridReduce(const Dev& D, GridSync& gs, double (&v)[K], double (&out)[K]) {
  ReduceScratch& sc = reduceScratch();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = HalfWarps ? 2 * ((blockDim.x + 31) >> 5) : (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = HalfWarps ? 8 : 16; o > 0; o >>= 1)
      v[k] = combine<Max>(v[k], __shfl_down_sync(0xffffffffu, v[k], o, HalfWarps ? 16 : 32));
  if (HalfWarps ? (lane & 15) == 0 : lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sc.red[k][HalfWarps ? 2 * w + (lane >> 4) : w] = v[k];
  __syncthreads();
  return gridCombine<K, Max>(D, gs, nw, out);
}

// Sums for a block that stands for one twice its size (at most 512 threads for 1024): thread t carries virtual
// threads t (lo) and t + blockDim.x (hi), so warp w's lo sums are virtual warp w's and its hi sums virtual warp
// w + nw's, in the order a block of the virtual size adds them.
template <int K>
__device__ inline bool gridReducePairs(const Dev& D, GridSync& gs, double (&lo)[K], double (&hi)[K],
                                       double (&out)[K]) {
  ReduceScratch& sc = reduceScratch();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] += __shfl_down_sync(0xffffffffu, lo[k], o);
      hi[k] += __shfl_down_sync(0xffffffffu, hi[k], o);
    }
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) {
      sc.red[k][w] = lo[k];
      sc.red[k][w + nw] = hi[k];
    }
  __syncthreads();
  return gridCombine<K, false>(D, gs, 2 * nw, out);
}

// Block `rank`'s contiguous share of [0, n) in a group of `size` blocks: the persistent kernels give each block one
// range of rows, so the neighbour gathers of the SpMV mostly hit rows the same block (hence the same SM's L1) just
// touched.
__device__ __forceinline__ void blockRange(uint32_t n, uint32_t rank, uint32_t size, uint32_t& r0, uint32_t& r1) {
  const uint32_t per = (n + size - 1) / size;
  r0 = min(n, rank * per);
  r1 = min(n, r0 + per);
}

__device__ __forceinline__ float3 filterContact(const Contact& c, float3 v) {
  if (c.active == 0u) return v;
  const float3 n = xyz(c.normal);
  return v - n * dot(n, v);
}

// The PCG's FP32 arithmetic with every rounding written out (products and sums fused or rounded explicitly, nothing
// left to the compiler's contraction), so that the reference-order kernels (pcgReferenceOrder over 1024-thread blocks,
// pcgResidentRows over 512-thread ones) round alike in whatever code surrounds them.
__device__ __forceinline__ float3 axpyRn(float3 x, float s, float3 y) {  // y + s x, one rounding per component
  return mk(__fmaf_rn(x.x, s, y.x), __fmaf_rn(x.y, s, y.y), __fmaf_rn(x.z, s, y.z));
}
__device__ __forceinline__ float dotRn(float a0, float a1, float a2, float3 b) {
  return __fmaf_rn(a2, b.z, __fmaf_rn(a1, b.y, __fmul_rn(a0, b.x)));
}
__device__ __forceinline__ float3 mulRn(const M3& a, float3 v) {
  return mk(dotRn(a.m[0], a.m[1], a.m[2], v), dotRn(a.m[3], a.m[4], a.m[5], v), dotRn(a.m[6], a.m[7], a.m[8], v));
}
// v - n (n . v) on active contact rows.
__device__ __forceinline__ float3 filterRn(const Contact& c, float3 v) {
  if (c.active == 0u) return v;
  const float3 n = xyz(c.normal);
  return axpyRn(n, -dotRn(n.x, n.y, n.z, v), v);
}
// acc += a v for a row-major 3x3 block a: each row's three products summed in order, then added to acc.
__device__ __forceinline__ void blockMulAddRn(float3& acc, const float (&a)[9], float3 v) {
  acc.x = __fadd_rn(acc.x, dotRn(a[0], a[1], a[2], v));
  acc.y = __fadd_rn(acc.y, dotRn(a[3], a[4], a[5], v));
  acc.z = __fadd_rn(acc.z, dotRn(a[6], a[7], a[8], v));
}

__device__ __forceinline__ float contactRadius(const Params& P, const Fabric& f) {
  return __fadd_rn(P.collisionOffset, __fmul_rn(0.5f, f.thickness));
}

__device__ __forceinline__ float3 ld3(const float4* p, uint32_t i) { return xyz(p[i]); }

__device__ __forceinline__ float seamTarget(const Dev& D, const Seam& s) {
  const Garment g = D.garment[s.garment];
  if (g.phase != 0) return 0.0f;
  return fmaxf(0.0f, s.startGap - D.P.closingSpeed * static_cast<float>(g.assemblyTime));
}

// ---------------------------------------------------------------------------------------------------------------
// Substep setup: predict (kernels.h:34-51) and contact setup (kernels.h:55-82).

__device__ inline void contactSetupOne(const Dev& D, uint32_t i, float3 xs, Contact& c) {
  const float lastForce = c.force;
  c.nearBody = 0u;
  c.active = 0u;
  c.frictionLambda = 0.0f;
  c.force = 0.0f;
  const Particle pa = D.particle[i];
  if (D.field.present && pa.pinned == 0u) {
    const float radius = contactRadius(D.P, D.fabric[pa.fabric]);
    const float phi = fieldSample(D.fieldValues, D.field, xs);
    if (phi < __fadd_rn(radius, D.P.contactReach)) {
      const float3 normal = fieldGradient(D.fieldValues, D.field, xs);
      if (!isZero(normal)) {
        c.nearBody = 1u;
        c.normal = f4(normal, __fsub_rn(radius, phi));
        c.frictionLambda = lastForce;
      }
    }
  }
}

// The point kernels' bodies take the block's rank in the blocks that cover the solver (the grid, or a garment's
// share of a batched launch) and that share's size.
__device__ inline void beginRows(const Dev& D, uint32_t rank, uint32_t size) {
  if (rank == 0 && threadIdx.x == 0) {
    D.ctl->newtonDone = 0;
    D.ctl->substeps += 1;
  }
  const float h = D.P.h;
  for (uint32_t i = rank * blockDim.x + threadIdx.x; i < D.P.n; i += size * blockDim.x) {
    const float4 x4 = D.x[i];
    D.xStart[i] = x4;
    const Particle pa = D.particle[i];
    if (pa.pinned != 0u) {
      D.yRel[i] = make_float4(0, 0, 0, 0);
      D.u[i] = make_float4(0, 0, 0, 0);
    } else {
      const float3 vel = ld3(D.v, i);
      const float3 g = D.garment[pa.garment].phase == 1 ? mk(D.P.gravity[0], D.P.gravity[1], D.P.gravity[2]) : mk(0, 0, 0);
      const float3 acc = g + div(ld3(D.fExt, i), pa.mass);
      D.yRel[i] = f4(vel * h + acc * (h * h));
      D.u[i] = f4(vel * h);
    }
    Contact c = D.contact[i];
    contactSetupOne(D, i, xyz(x4), c);
    D.contact[i] = c;
  }
}

// Holds near particles on their plane for this Newton iteration, projecting any below it (kernels.h:85-99).
__device__ inline void activateRows(const Dev& D, uint32_t rank, uint32_t size) {
  if (D.ctl->newtonDone) return;
  for (uint32_t i = rank * blockDim.x + threadIdx.x; i < D.P.n; i += size * blockDim.x) {
    Contact c = D.contact[i];
    if (c.nearBody == 0u) continue;
    const float3 n = xyz(c.normal);
    float3 ui = ld3(D.u, i);
    const float gap = c.normal.w - dot(n, ui);
    if (gap > -D.P.contactSnap) c.active = 1u;
    if (c.active != 0u && gap > 0.0f) {
      ui += n * gap;
      D.u[i] = f4(ui);
    }
    D.contact[i].active = c.active;
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Assembly in two passes. termsRows evaluates every stretch and hinge term once into a derivative record;
// assembleSlots then gives every block slot (i, j) one thread, which adds block (a, b) of each incident term that
// couples i (its vertex a) with j (its vertex b), formed from the term's record, in row i's incidence order (the
// reference's fixed gather order, gpu_solver_core.cpp:184-224). The diagonal slot walks row i's whole incidence list
// (every entry's block (a, a)) after the particle's own inertia and friction term and also sums the row's gradient;
// an off-diagonal slot walks its own contribution list (the reference's per-slot gather list). Deterministic, no
// atomics, no shared memory.

__device__ inline float3 relPos(const Dev& D, uint32_t v0, uint32_t vk) {
  return (ld3(D.xStart, vk) - ld3(D.xStart, v0)) + ld3(D.u, vk);
}

__device__ inline StretchIn stretchIn(const Dev& D, const Stretch& t) {
  const Fabric f = D.fabric[t.fabric];
  StretchIn s;
  s.d = t.d;
  s.area = t.area;
  s.k[0] = f.k[0];
  s.k[1] = f.k[1];
  s.k[2] = f.k[2];
  s.limit[0] = f.limit[0];
  s.limit[1] = f.limit[1];
  s.limitScale = D.P.limitScale;
  return s;
}

// Per-term derivative records of one Newton iteration (every stretch and hinge term evaluated once, one thread per
// term); the assembly then forms each incident row from them.
__device__ inline void termsRows(const Dev& D, uint32_t rank, uint32_t size) {
  if (D.ctl->newtonDone) return;
  const uint32_t S = D.P.nStretch, total = S + D.P.nHinge;
  for (uint32_t idx = rank * blockDim.x + threadIdx.x; idx < total; idx += size * blockDim.x) {
    if (idx < S) {
      const Stretch t = D.stretch[idx];
      float3 x[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) x[k] = relPos(D, t.v[0], t.v[k]);
      StretchDer o;
      stretchDerivs(stretchIn(D, t), x, o);
#pragma unroll
      for (int k = 0; k < 6; ++k) D.stretchDer[6ull * idx + k] = o.w[k];
    } else {
      const uint32_t h = idx - S;
      const Hinge t = D.hinge[h];
      float3 x[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) x[k] = relPos(D, t.v[0], t.v[k]);
      HingeDer o;
      hingeDerivs(t.K, t.rest, x, o);
#pragma unroll
      for (int k = 0; k < 4; ++k) D.hingeDer[4ull * h + k] = o.w[k];
    }
  }
}

// Block (a, b) of the term an incidence entry names, and with Grad the gradient of its vertex a (seam springs, a few
// hundred per garment, are evaluated here; stretch and hinge terms come from their records).
template <bool Grad>
__device__ inline void entryBlock(const Dev& D, uint32_t code, int b, float3& g, M3& H) {
  const uint32_t kind = code >> 30, term = (code >> 2) & 0x0FFFFFFFu;
  const int a = static_cast<int>(code & 3u);
  if (kind == 0) {
    stretchBlockFrom<Grad>(D.stretch[term].d, D.stretchDer + 6ull * term, a, b, g, H);
  } else if (kind == 1) {
    hingeBlockFrom<Grad>(D.hingeDer + 4ull * term, a, b, g, H);
  } else {
    const Seam sp = D.seam[term];
    M3 H2[2];
    seamRow(D.P.seamStiffness, seamTarget(D, sp), ld3(D.u, sp.a), relPos(D, sp.a, sp.b), a, g, H2);
    H = b == 0 ? H2[0] : H2[1];
  }
}

// Diagonal slot of row i: the particle's own inertia and friction term, then block (a, a) of every incident entry
// (vertex a of an entry is i itself); also the row's gradient, the block-Jacobi inverse and the contact release.
__device__ inline void diagonalSlot(const Dev& D, uint32_t i, uint32_t SP) {
  const uint32_t s = D.diagSlot[i];
  const Particle pa = D.particle[i];
  const Contact c = D.contact[i];
  M3 acc;
  zero(acc);
  float3 gAcc = mk(0, 0, 0);
  // The particle's own term: inertia 1/2 (m/h^2)|u - yRel|^2 and friction (kernels.h:104-129).
  if (pa.pinned == 0u) {
    const float k = pa.mass * D.P.invH2;
    gAcc = (ld3(D.u, i) - ld3(D.yRel, i)) * k;
    acc.m[0] = acc.m[4] = acc.m[8] = k;
  }
  if (c.frictionLambda > 0.0f)
    frictionRow(ld3(D.u, i), xyz(c.normal), D.fabric[pa.fabric].friction * c.frictionLambda,
                D.P.frictionSlip * D.P.h, gAcc, acc);
  const uint32_t ee = D.incStart[i + 1];
  for (uint32_t e = D.incStart[i]; e < ee; ++e) {
    const uint32_t code = D.incEntry[e];
    float3 g;
    M3 H;
    entryBlock<true>(D, code, static_cast<int>(code & 3u), g, H);
#pragma unroll
    for (int k = 0; k < 9; ++k) acc.m[k] += H.m[k];
    gAcc += g;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) D.blocks[k * SP + s] = acc.m[k];
  // Block-Jacobi inverse of the diagonal block (kernels.h:237-249); zero for pinned particles.
  M3 inv;
  if (pa.pinned != 0u) {
    zero(inv);
  } else {
    bool ok = false;
    inv = invertSpd(acc, ok);
  }
  D.precond[3 * i + 0] = make_float4(inv.m[0], inv.m[1], inv.m[2], 0.0f);
  D.precond[3 * i + 1] = make_float4(inv.m[3], inv.m[4], inv.m[5], 0.0f);
  D.precond[3 * i + 2] = make_float4(inv.m[6], inv.m[7], inv.m[8], 0.0f);
  // Gradient (pinned rows zero) and contact release (kernels.h:204-231).
  const float3 gi = pa.pinned != 0u ? mk(0, 0, 0) : gAcc;
  D.grad[i] = f4(gi);
  if (c.active != 0u && dot(gi, xyz(c.normal)) < 0.0f) D.contact[i].active = 0u;
}

// Off-diagonal slot k (offSlot[k] = row << 6 | row-local position): its contributions (incidence entry, block b of
// the entry's term) in gather order.
__device__ inline void offDiagonalSlot(const Dev& D, uint32_t k, uint32_t SP) {
  const uint32_t packed = D.offSlot[k];
  const uint32_t s = D.rowStart[packed >> 6] + (packed & 63u);
  M3 acc;
  zero(acc);
  const uint32_t ce = D.offStart[k + 1];
  for (uint32_t c = D.offStart[k]; c < ce; ++c) {
    const uint32_t v = D.offCode[c];
    float3 g;
    M3 H;
    // The incidence-entry code (kind 2 bits, term 28, vertex 2) and the block.
    entryBlock<false>(D, (v & 0xC0000000u) | (((v >> 4) & 0x03FFFFFFu) << 2) | ((v >> 2) & 3u), static_cast<int>(v & 3u),
                      g, H);
#pragma unroll
    for (int q = 0; q < 9; ++q) acc.m[q] += H.m[q];
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) D.blocks[q * SP + s] = acc.m[q];
}

// Thread k of the n + (B - n) assembly threads: the diagonal slot of row k for k < n, else off-diagonal slot k - n, so
// that the diagonal slots (every incident entry) and the off-diagonal ones (a few entries each) fill separate warps.
__device__ inline void assembleSlots(const Dev& D, uint32_t rank, uint32_t size) {
  if (D.ctl->newtonDone) return;
  const uint32_t n = D.P.n, SP = D.P.slotsPadded;
  for (uint32_t k = rank * blockDim.x + threadIdx.x; k < D.P.nBlocks; k += size * blockDim.x) {
    if (k < n)
      diagonalSlot(D, k, SP);
    else
      offDiagonalSlot(D, k - n, SP);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Energy at u + alpha * step, in FP64, summed per thread over particles (inertia + friction) and terms.

// Virtual thread vt of a block of vdim threads: the elements idx = rank * vdim + vt + k * size * vdim (a kernel whose
// blocks stand for larger ones sums in the larger blocks' order).
__device__ inline double energyPartial(const Dev& D, const GridSync& gs, double alpha, uint32_t vt, uint32_t vdim) {
  double e = 0.0;
  const uint32_t n = D.P.n, S = D.P.nStretch, H = D.P.nHinge, K = D.P.nSeam;
  const uint32_t total = n + S + H + K;
  const uint32_t stride = gs.size * vdim;
  auto pos = [&](uint32_t v0, uint32_t vk) -> d3 {
    const d3 rel = toD(ld3(D.xStart, vk)) - toD(ld3(D.xStart, v0));
    return rel + (toD(ld3(D.u, vk)) + alpha * toD(ld3(D.step, vk)));
  };
  const double invH2 = 1.0 / (D.P.hD * D.P.hD);
  for (uint32_t idx = gs.rank * vdim + vt; idx < total; idx += stride) {
    if (idx < n) {
      const uint32_t i = idx;
      const Particle pa = D.particle[i];
      const d3 ui = toD(ld3(D.u, i)) + alpha * toD(ld3(D.step, i));
      if (pa.pinned == 0u) {
        const d3 dd = ui - toD(ld3(D.yRel, i));
        e += 0.5 * static_cast<double>(pa.mass) * invH2 * dotd(dd, dd);
      }
      const Contact c = D.contact[i];
      if (c.frictionLambda > 0.0f)
        e += frictionEnergy(ui, toD(xyz(c.normal)),
                            static_cast<double>(D.fabric[pa.fabric].friction) * static_cast<double>(c.frictionLambda),
                            static_cast<double>(D.P.frictionSlip) * D.P.hD);
    } else if (idx < n + S) {
      const Stretch t = D.stretch[idx - n];
      d3 x[3];
      for (int k = 0; k < 3; ++k) x[k] = pos(t.v[0], t.v[k]);
      e += stretchEnergy(stretchIn(D, t), x);
    } else if (idx < n + S + H) {
      const Hinge t = D.hinge[idx - n - S];
      d3 x[4];
      for (int k = 0; k < 4; ++k) x[k] = pos(t.v[0], t.v[k]);
      e += hingeEnergy(t.K, t.rest, x);
    } else {
      const Seam s = D.seam[idx - n - S - H];
      e += seamEnergy(D.P.seamStiffness, seamTarget(D, s), pos(s.a, s.a), pos(s.a, s.b));
    }
  }
  return e;
}

__device__ inline double energyPartial(const Dev& D, const GridSync& gs, double alpha) {
  return energyPartial(D, gs, alpha, threadIdx.x, blockDim.x);
}

// ---------------------------------------------------------------------------------------------------------------
// Persistent solve: PCG with FP64 dot products, then the Newton line search. Every block computes the same scalars
// from the same partials, so all blocks take the same branches.
//
// Each block owns a contiguous range of rows; at the start of the launch it copies its rows' blocks and column
// indices into shared memory (up to P.smemSlots slots; any excess is read from global memory), and every CG
// iteration's SpMV reads them from there.
//
// The PCG follows the reference's order (cpu_solver.cpp:169-213): two grid reductions per iteration (p.Ap, then
// r.r with r.z); the direction update p = z + beta p is folded into the next SpMV (A p = A z + beta A pPrev).

__device__ __forceinline__ M3 loadPrecond(const Dev& D, uint32_t i) {
  const float4 a = D.precond[3 * i], b = D.precond[3 * i + 1], c = D.precond[3 * i + 2];
  return M3{{a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z}};
}

__device__ __forceinline__ double dotd3(float3 a, float3 b) {
  return static_cast<double>(a.x) * b.x + static_cast<double>(a.y) * b.y + static_cast<double>(a.z) * b.z;
}

struct SmemMatrix {
  const float* planes;  // 9 planes of `stride` floats in shared memory
  const uint32_t* cols;
  uint32_t base, cap, stride, SP;  // slots [base, base + cap) are in shared memory
  const float* gblocks;
  const uint32_t* gcols;
  __device__ __forceinline__ bool local(uint32_t s) const { return s - base < cap; }
  __device__ __forceinline__ uint32_t col(uint32_t s) const {
    return local(s) ? cols[s - base] : __ldg(gcols + s);
  }
  // Row-major block at slot s.
  __device__ __forceinline__ void block(uint32_t s, float a[9]) const {
    if (local(s)) {
      const float* p = planes + (s - base);
#pragma unroll
      for (int k = 0; k < 9; ++k) a[k] = p[k * stride];
    } else {
#pragma unroll
      for (int k = 0; k < 9; ++k) a[k] = __ldg(gblocks + k * SP + s);
    }
  }
};

extern __shared__ float4 solveSmem[];

// Copies this block's slot range into shared memory (all threads; ends with a block barrier).
__device__ inline SmemMatrix stageMatrix(const Dev& D, uint32_t r0, uint32_t r1) {
  SmemMatrix A;
  const uint32_t cap = D.P.smemSlots;
  float* planes = reinterpret_cast<float*>(solveSmem);
  uint32_t* cols = reinterpret_cast<uint32_t*>(planes + 9 * cap);
  A.planes = planes;
  A.cols = cols;
  A.SP = D.P.slotsPadded;
  A.gblocks = D.blocks;
  A.gcols = D.colIndex;
  A.base = r0 < r1 ? __ldg(D.rowStart + r0) : 0;
  const uint32_t end = r0 < r1 ? __ldg(D.rowStart + r1) : 0;
  const uint32_t count = min(end - A.base, cap);
  A.stride = cap;
  A.cap = count;
  for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) {
    const uint32_t s = A.base + k;
#pragma unroll
    for (int c = 0; c < 9; ++c) planes[c * cap + k] = __ldg(D.blocks + c * A.SP + s);
    cols[k] = __ldg(D.colIndex + s);
  }
  __syncthreads();
  return A;
}

// y_i (unfiltered) = sum over unpinned columns j of A_ij x_j for row i, by RL lanes (lane `sub`), reduced over the
// lanes; x_j given by a functor. Each lane takes its slots kGatherDepth at a time: their column indices first, then
// all their x_j loads (predicated, so they are in flight together), then the products in slot order; the sums are the
// same as one slot at a time.
constexpr int kGatherDepth = 4;

template <int RL, class X>
__device__ __forceinline__ float3 rowProduct(const SmemMatrix& A, uint32_t rs, uint32_t re, int sub, unsigned mask,
                                             X&& xj) {
  float3 acc = mk(0, 0, 0);
  for (uint32_t s0 = rs + sub; s0 < re; s0 += kGatherDepth * RL) {
    uint32_t col[kGatherDepth];
#pragma unroll
    for (int k = 0; k < kGatherDepth; ++k) {
      const uint32_t s = s0 + k * RL;
      col[k] = s < re ? A.col(s) : kPinnedBit;
    }
    float3 v[kGatherDepth];
#pragma unroll
    for (int k = 0; k < kGatherDepth; ++k) v[k] = (col[k] & kPinnedBit) ? mk(0, 0, 0) : xj(col[k]);
#pragma unroll
    for (int k = 0; k < kGatherDepth; ++k) {
      if (col[k] & kPinnedBit) continue;
      float a[9];
      A.block(s0 + k * RL, a);
      blockMulAddRn(acc, a, v[k]);
    }
  }
#pragma unroll
  for (int o = RL / 2; o > 0; o >>= 1) {
    acc.x = __fadd_rn(acc.x, __shfl_xor_sync(mask, acc.x, o));
    acc.y = __fadd_rn(acc.y, __shfl_xor_sync(mask, acc.y, o));
    acc.z = __fadd_rn(acc.z, __shfl_xor_sync(mask, acc.z, o));
  }
  return acc;
}

// The PCG's product Ap for the direction p = z + beta * pPrev (p = z on the first iteration) over this block's rows
// [r0, r1). The row's product is handed to `out(i, p_i, Ap_i)` (pinned rows: Ap_i = 0; pinned columns add nothing).
// Two schemes, chosen at compile time:
//   RL > 0  RL lanes per row, the lanes' partial sums reduced by shuffles (the matrix mostly in shared memory or L2:
//           no block barriers);
//   RL = 0  slot-parallel (an HBM-resident matrix): the rows are taken kSpmvRows at a time and their slots in passes
//           of kSpmvChunk, each thread computing the products A_s p_j of consecutive slots (coalesced loads of the
//           block planes and column indices); the products are staged in shared memory and the row's thread adds
//           them in slot order.
constexpr uint32_t kSpmvRows = 128;    // slot-parallel: rows per pass (the block needs more threads than this)
constexpr uint32_t kSpmvChunk = 1024;  // slot-parallel: slot products staged per pass

struct SpmvStage {
  uint32_t rowOff[kSpmvRows + 1];
  float prod[3][kSpmvChunk];
};

// The one staging area of a block (every instantiation of directionProducts shares it; its uses never overlap).
__device__ __forceinline__ SpmvStage& spmvStage() {
  __shared__ SpmvStage st;
  return st;
}

template <int RL, class Dir, class Out>
__device__ inline void directionProducts(const Dev& D, const SmemMatrix& A, uint32_t r0, uint32_t r1, Dir&& dir,
                                         Out&& out) {
  if constexpr (RL > 0) {
    const uint32_t groups = blockDim.x / RL;
    const int sub = threadIdx.x & (RL - 1);
    const unsigned groupMask = ((1u << RL) - 1u) << ((threadIdx.x & 31) & ~(RL - 1));
    for (uint32_t i = r0 + threadIdx.x / RL; i < r1; i += groups) {
      const uint32_t rs = __ldg(D.rowStart + i), re = D.particle[i].pinned == 0u ? __ldg(D.rowStart + i + 1) : rs;
      const float3 acc = rowProduct<RL>(A, rs, re, sub, groupMask, dir);
      if (sub == 0) out(i, dir(i), acc);
    }
  } else {
    SpmvStage& st = spmvStage();
    const uint32_t t = threadIdx.x;
    for (uint32_t rr = r0; rr < r1; rr += kSpmvRows) {
      const uint32_t R = min(kSpmvRows, r1 - rr);
      const uint32_t s0 = __ldg(D.rowStart + rr);
      if (t <= R) st.rowOff[t] = __ldg(D.rowStart + rr + t) - s0;
      __syncthreads();
      const uint32_t S = st.rowOff[R];
      float3 acc = mk(0, 0, 0);
      for (uint32_t c = 0; c < S; c += kSpmvChunk) {
        const uint32_t cn = min(kSpmvChunk, S - c);
        for (uint32_t k = t; k < cn; k += blockDim.x) {
          const uint32_t s = s0 + c + k;
          const uint32_t col = A.col(s);
          float3 v = mk(0, 0, 0);
          if (!(col & kPinnedBit)) {
            float a[9];
            A.block(s, a);
            const float3 x = dir(col);
            v.x = a[0] * x.x + a[1] * x.y + a[2] * x.z;
            v.y = a[3] * x.x + a[4] * x.y + a[5] * x.z;
            v.z = a[6] * x.x + a[7] * x.y + a[8] * x.z;
          }
          st.prod[0][k] = v.x;
          st.prod[1][k] = v.y;
          st.prod[2][k] = v.z;
        }
        __syncthreads();
        if (t < R) {
          const uint32_t lo = max(st.rowOff[t], c), hi = min(st.rowOff[t + 1], c + cn);
          for (uint32_t q = lo; q < hi; ++q) {
            acc.x += st.prod[0][q - c];
            acc.y += st.prod[1][q - c];
            acc.z += st.prod[2][q - c];
          }
        }
        __syncthreads();
      }
      if (t < R) {
        const uint32_t i = rr + t;
        out(i, dir(i), D.particle[i].pinned != 0u ? mk(0, 0, 0) : acc);
      }
      __syncthreads();  // rowOff is rewritten for the next rows
    }
  }
}

// One PCG iteration's product for the direction p = z + beta * pPrev without materialising p first: the rows gather
// only z_j and add beta times their previous product A pPrev (apFull). Writes p_i (pCur), Ap_i (apFull) and the
// contact-filtered Ap_i (ap); returns this thread's share of p . filtered Ap.
template <int RL>
__device__ inline double directionStep(const Dev& D, const SmemMatrix& A, uint32_t r0, uint32_t r1,
                                       const float4* pPrev, float4* pCur, float fb, bool first) {
  double vpap = 0.0;
  directionProducts<RL>(
      D, A, r0, r1, [&](uint32_t j) { return ld3(D.z, j); },
      [&](uint32_t i, float3 zi, float3 az) {
        // A p = A z + beta A pPrev: the previous direction's product is this row's apFull.
        const float3 pi = first ? zi : axpyRn(ld3(pPrev, i), fb, zi);
        const float3 acc = first ? az : axpyRn(ld3(D.apFull, i), fb, az);
        pCur[i] = f4(pi);
        const float3 filtered = filterRn(D.contact[i], acc);
        D.apFull[i] = f4(acc);
        D.ap[i] = f4(filtered);
        vpap += dotd3(pi, filtered);
      });
  return vpap;
}

// Contact-filtered block-Jacobi PCG in the reference's order. Writes step, resid; returns the iteration count, or -1
// when a grid barrier gave up.
// At most `budget` iterations (negative: P.maxCg). *r0out gets |r0|; *finished is false only when the budget, not
// the convergence test or pAp <= 0, ended the loop.
template <int PL>
__device__ inline int pcgReferenceOrder(const Dev& D, GridSync& gs, const SmemMatrix& A, int budget = -1,
                                        double* r0out = nullptr, bool* finished = nullptr) {
  const uint32_t n = D.P.n;
  uint32_t r0i, r1i;
  blockRange(n, gs.rank, gs.size, r0i, r1i);
  // CG init (kernels.h:252-268): step = 0, resid = -grad, r = filter(resid), z = filter(M r).
  double tot[2];
  {
    double v[2] = {0.0, 0.0};
    for (uint32_t i = r0i + threadIdx.x; i < r1i; i += blockDim.x) {
      const Contact c = D.contact[i];
      const float3 res = -ld3(D.grad, i);
      const float3 ri = filterRn(c, res);
      const float3 zi = filterRn(c, mulRn(loadPrecond(D, i), ri));
      D.step[i] = make_float4(0, 0, 0, 0);
      D.resid[i] = f4(res);
      D.r[i] = f4(ri);
      D.z[i] = f4(zi);
      v[0] += dotd3(ri, zi);
      v[1] += dotd3(ri, ri);
    }
    if (!gridReduce<2>(D, gs, v, tot)) return -1;
  }
  double rz = tot[0];
  const double r0 = sqrt(tot[1]);
  if (r0out) *r0out = r0;
  bool done = !(r0 > 0.0);
  double beta = 0.0;
  float4* pPrev = D.p0;
  float4* pCur = D.p1;
  int it = 0;
  const int maxCg = budget < 0 ? D.P.maxCg : min(budget, D.P.maxCg);
  if (finished) *finished = true;
  while (!done && it < maxCg) {
    // SpMV with the direction update folded in: p_j = z_j + beta * pPrev_j.
    double vpap[1] = {directionStep<PL>(D, A, r0i, r1i, pPrev, pCur, static_cast<float>(beta), it == 0)};
    double pAp[1];
    if (!gridReduce<1>(D, gs, vpap, pAp)) return -1;
    if (!(pAp[0] > 0.0)) return it;
    const double alpha = rz / pAp[0];
    const float fa = static_cast<float>(alpha);
    ++it;
    // Update (kernels.h:304-315) fused with the preconditioner apply (kernels.h:324-332).
    double v[2] = {0.0, 0.0};
    for (uint32_t i = r0i + threadIdx.x; i < r1i; i += blockDim.x) {
      const Contact c = D.contact[i];
      const float3 pi = ld3(pCur, i);
      D.step[i] = f4(axpyRn(pi, fa, ld3(D.step, i)));
      const float3 ri = axpyRn(ld3(D.ap, i), -fa, ld3(D.r, i));
      D.r[i] = f4(ri);
      D.resid[i] = f4(axpyRn(ld3(D.apFull, i), -fa, ld3(D.resid, i)));
      const float3 zi = filterRn(c, mulRn(loadPrecond(D, i), ri));
      D.z[i] = f4(zi);
      v[0] += dotd3(ri, ri);
      v[1] += dotd3(ri, zi);
    }
    double t2[2];
    if (!gridReduce<2>(D, gs, v, t2)) return -1;
    if (sqrt(t2[0]) <= D.P.cgTolerance * r0) return it;
    beta = t2[1] / rz;
    rz = t2[1];
    float4* tmp = pPrev;
    pPrev = pCur;
    pCur = tmp;
  }
  if (finished && !done) *finished = false;
  return it;
}

// ---------------------------------------------------------------------------------------------------------------
// Reference-order PCG with resident rows (k_solve_rows; the form pcgVariant 0 runs where a scene fits it). One thread owns one row of its block for the
// whole solve and keeps the row's PCG state (p, A p and its filtered copy, r, step, resid, z, the contact plane and
// the preconditioner block) in registers, so an iteration's only global traffic is the gather of z_j over the row's
// columns and the store of the new z_i: the reference-order kernel re-reads the row vectors from L2 in both passes.
// The block's slots sit in shared memory in a sliced layout: the rows in warps of 32, warp w's slots padded to its
// longest row L_w, slot k of lane l at base_w + 32 k + l (nine planes, then the columns; padding holds kPinnedBit),
// so a warp's 32 row threads read 32 consecutive words. The row's product keeps the two-lane order of
// pcgReferenceOrder<2> (the even slots in one sum, the odd slots in another, added at the end) and the FP64 partials
// are grouped as that kernel groups them (p.Ap by half-warps; the others fall on the same threads), so the iterates
// are that kernel's bit for bit.
constexpr int kRowThreads = 512;     // k_solve_rows block size: a block's rows must not exceed it
constexpr int kResidentRows = 4;     // the solve templates' Variant value of this form
constexpr int kSlicedDepth = 12;     // gathers a row thread has in flight (even, so k0 + k has the parity of k)

struct SlicedMatrix {
  const float* planes;   // 9 planes of `stride` floats
  const uint32_t* cols;  // `stride` column indices (bit 31: pinned column or padding)
  uint32_t stride;       // padded slots of the block
  uint32_t base, len;    // this thread's warp: its first position and its padded row length
};

// Copies this block's rows [r0, r1) into the sliced layout (all threads; ends with a block barrier). Returns false,
// after raising error 4, when the padded slots exceed P.slicedSlots (the host picks k_solve_rows only for scenes whose
// every block fits, so this is a guard).
__device__ inline bool stageSliced(const Dev& D, uint32_t r0, uint32_t r1, SlicedMatrix& A) {
  constexpr int kWarps = kRowThreads / 32;
  // The rows' first slots relative to the block's first, bit 31 set for pinned rows (they take no product).
  __shared__ uint32_t off[kRowThreads + 1];
  __shared__ uint32_t warpLen[kWarps], warpBase[kWarps + 1];
  const uint32_t t = threadIdx.x, lane = t & 31u, w = t >> 5;
  const uint32_t R = r1 - r0;
  if (R > static_cast<uint32_t>(kRowThreads) || blockDim.x != static_cast<unsigned>(kRowThreads)) {
    if (t == 0) atomicExch(&D.ctl->error, 4);
    return false;
  }
  const uint32_t first = __ldg(D.rowStart + r0);  // r0 <= n: rowStart has n + 1 entries
  uint32_t c = 0;
  if (t < R) {
    const uint32_t rs = __ldg(D.rowStart + r0 + t);
    const bool pinned = D.particle[r0 + t].pinned != 0u;
    off[t] = (rs - first) | (pinned ? kPinnedBit : 0u);
    if (!pinned) c = __ldg(D.rowStart + r0 + t + 1) - rs;
  }
  if (t == 0) off[R] = __ldg(D.rowStart + r1) - first;
  const uint32_t len = __reduce_max_sync(0xffffffffu, c);
  if (lane == 0) warpLen[w] = len;
  __syncthreads();
  if (t == 0) {
    uint32_t acc = 0;
    for (int k = 0; k < kWarps; ++k) {
      warpBase[k] = acc;
      acc += 32u * warpLen[k];
    }
    warpBase[kWarps] = acc;
  }
  __syncthreads();
  const uint32_t total = warpBase[kWarps];
  if (total > D.P.slicedSlots) {
    if (t == 0) atomicExch(&D.ctl->error, 4);
    return false;
  }
  float* planes = reinterpret_cast<float*>(solveSmem);
  uint32_t* cols = reinterpret_cast<uint32_t*>(planes + 9 * total);
  A.planes = planes;
  A.cols = cols;
  A.stride = total;
  A.base = warpBase[w];
  A.len = warpLen[w];
  // Padding of this thread's row: positions [c, len) of its lane.
  for (uint32_t k = c; k < len; ++k) cols[A.base + 32u * k + lane] = kPinnedBit;
  // The slots, read in slot order (coalesced); each finds its row by bisection over off[].
  const uint32_t S = off[R];
  const uint32_t SP = D.P.slotsPadded;
  for (uint32_t k = t; k < S; k += blockDim.x) {
    uint32_t lo = 0, hi = R;  // row lo's first slot <= k < row hi's first slot
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if ((off[mid] & ~kPinnedBit) <= k) lo = mid; else hi = mid;
    }
    if (off[lo] & kPinnedBit) continue;  // a pinned row's slot
    const uint32_t j = k - off[lo];
    const uint32_t pos = warpBase[lo >> 5] + 32u * j + (lo & 31u);
    const uint32_t s = first + k;
#pragma unroll
    for (int q = 0; q < 9; ++q) planes[q * total + pos] = __ldg(D.blocks + q * SP + s);
    cols[pos] = __ldg(D.colIndex + s);
  }
  __syncthreads();
  return true;
}

// y_i (unfiltered) = sum over the row's unpinned columns j of A_ij x_j, for this thread's row, in pcgReferenceOrder<2>'s
// order: slot k of the row into sum k mod 2, each sum in slot order, the odd sum added to the even one last.
__device__ __forceinline__ float3 slicedProduct(const SlicedMatrix& A, const float4* x) {
  float3 acc0 = mk(0, 0, 0), acc1 = mk(0, 0, 0);
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t k0 = 0; k0 < A.len; k0 += kSlicedDepth) {
    uint32_t col[kSlicedDepth];
#pragma unroll
    for (int k = 0; k < kSlicedDepth; ++k)
      col[k] = k0 + k < A.len ? A.cols[A.base + 32u * (k0 + k) + lane] : kPinnedBit;
    float3 v[kSlicedDepth];
#pragma unroll
    for (int k = 0; k < kSlicedDepth; ++k) v[k] = (col[k] & kPinnedBit) ? mk(0, 0, 0) : ld3(x, col[k]);
#pragma unroll
    for (int k = 0; k < kSlicedDepth; ++k) {
      if (col[k] & kPinnedBit) continue;
      const uint32_t pos = A.base + 32u * (k0 + k) + lane;
      float a[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) a[q] = A.planes[q * A.stride + pos];
      blockMulAddRn((k & 1) ? acc1 : acc0, a, v[k]);
    }
  }
  return mk(__fadd_rn(acc0.x, acc1.x), __fadd_rn(acc0.y, acc1.y), __fadd_rn(acc0.z, acc1.z));
}

// The reference-order PCG of pcgReferenceOrder (same recurrences, same stopping tests) over resident rows. Writes
// step, resid, r and z of the block's rows; returns the iteration count, or -1 when a grid barrier gave up.
__device__ inline int pcgResidentRows(const Dev& D, GridSync& gs, const SlicedMatrix& A) {
  uint32_t r0i, r1i;
  blockRange(D.P.n, gs.rank, gs.size, r0i, r1i);
  const uint32_t i = r0i + threadIdx.x;
  const bool own = i < r1i;
  Contact c{};
  M3 M{};
  float3 step = mk(0, 0, 0), resid = mk(0, 0, 0), r = mk(0, 0, 0), z = mk(0, 0, 0);
  float3 p = mk(0, 0, 0), apFull = mk(0, 0, 0), ap = mk(0, 0, 0);
  // CG init (kernels.h:252-268): step = 0, resid = -grad, r = filter(resid), z = filter(M r).
  double tot[2];
  {
    double v[2] = {0.0, 0.0};
    if (own) {
      c = D.contact[i];
      M = loadPrecond(D, i);
      resid = -ld3(D.grad, i);
      r = filterRn(c, resid);
      z = filterRn(c, mulRn(M, r));
      D.z[i] = f4(z);
      v[0] += dotd3(r, z);
      v[1] += dotd3(r, r);
    }
    if (!gridReduce<2>(D, gs, v, tot)) return -1;
  }
  double rz = tot[0];
  const double r0 = sqrt(tot[1]);
  double beta = 0.0;
  int it = 0;
  const int maxCg = D.P.maxCg;
  if (r0 > 0.0) {
    while (it < maxCg) {
      // A p = A z + beta A pPrev, p = z + beta pPrev (the direction update folded into the product).
      const float fb = static_cast<float>(beta);
      const bool firstIt = it == 0;
      double vpap[1] = {0.0};
      const float3 az = slicedProduct(A, D.z);
      if (own) {
        p = firstIt ? z : axpyRn(p, fb, z);
        const float3 acc = firstIt ? az : axpyRn(apFull, fb, az);
        ap = filterRn(c, acc);
        apFull = acc;
        vpap[0] += dotd3(p, ap);
      }
      double pAp[1];
      if (!gridReduce<1, false, true>(D, gs, vpap, pAp)) return -1;
      if (!(pAp[0] > 0.0)) break;
      const double alpha = rz / pAp[0];
      const float fa = static_cast<float>(alpha);
      ++it;
      // Update (kernels.h:304-315) fused with the preconditioner apply (kernels.h:324-332).
      double v[2] = {0.0, 0.0};
      if (own) {
        step = axpyRn(p, fa, step);
        r = axpyRn(ap, -fa, r);
        resid = axpyRn(apFull, -fa, resid);
        z = filterRn(c, mulRn(M, r));
        D.z[i] = f4(z);
        v[0] += dotd3(r, r);
        v[1] += dotd3(r, z);
      }
      double t2[2];
      if (!gridReduce<2>(D, gs, v, t2)) return -1;
      if (sqrt(t2[0]) <= D.P.cgTolerance * r0) break;
      beta = t2[1] / rz;
      rz = t2[1];
    }
  }
  if (own) {
    D.step[i] = f4(step);
    D.resid[i] = f4(resid);
    D.r[i] = f4(r);
  }
  return it;
}

constexpr int kLearnedDepth = 4;  // slots whose factor rows and gathered vector a row thread has in flight

// acc += B x (Upper: B^T x) for this thread's row over its slots [k0, k1) of the block's sliced column layout (slot k
// is global slot rs + k; the columns are sorted, so the lower part j <= i is [0, kd] and the upper part j >= i is
// [kd, end) with kd the diagonal's position), the blocks from the factor by rows (D.LfRows); padding and pinned columns
// carry bit 31 and are skipped. kLearnedDepth slots' loads are issued before their first FMA.
template <bool Upper>
__device__ __forceinline__ float3 factorProduct(const Dev& D, const SlicedMatrix& A, uint32_t rs, uint32_t kBegin,
                                                uint32_t kEnd, const float4* x) {
  const uint32_t lane = threadIdx.x & 31u;
  float3 acc = mk(0, 0, 0);
  for (uint32_t k0 = kBegin; k0 < kEnd; k0 += kLearnedDepth) {
    bool use[kLearnedDepth];
    float3 v[kLearnedDepth];
    float4 m[kLearnedDepth][3];
#pragma unroll
    for (int u = 0; u < kLearnedDepth; ++u) {
      const uint32_t k = k0 + u;
      const uint32_t col = k < kEnd ? A.cols[A.base + 32u * k + lane] : kPinnedBit;
      use[u] = !(col & kPinnedBit);
      v[u] = mk(0, 0, 0);
      m[u][0] = m[u][1] = m[u][2] = make_float4(0, 0, 0, 0);
      if (use[u]) {
        v[u] = ld3(x, col);
        const float4* row = D.LfRows + 3 * static_cast<size_t>(rs + k);
        m[u][0] = __ldg(row);
        m[u][1] = __ldg(row + 1);
        m[u][2] = __ldg(row + 2);
      }
    }
#pragma unroll
    for (int u = 0; u < kLearnedDepth; ++u) {
      if (!use[u]) continue;
      const float4 a = m[u][0], b = m[u][1], c = m[u][2];
      const float3 w = v[u];
      if (Upper) {  // L_ji^T x_j
        acc.x += a.x * w.x + b.x * w.y + c.x * w.z;
        acc.y += a.y * w.x + b.y * w.y + c.y * w.z;
        acc.z += a.z * w.x + b.z * w.y + c.z * w.z;
      } else {  // L_ij x_j
        acc.x += a.x * w.x + a.y * w.y + a.z * w.z;
        acc.y += b.x * w.x + b.y * w.y + b.z * w.z;
        acc.z += c.x * w.x + c.y * w.y + c.z * w.z;
      }
    }
  }
  return acc;
}

// z_i = F(L L^T r)_i for this thread's row over resident rows (pcgLearnedResident). y = L^T r goes through D.ap (r was
// published by the caller's reduction; a grid barrier publishes y); returns false when the barrier gave up.
__device__ inline bool applyLearnedResident(const Dev& D, GridSync& gs, const SlicedMatrix& A, uint32_t i, bool own,
                                            uint32_t rs, uint32_t kd, uint32_t len, const Contact& c, float3& z) {
  // y_i = sum over the row's slots (i, j), j >= i, of L_(j, i)^T r_j.
  if (own) D.ap[i] = f4(factorProduct<true>(D, A, rs, kd, len, D.r));  // pinned rows: kd = len = 0
  if (!gs.sync()) return false;
  // z_i = F(sum over the row's slots (i, j), j <= i, of L_(i, j) y_j).
  if (own) {
    z = filterContact(c, factorProduct<false>(D, A, rs, 0, min(kd + 1, len), D.ap));
    D.z[i] = f4(z);
  }
  return true;
}

// The learned-preconditioner PCG of pcgLearned (M^-1 = L L^T, contact-filtered, the same stopping tests and breakdown
// rules) over resident rows: each thread keeps its row's step, resid, r, z, p, A p and its filtered copy in registers;
// the matrix is the block's sliced shared-memory copy; r and z are published for the neighbours' gathers. Four grid
// exchanges an iteration (p.Ap; r.r, which publishes r; y = L^T r; r.z, which publishes z), as in pcgLearned. Returns
// the iteration count, -1 when a barrier gave up, or -2 - iterations on a breakdown (the caller then solves with
// block-Jacobi).
__device__ inline int pcgLearnedResident(const Dev& D, GridSync& gs, const SlicedMatrix& A) {
  uint32_t r0i, r1i;
  blockRange(D.P.n, gs.rank, gs.size, r0i, r1i);
  const uint32_t i = r0i + threadIdx.x;
  const bool own = i < r1i;
  const uint32_t rs = own ? __ldg(D.rowStart + i) : 0u;
  // The row's length and its diagonal's position (the factor's lower part is [0, kd], the upper [kd, len)); a pinned
  // row has no slots in the sliced layout (its L is zero) and takes none, and no range passes the warp's length.
  const bool live = own && D.particle[i].pinned == 0u;
  const uint32_t len = live ? min(__ldg(D.rowStart + i + 1) - rs, A.len) : 0u;
  const uint32_t kd = live ? min(__ldg(D.diagSlot + i) - rs, len) : 0u;
  Contact c{};
  float3 step = mk(0, 0, 0), resid = mk(0, 0, 0), r = mk(0, 0, 0), z = mk(0, 0, 0);
  float3 p = mk(0, 0, 0), ap = mk(0, 0, 0), apFull = mk(0, 0, 0);
  auto writeBack = [&] {
    if (own) {
      D.step[i] = f4(step);
      D.resid[i] = f4(resid);
      D.r[i] = f4(r);
    }
  };
  double rr0;
  {
    double v[1] = {0.0}, t[1];
    if (own) {
      c = D.contact[i];
      resid = -ld3(D.grad, i);
      r = filterContact(c, resid);
      D.r[i] = f4(r);
      v[0] = dotd3(r, r);
    }
    if (!gridReduce<1>(D, gs, v, t)) return -1;
    rr0 = t[0];
  }
  const double r0 = sqrt(rr0);
  if (!(r0 > 0.0) || !(rr0 > 0.0)) {
    writeBack();
    return 0;
  }
  double rz;
  {
    if (!applyLearnedResident(D, gs, A, i, own, rs, kd, len, c, z)) return -1;
    double v[1] = {own ? dotd3(r, z) : 0.0}, t[1];
    if (!gridReduce<1>(D, gs, v, t)) return -1;
    rz = t[0];
  }
  if (!isfinite(rz)) return -2;
  double beta = 0.0;
  int it = 0;
  while (it < D.P.maxCg) {
    // A p = A z + beta A pPrev, p = z + beta pPrev.
    const float fb = static_cast<float>(beta);
    const float3 az = slicedProduct(A, D.z);
    double vpap[1] = {0.0}, pAp[1];
    if (own) {
      p = it == 0 ? z : z + p * fb;
      apFull = it == 0 ? az : az + apFull * fb;
      ap = filterContact(c, apFull);
      vpap[0] = dotd3(p, ap);
    }
    if (!gridReduce<1>(D, gs, vpap, pAp)) return -1;
    if (!isfinite(pAp[0])) return -2 - it;
    if (!(pAp[0] > 0.0)) break;
    const float fa = static_cast<float>(rz / pAp[0]);
    ++it;
    double v[1] = {0.0}, rr[1];
    if (own) {
      step = step + p * fa;
      r = r - ap * fa;
      resid = resid - apFull * fa;
      D.r[i] = f4(r);
      v[0] = dotd3(r, r);
    }
    if (!gridReduce<1>(D, gs, v, rr)) return -1;
    if (!isfinite(rr[0])) return -2 - it;
    if (sqrt(rr[0]) <= D.P.cgTolerance * r0) break;
    if (rr[0] > 1e6 * rr0) return -2 - it;
    if (!applyLearnedResident(D, gs, A, i, own, rs, kd, len, c, z)) return -1;
    double vz[1] = {own ? dotd3(r, z) : 0.0}, rzNew[1];
    if (!gridReduce<1>(D, gs, vz, rzNew)) return -1;
    if (!isfinite(rzNew[0])) return -2 - it;
    beta = rzNew[0] / rz;
    rz = rzNew[0];
  }
  writeBack();
  return it;
}

// Pipelined contact-filtered block-Jacobi PCG (Ghysels and Vanroose, "Hiding global synchronization latency in the
// preconditioned conjugate gradient algorithm", Parallel Computing 40 (2014) 224-238, Alg. 3). In exact arithmetic
// its iterates, iteration count and stopping tests are those of pcgReferenceOrder (operator F A F, preconditioner
// F M F, the same |r| <= tol |r0| and p.Ap <= 0 tests): besides u = M r and w = A u it carries s = A p, q = M s and
// z = A q by recurrence, so each iteration is one pass over the rows and ONE grid exchange instead of two. The pass
// forms n = F A m for the m = F M w of the previous exchange (the only gather), updates the row's z, q, s, p, x, r,
// u, w and forms the next exchange's FP64 partials (r.u, w.u, r.r) and the next m; the exchange (gridReduce<3>)
// publishes partials and m together. m alternates between two buffers: a block cannot pass the next exchange before
// every block has arrived at it, hence before any block still gathers the m it would overwrite. The unfiltered
// residual for the contact force, resid = -grad - A step, is formed once after the loop. Vectors: x = step, r = r,
// u = z, w = ap, s = apFull, p = p0, q = p1, z = pz, m = pm0 / pm1. Returns the iteration count, or -1 when a grid
// barrier gave up.
template <int PL>
__device__ inline int pcgPipelined(const Dev& D, GridSync& gs, const SmemMatrix& A) {
  uint32_t r0i, r1i;
  blockRange(D.P.n, gs.rank, gs.size, r0i, r1i);
  float4 *x = D.step, *r = D.r, *u = D.z, *w = D.ap, *s = D.apFull, *p = D.p0, *q = D.p1, *zq = D.pz;
  // x = 0, r = F(-grad), u = F(M r); u is gathered next, so a plain barrier publishes it.
  for (uint32_t i = r0i + threadIdx.x; i < r1i; i += blockDim.x) {
    const Contact c = D.contact[i];
    const float3 ri = filterContact(c, -ld3(D.grad, i));
    x[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    r[i] = f4(ri);
    u[i] = f4(filterContact(c, mul(loadPrecond(D, i), ri)));
  }
  if (!gs.sync()) return -1;
  // w = F A u, the first partials and m.
  double t[3];
  {
    double v[3] = {0.0, 0.0, 0.0};
    directionProducts<PL>(
        D, A, r0i, r1i, [&](uint32_t j) { return ld3(u, j); },
        [&](uint32_t i, float3 ui, float3 au) {
          const Contact c = D.contact[i];
          const float3 wi = filterContact(c, au);
          const float3 ri = ld3(r, i);
          w[i] = f4(wi);
          v[0] += dotd3(ri, ui);
          v[1] += dotd3(wi, ui);
          v[2] += dotd3(ri, ri);
          D.pm0[i] = f4(filterContact(c, mul(loadPrecond(D, i), wi)));
        });
    if (!gridReduce<3>(D, gs, v, t)) return -1;
  }
  const double r0 = sqrt(t[2]);
  double gammaPrev = 0.0, alphaPrev = 0.0;
  int it = 0;
  while (it < D.P.maxCg) {
    if (!(r0 > 0.0)) break;
    if (it > 0 && sqrt(t[2]) <= D.P.cgTolerance * r0) break;
    const double gamma = t[0], delta = t[1];
    const double beta = it == 0 ? 0.0 : gamma / gammaPrev;
    const double pAp = it == 0 ? delta : delta - beta * gamma / alphaPrev;
    if (!(pAp > 0.0)) break;
    const double alpha = gamma / pAp;
    const float fa = static_cast<float>(alpha), fb = static_cast<float>(beta);
    const bool first = it == 0;
    const float4* mCur = (it & 1) ? D.pm1 : D.pm0;
    float4* mNext = (it & 1) ? D.pm0 : D.pm1;
    double v[3] = {0.0, 0.0, 0.0};
    directionProducts<PL>(
        D, A, r0i, r1i, [&](uint32_t j) { return ld3(mCur, j); },
        [&](uint32_t i, float3 mi, float3 am) {
          // Each recurrence is formed and stored in turn (z, w, s, r, q, u, p, x), so that only r, u and w stay live.
          const Contact c = D.contact[i];
          const float3 zi = first ? filterContact(c, am) : filterContact(c, am) + ld3(zq, i) * fb;
          zq[i] = f4(zi);
          const float3 wi0 = ld3(w, i);
          const float3 wi = wi0 - zi * fa;
          w[i] = f4(wi);
          const float3 si = first ? wi0 : wi0 + ld3(s, i) * fb;
          s[i] = f4(si);
          const float3 ri = ld3(r, i) - si * fa;
          r[i] = f4(ri);
          const float3 qi = first ? mi : mi + ld3(q, i) * fb;
          q[i] = f4(qi);
          const float3 ui0 = ld3(u, i);
          const float3 ui = ui0 - qi * fa;
          u[i] = f4(ui);
          const float3 pi = first ? ui0 : ui0 + ld3(p, i) * fb;
          p[i] = f4(pi);
          x[i] = f4(ld3(x, i) + pi * fa);
          v[0] += dotd3(ri, ui);
          v[1] += dotd3(wi, ui);
          v[2] += dotd3(ri, ri);
          mNext[i] = f4(filterContact(c, mul(loadPrecond(D, i), wi)));
        });
    ++it;
    gammaPrev = gamma;
    alphaPrev = alpha;
    if (!gridReduce<3>(D, gs, v, t)) return -1;
  }
  // resid = -grad - A step over unpinned rows and columns (the reference-order PCG's recurrence, formed directly). Every
  // exit of the loop follows a grid exchange, whose barrier has published every block's last x.
  directionProducts<PL>(
      D, A, r0i, r1i, [&](uint32_t j) { return ld3(x, j); },
      [&](uint32_t i, float3, float3 ax) { D.resid[i] = f4(-ld3(D.grad, i) - ax); });
  return it;
}

// Contact-filtered block-Jacobi PCG in the Chronopoulos-Gear form ("s-step iterative methods for symmetric linear
// systems", J. Comput. Appl. Math. 25 (1989) 153-168): the same iterates and stopping tests as pcgReferenceOrder in
// exact arithmetic. Each iteration forms w = F A z exactly (the only gather), reduces r.z, w.z and r.r in one FP64 grid
// reduction, and takes alpha = (r.z) / (w.z - beta (r.z) / alpha_prev) (= r.z / p.Ap) with beta = (r.z) / (r.z)_prev;
// A p is carried as s = w + beta s, as the reference-order form carries it. The exchange that publishes the new z is a
// plain barrier instead of the reference order's second reduction. resid = -grad - A step is formed after the loop.
// Vectors: x = step, r = r, z = z, p = p0, s = ap, w = apFull. Returns the iteration count, or -1 when a grid barrier
// gave up.
template <int PL>
__device__ inline int pcgSingleReduction(const Dev& D, GridSync& gs, const SmemMatrix& A) {
  uint32_t r0i, r1i;
  blockRange(D.P.n, gs.rank, gs.size, r0i, r1i);
  float4 *x = D.step, *r = D.r, *z = D.z, *p = D.p0, *s = D.ap, *w = D.apFull;
  for (uint32_t i = r0i + threadIdx.x; i < r1i; i += blockDim.x) {
    const Contact c = D.contact[i];
    const float3 ri = filterContact(c, -ld3(D.grad, i));
    x[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    r[i] = f4(ri);
    z[i] = f4(filterContact(c, mul(loadPrecond(D, i), ri)));
  }
  if (!gs.sync()) return -1;
  double r0 = 0.0, gammaPrev = 0.0, alphaPrev = 0.0;
  int it = 0;
  while (true) {
    // w = F A z and the three partials.
    double v[3] = {0.0, 0.0, 0.0};
    directionProducts<PL>(
        D, A, r0i, r1i, [&](uint32_t j) { return ld3(z, j); },
        [&](uint32_t i, float3 zi, float3 az) {
          const float3 wi = filterContact(D.contact[i], az);
          const float3 ri = ld3(r, i);
          w[i] = f4(wi);
          v[0] += dotd3(ri, zi);
          v[1] += dotd3(wi, zi);
          v[2] += dotd3(ri, ri);
        });
    double t[3];
    if (!gridReduce<3>(D, gs, v, t)) return -1;
    if (it == 0) r0 = sqrt(t[2]);
    if (!(r0 > 0.0)) break;
    if (it > 0 && sqrt(t[2]) <= D.P.cgTolerance * r0) break;
    if (it >= D.P.maxCg) break;
    const double gamma = t[0];
    const double beta = it == 0 ? 0.0 : gamma / gammaPrev;
    const double pAp = it == 0 ? t[1] : t[1] - beta * gamma / alphaPrev;
    if (!(pAp > 0.0)) break;
    const double alpha = gamma / pAp;
    const float fa = static_cast<float>(alpha), fb = static_cast<float>(beta);
    const bool first = it == 0;
    for (uint32_t i = r0i + threadIdx.x; i < r1i; i += blockDim.x) {
      const Contact c = D.contact[i];
      const float3 pi = first ? ld3(z, i) : ld3(z, i) + ld3(p, i) * fb;
      p[i] = f4(pi);
      const float3 si = first ? ld3(w, i) : ld3(w, i) + ld3(s, i) * fb;
      s[i] = f4(si);
      x[i] = f4(ld3(x, i) + pi * fa);
      const float3 ri = ld3(r, i) - si * fa;
      r[i] = f4(ri);
      z[i] = f4(filterContact(c, mul(loadPrecond(D, i), ri)));
    }
    ++it;
    gammaPrev = gamma;
    alphaPrev = alpha;
    if (!gs.sync()) return -1;
  }
  // resid = -grad - A step over unpinned rows and columns; the last exchange has published every block's x.
  directionProducts<PL>(
      D, A, r0i, r1i, [&](uint32_t j) { return ld3(x, j); },
      [&](uint32_t i, float3, float3 ax) { D.resid[i] = f4(-ld3(D.grad, i) - ax); });
  return it;
}

// z = F(L L^T r) over this block's rows, with L the learned factor (planes D.Lf, lower slots) and y = L^T r kept in
// D.ap between the two products; returns false when a grid barrier gave up. Adds r.z of its rows to *rz.
template <int RL>
__device__ inline bool applyLearned(const Dev& D, GridSync& gs, uint32_t r0i, uint32_t r1i, double* rz) {
  const uint32_t groups = blockDim.x / RL;
  const int sub = threadIdx.x & (RL - 1);
  const unsigned groupMask = ((1u << RL) - 1u) << ((threadIdx.x & 31) & ~(RL - 1));
  const uint32_t SP = D.P.slotsPadded;
  // y_j = sum over slots (j, i), i >= j, of L_(i, j)^T r_i.
  for (uint32_t j = r0i + threadIdx.x / RL; j < r1i; j += groups) {
    float3 acc = mk(0, 0, 0);
    for (uint32_t s = __ldg(D.rowStart + j) + sub; s < __ldg(D.rowStart + j + 1); s += RL) {
      const uint32_t col = __ldg(D.colIndex + s);
      if ((col & kPinnedBit) || col < j) continue;
      const uint32_t t = __ldg(D.tslot + s);
      const float3 v = ld3(D.r, col);
      const float* L = D.Lf + t;
      acc.x += L[0] * v.x + L[3 * SP] * v.y + L[6 * SP] * v.z;
      acc.y += L[SP] * v.x + L[4 * SP] * v.y + L[7 * SP] * v.z;
      acc.z += L[2 * SP] * v.x + L[5 * SP] * v.y + L[8 * SP] * v.z;
    }
#pragma unroll
    for (int o = RL / 2; o > 0; o >>= 1) {
      acc.x += __shfl_xor_sync(groupMask, acc.x, o);
      acc.y += __shfl_xor_sync(groupMask, acc.y, o);
      acc.z += __shfl_xor_sync(groupMask, acc.z, o);
    }
    if (sub == 0) D.ap[j] = f4(acc);
  }
  if (!gs.sync()) return false;
  // z_i = F(sum over slots (i, j), j <= i, of L_(i, j) y_j).
  for (uint32_t i = r0i + threadIdx.x / RL; i < r1i; i += groups) {
    float3 acc = mk(0, 0, 0);
    for (uint32_t s = __ldg(D.rowStart + i) + sub; s < __ldg(D.rowStart + i + 1); s += RL) {
      const uint32_t col = __ldg(D.colIndex + s);
      if ((col & kPinnedBit) || col > i) continue;
      const float3 v = ld3(D.ap, col);
      const float* L = D.Lf + s;
      acc.x += L[0] * v.x + L[SP] * v.y + L[2 * SP] * v.z;
      acc.y += L[3 * SP] * v.x + L[4 * SP] * v.y + L[5 * SP] * v.z;
      acc.z += L[6 * SP] * v.x + L[7 * SP] * v.y + L[8 * SP] * v.z;
    }
#pragma unroll
    for (int o = RL / 2; o > 0; o >>= 1) {
      acc.x += __shfl_xor_sync(groupMask, acc.x, o);
      acc.y += __shfl_xor_sync(groupMask, acc.y, o);
      acc.z += __shfl_xor_sync(groupMask, acc.z, o);
    }
    if (sub == 0) {
      const float3 zi = filterContact(D.contact[i], acc);
      D.z[i] = f4(zi);
      *rz += dotd3(ld3(D.r, i), zi);
    }
  }
  return true;
}

// PCG with the learned preconditioner M^-1 = L L^T (contact-filtered), in the reference's order otherwise: four grid
// synchronisations per iteration (p.Ap, r.r, y = L^T r, r.z). The convergence test is the reference's, on the
// unpreconditioned residual. Returns the iteration count, -1 when a barrier gave up, or -2 - iterations when the
// solve broke down (a non-finite scalar, or |r|^2 above 1e6 |r0|^2): the caller then solves again with block-Jacobi.
// M^-1 = L L^T is SPD for any finite L with a positive block diagonal, so a finite solve converges like any PCG; its
// unpreconditioned |r| is not monotone and is no stall signal. With `warm`, step, resid and r hold a partial solve
// (a block-Jacobi phase) and the iteration continues from them, with `r0In` (that solve's initial |r|) in the
// convergence test; `budget` bounds the iterations.
template <int PL>
__device__ inline int pcgLearned(const Dev& D, GridSync& gs, const SmemMatrix& A, bool warm = false,
                                 double r0In = 0.0, int budget = -1) {
  const uint32_t n = D.P.n;
  uint32_t r0i, r1i;
  blockRange(n, gs.rank, gs.size, r0i, r1i);
  double rr0;
  {
    double v[1] = {0.0};
    for (uint32_t i = r0i + threadIdx.x; i < r1i; i += blockDim.x) {
      if (warm) {
        v[0] += dotd3(ld3(D.r, i), ld3(D.r, i));
        continue;
      }
      const float3 res = -ld3(D.grad, i);
      const float3 ri = filterContact(D.contact[i], res);
      D.step[i] = make_float4(0, 0, 0, 0);
      D.resid[i] = f4(res);
      D.r[i] = f4(ri);
      v[0] += dotd3(ri, ri);
    }
    double t[1];
    if (!gridReduce<1>(D, gs, v, t)) return -1;
    rr0 = t[0];
  }
  const double r0 = warm ? r0In : sqrt(rr0);
  if (!(r0 > 0.0) || !(rr0 > 0.0)) return 0;
  double rz;
  {
    double v[1] = {0.0};
    if (!applyLearned<(PL > 0 ? PL : kRowLanes)>(D, gs, r0i, r1i, &v[0])) return -1;
    double t[1];
    if (!gridReduce<1>(D, gs, v, t)) return -1;
    rz = t[0];
  }
  if (!isfinite(rz)) return -2;
  double beta = 0.0;
  float4* pPrev = D.p0;
  float4* pCur = D.p1;
  int it = 0;
  const int maxCg = budget < 0 ? D.P.maxCg : min(budget, D.P.maxCg);
  while (it < maxCg) {
    // SpMV with the direction update folded in: p_j = z_j + beta * pPrev_j.
    double vpap[1] = {directionStep<PL>(D, A, r0i, r1i, pPrev, pCur, static_cast<float>(beta), it == 0)};
    double pAp[1];
    if (!gridReduce<1>(D, gs, vpap, pAp)) return -1;
    if (!isfinite(pAp[0])) return -2 - it;
    if (!(pAp[0] > 0.0)) break;
    const float fa = static_cast<float>(rz / pAp[0]);
    ++it;
    double v[1] = {0.0};
    for (uint32_t i = r0i + threadIdx.x; i < r1i; i += blockDim.x) {
      const float3 pi = ld3(pCur, i);
      D.step[i] = f4(ld3(D.step, i) + pi * fa);
      const float3 ri = ld3(D.r, i) - ld3(D.ap, i) * fa;
      D.r[i] = f4(ri);
      D.resid[i] = f4(ld3(D.resid, i) - ld3(D.apFull, i) * fa);
      v[0] += dotd3(ri, ri);
    }
    double rr[1];
    if (!gridReduce<1>(D, gs, v, rr)) return -1;
    if (!isfinite(rr[0])) return -2 - it;
    if (sqrt(rr[0]) <= D.P.cgTolerance * r0) break;
    if (rr[0] > 1e6 * rr0) return -2 - it;
    double vz[1] = {0.0};
    if (!applyLearned<(PL > 0 ? PL : kRowLanes)>(D, gs, r0i, r1i, &vz[0])) return -1;
    double rzNew[1];
    if (!gridReduce<1>(D, gs, vz, rzNew)) return -1;
    if (!isfinite(rzNew[0])) return -2 - it;
    beta = rzNew[0] / rz;
    rz = rzNew[0];
    float4* tmp = pPrev;
    pPrev = pCur;
    pCur = tmp;
  }
  return it;
}

// The solve's PCG: block-Jacobi (reference order), or the learned schedule: P.learnedSwitch block-Jacobi iterations
// first (0: none), then, when the solve has not converged, the learned preconditioner from the current iterate within
// the remaining iteration budget; a learned phase that stalls is followed by a full block-Jacobi solve. Returns the
// total iteration count of all phases, or -1 when a barrier gave up.
// Variant (block-Jacobi only): 0 the reference's order (pcgReferenceOrder), 1 pipelined (pcgPipelined; needs the
// pm0/pm1/pz vectors), 2 Chronopoulos-Gear (pcgSingleReduction). A compile-time choice, so each solve kernel carries
// one PCG's registers.
template <bool Learned, int PL, int Variant>
__device__ inline int pcgSolveStaged(const Dev& D, GridSync& gs, const SmemMatrix& A);

template <bool Learned, int PL, int Variant = 0>
__device__ inline int pcgSolve(const Dev& D, GridSync& gs) {
  uint32_t r0i, r1i;
  blockRange(D.P.n, gs.rank, gs.size, r0i, r1i);
  if constexpr (Variant == kResidentRows) {
    SlicedMatrix A;
    if (!stageSliced(D, r0i, r1i, A)) return -1;
    const unsigned long long t0 = globalTimerNs();
    int it;
    if constexpr (Learned) {
      // The learned schedule without block-Jacobi iterations first (the host picks this kernel only then): a learned
      // solve that breaks down is followed by a full block-Jacobi solve, as in pcgSolveStaged.
      it = pcgLearnedResident(D, gs, A);
      if (gs.rank == 0 && threadIdx.x == 0) D.ctl->learnedSolves += 1;
      if (it < -1) {
        if (gs.rank == 0 && threadIdx.x == 0) D.ctl->precondFallbacks += 1;
        const int jac = pcgResidentRows(D, gs, A);
        it = jac < 0 ? jac : jac + (-2 - it);
      }
    } else {
      it = pcgResidentRows(D, gs, A);
    }
    if (gs.rank == 0 && threadIdx.x == 0) D.ctl->pcgNs += static_cast<long long>(globalTimerNs() - t0);
    return it;
  } else {
    const SmemMatrix A = stageMatrix(D, r0i, r1i);
    const unsigned long long t0 = globalTimerNs();
    const int it = pcgSolveStaged<Learned, PL, Variant>(D, gs, A);
    if (gs.rank == 0 && threadIdx.x == 0) D.ctl->pcgNs += static_cast<long long>(globalTimerNs() - t0);
    return it;
  }
}

template <bool Learned, int PL, int Variant>
__device__ inline int pcgSolveStaged(const Dev& D, GridSync& gs, const SmemMatrix& A) {
  if constexpr (!Learned) {
    if constexpr (Variant == 1) {
      return pcgPipelined<PL>(D, gs, A);
    } else if constexpr (Variant == 2) {
      return pcgSingleReduction<PL>(D, gs, A);
    } else {
      return pcgReferenceOrder<PL>(D, gs, A);
    }
  }
  int first = 0;
  double r0 = 0.0;
  const int sw = D.P.learnedSwitch;
  if (sw > 0) {
    bool finished = false;
    first = pcgReferenceOrder<PL>(D, gs, A, sw, &r0, &finished);
    if (first < 0 || finished || first >= D.P.maxCg) return first;
  }
  const int it = pcgLearned<PL>(D, gs, A, sw > 0, r0, D.P.maxCg - first);
  if (gs.rank == 0 && threadIdx.x == 0) D.ctl->learnedSolves += 1;
  if (it >= -1) return it < 0 ? it : first + it;
  if (gs.rank == 0 && threadIdx.x == 0) D.ctl->precondFallbacks += 1;
  const int jac = pcgReferenceOrder<PL>(D, gs, A);
  return jac < 0 ? jac : jac + first + (-2 - it);
}

// One Newton iteration's solve for the blocks of one group (the whole grid for one solver, or a garment's blocks in
// a batched launch); gs is initialised. PL: the scheme of the PCG's product A p (lanes per row, or 0 for
// slot-parallel; see directionProducts), also the lanes of the learned factor's products when positive.
template <bool Learned, int PL, int Variant = 0>
__device__ inline void solveGroup(const Dev& D, GridSync& gs) {
  Control* ctl = D.ctl;
  const uint32_t n = D.P.n;
  uint32_t r0i, r1i;
  blockRange(n, gs.rank, gs.size, r0i, r1i);
  const int it = pcgSolve<Learned, PL, Variant>(D, gs);
  if (it < 0) return;
  if (gs.rank == 0 && threadIdx.x == 0) {
    if (D.cgLog) D.cgLog[static_cast<unsigned long long>(ctl->newtonIterations) % kCgLogCapacity] = it;
    ctl->cgIterations += it;
    ctl->newtonIterations += 1;
    ctl->lastCg = it;
    ctl->energyEvaluations += 1;  // E(0) below
  }

  // The resident-row kernel's 512-thread blocks stand for the reference-order kernel's 1024-thread ones: its energies
  // are summed as two virtual threads per thread, in that kernel's order, so both kernels take the same line-search
  // decisions (its rows, at most 512 per block, already sit on the same threads).
  constexpr bool kVirtual = Variant == kResidentRows;
  // Contact normal force from the residual (kernels.h:391-396), Newton slope grad . step and E(0), in FP64.
  double se[2];
  {
    double v[2] = {0.0, 0.0};
    for (uint32_t i = r0i + threadIdx.x; i < r1i; i += blockDim.x) {
      const Contact c = D.contact[i];
      const float3 res = ld3(D.resid, i);
      D.contact[i].force = c.active != 0u ? fmaxf(0.0f, -dot(res, xyz(c.normal))) : 0.0f;
      v[0] += dotd3(ld3(D.grad, i), ld3(D.step, i));
    }
    if constexpr (kVirtual) {
      v[1] = energyPartial(D, gs, 0.0, threadIdx.x, 2 * blockDim.x);
      double hi[2] = {0.0, energyPartial(D, gs, 0.0, threadIdx.x + blockDim.x, 2 * blockDim.x)};
      if (!gridReducePairs<2>(D, gs, v, hi, se)) return;
    } else {
      v[1] = energyPartial(D, gs, 0.0);
      if (!gridReduce<2>(D, gs, v, se)) return;
    }
  }
  const double slope = se[0], e0 = se[1];
  if (!(slope < 0.0)) {
    if (gs.rank == 0 && threadIdx.x == 0) {
      ctl->newtonDone = 1;
      ctl->lastSlope = slope;
    }
    return;
  }
  // Backtracking line search, Armijo c = 1e-4, at most 20 halvings (cpu_solver.cpp:269-274).
  double alpha = 1.0;
  for (int ls = 0; ls < 20; ++ls) {
    if (gs.rank == 0 && threadIdx.x == 0) ctl->energyEvaluations += 1;
    double e[1];
    if constexpr (kVirtual) {
      double lo[1] = {energyPartial(D, gs, alpha, threadIdx.x, 2 * blockDim.x)};
      double hi[1] = {energyPartial(D, gs, alpha, threadIdx.x + blockDim.x, 2 * blockDim.x)};
      if (!gridReducePairs<1>(D, gs, lo, hi, e)) return;
    } else {
      double v[1] = {energyPartial(D, gs, alpha)};
      if (!gridReduce<1>(D, gs, v, e)) return;
    }
    if (e[0] <= e0 + 1e-4 * alpha * slope) break;
    alpha *= 0.5;
    if (gs.rank == 0 && threadIdx.x == 0) ctl->lineSearchHalvings += 1;
  }
  // Apply the step; max move; the next Newton iteration's friction uses this solve's forces (kernels.h:407-414).
  double mv[1] = {0.0};
  const float fa = static_cast<float>(alpha);
  for (uint32_t i = r0i + threadIdx.x; i < r1i; i += blockDim.x) {
    const float3 d = ld3(D.step, i) * fa;
    D.u[i] = f4(ld3(D.u, i) + d);
    mv[0] = fmax(mv[0], static_cast<double>(fmaxf(fabsf(d.x), fmaxf(fabsf(d.y), fabsf(d.z)))));
    const Contact c = D.contact[i];
    D.contact[i].frictionLambda = c.active != 0u ? c.force : 0.0f;
  }
  double maxMove[1];
  if (!gridReduce<1, true>(D, gs, mv, maxMove)) return;
  if (gs.rank == 0 && threadIdx.x == 0) {
    ctl->lastAlpha = alpha;
    ctl->lastSlope = slope;
    ctl->lastE0 = e0;
    ctl->lastMaxMove = maxMove[0];
    if (maxMove[0] < 1e-9) ctl->newtonDone = 1;
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Finish: x = xStart + u, post-solve push-out below the snap tolerance, pins, damped velocity (kernels.h:419-448,
// cpu_solver.cpp:285-313); the assembly clock of Assembling garments advances by h.

__device__ inline void finishRows(const Dev& D, uint32_t rank, uint32_t size) {
  const float h = D.P.h;
  for (uint32_t i = rank * blockDim.x + threadIdx.x; i < D.P.n; i += size * blockDim.x) {
    const Particle pa = D.particle[i];
    const Fabric fab = D.fabric[pa.fabric];
    const float3 xs = ld3(D.xStart, i);
    float3 xn = xs + ld3(D.u, i);
    if (pa.pinned != 0u) {
      xn = ld3(D.pinPos, i);
    } else if (D.field.present) {
      const float radius = contactRadius(D.P, fab);
      if (fieldSample(D.fieldValues, D.field, xn) < radius - D.P.contactSnap) {
        if (isZero(fieldGradient(D.fieldValues, D.field, xn))) {
          xn = landOnBody(D.fieldValues, D.field, radius, xs, xn);
        } else {
          collideBody(D.fieldValues, D.field, radius, fab.friction, xs, xn);
        }
      }
    }
    float c = D.P.dampingScale * fab.damping;
    if (D.garment[pa.garment].phase == 0) c += D.P.assemblyExtraDamping;
    const float3 vel = div(xn - xs, h) * fmaxf(0.0f, 1.0f - c * h);
    D.x[i] = f4(xn);
    D.v[i] = f4(vel);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Statistics of one solver or one garment (sim_model.cpp:222-241), reduced on the device in FP64.

struct StatsOut {
  double kineticEnergy, sumV2, maxSeamGap, maxPenetration;
  unsigned long long moving;
  int nonFinite;
  int pad;
  unsigned long long beginNs, endNs;  // %globaltimer at the frame's first kernel and at its statistics' end
};

}  // namespace dcu
