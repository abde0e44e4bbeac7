// The single solver's kernels (one solver per launch grid) over the device functions of kernels.cuh; the batch
// (batch.cu) launches its own wrappers of the same functions.
#pragma once

#include "kernels.cuh"

namespace dcu {

__global__ void k_begin(Dev D) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && D.ctl->frameBeginNs == 0ull) D.ctl->frameBeginNs = globalTimerNs();
  beginRows(D, blockIdx.x, gridDim.x);
}

// Contact candidates for given positions (test entry point; same code as k_begin).
__global__ void k_contact_candidates(Dev D, const float4* xs, Contact* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < D.P.n; i += gridDim.x * blockDim.x) {
    Contact c{};
    contactSetupOne(D, i, xyz(xs[i]), c);
    out[i] = c;
  }
}

__global__ void k_activate(Dev D) { activateRows(D, blockIdx.x, gridDim.x); }

constexpr int kTermThreads = 256;  // k_terms block size

__global__ void __launch_bounds__(kTermThreads) k_terms(Dev D) { termsRows(D, blockIdx.x, gridDim.x); }

// Four 256-thread blocks per SM (64 registers): with each stretch record loaded in one round (24 floats live), 1.9 %
// faster per drape frame than five (48 registers, spilling); with the record read in two dependent rounds five had been
// 3 % faster than four.
__global__ void __launch_bounds__(kAssembleThreads, 4) k_assemble(Dev D) {
  assembleSlots(D, blockIdx.x, gridDim.x);
}

// One Newton iteration's persistent solve; the whole grid is one group.
// Variant: the block-Jacobi PCG's form (0 reference order, 1 pipelined; see pcgSolveStaged).
template <bool Learned, int Variant = 0>
__global__ void __launch_bounds__(kSolveThreads, 1) k_solve(Dev D) {
  if (D.ctl->newtonDone) return;
  GridSync gs;
  gs.init(D.ctl, D.P.barrierLimitNs);
  solveGroup<Learned, kRowLanes, Variant>(D, gs);
}

// The same Newton iteration with the reference-order PCG over resident rows (pcgResidentRows): 512-thread blocks, so a
// row thread has the registers to keep its row's PCG state; launched only for scenes whose blocks have at most 512
// rows and whose sliced matrix fits in shared memory.
__global__ void __launch_bounds__(kRowThreads, 1) k_solve_rows(Dev D) {
  if (D.ctl->newtonDone) return;
  GridSync gs;
  gs.init(D.ctl, D.P.barrierLimitNs);
  solveGroup<false, kRowLanes, kResidentRows>(D, gs);
}

// The same with the learned preconditioner (pcgLearnedResident; block-Jacobi after a breakdown), for scenes that fit
// resident rows and solves that start with the learned preconditioner.
__global__ void __launch_bounds__(kRowThreads, 1) k_solve_rows_learned(Dev D) {
  if (D.ctl->newtonDone) return;
  GridSync gs;
  gs.init(D.ctl, D.P.barrierLimitNs);
  solveGroup<true, kRowLanes, kResidentRows>(D, gs);
}

__global__ void k_finish(Dev D) { finishRows(D, blockIdx.x, gridDim.x); }

__global__ void k_advance_clock(Dev D) {
  for (uint32_t g = threadIdx.x; g < D.P.nGarments; g += blockDim.x)
    if (D.garment[g].phase == 0) D.garment[g].assemblyTime += D.P.hD;
}

// Statistics: per-block partials, the last block to finish combines them.
__global__ void k_stats(Dev D, double* part, unsigned int* done, StatsOut* out) {
  double ke = 0, v2s = 0, gap = 0, pen = 0;
  unsigned long long moving = 0;
  int bad = 0;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (uint32_t i = tid; i < D.P.n; i += stride) {
    const float3 x = ld3(D.x, i), v = ld3(D.v, i);
    if (!isfinite(x.x) || !isfinite(x.y) || !isfinite(x.z) || !isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) bad = 1;
    if (D.field.present) {
      const double phi = fieldSampleD(D.fieldValues, D.field, x.x, x.y, x.z, D.fieldOrigin[0], D.fieldOrigin[1],
                                      D.fieldOrigin[2], D.fieldCell);
      pen = fmax(pen, -phi);
    }
    const Particle pa = D.particle[i];
    if (pa.pinned != 0u) continue;
    const double vv = static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y + static_cast<double>(v.z) * v.z;
    ke += 0.5 * static_cast<double>(pa.mass) * vv;
    v2s += vv;
    ++moving;
  }
  for (uint32_t k = tid; k < D.P.nSeam; k += stride) {
    const Seam s = D.seam[k];
    const float3 d = ld3(D.x, s.a) - ld3(D.x, s.b);
    gap = fmax(gap, static_cast<double>(sqrtf(d.x * d.x + d.y * d.y + d.z * d.z)));
  }
  double sums[2] = {ke, v2s};
  __shared__ double r2[2];
  blockSum<2>(sums, r2);
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
    double g = 0, p = 0;
    unsigned long long m = 0;
    int b = 0;
    for (int k = 0; k < nw; ++k) {
      g = fmax(g, mx[0][k]);
      p = fmax(p, mx[1][k]);
      m += mv[k];
      b |= bd[k];
    }
    double* row = part + blockIdx.x * 8;
    row[0] = r2[0];
    row[1] = r2[1];
    row[2] = g;
    row[3] = p;
    row[4] = static_cast<double>(m);
    row[5] = b;
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  // The last block combines the blocks' rows: thread t reads rows t, t + blockDim, ... (their loads in flight
  // together across the block), then fixed-shape block reductions.
  __threadfence();
  double sum3[3] = {0.0, 0.0, 0.0}, max2[2] = {0.0, 0.0};
  int nonFinite = 0;
  for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    const double* row = part + b * 8;
    sum3[0] += __ldcg(row + 0);
    sum3[1] += __ldcg(row + 1);
    max2[0] = fmax(max2[0], __ldcg(row + 2));
    max2[1] = fmax(max2[1], __ldcg(row + 3));
    sum3[2] += __ldcg(row + 4);
    nonFinite |= __ldcg(row + 5) != 0.0;
  }
  __shared__ double tot3[3], tot2[2];
  blockSum<3>(sum3, tot3);
  blockReduce<2, true>(max2, tot2);
  nonFinite = __syncthreads_or(nonFinite);
  if (threadIdx.x == 0) {
    StatsOut s{};
    s.kineticEnergy = tot3[0];
    s.sumV2 = tot3[1];
    s.moving = static_cast<unsigned long long>(tot3[2]);
    s.maxSeamGap = tot2[0];
    s.maxPenetration = tot2[1];
    s.nonFinite = nonFinite != 0;
    s.beginNs = D.ctl->frameBeginNs;
    s.endNs = globalTimerNs();
    D.ctl->frameBeginNs = 0ull;
    *out = s;
    *done = 0;
  }
}

// PCG on a given system (test and measurement entry point): block-Jacobi inverse of each diagonal block, then the
// same persistent PCG as k_solve.
__global__ void k_pcg_precondition(Dev D, const uint32_t* __restrict__ diag) {
  const uint32_t SP = D.P.slotsPadded;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < D.P.n; i += gridDim.x * blockDim.x) {
    M3 A;
#pragma unroll
    for (int k = 0; k < 9; ++k) A.m[k] = D.blocks[k * SP + diag[i]];
    M3 inv;
    if (D.particle[i].pinned != 0u) {
      zero(inv);
    } else {
      bool ok = false;
      inv = invertSpd(A, ok);
    }
    D.precond[3 * i + 0] = make_float4(inv.m[0], inv.m[1], inv.m[2], 0.0f);
    D.precond[3 * i + 1] = make_float4(inv.m[3], inv.m[4], inv.m[5], 0.0f);
    D.precond[3 * i + 2] = make_float4(inv.m[6], inv.m[7], inv.m[8], 0.0f);
  }
}

__global__ void __launch_bounds__(kSolveThreads, 1) k_pcg_only(Dev D) {
  GridSync gs;
  gs.init(D.ctl, D.P.barrierLimitNs);
  const int it = pcgSolve<false, kRowLanes>(D, gs);
  if (it >= 0 && blockIdx.x == 0 && threadIdx.x == 0) D.ctl->lastCg = it;
}

// Standalone block-CSR SpMV, y = A x over unpinned rows and columns, slot-parallel: block b owns rows
// [b * Rows, (b + 1) * Rows) and walks their slots in chunks of Chunk, each thread computing the products A_s x_j of
// consecutive slots (coalesced loads of every block plane and column index), staged in shared memory; one thread per
// row then adds its slots' products in slot order. Configuration: 256 threads, 128 rows, 1024-slot chunks (4.36 TB/s
// on the tiled 60k-tube system; a 128-thread, 64-row variant held to 32 registers reached 4.19 there).
constexpr uint32_t kSpmvThreads = 256, kSpmvBlockRows = 128, kSpmvBlockChunk = 1024;

__global__ void __launch_bounds__(kSpmvThreads) k_spmv(uint32_t n, const uint32_t* __restrict__ rowStart,
                                                           const uint32_t* __restrict__ colIndex,
                                                           const float* __restrict__ blocks, uint32_t SP,
                                                           const uint8_t* __restrict__ pinned,
                                                           const float4* __restrict__ x, float4* __restrict__ y) {
  __shared__ uint32_t rowOff[kSpmvBlockRows + 1];
  __shared__ float prod[3][kSpmvBlockChunk];
  const uint32_t t = threadIdx.x;
  for (uint32_t r0 = blockIdx.x * kSpmvBlockRows; r0 < n; r0 += gridDim.x * kSpmvBlockRows) {
    const uint32_t R = min(kSpmvBlockRows, n - r0);
    const uint32_t s0 = __ldg(rowStart + r0);
    if (t <= R) rowOff[t] = __ldg(rowStart + r0 + t) - s0;
    __syncthreads();
    const uint32_t S = rowOff[R];
    float3 acc = mk(0, 0, 0);
    const bool rowLive = t < R && pinned[r0 + t] == 0;
    for (uint32_t c = 0; c < S; c += kSpmvBlockChunk) {
      const uint32_t cn = min(kSpmvBlockChunk, S - c);
#pragma unroll 4
      for (uint32_t k = t; k < cn; k += kSpmvThreads) {
        const uint32_t s = s0 + c + k;
        const uint32_t j = __ldg(colIndex + s);
        float a[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) a[q] = __ldg(blocks + q * SP + s);
        float3 v = mk(0, 0, 0);
        if (pinned[j] == 0) {
          const float3 xj = xyz(__ldg(x + j));
          v.x = a[0] * xj.x + a[1] * xj.y + a[2] * xj.z;
          v.y = a[3] * xj.x + a[4] * xj.y + a[5] * xj.z;
          v.z = a[6] * xj.x + a[7] * xj.y + a[8] * xj.z;
        }
        prod[0][k] = v.x;
        prod[1][k] = v.y;
        prod[2][k] = v.z;
      }
      __syncthreads();
      if (t < R) {
        const uint32_t lo = max(rowOff[t], c), hi = min(rowOff[t + 1], c + cn);
        for (uint32_t q = lo; q < hi; ++q) {
          acc.x += prod[0][q - c];
          acc.y += prod[1][q - c];
          acc.z += prod[2][q - c];
        }
      }
      __syncthreads();
    }
    if (t < R) y[r0 + t] = f4(rowLive ? acc : mk(0, 0, 0));
    __syncthreads();  // rowOff is rewritten for the next row range
  }
}

// A barrier that waits for one more block than the grid has: it can only end by its time limit. Used by the test of
// the bounded wait; returns the status the blocks read back in *out (1: gave up).
__global__ void k_barrier_probe(Control* ctl, unsigned long long limitNs, int* out) {
  GridSync gs;
  gs.init(ctl, limitNs);
  gs.target += 1;  // one arrival that never comes
  const bool released = gs.sync();
  if (threadIdx.x == 0 && blockIdx.x == 0) *out = released ? 0 : ctl->error;
}

// The persistent solve's synchronisation floor: `iterations` rounds of grid-wide exchanges on the solve's grid, with no
// other work, timed by block 0 with %globaltimer (nanoseconds for all rounds in *ns, or 0 if a barrier gave up).
//   mode 0: gridReduce<1> + gridReduce<2>  (a reference-order PCG iteration's two reductions: p.Ap, then r.r and r.z)
//   mode 1: gridReduce<3> + a plain barrier (one merged reduction plus the direction's exchange before the next SpMV)
//   mode 2: gridReduce<3> alone
//   mode 3: two plain barriers
// Each round feeds its result into the next, so no round can be skipped or overlapped. Threads: the block size of the
// solve kernel measured (k_solve 1024, k_solve_rows 512).
template <int Threads>
__global__ void __launch_bounds__(Threads, 1) k_reduction_floor(Dev D, int mode, int iterations,
                                                                  unsigned long long* ns) {
  GridSync gs;
  gs.init(D.ctl, D.P.barrierLimitNs);
  double x = 1e-3 * threadIdx.x;
  const unsigned long long t0 = globalTimerNs();
  for (int it = 0; it < iterations; ++it) {
    if (mode == 0) {
      double a[1] = {x}, b[1];
      if (!gridReduce<1>(D, gs, a, b)) return;
      double c[2] = {x, b[0]}, d[2];
      if (!gridReduce<2>(D, gs, c, d)) return;
      x = 1e-9 * d[1];
    } else if (mode == 1 || mode == 2) {
      double a[3] = {x, 2.0 * x, 1.0}, b[3];
      if (!gridReduce<3>(D, gs, a, b)) return;
      if (mode == 1 && !gs.sync()) return;
      x = 1e-9 * b[0];
    } else {
      if (!gs.sync() || !gs.sync()) return;
      x += 1e-9;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *ns = (x > -1.0) ? globalTimerNs() - t0 : 0ull;
}

}  // namespace dcu
