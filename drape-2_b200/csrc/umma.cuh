// tcgen05 (5th-generation tensor core) helpers for sm_100a: TMEM allocation, BF16 x BF16 -> FP32 MMAs issued by one
// thread with both operands in shared memory, completion through an mbarrier, and TMEM -> register loads.
//
// Operand layout in shared memory: K-major, no swizzle ("interleaved" core matrices). A core matrix is 8 rows x
// 16 bytes (8 BF16 along K), stored as 128 contiguous bytes. For an R x K tile (R rows of the M or N dimension):
//   byte offset of element (r, k) = (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,  SBO = 16 * K,
// i.e. the leading-dimension byte offset (between K-adjacent core matrices) is 128 and the stride-dimension byte
// offset (between 8-row groups) is 16 * K. One MMA consumes K = 16 (two core matrices along K); the next K step
// starts 256 bytes further.
//
// Every wait on an mbarrier is bounded; on expiry the caller's error flag is set and the wait returns false.
#pragma once
#include <cstdint>

namespace umma {

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t kmajorOffset(uint32_t r, uint32_t k, uint32_t K) {
  return (r >> 3) * (16u * K) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor (no swizzle, K-major): start address, LBO = 128, SBO = 16 * K, version 1.
__device__ __forceinline__ uint64_t smemDesc(const void* tile, uint32_t K) {
  const uint64_t addr = smemAddr(tile);
  return ((addr & 0x3FFFFull) >> 4) | (static_cast<uint64_t>(128u >> 4) << 16) |
         (static_cast<uint64_t>((16u * K) >> 4) << 32) | (1ull << 46);
}

// The same with an explicit stride-dimension byte offset (a K-major operand whose 8-row groups lie `sbo` bytes apart,
// e.g. columns [64, 128) of a K = 128 tile read as a K = 64 operand: start + 1024, SBO = 2048).
__device__ __forceinline__ uint64_t smemDescSbo(const void* tile, uint32_t sbo) {
  const uint64_t addr = smemAddr(tile);
  return ((addr & 0x3FFFFull) >> 4) | (static_cast<uint64_t>(128u >> 4) << 16) |
         (static_cast<uint64_t>(sbo >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major, shape M x N.
__host__ __device__ constexpr uint32_t instrDescBf16(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// Whole warp: allocate `cols` TMEM columns (a power of two >= 32); the base address lands in *dst (shared memory).
__device__ __forceinline__ void tmemAlloc(uint32_t* dst, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(dst)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Whole warp (the one that allocated).
__device__ __forceinline__ void tmemFree(uint32_t base, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's generic-proxy shared-memory writes visible to the tensor core (async proxy).
__device__ __forceinline__ void fenceSmemForMma() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One thread: D[tmem] (+)= A * B^T for an M x N x 16 step.
__device__ __forceinline__ void mma(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dTmem),
      "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate ? 1u : 0u)
      : "memory");
}

// One thread: arrive on `bar` once all MMAs this thread issued so far have completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddr(bar))
               : "memory");
}

__device__ __forceinline__ void mbarInit(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smemAddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t nowNs() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait (1 s) for the phase with the given parity to complete. Returns false (and raises *error) when it
// gives up.
__device__ __forceinline__ bool mbarWait(uint64_t* bar, uint32_t parity, int* error) {
  if (mbarTryWait(bar, parity)) return true;
  const uint64_t start = nowNs();
  for (uint32_t spin = 1;; ++spin) {
    if (mbarTryWait(bar, parity)) return true;
    if ((spin & 255u) == 0 && nowNs() - start > 1000000000ull) break;
  }
  if (error) atomicExch(error, 1);
  return false;
}

// Warp: 16 consecutive FP32 columns of this warp's 32 TMEM lanes (lane = row); thread t gets row 32 * (warp % 4) + t.
__device__ __forceinline__ void load16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// TMEM address of (lane, column) relative to an allocation base.
__device__ __forceinline__ uint32_t tmemAt(uint32_t base, uint32_t lane, uint32_t col) {
  return base + (lane << 16) + col;
}

// One thread issues D = A(M x K) * B(N x K)^T over K in steps of 16 (A and B K-major tiles, see above); the
// accumulator is overwritten unless `accumulate`. The caller commits (one commit covers every MMA issued before it).
__device__ __forceinline__ void gemmIssue(uint32_t dTmem, const void* a, const void* b, uint32_t M, uint32_t N,
                                          uint32_t K, bool accumulate) {
  const uint32_t idesc = instrDescBf16(M, N);
  const uint64_t aDesc = smemDesc(a, K), bDesc = smemDesc(b, K);
  for (uint32_t k = 0; k < K; k += 16) {
    // Advance the start address by 256 bytes per K step (address field is in 16-byte units).
    const uint64_t step = static_cast<uint64_t>((k / 16) * 256u) >> 4;
    mma(dTmem, aDesc + step, bDesc + step, idesc, accumulate || k > 0);
  }
}

// gemmIssue with the operands' descriptors given (smemDesc / smemDescSbo).
__device__ __forceinline__ void gemmIssueDesc(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t M, uint32_t N,
                                              uint32_t K, bool accumulate) {
  const uint32_t idesc = instrDescBf16(M, N);
  for (uint32_t k = 0; k < K; k += 16) {
    const uint64_t step = static_cast<uint64_t>((k / 16) * 256u) >> 4;
    mma(dTmem, aDesc + step, bDesc + step, idesc, accumulate || k > 0);
  }
}

}  // namespace umma
