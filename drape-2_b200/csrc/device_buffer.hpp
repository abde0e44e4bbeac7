// Host-side ownership of device and pinned host memory for the solver and the batch: error checks that throw
// std::runtime_error("cuda: ..."), device buffers zeroed at allocation, and the per-thread host -> device byte counter
// of the handle whose public call is running.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace dbuf {

inline void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("cuda: ") + what + ": " + cudaGetErrorString(e));
}

// Host -> device byte counter of the handle whose public call is running on this thread (see CountTransfers).
inline thread_local uint64_t* g_h2d = nullptr;

struct CountTransfers {
  uint64_t* prev;
  explicit CountTransfers(uint64_t* c) : prev(g_h2d) { g_h2d = c; }
  ~CountTransfers() { g_h2d = prev; }
};

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  // The zeroing runs on the legacy default stream, which is not ordered with the handles' non-blocking streams: wait
  // for it here, or it could land after the uploads and kernels that follow.
  // An allocation of the same size is reused (a rebuild of the same scene allocates nothing).
  void alloc(size_t count) {
    if (!p || count != n) {
      release();
      check(cudaMalloc(&p, sizeof(T) * std::max<size_t>(count, 1)), "cudaMalloc");
      n = count;
    }
    check(cudaMemset(p, 0, sizeof(T) * std::max<size_t>(count, 1)), "cudaMemset");
    check(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize(legacy stream)");
  }
  void upload(const T* src, size_t count, cudaStream_t s) {
    if (count > n || !p) alloc(count);
    if (count) check(cudaMemcpyAsync(p, src, sizeof(T) * count, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(H2D)");
    if (g_h2d) *g_h2d += sizeof(T) * count;
  }
  void upload(const std::vector<T>& v, cudaStream_t s) { upload(v.data(), v.size(), s); }
};

// `count` T in page-locked host memory (zeroed), for copies that graph nodes and async calls read or write.
template <class T>
struct HostPinned {
  T* p = nullptr;
  size_t n = 0;
  HostPinned() = default;
  HostPinned(const HostPinned&) = delete;
  HostPinned& operator=(const HostPinned&) = delete;
  ~HostPinned() { release(); }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count = 1) {
    if (p && n == count) return;
    release();
    check(cudaMallocHost(&p, sizeof(T) * std::max<size_t>(count, 1)), "cudaMallocHost");
    std::memset(static_cast<void*>(p), 0, sizeof(T) * std::max<size_t>(count, 1));
    n = count;
  }
};

}  // namespace dbuf
