// Shared host/device plumbing: status propagation, device buffers, launch sizing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <stdexcept>
#include <string>

#include "../../include/ppf_b200.h"

namespace ppf {

// Error carried out of the engine to the C ABI (which turns it into a
// ppf_status and a thread-local message; nothing in the engine exits).
struct Error : public std::runtime_error {
  ppf_status status;
  Error(ppf_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define PPF_CUDA(x)                                                                      \
  do {                                                                                   \
    cudaError_t e_ = (x);                                                                \
    if (e_ != cudaSuccess) {                                                             \
      throw ::ppf::Error(e_ == cudaErrorMemoryAllocation ? PPF_ERR_OOM : PPF_ERR_CUDA,   \
                         std::string(#x) + ": " + cudaGetErrorString(e_) + " (" __FILE__ \
                         ":" + std::to_string(__LINE__) + ")");                          \
    }                                                                                    \
  } while (0)

#define PPF_REQUIRE(cond, status, msg)               \
  do {                                               \
    if (!(cond)) throw ::ppf::Error((status), (msg)); \
  } while (0)

// The stream that device allocations of the current call are ordered on.
// Every C-ABI entry point that allocates sets it to its context's stream
// (StreamScope); allocations then come from the device's stream-ordered pool
// and freed blocks are reused by later calls without a device synchronise.
inline cudaStream_t& alloc_stream() {
  thread_local cudaStream_t s = nullptr;
  return s;
}

struct StreamScope {
  cudaStream_t prev;
  explicit StreamScope(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
  ~StreamScope() { alloc_stream() = prev; }
};

// Failure injection for tests: when positive, the device allocation that
// brings it to zero fails with PPF_ERR_OUT_OF_MEMORY as a failed cudaMalloc
// would.  Armed per process from PPF_B200_TEST_FAIL_ALLOC=<n> when a context
// is created; zero (off) otherwise.
inline std::atomic<long long>& alloc_failure_countdown() {
  static std::atomic<long long> n{0};
  return n;
}

// Owning device allocation, grown on demand, never shrunk implicitly.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;  // stream the block was allocated on (freed there too)
  bool pooled = false;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes), stream(o.stream), pooled(o.pooled) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      bytes = o.bytes;
      stream = o.stream;
      pooled = o.pooled;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (ptr) {
      if (pooled) cudaFreeAsync(ptr, stream);
      else cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
  }
  void reserve(size_t b) {
    if (b <= bytes) return;
    if (alloc_failure_countdown().load(std::memory_order_relaxed) > 0 &&
        alloc_failure_countdown().fetch_sub(1) == 1)
      throw Error(PPF_ERR_OOM, "device allocation of " + std::to_string(b) + " bytes failed (injected)");
    release();
    size_t want = b < 256 ? 256 : b;
    stream = alloc_stream();
    pooled = stream != nullptr;
    if (pooled) PPF_CUDA(cudaMallocAsync(&ptr, want, stream));
    else PPF_CUDA(cudaMalloc(&ptr, want));
    bytes = want;
  }
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(ptr);
  }
};

inline int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

inline unsigned grid_for(size_t n, int threads, int waves_per_sm = 8) {
  size_t g = (n + threads - 1) / threads;
  size_t cap = (size_t)sm_count() * waves_per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

// Error flags a kernel raises instead of trapping (bounded waits that ran out,
// capacity overflows); the host reads them after the stream synchronises.
enum DeviceFlag : uint32_t {
  kFlagSpinTimeout = 1u << 0,
  kFlagCandidateOverflow = 1u << 1,
  kFlagBadInput = 1u << 2,
  kFlagBadIndex = 1u << 3,
};

}  // namespace ppf
