// Shared-memory atomic throughput of a B200 SM, measured the way the vote
// pass uses shared memory: one persistent 1024-thread block per SM with a
// large dynamic shared accumulator, non-returning 32-bit atomicAdd, kUnroll
// independent atomics per lane per pass.  The vote pass is limited by these
// atomics, not by DRAM, so bench.py rates it against this measured rate as
// well as against the copy bandwidth.
//
// Address patterns (lane l of warp w, pass p, atomic u; every base is a
// multiple of 64 words, so a word's bank is its offset from the base):
//   0  32 distinct words in 32 distinct banks (one bank wavefront);
//   1  16 banks, two distinct words in each (two wavefronts);
//   2  one word for all 32 lanes.
// Each block records its SM cycles (clock64) between two block barriers.
#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

namespace {

constexpr int kThreads = 1024;
constexpr int kWarps = kThreads / 32;
constexpr int kUnroll = 8;
// 128 KiB of accumulator (one block per SM either way: 1024 threads need
// half of the SM's 2048, and two blocks' accumulators would not fit).  One
// pass covers half of it (kUnroll x kWarps x 64 words), and passes alternate
// halves, so each atomic's address is a per-pass register plus a constant.
constexpr uint32_t kWords = 32768;
constexpr uint32_t kHalf = kUnroll * kWarps * 64;
static_assert(2 * kHalf == kWords, "one pass covers half the accumulator");

__global__ void __launch_bounds__(kThreads, 1)
shared_atomic_kernel(int pattern, uint32_t passes, unsigned long long* cycles, uint32_t* sink) {
  extern __shared__ uint32_t acc[];
  for (uint32_t i = threadIdx.x; i < kWords; i += kThreads) acc[i] = 0u;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t off;
  if (pattern == 0) off = lane;
  else if (pattern == 1) off = (lane & 15u) + (lane >> 4) * 32u;
  else off = 0u;
  const unsigned long long t0 = clock64();
  for (uint32_t p = 0; p < passes; ++p) {
    uint32_t* const row = acc + (p & 1u) * kHalf + warp * 64u + off;
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) atomicAdd(row + u * kWarps * 64u, 1u);
  }
  __syncthreads();
  const unsigned long long t1 = clock64();
  if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
  // keep the counts observable
  uint32_t s = 0;
  for (uint32_t i = threadIdx.x; i < kWords; i += kThreads) s += acc[i];
  atomicAdd(sink, s);
}

}  // namespace

extern "C" {

// Runs the probe on `device` with one block per SM and returns, in
// *warp_atomics_per_sm_cycle, the warp-wide atomic instructions one SM
// completes per cycle (the mean over blocks of 32 warps x passes x kUnroll /
// cycles), and in *ms the launch's duration by CUDA events.  0 on success,
// else the CUDA error code.  Allocates and frees its own 2 small buffers.
int ppf_peak_shared_atomics(int device, int pattern, uint32_t passes, double* warp_atomics_per_sm_cycle,
                            double* ms) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return (int)e;
  int sms = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return (int)e;
  const size_t smem = kWords * sizeof(uint32_t);
  if ((e = cudaFuncSetAttribute(shared_atomic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
      cudaSuccess)
    return (int)e;
  unsigned long long* cycles = nullptr;
  uint32_t* sink = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  std::vector<unsigned long long> host;
  double sum = 0.0;
  float t = 0.f;
  if ((e = cudaMalloc(&cycles, sizeof(unsigned long long) * sms)) != cudaSuccess) goto done;
  if ((e = cudaMalloc(&sink, sizeof(uint32_t))) != cudaSuccess) goto done;
  if ((e = cudaEventCreate(&a)) != cudaSuccess || (e = cudaEventCreate(&b)) != cudaSuccess) goto done;
  cudaEventRecord(a);
  shared_atomic_kernel<<<sms, kThreads, smem>>>(pattern, passes, cycles, sink);
  cudaEventRecord(b);
  if ((e = cudaGetLastError()) != cudaSuccess) goto done;
  if ((e = cudaEventSynchronize(b)) != cudaSuccess) goto done;
  cudaEventElapsedTime(&t, a, b);
  host.resize(sms);
  if ((e = cudaMemcpy(host.data(), cycles, sizeof(unsigned long long) * sms, cudaMemcpyDeviceToHost)) !=
      cudaSuccess)
    goto done;
  for (int i = 0; i < sms; ++i) sum += (double)kWarps * passes * kUnroll / (double)host[i];
  *warp_atomics_per_sm_cycle = sum / sms;
  *ms = t;
done:
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (cycles) cudaFree(cycles);
  if (sink) cudaFree(sink);
  return (int)e;
}

}  // extern "C"
