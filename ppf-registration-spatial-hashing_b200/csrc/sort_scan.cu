#include "sort_scan.cuh"

namespace ppf {
namespace {

constexpr int kThreads = 256;                    // one thread per digit value
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;         // 2048 keys per tile
constexpr int kRadix = 256;
constexpr unsigned long long kAgg = 1ull << 32;  // status: tile aggregate only
constexpr unsigned long long kInc = 2ull << 32;  // status: inclusive prefix
constexpr int kSpinLimit = 1 << 22;

// Status words of other tiles change while a tile waits on them: read them
// with a load the compiler must repeat.
__device__ __forceinline__ unsigned long long load_status(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ void store_status(unsigned long long* p, unsigned long long v) {
  *reinterpret_cast<volatile unsigned long long*>(p) = v;
}

// Exclusive scan of one value per thread over a 256-thread block.
__device__ __forceinline__ uint32_t block_excl_scan256(uint32_t v, uint32_t* s_warp,
                                                       uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kWarps ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kWarps) s_warp[lane] = w;
  }
  __syncthreads();
  uint32_t warp_excl = warp ? s_warp[warp - 1] : 0;
  if (total) *total = s_warp[kWarps - 1];
  uint32_t r = warp_excl + x - v;
  __syncthreads();
  return r;
}

template <typename K>
__global__ void __launch_bounds__(kThreads) rs_histogram(const K* __restrict__ keys, size_t n,
                                                         int begin_bit, int passes,
                                                         uint32_t* __restrict__ hist) {
  __shared__ uint32_t sh[8][kRadix];
  for (int i = threadIdx.x; i < 8 * kRadix; i += blockDim.x) sh[i / kRadix][i % kRadix] = 0;
  __syncthreads();
  // one shared atomic per distinct digit of a warp: sorted or skewed keys
  // (long runs of equal digits) would otherwise serialise on one counter
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    K k = keys[i];
    const uint32_t active = __activemask();
    const int lane = threadIdx.x & 31;
    for (int p = 0; p < passes; ++p) {
      const uint32_t d = (uint32_t)(k >> (begin_bit + 8 * p)) & 0xffu;
      const uint32_t peers = __match_any_sync(active, d);
      if (lane == __ffs(peers) - 1) atomicAdd(&sh[p][d], (uint32_t)__popc(peers));
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) {
    uint32_t v = sh[i / kRadix][i % kRadix];
    if (v) atomicAdd(&hist[i], v);
  }
}

template <typename K>
__global__ void __launch_bounds__(kThreads) rs_onesweep(
    const K* __restrict__ kin, const uint32_t* __restrict__ vin, bool vin_iota,
    K* __restrict__ kout, uint32_t* __restrict__ vout, size_t n, int shift,
    const uint32_t* __restrict__ pass_hist, unsigned long long* status, uint32_t* tile_counter,
    uint32_t* flags, uint32_t stall_tile, int spin_limit) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_whist[kWarps][kRadix];
  __shared__ uint32_t s_tile_start[kRadix];
  __shared__ uint32_t s_global[kRadix];
  __shared__ uint32_t s_scan[kWarps];
  __shared__ K s_keys[kTile];
  __shared__ uint32_t s_vals[kTile];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
  for (int i = tid; i < kWarps * kRadix; i += kThreads) (&s_whist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const size_t base = (size_t)tile * kTile;

  K key[kItems];
  uint32_t val[kItems], dig[kItems], rank[kItems];
  const size_t wbase = base + (size_t)warp * 32 * kItems;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    size_t idx = wbase + (size_t)i * 32 + lane;
    bool ok = idx < n;
    key[i] = ok ? kin[idx] : K(0);
    val[i] = ok ? (vin_iota ? (uint32_t)idx : vin[idx]) : 0u;
    dig[i] = ok ? ((uint32_t)(key[i] >> shift) & 0xffu) : 256u;
  }
  // Warp multisplit: rank of each item among equal digits, in input order.
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    uint32_t d = dig[i];
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t before = d < 256u ? s_whist[warp][d] : 0u;
    __syncwarp();
    if (d < 256u && lane == __ffs(peers) - 1) s_whist[warp][d] = before + __popc(peers);
    __syncwarp();
    rank[i] = before + __popc(peers & lt);
  }
  __syncthreads();
  // Per digit (thread tid = digit): warp exclusive offsets and the tile count.
  uint32_t run = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    uint32_t c = s_whist[w][tid];
    s_whist[w][tid] = run;
    run += c;
  }
  const uint32_t tile_cnt = run;
  s_tile_start[tid] = block_excl_scan256(tile_cnt, s_scan, nullptr);
  const uint32_t pass_base = block_excl_scan256(pass_hist[tid], s_scan, nullptr);
  // Decoupled look-back for this digit.
  unsigned long long* my = status + (size_t)tile * kRadix + tid;
  uint32_t excl = 0;
  const bool publish = tile != stall_tile;  // the test hook's silent tile
  if (tile == 0) {
    store_status(my, kInc | (unsigned long long)tile_cnt);
  } else {
    if (publish) store_status(my, kAgg | (unsigned long long)tile_cnt);
    long long t = (long long)tile - 1;
    while (t >= 0) {
      const unsigned long long* p = status + (size_t)t * kRadix + tid;
      unsigned long long v = load_status(p);
      int spins = 0;
      while ((v >> 32) == 0) {
        if (++spins > spin_limit) {
          atomicOr(flags, (uint32_t)kFlagSpinTimeout);
          v = kInc;
          break;
        }
        __nanosleep(32);
        v = load_status(p);
      }
      excl += (uint32_t)v;
      if ((v >> 32) == 2) break;
      --t;
    }
    if (publish) store_status(my, kInc | (unsigned long long)(excl + tile_cnt));
  }
  s_global[tid] = pass_base + excl;
  __syncthreads();
  // Tile-local sort through shared memory, then digit-contiguous writes.
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    uint32_t d = dig[i];
    if (d < 256u) {
      uint32_t pos = s_tile_start[d] + s_whist[warp][d] + rank[i];
      s_keys[pos] = key[i];
      s_vals[pos] = val[i];
    }
  }
  __syncthreads();
  const size_t remain = n - base;
  const uint32_t valid = remain < (size_t)kTile ? (uint32_t)remain : (uint32_t)kTile;
  for (uint32_t p = tid; p < valid; p += kThreads) {
    K k = s_keys[p];
    uint32_t d = (uint32_t)(k >> shift) & 0xffu;
    size_t o = (size_t)s_global[d] + (p - s_tile_start[d]);
    kout[o] = k;
    vout[o] = s_vals[p];
  }
}

// ---- run tables --------------------------------------------------------
constexpr int kRunThreads = 256;
constexpr int kRunItems = 16;
constexpr int kRunTile = kRunThreads * kRunItems;

__global__ void __launch_bounds__(kRunThreads) runs_count(const uint32_t* __restrict__ k,
                                                           size_t n, uint32_t* __restrict__ tile_heads) {
  __shared__ uint32_t s_scan[kWarps];
  size_t base = (size_t)blockIdx.x * kRunTile + (size_t)threadIdx.x * kRunItems;
  uint32_t c = 0;
  for (int i = 0; i < kRunItems; ++i) {
    size_t p = base + i;
    if (p < n && (p == 0 || k[p] != k[p - 1])) ++c;
  }
  uint32_t total;
  block_excl_scan256(c, s_scan, &total);
  if (threadIdx.x == 0) tile_heads[blockIdx.x] = total;
}

// Exclusive scan of the per-tile head counts by one block (serial chunks).
__global__ void __launch_bounds__(kRunThreads) runs_scan_tiles(uint32_t* __restrict__ v, size_t m,
                                                               uint32_t* __restrict__ total_out) {
  __shared__ uint32_t s_scan[kWarps];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (size_t b = 0; b < m; b += kRunThreads) {
    size_t i = b + threadIdx.x;
    uint32_t x = i < m ? v[i] : 0u;
    uint32_t tot;
    uint32_t e = block_excl_scan256(x, s_scan, &tot);
    if (i < m) v[i] = s_carry + e;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total_out = s_carry;
}

__global__ void __launch_bounds__(kRunThreads) runs_emit(const uint32_t* __restrict__ k, size_t n,
                                                          const uint32_t* __restrict__ tile_off,
                                                          uint32_t* __restrict__ uniq,
                                                          uint32_t* __restrict__ first) {
  __shared__ uint32_t s_scan[kWarps];
  size_t base = (size_t)blockIdx.x * kRunTile + (size_t)threadIdx.x * kRunItems;
  uint32_t c = 0;
  for (int i = 0; i < kRunItems; ++i) {
    size_t p = base + i;
    if (p < n && (p == 0 || k[p] != k[p - 1])) ++c;
  }
  uint32_t r = tile_off[blockIdx.x] + block_excl_scan256(c, s_scan, nullptr);
  for (int i = 0; i < kRunItems; ++i) {
    size_t p = base + i;
    if (p < n && (p == 0 || k[p] != k[p - 1])) {
      uniq[r] = k[p];
      first[r] = (uint32_t)p;
      ++r;
    }
  }
}

__global__ void runs_lengths(const uint32_t* __restrict__ first, size_t K, size_t n,
                             uint32_t* __restrict__ count) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < K;
       r += (size_t)gridDim.x * blockDim.x) {
    size_t end = (r + 1 < K) ? first[r + 1] : n;
    count[r] = (uint32_t)(end - first[r]);
  }
}

}  // namespace

template <typename K>
void RadixSorter<K>::sort(K* keys, uint32_t* vals, bool vals_iota, size_t n, int begin_bit,
                          int end_bit, cudaStream_t st, uint32_t* d_flags) {
  if (n == 0) return;
  PPF_REQUIRE(n < (1ull << 32), PPF_ERR_INVALID_ARGUMENT, "radix sort: more than 2^32 elements");
  const int passes = (end_bit - begin_bit + 7) / 8;
  if (passes <= 0) {
    if (vals_iota) {
      // identity permutation: still produce the values
      PPF_REQUIRE(false, PPF_ERR_INTERNAL, "radix sort with no digits");
    }
    return;
  }
  const size_t tiles = (n + kTile - 1) / kTile;
  kalt_.reserve(n * sizeof(K));
  valt_.reserve(n * sizeof(uint32_t));
  hist_.reserve(8 * kRadix * sizeof(uint32_t));
  status_.reserve(tiles * kRadix * sizeof(unsigned long long));
  counters_.reserve(8 * sizeof(uint32_t));
  PPF_CUDA(cudaMemsetAsync(hist_.ptr, 0, passes * kRadix * sizeof(uint32_t), st));
  rs_histogram<K><<<grid_for(n, kThreads, 4), kThreads, 0, st>>>(keys, n, begin_bit, passes,
                                                                  hist_.as<uint32_t>());
  PPF_CUDA(cudaGetLastError());
  launches_ += 1;
  K* kin = keys;
  uint32_t* vin = vals;
  K* kout = kalt_.as<K>();
  uint32_t* vout = valt_.as<uint32_t>();
  bool iota = vals_iota;
  // the test hook (arm_stall) applies to the first pass of a sort with a tile 1
  const bool stall = stall_ && tiles > 1;
  if (stall) stall_ = false;
  for (int p = 0; p < passes; ++p) {
    PPF_CUDA(cudaMemsetAsync(status_.ptr, 0, tiles * kRadix * sizeof(unsigned long long), st));
    PPF_CUDA(cudaMemsetAsync(counters_.ptr, 0, sizeof(uint32_t), st));
    const bool stall_here = stall && p == 0;
    rs_onesweep<K><<<(unsigned)tiles, kThreads, 0, st>>>(
        kin, vin, iota, kout, vout, n, begin_bit + 8 * p, hist_.as<uint32_t>() + p * kRadix,
        status_.as<unsigned long long>(), counters_.as<uint32_t>(), d_flags, stall_here ? 1u : 0xffffffffu,
        stall_here ? 4096 : kSpinLimit);
    PPF_CUDA(cudaGetLastError());
    launches_ += 1;
    iota = false;
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  if (kin != keys) {
    PPF_CUDA(cudaMemcpyAsync(keys, kin, n * sizeof(K), cudaMemcpyDeviceToDevice, st));
    PPF_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  }
  // A look-back that gave up leaves the order undefined: stop here.
  uint32_t f = 0;
  PPF_CUDA(cudaMemcpyAsync(&f, d_flags, sizeof(f), cudaMemcpyDeviceToHost, st));
  PPF_CUDA(cudaStreamSynchronize(st));
  if (f & kFlagSpinTimeout) {
    const uint32_t clear = f & ~(uint32_t)kFlagSpinTimeout;
    PPF_CUDA(cudaMemcpyAsync(d_flags, &clear, sizeof(clear), cudaMemcpyHostToDevice, st));
    PPF_CUDA(cudaStreamSynchronize(st));
    throw Error(PPF_ERR_TIMEOUT, "radix sort look-back timed out (" + std::to_string(n) + " keys)");
  }
}

template class RadixSorter<uint32_t>;
template class RadixSorter<unsigned long long>;

void exclusive_scan_small(uint32_t* v, size_t n, uint32_t* total_dev, cudaStream_t st) {
  runs_scan_tiles<<<1, kRunThreads, 0, st>>>(v, n, total_dev);
  PPF_CUDA(cudaGetLastError());
}

namespace {
// Run heads per tile, scanned: scratch[t] = runs before tile t,
// scratch[tiles] = K.  Returns K (one stream synchronisation).
size_t count_runs(const uint32_t* sorted_keys, size_t n, DevBuf& scratch, cudaStream_t st) {
  const size_t tiles = (n + kRunTile - 1) / kRunTile;
  scratch.reserve((tiles + 1) * sizeof(uint32_t));
  uint32_t* th = scratch.as<uint32_t>();
  runs_count<<<(unsigned)tiles, kRunThreads, 0, st>>>(sorted_keys, n, th);
  runs_scan_tiles<<<1, kRunThreads, 0, st>>>(th, tiles, th + tiles);
  PPF_CUDA(cudaGetLastError());
  uint32_t K = 0;
  PPF_CUDA(cudaMemcpyAsync(&K, th + tiles, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  PPF_CUDA(cudaStreamSynchronize(st));
  return K;
}

void emit_runs(const uint32_t* sorted_keys, size_t n, size_t K, uint32_t* uniq, uint32_t* first, uint32_t* count,
               DevBuf& scratch, cudaStream_t st) {
  const size_t tiles = (n + kRunTile - 1) / kRunTile;
  runs_emit<<<(unsigned)tiles, kRunThreads, 0, st>>>(sorted_keys, n, scratch.as<uint32_t>(), uniq, first);
  runs_lengths<<<grid_for(K, 256), 256, 0, st>>>(first, K, n, count);
  PPF_CUDA(cudaGetLastError());
}
}  // namespace

size_t build_runs(const uint32_t* sorted_keys, size_t n, uint32_t* uniq, uint32_t* first,
                  uint32_t* count, DevBuf& scratch, cudaStream_t st, size_t* launches) {
  if (n == 0) return 0;
  const size_t K = count_runs(sorted_keys, n, scratch, st);
  emit_runs(sorted_keys, n, K, uniq, first, count, scratch, st);
  if (launches) *launches += 4;
  return K;
}

size_t build_runs(const uint32_t* sorted_keys, size_t n, DevBuf& uniq, DevBuf& first, DevBuf& count,
                  DevBuf& scratch, cudaStream_t st, size_t* launches) {
  if (n == 0) return 0;
  const size_t K = count_runs(sorted_keys, n, scratch, st);
  uniq.reserve(K * sizeof(uint32_t));
  first.reserve(K * sizeof(uint32_t));
  count.reserve(K * sizeof(uint32_t));
  emit_runs(sorted_keys, n, K, uniq.as<uint32_t>(), first.as<uint32_t>(), count.as<uint32_t>(), scratch, st);
  if (launches) *launches += 4;
  return K;
}

}  // namespace ppf
