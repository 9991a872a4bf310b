// Model hash array build (the work of Model::Model, src/cuda/model.cu:43-82):
// pair features and keys of all ordered model pairs, a stable key sort, run
// tables, per-pair vote entries and the key -> run lookup table.
#include <algorithm>

#include "engine.h"
#include "ppf_math.cuh"

namespace ppf {
namespace {

__global__ void pack_points_kernel(const float* __restrict__ xyz, size_t n,
                                   float4* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.f);
}

// Per model point: rows 1-2 of its reference frame and the frame angles.
__global__ void model_points_kernel(const float4* __restrict__ pts, const float4* __restrict__ nrm,
                                    uint32_t n, float4* __restrict__ r1, float4* __restrict__ r2,
                                    float2* __restrict__ ang) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 p4 = pts[i], n4 = nrm[i];
    float3 p = make_float3(p4.x, p4.y, p4.z), q = make_float3(n4.x, n4.y, n4.z);
    FrameYZ f = frame_yz(p, q);
    r1[i] = f.r1;
    r2[i] = f.r2;
    FrameAngles a = frame_angles(q);
    ang[i] = make_float2(a.roty, a.rotz);
  }
}

// Keys of ordered pairs (row r, column i) -> keys[r * n + i]; rows with
// r % ref_df != 0 and self pairs get 0 (src/cuda/kernel.cu:404-477).
// grid.y walks rows, x-blocks walk columns (coalesced key writes).
__global__ void pair_keys_kernel(const float4* __restrict__ pts, const float4* __restrict__ nrm,
                                 uint32_t n, uint32_t ref_df, float d_dist,
                                 uint32_t* __restrict__ keys) {
  for (uint32_t r = blockIdx.y; r < n; r += gridDim.y) {
    uint32_t* row = keys + (size_t)r * n;
    const bool ref_row = (r % ref_df) == 0 && n > 1;
    float4 pr4 = pts[r], nr4 = nrm[r];
    float3 pr = make_float3(pr4.x, pr4.y, pr4.z), nr = make_float3(nr4.x, nr4.y, nr4.z);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      uint32_t k = 0;
      if (ref_row && i != r) {
        float4 pi4 = pts[i], ni4 = nrm[i];
        float4 f = pair_feature(pr, nr, make_float3(pi4.x, pi4.y, pi4.z),
                                make_float3(ni4.x, ni4.y, ni4.z), d_dist);
        k = feature_key(f);
      }
      row[i] = k;
    }
  }
}

// Vote order of the run entries: by key, then m_r, then a hash of the pair
// index.  Grouping a run by m_r lets the vote pass split it into m_r chunks;
// the hash scatters the pairs of one m_r over angles, so that neighbouring
// lanes of a warp rarely count into the same (m_r, bin) cell even when the
// cloud's points come in scan order.
__global__ void order_words_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ pairs,
                                   size_t P, uint32_t n, unsigned long long* __restrict__ words) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < P;
       j += (size_t)gridDim.x * blockDim.x) {
    uint32_t pr = pairs[j];
    uint32_t mr = pr / n;
    words[j] = ((unsigned long long)keys[j] << 32) | (mr << 16) | ((pr * 0x9E3779B1u) >> 16);
  }
}

// Vote entry of each pair in vote order: (m_r mod chunk) << 21 | angle21(u),
// u = the pair's second point in the frame of the first: the top 11 bits are
// the pair's m_r inside its chunk, so the vote kernel forms the cell index
// row * 31 + bin with one multiply-add.  A pair whose u is
// (numerically) zero cannot be binned from angles; its run is flagged for
// exact binning.
__global__ void entries_kernel(const uint32_t* __restrict__ epairs, size_t P, uint32_t n,
                               uint32_t chunk, const float4* __restrict__ pts, const float4* __restrict__ r1,
                               const float4* __restrict__ r2, const uint32_t* __restrict__ first,
                               size_t K, uint32_t* __restrict__ entries,
                               uint8_t* __restrict__ run_flags) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < P;
       j += (size_t)gridDim.x * blockDim.x) {
    uint32_t pr = epairs[j];
    uint32_t mr = pr / n, mi = pr - mr * n;
    FrameYZ f;
    f.r1 = r1[mr];
    f.r2 = r2[mr];
    float4 q4 = pts[mi];
    float2 u = frame_point_yz(f, make_float3(q4.x, q4.y, q4.z));
    entries[j] = ((mr % chunk) << PPF_ANGLE_BITS) | angle21(u);
    if (fabsf(u.x) + fabsf(u.y) < 1e-12f || !isfinite(u.x) || !isfinite(u.y)) {
      // run of position j: last run start <= j
      size_t lo = 0, hi = K;
      while (hi - lo > 1) {
        size_t mid = (lo + hi) >> 1;
        if (first[mid] <= j) lo = mid;
        else hi = mid;
      }
      run_flags[lo] = 1;
    }
  }
}

__device__ __forceinline__ uint32_t ht_slot(uint32_t key, uint32_t mask) {
  return (key * 0x9E3779B1u) & mask;
}

__global__ void ht_build_kernel(const uint32_t* __restrict__ uniq, size_t K, uint32_t mask,
                                uint32_t* __restrict__ ht_keys, uint32_t* __restrict__ ht_runs) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < K;
       r += (size_t)gridDim.x * blockDim.x) {
    uint32_t key = uniq[r];
    if (key == 0) continue;  // key 0 never votes (src/cuda/kernel.cu:491)
    uint32_t s = ht_slot(key, mask);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      uint32_t prev = atomicCAS(&ht_keys[s], 0u, key);
      if (prev == 0u || prev == key) {
        ht_runs[s] = (uint32_t)r;
        break;
      }
      s = (s + 1) & mask;
    }
  }
}

// split[r*(C+1) + c] = first position of run r whose m_r >= c*chunk
// (entries of a run are in m_r order).
__global__ void split_kernel(const uint32_t* __restrict__ epairs, uint32_t n,
                             const uint32_t* __restrict__ first,
                             const uint32_t* __restrict__ count, size_t K, uint32_t chunk,
                             uint32_t n_chunks, uint32_t* __restrict__ split) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < K;
       r += (size_t)gridDim.x * blockDim.x) {
    uint32_t b = first[r], e = b + count[r];
    uint32_t* out = split + r * (n_chunks + 1);
    out[0] = b;
    for (uint32_t c = 1; c < n_chunks; ++c) {
      uint32_t bound = c * chunk;
      uint32_t lo = b, hi = e;  // first position with m_r >= bound
      while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (epairs[mid] / n < bound) lo = mid + 1;
        else hi = mid;
      }
      out[c] = lo;
    }
    out[n_chunks] = e;
  }
}

// Self-checking build (PPF_B200_CHECKS=1): verifies the invariants the vote
// pass relies on and records the first violation as (site, index) in bad[].
__global__ void validate_tables_kernel(const uint32_t* __restrict__ keys, size_t P,
                                       const uint32_t* __restrict__ uniq, const uint32_t* __restrict__ first,
                                       const uint32_t* __restrict__ count, size_t K,
                                       const uint32_t* __restrict__ epairs,
                                       const uint32_t* __restrict__ entries, uint32_t n, uint32_t chunk,
                                       uint32_t n_chunks, const uint32_t* __restrict__ split,
                                       unsigned long long* bad, uint32_t* flags) {
  auto report = [&](unsigned long long site, unsigned long long idx) {
    if (atomicCAS(&bad[0], 0ull, site) == 0ull) bad[1] = idx;
    atomicOr(flags, (uint32_t)kFlagBadIndex);
  };
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < P;
       j += (size_t)gridDim.x * blockDim.x) {
    if (j + 1 < P && keys[j] > keys[j + 1]) report(101, j);
    const uint32_t pr = epairs[j];
    if (pr >= (uint32_t)(n * n)) report(102, j);
    const uint32_t mr = pr / n;
    if ((entries[j] >> PPF_ANGLE_BITS) != mr % chunk) report(103, j);
  }
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < K;
       r += (size_t)gridDim.x * blockDim.x) {
    const uint32_t b = first[r], e = b + count[r];
    if (e > P || count[r] == 0) report(104, r);
    if (r + 1 < K && (uniq[r] >= uniq[r + 1] || first[r + 1] != e)) report(105, r);
    if (keys[b] != uniq[r]) report(106, r);
    for (uint32_t j = b + 1; j < e && j < P; ++j)
      if (epairs[j] / n / chunk < epairs[j - 1] / n / chunk) {
        report(107, r);
        break;
      }
    const uint32_t* sp = split + r * (n_chunks + 1);
    if (sp[0] != b || sp[n_chunks] != e) report(108, r);
    for (uint32_t c = 0; c < n_chunks; ++c) {
      if (sp[c] > sp[c + 1]) report(109, r);
      for (uint32_t j = sp[c]; j < sp[c + 1] && j < P; ++j) {
        const uint32_t mr = epairs[j] / n;
        if (mr < c * chunk || mr >= (c + 1) * chunk) {
          report(110, r);
          break;
        }
      }
    }
  }
}

__global__ void fill_f32(float* p, size_t n, float v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace

bool is_any_device_pointer(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool is_device_pointer(const void* p, int device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  if (a.type != cudaMemoryTypeDevice) return false;
  // A kernel of this context would read another GPU's memory as a peer
  // without peer access enabled: refused before any launch.
  PPF_REQUIRE(a.device == device, PPF_ERR_INVALID_ARGUMENT,
              "device pointer on GPU " + std::to_string(a.device) + " passed to a context on GPU " +
                  std::to_string(device));
  return true;
}

void upload_points(Context& ctx, const float* xyz, size_t n, DevBuf& dst) {
  dst.reserve(n * sizeof(float4));
  if (n == 0) return;
  DevBuf tmp;
  const float* src = xyz;
  if (!is_device_pointer(xyz, ctx.device)) {
    tmp.reserve(n * 3 * sizeof(float));
    PPF_CUDA(cudaMemcpyAsync(tmp.ptr, xyz, n * 3 * sizeof(float), cudaMemcpyHostToDevice,
                             ctx.stream));
    src = tmp.as<float>();
  }
  pack_points_kernel<<<grid_for(n, 256), 256, 0, ctx.stream>>>(src, n, dst.as<float4>());
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
}

void pair_keys_device(Context& ctx, const float4* pts, const float4* nrm, uint32_t n,
                      uint32_t ref_df, float d_dist, uint32_t* keys) {
  if (n == 0) return;
  dim3 block(256);
  dim3 grid((n + 255) / 256, std::min<uint32_t>(n, 65535u));
  pair_keys_kernel<<<grid, block, 0, ctx.stream>>>(pts, nrm, n, ref_df ? ref_df : 1, d_dist, keys);
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
}

void build_model(Context& ctx, ModelTables& t, const float* xyz, const float* nxyz, size_t n,
                 float d_dist) {
  PPF_REQUIRE(n >= 2 && n <= 65535, PPF_ERR_INVALID_ARGUMENT,
              "model size must be in [2, 65535] points");
  PPF_REQUIRE(d_dist > 0.f && std::isfinite(d_dist), PPF_ERR_INVALID_ARGUMENT,
              "d_dist must be a positive finite number");
  cudaStream_t st = ctx.stream;
  t.n = (uint32_t)n;
  t.d_dist = d_dist;
  upload_points(ctx, xyz, n, t.pts);
  upload_points(ctx, nxyz, n, t.nrm);
  t.frame_r1.reserve(n * sizeof(float4));
  t.frame_r2.reserve(n * sizeof(float4));
  t.angles.reserve(n * sizeof(float2));
  t.weights.reserve(n * sizeof(float));
  fill_f32<<<grid_for(n, 256), 256, 0, st>>>(t.weights.as<float>(), n, 1.0f);
  model_points_kernel<<<grid_for(n, 128), 128, 0, st>>>(
      t.pts.as<float4>(), t.nrm.as<float4>(), t.n, t.frame_r1.as<float4>(),
      t.frame_r2.as<float4>(), t.angles.as<float2>());
  PPF_CUDA(cudaGetLastError());
  ctx.launches += 2;

  // keys of all ordered pairs, then the stable sort by key
  t.P = n * n;
  t.keys.reserve(t.P * sizeof(uint32_t));
  t.pairs.reserve(t.P * sizeof(uint32_t));
  pair_keys_device(ctx, t.pts.as<float4>(), t.nrm.as<float4>(), t.n, 1, d_dist,
                   t.keys.as<uint32_t>());
  PPF_CUDA(cudaMemsetAsync(ctx.flags.ptr, 0, sizeof(uint32_t), st));
  size_t l0 = ctx.sort32.launches();
  ctx.sort32.sort(t.keys.as<uint32_t>(), t.pairs.as<uint32_t>(), true, t.P, 0, 32, st,
                  ctx.flags.as<uint32_t>());
  ctx.launches += ctx.sort32.launches() - l0;

  // run tables (the hash array's unique keys, counts and first offsets)
  t.K = build_runs(t.keys.as<uint32_t>(), t.P, t.uniq, t.first, t.count, ctx.scratch, st, &ctx.launches);

  // m_r chunks sized to the vote kernel's shared-memory accumulator
  uint32_t max_chunk = 64;
  // (m_r mod chunk fits the 11 bits above an entry's 21-bit angle)
  while (vote_acc_words(max_chunk + 1) * 4 + kVoteQueueBytes <= (size_t)ctx.vote_smem_limit &&
         max_chunk < (1u << (32 - PPF_ANGLE_BITS)))
    ++max_chunk;
  t.n_chunks = (t.n + max_chunk - 1) / max_chunk;
  t.chunk = (t.n + t.n_chunks - 1) / t.n_chunks;

  // vote entries in vote order; epairs keeps each entry's pair index
  t.entries.reserve(t.P * sizeof(uint32_t));
  t.epairs.reserve(t.P * sizeof(uint32_t));
  t.run_flags.reserve(t.K);
  t.split.reserve(t.K * (t.n_chunks + 1) * sizeof(uint32_t));
  PPF_CUDA(cudaMemsetAsync(t.run_flags.ptr, 0, t.K, st));
  {
    DevBuf words;
    words.reserve(t.P * sizeof(unsigned long long));
    order_words_kernel<<<grid_for(t.P, 256), 256, 0, st>>>(t.keys.as<uint32_t>(), t.pairs.as<uint32_t>(),
                                                            t.P, t.n, words.as<unsigned long long>());
    PPF_CUDA(cudaMemcpyAsync(t.epairs.ptr, t.pairs.ptr, t.P * 4, cudaMemcpyDeviceToDevice, st));
    PPF_CUDA(cudaGetLastError());
    size_t l1 = ctx.sort64.launches();
    ctx.sort64.sort(words.as<unsigned long long>(), t.epairs.as<uint32_t>(), false, t.P, 0, 64, st,
                    ctx.flags.as<uint32_t>());
    ctx.launches += ctx.sort64.launches() - l1 + 1;
    // chunk boundaries of every run (entries are in chunk order within a run)
    split_kernel<<<grid_for(t.K, 256), 256, 0, st>>>(t.epairs.as<uint32_t>(), t.n, t.first.as<uint32_t>(),
                                                      t.count.as<uint32_t>(), t.K, t.chunk, t.n_chunks,
                                                      t.split.as<uint32_t>());
    PPF_CUDA(cudaGetLastError());
    ctx.launches++;
    entries_kernel<<<grid_for(t.P, 256), 256, 0, st>>>(
        t.epairs.as<uint32_t>(), t.P, t.n, t.chunk, t.pts.as<float4>(), t.frame_r1.as<float4>(),
        t.frame_r2.as<float4>(), t.first.as<uint32_t>(), t.K, t.entries.as<uint32_t>(),
        t.run_flags.as<uint8_t>());
    PPF_CUDA(cudaGetLastError());
    ctx.launches++;
  }

  // key -> run table, load factor <= 0.5
  uint32_t cap = 1024;
  while (cap < 2 * t.K) cap <<= 1;
  t.ht_mask = cap - 1;
  t.ht_keys.reserve(cap * sizeof(uint32_t));
  t.ht_runs.reserve(cap * sizeof(uint32_t));
  PPF_CUDA(cudaMemsetAsync(t.ht_keys.ptr, 0, cap * sizeof(uint32_t), st));
  ht_build_kernel<<<grid_for(t.K, 256), 256, 0, st>>>(t.uniq.as<uint32_t>(), t.K, t.ht_mask,
                                                       t.ht_keys.as<uint32_t>(),
                                                       t.ht_runs.as<uint32_t>());
  PPF_CUDA(cudaGetLastError());

  ctx.launches += 1;
  unsigned long long* bad = reinterpret_cast<unsigned long long*>(ctx.flags.as<uint32_t>() + 8);
  if (ctx.checks) {
    PPF_CUDA(cudaMemsetAsync(bad, 0, 24, st));
    validate_tables_kernel<<<grid_for(t.P, 256), 256, 0, st>>>(
        t.keys.as<uint32_t>(), t.P, t.uniq.as<uint32_t>(), t.first.as<uint32_t>(),
        t.count.as<uint32_t>(), t.K, t.epairs.as<uint32_t>(), t.entries.as<uint32_t>(), t.n, t.chunk,
        t.n_chunks, t.split.as<uint32_t>(), bad, ctx.flags.as<uint32_t>());
    PPF_CUDA(cudaGetLastError());
  }
  uint32_t flags = 0;
  unsigned long long badh[2] = {0, 0};
  PPF_CUDA(cudaMemcpyAsync(&flags, ctx.flags.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (ctx.checks) PPF_CUDA(cudaMemcpyAsync(badh, bad, 16, cudaMemcpyDeviceToHost, st));
  PPF_CUDA(cudaStreamSynchronize(st));
  PPF_REQUIRE(!(flags & kFlagSpinTimeout), PPF_ERR_TIMEOUT, "radix sort look-back timed out");
  PPF_REQUIRE(!(flags & kFlagBadIndex), PPF_ERR_INTERNAL,
              "model tables inconsistent: check " + std::to_string(badh[0]) + " at " +
                  std::to_string(badh[1]));
  // The sorts keep scratch of about 22 bytes per sorted pair for reuse by
  // later builds; past 2^28 pairs (16k-point models) that is gigabytes, so
  // it goes back to the pool now.
  if (t.P > (size_t(1) << 28)) {
    ctx.sort32.release();
    ctx.sort64.release();
  }
}

}  // namespace ppf
