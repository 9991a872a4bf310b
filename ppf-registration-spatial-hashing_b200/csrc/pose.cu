// After the vote pass: threshold and order the votes, one pose per kept vote,
// spatial-hash pose clustering and the best pose
// (src/cuda/model.cu:155-244,293-295, src/cuda/ppf.cu:78-93).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.h"
#include "ppf_math.cuh"

namespace ppf {
namespace {

// The rotation and translation tests' dot products with the contraction
// written out, so that the rounding does not depend on how the compiler
// contracts the expression where it is inlined: y*y' rounded, x*x' fused onto
// it, then z*z' and w*w' fused in turn.  This is the rounding of the
// reference's dot() in its clustering kernel (src/cuda/kernel.cu:737-743, as
// nvcc contracts x*x' + y*y' + z*z' + w*w'): on the bench's 31 M poses every
// score equals theirs, while fusing y*y' onto a rounded x*x' instead, in
// either sum, changed scores (up to 950 of them).
__device__ __forceinline__ float dot4_fused(float4 a, float4 b) {
  return fmaf(a.w, b.w, fmaf(a.z, b.z, fmaf(a.x, b.x, __fmul_rn(a.y, b.y))));
}
__device__ __forceinline__ float dot3_fused(float3 a) {
  return fmaf(a.z, a.z, fmaf(a.x, a.x, __fmul_rn(a.y, a.y)));
}

// Keep candidates with count > min_votecount (compared in float, as the
// reference's count_if lambda does, src/cuda/model.cu:164-167).
__global__ void filter_kernel(const unsigned long long* __restrict__ code,
                              const uint32_t* __restrict__ count, size_t n, float min_votecount,
                              unsigned long long* __restrict__ out_code, uint32_t* __restrict__ out_count,
                              uint32_t* __restrict__ n_out) {
  const int lane = threadIdx.x & 31;
  for (size_t b = blockIdx.x * (size_t)blockDim.x; b < n; b += (size_t)gridDim.x * blockDim.x) {
    size_t i = b + threadIdx.x;
    bool keep = i < n && (float)count[i] > min_votecount;
    uint32_t ballot = __ballot_sync(0xffffffffu, keep);
    if (!ballot) continue;
    uint32_t s0 = 0;
    if (lane == 0) s0 = atomicAdd(n_out, (uint32_t)__popc(ballot));
    s0 = __shfl_sync(0xffffffffu, s0, 0);
    if (keep) {
      uint32_t s = s0 + __popc(ballot & ((1u << lane) - 1u));
      out_code[s] = code[i];
      out_count[s] = count[i];
    }
  }
}

// Descending order of the count as a float (the reference sorts with
// thrust::greater<float>, src/cuda/model.cu:155-158): complement of the
// float's bits, which are monotone for non-negative floats.
__global__ void count_key_kernel(const uint32_t* __restrict__ count, size_t n,
                                 uint32_t* __restrict__ key) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    key[i] = ~__float_as_uint((float)count[i]);
}

// Descending count as max_count - count.  For counts below 2^24 the float
// order of the reference's sort and the integer order agree, and the key
// needs only the bits of max_count.
__global__ void count_desc_kernel(const uint32_t* __restrict__ count, size_t n, uint32_t max_count,
                                  uint32_t* __restrict__ key) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    key[i] = max_count - count[i];
}

// Vote codes s_r << 32 | m_r << 6 | bin packed to s_r << kb | m_r << 6 | bin,
// kb = 6 + the bits of the largest m_r: the same order in fewer bits.
template <typename K>
__global__ void pack_codes_kernel(const unsigned long long* code, size_t n, int kb, K* out) {  // may alias
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const unsigned long long c = code[i];
    out[i] = (K)(((c >> 32) << kb) | (uint32_t)c);
  }
}

template <typename K>
__global__ void gather_packed_kernel(const uint32_t* __restrict__ perm, const K* __restrict__ packed,
                                     const uint32_t* __restrict__ count_in, size_t n, int kb,
                                     unsigned long long* __restrict__ code_out,
                                     uint32_t* __restrict__ count_out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t p = perm[i];
    const unsigned long long k = packed[p];
    code_out[i] = ((k >> kb) << 32) | (k & ((1ull << kb) - 1));
    count_out[i] = count_in[p];
  }
}

struct PoseArgs {
  const unsigned long long* codes;
  const uint32_t* counts;
  size_t U;
  const float4* m_pts;
  const float2* m_ang;
  const float* m_w;
  const float4* s_pts;
  const float4* s_nrm;
  float d_dist;
  float* transforms;
  float* trans0;
  float* quats;
  float* weighted;
  uint32_t* cell_keys;
  uint32_t* adj;
  int4* cells3;
};

// trans_calc_kernel2 + vote_weight_kernel + mat2transquat_kernel +
// trans2idx_kernel (src/cuda/kernel.cu:605-699,766-782) for one kept vote.
__global__ void poses_kernel(PoseArgs a) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < a.U;
       i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long code = a.codes[i];
    uint32_t sr = (uint32_t)(code >> 32), mc = (uint32_t)code;
    uint32_t mr = mc >> 6, bin = mc & 63u;
    float T[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) T[k] = 0.f;
    if (!(sr == 0 && mr == 0 && bin == 0)) {  // vote code 0 is skipped (kernel.cu:628)
      float4 mp = a.m_pts[mr];
      float2 ma2 = a.m_ang[mr];
      FrameAngles ma;
      ma.roty = ma2.x;
      ma.rotz = ma2.y;
      float4 sp = a.s_pts[sr], sn = a.s_nrm[sr];
      FrameAngles sa = frame_angles(make_float3(sn.x, sn.y, sn.z));
      vote_pose(bin, make_float3(mp.x, mp.y, mp.z), ma, make_float3(sp.x, sp.y, sp.z), sa, T);
    }
    float* Tout = a.transforms + 16 * i;
#pragma unroll
    for (int k = 0; k < 16; ++k) Tout[k] = T[k];
    float3 t = make_float3(T[3], T[7], T[11]);
    a.trans0[3 * i] = t.x;
    a.trans0[3 * i + 1] = t.y;
    a.trans0[3 * i + 2] = t.z;
    float4 q = pose_quaternion(T);
    a.quats[4 * i] = q.x;
    a.quats[4 * i + 1] = q.y;
    a.quats[4 * i + 2] = q.z;
    a.quats[4 * i + 3] = q.w;
    a.weighted[i] = a.m_w[mr] * a.counts[i];
    int3 c = trans_cell(t, a.d_dist);
    a.cell_keys[i] = cell_key(c.x, c.y, c.z);
    a.cells3[i] = make_int4(c.x, c.y, c.z, 0);
    uint32_t* adj = a.adj + 27 * i;
    int idx = 0;
    for (int di = -1; di < 2; ++di)
      for (int dj = -1; dj < 2; ++dj)
        for (int dk = -1; dk < 2; ++dk, ++idx)
          adj[idx] = (di == 0 && dj == 0 && dk == 0) ? 0u : cell_key(c.x + di, c.y + dj, c.z + dk);
  }
}

struct ClusterArgs {
  size_t U;
  const float* trans0;
  const float* quats;
  const float* weighted;
  const uint32_t* adj;
  const uint32_t* uniq;
  const uint32_t* first;
  const uint32_t* count;
  const uint32_t* map;
  size_t Kc;
  float d_dist;
  int use_l1, use_avg;
  float* scores;
  float* trans;
};

// rot_clustering_kernel (src/cuda/kernel.cu:702-763).  Neighbour translations
// are read from the pre-clustering snapshot (the reference updates them in
// place while other threads read them).
__global__ void cluster_kernel(ClusterArgs a) {
  const float rot_sq = PPF_ROT_THRESH * PPF_ROT_THRESH;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < a.U;
       i += (size_t)gridDim.x * blockDim.x) {
    float3 t = make_float3(a.trans0[3 * i], a.trans0[3 * i + 1], a.trans0[3 * i + 2]);
    float4 q = make_float4(a.quats[4 * i], a.quats[4 * i + 1], a.quats[4 * i + 2], a.quats[4 * i + 3]);
    float c = 1;
    float3 to = t;
    for (int b = 0; b < 27; ++b) {
      uint32_t key = a.adj[27 * i + b];
      if (key == 0u) continue;
      size_t lo = 0, hi = a.Kc;
      while (lo < hi) {
        size_t mid = (lo + hi) >> 1;
        if (a.uniq[mid] < key) lo = mid + 1;
        else hi = mid;
      }
      if (lo == a.Kc || a.uniq[lo] != key) continue;
      uint32_t f = a.first[lo], cnt = a.count[lo];
      for (uint32_t e = 0; e < cnt; ++e) {
        uint32_t j = a.map[f + e];
        float w = a.weighted[j];
        float4 qj = make_float4(a.quats[4 * j], a.quats[4 * j + 1], a.quats[4 * j + 2], a.quats[4 * j + 3]);
        float qd = fabsf(8 * (1 - dot4_fused(q, qj)));
        if (qd < rot_sq) {
          float3 tj = make_float3(a.trans0[3 * j], a.trans0[3 * j + 1], a.trans0[3 * j + 2]);
          if (!a.use_l1) {
            float nd = sqrtf(dot3_fused(v3_sub(t, tj)));
            if (!(nd < a.d_dist)) continue;
          }
          if (a.use_avg) {
            to = v3_scale(c, to);
            to = v3_add(to, v3_scale(w, tj));
            to = v3_scale(1 / (c + w), to);
          }
          c += w;
        }
      }
    }
    a.scores[i] = c;
    a.trans[3 * i] = to.x;
    a.trans[3 * i + 1] = to.y;
    a.trans[3 * i + 2] = to.z;
  }
}

constexpr int kGroup = 32;  // clustering targets per warp

// Also folds the largest squared norm of a finite quaternion into *max_qq
// (float bits; non-negative floats order as their bits).
__global__ void gather_sorted_kernel(const uint32_t* __restrict__ map, size_t U,
                                     const float* __restrict__ quats, const float* __restrict__ trans0,
                                     const float* __restrict__ weighted, float4* __restrict__ qs,
                                     float4* __restrict__ tws, uint32_t* __restrict__ max_qq) {
  float m = 0.f;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < U;
       p += (size_t)gridDim.x * blockDim.x) {
    uint32_t o = map[p];
    const float4 q = make_float4(quats[4 * o], quats[4 * o + 1], quats[4 * o + 2], quats[4 * o + 3]);
    qs[p] = q;
    tws[p] = make_float4(trans0[3 * o], trans0[3 * o + 1], trans0[3 * o + 2], weighted[o]);
    const float qq = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (isfinite(qq)) m = fmaxf(m, qq);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(max_qq, __float_as_uint(m));
}

// Quaternion half-width of the box filters.  The reference's rotation test
// passes only if |8 (1 - q.s)| < rot_sq, so q.s > 1 - rot_sq / 8, and then
// |q - s|^2 = |q|^2 + |s|^2 - 2 q.s < 2 R^2 - 2 + rot_sq / 4 for quaternions
// of norm at most R: every component of q - s is within that root (0.2095
// for unit quaternions).  The small additions cover float rounding.
float quat_margin(float max_qq) {
  const double rot_sq = (double)(2 * PPF_D_ANGLE_HOST) * (double)(2 * PPF_D_ANGLE_HOST);
  const double r2 = std::max(0.0, 2.0 * (double)max_qq - 2.0);
  return (float)(std::sqrt(r2 + rot_sq / 4.0 + 1e-5) + 1e-5);
}

// Whether two different int3 cells share one cell key (then the per-pose
// neighbour lists of cluster_kernel are needed): a sorted position whose key
// equals its predecessor's but whose cell differs.
__global__ void mixed_cells_kernel(const uint32_t* __restrict__ sorted_keys, const uint32_t* __restrict__ map,
                                   const int4* __restrict__ cells3, size_t U, uint32_t* __restrict__ mixed) {
  for (size_t p = 1 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < U;
       p += (size_t)gridDim.x * blockDim.x) {
    if (sorted_keys[p] != sorted_keys[p - 1]) continue;
    const int4 c = cells3[map[p]], c0 = cells3[map[p - 1]];
    if (c.x != c0.x || c.y != c0.y || c.z != c0.z) atomicOr(mixed, 1u);
  }
}

// 4-D grid bucket of a unit quaternion, 16 cells of 0.125 per component.
__device__ __forceinline__ uint32_t quat_bucket(float4 q) {
  auto b = [](float x) { return (uint32_t)min(max(__float2int_rd((x + 1.f) * 8.f), 0), 15); };
  return (b(q.w) << 12) | (b(q.z) << 8) | (b(q.y) << 4) | b(q.x);
}

// Sort key of each pose as a clustering target: its cell key, then its
// rotation bucket, then its quarter-cell of translation (4x4x4 sub-cells of
// d_dist / 4), so the 32 targets of a warp hold similar rotations and, where
// a rotation bucket is crowded, nearby translations.  54 bits.  On the bench's
// pose-dense model the warp boxes then hold 9.0% of the neighbour poses,
// against 13.7% with the rotation bucket alone.
constexpr int kTargetKeyBits = 54;
__global__ void target_keys_kernel(const uint32_t* __restrict__ sorted_keys, const float4* __restrict__ qs,
                                   const float4* __restrict__ tws, float sub_scale, size_t U,
                                   unsigned long long* __restrict__ keys) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < U;
       p += (size_t)gridDim.x * blockDim.x) {
    const float4 tw = tws[p];
    const uint32_t sub = ((uint32_t)__float2int_rd(tw.x * sub_scale) & 3u) << 4 |
                         ((uint32_t)__float2int_rd(tw.y * sub_scale) & 3u) << 2 |
                         ((uint32_t)__float2int_rd(tw.z * sub_scale) & 3u);
    keys[p] = ((unsigned long long)sorted_keys[p] << 22) | ((unsigned long long)quat_bucket(qs[p]) << 6) | sub;
  }
}

// The translation test of the clustering kernels is sqrtf(|t - s|^2) < d.
// sqrtf is non-decreasing in its argument wherever it is checked here, so the
// test equals |t - s|^2 < x_star for x_star the smallest float whose sqrtf
// reaches d, and the square root can be left out.  Every block finds x_star
// by bisection over the float bit patterns with the device's own sqrtf (the
// one the clustering kernels would call), then compares both forms of the
// test on its share of the 2^21 + 1 floats around x_star; out[1] is set on
// any disagreement (or a subnormal x_star, which ftz comparisons would flush),
// and the kernels then keep the square root.  Further from x_star than 2^20
// ulps the argument differs from x_star by more than 1/16 of it, far beyond
// the error of the approximate square root, so both forms agree there too.
constexpr uint32_t kDistWindow = 1u << 20;
__global__ void dist_threshold_kernel(float d, uint32_t* __restrict__ out) {
  __shared__ uint32_t s_star;
  if (threadIdx.x == 0) {
    uint32_t lo = 0u, hi = 0x7f800000u;  // sqrtf(0) < d <= sqrtf(inf) for finite d > 0
    while (hi - lo > 1u) {
      const uint32_t mid = lo + (hi - lo) / 2u;
      if (sqrtf(__uint_as_float(mid)) < d) lo = mid;
      else hi = mid;
    }
    s_star = hi;
    if (blockIdx.x == 0) out[0] = hi;
  }
  __syncthreads();
  const uint32_t star = s_star;
  const float x_star = __uint_as_float(star);
  const uint32_t first = star > kDistWindow ? star - kDistWindow : 0u;
  const uint32_t last = min(star + kDistWindow, 0x7f800000u);
  const uint32_t b = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (b <= last) {
    const float x = __uint_as_float(b);
    if ((sqrtf(x) < d) != (x < x_star)) atomicOr(out + 1, 1u);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && star < 0x00800000u) atomicOr(out + 1, 1u);
}

// Per cell run: its 27 neighbour runs (-1: none / the centre), the number of
// 32-target groups and, if items32 is set, the number of split items (32-target
// tiles x 27 neighbours).
__global__ void run_adjacency_kernel(const uint32_t* __restrict__ first, const uint32_t* __restrict__ count,
                                     size_t Kc, const uint32_t* __restrict__ map,
                                     const int4* __restrict__ cells3, const uint32_t* __restrict__ uniq,
                                     int* __restrict__ adjrun, uint32_t* __restrict__ groups,
                                     uint32_t* __restrict__ items32) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < Kc;
       r += (size_t)gridDim.x * blockDim.x) {
    const uint32_t f = first[r], n = count[r];
    const int4 c0 = cells3[map[f]];
    int b = 0;
    for (int di = -1; di < 2; ++di)
      for (int dj = -1; dj < 2; ++dj)
        for (int dk = -1; dk < 2; ++dk, ++b) {
          int run = -1;
          if (!(di == 0 && dj == 0 && dk == 0)) {
            uint32_t key = cell_key(c0.x + di, c0.y + dj, c0.z + dk);
            size_t lo = 0, hi = Kc;
            while (lo < hi) {
              size_t mid = (lo + hi) >> 1;
              if (uniq[mid] < key) lo = mid + 1;
              else hi = mid;
            }
            if (key != 0u && lo < Kc && uniq[lo] == key) run = (int)lo;
          }
          adjrun[r * 27 + b] = run;
        }
    groups[r] = (n + kGroup - 1) / kGroup;
    if (items32) items32[r] = (n + 31) / 32 * 27;
  }
}

struct GroupArgs {
  const uint32_t* first;
  const uint32_t* count;
  const uint32_t* map;
  const uint32_t* tperm;  // target order: positions sorted by (cell, rotation bucket)
  const int* adjrun;
  const uint32_t* item_off;  // exclusive scan of tiles per run
  size_t Kc;
  uint32_t n_items;
  const float4* qs;
  const float4* tws;
  float d_dist;
  float qmargin;  // quaternion half-width of the box filter (quat_margin)
  float x_star;   // |t - s|^2 < x_star equals sqrtf(|t - s|^2) < d_dist (dist_threshold_kernel)
  int use_x_star;
  int use_l1, use_avg;
  float* scores;
  float* trans;
};

// The reference's two tests for a source pose (rot_clustering_kernel,
// src/cuda/kernel.cu:702-763): |8 (1 - q.s)| < rot_sq, and in L2 mode
// sqrtf(|t - s|^2) < d_dist.  Multiplying by 8 is exact, so the first equals
// |1 - q.s| < rot_sq / 8; the second uses the calibrated threshold when the
// host found it valid.  The dot products round as the reference's.
// Translation test of a clustering launch: none (L1 mode), the calibrated
// threshold, or the square root.
enum TransTest : int { kTransNone = 0, kTransThreshold = 1, kTransSqrt = 2 };

template <int TT>
__device__ __forceinline__ bool cluster_match_t(const GroupArgs& a, float4 q, float3 t, float4 s, float4 sw,
                                                float rot_sq8) {
  bool ok = fabsf(1 - dot4_fused(q, s)) < rot_sq8;
  if (TT != kTransNone) {
    const float3 v = v3_sub(t, make_float3(sw.x, sw.y, sw.z));
    const float d2 = dot3_fused(v);
    ok = ok && (TT == kTransThreshold ? d2 < a.x_star : sqrtf(d2) < a.d_dist);
  }
  return ok;
}

__device__ __forceinline__ bool cluster_match(const GroupArgs& a, float4 q, float3 t, float4 s, float4 sw,
                                              float rot_sq8) {
  return a.use_l1 ? cluster_match_t<kTransNone>(a, q, t, s, sw, rot_sq8)
         : a.use_x_star ? cluster_match_t<kTransThreshold>(a, q, t, s, sw, rot_sq8)
                        : cluster_match_t<kTransSqrt>(a, q, t, s, sw, rot_sq8);
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---- warp-group clustering -------------------------------------------------
// Scores of rot_clustering_kernel (src/cuda/kernel.cu:702-763), cell-major.
// A warp takes 32 targets of one cell (a group; targets ordered by rotation
// bucket, then quarter-cell) and streams the poses of the cell's neighbour
// cells, 32 at a time, into a private ring of kRingStages chunks in shared
// memory with cp.async, kRingStages - 1 chunks ahead of its tests.  For each
// chunk it marks, with one ballot, the sources inside a box around its
// targets: quaternion components within quat_margin of some target's (about
// 0.21: the rotation test bounds the quaternion distance) and, in L2 mode,
// translation components within 1.0001 d_dist.  It then runs the reference's
// tests on the marked sources only, in ascending order.  Sources are visited
// in the reference's order (neighbour b = 0..26, then position), so every
// target adds the same weights in the same order as the reference.  No block
// barrier couples the warps of a block.

constexpr int kWarpBlock = 128;  // threads per block: independent warps
constexpr int kRingStages = 4;

// Position in a group's stream of source chunks: neighbour b, offset o into
// that neighbour run [f, f + n).
struct ChunkPos {
  int b;
  uint32_t o, f, n;
};

// Advances to the next chunk of 32 sources; false past the last neighbour.
__device__ __forceinline__ bool next_chunk(const GroupArgs& a, size_t r, ChunkPos& c) {
  c.o += 32u;
  while (c.o >= c.n) {
    if (++c.b >= 27) return false;
    const int nr = a.adjrun[r * 27 + c.b];
    if (nr < 0) continue;
    c.f = a.first[nr];
    c.n = a.count[nr];
    c.o = 0u;
  }
  return true;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <bool AVG, int TT>
__global__ void __launch_bounds__(kWarpBlock, 8) cluster_warp_kernel(GroupArgs a) {
  __shared__ float4 ring[kWarpBlock / 32][kRingStages][2][32];
  __shared__ float4 marked[kWarpBlock / 32][2][32];
  __shared__ uint32_t ring_len[kWarpBlock / 32][kRingStages];
  const float rot_sq8 = PPF_ROT_THRESH * PPF_ROT_THRESH * 0.125f;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t item = blockIdx.x * (kWarpBlock / 32) + warp;
  if (item >= a.n_items) return;  // uniform over the warp
  size_t lo = 0, hi = a.Kc;  // run r with item_off[r] <= item < item_off[r + 1]
  while (hi - lo > 1) {
    size_t mid = (lo + hi) >> 1;
    if (a.item_off[mid] <= item) lo = mid;
    else hi = mid;
  }
  const size_t r = lo;
  const float kQuatMargin = a.qmargin;
  const float t_margin = a.d_dist * 1.0001f + 1e-6f;
  const uint32_t slot = a.first[r] + (item - a.item_off[r]) * kGroup + lane;
  const bool valid = slot < a.first[r] + a.count[r];
  const uint32_t p = valid ? a.tperm[slot] : 0u;
  // a lane without a target keeps q = 0, which fails the rotation test
  float4 q = make_float4(0, 0, 0, 0), tw = make_float4(0, 0, 0, 0);
  if (valid) {
    q = a.qs[p];
    tw = a.tws[p];
  }
  const float3 t = make_float3(tw.x, tw.y, tw.z);
  const float4 qlo = make_float4(warp_min(valid ? q.x : INFINITY) - kQuatMargin,
                                 warp_min(valid ? q.y : INFINITY) - kQuatMargin,
                                 warp_min(valid ? q.z : INFINITY) - kQuatMargin,
                                 warp_min(valid ? q.w : INFINITY) - kQuatMargin);
  const float4 qhi = make_float4(warp_max(valid ? q.x : -INFINITY) + kQuatMargin,
                                 warp_max(valid ? q.y : -INFINITY) + kQuatMargin,
                                 warp_max(valid ? q.z : -INFINITY) + kQuatMargin,
                                 warp_max(valid ? q.w : -INFINITY) + kQuatMargin);
  float3 tlo = make_float3(0, 0, 0), thi = make_float3(0, 0, 0);
  if (TT != kTransNone) {
    tlo = make_float3(warp_min(valid ? t.x : INFINITY) - t_margin, warp_min(valid ? t.y : INFINITY) - t_margin,
                      warp_min(valid ? t.z : INFINITY) - t_margin);
    thi = make_float3(warp_max(valid ? t.x : -INFINITY) + t_margin, warp_max(valid ? t.y : -INFINITY) + t_margin,
                      warp_max(valid ? t.z : -INFINITY) + t_margin);
  }
  float4(*const wr)[2][32] = ring[warp];
  float4(*const mk)[32] = marked[warp];
  uint32_t* const wm = ring_len[warp];
  // The producer walks the chunk stream kRingStages - 1 chunks ahead of the
  // tests and records each chunk's length; it commits one cp.async group per
  // step (empty past the end), so wait_group<kRingStages - 1> leaves the
  // chunk under test complete.
  ChunkPos pc{-1, 0u, 0u, 0u};
  bool more = next_chunk(a, r, pc);
  uint32_t issued = 0;
  auto produce = [&]() {
    if (more) {
      const uint32_t k = issued % kRingStages;
      if (pc.o + lane < pc.n) {
        cp_async16(&wr[k][0][lane], a.qs + pc.f + pc.o + lane);
        cp_async16(&wr[k][1][lane], a.tws + pc.f + pc.o + lane);
      }
      if (lane == 0) wm[k] = min(32u, pc.n - pc.o);
      ++issued;
      more = next_chunk(a, r, pc);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int s = 0; s < kRingStages - 1; ++s) produce();
  const uint32_t lanes_below = (1u << lane) - 1u;
  float c = 1;
  float3 to = t;
  for (uint32_t used = 0; used < issued; ++used) {
    produce();
    cp_async_wait<kRingStages - 1>();
    __syncwarp();
    const uint32_t k = used % kRingStages;
    bool in = false;
    float4 sj, wj;
    if ((uint32_t)lane < wm[k]) {
      sj = wr[k][0][lane];
      wj = wr[k][1][lane];
      in = sj.x >= qlo.x && sj.x <= qhi.x && sj.y >= qlo.y && sj.y <= qhi.y && sj.z >= qlo.z && sj.z <= qhi.z &&
           sj.w >= qlo.w && sj.w <= qhi.w;
      if (TT != kTransNone)
        in = in && wj.x >= tlo.x && wj.x <= thi.x && wj.y >= tlo.y && wj.y <= thi.y && wj.z >= tlo.z &&
             wj.z <= thi.z;
    }
    const uint32_t mask = __ballot_sync(0xffffffffu, in);
    if (mask) {  // uniform
      // the marked sources, in ascending position, as one list
      if (in) {
        const uint32_t at = __popc(mask & lanes_below);
        mk[0][at] = sj;
        mk[1][at] = wj;
      }
      __syncwarp();
      const int n = __popc(mask);
#pragma unroll 2
      for (int e = 0; e < n; ++e) {
        const float4 sv = mk[0][e], wv = mk[1][e];
        if (cluster_match_t<TT>(a, q, t, sv, wv, rot_sq8)) {
          if (AVG) {
            const float3 tj = make_float3(wv.x, wv.y, wv.z);
            to = v3_scale(c, to);
            to = v3_add(to, v3_scale(wv.w, tj));
            to = v3_scale(1 / (c + wv.w), to);
          }
          c += wv.w;
        }
      }
    }
    __syncwarp();  // every lane is done with this slot and the list before both are refilled
  }
  cp_async_wait<0>();
  if (valid) {
    const uint32_t o = a.map[p];
    a.scores[o] = c;
    a.trans[3 * o] = to.x;
    a.trans[3 * o + 1] = to.y;
    a.trans[3 * o + 2] = to.z;
  }
}

// ---- split clustering (exact sums) ----------------------------------------
// When every weight is an integer and the weights' absolute sum is below
// 2^24, every partial score is an integer that a float holds exactly, so a
// target's score is the same whatever the order of its additions.  The work
// can then be split per (32-target tile, neighbour cell): each warp tests one
// neighbour cell's poses against its 32 targets, in the same box-filtered way
// as cluster_warp_kernel, and adds its partial sum with a float atomic.  A
// lookup with few poses then spreads over up to 27x more warps.

// nonint: some weight is not an integer below 2^24 (or is NaN); abs_sum: the
// sum of |weight| over all poses.
__global__ void weight_check_kernel(const float* __restrict__ w, size_t U, uint32_t* __restrict__ nonint,
                                    unsigned long long* __restrict__ abs_sum) {
  unsigned long long s = 0;
  bool bad = false;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < U; i += (size_t)gridDim.x * blockDim.x) {
    const float x = w[i], ax = fabsf(x);
    if (!(ax < 16777216.f) || x != truncf(x)) bad = true;
    else s += (unsigned long long)ax;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  bad = __any_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
    if (bad) atomicOr(nonint, 1u);
    if (s) atomicAdd(abs_sum, s);
  }
}

// Scores start at 1 (the pose itself); translations stay the snapshot's.
__global__ void split_init_kernel(size_t U, const float* __restrict__ trans0, float* __restrict__ scores,
                                  float* __restrict__ trans) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < U; i += (size_t)gridDim.x * blockDim.x) {
    scores[i] = 1.f;
    trans[3 * i] = trans0[3 * i];
    trans[3 * i + 1] = trans0[3 * i + 1];
    trans[3 * i + 2] = trans0[3 * i + 2];
  }
}

constexpr int kSplitBlock = 256;

__global__ void __launch_bounds__(kSplitBlock) cluster_split_kernel(GroupArgs a) {
  const float rot_sq8 = PPF_ROT_THRESH * PPF_ROT_THRESH * 0.125f;
  const int lane = threadIdx.x & 31;
  const float kQuatMargin = a.qmargin;  // as cluster_warp_kernel
  const float t_margin = a.use_l1 ? INFINITY : a.d_dist * 1.0001f + 1e-6f;
  const uint32_t n_warps = gridDim.x * (kSplitBlock / 32);
  for (uint32_t item = blockIdx.x * (kSplitBlock / 32) + (threadIdx.x >> 5); item < a.n_items;
       item += n_warps) {
    size_t lo = 0, hi = a.Kc;  // run r with item_off[r] <= item < item_off[r + 1]
    while (hi - lo > 1) {
      size_t mid = (lo + hi) >> 1;
      if (a.item_off[mid] <= item) lo = mid;
      else hi = mid;
    }
    const size_t r = lo;
    const uint32_t k = item - a.item_off[r];
    const int nr = a.adjrun[r * 27 + k % 27];
    if (nr < 0) continue;  // uniform over the warp
    const uint32_t slot = a.first[r] + (k / 27) * 32 + lane;
    const bool valid = slot < a.first[r] + a.count[r];
    const uint32_t p = valid ? a.tperm[slot] : 0u;
    float4 q = make_float4(0, 0, 0, 0), tw = make_float4(0, 0, 0, 0);
    if (valid) {
      q = a.qs[p];
      tw = a.tws[p];
    }
    const float3 t = make_float3(tw.x, tw.y, tw.z);
    const float4 qlo = make_float4(warp_min(valid ? q.x : INFINITY) - kQuatMargin,
                                   warp_min(valid ? q.y : INFINITY) - kQuatMargin,
                                   warp_min(valid ? q.z : INFINITY) - kQuatMargin,
                                   warp_min(valid ? q.w : INFINITY) - kQuatMargin);
    const float4 qhi = make_float4(warp_max(valid ? q.x : -INFINITY) + kQuatMargin,
                                   warp_max(valid ? q.y : -INFINITY) + kQuatMargin,
                                   warp_max(valid ? q.z : -INFINITY) + kQuatMargin,
                                   warp_max(valid ? q.w : -INFINITY) + kQuatMargin);
    const float3 tlo = make_float3(warp_min(valid ? t.x : INFINITY) - t_margin,
                                   warp_min(valid ? t.y : INFINITY) - t_margin,
                                   warp_min(valid ? t.z : INFINITY) - t_margin);
    const float3 thi = make_float3(warp_max(valid ? t.x : -INFINITY) + t_margin,
                                   warp_max(valid ? t.y : -INFINITY) + t_margin,
                                   warp_max(valid ? t.z : -INFINITY) + t_margin);
    const uint32_t f = a.first[nr], n = a.count[nr];
    float c = 0;
    for (uint32_t j0 = 0; j0 < n; j0 += 32) {
      float4 sj = make_float4(0, 0, 0, 0), wj = make_float4(0, 0, 0, 0);
      bool in = false;
      if (j0 + lane < n) {
        sj = a.qs[f + j0 + lane];
        wj = a.tws[f + j0 + lane];
        in = sj.x >= qlo.x && sj.x <= qhi.x && sj.y >= qlo.y && sj.y <= qhi.y && sj.z >= qlo.z &&
             sj.z <= qhi.z && sj.w >= qlo.w && sj.w <= qhi.w && wj.x >= tlo.x && wj.x <= thi.x &&
             wj.y >= tlo.y && wj.y <= thi.y && wj.z >= tlo.z && wj.z <= thi.z;
      }
      uint32_t mask = __ballot_sync(0xffffffffu, in);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const float4 s = make_float4(__shfl_sync(0xffffffffu, sj.x, src), __shfl_sync(0xffffffffu, sj.y, src),
                                     __shfl_sync(0xffffffffu, sj.z, src), __shfl_sync(0xffffffffu, sj.w, src));
        const float4 sw = make_float4(__shfl_sync(0xffffffffu, wj.x, src), __shfl_sync(0xffffffffu, wj.y, src),
                                      __shfl_sync(0xffffffffu, wj.z, src), __shfl_sync(0xffffffffu, wj.w, src));
        if (valid && cluster_match(a, q, t, s, sw, rot_sq8)) c += sw.w;
      }
    }
    if (valid && c != 0.f) atomicAdd(&a.scores[a.map[p]], c);
  }
}

// First index of the largest score (thrust::max_element semantics: NaN never
// wins, the first of equal maxima does), in two steps: each block reduces a
// strided share of the scores to (value, index) pairs, then one block
// reduces those and assembles the pose of ppf.cu:78-93 into best[0..15];
// best[16] = score and best[18..19] = index (uint64).
__device__ __forceinline__ void argmax_take(float v, unsigned long long i, float& bv, unsigned long long& bi) {
  if (v > bv || (v == bv && i < bi)) {
    bv = v;
    bi = i;
  }
}

__device__ __forceinline__ void block_argmax(float& bv, unsigned long long& bi) {
  __shared__ float s_v[32];
  __shared__ unsigned long long s_i[32];
  for (int o = 16; o; o >>= 1)
    argmax_take(__shfl_xor_sync(0xffffffffu, bv, o), __shfl_xor_sync(0xffffffffu, bi, o), bv, bi);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s_v[warp] = bv;
    s_i[warp] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) / 32;
    for (int w = 1; w < nw; ++w) argmax_take(s_v[w], s_i[w], bv, bi);
  }
}

__global__ void argmax_partial_kernel(const float* __restrict__ scores, size_t U, float* __restrict__ part_v,
                                      unsigned long long* __restrict__ part_i) {
  float bv = -INFINITY;
  unsigned long long bi = ~0ull;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < U; i += (size_t)gridDim.x * blockDim.x)
    argmax_take(scores[i], i, bv, bi);
  block_argmax(bv, bi);
  if (threadIdx.x == 0) {
    part_v[blockIdx.x] = bv;
    part_i[blockIdx.x] = bi;
  }
}

__global__ void argmax_pose_kernel(const float* __restrict__ part_v, const unsigned long long* __restrict__ part_i,
                                   uint32_t n_part, const float* __restrict__ scores,
                                   const float* __restrict__ transforms, const float* __restrict__ trans,
                                   float* __restrict__ best) {
  float bv = -INFINITY;
  unsigned long long bi = ~0ull;
  for (uint32_t k = threadIdx.x; k < n_part; k += blockDim.x) argmax_take(part_v[k], part_i[k], bv, bi);
  block_argmax(bv, bi);
  if (threadIdx.x == 0) {
    if (bi == ~0ull) bi = 0;  // all scores NaN: first element, as max_element
    for (int k = 0; k < 16; ++k) best[k] = transforms[16 * bi + k];
    best[3] = trans[3 * bi];
    best[7] = trans[3 * bi + 1];
    best[11] = trans[3 * bi + 2];
    best[16] = scores[bi];
    *reinterpret_cast<unsigned long long*>(best + 18) = bi;
  }
}

template <typename T>
T* grow(DevBuf& b, size_t n) {
  b.reserve(n * sizeof(T));
  return b.as<T>();
}

}  // namespace

size_t select_votes(Context& ctx, const Model& m, const SceneData& s, LookupState& st,
                    const unsigned long long* cand_code, const uint32_t* cand_count, size_t n_cand,
                    float min_votecount, uint32_t max_count) {
  cudaStream_t stream = ctx.stream;
  unsigned long long* fcode = grow<unsigned long long>(st.tmp64, n_cand + 1);
  uint32_t* fcount = grow<uint32_t>(st.tmp32a, n_cand + 1);
  PPF_CUDA(cudaMemsetAsync(ctx.counters.ptr, 0, 4, stream));
  filter_kernel<<<grid_for(n_cand, 256), 256, 0, stream>>>(
      cand_code, cand_count, n_cand, min_votecount,
      fcode, fcount, ctx.counters.as<uint32_t>());
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
  uint32_t U = 0;
  PPF_CUDA(cudaMemcpyAsync(&U, ctx.counters.ptr, 4, cudaMemcpyDeviceToHost, stream));
  PPF_CUDA(cudaStreamSynchronize(stream));
  st.U = U;
  if (U == 0) return 0;
  // code ascending (codes are unique), counts carried as values; codes are
  // packed to the bits that s_r and m_r need
  auto bits_for = [](uint64_t x) {
    int b = 0;
    while (b < 64 && (x >> b) != 0) ++b;
    return b;
  };
  const int kb = 6 + bits_for(m.t.n > 1 ? m.t.n - 1 : 1);
  const int code_bits = kb + bits_for(s.n > 1 ? s.n - 1 : 1);
  PPF_CUDA(cudaMemsetAsync(ctx.flags.ptr, 0, 4, stream));
  size_t l0 = ctx.sort64.launches() + ctx.sort32.launches();
  uint32_t* packed32 = nullptr;
  if (code_bits <= 32) {
    packed32 = grow<uint32_t>(st.tmp32c, U);
    pack_codes_kernel<uint32_t><<<grid_for(U, 256), 256, 0, stream>>>(fcode, U, kb, packed32);
    ctx.sort32.sort(packed32, fcount, false, U, 0, code_bits, stream, ctx.flags.as<uint32_t>());
  } else {
    pack_codes_kernel<unsigned long long><<<grid_for(U, 256), 256, 0, stream>>>(fcode, U, kb, fcode);
    ctx.sort64.sort(fcode, fcount, false, U, 0, code_bits, stream, ctx.flags.as<uint32_t>());
  }
  // then stable by count descending
  uint32_t* key2 = grow<uint32_t>(st.tmp32b, U);
  uint32_t* perm = grow<uint32_t>(st.perm, U);
  if (max_count < (1u << 24)) {
    count_desc_kernel<<<grid_for(U, 256), 256, 0, stream>>>(fcount, U, max_count, key2);
    ctx.sort32.sort(key2, perm, true, U, 0, std::max(1, bits_for(max_count)), stream, ctx.flags.as<uint32_t>());
  } else {
    count_key_kernel<<<grid_for(U, 256), 256, 0, stream>>>(fcount, U, key2);
    ctx.sort32.sort(key2, perm, true, U, 0, 32, stream, ctx.flags.as<uint32_t>());
  }
  unsigned long long* codes = grow<unsigned long long>(st.codes, U);
  uint32_t* counts = grow<uint32_t>(st.counts, U);
  if (packed32)
    gather_packed_kernel<uint32_t><<<grid_for(U, 256), 256, 0, stream>>>(perm, packed32, fcount, U, kb, codes,
                                                                         counts);
  else
    gather_packed_kernel<unsigned long long><<<grid_for(U, 256), 256, 0, stream>>>(perm, fcode, fcount, U, kb,
                                                                                   codes, counts);
  PPF_CUDA(cudaGetLastError());
  ctx.launches += 3 + (ctx.sort64.launches() + ctx.sort32.launches() - l0);
  return U;
}

void sort_by_code(Context& ctx, LookupState& st, size_t n) {
  if (n == 0) return;
  cudaStream_t stream = ctx.stream;
  unsigned long long* code = grow<unsigned long long>(st.codes, n);
  uint32_t* count = grow<uint32_t>(st.counts, n);
  PPF_CUDA(cudaMemcpyAsync(code, ctx.cand_codes.ptr, n * 8, cudaMemcpyDeviceToDevice, stream));
  PPF_CUDA(cudaMemcpyAsync(count, ctx.cand_counts.ptr, n * 4, cudaMemcpyDeviceToDevice, stream));
  PPF_CUDA(cudaMemsetAsync(ctx.flags.ptr, 0, 4, stream));
  size_t l0 = ctx.sort64.launches();
  ctx.sort64.sort(code, count, false, n, 0, 64, stream, ctx.flags.as<uint32_t>());
  ctx.launches += ctx.sort64.launches() - l0;
}

void compute_poses(Context& ctx, const Model& m, const SceneData& s, LookupState& st) {
  const size_t U = st.U;
  cudaStream_t stream = ctx.stream;
  PoseArgs a;
  a.codes = st.codes.as<unsigned long long>();
  a.counts = st.counts.as<uint32_t>();
  a.U = U;
  a.m_pts = m.t.pts.as<float4>();
  a.m_ang = m.t.angles.as<float2>();
  a.m_w = m.t.weights.as<float>();
  a.s_pts = s.pts.as<float4>();
  a.s_nrm = s.nrm.as<float4>();
  a.d_dist = m.t.d_dist;
  a.transforms = grow<float>(st.transforms, U * 16);
  a.trans0 = grow<float>(st.trans0, U * 3);
  a.quats = grow<float>(st.quats, U * 4);
  a.weighted = grow<float>(st.weighted, U);
  a.cell_keys = grow<uint32_t>(st.cell_keys, U);
  a.adj = grow<uint32_t>(st.adj, U * 27);
  a.cells3 = grow<int4>(st.cells3, U);
  grow<float>(st.trans, U * 3);
  grow<float>(st.scores, U);
  if (U <= 1) {
    // Every per-vote kernel of the reference returns early when its count is
    // <= 1 (src/cuda/kernel.cu:609,651,667,712,769): a single kept vote leaves
    // zero transforms, zero scores and an all-zero pose.
    PPF_CUDA(cudaMemsetAsync(a.transforms, 0, U * 64, stream));
    PPF_CUDA(cudaMemsetAsync(a.trans0, 0, U * 12, stream));
    PPF_CUDA(cudaMemsetAsync(st.trans.ptr, 0, U * 12, stream));
    PPF_CUDA(cudaMemsetAsync(a.quats, 0, U * 16, stream));
    PPF_CUDA(cudaMemsetAsync(a.weighted, 0, U * 4, stream));
    PPF_CUDA(cudaMemsetAsync(a.cell_keys, 0, U * 4, stream));
    PPF_CUDA(cudaMemsetAsync(st.scores.ptr, 0, U * 4, stream));
    return;
  }
  poses_kernel<<<grid_for(U, 128), 128, 0, stream>>>(a);
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
}

size_t cluster_poses_gpu(Context& ctx, const Model& m, LookupState& st, float* best_score) {
  const size_t U = st.U;
  cudaStream_t stream = ctx.stream;
  float* best = grow<float>(st.best, 32);
  st.cluster_path = 0;
  if (U <= 1) {
    PPF_CUDA(cudaMemsetAsync(best, 0, 32 * sizeof(float), stream));
    *best_score = 0;
    return 0;
  }
  // hash array of the pose cells (src/cuda/model.cu:222-226)
  uint32_t* ck = grow<uint32_t>(st.cells_sorted, U);
  uint32_t* map = grow<uint32_t>(st.cells_map, U);
  PPF_CUDA(cudaMemcpyAsync(ck, st.cell_keys.ptr, U * 4, cudaMemcpyDeviceToDevice, stream));
  PPF_CUDA(cudaMemsetAsync(ctx.flags.ptr, 0, 4, stream));
  size_t l0 = ctx.sort32.launches();
  ctx.sort32.sort(ck, map, true, U, 0, 32, stream, ctx.flags.as<uint32_t>());
  ctx.launches += ctx.sort32.launches() - l0;
  uint32_t* uq = grow<uint32_t>(st.cells_uniq, U);
  uint32_t* fi = grow<uint32_t>(st.cells_first, U);
  uint32_t* ct = grow<uint32_t>(st.cells_count, U);
  size_t Kc = build_runs(ck, U, uq, fi, ct, ctx.scratch, stream, &ctx.launches);
  ClusterArgs a;
  a.U = U;
  a.trans0 = st.trans0.as<float>();
  a.quats = st.quats.as<float>();
  a.weighted = st.weighted.as<float>();
  a.adj = st.adj.as<uint32_t>();
  a.uniq = uq;
  a.first = fi;
  a.count = ct;
  a.map = map;
  a.Kc = Kc;
  a.d_dist = m.t.d_dist;
  a.use_l1 = m.use_l1_norm;
  a.use_avg = m.use_averaged_clusters;
  a.scores = st.scores.as<float>();
  a.trans = st.trans.as<float>();
  // cell-major group scores; per-pose neighbour lists only if two different
  // cells share a hash inside one run
  float4* qs = grow<float4>(st.qs, U);
  float4* tws = grow<float4>(st.tws, U);
  int* adjrun = grow<int>(st.adjrun, Kc * 27);
  uint32_t* item_off = grow<uint32_t>(st.item_off, Kc + 1);
  // Without running averages the score sums may be split across warps when
  // they are exact in any order (integer weights, absolute sum below 2^24).
  const bool may_split = ctx.cluster_split && !m.use_averaged_clusters;
  uint32_t* item_off32 = may_split ? grow<uint32_t>(st.item_off32, Kc + 1) : nullptr;
  // counters: [0] mixed cells, [1] tiles, [2] split items, [3] non-integer
  // weight, [4..5] sum of |weight|, [6] largest squared quaternion norm,
  // [7] x_star of the translation test, [8] x_star unusable
  PPF_CUDA(cudaMemsetAsync(ctx.counters.ptr, 0, 36, stream));
  uint32_t* mixed = ctx.counters.as<uint32_t>();
  const float d_dist = m.t.d_dist;
  const bool calibrate = !m.use_l1_norm && d_dist > 0.f && std::isfinite(d_dist);
  if (calibrate) {
    dist_threshold_kernel<<<(2 * kDistWindow + 1 + 255) / 256, 256, 0, stream>>>(d_dist, mixed + 7);
    ctx.launches++;
  }
  gather_sorted_kernel<<<grid_for(U, 256), 256, 0, stream>>>(map, U, a.quats, a.trans0, a.weighted, qs, tws,
                                                              mixed + 6);
  mixed_cells_kernel<<<grid_for(U, 256), 256, 0, stream>>>(ck, map, st.cells3.as<int4>(), U, mixed);
  run_adjacency_kernel<<<grid_for(Kc, 128), 128, 0, stream>>>(fi, ct, Kc, map, st.cells3.as<int4>(), uq,
                                                              adjrun, item_off, item_off32);
  exclusive_scan_small(item_off, Kc, mixed + 1, stream);
  ctx.launches += 4;
  if (may_split) {
    exclusive_scan_small(item_off32, Kc, mixed + 2, stream);
    weight_check_kernel<<<grid_for(U, 256), 256, 0, stream>>>(a.weighted, U, mixed + 3,
                                                              reinterpret_cast<unsigned long long*>(mixed + 4));
    ctx.launches += 2;
  }
  uint32_t hc[9];
  PPF_CUDA(cudaMemcpyAsync(hc, mixed, sizeof(hc), cudaMemcpyDeviceToHost, stream));
  PPF_CUDA(cudaStreamSynchronize(stream));
  float max_qq, x_star;
  std::memcpy(&max_qq, hc + 6, sizeof(max_qq));
  std::memcpy(&x_star, hc + 7, sizeof(x_star));
  const float qmargin = quat_margin(max_qq);
  const int use_x_star = calibrate && !hc[8] && !ctx.cluster_sqrt;
  // quarter-cell translation bins of the target order
  const float sub_scale = d_dist > 0.f && std::isfinite(d_dist) ? 4.f / d_dist : 0.f;
  const unsigned long long abs_sum = hc[4] | ((unsigned long long)hc[5] << 32);
  const bool split = may_split && !hc[0] && !hc[3] && abs_sum < (1ull << 24) - 1;
  st.cluster_path = split ? 3 : hc[0] ? 2 : 1;
  if (split) {
    // targets of each cell ordered by rotation bucket, as below
    unsigned long long* tkeys = grow<unsigned long long>(st.tmp64, U);
    uint32_t* tperm = grow<uint32_t>(st.tperm, U);
    target_keys_kernel<<<grid_for(U, 256), 256, 0, stream>>>(ck, qs, tws, sub_scale, U, tkeys);
    const size_t l1 = ctx.sort64.launches();
    ctx.sort64.sort(tkeys, tperm, true, U, 0, kTargetKeyBits, stream, ctx.flags.as<uint32_t>());
    ctx.launches += 1 + ctx.sort64.launches() - l1;
    split_init_kernel<<<grid_for(U, 256), 256, 0, stream>>>(U, a.trans0, a.scores, a.trans);
    GroupArgs ta;
    ta.tperm = tperm;
    ta.first = fi;
    ta.count = ct;
    ta.map = map;
    ta.adjrun = adjrun;
    ta.item_off = item_off32;
    ta.Kc = Kc;
    ta.n_items = hc[2];
    ta.qs = qs;
    ta.tws = tws;
    ta.d_dist = m.t.d_dist;
    ta.qmargin = qmargin;
    ta.x_star = x_star;
    ta.use_x_star = use_x_star;
    ta.use_l1 = m.use_l1_norm;
    ta.use_avg = 0;
    ta.scores = a.scores;
    ta.trans = a.trans;
    const size_t blocks = (hc[2] + kSplitBlock / 32 - 1) / (kSplitBlock / 32);
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>(blocks, (size_t)sm_count() * 8));
    cluster_split_kernel<<<grid, kSplitBlock, 0, stream>>>(ta);
    ctx.launches += 2;
  } else if (hc[0]) {
    cluster_kernel<<<grid_for(U, 128), 128, 0, stream>>>(a);
  } else {
    // targets of each cell ordered by rotation bucket
    unsigned long long* tkeys = grow<unsigned long long>(st.tmp64, U);
    uint32_t* tperm = grow<uint32_t>(st.tperm, U);
    target_keys_kernel<<<grid_for(U, 256), 256, 0, stream>>>(ck, qs, tws, sub_scale, U, tkeys);
    ctx.launches++;
    const size_t l1 = ctx.sort64.launches();
    ctx.sort64.sort(tkeys, tperm, true, U, 0, kTargetKeyBits, stream, ctx.flags.as<uint32_t>());
    ctx.launches += ctx.sort64.launches() - l1;
    GroupArgs ta;
    ta.tperm = tperm;
    ta.first = fi;
    ta.count = ct;
    ta.map = map;
    ta.adjrun = adjrun;
    ta.item_off = item_off;
    ta.Kc = Kc;
    ta.n_items = hc[1];
    ta.qs = qs;
    ta.tws = tws;
    ta.d_dist = m.t.d_dist;
    ta.qmargin = qmargin;
    ta.x_star = x_star;
    ta.use_x_star = use_x_star;
    ta.use_l1 = m.use_l1_norm;
    ta.use_avg = m.use_averaged_clusters;
    ta.scores = a.scores;
    ta.trans = a.trans;
    const size_t blocks = (hc[1] + kWarpBlock / 32 - 1) / (kWarpBlock / 32);
    const unsigned grid = (unsigned)std::max<size_t>(1, blocks);
    const int tt = m.use_l1_norm ? kTransNone : use_x_star ? kTransThreshold : kTransSqrt;
    auto launch = [&](auto kernel) { kernel<<<grid, kWarpBlock, 0, stream>>>(ta); };
    if (m.use_averaged_clusters) {
      if (tt == kTransNone) launch(cluster_warp_kernel<true, kTransNone>);
      else if (tt == kTransThreshold) launch(cluster_warp_kernel<true, kTransThreshold>);
      else launch(cluster_warp_kernel<true, kTransSqrt>);
    } else {
      if (tt == kTransNone) launch(cluster_warp_kernel<false, kTransNone>);
      else if (tt == kTransThreshold) launch(cluster_warp_kernel<false, kTransThreshold>);
      else launch(cluster_warp_kernel<false, kTransSqrt>);
    }
  }
  const unsigned n_part = grid_for(U, 256, 2);
  float* part_v = grow<float>(st.argmax_v, n_part);
  unsigned long long* part_i = grow<unsigned long long>(st.argmax_i, n_part);
  argmax_partial_kernel<<<n_part, 256, 0, stream>>>(a.scores, U, part_v, part_i);
  argmax_pose_kernel<<<1, 256, 0, stream>>>(part_v, part_i, n_part, a.scores, st.transforms.as<float>(), a.trans,
                                            best);
  PPF_CUDA(cudaGetLastError());
  ctx.launches += 3;
  float h[20];
  PPF_CUDA(cudaMemcpyAsync(h, best, sizeof(h), cudaMemcpyDeviceToHost, stream));
  PPF_CUDA(cudaStreamSynchronize(stream));
  *best_score = h[16];
  unsigned long long idx;
  memcpy(&idx, h + 18, sizeof(idx));
  return (size_t)idx;
}

}  // namespace ppf
