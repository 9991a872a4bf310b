// The reference's cpu_clustering path on the device: greedy pose clustering
// (Model::ClusterTransformationsCPU, src/cuda/model.cu:246-266, clusterPoses
// and posesWithinErrorBounds, src/transformation_clustering.cpp:62-137).
//
// Poses are taken in vote order (the kept votes come ordered by count
// descending, so the reference's sort by votes keeps them as they are, ties
// in vote code order).  A pose joins the first existing cluster whose first
// pose is within d_dist in translation and 2*pi/30 in rotation, or starts a
// new cluster.  Done in chunks of poses: one grid-wide pass finds, for every
// pose of the chunk, its first matching cluster among those that existed
// before the chunk; one block then walks the chunk's remaining poses in
// order, each unassigned one starting a cluster that the block's threads
// test against every later unassigned pose at once.  The three clusters with
// most votes (ties: the earlier cluster) are averaged over their poses in
// order: translations, and quaternions in 4-D, renormalised.  The float
// arithmetic is that of the host restatement, operation for operation
// (correctly rounded square roots and divisions, no fused multiply-adds);
// atan2f is CUDA's, so a rotation difference within an ulp or two of the
// threshold may decide differently from the host's.
#include <cstring>

#include "engine.h"

namespace ppf {
namespace {

constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kGreedyChunk = 16384;

struct GPose {
  float4 a, b, c;  // R00 R01 R02 R10 | R11 R12 R20 R21 | R22 tx ty tz
};

// Barrier that every warp reaches converged, with shared memory fenced on
// both sides (single-thread work precedes several barriers here).
__device__ __forceinline__ void block_sync() {
  __syncwarp();
  __threadfence_block();
  __syncthreads();
  __threadfence_block();
}

__device__ __forceinline__ float fadd(float x, float y) { return __fadd_rn(x, y); }
__device__ __forceinline__ float fsub(float x, float y) { return __fsub_rn(x, y); }
__device__ __forceinline__ float fmul(float x, float y) { return __fmul_rn(x, y); }

__device__ __forceinline__ void unpack(const GPose& p, float R[9], float t[3]) {
  R[0] = p.a.x; R[1] = p.a.y; R[2] = p.a.z; R[3] = p.a.w;
  R[4] = p.b.x; R[5] = p.b.y; R[6] = p.b.z; R[7] = p.b.w;
  R[8] = p.c.x; t[0] = p.c.y; t[1] = p.c.z; t[2] = p.c.w;
}

// Quaternion (x, y, z, w) of a rotation matrix (trace / largest diagonal).
__device__ void quat_xyzw(const float* m, float q[4]) {
  const float tr = fadd(fadd(m[0], m[4]), m[8]);
  if (tr > 0.f) {
    float s = __fsqrt_rn(fadd(tr, 1.0f));
    q[3] = fmul(0.5f, s);
    s = __fdiv_rn(0.5f, s);
    q[0] = fmul(fsub(m[7], m[5]), s);
    q[1] = fmul(fsub(m[2], m[6]), s);
    q[2] = fmul(fsub(m[3], m[1]), s);
    return;
  }
  int i = 0;
  if (m[4] > m[0]) i = 1;
  if (m[8] > m[4 * i]) i = 2;
  const int j = (i + 1) % 3, k = (j + 1) % 3;
  float s = __fsqrt_rn(fadd(fsub(fsub(m[4 * i], m[4 * j]), m[4 * k]), 1.0f));
  q[i] = fmul(0.5f, s);
  s = __fdiv_rn(0.5f, s);
  q[3] = fmul(fsub(m[3 * k + j], m[3 * j + k]), s);
  q[j] = fmul(fadd(m[3 * j + i], m[3 * i + j]), s);
  q[k] = fmul(fadd(m[3 * k + i], m[3 * i + k]), s);
}

__device__ bool close_enough(const GPose& A, const GPose& B, float trans_thresh, float rot_thresh) {
  float Ra[9], Rb[9], ta[3], tb[3];
  unpack(A, Ra, ta);
  unpack(B, Rb, tb);
  const float dx = fsub(ta[0], tb[0]), dy = fsub(ta[1], tb[1]), dz = fsub(ta[2], tb[2]);
  const float dist = __fsqrt_rn(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
  if (!(dist < trans_thresh)) return false;
  float M[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float s = 0.f;
      for (int k = 0; k < 3; ++k) s = fadd(s, fmul(Ra[3 * k + i], Rb[3 * k + j]));
      M[3 * i + j] = s;
    }
  float q[4];
  quat_xyzw(M, q);
  const float nv = __fsqrt_rn(fadd(fadd(fmul(q[0], q[0]), fmul(q[1], q[1])), fmul(q[2], q[2])));
  const float angle = nv != 0.f ? fmul(2.f, atan2f(nv, fabsf(q[3]))) : 0.f;
  return fabsf(angle) < rot_thresh;
}

// Rotation block and translation of each row-major pose; an all-zero block
// (a pose never computed) is the identity, the polar factor Eigen returns.
__global__ void prep_kernel(const float* __restrict__ T, size_t U, GPose* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < U; i += (size_t)gridDim.x * blockDim.x) {
    const float* P = T + 16 * i;
    float R[9];
    bool zero = true;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        R[3 * r + c] = P[4 * r + c];
        zero = zero && R[3 * r + c] == 0.f;
      }
    if (zero)
      for (int k = 0; k < 9; ++k) R[k] = (k % 4 == 0) ? 1.f : 0.f;
    GPose g;
    g.a = make_float4(R[0], R[1], R[2], R[3]);
    g.b = make_float4(R[4], R[5], R[6], R[7]);
    g.c = make_float4(R[8], P[3], P[7], P[11]);
    out[i] = g;
  }
}

// First cluster (among those existing before the chunk) that each pose of
// [b, e) matches.
__global__ void match_kernel(const GPose* __restrict__ poses, size_t b, size_t e,
                             const GPose* __restrict__ seeds, const uint32_t* __restrict__ n_seeds,
                             uint32_t* __restrict__ assign, float tt, float rt) {
  const uint32_t C = *n_seeds;
  for (size_t i = b + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < e; i += (size_t)gridDim.x * blockDim.x) {
    const GPose p = poses[i];
    uint32_t a = kNone;
    for (uint32_t c = 0; c < C; ++c)
      if (close_enough(p, seeds[c], tt, rt)) {
        a = c;
        break;
      }
    assign[i] = a;
  }
}

// One block: the chunk's poses without a cluster, in order; each one still
// unassigned starts a cluster, which every later unassigned pose of the chunk
// then tests.
__global__ void __launch_bounds__(1024) resolve_kernel(const GPose* __restrict__ poses, size_t b, size_t e,
                                                       GPose* __restrict__ seeds, uint32_t* __restrict__ n_seeds,
                                                       uint32_t* __restrict__ assign, uint32_t* __restrict__ unm,
                                                       float tt, float rt) {
  __shared__ uint32_t s_warp[32], s_n, s_c;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // compact the unassigned positions of the chunk, in order
  if (tid == 0) s_n = 0;
  block_sync();
  for (size_t t0 = b; t0 < e; t0 += 1024) {
    const size_t i = t0 + tid;
    const bool u = i < e && assign[i] == kNone;
    const uint32_t bal = __ballot_sync(0xffffffffu, u);
    if (lane == 0) s_warp[warp] = __popc(bal);
    block_sync();
    uint32_t off = s_n;
    for (int w = 0; w < warp; ++w) off += s_warp[w];
    if (u) unm[off + __popc(bal & ((1u << lane) - 1u))] = (uint32_t)i;
    block_sync();
    if (tid == 0)
      for (int w = 0; w < 32; ++w) s_n += s_warp[w];
    block_sync();
  }
  const uint32_t n = s_n;
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t j = unm[k];
    if (assign[j] != kNone) continue;  // uniform: written before the last barrier
    if (tid == 0) {
      const uint32_t c = *n_seeds;
      seeds[c] = poses[j];
      assign[j] = c;
      *n_seeds = c + 1;
      s_c = c;
    }
    block_sync();
    const uint32_t c = s_c;
    const GPose pj = poses[j];
    for (uint32_t m = k + 1 + tid; m < n; m += 1024) {
      const uint32_t i = unm[m];
      if (assign[i] == kNone && close_enough(poses[i], pj, tt, rt)) assign[i] = c;
    }
    block_sync();
  }
}

__global__ void totals_kernel(const uint32_t* __restrict__ assign, const uint32_t* __restrict__ votes, size_t U,
                              uint32_t* __restrict__ totals) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < U; i += (size_t)gridDim.x * blockDim.x)
    atomicAdd(totals + assign[i], votes[i]);
}

// The three clusters with most votes (ties: lower cluster index), then the
// average pose of each, written as three row-major poses.  One block.
__global__ void __launch_bounds__(1024) top3_average_kernel(const GPose* __restrict__ poses, size_t U,
                                                            const uint32_t* __restrict__ assign,
                                                            const uint32_t* __restrict__ totals,
                                                            const uint32_t* __restrict__ n_seeds,
                                                            float* __restrict__ out, uint32_t* __restrict__ out_info) {
  __shared__ unsigned long long s_best[32];
  __shared__ uint32_t s_top[3], s_list[1024], s_cnt;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t C = *n_seeds;
  const int nc = C < 3 ? (int)C : 3;
  for (int r = 0; r < nc; ++r) {
    // key: total (high), ~cluster (low) -> max picks most votes, then lowest index
    unsigned long long best = 0;
    for (uint32_t c = tid; c < C; c += 1024) {
      bool taken = false;
      for (int q = 0; q < r; ++q) taken = taken || s_top[q] == c;
      if (!taken) best = max(best, ((unsigned long long)totals[c] << 32) | (0xffffffffu - c));
    }
    for (int o = 16; o; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) s_best[warp] = best;
    block_sync();
    if (tid == 0) {
      unsigned long long m = 0;
      for (int w = 0; w < 32; ++w) m = max(m, s_best[w]);
      s_top[r] = 0xffffffffu - (uint32_t)(m & 0xffffffffu);
    }
    block_sync();
  }
  for (int r = 0; r < nc; ++r) {
    const uint32_t c = s_top[r];
    float t[3] = {0.f, 0.f, 0.f}, qs[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t size = 0;
    for (size_t t0 = 0; t0 < U; t0 += 1024) {
      // members of this tile, in order, then summed by one thread
      const size_t i = t0 + tid;
      const bool mem = i < U && assign[i] == c;
      const uint32_t bal = __ballot_sync(0xffffffffu, mem);
      if (lane == 0) s_best[warp] = __popc(bal);
      block_sync();
      uint32_t off = 0;
      for (int w = 0; w < warp; ++w) off += (uint32_t)s_best[w];
      if (mem) s_list[off + __popc(bal & ((1u << lane) - 1u))] = (uint32_t)i;
      if (tid == 0) {
        uint32_t cnt = 0;
        for (int w = 0; w < 32; ++w) cnt += (uint32_t)s_best[w];
        s_cnt = cnt;
      }
      block_sync();
      if (tid == 0) {
        for (uint32_t k = 0; k < s_cnt; ++k) {
          float R[9], tr[3], q[4];
          unpack(poses[s_list[k]], R, tr);
          for (int d = 0; d < 3; ++d) t[d] = fadd(t[d], tr[d]);
          quat_xyzw(R, q);
          for (int d = 0; d < 4; ++d) qs[d] = fadd(qs[d], q[d]);
        }
        size += s_cnt;
      }
      block_sync();
    }
    if (tid == 0) {
      const float sz = (float)size;
      for (int d = 0; d < 3; ++d) t[d] = __fdiv_rn(t[d], sz);
      for (int d = 0; d < 4; ++d) qs[d] = __fdiv_rn(qs[d], sz);
      const float qn = __fsqrt_rn(
          fadd(fadd(fadd(fmul(qs[0], qs[0]), fmul(qs[1], qs[1])), fmul(qs[2], qs[2])), fmul(qs[3], qs[3])));
      const float x = __fdiv_rn(qs[0], qn), y = __fdiv_rn(qs[1], qn), z = __fdiv_rn(qs[2], qn),
                  w = __fdiv_rn(qs[3], qn);
      const float tx = fmul(2.f, x), ty = fmul(2.f, y), tz = fmul(2.f, z);
      float* O = out + 16 * r;
      O[0] = fsub(1.f, fadd(fmul(ty, y), fmul(tz, z)));
      O[1] = fsub(fmul(ty, x), fmul(tz, w));
      O[2] = fadd(fmul(tz, x), fmul(ty, w));
      O[3] = t[0];
      O[4] = fadd(fmul(ty, x), fmul(tz, w));
      O[5] = fsub(1.f, fadd(fmul(tx, x), fmul(tz, z)));
      O[6] = fsub(fmul(tz, y), fmul(tx, w));
      O[7] = t[1];
      O[8] = fsub(fmul(tz, x), fmul(ty, w));
      O[9] = fadd(fmul(tz, y), fmul(tx, w));
      O[10] = fsub(1.f, fadd(fmul(tx, x), fmul(ty, y)));
      O[11] = t[2];
      O[12] = 0.f;
      O[13] = 0.f;
      O[14] = 0.f;
      O[15] = 1.f;
      out_info[1 + r] = totals[c];
    }
    block_sync();
  }
  if (tid == 0) out_info[0] = (uint32_t)nc;
}

__global__ void invert_kernel(const uint32_t* __restrict__ v, size_t n, uint32_t* __restrict__ k) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    k[i] = ~v[i];  // ascending order of ~votes = descending votes
}

__global__ void gather_poses_kernel(const uint32_t* __restrict__ perm, const float* __restrict__ T,
                                    const uint32_t* __restrict__ v, size_t n, float* __restrict__ To,
                                    uint32_t* __restrict__ vo) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t p = perm[i];
    for (int k = 0; k < 16; ++k) To[16 * i + k] = T[16 * p + k];
    vo[i] = v[p];
  }
}

}  // namespace

int cluster_poses_greedy_gpu(Context& ctx, const float* transforms_dev, const uint32_t* votes_dev, size_t U,
                             float trans_thresh, float rot_thresh, float out_poses[3 * 16], uint32_t out_votes[3]) {
  if (U == 0) return 0;
  cudaStream_t st = ctx.stream;
  PPF_REQUIRE(U < 0xffffffffull, PPF_ERR_INVALID_ARGUMENT, "more than 2^32 - 1 poses");
  DevBuf poses, seeds, assign, unm, totals, out;
  poses.reserve(U * sizeof(GPose));
  seeds.reserve(U * sizeof(GPose));
  assign.reserve(U * 4);
  unm.reserve(std::min<size_t>(U, kGreedyChunk) * 4);
  totals.reserve(U * 4);
  out.reserve(64 + 48 * 4);
  uint32_t* n_seeds = out.as<uint32_t>();  // [0] clusters, [1..3] top totals; poses at byte 64
  PPF_CUDA(cudaMemsetAsync(out.ptr, 0, 64, st));
  PPF_CUDA(cudaMemsetAsync(totals.ptr, 0, U * 4, st));
  GPose* P = poses.as<GPose>();
  prep_kernel<<<grid_for(U, 256), 256, 0, st>>>(transforms_dev, U, P);
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
  uint32_t* seed_count = n_seeds + 8;  // separate word for the running cluster count
  for (size_t b = 0; b < U; b += kGreedyChunk) {
    const size_t e = std::min(U, b + kGreedyChunk);
    match_kernel<<<grid_for(e - b, 128), 128, 0, st>>>(P, b, e, seeds.as<GPose>(), seed_count,
                                                         assign.as<uint32_t>(), trans_thresh, rot_thresh);
    resolve_kernel<<<1, 1024, 0, st>>>(P, b, e, seeds.as<GPose>(), seed_count, assign.as<uint32_t>(),
                                       unm.as<uint32_t>(), trans_thresh, rot_thresh);
    PPF_CUDA(cudaGetLastError());
    ctx.launches += 2;
  }
  totals_kernel<<<grid_for(U, 256), 256, 0, st>>>(assign.as<uint32_t>(), votes_dev, U, totals.as<uint32_t>());
  top3_average_kernel<<<1, 1024, 0, st>>>(P, U, assign.as<uint32_t>(), totals.as<uint32_t>(), seed_count,
                                          reinterpret_cast<float*>(out.as<char>() + 64), n_seeds);
  PPF_CUDA(cudaGetLastError());
  ctx.launches += 2;
  uint32_t info[4];
  float h[48];
  PPF_CUDA(cudaMemcpyAsync(info, n_seeds, sizeof(info), cudaMemcpyDeviceToHost, st));
  PPF_CUDA(cudaMemcpyAsync(h, out.as<char>() + 64, sizeof(h), cudaMemcpyDeviceToHost, st));
  PPF_CUDA(cudaStreamSynchronize(st));
  const int nc = (int)info[0];
  std::memcpy(out_poses, h, sizeof(float) * 16 * nc);
  for (int r = 0; r < nc; ++r) out_votes[r] = info[1 + r];
  return nc;
}

// clusterPoses on arbitrary poses: the stable sort by votes (descending)
// first, then the greedy pass above.
int cluster_poses_sorted_gpu(Context& ctx, const float* transforms_dev, const uint32_t* votes_dev, size_t U,
                             float trans_thresh, float rot_thresh, float out_poses[3 * 16], uint32_t out_votes[3]) {
  if (U == 0) return 0;
  cudaStream_t st = ctx.stream;
  DevBuf keys, perm, T, V;
  keys.reserve(U * 4);
  perm.reserve(U * 4);
  T.reserve(U * 64);
  V.reserve(U * 4);
  invert_kernel<<<grid_for(U, 256), 256, 0, st>>>(votes_dev, U, keys.as<uint32_t>());
  PPF_CUDA(cudaMemsetAsync(ctx.flags.ptr, 0, 4, st));
  const size_t l0 = ctx.sort32.launches();
  ctx.sort32.sort(keys.as<uint32_t>(), perm.as<uint32_t>(), true, U, 0, 32, st, ctx.flags.as<uint32_t>());
  ctx.launches += ctx.sort32.launches() - l0 + 2;
  gather_poses_kernel<<<grid_for(U, 256), 256, 0, st>>>(perm.as<uint32_t>(), transforms_dev, votes_dev, U,
                                                         T.as<float>(), V.as<uint32_t>());
  PPF_CUDA(cudaGetLastError());
  return cluster_poses_greedy_gpu(ctx, T.as<float>(), V.as<uint32_t>(), U, trans_thresh, rot_thresh, out_poses,
                                  out_votes);
}

}  // namespace ppf
