// The vote pass: the work of Scene::Scene + Model::ComputeUniqueVotes
// (src/cuda/scene.cu:24-55, src/cuda/model.cu:95-171) without materialising
// scene pair features or individual votes.
//
// One work item = (scene reference point s_r, chunk of model reference points).
// A persistent block (1024 threads, one per SM) takes items from an atomic
// counter.  For its s_r it walks all scene points in tiles of 1024: each
// thread computes one pair feature, its FNV key, and looks the key up in the
// model's key -> run table.  Every matched pair's sub-run (the run entries
// whose m_r falls in this chunk) is cut into segments of at most kSeg entries;
// warps take segments from a shared counter and stream their entries with
// consecutive lanes on consecutive entries, counting each vote into a
// shared-memory accumulator of 32-bit (m_r, alpha bin) counters.  When an
// item is done, the block folds its largest count into a global running
// maximum and emits every cell whose count exceeds threshold x running
// maximum: a superset of the cells the final threshold (threshold x global
// maximum) keeps.
#include "engine.h"
#include "ppf_math.cuh"

namespace ppf {
namespace {

constexpr uint32_t kSeg = 1024;   // entries per segment
constexpr int kUnroll = 8;        // independent entry loads per lane
constexpr uint32_t kNoRun = 0xffffffffu;

struct VoteArgs {
  // model
  const uint32_t* entries;
  const uint32_t* epairs;
  const uint32_t* split;
  const uint32_t* run_count;
  const uint8_t* run_flags;
  const uint32_t* ht_keys;
  const uint32_t* ht_runs;
  uint32_t ht_mask;
  const float4* m_r1;
  const float4* m_r2;
  const float4* m_pts;
  uint32_t n_m, chunk, n_chunks;
  // scene
  const float4* s_pts;
  const float4* s_nrm;
  uint32_t n_s, ref_df, n_ref, perm_mul;
  float d_dist, thr, floor;
  int emit_all;
  // control / outputs
  uint32_t n_items;
  uint32_t* work_counter;
  uint32_t* global_max;
  unsigned long long* stats;  // [0] votes, [1] matched pairs, [2] exact bins
  unsigned long long* cand_code;
  uint32_t* cand_count;
  uint32_t* n_cand;
  uint32_t cand_cap;
  uint32_t* flags;
};

__device__ __forceinline__ uint32_t ht_lookup(const uint32_t* __restrict__ keys,
                                              const uint32_t* __restrict__ runs, uint32_t mask,
                                              uint32_t key) {
  uint32_t s = (key * 0x9E3779B1u) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    uint32_t k = __ldg(keys + s);
    if (k == key) return __ldg(runs + s);
    if (k == 0u) return kNoRun;
    s = (s + 1) & mask;
  }
  return kNoRun;
}

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
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
    uint32_t w = lane < kVoteWarps ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kVoteWarps) s_warp[lane] = w;
  }
  __syncthreads();
  uint32_t r = (warp ? s_warp[warp - 1] : 0u) + x - v;
  if (total) *total = s_warp[kVoteWarps - 1];
  __syncthreads();
  return r;
}

// Exact bin of one vote: the reference's own arithmetic for it.
__device__ __forceinline__ uint32_t exact_bin(const VoteArgs& a, uint32_t pos, uint32_t mr,
                                              float2 v) {
  const uint32_t mi = __ldg(a.epairs + pos) - mr * a.n_m;
  FrameYZ fm;
  fm.r1 = __ldg(a.m_r1 + mr);
  fm.r2 = __ldg(a.m_r2 + mr);
  float4 q4 = __ldg(a.m_pts + mi);
  float2 u = frame_point_yz(fm, make_float3(q4.x, q4.y, q4.z));
  return alpha_bin_exact(u, v);
}

__global__ void __launch_bounds__(kVoteThreads, 1) vote_kernel(VoteArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* q_lo = smem;                        // [kVoteThreads]
  uint32_t* q_len = q_lo + kVoteThreads;        // [kVoteThreads]
  uint32_t* q_beta = q_len + kVoteThreads;      // [kVoteThreads]
  float2* q_v = reinterpret_cast<float2*>(q_beta + kVoteThreads);       // [kVoteThreads]
  uint32_t* q_seg = reinterpret_cast<uint32_t*>(q_v + kVoteThreads);    // [kVoteThreads + 4]
  uint32_t* acc = q_seg + kVoteThreads + 4;

  __shared__ uint32_t s_item, s_next, s_max;
  __shared__ uint32_t s_warp[kVoteWarps];
  __shared__ float4 s_fr[2];  // scene frame rows 1, 2
  __shared__ float4 s_pr, s_nr;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t cells = a.chunk * kBins;
  unsigned long long my_votes = 0, my_matched = 0, my_exact = 0;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(a.work_counter, 1u);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= a.n_items) break;
    const uint32_t c = item % a.n_chunks;
    const uint32_t ref = (uint32_t)(((unsigned long long)(item / a.n_chunks) * a.perm_mul) % a.n_ref);
    const uint32_t sr = ref * a.ref_df;
    const uint32_t mr_lo = c * a.chunk;
    if (tid == 0) {
      float4 p = a.s_pts[sr], q = a.s_nrm[sr];
      FrameYZ f = frame_yz(make_float3(p.x, p.y, p.z), make_float3(q.x, q.y, q.z));
      s_fr[0] = f.r1;
      s_fr[1] = f.r2;
      s_pr = p;
      s_nr = q;
    }
    for (uint32_t i = tid; i < cells; i += kVoteThreads) acc[i] = 0u;
    __syncthreads();
    const float3 pr = make_float3(s_pr.x, s_pr.y, s_pr.z);
    const float3 nr = make_float3(s_nr.x, s_nr.y, s_nr.z);
    FrameYZ fs;
    fs.r1 = s_fr[0];
    fs.r2 = s_fr[1];

    for (uint32_t base = 0; base < a.n_s; base += kVoteThreads) {
      // ---- one scene pair per thread: feature, key, lookup, sub-run
      const uint32_t i = base + tid;
      uint32_t len = 0, lo = 0, beta = 0;
      float2 v = make_float2(0.f, 0.f);
      if (i < a.n_s && i != sr) {
        float4 pi4 = a.s_pts[i], ni4 = a.s_nrm[i];
        float3 pi = make_float3(pi4.x, pi4.y, pi4.z);
        float4 f = pair_feature(pr, nr, pi, make_float3(ni4.x, ni4.y, ni4.z), a.d_dist);
        uint32_t key = feature_key(f);
        if (key != 0u) {
          uint32_t run = ht_lookup(a.ht_keys, a.ht_runs, a.ht_mask, key);
          if (run != kNoRun) {
            const uint32_t* sp = a.split + (size_t)run * (a.n_chunks + 1);
            lo = __ldg(sp + c);
            len = __ldg(sp + c + 1) - lo;
            if (c == 0) {
              my_votes += __ldg(a.run_count + run);
              my_matched += 1;
            }
            if (len) {
              v = frame_point_yz(fs, pi);
              bool degenerate = fabsf(v.x) + fabsf(v.y) < 1e-12f || !isfinite(v.x) || !isfinite(v.y);
              beta = angle16(v) | ((degenerate || __ldg(a.run_flags + run)) ? 0x10000u : 0u);
            }
          }
        }
      }
      uint32_t n_seg_total;
      uint32_t seg0 = block_excl_scan((len + kSeg - 1) / kSeg, s_warp, &n_seg_total);
      q_lo[tid] = lo;
      q_len[tid] = len;
      q_beta[tid] = beta;
      q_v[tid] = v;
      q_seg[tid] = seg0;
      if (tid == 0) {
        q_seg[kVoteThreads] = n_seg_total;
        s_next = kVoteWarps;
      }
      __syncthreads();

      // ---- warps take segments; lanes stream consecutive entries
      uint32_t s = warp;
      while (s < n_seg_total) {
        uint32_t plo = 0, phi = kVoteThreads;  // pair p with q_seg[p] <= s < q_seg[p+1]
        while (phi - plo > 1) {
          uint32_t mid = (plo + phi) >> 1;
          if (q_seg[mid] <= s) plo = mid;
          else phi = mid;
        }
        const uint32_t p = plo;
        const uint32_t start = q_lo[p] + (s - q_seg[p]) * kSeg;
        const uint32_t end = min(q_lo[p] + q_len[p], start + kSeg);
        const uint32_t bw = q_beta[p];
        const uint32_t bsp = bw + 32768u;  // bits above 16 shift out below
        const float2 vv = q_v[p];
        // Each entry holds its accumulator row (m_r - mr_lo) * 31 in the high
        // half and the model angle beta_m in the low half.  With y = (beta_s +
        // 2^15 - beta_m) << 16, i.e. alpha + pi in 2^-32 turns, the bin is the
        // high word of y * 30 and the low word is the position inside the bin.
        const uint32_t bsh = bsp << 16;
        constexpr uint32_t m_lo = (PPF_BIN_MARGIN_UNITS * PPF_N_ANGLE) << 16;
        constexpr uint32_t m_span = (65536u - 2 * PPF_BIN_MARGIN_UNITS * PPF_N_ANGLE) << 16;
        const uint32_t* ep = a.entries + start + lane;
        const uint32_t n_here = end - start;
        if (bw & 0x10000u) {
          // degenerate frame vector or run: every vote takes the exact path
          for (uint32_t k = lane; k < n_here; k += 32) {
            const uint32_t row = __ldg(a.entries + start + k) >> 16;
            atomicAdd(&acc[row + exact_bin(a, start + k, mr_lo + row / kBins, vv)], 1u);
            ++my_exact;
          }
        } else {
          const uint32_t nfull = n_here / (32 * kUnroll);
          for (uint32_t it = 0; it < nfull; ++it, ep += 32 * kUnroll) {
            uint32_t e[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) e[u] = __ldg(ep + 32 * u);
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
              const uint32_t y = bsh - (e[u] << 16);
              uint32_t cell = (e[u] >> 16) + __umulhi(y, (uint32_t)PPF_N_ANGLE);
              if (y * (uint32_t)PPF_N_ANGLE - m_lo > m_span) {  // near a bin edge
                const uint32_t row = e[u] >> 16;
                cell = row + exact_bin(a, (uint32_t)(ep + 32 * u - a.entries), mr_lo + row / kBins, vv);
                ++my_exact;
              }
              atomicAdd(&acc[cell], 1u);
            }
          }
          for (uint32_t k = nfull * 32 * kUnroll + lane; k < n_here; k += 32) {
            const uint32_t e = __ldg(a.entries + start + k);
            const uint32_t y = bsh - (e << 16);
            uint32_t cell = (e >> 16) + __umulhi(y, (uint32_t)PPF_N_ANGLE);
            if (y * (uint32_t)PPF_N_ANGLE - m_lo > m_span) {
              const uint32_t row = e >> 16;
              cell = row + exact_bin(a, start + k, mr_lo + row / kBins, vv);
              ++my_exact;
            }
            atomicAdd(&acc[cell], 1u);
          }
        }
        if (lane == 0) s = atomicAdd(&s_next, 1u);
        s = __shfl_sync(0xffffffffu, s, 0);
      }
      __syncthreads();
    }

    // ---- running maximum, emission
    uint32_t lmax = 0;
    for (uint32_t w = tid; w < cells; w += kVoteThreads) lmax = max(lmax, acc[w]);
#pragma unroll
    for (int o = 16; o; o >>= 1) lmax = max(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if (lane == 0) s_warp[warp] = lmax;
    __syncthreads();
    if (tid == 0) {
      uint32_t m = 0;
      for (int w = 0; w < kVoteWarps; ++w) m = max(m, s_warp[w]);
      uint32_t old = atomicMax(a.global_max, m);
      s_max = max(old, m);
    }
    __syncthreads();
    const float floor_v = a.floor >= 0.f ? a.floor : a.thr * (float)s_max;
    for (uint32_t b0 = 0; b0 < cells; b0 += kVoteThreads) {
      const uint32_t cell = b0 + tid;
      const uint32_t cnt = cell < cells ? acc[cell] : 0u;
      bool keep = cnt != 0u && (a.emit_all || (float)cnt > floor_v);
      uint32_t ballot = __ballot_sync(0xffffffffu, keep);
      if (!ballot) continue;
      uint32_t slot0 = 0;
      if (lane == 0) slot0 = atomicAdd(a.n_cand, (uint32_t)__popc(ballot));
      slot0 = __shfl_sync(0xffffffffu, slot0, 0);
      if (keep) {
        uint32_t sl = slot0 + __popc(ballot & ((1u << lane) - 1u));
        if (sl < a.cand_cap) {
          uint32_t mr = mr_lo + cell / kBins, bin = cell % kBins;
          a.cand_code[sl] = ((unsigned long long)sr << 32) | ((unsigned long long)mr << 6) | bin;
          a.cand_count[sl] = cnt;
        } else {
          atomicOr(a.flags, (uint32_t)kFlagCandidateOverflow);
        }
      }
    }
    __syncthreads();
  }

  // per-block statistics
  for (int o = 16; o; o >>= 1) {
    my_votes += __shfl_xor_sync(0xffffffffu, my_votes, o);
    my_matched += __shfl_xor_sync(0xffffffffu, my_matched, o);
    my_exact += __shfl_xor_sync(0xffffffffu, my_exact, o);
  }
  if (lane == 0) {
    if (my_votes) atomicAdd(&a.stats[0], my_votes);
    if (my_matched) atomicAdd(&a.stats[1], my_matched);
    if (my_exact) atomicAdd(&a.stats[2], my_exact);
  }
}

// counts[r * n_s + i]: model run length of a matching scene pair (r, i).
__global__ void pair_vote_counts_kernel(VoteArgs a, unsigned long long* __restrict__ out) {
  for (uint32_t r = blockIdx.y; r < a.n_s; r += gridDim.y) {
    unsigned long long* row = out + (size_t)r * a.n_s;
    const bool ref_row = (r % a.ref_df) == 0 && a.n_s > 1;
    float4 p4 = a.s_pts[r], n4 = a.s_nrm[r];
    float3 pr = make_float3(p4.x, p4.y, p4.z), nr = make_float3(n4.x, n4.y, n4.z);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_s;
         i += gridDim.x * blockDim.x) {
      unsigned long long cnt = 0;
      if (ref_row && i != r) {
        float4 q4 = a.s_pts[i], m4 = a.s_nrm[i];
        float4 f = pair_feature(pr, nr, make_float3(q4.x, q4.y, q4.z),
                                make_float3(m4.x, m4.y, m4.z), a.d_dist);
        uint32_t key = feature_key(f);
        if (key) {
          uint32_t run = ht_lookup(a.ht_keys, a.ht_runs, a.ht_mask, key);
          if (run != kNoRun) cnt = a.run_count[run];
        }
      }
      row[i] = cnt;
    }
  }
}

uint32_t gcd_u32(uint32_t x, uint32_t y) {
  while (y) {
    uint32_t t = x % y;
    x = y;
    y = t;
  }
  return x;
}

VoteArgs make_args(const Model& m, const SceneData& s) {
  const ModelTables& t = m.t;
  VoteArgs a{};
  a.entries = t.entries.as<uint32_t>();
  a.epairs = t.epairs.as<uint32_t>();
  a.split = t.split.as<uint32_t>();
  a.run_count = t.count.as<uint32_t>();
  a.run_flags = t.run_flags.as<uint8_t>();
  a.ht_keys = t.ht_keys.as<uint32_t>();
  a.ht_runs = t.ht_runs.as<uint32_t>();
  a.ht_mask = t.ht_mask;
  a.m_r1 = t.frame_r1.as<float4>();
  a.m_r2 = t.frame_r2.as<float4>();
  a.m_pts = t.pts.as<float4>();
  a.n_m = t.n;
  a.chunk = t.chunk;
  a.n_chunks = t.n_chunks;
  a.s_pts = s.pts.as<float4>();
  a.s_nrm = s.nrm.as<float4>();
  a.n_s = s.n;
  a.ref_df = s.ref_df ? s.ref_df : 1;
  a.n_ref = (s.n + a.ref_df - 1) / a.ref_df;
  a.d_dist = s.d_dist;  // scene pair features use the scene's quantum
  a.thr = m.vote_count_threshold;
  // ref visiting order: j -> j * perm_mul mod n_ref (a bijection)
  uint32_t pm = a.n_ref > 1 ? (0x9E3779B1u % a.n_ref) : 1u;
  if (pm == 0) pm = 1;
  while (a.n_ref > 1 && gcd_u32(pm, a.n_ref) != 1) ++pm;
  a.perm_mul = pm;
  return a;
}

}  // namespace

VoteResult run_votes(Context& ctx, const Model& m, const SceneData& s, LookupState& st,
                     bool emit_all, float floor, size_t cand_cap) {
  VoteResult r;
  cudaStream_t stream = ctx.stream;
  VoteArgs a = make_args(m, s);
  a.emit_all = emit_all ? 1 : 0;
  a.floor = floor;
  a.n_items = a.n_ref * a.n_chunks;
  if (s.n < 2 || a.n_items == 0) return r;
  // counters: [0] work, [1] max, [2] n_cand, [3] pad, [4..9] 3 x u64 stats
  ctx.counters.reserve(64);
  PPF_CUDA(cudaMemsetAsync(ctx.counters.ptr, 0, 64, stream));
  PPF_CUDA(cudaMemsetAsync(ctx.flags.ptr, 0, sizeof(uint32_t), stream));
  uint32_t* cnt = ctx.counters.as<uint32_t>();
  a.work_counter = cnt + 0;
  a.global_max = cnt + 1;
  a.n_cand = cnt + 2;
  a.stats = reinterpret_cast<unsigned long long*>(cnt + 4);
  a.flags = ctx.flags.as<uint32_t>();
  st.cand_codes.reserve(cand_cap * sizeof(unsigned long long));
  st.cand_counts.reserve(cand_cap * sizeof(uint32_t));
  a.cand_code = st.cand_codes.as<unsigned long long>();
  a.cand_count = st.cand_counts.as<uint32_t>();
  a.cand_cap = (uint32_t)cand_cap;

  const size_t smem = kVoteQueueBytes + vote_acc_words(a.chunk) * 4;
  PPF_REQUIRE((int)smem <= ctx.vote_smem_limit, PPF_ERR_INTERNAL, "vote accumulator too large");
  PPF_CUDA(cudaFuncSetAttribute(vote_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PPF_CUDA(cudaEventRecord(ctx.ev[0], stream));
  vote_kernel<<<(unsigned)std::min<size_t>(a.n_items, (size_t)sm_count()), kVoteThreads, smem, stream>>>(a);
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
  PPF_CUDA(cudaEventRecord(ctx.ev[1], stream));
  uint32_t h[16];
  PPF_CUDA(cudaMemcpyAsync(h, ctx.counters.ptr, 64, cudaMemcpyDeviceToHost, stream));
  PPF_CUDA(cudaStreamSynchronize(stream));
  PPF_CUDA(cudaEventElapsedTime(&r.vote_ms, ctx.ev[0], ctx.ev[1]));
  r.max_count = h[1];
  r.n_cand = h[2];
  unsigned long long* s64 = reinterpret_cast<unsigned long long*>(h + 4);
  r.n_votes = s64[0];
  r.n_matched = s64[1];
  r.n_exact = s64[2];
  return r;
}

void pair_vote_counts(Context& ctx, const Model& m, const SceneData& s, uint64_t* out_dev) {
  VoteArgs a = make_args(m, s);
  dim3 grid((s.n + 255) / 256, std::min<uint32_t>(s.n, 65535u));
  pair_vote_counts_kernel<<<grid, 256, 0, ctx.stream>>>(a, reinterpret_cast<unsigned long long*>(out_dev));
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
}

}  // namespace ppf
