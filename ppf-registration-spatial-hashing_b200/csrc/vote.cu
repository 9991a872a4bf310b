// The vote pass: the work of Scene::Scene + Model::ComputeUniqueVotes
// (src/cuda/scene.cu:24-55, src/cuda/model.cu:95-171) without materialising
// scene pair features or individual votes.
//
// One work item = (scene reference point s_r, chunk of model reference points).
// A persistent block (1024 threads, one per SM) takes items from an atomic
// counter.  For its s_r it walks all scene points in tiles of 1024: each
// thread computes one pair feature, its FNV key, and looks the key up in the
// model's key -> run table.  Every matched pair's sub-run (the run entries
// whose m_r falls in this chunk) is cut into segments of at most 2^seg_shift entries;
// warps take segments from a shared counter and stream their entries with
// consecutive lanes on consecutive entries, counting each vote into a
// shared-memory accumulator of 32-bit (m_r, alpha bin) counters.  When an
// item is done, the block folds its largest count into a global running
// maximum and emits every cell whose count exceeds threshold x running
// maximum: a superset of the cells the final threshold (threshold x global
// maximum) keeps.
#include <cstring>
#include <mutex>
#include <string>

#include "engine.h"
#include "ppf_math.cuh"

namespace ppf {
namespace {

// Entries per segment: 1 << VoteArgs::seg_shift.  A warp streams a segment
// in passes of 256 entries and pays the L2 latency of its first loads and the
// segment search once per segment; longer segments leave more warps idle at
// the end of a tile.  Fixed lengths of 1024/2048/4096/8192 measured
// 57.8/53.2/51.5/51.6 ms on the bench's first model (ref_point_df 50) and
// 92.1/83.8/79.8/78.3 ms on its fourth: the best length depends on the model,
// so tune_vote_segments chooses it per model among kSegShifts.
constexpr uint32_t kSegShifts[] = {11, 12, 13};
constexpr int kUnroll = 8;        // independent entry loads per lane
constexpr uint32_t kNoRun = 0xffffffffu;
constexpr uint32_t kExactOnly = 1u << 31;  // scene angle flag: every vote of the pair takes the exact path

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
  uint32_t seg_shift;  // log2 of the segment length
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
  unsigned long long* n_needed;  // cells all items asked to emit
  uint32_t* redo_items;          // items that did not fit the buffer
  uint32_t* n_redo;
  uint32_t n_items_total;        // capacity of redo_items
  const uint32_t* item_list;     // second launch: the items to redo (else all items)
  uint32_t* flags;
  // bounds for the self-checking build (PPF_B200_CHECKS=1)
  size_t P, K;
  unsigned long long* bad;  // first out-of-range access: site, value, bound
};

// Self-checking build: every index the kernel derives is compared with its
// bound; the first violation is recorded (site, value, bound) in bad[0..2],
// kFlagBadIndex is raised and the access is skipped.
template <bool kCheck>
__device__ __forceinline__ bool in_range(const VoteArgs& a, uint32_t site, unsigned long long v,
                                         unsigned long long bound) {
  if (!kCheck) return true;
  if (v < bound) return true;
  if (atomicCAS(&a.bad[0], 0ull, (unsigned long long)site) == 0ull) {
    a.bad[1] = v;
    a.bad[2] = bound;
  }
  atomicOr(a.flags, (uint32_t)kFlagBadIndex);
  return false;
}

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

// Block barrier of the vote kernel.  __syncthreads() is an .aligned barrier:
// every lane of a warp must reach it together.  Each barrier here follows
// lane-conditional code (lane 31 stores a warp total before the scan
// barriers, lane 0 stores sh.item, sh.base and the counters), and with
// independent thread scheduling an optimised build may bring a warp to the
// barrier in two groups, so that the barrier releases on the first and the
// rest of the warp runs one barrier phase behind.  That is what a -O3 build
// without the __syncwarp() did on one 60000-point scene (the other warps
// read the segment scan before warp 0 had written it; -O1 and -O0 builds
// did not).
// __syncwarp() reconverges the warp first; the fences around the barrier
// order the shared-memory stores and loads on both sides.
__device__ __forceinline__ void block_sync() {
  __syncwarp();
  __threadfence_block();
  __syncthreads();
  __threadfence_block();
}

// Exclusive block scan of one value per thread; `total` receives the sum.
// s_warp is this call site's own 32-word scratch; the caller places a barrier
// between two scans on the same scratch (both call sites have several).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  block_sync();
  if (warp == 0) {
    uint32_t w = s_warp[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    s_warp[lane] = w;
  }
  block_sync();
  const uint32_t r = (warp ? s_warp[warp - 1] : 0u) + x - v;
  total = s_warp[kVoteWarps - 1];
  return r;
}

// Exact bin of one vote: the reference's own arithmetic for it.  The model
// pair comes from the entry's pair index, so every index is in range by
// construction.
template <bool kCheck>
__device__ __forceinline__ uint32_t exact_bin(const VoteArgs& a, uint32_t pos, float2 v) {
  if (!in_range<kCheck>(a, 20, pos, a.P)) return 0;
  const uint32_t pr = __ldg(a.epairs + pos);
  const uint32_t mr = pr / a.n_m, mi = pr - mr * a.n_m;
  if (!in_range<kCheck>(a, 21, mr, a.n_m) || !in_range<kCheck>(a, 22, mi, a.n_m)) return 0;
  FrameYZ fm;
  fm.r1 = __ldg(a.m_r1 + mr);
  fm.r2 = __ldg(a.m_r2 + mr);
  float4 q4 = __ldg(a.m_pts + mi);
  float2 u = frame_point_yz(fm, make_float3(q4.x, q4.y, q4.z));
  return alpha_bin_exact(u, v);
}

// Per-block shared state of a vote kernel besides the dynamic queue and
// accumulator.
struct VoteShared {
  // the item's scene reference point, its normal and rows 1-2 of its frame:
  // read from here by the scene walk of each tile, so that they do not hold
  // 14 registers through the vote passes between walks
  float4 p_r, n_r, f_r1, f_r2;
  uint32_t item, next, max, base;
  uint32_t scan_seg[kVoteWarps];   // scratch of the per-tile segment scan
  uint32_t scan_emit[kVoteWarps];  // scratch of the emission scan
  // q_seg at the first pair of each warp's 32 (q_seg[32 l]), kept
  // contiguous: the segment search reads all 32 in one conflict-free access
  // (read in place they sit in one bank, 32 accesses per search)
  uint32_t seg_blk[kVoteWarps];
  uint32_t wmax[kVoteWarps];       // per-warp maxima of the accumulator
};

// Per-thread vote statistics, folded into a request's counters when the
// block leaves the request.
struct VoteStats {
  unsigned long long votes = 0, matched = 0, exact = 0;
};

__device__ __forceinline__ void flush_stats(const VoteArgs& a, VoteStats& st) {
  for (int o = 16; o; o >>= 1) {
    st.votes += __shfl_xor_sync(0xffffffffu, st.votes, o);
    st.matched += __shfl_xor_sync(0xffffffffu, st.matched, o);
    st.exact += __shfl_xor_sync(0xffffffffu, st.exact, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (st.votes) atomicAdd(&a.stats[0], st.votes);
    if (st.matched) atomicAdd(&a.stats[1], st.matched);
    if (st.exact) atomicAdd(&a.stats[2], st.exact);
  }
  st = VoteStats();
}

// Fetches the next work item into sh.item (one atomic per block).
__device__ __forceinline__ uint32_t fetch_item(uint32_t* work_counter, VoteShared& sh) {
  if ((threadIdx.x >> 5) == 0) {
    uint32_t next = 0;
    if ((threadIdx.x & 31) == 0) next = atomicAdd(work_counter, 1u);
    next = __shfl_sync(0xffffffffu, next, 0);
    if ((threadIdx.x & 31) == 0) sh.item = next;
  }
  block_sync();
  return sh.item;
}

// One work item (s_r, chunk) of request `a`: slot_of_item indexes a's items
// (or a.item_list).  Called by every thread of the block.
template <bool kCheck>
__device__ __forceinline__ void vote_item(const VoteArgs& a, uint32_t slot_of_item, VoteShared& sh,
                                          VoteStats& st) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* q_lo = smem;                        // [kVoteThreads]
  uint32_t* q_len = q_lo + kVoteThreads;        // [kVoteThreads]
  uint32_t* q_beta = q_len + kVoteThreads;      // [kVoteThreads]
  float2* q_v = reinterpret_cast<float2*>(q_beta + kVoteThreads);       // [kVoteThreads]
  uint32_t* q_seg = reinterpret_cast<uint32_t*>(q_v + kVoteThreads);    // [kVoteThreads + 4]
  uint32_t* acc = q_seg + kVoteThreads + 4;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t cells = a.chunk * kBins;
  const uint32_t seg_len = 1u << a.seg_shift;
  {
    const uint32_t item = a.item_list ? a.item_list[slot_of_item] : slot_of_item;
    const uint32_t c = item % a.n_chunks;
    // ref < n_ref, so sr = ref * ref_df < n_s
    const uint32_t ref = (uint32_t)(((unsigned long long)(item / a.n_chunks) * a.perm_mul) % a.n_ref);
    const uint32_t sr = ref * a.ref_df;
    const uint32_t mr_lo = c * a.chunk;
    // thread 0 publishes the frame of s_r; the barrier after the clear makes
    // it visible, and the previous item's readers are past the item-fetch
    // barrier before it is overwritten
    if (tid == 0) {
      const float4 p4 = a.s_pts[sr], n4 = a.s_nrm[sr];
      const FrameYZ f = frame_yz(make_float3(p4.x, p4.y, p4.z), make_float3(n4.x, n4.y, n4.z));
      sh.p_r = p4;
      sh.n_r = n4;
      sh.f_r1 = f.r1;
      sh.f_r2 = f.r2;
    }
    for (uint32_t i = tid; i < cells; i += kVoteThreads) acc[i] = 0u;
    block_sync();

    for (uint32_t base = 0; base < a.n_s; base += kVoteThreads) {
      // ---- one scene pair per thread: feature, key, lookup, sub-run
      const uint32_t i = base + tid;
      uint32_t len = 0, lo = 0, beta = 0;
      float2 v = make_float2(0.f, 0.f);
      if (i < a.n_s && i != sr) {
        float4 pi4 = a.s_pts[i], ni4 = a.s_nrm[i];
        float3 pi = make_float3(pi4.x, pi4.y, pi4.z);
        const float4 p4 = sh.p_r, n4 = sh.n_r;
        float4 f = pair_feature(make_float3(p4.x, p4.y, p4.z), make_float3(n4.x, n4.y, n4.z), pi,
                                make_float3(ni4.x, ni4.y, ni4.z), a.d_dist);
        uint32_t key = feature_key(f);
        if (key != 0u) {
          uint32_t run = ht_lookup(a.ht_keys, a.ht_runs, a.ht_mask, key);
          if (run != kNoRun && in_range<kCheck>(a, 2, run, a.K)) {
            const uint32_t* sp = a.split + (size_t)run * (a.n_chunks + 1);
            lo = __ldg(sp + c);
            len = __ldg(sp + c + 1) - lo;
            if (kCheck && !in_range<kCheck>(a, 3, (unsigned long long)lo + len, a.P + 1)) len = 0;
            if (c == 0 && !a.item_list) {
              st.votes += __ldg(a.run_count + run);
              st.matched += 1;
            }
            if (len) {
              FrameYZ fs;
              fs.r1 = sh.f_r1;
              fs.r2 = sh.f_r2;
              v = frame_point_yz(fs, pi);
              bool degenerate = fabsf(v.x) + fabsf(v.y) < 1e-12f || !isfinite(v.x) || !isfinite(v.y);
              beta = angle21(v) | ((degenerate || __ldg(a.run_flags + run)) ? kExactOnly : 0u);
            }
          }
        }
      }
      uint32_t n_seg_total;
      const uint32_t seg0 = block_excl_scan((len + seg_len - 1) >> a.seg_shift, sh.scan_seg, n_seg_total);
      q_lo[tid] = lo;
      q_len[tid] = len;
      q_beta[tid] = beta;
      q_v[tid] = v;
      q_seg[tid] = seg0;
      if (lane == 0) sh.seg_blk[warp] = seg0;
      if (tid == 0) {
        q_seg[kVoteThreads] = n_seg_total;
        sh.next = kVoteWarps;
      }
      block_sync();
      if (kCheck) {
        const uint32_t want = q_seg[tid] + ((q_len[tid] + seg_len - 1) >> a.seg_shift);
        if (q_seg[tid] != seg0 || q_seg[tid + 1] != want)
          in_range<kCheck>(a, 11, ((unsigned long long)tid << 32) | q_seg[tid + 1], want);
      }

      // ---- warps take segments; lanes stream consecutive entries
      uint32_t s = warp;
      while (s < n_seg_total) {
        // pair p with q_seg[p] <= s < q_seg[p+1]: the last index whose segment
        // offset is <= s (q_seg is nondecreasing and q_seg[0] = 0), found with
        // two ballots: first over q_seg[32 l] (its copy seg_blk[l]), then
        // inside that block of 32
        const uint32_t blk = 31u - __clz(__ballot_sync(0xffffffffu, sh.seg_blk[lane] <= s));
        const uint32_t plo = 32u * blk + 31u - __clz(__ballot_sync(0xffffffffu, q_seg[32 * blk + lane] <= s));
        const uint32_t p = plo;
        const uint32_t start = q_lo[p] + ((s - q_seg[p]) << a.seg_shift);
        uint32_t end = min(q_lo[p] + q_len[p], start + seg_len);
        // Always-on guard (one compare per segment of up to 1024 votes): a
        // segment outside its sub-run or the entry array is recorded, raises
        // kFlagBadIndex and is skipped, so the lookup fails instead of the
        // kernel reading outside the entries.
        if (start >= end || end > a.P) {
          if (lane == 0) {
            if (atomicCAS(&a.bad[3], 0ull, 1ull) == 0ull) {
              a.bad[4] = ((unsigned long long)p << 32) | s;
              a.bad[5] = ((unsigned long long)q_seg[p] << 32) | q_seg[p + 1];
              a.bad[6] = ((unsigned long long)q_lo[p] << 32) | q_len[p];
              a.bad[7] = ((unsigned long long)n_seg_total << 32) | q_seg[kVoteThreads];
              a.bad[8] = ((unsigned long long)base << 32) | item;
              a.bad[9] = ((unsigned long long)warp << 32) | plo;
            }
            atomicOr(a.flags, (uint32_t)kFlagBadIndex);
          }
          end = start;
        }
        const uint32_t bw = q_beta[p];
        const float2 vv = q_v[p];
        // Each entry holds the pair's m_r inside the chunk in its top 11 bits
        // and the model angle beta_m in its low 21.  With y = (beta_s + 2^20 -
        // beta_m) << 11, i.e. alpha + pi in 2^-32 turns (the row bits and the
        // exact-only flag shift out), the bin is the high word of y * 30 and
        // the low word the position inside the bin; a vote is ambiguous when
        // that position is within the margin m = 6 units of an edge.  One
        // 32 x 32 -> 64 multiply gives both words of the margin-shifted angle
        // y' = y - m:  30 y' = 30 y - 30 m, so a vote is unambiguous exactly
        // when the low word of 30 y' is at most m_span, and its high word is
        // then the bin of y.  For the ambiguous votes the high word is still
        // in [0, 29] (y' wraps to 2^32 + y - m only when 30 y < 30 m, giving
        // 29), so their provisional fast cell stays inside the accumulator.
        constexpr int kShift = 32 - PPF_ANGLE_BITS;
        const uint32_t bsh = ((bw + (1u << (PPF_ANGLE_BITS - 1))) << kShift) -
                             ((uint32_t)PPF_BIN_MARGIN_UNITS << kShift);
        constexpr uint32_t m_span =
            ((1u << PPF_ANGLE_BITS) - 2 * PPF_BIN_MARGIN_UNITS * PPF_N_ANGLE) << kShift;
        // (bin, position) of a margin-shifted angle: high and low word of 30 y'
        auto bin_pos = [](uint32_t yp) { return (unsigned long long)yp * (uint32_t)PPF_N_ANGLE; };
        const uint32_t* ep = a.entries + start + lane;
        const uint32_t n_here = end - start;
        // Votes near a bin edge were counted in their fast cell; move them to
        // the cell of the reference's exact arithmetic (rare: ~1.7e-4 of
        // votes).  The pass's entries are still in registers (c), so only the
        // exact path's own loads remain; pass_pos is the position of this
        // lane's first entry of the pass.
        auto fix_up = [&](uint32_t pass_pos, const uint32_t(&c)[kUnroll]) {
          uint32_t mask = 0;
#pragma unroll
          for (int u = 0; u < kUnroll; ++u)
            if ((uint32_t)bin_pos(bsh - (c[u] << kShift)) > m_span) mask |= 1u << u;
          while (mask) {
            const int u = __ffs(mask) - 1;
            mask &= mask - 1;
            uint32_t e = c[0];
#pragma unroll
            for (int k = 1; k < kUnroll; ++k) e = (u == k) ? c[k] : e;
            const uint32_t pos = pass_pos + 32u * (uint32_t)u;
            const unsigned long long bp = bin_pos(bsh - (e << kShift));
            const uint32_t row = (e >> PPF_ANGLE_BITS) * kBins;
            const uint32_t fast = row + (uint32_t)(bp >> 32);
            const uint32_t exact = row + exact_bin<kCheck>(a, pos, vv);
            if (exact != fast && in_range<kCheck>(a, 7, exact, cells)) {
              atomicAdd(&acc[fast], 0xffffffffu);
              atomicAdd(&acc[exact], 1u);
            }
            ++st.exact;
          }
        };
        if (bw & kExactOnly) {
          // degenerate frame vector or run: every vote takes the exact path
          for (uint32_t k = lane; k < n_here; k += 32) {
            const uint32_t row = (__ldg(a.entries + start + k) >> PPF_ANGLE_BITS) * kBins;
            const uint32_t cell = row + exact_bin<kCheck>(a, start + k, vv);
            if (in_range<kCheck>(a, 6, cell, cells)) atomicAdd(&acc[cell], 1u);
            ++st.exact;
          }
        } else {
          // kUnroll entries per lane per pass, branch-free: the fast cell of
          // every vote is counted, and the rare votes near a bin edge are
          // moved afterwards.  The last pass is masked to the segment's end.
          const uint32_t nfull = n_here / (32 * kUnroll);
          for (uint32_t it = 0; it < nfull; ++it, ep += 32 * kUnroll) {
            uint32_t c[kUnroll];
            bool amb = false;
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) c[u] = __ldg(ep + 32 * u);
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
              const unsigned long long bp = bin_pos(bsh - (c[u] << kShift));
              amb |= (uint32_t)bp > m_span;
              const uint32_t cell = (c[u] >> PPF_ANGLE_BITS) * kBins + (uint32_t)(bp >> 32);
              if (in_range<kCheck>(a, 8, cell, cells)) atomicAdd(&acc[cell], 1u);
            }
            if (amb) fix_up(start + it * 32u * kUnroll + lane, c);
          }
          for (uint32_t k = nfull * 32 * kUnroll + lane; k < n_here; k += 32) {
            const uint32_t e = __ldg(a.entries + start + k);
            const unsigned long long bp = bin_pos(bsh - (e << kShift));
            uint32_t cell = (e >> PPF_ANGLE_BITS) * kBins + (uint32_t)(bp >> 32);
            if ((uint32_t)bp > m_span) {
              cell = (e >> PPF_ANGLE_BITS) * kBins + exact_bin<kCheck>(a, start + k, vv);
              ++st.exact;
            }
            if (in_range<kCheck>(a, 8, cell, cells)) atomicAdd(&acc[cell], 1u);
          }
        }
        if (lane == 0) s = atomicAdd(&sh.next, 1u);
        s = __shfl_sync(0xffffffffu, s, 0);
      }
      if (kCheck && (q_seg[tid] != seg0 || q_len[tid] != len || q_lo[tid] != lo))
        in_range<kCheck>(a, 12, ((unsigned long long)tid << 32) | q_seg[tid], seg0);
      // No barrier here: the next tile writes the queue only after the two
      // barriers of its segment scan, which every warp reaches after its
      // last segment.
    }
    block_sync();  // all votes of the item are counted

    // ---- running maximum, emission
    uint32_t lmax = 0;
    for (uint32_t w = tid; w < cells; w += kVoteThreads) lmax = max(lmax, acc[w]);
#pragma unroll
    for (int o = 16; o; o >>= 1) lmax = max(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if (lane == 0) sh.wmax[warp] = lmax;
    block_sync();
    if (warp == 0) {
      uint32_t m = sh.wmax[lane];
#pragma unroll
      for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
      uint32_t old = 0;
      if (lane == 0) old = atomicMax(a.global_max, m);
      old = __shfl_sync(0xffffffffu, old, 0);
      if (lane == 0) sh.max = max(old, m);
    }
    block_sync();
    const float floor_v = a.floor >= 0.f ? a.floor : a.thr * (float)sh.max;
    // All-or-nothing slot reservation for the item's cells: an item that does
    // not fit writes nothing and is queued for a second launch after the
    // buffer has grown, so the buffer never holds a partial item.
    uint32_t my_n = 0;
    for (uint32_t cell = tid; cell < cells; cell += kVoteThreads) {
      const uint32_t cnt = acc[cell];
      my_n += (cnt != 0u && (a.emit_all || (float)cnt > floor_v)) ? 1u : 0u;
    }
    uint32_t item_total;
    const uint32_t my_off = block_excl_scan(my_n, sh.scan_emit, item_total);
    if (warp == 0) {
      // The whole warp walks the reservation loop in lockstep (lane 0 issues
      // the atomics, every exit condition is warp-uniform).
      uint32_t base_slot = 0xffffffffu;
      if (item_total) {
        if (lane == 0) atomicAdd(a.n_needed, (unsigned long long)item_total);
        uint32_t old = 0;
        if (lane == 0) old = *(volatile uint32_t*)a.n_cand;
        old = __shfl_sync(0xffffffffu, old, 0);
        for (int tries = 0; tries < (1 << 20); ++tries) {
          if ((unsigned long long)old + item_total > a.cand_cap) break;
          uint32_t prev = 0;
          if (lane == 0) prev = atomicCAS(a.n_cand, old, old + item_total);
          prev = __shfl_sync(0xffffffffu, prev, 0);
          if (prev == old) {
            base_slot = old;
            break;
          }
          old = prev;
        }
        if (base_slot == 0xffffffffu && lane == 0) {
          const uint32_t k = atomicAdd(a.n_redo, 1u);
          if (in_range<kCheck>(a, 9, k, a.n_items_total)) a.redo_items[k] = item;
        }
      }
      if (lane == 0) sh.base = base_slot;
    }
    block_sync();
    const uint32_t item_base = sh.base;
    if (item_base != 0xffffffffu) {
      uint32_t slot = item_base + my_off;
      for (uint32_t cell = tid; cell < cells; cell += kVoteThreads) {
        const uint32_t cnt = acc[cell];
        if (cnt != 0u && (a.emit_all || (float)cnt > floor_v)) {
          const uint32_t mr = mr_lo + cell / kBins, bin = cell % kBins;
          if (in_range<kCheck>(a, 10, slot, a.cand_cap)) {
            a.cand_code[slot] = ((unsigned long long)sr << 32) | ((unsigned long long)mr << 6) | bin;
            a.cand_count[slot] = cnt;
          }
          ++slot;
        }
      }
    }
    // The item-fetch barrier of the caller separates these reads of the
    // accumulator from the next item's clear.
  }
}

template <bool kCheck>
__global__ void __launch_bounds__(kVoteThreads, 1) vote_kernel(VoteArgs a) {
  __shared__ VoteShared sh;
  VoteStats st;
  for (;;) {
    const uint32_t slot = fetch_item(a.work_counter, sh);
    if (slot >= a.n_items) break;
    vote_item<kCheck>(a, slot, sh, st);
  }
  flush_stats(a, st);
}

// Several requests (model, scene) in one persistent launch: work items of
// all requests are numbered consecutively (request r owns items
// [item_off[r], item_off[r+1])) and fetched from one counter.  A block copies
// the arguments of an item's request into shared memory when the request
// changes; each request keeps its own running maximum, counters, candidate
// region and list of items that did not fit.
struct BatchArgs {
  const VoteArgs* reqs;
  const uint32_t* item_off;  // n_reqs + 1
  uint32_t n_reqs, n_items;
  uint32_t* work_counter;
};

template <bool kCheck>
__global__ void __launch_bounds__(kVoteThreads, 1) vote_batch_kernel(BatchArgs b) {
  __shared__ VoteShared sh;
  __shared__ VoteArgs s_args;
  VoteStats st;
  uint32_t cur = 0xffffffffu;
  for (;;) {
    const uint32_t g = fetch_item(b.work_counter, sh);
    if (g >= b.n_items) break;
    uint32_t lo = 0, hi = b.n_reqs;  // request r with item_off[r] <= g < item_off[r + 1]
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(b.item_off + mid) <= g) lo = mid;
      else hi = mid;
    }
    if (lo != cur) {  // uniform: every thread found the same request
      if (cur != 0xffffffffu) flush_stats(s_args, st);
      block_sync();
      constexpr int kWords = sizeof(VoteArgs) / 4;
      static_assert(sizeof(VoteArgs) % 4 == 0 && kWords <= kVoteThreads, "request arguments fit one copy pass");
      if (threadIdx.x < kWords)
        reinterpret_cast<uint32_t*>(&s_args)[threadIdx.x] = reinterpret_cast<const uint32_t*>(b.reqs + lo)[threadIdx.x];
      block_sync();
      cur = lo;
    }
    vote_item<kCheck>(s_args, g - __ldg(b.item_off + lo), sh, st);
  }
  if (cur != 0xffffffffu) flush_stats(s_args, st);
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
  a.P = t.P;
  a.K = t.K;
  a.m_r1 = t.frame_r1.as<float4>();
  a.m_r2 = t.frame_r2.as<float4>();
  a.m_pts = t.pts.as<float4>();
  a.n_m = t.n;
  a.chunk = t.chunk;
  a.n_chunks = t.n_chunks;
  const uint32_t shift = m.seg_shift.load(std::memory_order_relaxed);
  a.seg_shift = shift ? shift : kSegShiftDefault;
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

VoteResult run_votes(Context& ctx, const Model& m, const SceneData& s, bool emit_all, float floor) {
  VoteResult r;
  cudaStream_t stream = ctx.stream;
  VoteArgs a = make_args(m, s);
  a.emit_all = emit_all ? 1 : 0;
  a.floor = floor;
  const uint32_t n_items = a.n_ref * a.n_chunks;
  if (s.n < 2 || n_items == 0) return r;
  // counters: [0] work, [1] max, [2] n_cand, [3] n_redo, [4..9] 3 x u64 stats,
  // [10..11] u64 n_needed, [12] work counter of the second launch
  ctx.counters.reserve(64);
  PPF_CUDA(cudaMemsetAsync(ctx.counters.ptr, 0, 64, stream));
  // flags word and the bad-index record at byte 32 (site, value, bound, 7 words of detail)
  PPF_CUDA(cudaMemsetAsync(ctx.flags.ptr, 0, 32 + 80, stream));
  uint32_t* cnt = ctx.counters.as<uint32_t>();
  a.work_counter = cnt + 0;
  a.global_max = cnt + 1;
  a.n_cand = cnt + 2;
  a.n_redo = cnt + 3;
  a.stats = reinterpret_cast<unsigned long long*>(cnt + 4);
  a.n_needed = reinterpret_cast<unsigned long long*>(cnt + 10);
  a.flags = ctx.flags.as<uint32_t>();
  ctx.cand_codes.reserve(ctx.cand_cap * sizeof(unsigned long long));
  ctx.cand_counts.reserve(ctx.cand_cap * sizeof(uint32_t));
  ctx.redo_items.reserve((size_t)n_items * sizeof(uint32_t));
  a.cand_code = ctx.cand_codes.as<unsigned long long>();
  a.cand_count = ctx.cand_counts.as<uint32_t>();
  a.cand_cap = (uint32_t)std::min<size_t>(ctx.cand_cap, 0xffffffffu);
  a.redo_items = ctx.redo_items.as<uint32_t>();
  a.item_list = nullptr;
  a.n_items = n_items;
  a.n_items_total = n_items;
  const bool check = ctx.checks;
  a.bad = reinterpret_cast<unsigned long long*>(ctx.flags.as<uint32_t>() + 8);
  auto kernel = check ? vote_kernel<true> : vote_kernel<false>;

  const size_t smem = kVoteQueueBytes + vote_acc_words(a.chunk) * 4;
  PPF_REQUIRE((int)smem <= ctx.vote_smem_limit, PPF_ERR_INTERNAL, "vote accumulator too large");
  PPF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PPF_CUDA(cudaEventRecord(ctx.ev[0], stream));
  kernel<<<(unsigned)std::min<size_t>(n_items, (size_t)sm_count()), kVoteThreads, smem, stream>>>(a);
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
  uint32_t h[16];
  PPF_CUDA(cudaMemcpyAsync(h, ctx.counters.ptr, 64, cudaMemcpyDeviceToHost, stream));
  PPF_CUDA(cudaStreamSynchronize(stream));
  if (h[3]) {
    // Items that did not fit: grow the buffer (keeping what was emitted) to
    // what every item asked for, then count those items again.
    unsigned long long needed;
    memcpy(&needed, h + 10, sizeof(needed));
    r.n_needed = needed;
    const size_t want = std::max<size_t>(needed, 2 * ctx.cand_cap);
    PPF_REQUIRE(want < 0xffffffffull, PPF_ERR_OUT_OF_MEMORY, "more than 2^32 vote candidates");
    DevBuf nc, nn, items;
    nc.reserve(want * sizeof(unsigned long long));
    nn.reserve(want * sizeof(uint32_t));
    items.reserve((size_t)h[3] * sizeof(uint32_t));
    PPF_CUDA(cudaMemcpyAsync(nc.ptr, ctx.cand_codes.ptr, (size_t)h[2] * 8, cudaMemcpyDeviceToDevice, stream));
    PPF_CUDA(cudaMemcpyAsync(nn.ptr, ctx.cand_counts.ptr, (size_t)h[2] * 4, cudaMemcpyDeviceToDevice, stream));
    PPF_CUDA(cudaMemcpyAsync(items.ptr, ctx.redo_items.ptr, (size_t)h[3] * 4, cudaMemcpyDeviceToDevice, stream));
    ctx.cand_codes = std::move(nc);
    ctx.cand_counts = std::move(nn);
    ctx.cand_cap = want;
    a.cand_code = ctx.cand_codes.as<unsigned long long>();
    a.cand_count = ctx.cand_counts.as<uint32_t>();
    a.cand_cap = (uint32_t)want;
    a.item_list = items.as<uint32_t>();
    a.n_items = h[3];
    a.work_counter = cnt + 12;
    PPF_CUDA(cudaMemsetAsync(a.n_redo, 0, 4, stream));
    kernel<<<(unsigned)std::min<size_t>(a.n_items, (size_t)sm_count()), kVoteThreads, smem, stream>>>(a);
    PPF_CUDA(cudaGetLastError());
    ctx.launches++;
    r.n_redo = h[3];
    PPF_CUDA(cudaMemcpyAsync(h, ctx.counters.ptr, 64, cudaMemcpyDeviceToHost, stream));
    PPF_CUDA(cudaStreamSynchronize(stream));
    PPF_REQUIRE(h[3] == 0, PPF_ERR_INTERNAL, "vote candidates still do not fit");
  }
  PPF_CUDA(cudaEventRecord(ctx.ev[1], stream));
  PPF_CUDA(cudaEventSynchronize(ctx.ev[1]));
  {
    // flags word and bad-index record in one read
    unsigned long long rec[14];
    PPF_CUDA(cudaMemcpyAsync(rec, ctx.flags.ptr, sizeof(rec), cudaMemcpyDeviceToHost, stream));
    PPF_CUDA(cudaStreamSynchronize(stream));
    const uint32_t f = (uint32_t)(rec[0] & 0xffffffffu);
    if (f & kFlagBadIndex) {
      const unsigned long long* bad = rec + 4;
      std::string detail;
      for (int k = 3; k < 10; ++k)
        detail += " " + std::to_string(bad[k] >> 32) + ":" + std::to_string(bad[k] & 0xffffffffu);
      throw Error(PPF_ERR_INTERNAL, "vote kernel index out of range: site " + std::to_string(bad[0]) +
                                        " value " + std::to_string(bad[1]) + " bound " +
                                        std::to_string(bad[2]) + " |" + detail);
    }
  }
  PPF_CUDA(cudaEventElapsedTime(&r.vote_ms, ctx.ev[0], ctx.ev[1]));
  r.max_count = h[1];
  r.n_cand = h[2];
  unsigned long long* s64 = reinterpret_cast<unsigned long long*>(h + 4);
  r.n_votes = s64[0];
  r.n_matched = s64[1];
  r.n_exact = s64[2];
  return r;
}

void run_votes_batch(Context& ctx, std::vector<BatchVote>& reqs) {
  cudaStream_t stream = ctx.stream;
  const size_t n = reqs.size();
  if (n == 0) return;
  PPF_REQUIRE(n < (1u << 24), PPF_ERR_INVALID_ARGUMENT, "too many requests in one batch");
  std::vector<VoteArgs> args(n);
  std::vector<uint32_t> item_off(n + 1, 0);
  // per request 16 counter words ([1] max, [2] n_cand, [3] n_redo, [4..9]
  // stats, [10..11] n_needed, [12] work counter of its redo launch), then the
  // batch's own work counter
  ctx.batch_counters.reserve((n + 1) * 64);
  PPF_CUDA(cudaMemsetAsync(ctx.batch_counters.ptr, 0, (n + 1) * 64, stream));
  PPF_CUDA(cudaMemsetAsync(ctx.flags.ptr, 0, 32 + 80, stream));
  uint32_t* cnt0 = ctx.batch_counters.as<uint32_t>();
  size_t total = 0, smem = kVoteQueueBytes;
  for (size_t i = 0; i < n; ++i) {
    const VoteArgs a0 = make_args(*reqs[i].m, *reqs[i].s);
    const uint64_t items = reqs[i].s->n < 2 ? 0 : (uint64_t)a0.n_ref * a0.n_chunks;
    total += items;
    PPF_REQUIRE(total < 0xffffffffull, PPF_ERR_INVALID_ARGUMENT, "more than 2^32 work items in one batch");
    item_off[i + 1] = (uint32_t)total;
    smem = std::max(smem, kVoteQueueBytes + vote_acc_words(a0.chunk) * 4);
  }
  PPF_REQUIRE((int)smem <= ctx.vote_smem_limit, PPF_ERR_INTERNAL, "vote accumulator too large");
  ctx.batch_redo.reserve(std::max<size_t>(total, 1) * sizeof(uint32_t));
  for (size_t i = 0; i < n; ++i) {
    VoteArgs& a = args[i];
    a = make_args(*reqs[i].m, *reqs[i].s);
    a.emit_all = 0;
    a.floor = -1.f;
    uint32_t* cnt = cnt0 + 16 * i;
    a.work_counter = nullptr;
    a.global_max = cnt + 1;
    a.n_cand = cnt + 2;
    a.n_redo = cnt + 3;
    a.stats = reinterpret_cast<unsigned long long*>(cnt + 4);
    a.n_needed = reinterpret_cast<unsigned long long*>(cnt + 10);
    a.flags = ctx.flags.as<uint32_t>();
    a.bad = reinterpret_cast<unsigned long long*>(ctx.flags.as<uint32_t>() + 8);
    reqs[i].cap = std::max<size_t>(reqs[i].cap, 1024);
    PPF_REQUIRE(reqs[i].cap < 0xffffffffull, PPF_ERR_INVALID_ARGUMENT, "candidate capacity beyond 2^32");
    reqs[i].codes.reserve(reqs[i].cap * sizeof(unsigned long long));
    reqs[i].counts.reserve(reqs[i].cap * sizeof(uint32_t));
    a.cand_code = reqs[i].codes.as<unsigned long long>();
    a.cand_count = reqs[i].counts.as<uint32_t>();
    a.cand_cap = (uint32_t)reqs[i].cap;
    a.redo_items = ctx.batch_redo.as<uint32_t>() + item_off[i];
    a.item_list = nullptr;
    a.n_items = item_off[i + 1] - item_off[i];
    a.n_items_total = a.n_items;
  }
  ctx.batch_args.reserve(n * sizeof(VoteArgs));
  ctx.batch_off.reserve((n + 1) * sizeof(uint32_t));
  PPF_CUDA(cudaMemcpyAsync(ctx.batch_args.ptr, args.data(), n * sizeof(VoteArgs), cudaMemcpyHostToDevice, stream));
  PPF_CUDA(cudaMemcpyAsync(ctx.batch_off.ptr, item_off.data(), (n + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice,
                           stream));
  BatchArgs b;
  b.reqs = ctx.batch_args.as<VoteArgs>();
  b.item_off = ctx.batch_off.as<uint32_t>();
  b.n_reqs = (uint32_t)n;
  b.n_items = (uint32_t)total;
  b.work_counter = cnt0 + 16 * n;
  const bool check = ctx.checks;
  auto bkernel = check ? vote_batch_kernel<true> : vote_batch_kernel<false>;
  auto kernel = check ? vote_kernel<true> : vote_kernel<false>;
  PPF_CUDA(cudaEventRecord(ctx.ev[0], stream));
  if (total) {
    PPF_CUDA(cudaFuncSetAttribute(bkernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    bkernel<<<(unsigned)std::min<size_t>(total, (size_t)sm_count()), kVoteThreads, smem, stream>>>(b);
    PPF_CUDA(cudaGetLastError());
    ctx.launches++;
  }
  std::vector<uint32_t> h((n + 1) * 16);
  PPF_CUDA(cudaMemcpyAsync(h.data(), cnt0, (n + 1) * 64, cudaMemcpyDeviceToHost, stream));
  PPF_CUDA(cudaStreamSynchronize(stream));
  // Requests whose cells did not all fit: grow their buffers (keeping what was
  // emitted) and count their remaining items again, one request at a time.
  for (size_t i = 0; i < n; ++i) {
    uint32_t* hc = h.data() + 16 * i;
    reqs[i].r.n_redo = hc[3];
    if (!hc[3]) continue;
    unsigned long long needed;
    memcpy(&needed, hc + 10, sizeof(needed));
    reqs[i].r.n_needed = needed;
    const size_t want = std::max<size_t>(needed, 2 * reqs[i].cap);
    PPF_REQUIRE(want < 0xffffffffull, PPF_ERR_OUT_OF_MEMORY, "more than 2^32 vote candidates");
    DevBuf nc, nn, items;
    nc.reserve(want * sizeof(unsigned long long));
    nn.reserve(want * sizeof(uint32_t));
    items.reserve((size_t)hc[3] * sizeof(uint32_t));
    PPF_CUDA(cudaMemcpyAsync(nc.ptr, reqs[i].codes.ptr, (size_t)hc[2] * 8, cudaMemcpyDeviceToDevice, stream));
    PPF_CUDA(cudaMemcpyAsync(nn.ptr, reqs[i].counts.ptr, (size_t)hc[2] * 4, cudaMemcpyDeviceToDevice, stream));
    PPF_CUDA(cudaMemcpyAsync(items.ptr, args[i].redo_items, (size_t)hc[3] * 4, cudaMemcpyDeviceToDevice, stream));
    reqs[i].codes = std::move(nc);
    reqs[i].counts = std::move(nn);
    reqs[i].cap = want;
    VoteArgs a = args[i];
    a.cand_code = reqs[i].codes.as<unsigned long long>();
    a.cand_count = reqs[i].counts.as<uint32_t>();
    a.cand_cap = (uint32_t)want;
    a.item_list = items.as<uint32_t>();
    a.n_items = hc[3];
    a.work_counter = cnt0 + 16 * i + 12;
    PPF_CUDA(cudaMemsetAsync(a.n_redo, 0, 4, stream));
    const size_t smem_i = kVoteQueueBytes + vote_acc_words(a.chunk) * 4;
    PPF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_i));
    kernel<<<(unsigned)std::min<size_t>(a.n_items, (size_t)sm_count()), kVoteThreads, smem_i, stream>>>(a);
    PPF_CUDA(cudaGetLastError());
    ctx.launches++;
    PPF_CUDA(cudaMemcpyAsync(hc, cnt0 + 16 * i, 64, cudaMemcpyDeviceToHost, stream));
    PPF_CUDA(cudaStreamSynchronize(stream));
    PPF_REQUIRE(hc[3] == 0, PPF_ERR_INTERNAL, "vote candidates still do not fit");
  }
  PPF_CUDA(cudaEventRecord(ctx.ev[1], stream));
  PPF_CUDA(cudaEventSynchronize(ctx.ev[1]));
  {
    unsigned long long rec[14];
    PPF_CUDA(cudaMemcpyAsync(rec, ctx.flags.ptr, sizeof(rec), cudaMemcpyDeviceToHost, stream));
    PPF_CUDA(cudaStreamSynchronize(stream));
    if ((uint32_t)(rec[0] & 0xffffffffu) & kFlagBadIndex)
      throw Error(PPF_ERR_INTERNAL, "vote kernel index out of range: site " + std::to_string(rec[4]) +
                                        " value " + std::to_string(rec[5]) + " bound " + std::to_string(rec[6]));
  }
  float ms = 0;
  PPF_CUDA(cudaEventElapsedTime(&ms, ctx.ev[0], ctx.ev[1]));
  for (size_t i = 0; i < n; ++i) {
    const uint32_t* hc = h.data() + 16 * i;
    VoteResult& r = reqs[i].r;
    r.max_count = hc[1];
    r.n_cand = hc[2];
    unsigned long long s64[3];
    memcpy(s64, hc + 4, sizeof(s64));
    r.n_votes = s64[0];
    r.n_matched = s64[1];
    r.n_exact = s64[2];
    // the batch's device time, split by work items
    r.vote_ms = total ? ms * (float)(item_off[i + 1] - item_off[i]) / (float)total : 0.f;
  }
}

void tune_vote_segments(Context& ctx, Model& m, const SceneData& s, uint64_t signature) {
  if (m.seg_shift) return;
  if (ctx.forced_seg_shift) {
    m.seg_shift = ctx.forced_seg_shift;
    return;
  }
  auto it = ctx.seg_tuned.find(signature);
  if (it != ctx.seg_tuned.end()) {
    m.seg_shift = it->second;
    return;
  }
  if (!ctx.tune || s.n < 2) {
    m.seg_shift = kSegShiftDefault;
    return;
  }
  cudaStream_t stream = ctx.stream;
  VoteArgs a = make_args(m, s);
  const uint32_t n_items = a.n_ref * a.n_chunks;
  // about two items per SM: the first items of the pass's scrambled order of
  // scene reference points, for every chunk of the model
  const uint32_t sample = std::min<uint32_t>(n_items, 2u * (uint32_t)sm_count());
  // The sample launches count and emit nothing: no cell exceeds an infinite
  // floor.  Their counters live in a buffer of their own.
  ctx.tune_counters.reserve(64 + 32 + 80);
  uint32_t* cnt = ctx.tune_counters.as<uint32_t>();
  a.emit_all = 0;
  a.floor = INFINITY;
  a.work_counter = cnt + 0;
  a.global_max = cnt + 1;
  a.n_cand = cnt + 2;
  a.n_redo = cnt + 3;
  a.stats = reinterpret_cast<unsigned long long*>(cnt + 4);
  a.n_needed = reinterpret_cast<unsigned long long*>(cnt + 10);
  a.flags = cnt + 16;
  a.bad = reinterpret_cast<unsigned long long*>(cnt + 24);
  a.cand_code = nullptr;
  a.cand_count = nullptr;
  a.cand_cap = 0;
  a.redo_items = nullptr;
  a.n_items_total = 0;
  a.item_list = nullptr;
  a.n_items = sample;
  const size_t smem = kVoteQueueBytes + vote_acc_words(a.chunk) * 4;
  PPF_REQUIRE((int)smem <= ctx.vote_smem_limit, PPF_ERR_INTERNAL, "vote accumulator too large");
  auto kernel = vote_kernel<false>;
  PPF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  constexpr int kCands = sizeof(kSegShifts) / sizeof(kSegShifts[0]);
  float best_ms[kCands];
  for (int c = 0; c < kCands; ++c) best_ms[c] = INFINITY;
  // two rounds over the candidates, the faster of each candidate's two times
  for (int round = 0; round < 2; ++round)
    for (int c = 0; c < kCands; ++c) {
      a.seg_shift = kSegShifts[c];
      PPF_CUDA(cudaMemsetAsync(cnt, 0, 64 + 32 + 80, stream));
      PPF_CUDA(cudaEventRecord(ctx.ev[0], stream));
      kernel<<<std::min<uint32_t>(sample, (uint32_t)sm_count()), kVoteThreads, smem, stream>>>(a);
      PPF_CUDA(cudaGetLastError());
      ctx.launches++;
      PPF_CUDA(cudaEventRecord(ctx.ev[1], stream));
      PPF_CUDA(cudaEventSynchronize(ctx.ev[1]));
      float ms = 0;
      PPF_CUDA(cudaEventElapsedTime(&ms, ctx.ev[0], ctx.ev[1]));
      best_ms[c] = std::min(best_ms[c], ms);
    }
  uint32_t flags = 0;
  PPF_CUDA(cudaMemcpyAsync(&flags, cnt + 16, sizeof(flags), cudaMemcpyDeviceToHost, stream));
  PPF_CUDA(cudaStreamSynchronize(stream));
  PPF_REQUIRE(!(flags & kFlagBadIndex), PPF_ERR_INTERNAL, "vote kernel index out of range while tuning");
  // the default stays unless another length is at least 2% faster
  int pick = -1;
  for (int c = 0; c < kCands; ++c)
    if (kSegShifts[c] == kSegShiftDefault) pick = c;
  for (int c = 0; c < kCands; ++c)
    if (best_ms[c] < 0.98f * best_ms[pick]) pick = c;
  m.seg_shift = kSegShifts[pick];
  ctx.seg_tuned[signature] = m.seg_shift;
}

void pair_vote_counts(Context& ctx, const Model& m, const SceneData& s, uint64_t* out_dev) {
  VoteArgs a = make_args(m, s);
  dim3 grid((s.n + 255) / 256, std::min<uint32_t>(s.n, 65535u));
  pair_vote_counts_kernel<<<grid, 256, 0, ctx.stream>>>(a, reinterpret_cast<unsigned long long*>(out_dev));
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;
}

// ---- allocation-free vote pass (ppf_model_vote_cells_noalloc)
//
// The same vote kernel as run_votes, for callers that must not allocate
// device memory while they run: a serving process whose device-memory budget
// was reserved at start-up (its own pool holds the rest of the device, so a
// further cudaMalloc fails or takes memory the budget does not have) and
// latency-bound loops that cannot take cudaMalloc/cudaFree latency or the
// device-wide synchronisation that cudaFree implies.  Everything the pass
// needs besides the caller's inputs and outputs lives in one static device
// array of this file, which every GPU that loads the library holds until the
// process exits:
//   [0, 256)        counters (the run_votes layout), the flags word at byte
//                   64 and the bad-index record at byte 96
//   items           the work items that did not fit the caller's output
//   points, normals the scene packed to float4
constexpr uint32_t kNoAllocMaxScenePoints = 65536;
constexpr uint32_t kNoAllocMaxItems = 262144;  // scene reference points x model chunks
constexpr size_t kNoAllocHeader = 256;
constexpr size_t kNoAllocItemsOff = kNoAllocHeader;
constexpr size_t kNoAllocPtsOff = kNoAllocItemsOff + (size_t)kNoAllocMaxItems * 4;
constexpr size_t kNoAllocNrmOff = kNoAllocPtsOff + (size_t)kNoAllocMaxScenePoints * 16;
constexpr size_t kNoAllocBytes = kNoAllocNrmOff + (size_t)kNoAllocMaxScenePoints * 16;  // 3 MiB + 256 B
static_assert(kNoAllocPtsOff % 256 == 0 && kNoAllocNrmOff % 256 == 0, "scratch sections stay aligned");

static __device__ __align__(256) unsigned char g_vote_scratch[kNoAllocBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_vote_scratch_mutex;
unsigned char* g_vote_scratch_ptr[kNoAllocMaxDevices] = {};

// Device address of g_vote_scratch on `device`, which must be current.  The
// first call per device looks it up; later calls reuse it.
unsigned char* vote_scratch(int device) {
  PPF_REQUIRE(device >= 0 && device < kNoAllocMaxDevices, PPF_ERR_INVALID_ARGUMENT,
              "device index beyond the allocation-free path's table of 64 devices");
  std::lock_guard<std::mutex> lock(g_vote_scratch_mutex);
  if (!g_vote_scratch_ptr[device]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_vote_scratch);
    if (e != cudaSuccess || !ptr)
      throw Error(PPF_ERR_CUDA, std::string("cudaGetSymbolAddress(vote scratch): ") + cudaGetErrorString(e));
    g_vote_scratch_ptr[device] = static_cast<unsigned char*>(ptr);
  }
  return g_vote_scratch_ptr[device];
}

__global__ void pack_scene_kernel(const float* __restrict__ xyz, const float* __restrict__ nxyz,
                                  uint32_t n, float4* __restrict__ pts, float4* __restrict__ nrm) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    pts[i] = make_float4(xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2], 0.f);
    nrm[i] = make_float4(nxyz[3 * (size_t)i], nxyz[3 * (size_t)i + 1], nxyz[3 * (size_t)i + 2], 0.f);
  }
}

}  // namespace

void vote_cells_noalloc(Context& ctx, const Model& m, const float* xyz, const float* nxyz,
                        uint64_t n, uint32_t ref_df, float vote_floor, uint64_t* codes,
                        uint32_t* counts, uint64_t capacity, uint64_t* n_out, uint32_t* max_out) {
  *n_out = 0;
  if (max_out) *max_out = 0;
  PPF_REQUIRE(n <= kNoAllocMaxScenePoints, PPF_ERR_INVALID_ARGUMENT,
              "scene of " + std::to_string(n) + " points exceeds the allocation-free limit of " +
                  std::to_string(kNoAllocMaxScenePoints));
  if (n < 2) return;
  PPF_REQUIRE(xyz && nxyz && is_device_pointer(xyz, ctx.device) && is_device_pointer(nxyz, ctx.device),
              PPF_ERR_INVALID_ARGUMENT, "scene points and normals must be device memory");
  PPF_REQUIRE(capacity == 0 || (codes && counts && is_device_pointer(codes, ctx.device) &&
                                   is_device_pointer(counts, ctx.device)),
              PPF_ERR_INVALID_ARGUMENT, "vote cell outputs must be device memory");
  PPF_REQUIRE(capacity <= 0xffffffffull, PPF_ERR_INVALID_ARGUMENT, "capacity beyond 2^32 - 1 cells");
  ref_df = ref_df ? ref_df : 1;
  const uint64_t n_ref = (n + ref_df - 1) / ref_df;
  const uint64_t n_items = n_ref * m.t.n_chunks;
  PPF_REQUIRE(n_items <= kNoAllocMaxItems, PPF_ERR_INVALID_ARGUMENT,
              std::to_string(n_ref) + " scene reference points x " + std::to_string(m.t.n_chunks) +
                  " model chunks exceed the allocation-free limit of " + std::to_string(kNoAllocMaxItems) +
                  " work items");
  const size_t smem = kVoteQueueBytes + vote_acc_words(m.t.chunk) * 4;
  PPF_REQUIRE((int)smem <= ctx.vote_smem_limit, PPF_ERR_INTERNAL, "vote accumulator too large");

  unsigned char* scratch = vote_scratch(ctx.device);
  cudaStream_t stream = ctx.stream;
  float4* pts = reinterpret_cast<float4*>(scratch + kNoAllocPtsOff);
  float4* nrm = reinterpret_cast<float4*>(scratch + kNoAllocNrmOff);
  // the counter header is the only part of the scratch that must start at zero
  PPF_CUDA(cudaMemsetAsync(scratch, 0, kNoAllocHeader, stream));
  pack_scene_kernel<<<grid_for(n, 256), 256, 0, stream>>>(xyz, nxyz, (uint32_t)n, pts, nrm);
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;

  // scene with no storage of its own: make_args takes n, d_dist and ref_df from it
  SceneData s;
  s.n = (uint32_t)n;
  s.d_dist = m.t.d_dist;  // ppf_registration builds each scene with its model's d_dist
  s.ref_df = ref_df;
  VoteArgs a = make_args(m, s);
  a.s_pts = pts;
  a.s_nrm = nrm;
  a.emit_all = 0;
  a.floor = vote_floor;
  uint32_t* cnt = reinterpret_cast<uint32_t*>(scratch);
  a.work_counter = cnt + 0;
  a.global_max = cnt + 1;
  a.n_cand = cnt + 2;
  a.n_redo = cnt + 3;
  a.stats = reinterpret_cast<unsigned long long*>(cnt + 4);
  a.n_needed = reinterpret_cast<unsigned long long*>(cnt + 10);
  a.flags = cnt + 16;
  a.bad = reinterpret_cast<unsigned long long*>(cnt + 24);
  a.cand_code = reinterpret_cast<unsigned long long*>(codes);
  a.cand_count = counts;
  a.cand_cap = (uint32_t)capacity;
  a.redo_items = reinterpret_cast<uint32_t*>(scratch + kNoAllocItemsOff);
  a.n_items_total = kNoAllocMaxItems;
  a.item_list = nullptr;
  a.n_items = (uint32_t)n_items;
  auto kernel = ctx.checks ? vote_kernel<true> : vote_kernel<false>;
  PPF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kernel<<<(unsigned)std::min<uint64_t>(n_items, (uint64_t)sm_count()), kVoteThreads, smem, stream>>>(a);
  PPF_CUDA(cudaGetLastError());
  ctx.launches++;

  unsigned long long h[22];  // bytes [0, 176): counters, flags, bad-index record
  PPF_CUDA(cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, stream));
  PPF_CUDA(cudaStreamSynchronize(stream));
  const uint32_t* h32 = reinterpret_cast<const uint32_t*>(h);
  if (h32[16] & kFlagBadIndex) {
    const unsigned long long* bad = h + 12;
    throw Error(PPF_ERR_INTERNAL, "vote kernel index out of range: site " + std::to_string(bad[0]) +
                                      " value " + std::to_string(bad[1]) + " bound " +
                                      std::to_string(bad[2]));
  }
  if (max_out) *max_out = h32[1];
  if (h32[3]) {
    const unsigned long long needed = h[5];
    *n_out = needed;
    throw Error(PPF_ERR_OUT_OF_MEMORY,
                "vote cell output of " + std::to_string(capacity) + " entries is too small: this call needed " +
                    std::to_string(needed) + " (the cells of the items that fit were written)");
  }
  *n_out = h32[2];
}

}  // namespace ppf
