// TEST INFRASTRUCTURE ONLY: the bit-exact GPU oracle.
//
// Drives the reference's OWN CUDA kernels (src/cuda/kernel.cu, compiled in
// place from the reference sources with its arithmetic flags; see
// oracle/Makefile) in the order Scene::Scene / Model::Model /
// Model::ppf_lookup run them (src/cuda/scene.cu:24-99,
// src/cuda/model.cu:43-306, include/impl/parallel_hash_array.hpp:55-92), and
// returns every intermediate the tests compare against.  The orchestration
// below is written for this harness: Thrust calls restate the reference's
// (same primitives, same comparators), and the hash-array key vectors get one
// padding element so the reference kernels' read of keys[lower_bound] when
// the bound equals the size (kernel.cu:492,521,728) stays inside the
// allocation.  Sizes are limited to n <= 46340 points (the reference indexes
// pairs with int, kernel.cu:409,433).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <thrust/binary_search.h>
#include <thrust/copy.h>
#include <thrust/count.h>
#include <thrust/device_vector.h>
#include <thrust/extrema.h>
#include <thrust/functional.h>
#include <thrust/host_vector.h>
#include <thrust/inner_product.h>
#include <thrust/iterator/constant_iterator.h>
#include <thrust/reduce.h>
#include <thrust/scan.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>

#include "kernel.h"

namespace {

#define RH_CHECK(x)                                                                    \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      snprintf(g_err, sizeof(g_err), "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
      return -1;                                                                       \
    }                                                                                  \
  } while (0)

char g_err[512];

int blocks_for(size_t count) {
  return std::min(((int)count + BLOCK_SIZE - 1) / BLOCK_SIZE, MAX_NBLOCKS);
}

// Sorted-input histogram: unique values and run counts (include/impl/util.hpp:30-52).
template <typename V, typename C>
void histogram(const thrust::device_vector<V>& input, thrust::device_vector<V>& values,
               thrust::device_vector<C>& counts) {
  if (input.empty()) {
    values.clear();
    counts.clear();
    return;
  }
  thrust::device_vector<V> data(input);
  C num_bins = thrust::inner_product(data.begin(), data.end() - 1, data.begin() + 1, C(1),
                                     thrust::plus<C>(), thrust::not_equal_to<V>());
  values.resize(num_bins);
  counts.resize(num_bins);
  thrust::reduce_by_key(data.begin(), data.end(), thrust::constant_iterator<C>(1),
                        values.begin(), counts.begin());
}

// ParallelHashArray<unsigned int> (parallel_hash_array.hpp:55-77); keys are
// sorted in place as in the reference.  `hashkeys` carries one extra 0 at the end.
struct Pha {
  thrust::device_vector<size_t> map;
  thrust::device_vector<unsigned int> hashkeys;  // K + 1 (padded)
  thrust::device_vector<size_t> counts, first;
  size_t K = 0;
  void build(thrust::device_vector<unsigned int>& data) {
    map.resize(data.size());
    thrust::sequence(map.begin(), map.end());
    thrust::sort_by_key(data.begin(), data.end(), map.begin());
    thrust::device_vector<unsigned int> uk;
    histogram(data, uk, counts);
    K = uk.size();
    hashkeys.resize(K + 1);
    thrust::copy(uk.begin(), uk.end(), hashkeys.begin());
    hashkeys[K] = 0;
    first.resize(K);
    thrust::exclusive_scan(counts.begin(), counts.end(), first.begin());
  }
  // GetIndices (parallel_hash_array.hpp:80-92)
  void indices(const thrust::device_vector<unsigned int>& q, thrust::device_vector<size_t>& out) {
    out.resize(q.size());
    thrust::lower_bound(hashkeys.begin(), hashkeys.begin() + K, q.begin(), q.end(), out.begin());
  }
};

struct Cloud {
  thrust::device_vector<float3> pts, nrm;
  int n = 0;
  void load(const float* p, const float* q, int count) {
    n = count;
    thrust::host_vector<float3> hp(n), hn(n);
    for (int i = 0; i < n; ++i) {
      hp[i] = make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
      hn[i] = make_float3(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
    }
    pts = hp;
    nrm = hn;
  }
};

// Scene::initPPFs + ppf_hash_kernel (scene.cu:44-54,64-99).
int cloud_keys(Cloud& c, float d_dist, unsigned ref_df, thrust::device_vector<unsigned int>& keys) {
  size_t nn = (size_t)c.n * c.n;
  thrust::device_vector<float4> ppfs(nn);
  int blocks = std::min(((int)(c.n + BLOCK_SIZE) - 1) / BLOCK_SIZE, MAX_NBLOCKS);
  ppf_kernel<<<blocks, BLOCK_SIZE>>>(thrust::raw_pointer_cast(c.pts.data()),
                                     thrust::raw_pointer_cast(c.nrm.data()),
                                     thrust::raw_pointer_cast(ppfs.data()), c.n, ref_df, d_dist);
  RH_CHECK(cudaGetLastError());
  RH_CHECK(cudaDeviceSynchronize());
  keys.assign(nn, 0u);
  ppf_hash_kernel<<<blocks_for(nn), BLOCK_SIZE>>>(thrust::raw_pointer_cast(ppfs.data()),
                                                  thrust::raw_pointer_cast(keys.data()), (int)nn);
  RH_CHECK(cudaGetLastError());
  RH_CHECK(cudaDeviceSynchronize());
  return 0;
}

}  // namespace

extern "C" {

const char* rh_last_error() { return g_err; }

// Keys of all n*n ordered pairs (Scene::Scene with the given ref_df).
int rh_pair_keys(const float* pts, const float* nrm, int n, float d_dist, unsigned ref_df,
                 uint32_t* keys_out) {
  if (n > 46340) return -2;
  Cloud c;
  c.load(pts, nrm, n);
  thrust::device_vector<unsigned int> keys;
  if (cloud_keys(c, d_dist, ref_df, keys)) return -1;
  thrust::copy(keys.begin(), keys.end(), keys_out);
  return 0;
}

// Model::Model hash array (model.cu:66-79): returns K and fills the sorted
// position map (n*n), unique keys, counts and first offsets (K each).
long long rh_model_tables(const float* pts, const float* nrm, int n, float d_dist, uint32_t* map_out,
                          uint32_t* uniq_out, uint32_t* counts_out, uint32_t* first_out,
                          long long cap) {
  if (n > 46340) return -2;
  Cloud c;
  c.load(pts, nrm, n);
  thrust::device_vector<unsigned int> keys;
  if (cloud_keys(c, d_dist, 1, keys)) return -1;
  Pha H;
  H.build(keys);
  if ((long long)H.K > cap) return -3;
  thrust::host_vector<size_t> m = H.map, cnt = H.counts, fst = H.first;
  thrust::host_vector<unsigned int> uk(H.hashkeys.begin(), H.hashkeys.begin() + H.K);
  for (size_t i = 0; i < m.size(); ++i) map_out[i] = (uint32_t)m[i];
  for (size_t k = 0; k < H.K; ++k) {
    uniq_out[k] = uk[k];
    counts_out[k] = (uint32_t)cnt[k];
    first_out[k] = (uint32_t)fst[k];
  }
  return (long long)H.K;
}

typedef struct rh_result {
  unsigned long long n_votes;
  unsigned long long n_unique;
  unsigned int max_count;
  float min_votecount;
  unsigned long long n_kept;
  unsigned long long max_idx;
  float pose[16];
  float elapsed_ms;  // device time of the timed stages (CUDA events)
} rh_result;

}  // extern "C"

namespace {

struct Timer {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  Timer() {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
  }
  float stop() {
    float ms = 0;
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
  }
  ~Timer() {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
};

// ComputeUniqueVotes up to the histogram (model.cu:95-151): every vote of the
// scene's reference rows, sorted, reduced to unique codes and their counts.
int unique_votes(Cloud& M, Cloud& S, Pha& H, thrust::device_vector<unsigned int>& skeys, float d_dist,
                 thrust::device_vector<unsigned long>& votes, thrust::device_vector<unsigned int>& vote_counts,
                 unsigned long long* n_votes, unsigned long long* pair_counts) {
  size_t nn = skeys.size();
  thrust::device_vector<size_t> sidx;
  H.indices(skeys, sidx);
  thrust::device_vector<unsigned long> vcounts(nn, 0ul);
  ppf_vote_count_kernel<<<blocks_for(nn), BLOCK_SIZE>>>(
      thrust::raw_pointer_cast(skeys.data()), thrust::raw_pointer_cast(sidx.data()),
      thrust::raw_pointer_cast(H.hashkeys.data()), thrust::raw_pointer_cast(H.counts.data()),
      thrust::raw_pointer_cast(vcounts.data()), (int)nn);
  RH_CHECK(cudaGetLastError());
  RH_CHECK(cudaDeviceSynchronize());
  if (pair_counts) thrust::copy(vcounts.begin(), vcounts.end(), pair_counts);
  thrust::device_vector<size_t> vidx(nn);
  thrust::exclusive_scan(vcounts.begin(), vcounts.end(), vidx.begin());
  size_t num_votes = (size_t)vcounts.back() + (size_t)vidx.back();
  *n_votes = num_votes;
  vcounts.clear();
  vcounts.shrink_to_fit();
  thrust::device_vector<unsigned long> votes_all(num_votes);
  ppf_vote_kernel<<<blocks_for(nn), BLOCK_SIZE>>>(
      thrust::raw_pointer_cast(skeys.data()), thrust::raw_pointer_cast(sidx.data()),
      thrust::raw_pointer_cast(H.hashkeys.data()), thrust::raw_pointer_cast(H.counts.data()),
      thrust::raw_pointer_cast(H.first.data()), thrust::raw_pointer_cast(H.map.data()),
      thrust::raw_pointer_cast(M.pts.data()), thrust::raw_pointer_cast(M.nrm.data()), M.n,
      thrust::raw_pointer_cast(S.pts.data()), thrust::raw_pointer_cast(S.nrm.data()), S.n,
      thrust::raw_pointer_cast(vidx.data()), thrust::raw_pointer_cast(votes_all.data()), (int)nn, d_dist);
  RH_CHECK(cudaGetLastError());
  RH_CHECK(cudaDeviceSynchronize());
  vidx.clear();
  vidx.shrink_to_fit();
  sidx.clear();
  sidx.shrink_to_fit();
  thrust::sort(votes_all.begin(), votes_all.end());
  histogram(votes_all, votes, vote_counts);
  return 0;
}

// ComputeTransformations, ComputeWeightedVoteCounts and ClusterTransformations
// (model.cu:173-244) on the kept votes (reference order), then the argmax and
// the pose assembly of ppf_registration (model.cu:293-295, ppf.cu:78-93).
int post_votes(Cloud& M, Cloud& S, thrust::device_vector<float>& wts, thrust::device_vector<unsigned long>& votes,
               thrust::device_vector<unsigned int>& vote_counts, float d_dist, int use_l1, int use_avg,
               rh_result* res, float* transforms, float* trans, float* quats, float* scores, long long cap) {
  const size_t U = votes.size();
  thrust::device_vector<float> T(U * 16, 0.f);
  trans_calc_kernel2<<<blocks_for(U), BLOCK_SIZE>>>(
      thrust::raw_pointer_cast(votes.data()), thrust::raw_pointer_cast(M.pts.data()),
      thrust::raw_pointer_cast(M.nrm.data()), thrust::raw_pointer_cast(S.pts.data()),
      thrust::raw_pointer_cast(S.nrm.data()), thrust::raw_pointer_cast(T.data()), (int)U);
  RH_CHECK(cudaGetLastError());
  thrust::device_vector<float> wvc(U, 0.f);
  vote_weight_kernel<<<blocks_for(U), BLOCK_SIZE>>>(
      thrust::raw_pointer_cast(votes.data()), thrust::raw_pointer_cast(vote_counts.data()),
      thrust::raw_pointer_cast(wts.data()), thrust::raw_pointer_cast(wvc.data()), (int)U);
  RH_CHECK(cudaGetLastError());
  thrust::device_vector<float3> tt(U, make_float3(0, 0, 0));
  thrust::device_vector<float4> tq(U, make_float4(0, 0, 0, 0));
  mat2transquat_kernel<<<blocks_for(U), BLOCK_SIZE>>>(thrust::raw_pointer_cast(T.data()),
                                                      thrust::raw_pointer_cast(tt.data()),
                                                      thrust::raw_pointer_cast(tq.data()), (int)U);
  RH_CHECK(cudaGetLastError());
  thrust::device_vector<unsigned int> th(U, 0u), adj(27 * U, 0u);
  trans2idx_kernel<<<blocks_for(U), BLOCK_SIZE>>>(thrust::raw_pointer_cast(tt.data()),
                                                  thrust::raw_pointer_cast(th.data()),
                                                  thrust::raw_pointer_cast(adj.data()), (int)U, d_dist);
  RH_CHECK(cudaGetLastError());
  RH_CHECK(cudaDeviceSynchronize());
  Pha P;
  P.build(th);
  thrust::device_vector<size_t> tidx;
  P.indices(adj, tidx);
  thrust::device_vector<float> vco(U, 0.f);
  rot_clustering_kernel<<<blocks_for(U), BLOCK_SIZE>>>(
      thrust::raw_pointer_cast(tt.data()), thrust::raw_pointer_cast(tq.data()),
      thrust::raw_pointer_cast(wvc.data()), thrust::raw_pointer_cast(adj.data()),
      thrust::raw_pointer_cast(tidx.data()), thrust::raw_pointer_cast(P.hashkeys.data()),
      thrust::raw_pointer_cast(P.counts.data()), thrust::raw_pointer_cast(P.first.data()),
      thrust::raw_pointer_cast(P.map.data()), thrust::raw_pointer_cast(vco.data()), (int)U, d_dist,
      use_l1 != 0, use_avg != 0);
  RH_CHECK(cudaGetLastError());
  size_t max_idx = thrust::max_element(vco.begin(), vco.end()) - vco.begin();
  RH_CHECK(cudaDeviceSynchronize());
  res->max_idx = max_idx;
  thrust::host_vector<float> hT(T.begin() + 16 * max_idx, T.begin() + 16 * max_idx + 16);
  float3 ht = tt[max_idx];
  for (int k = 0; k < 16; ++k) res->pose[k] = hT[k];
  res->pose[3] = ht.x;
  res->pose[7] = ht.y;
  res->pose[11] = ht.z;
  if ((long long)U <= cap) {
    if (transforms) thrust::copy(T.begin(), T.end(), transforms);
    if (trans) {
      thrust::host_vector<float3> h = tt;
      for (size_t i = 0; i < U; ++i) {
        trans[3 * i] = h[i].x;
        trans[3 * i + 1] = h[i].y;
        trans[3 * i + 2] = h[i].z;
      }
    }
    if (quats) {
      thrust::host_vector<float4> h = tq;
      for (size_t i = 0; i < U; ++i) {
        quats[4 * i] = h[i].x;
        quats[4 * i + 1] = h[i].y;
        quats[4 * i + 2] = h[i].z;
        quats[4 * i + 3] = h[i].w;
      }
    }
    if (scores) thrust::copy(vco.begin(), vco.end(), scores);
  }
  return 0;
}

}  // namespace

extern "C" {

// Model::Model + Scene::Scene + Model::ppf_lookup with GPU clustering, then the
// pose assembly of ppf_registration (ppf.cu:67-93).  Output arrays are
// optional (NULL skips); capacities in elements.  all_codes/all_counts receive
// the unique votes before the threshold in code order; codes/counts the kept
// votes in the reference's order; transforms U*16, trans U*3, quats U*4,
// scores U; pair_counts n_s*n_s per-scene-pair vote counts.
int rh_lookup(const float* m_pts, const float* m_nrm, int n_m, const float* s_pts,
              const float* s_nrm, int n_s, float d_dist, unsigned ref_df, float thr, int use_l1,
              int use_avg, const float* weights, rh_result* res, unsigned long long* all_codes,
              uint32_t* all_counts, long long all_cap, unsigned long long* codes, uint32_t* counts,
              float* transforms, float* trans, float* quats, float* scores, long long cap,
              unsigned long long* pair_counts) {
  memset(res, 0, sizeof(*res));
  if (n_m > 46340 || n_s > 46340) return -2;
  Cloud M, S;
  M.load(m_pts, m_nrm, n_m);
  S.load(s_pts, s_nrm, n_s);
  thrust::device_vector<unsigned int> mkeys, skeys;
  if (cloud_keys(M, d_dist, 1, mkeys)) return -1;
  Pha H;
  H.build(mkeys);
  thrust::device_vector<float> wts(n_m, 1.0f);
  if (weights) thrust::copy(weights, weights + n_m, wts.begin());
  if (cloud_keys(S, d_dist, ref_df, skeys)) return -1;
  RH_CHECK(cudaDeviceSynchronize());

  Timer timer;
  thrust::device_vector<unsigned long> votes;
  thrust::device_vector<unsigned int> vote_counts;
  if (unique_votes(M, S, H, skeys, d_dist, votes, vote_counts, &res->n_votes, pair_counts)) return -1;
  res->n_unique = votes.size();
  if (all_codes && (long long)votes.size() <= all_cap) {
    thrust::copy(votes.begin(), votes.end(), all_codes);
    thrust::copy(vote_counts.begin(), vote_counts.end(), all_counts);
  }
  if (votes.empty()) {
    res->elapsed_ms = timer.stop();
    return 1;
  }
  // threshold and order (model.cu:155-170)
  thrust::sort_by_key(vote_counts.begin(), vote_counts.end(), votes.begin(), thrust::greater<float>());
  unsigned int top = vote_counts[0];
  float min_votecount = thr * top;
  size_t U = thrust::count_if(vote_counts.begin(), vote_counts.end(),
                              [min_votecount] __device__(unsigned int x) { return x > min_votecount; });
  res->max_count = top;
  res->min_votecount = min_votecount;
  res->n_kept = U;
  votes.resize(U);
  vote_counts.resize(U);
  if (post_votes(M, S, wts, votes, vote_counts, d_dist, use_l1, use_avg, res, transforms, trans, quats, scores,
                 cap))
    return -1;
  res->elapsed_ms = timer.stop();
  if (codes && (long long)U <= cap) {
    thrust::copy(votes.begin(), votes.end(), codes);
    thrust::copy(vote_counts.begin(), vote_counts.end(), counts);
  }
  return 0;
}

// The unique votes of one scene against one model (model.cu:95-151): every
// nonzero (s_r, m_r, alpha) cell in code order with its count.  *n_unique is
// set even when cap is too small (nothing is copied then); res->elapsed_ms
// is the device time of the vote count, vote, sort and histogram stages.
int rh_unique_votes(const float* m_pts, const float* m_nrm, int n_m, const float* s_pts, const float* s_nrm,
                    int n_s, float d_dist, unsigned ref_df, rh_result* res, unsigned long long* codes,
                    uint32_t* counts, long long cap) {
  memset(res, 0, sizeof(*res));
  if (n_m > 46340 || n_s > 46340) return -2;
  Cloud M, S;
  M.load(m_pts, m_nrm, n_m);
  S.load(s_pts, s_nrm, n_s);
  thrust::device_vector<unsigned int> mkeys, skeys;
  if (cloud_keys(M, d_dist, 1, mkeys)) return -1;
  Pha H;
  H.build(mkeys);
  if (cloud_keys(S, d_dist, ref_df, skeys)) return -1;
  RH_CHECK(cudaDeviceSynchronize());
  Timer timer;
  thrust::device_vector<unsigned long> votes;
  thrust::device_vector<unsigned int> vote_counts;
  if (unique_votes(M, S, H, skeys, d_dist, votes, vote_counts, &res->n_votes, nullptr)) return -1;
  res->elapsed_ms = timer.stop();
  res->n_unique = votes.size();
  if (codes && (long long)votes.size() <= cap) {
    thrust::copy(votes.begin(), votes.end(), codes);
    thrust::copy(vote_counts.begin(), vote_counts.end(), counts);
  }
  return 0;
}

// The stages of Model::ppf_lookup after the threshold (model.cu:173-244,
// 293-295) and the pose assembly of ppf_registration (ppf.cu:78-93), on U
// kept votes given in the reference's order (count descending, code
// ascending).  res->elapsed_ms is their device time.
int rh_post(const float* m_pts, const float* m_nrm, int n_m, const float* s_pts, const float* s_nrm, int n_s,
            float d_dist, int use_l1, int use_avg, const float* weights, const unsigned long long* codes,
            const uint32_t* counts, long long U, rh_result* res, float* transforms, float* trans, float* quats,
            float* scores) {
  memset(res, 0, sizeof(*res));
  if (n_m > 46340 || U < 1) return -2;
  Cloud M, S;
  M.load(m_pts, m_nrm, n_m);
  S.load(s_pts, s_nrm, n_s);
  thrust::device_vector<float> wts(n_m, 1.0f);
  if (weights) thrust::copy(weights, weights + n_m, wts.begin());
  thrust::host_vector<unsigned long> hv(U);
  thrust::host_vector<unsigned int> hc(U);
  for (long long i = 0; i < U; ++i) {
    hv[i] = (unsigned long)codes[i];
    hc[i] = counts[i];
  }
  thrust::device_vector<unsigned long> votes = hv;
  thrust::device_vector<unsigned int> vote_counts = hc;
  RH_CHECK(cudaDeviceSynchronize());
  res->n_kept = (unsigned long long)U;
  Timer timer;
  if (post_votes(M, S, wts, votes, vote_counts, d_dist, use_l1, use_avg, res, transforms, trans, quats, scores,
                 U))
    return -1;
  res->elapsed_ms = timer.stop();
  return 0;
}

}  // extern "C"
