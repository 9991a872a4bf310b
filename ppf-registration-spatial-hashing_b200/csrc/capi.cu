// Host orchestration and the C ABI (include/ppf_b200.h).  Every entry point
// catches engine errors and returns a status; the message is kept per thread.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "engine.h"

namespace ppf {

Context::~Context() {
  // device blocks go back to the pool on this stream, so free them first
  flags.release();
  counters.release();
  scratch.release();
  cand_codes.release();
  cand_counts.release();
  batch_args.release();
  batch_off.release();
  batch_counters.release();
  batch_redo.release();
  redo_items.release();
  tune_counters.release();
  sort32.release();
  sort64.release();
  if (stream) cudaStreamSynchronize(stream);
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
}

namespace {

thread_local std::string g_last_error;

ppf_status fail(ppf_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

template <typename F>
ppf_status guarded(F&& f) {
  try {
    g_last_error.clear();
    return f();
  } catch (const Error& e) {
    return fail(e.status, e.what());
  } catch (const std::bad_alloc&) {
    return fail(PPF_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(PPF_ERR_INTERNAL, e.what());
  }
}

// Reference counts of the handles (see engine.h): releasing the last
// reference waits for the object's stream and frees it.
void release_context(ppf_context_s* c) {
  if (c && c->refs.fetch_sub(1) == 1) {
    cudaSetDevice(c->c.device);
    cudaStreamSynchronize(c->c.stream);
    delete c;
  }
}

void release_model(ppf_model_s* m) {
  if (m && m->refs.fetch_sub(1) == 1) {
    ppf_context_s* owner = m->owner;
    {
      cudaSetDevice(m->m.ctx->device);
      StreamScope scope(m->m.ctx->stream);
      cudaStreamSynchronize(m->m.ctx->stream);
      delete m;
    }
    release_context(owner);
  }
}

void copy_out(void* dst, const void* src_dev, size_t bytes, cudaStream_t st) {
  if (!dst || !bytes) return;
  PPF_CUDA(cudaMemcpyAsync(dst, src_dev, bytes, cudaMemcpyDefault, st));
}

}  // namespace

uint64_t model_signature(const Model& m) {
  uint32_t d, t;
  std::memcpy(&d, &m.t.d_dist, 4);
  std::memcpy(&t, &m.vote_count_threshold, 4);
  return ((uint64_t)m.t.n * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)d << 21) ^ ((uint64_t)t * 0xC2B2AE3Dull);
}

// The part of Model::ppf_lookup after the vote pass (threshold, order,
// poses, clustering) and the pose extraction of ppf_registration, on the
// candidate cells of one vote pass.  ev[2] marks the lookup's start.
LookupOut finish_lookup(Context& ctx, Model& m, LookupState& st, const SceneData& s, const VoteResult& vr,
                        const unsigned long long* cand_code, const uint32_t* cand_count,
                        size_t launches0, bool own_state) {
  LookupOut out;
  // After an overflow the recounted items emit against a higher running
  // maximum, so the cells the first launch asked for are the better size.
  const size_t hint = std::max<size_t>(vr.n_cand, vr.n_needed);
  if (own_state) m.cand_hint = hint;
  ctx.cand_hints[model_signature(m)] = hint;
  out.cand_hint = hint;
  st.U = 0;
  out.stats.n_votes = vr.n_votes;
  out.stats.n_matched_pairs = vr.n_matched;
  out.stats.n_exact_bins = vr.n_exact;
  out.stats.max_vote_count = vr.max_count;
  out.stats.vote_ms = vr.vote_ms;
  const uint32_t shift = m.seg_shift.load(std::memory_order_relaxed);
  out.stats.vote_segment = 1u << (shift ? shift : kSegShiftDefault);
  out.stats.n_redo_items = vr.n_redo;
  if (vr.max_count == 0) {
    out.status = PPF_ERR_NO_VOTES;
    return out;
  }
  const float min_votecount = m.vote_count_threshold * (float)vr.max_count;
  out.stats.min_votecount = min_votecount;
  out.stats.n_candidates = vr.n_cand;
  const size_t U = select_votes(ctx, m, s, st, cand_code, cand_count, vr.n_cand, min_votecount, vr.max_count);
  out.stats.n_kept = U;
  if (U == 0) {
    out.status = PPF_ERR_NO_VOTES;
    return out;
  }
  compute_poses(ctx, m, s, st);
  if (m.cpu_clustering) {
    float poses[48];
    uint32_t votes[3];
    const int nc = cluster_poses_greedy_gpu(ctx, st.transforms.as<float>(), st.counts.as<uint32_t>(), U,
                                            m.t.d_dist, PPF_D_ANGLE_HOST, poses, votes);
    st.cpu_poses.assign(poses, poses + 16 * nc);
    if (nc > 0) std::memcpy(out.pose, poses, sizeof(out.pose));
    out.stats.max_idx = 0;
    out.stats.best_score = nc > 0 ? (float)votes[0] : 0.f;
    out.stats.cluster_path = 4;
  } else {
    float best_score = 0;
    size_t idx = cluster_poses_gpu(ctx, m, st, &best_score);
    PPF_CUDA(cudaMemcpyAsync(out.pose, st.best.ptr, sizeof(out.pose), cudaMemcpyDeviceToHost, ctx.stream));
    out.stats.max_idx = idx;
    out.stats.best_score = best_score;
    out.stats.cluster_path = st.cluster_path;
  }
  PPF_CUDA(cudaEventRecord(ctx.ev[3], ctx.stream));
  PPF_CUDA(cudaStreamSynchronize(ctx.stream));
  uint32_t flags = 0;
  PPF_CUDA(cudaMemcpyAsync(&flags, ctx.flags.ptr, 4, cudaMemcpyDeviceToHost, ctx.stream));
  PPF_CUDA(cudaStreamSynchronize(ctx.stream));
  PPF_REQUIRE(!(flags & kFlagSpinTimeout), PPF_ERR_TIMEOUT, "radix sort look-back timed out");
  PPF_CUDA(cudaEventElapsedTime(&out.stats.total_ms, ctx.ev[2], ctx.ev[3]));
  out.stats.gpu_launches = (uint32_t)(ctx.launches - launches0);
  return out;
}

// Model::ppf_lookup + the pose extraction of ppf_registration.
LookupOut lookup(Model& m, const SceneData& s) {
  Context& ctx = *m.ctx;
  const size_t launches0 = ctx.launches;
  tune_vote_segments(ctx, m, s, model_signature(m));
  PPF_CUDA(cudaEventRecord(ctx.ev[2], ctx.stream));
  VoteResult vr = run_votes(ctx, m, s, false, -1.f);
  return finish_lookup(ctx, m, m.last, s, vr, ctx.cand_codes.as<unsigned long long>(),
                       ctx.cand_counts.as<uint32_t>(), launches0, true);
}

// Several lookups with one batched vote pass: request i is (models[i],
// scenes[i]).  Candidate buffers are sized from each model's last pass,
// within a budget shared by the batch.
std::vector<LookupOut> lookup_batch(Context& ctx, const std::vector<Model*>& models,
                                    const std::vector<const SceneData*>& scenes, LookupState* states,
                                    const size_t* caps) {
  const size_t n = models.size();
  const size_t launches0 = ctx.launches;
  for (size_t i = 0; i < n; ++i) tune_vote_segments(ctx, *models[i], *scenes[i], model_signature(*models[i]));
  PPF_CUDA(cudaEventRecord(ctx.ev[2], ctx.stream));
  std::vector<BatchVote> reqs(n);
  constexpr size_t kBudgetCells = size_t(1) << 28;  // 3 GB of candidate cells over the batch
  size_t want = 0;
  for (size_t i = 0; i < n; ++i) {
    reqs[i].m = models[i];
    reqs[i].s = scenes[i];
    size_t hint = caps ? caps[i] : models[i]->cand_hint;
    if (!hint) {
      auto it = ctx.cand_hints.find(model_signature(*models[i]));
      if (it != ctx.cand_hints.end()) hint = it->second;
    }
    reqs[i].cap = hint ? hint + hint / 4 + 65536 : (size_t(1) << 22);
    want += reqs[i].cap;
  }
  if (want > kBudgetCells)
    for (auto& r : reqs) r.cap = std::max<size_t>(r.cap * (double)kBudgetCells / (double)want, 65536);
  // test hook: a small capacity exercises the per-request growth path
  if (const char* e = std::getenv("PPF_B200_BATCH_CAP")) {
    const long long v = std::atoll(e);
    if (v > 0)
      for (auto& r : reqs) r.cap = (size_t)v;
  }
  run_votes_batch(ctx, reqs);
  std::vector<LookupOut> out(n);
  for (size_t i = 0; i < n; ++i) {
    Model& m = *models[i];
    out[i] = finish_lookup(ctx, m, states ? states[i] : m.last, *scenes[i], reqs[i].r,
                           reqs[i].codes.as<unsigned long long>(), reqs[i].counts.as<uint32_t>(),
                           i == 0 ? launches0 : ctx.launches, states == nullptr);
    PPF_CUDA(cudaEventRecord(ctx.ev[2], ctx.stream));
  }
  return out;
}

void check_cloud(const float* xyz, const float* nxyz, uint64_t n) {
  PPF_REQUIRE(xyz && nxyz, PPF_ERR_INVALID_ARGUMENT, "null point or normal pointer");
  PPF_REQUIRE(n >= 1, PPF_ERR_INVALID_ARGUMENT, "empty cloud");
}

void init_context(Context& c, int device) {
  int count = 0;
  PPF_CUDA(cudaGetDeviceCount(&count));
  PPF_REQUIRE(count > 0, PPF_ERR_CUDA, "no CUDA device");
  c.device = std::max(0, std::min(count - 1, device));
  PPF_CUDA(cudaSetDevice(c.device));
  PPF_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  for (auto& e : c.ev) PPF_CUDA(cudaEventCreate(&e));
  // keep freed blocks in the device's stream-ordered pool for reuse
  cudaMemPool_t pool;
  PPF_CUDA(cudaDeviceGetDefaultMemPool(&pool, c.device));
  uint64_t keep = UINT64_MAX;
  PPF_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  StreamScope scope(c.stream);
  c.flags.reserve(256);
  c.counters.reserve(256);
  PPF_CUDA(cudaMemsetAsync(c.flags.ptr, 0, 256, c.stream));
  PPF_CUDA(cudaStreamSynchronize(c.stream));
  int optin = 0;
  PPF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
  c.vote_smem_limit = optin - 2048;  // static shared memory of the vote kernel
  if (const char* e = std::getenv("PPF_B200_CHECKS")) c.checks = e[0] == '1';
  if (const char* e = std::getenv("PPF_B200_CLUSTER_SPLIT")) c.cluster_split = e[0] != '0';
  if (const char* e = std::getenv("PPF_B200_CLUSTER_SQRT")) c.cluster_sqrt = e[0] == '1';
  if (const char* e = std::getenv("PPF_B200_TUNE")) c.tune = e[0] != '0';
  if (const char* e = std::getenv("PPF_B200_VOTE_SEGMENT")) {
    // a power of two from 256 to 65536 entries
    const long long v = std::atoll(e);
    for (uint32_t k = 8; k <= 16; ++k)
      if (v == (1ll << k)) c.forced_seg_shift = k;
  }
  // test hooks: the n-th device allocation from now fails; the next 32-bit
  // radix sort on this context has one tile withhold its look-back status,
  // so that the tiles waiting on it give up after a short bounded spin
  if (const char* e = std::getenv("PPF_B200_TEST_FAIL_ALLOC")) alloc_failure_countdown() = std::atoll(e);
  if (const char* e = std::getenv("PPF_B200_TEST_SORT_STALL"))
    if (e[0] == '1') c.sort32.arm_stall();
  // test hook: a small initial candidate buffer exercises its growth path
  if (const char* e = std::getenv("PPF_B200_CANDIDATE_CAP")) {
    long long v = std::atoll(e);
    if (v > 0) c.cand_cap = (size_t)v;
  }
}

}  // namespace ppf

using namespace ppf;

extern "C" {

const char* ppf_last_error(void) { return g_last_error.c_str(); }
int ppf_abi_version(void) { return PPF_B200_ABI_VERSION; }

ppf_status ppf_context_create(int device, ppf_context_t* out) {
  return guarded([&]() {
    PPF_REQUIRE(out, PPF_ERR_INVALID_ARGUMENT, "null output handle");
    std::unique_ptr<ppf_context_s> c(new ppf_context_s());
    init_context(c->c, device);
    *out = c.release();
    return PPF_OK;
  });
}

ppf_status ppf_context_destroy(ppf_context_t ctx) {
  return guarded([&]() {
    release_context(ctx);
    return PPF_OK;
  });
}

ppf_status ppf_context_synchronize(ppf_context_t ctx) {
  return guarded([&]() {
    PPF_REQUIRE(ctx, PPF_ERR_INVALID_ARGUMENT, "null context");
    PPF_CUDA(cudaStreamSynchronize(ctx->c.stream));
    return PPF_OK;
  });
}

void* ppf_context_stream(ppf_context_t ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }
uint64_t ppf_context_kernel_launches(ppf_context_t ctx) { return ctx ? ctx->c.launches : 0; }
int ppf_context_device(ppf_context_t ctx) { return ctx ? ctx->c.device : -1; }

ppf_status ppf_model_create(ppf_context_t ctx, const float* xyz, const float* nxyz, uint64_t n,
                            float d_dist, float vote_count_threshold, int cpu_clustering,
                            int use_l1_norm, int use_averaged_clusters, ppf_model_t* out) {
  return guarded([&]() {
    PPF_REQUIRE(ctx && out, PPF_ERR_INVALID_ARGUMENT, "null context or output handle");
    check_cloud(xyz, nxyz, n);
    PPF_REQUIRE(std::isfinite(vote_count_threshold) && vote_count_threshold >= 0.f,
                PPF_ERR_INVALID_ARGUMENT, "vote_count_threshold must be finite and >= 0");
    PPF_CUDA(cudaSetDevice(ctx->c.device));
    StreamScope scope(ctx->c.stream);
    std::unique_ptr<ppf_model_s> m(new ppf_model_s());
    m->m.ctx = &ctx->c;
    m->m.vote_count_threshold = vote_count_threshold;
    m->m.cpu_clustering = cpu_clustering != 0;
    m->m.use_l1_norm = use_l1_norm != 0;
    m->m.use_averaged_clusters = use_averaged_clusters != 0;
    build_model(ctx->c, m->m.t, xyz, nxyz, n, d_dist);
    m->owner = ctx;
    ctx->refs.fetch_add(1);
    *out = m.release();
    return PPF_OK;
  });
}

ppf_status ppf_model_set_point_vote_weights(ppf_model_t m, const float* w, uint64_t n) {
  return guarded([&]() {
    PPF_REQUIRE(m && w, PPF_ERR_INVALID_ARGUMENT, "null model or weights");
    PPF_REQUIRE(n == m->m.t.n, PPF_ERR_INVALID_ARGUMENT, "one weight per model point required");
    PPF_CUDA(cudaSetDevice(m->m.ctx->device));
    StreamScope scope(m->m.ctx->stream);
    PPF_CUDA(cudaMemcpyAsync(m->m.t.weights.ptr, w, n * sizeof(float), cudaMemcpyDefault,
                             m->m.ctx->stream));
    PPF_CUDA(cudaStreamSynchronize(m->m.ctx->stream));
    return PPF_OK;
  });
}

ppf_status ppf_model_destroy(ppf_model_t m) {
  return guarded([&]() {
    release_model(m);
    return PPF_OK;
  });
}

uint64_t ppf_model_num_points(ppf_model_t m) { return m ? m->m.t.n : 0; }
uint64_t ppf_model_num_keys(ppf_model_t m) { return m ? m->m.t.K : 0; }
uint64_t ppf_model_num_chunks(ppf_model_t m) { return m ? m->m.t.n_chunks : 0; }

ppf_status ppf_scene_create(ppf_context_t ctx, const float* xyz, const float* nxyz, uint64_t n,
                            float d_dist, uint32_t ref_point_df, ppf_scene_t* out) {
  return guarded([&]() {
    PPF_REQUIRE(ctx && out, PPF_ERR_INVALID_ARGUMENT, "null context or output handle");
    check_cloud(xyz, nxyz, n);
    PPF_REQUIRE(n < (1ull << 31), PPF_ERR_INVALID_ARGUMENT, "scene larger than 2^31 points");
    PPF_REQUIRE(d_dist > 0.f && std::isfinite(d_dist), PPF_ERR_INVALID_ARGUMENT,
                "d_dist must be a positive finite number");
    PPF_CUDA(cudaSetDevice(ctx->c.device));
    StreamScope scope(ctx->c.stream);
    std::unique_ptr<ppf_scene_s> s(new ppf_scene_s());
    s->ctx = &ctx->c;
    s->s.n = (uint32_t)n;
    s->s.d_dist = d_dist;
    s->s.ref_df = ref_point_df ? ref_point_df : 1;
    upload_points(ctx->c, xyz, n, s->s.pts);
    upload_points(ctx->c, nxyz, n, s->s.nrm);
    s->owner = ctx;
    ctx->refs.fetch_add(1);
    *out = s.release();
    return PPF_OK;
  });
}

ppf_status ppf_scene_destroy(ppf_scene_t s) {
  return guarded([&]() {
    if (s) {
      ppf_context_s* owner = s->owner;
      {
        cudaSetDevice(s->ctx->device);
        StreamScope scope(s->ctx->stream);
        cudaStreamSynchronize(s->ctx->stream);
        delete s;
      }
      release_context(owner);
    }
    return PPF_OK;
  });
}

ppf_status ppf_model_lookup(ppf_model_t m, ppf_scene_t s, float* pose_out, ppf_stats* stats) {
  return guarded([&]() {
    PPF_REQUIRE(m && s && pose_out, PPF_ERR_INVALID_ARGUMENT, "null model, scene or pose");
    PPF_REQUIRE(m->m.ctx == s->ctx, PPF_ERR_INVALID_ARGUMENT, "model and scene on different contexts");
    PPF_CUDA(cudaSetDevice(m->m.ctx->device));
    StreamScope scope(m->m.ctx->stream);
    LookupOut r = lookup(m->m, s->s);
    PPF_CUDA(cudaMemcpy(pose_out, r.pose, sizeof(r.pose), cudaMemcpyDefault));
    if (stats) *stats = r.stats;
    if (r.status != PPF_OK) return fail(r.status, "no vote passed the threshold");
    return PPF_OK;
  });
}

ppf_status ppf_lookup_batch(ppf_context_t ctx, uint64_t n, const ppf_model_t* models,
                            const ppf_scene_t* scenes, float* poses_out, ppf_stats* stats_out) {
  return guarded([&]() {
    PPF_REQUIRE(ctx, PPF_ERR_INVALID_ARGUMENT, "null context");
    if (n == 0) return PPF_OK;
    PPF_REQUIRE(models && scenes && poses_out, PPF_ERR_INVALID_ARGUMENT, "null models, scenes or poses");
    std::vector<Model*> ms(n);
    std::vector<const SceneData*> ss(n);
    for (uint64_t i = 0; i < n; ++i) {
      PPF_REQUIRE(models[i] && scenes[i], PPF_ERR_INVALID_ARGUMENT, "null model or scene in the batch");
      PPF_REQUIRE(models[i]->m.ctx == &ctx->c && scenes[i]->ctx == &ctx->c, PPF_ERR_INVALID_ARGUMENT,
                  "batch model or scene on another context");
      ms[i] = &models[i]->m;
      ss[i] = &scenes[i]->s;
    }
    PPF_CUDA(cudaSetDevice(ctx->c.device));
    StreamScope scope(ctx->c.stream);
    std::vector<LookupOut> r = lookup_batch(ctx->c, ms, ss, nullptr, nullptr);
    std::vector<float> poses(n * 16);
    ppf_status worst = PPF_OK;
    for (uint64_t i = 0; i < n; ++i) {
      std::memcpy(&poses[16 * i], r[i].pose, sizeof(r[i].pose));
      if (stats_out) stats_out[i] = r[i].stats;
      if (r[i].status != PPF_OK) worst = r[i].status;
    }
    PPF_CUDA(cudaMemcpy(poses_out, poses.data(), poses.size() * sizeof(float), cudaMemcpyDefault));
    if (worst != PPF_OK) return fail(worst, "no vote passed the threshold for at least one request");
    return PPF_OK;
  });
}

namespace {
// n x 3 floats on the device: the caller's pointer, or a copy of host memory
const float* device_xyz(Context& c, const float* p, size_t n, DevBuf& tmp) {
  if (is_device_pointer(p, c.device)) return p;
  tmp.reserve(std::max<size_t>(n, 1) * 12);
  if (n) PPF_CUDA(cudaMemcpyAsync(tmp.ptr, p, n * 12, cudaMemcpyHostToDevice, c.stream));
  return tmp.as<float>();
}
}  // namespace

ppf_status ppf_cloud_extent(ppf_context_t ctx, const float* xyz, uint64_t n, float* min_out, float* max_out) {
  return guarded([&]() {
    PPF_REQUIRE(ctx && xyz && min_out && max_out, PPF_ERR_INVALID_ARGUMENT, "null argument");
    PPF_CUDA(cudaSetDevice(ctx->c.device));
    StreamScope scope(ctx->c.stream);
    DevBuf tmp;
    const float* d = device_xyz(ctx->c, xyz, n, tmp);
    float lo[3], hi[3];
    PPF_REQUIRE(cloud_extent(ctx->c, d, n, lo, hi), PPF_ERR_INVALID_ARGUMENT, "no finite point");
    std::memcpy(min_out, lo, sizeof(lo));
    std::memcpy(max_out, hi, sizeof(hi));
    return PPF_OK;
  });
}

ppf_status ppf_voxel_downsample(ppf_context_t ctx, const float* xyz, const float* nxyz, uint64_t n, float leaf,
                                float* out_xyz, float* out_nxyz, uint64_t cap, uint64_t* n_out) {
  return guarded([&]() {
    PPF_REQUIRE(ctx && xyz && nxyz && n_out, PPF_ERR_INVALID_ARGUMENT, "null argument");
    PPF_CUDA(cudaSetDevice(ctx->c.device));
    StreamScope scope(ctx->c.stream);
    DevBuf ta, tb, ox, on;
    const float* dx = device_xyz(ctx->c, xyz, n, ta);
    const float* dn = device_xyz(ctx->c, nxyz, n, tb);
    const size_t K = voxel_downsample(ctx->c, dx, dn, n, leaf, ox, on);
    *n_out = K;
    PPF_REQUIRE(K <= cap, PPF_ERR_INVALID_ARGUMENT,
                "output capacity " + std::to_string(cap) + " below the " + std::to_string(K) + " voxels");
    PPF_REQUIRE(!K || (out_xyz && out_nxyz), PPF_ERR_INVALID_ARGUMENT, "null output");
    copy_out(out_xyz, ox.ptr, K * 12, ctx->c.stream);
    copy_out(out_nxyz, on.ptr, K * 12, ctx->c.stream);
    PPF_CUDA(cudaStreamSynchronize(ctx->c.stream));
    return PPF_OK;
  });
}

ppf_status ppf_cluster_poses(ppf_context_t ctx, const float* transforms, const uint32_t* votes, uint64_t n,
                             float trans_thresh, float rot_thresh, float* out_poses, uint32_t* out_votes,
                             uint32_t* n_clusters) {
  return guarded([&]() {
    PPF_REQUIRE(ctx && out_poses && out_votes && n_clusters && (n == 0 || (transforms && votes)),
                PPF_ERR_INVALID_ARGUMENT, "null argument");
    PPF_CUDA(cudaSetDevice(ctx->c.device));
    StreamScope scope(ctx->c.stream);
    DevBuf tT, tV;
    const float* T = transforms;
    const uint32_t* V = votes;
    if (n && !is_device_pointer(transforms, ctx->c.device)) {
      tT.reserve(n * 64);
      PPF_CUDA(cudaMemcpyAsync(tT.ptr, transforms, n * 64, cudaMemcpyHostToDevice, ctx->c.stream));
      T = tT.as<float>();
    }
    if (n && !is_device_pointer(votes, ctx->c.device)) {
      tV.reserve(n * 4);
      PPF_CUDA(cudaMemcpyAsync(tV.ptr, votes, n * 4, cudaMemcpyHostToDevice, ctx->c.stream));
      V = tV.as<uint32_t>();
    }
    float p[48];
    uint32_t v[3];
    const int nc = cluster_poses_sorted_gpu(ctx->c, T, V, n, trans_thresh, rot_thresh, p, v);
    std::memcpy(out_poses, p, sizeof(float) * 16 * nc);
    std::memcpy(out_votes, v, sizeof(uint32_t) * nc);
    *n_clusters = (uint32_t)nc;
    return PPF_OK;
  });
}

ppf_status ppf_ply_read(const char* path, float* xyz, float* nxyz, uint64_t cap, uint64_t* n_out) {
  return guarded([&]() {
    std::string err;
    const ppf_status st = ply_read(path, xyz, nxyz, cap, n_out, &err);
    if (st != PPF_OK) return fail(st, err);
    return PPF_OK;
  });
}

ppf_status ppf_ply_write(const char* path, const float* xyz, const float* nxyz, uint64_t n) {
  return guarded([&]() {
    const ppf_status st = ply_write(path, xyz, nxyz, n);
    if (st != PPF_OK) return fail(st, std::string("cannot write ") + (path ? path : "(null)"));
    return PPF_OK;
  });
}

ppf_status ppf_server_create(int device, uint64_t n_models, const ppf_model_t* models,
                             uint64_t memory_budget, uint32_t n_workers, uint32_t max_batch,
                             ppf_server_t* out) {
  return guarded([&]() {
    PPF_REQUIRE(out && models && n_models, PPF_ERR_INVALID_ARGUMENT, "null output or empty library");
    std::vector<Model*> ms(n_models);
    for (uint64_t j = 0; j < n_models; ++j) {
      PPF_REQUIRE(models[j], PPF_ERR_INVALID_ARGUMENT, "null model in the library");
      ms[j] = &models[j]->m;
    }
    std::unique_ptr<ppf_server_s> s(new ppf_server_s());
    s->srv = server_create(device, ms, memory_budget, n_workers, max_batch);
    // the server holds each library model (and through it its context)
    for (uint64_t j = 0; j < n_models; ++j) {
      models[j]->refs.fetch_add(1);
      s->library.push_back(models[j]);
    }
    *out = s.release();
    return PPF_OK;
  });
}

ppf_status ppf_server_submit(ppf_server_t srv, const float* xyz, const float* nxyz, uint64_t n,
                             uint32_t ref_point_df, uint64_t n_targets, const uint32_t* model_ids,
                             uint64_t* ticket) {
  return guarded([&]() {
    PPF_REQUIRE(srv && srv->srv && ticket, PPF_ERR_INVALID_ARGUMENT, "null server or ticket");
    *ticket = server_submit(srv->srv, xyz, nxyz, n, ref_point_df, model_ids, n_targets);
    return PPF_OK;
  });
}

ppf_status ppf_server_wait(ppf_server_t srv, uint64_t ticket, float* poses_out, ppf_stats* stats_out,
                           double* latency_ms) {
  return guarded([&]() {
    PPF_REQUIRE(srv && srv->srv, PPF_ERR_INVALID_ARGUMENT, "null server");
    std::string err;
    const ppf_status st = server_wait(srv->srv, ticket, poses_out, stats_out, latency_ms, &err);
    if (st != PPF_OK)
      return fail(st, err.empty() ? "no vote passed the threshold for at least one target" : err);
    return PPF_OK;
  });
}

ppf_status ppf_server_destroy(ppf_server_t srv) {
  return guarded([&]() {
    if (srv) {
      if (srv->srv) server_destroy(srv->srv);
      for (ppf_model_s* m : srv->library) release_model(m);
      delete srv;
    }
    return PPF_OK;
  });
}

ppf_status ppf_registration(ppf_context_t ctx, uint64_t n_scenes, const float* const* scene_xyz,
                            const float* const* scene_nxyz, const uint64_t* scene_n,
                            uint64_t n_models, const float* const* model_xyz,
                            const float* const* model_nxyz, const uint64_t* model_n,
                            const float* model_d_dists, uint32_t ref_point_df,
                            float vote_count_threshold, int cpu_clustering, int use_l1_norm,
                            int use_averaged_clusters, int dev_use, const float* model_weights,
                            float* poses_out, ppf_stats* stats_out) {
  (void)model_weights;  // accepted and unused, as src/cuda/ppf.cu:35
  return guarded([&]() {
    PPF_REQUIRE(poses_out || (n_scenes * n_models == 0), PPF_ERR_INVALID_ARGUMENT, "null pose output");
    PPF_REQUIRE(n_models == 0 || (model_xyz && model_nxyz && model_n && model_d_dists),
                PPF_ERR_INVALID_ARGUMENT, "null model arrays");
    PPF_REQUIRE(n_scenes == 0 || (scene_xyz && scene_nxyz && scene_n), PPF_ERR_INVALID_ARGUMENT,
                "null scene arrays");
    std::unique_ptr<ppf_context_s, void (*)(ppf_context_s*)> own(nullptr, release_context);
    ppf_context_t c = ctx;
    if (!c) {
      std::unique_ptr<ppf_context_s> fresh(new ppf_context_s());
      init_context(fresh->c, dev_use);
      own.reset(fresh.release());
      c = own.get();
    }
    PPF_CUDA(cudaSetDevice(c->c.device));
    StreamScope scope(c->c.stream);
    std::vector<float> host_poses(n_scenes * n_models * 16, 0.f);
    ppf_status worst = PPF_OK;
    using ModelPtr = std::unique_ptr<ppf_model_s, ppf_status (*)(ppf_model_t)>;
    using ScenePtr = std::unique_ptr<ppf_scene_s, ppf_status (*)(ppf_scene_t)>;
    // The reference builds each model again for every scene; a model built
    // once gives the same results.  Models are built in groups whose tables
    // (about 17 bytes per ordered pair) fit a device budget, and all (scene,
    // model) pairs of a group share one batched vote pass.
    constexpr double kGroupBytes = 48e9;
    for (uint64_t j0 = 0; j0 < n_models;) {
      uint64_t j1 = j0;
      double bytes = 0;
      while (j1 < n_models && (j1 == j0 || bytes + 17.0 * model_n[j1] * model_n[j1] <= kGroupBytes))
        bytes += 17.0 * model_n[j1] * model_n[j1], ++j1;
      std::vector<ModelPtr> models;
      for (uint64_t j = j0; j < j1; ++j) {
        ppf_model_t m = nullptr;
        ppf_status st = ppf_model_create(c, model_xyz[j], model_nxyz[j], model_n[j], model_d_dists[j],
                                         vote_count_threshold, cpu_clustering, use_l1_norm,
                                         use_averaged_clusters, &m);
        if (st != PPF_OK) throw Error(st, g_last_error);
        models.emplace_back(m, ppf_model_destroy);
      }
      std::vector<ScenePtr> scenes;
      std::vector<Model*> ms;
      std::vector<const SceneData*> ss;
      std::vector<size_t> slot;
      for (uint64_t i = 0; i < n_scenes; ++i)
        for (uint64_t j = j0; j < j1; ++j) {
          ppf_scene_t s = nullptr;
          ppf_status st = ppf_scene_create(c, scene_xyz[i], scene_nxyz[i], scene_n[i], model_d_dists[j],
                                           ref_point_df, &s);
          if (st != PPF_OK) throw Error(st, g_last_error);
          scenes.emplace_back(s, ppf_scene_destroy);
          ms.push_back(&models[j - j0]->m);
          ss.push_back(&s->s);
          slot.push_back(i * n_models + j);
        }
      std::vector<LookupOut> r = lookup_batch(c->c, ms, ss, nullptr, nullptr);
      for (size_t k = 0; k < r.size(); ++k) {
        std::memcpy(&host_poses[slot[k] * 16], r[k].pose, sizeof(r[k].pose));
        if (stats_out) stats_out[slot[k]] = r[k].stats;
        if (r[k].status != PPF_OK) worst = r[k].status;
      }
      j0 = j1;
    }
    if (!host_poses.empty())
      PPF_CUDA(cudaMemcpy(poses_out, host_poses.data(), host_poses.size() * sizeof(float),
                          cudaMemcpyDefault));
    if (worst != PPF_OK) return fail(worst, "at least one (scene, model) pair had no votes");
    return PPF_OK;
  });
}

ppf_status ppf_model_get_votes(ppf_model_t m, uint64_t* codes, uint32_t* counts, uint64_t cap,
                               uint64_t* n) {
  return guarded([&]() {
    PPF_REQUIRE(m && n, PPF_ERR_INVALID_ARGUMENT, "null model or count");
    const size_t U = m->m.last.U;
    *n = U;
    if (U && cap >= U) {
      copy_out(codes, m->m.last.codes.ptr, U * 8, m->m.ctx->stream);
      copy_out(counts, m->m.last.counts.ptr, U * 4, m->m.ctx->stream);
      PPF_CUDA(cudaStreamSynchronize(m->m.ctx->stream));
    }
    return PPF_OK;
  });
}

ppf_status ppf_model_get_transformations(ppf_model_t m, float* T, uint64_t cap, uint64_t* n) {
  return guarded([&]() {
    PPF_REQUIRE(m && n, PPF_ERR_INVALID_ARGUMENT, "null model or count");
    const size_t U = m->m.last.U;
    *n = U;
    if (U && cap >= U) {
      copy_out(T, m->m.last.transforms.ptr, U * 64, m->m.ctx->stream);
      PPF_CUDA(cudaStreamSynchronize(m->m.ctx->stream));
    }
    return PPF_OK;
  });
}

ppf_status ppf_model_get_cluster_state(ppf_model_t m, float* trans, float* quats, float* scores,
                                       uint64_t cap, uint64_t* n) {
  return guarded([&]() {
    PPF_REQUIRE(m && n, PPF_ERR_INVALID_ARGUMENT, "null model or count");
    const size_t U = m->m.last.U;
    *n = U;
    if (U && cap >= U && !m->m.cpu_clustering) {
      copy_out(trans, m->m.last.trans.ptr, U * 12, m->m.ctx->stream);
      copy_out(quats, m->m.last.quats.ptr, U * 16, m->m.ctx->stream);
      copy_out(scores, m->m.last.scores.ptr, U * 4, m->m.ctx->stream);
      PPF_CUDA(cudaStreamSynchronize(m->m.ctx->stream));
    }
    return PPF_OK;
  });
}

ppf_status ppf_model_get_hash_array(ppf_model_t m, uint32_t* keys, uint32_t* counts,
                                    uint32_t* first, uint64_t cap_k, uint32_t* map, uint64_t cap_p,
                                    uint64_t* K, uint64_t* P) {
  return guarded([&]() {
    PPF_REQUIRE(m && K && P, PPF_ERR_INVALID_ARGUMENT, "null model or sizes");
    const ModelTables& t = m->m.t;
    *K = t.K;
    *P = t.P;
    cudaStream_t st = m->m.ctx->stream;
    if (cap_k >= t.K) {
      copy_out(keys, t.uniq.ptr, t.K * 4, st);
      copy_out(counts, t.count.ptr, t.K * 4, st);
      copy_out(first, t.first.ptr, t.K * 4, st);
    }
    if (cap_p >= t.P) copy_out(map, t.pairs.ptr, t.P * 4, st);
    PPF_CUDA(cudaStreamSynchronize(st));
    return PPF_OK;
  });
}

ppf_status ppf_pair_keys(ppf_context_t ctx, const float* xyz, const float* nxyz, uint64_t n,
                         float d_dist, uint32_t ref_point_df, uint32_t* keys) {
  return guarded([&]() {
    PPF_REQUIRE(ctx && keys, PPF_ERR_INVALID_ARGUMENT, "null context or keys");
    check_cloud(xyz, nxyz, n);
    PPF_REQUIRE(n <= 65535, PPF_ERR_INVALID_ARGUMENT, "pair keys limited to 65535 points");
    Context& c = ctx->c;
    PPF_CUDA(cudaSetDevice(c.device));
    StreamScope scope(c.stream);
    DevBuf p, q, k;
    upload_points(c, xyz, n, p);
    upload_points(c, nxyz, n, q);
    uint32_t* dst = keys;
    if (!is_device_pointer(keys, c.device)) {
      k.reserve(n * n * 4);
      dst = k.as<uint32_t>();
    }
    pair_keys_device(c, p.as<float4>(), q.as<float4>(), (uint32_t)n, ref_point_df, d_dist, dst);
    if (dst != keys) PPF_CUDA(cudaMemcpyAsync(keys, dst, n * n * 4, cudaMemcpyDeviceToHost, c.stream));
    PPF_CUDA(cudaStreamSynchronize(c.stream));
    return PPF_OK;
  });
}

ppf_status ppf_model_all_votes(ppf_model_t m, ppf_scene_t s, uint64_t* codes, uint32_t* counts,
                               uint64_t cap, uint64_t* n) {
  return guarded([&]() {
    PPF_REQUIRE(m && s && n, PPF_ERR_INVALID_ARGUMENT, "null model, scene or count");
    Context& c = *m->m.ctx;
    PPF_CUDA(cudaSetDevice(c.device));
    StreamScope scope(c.stream);
    LookupState& st = m->m.last;
    VoteResult vr = run_votes(c, m->m, s->s, true, -1.f);
    sort_by_code(c, st, vr.n_cand);
    st.U = 0;
    *n = vr.n_cand;
    if (cap >= vr.n_cand) {
      copy_out(codes, st.codes.ptr, vr.n_cand * 8, c.stream);
      copy_out(counts, st.counts.ptr, vr.n_cand * 4, c.stream);
    }
    PPF_CUDA(cudaStreamSynchronize(c.stream));
    return PPF_OK;
  });
}

ppf_status ppf_model_vote_cells_noalloc(ppf_model_t m, const float* scene_xyz,
                                        const float* scene_nxyz, uint64_t n_scene,
                                        uint32_t ref_point_df, float vote_floor, uint64_t* codes,
                                        uint32_t* counts, uint64_t capacity, uint64_t* n_out,
                                        uint32_t* max_count) {
  return guarded([&]() {
    PPF_REQUIRE(m && n_out, PPF_ERR_INVALID_ARGUMENT, "null model or count");
    Context& c = *m->m.ctx;
    PPF_CUDA(cudaSetDevice(c.device));
    vote_cells_noalloc(c, m->m, scene_xyz, scene_nxyz, n_scene, ref_point_df, vote_floor, codes,
                       counts, capacity, n_out, max_count);
    return PPF_OK;
  });
}

ppf_status ppf_model_pair_vote_counts(ppf_model_t m, ppf_scene_t s, uint64_t* counts) {
  return guarded([&]() {
    PPF_REQUIRE(m && s && counts, PPF_ERR_INVALID_ARGUMENT, "null model, scene or counts");
    Context& c = *m->m.ctx;
    PPF_CUDA(cudaSetDevice(c.device));
    StreamScope scope(c.stream);
    const size_t nn = (size_t)s->s.n * s->s.n;
    DevBuf tmp;
    uint64_t* dst = counts;
    if (!is_device_pointer(counts, c.device)) {
      tmp.reserve(nn * 8);
      dst = tmp.as<uint64_t>();
    }
    pair_vote_counts(c, m->m, s->s, dst);
    if (dst != counts) PPF_CUDA(cudaMemcpyAsync(counts, dst, nn * 8, cudaMemcpyDeviceToHost, c.stream));
    PPF_CUDA(cudaStreamSynchronize(c.stream));
    return PPF_OK;
  });
}

}  // extern "C"
