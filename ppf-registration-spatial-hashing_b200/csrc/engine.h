// Engine objects behind the C ABI: context, resident model hash arrays,
// resident scenes, and the device-side layout the kernels consume.
#pragma once

#include <atomic>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "sort_scan.cuh"

struct ppf_context_s;

namespace ppf {

// Angle bins per model reference point in the vote accumulator (alpha bins
// 0..30; bin 30 is only reached at alpha == pi exactly).
constexpr int kBins = 31;
#define PPF_N_ANGLE_CELLS 31
// Vote kernel launch shape: one 1024-thread block per SM.
constexpr int kVoteThreads = 1024;
constexpr int kVoteWarps = kVoteThreads / 32;
// Shared memory of the vote block besides its accumulator: per scene pair of
// a tile its sub-run start and length, angle word, frame vector (y, z) and
// segment offset (+1 entry).
constexpr int kVoteQueueBytes = kVoteThreads * (4 + 4 + 4 + 8) + (kVoteThreads + 4) * 4;
// Accumulator words of a chunk: one 32-bit counter per (m_r, alpha bin) cell
// (the reference counts votes in unsigned int too, include/impl/util.hpp:30-52).
inline size_t vote_acc_words(uint32_t chunk) { return ((size_t)chunk * kBins + 3) & ~size_t(3); }
// Angle quantum on the host (include/kernel.h:16 evaluated in float).
#define PPF_D_ANGLE_HOST ((2.0f * 3.141592654f) / float(30))

// Every DevBuf member must be released in ~Context (capi.cu) before the
// stream its blocks are freed on is destroyed.
struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  RadixSorter<uint32_t> sort32;
  RadixSorter<unsigned long long> sort64;
  DevBuf flags;      // uint32 device flags (kFlag*)
  DevBuf counters;   // small device counters for kernels
  DevBuf scratch;    // run-table scratch
  // vote-pass candidate cells (code, count), kept and grown across lookups
  DevBuf cand_codes, cand_counts, redo_items;
  DevBuf batch_args, batch_off, batch_counters, batch_redo;  // batched vote pass
  // candidate cells the last vote pass of a model with this signature
  // (points, d_dist, threshold) emitted; sizes the next batch's buffers when
  // the same model is built again
  std::unordered_map<uint64_t, size_t> cand_hints;
  // vote segment length chosen by the tuner per model signature
  // (tune_vote_segments); PPF_B200_TUNE=0 keeps the default
  std::unordered_map<uint64_t, uint32_t> seg_tuned;
  bool tune = true;
  uint32_t forced_seg_shift = 0;  // PPF_B200_VOTE_SEGMENT=<2^k>: every model uses it
  DevBuf tune_counters;
  size_t cand_cap = size_t(1) << 24;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  int vote_smem_limit = 0;  // max dynamic shared memory per vote block
  size_t launches = 0;      // kernels launched (running total)
  bool checks = false;      // self-checking kernels (PPF_B200_CHECKS=1)
  bool cluster_split = true; // exact-sum split clustering allowed (PPF_B200_CLUSTER_SPLIT=0: never)
  bool cluster_sqrt = false; // PPF_B200_CLUSTER_SQRT=1: translation test with the square root
  ~Context();
};

// Model hash array resident in HBM (built once by ppf_model_create).
struct ModelTables {
  uint32_t n = 0;        // model points
  float d_dist = 0;
  // per model point
  DevBuf pts, nrm;       // float4 (x, y, z, 0)
  DevBuf frame_r1, frame_r2;  // rows 1 and 2 of the point's reference frame
  DevBuf angles;         // float2 (roty, rotz) of the frame
  DevBuf weights;        // float vote weights (default 1)
  // all ordered pairs, sorted by feature key (stable: pair index order)
  size_t P = 0;
  DevBuf keys;           // uint32 sorted keys
  DevBuf pairs;          // uint32 pair index r*n + i (the hash array's data map)
  DevBuf entries;        // uint32 (m_r mod chunk) << 21 | 21-bit angle of u,
                         // vote order: by key, then m_r, then a hash of the pair
  DevBuf epairs;         // uint32 pair index of each entry (vote order)
  // runs
  size_t K = 0;
  DevBuf uniq, first, count;  // uint32 each
  DevBuf run_flags;           // uint8: 1 = run holds a degenerate pair (exact bins only)
  // key -> run open-addressing table (key 0 is the empty marker)
  DevBuf ht_keys, ht_runs;
  uint32_t ht_mask = 0;
  // m_r chunking of the vote accumulator
  uint32_t chunk = 0, n_chunks = 0;
  DevBuf split;  // uint32 [K * (n_chunks + 1)] first run position per chunk
};

struct SceneData {
  uint32_t n = 0;
  float d_dist = 0;
  uint32_t ref_df = 1;
  DevBuf pts, nrm;  // float4
};

// Results of the last lookup, kept on the device for the inspection calls.
struct LookupState {
  size_t U = 0;
  DevBuf codes;       // uint64 kept vote codes, reference order
  DevBuf counts;      // uint32
  DevBuf weighted;    // float
  DevBuf transforms;  // float U*16
  DevBuf trans;       // float U*3 (after clustering)
  DevBuf trans0;      // float U*3 (before clustering)
  DevBuf quats;       // float U*4
  DevBuf cell_keys;   // uint32 U
  DevBuf adj;         // uint32 U*27
  DevBuf scores;      // float U
  DevBuf cells_sorted, cells_map, cells_uniq, cells_first, cells_count;
  DevBuf cells3;      // int4 U: integer cell of each pose
  DevBuf qs, tws, adjrun, item_off;  // cell-major clustering tables
  DevBuf item_off32;  // split clustering: (32-target tile, neighbour) items per run
  DevBuf tmp64, tmp32a, tmp32b, tmp32c, perm;
  DevBuf tperm;       // clustering target order (cell, rotation bucket)
  DevBuf best;        // float[16] pose + int idx
  DevBuf argmax_v, argmax_i;  // per-block partial maxima of the scores
  uint32_t cluster_path = 0;  // ppf_stats::cluster_path of the last clustering
  std::vector<float> cpu_poses;
};

struct Model {
  Context* ctx = nullptr;
  ModelTables t;
  float vote_count_threshold = 0.4f;
  bool cpu_clustering = false, use_l1_norm = false, use_averaged_clusters = false;
  size_t cand_hint = 0;  // candidate cells of the last vote pass (sizes batch buffers)
  // log2 of the vote pass's segment length (entries a warp streams per
  // segment); 0 until the tuner has chosen it (the default is used)
  // (atomic: the workers of a server may tune one library model at once)
  std::atomic<uint32_t> seg_shift{0};
  LookupState last;
};

// ---- model build (model.cu)
void build_model(Context& ctx, ModelTables& t, const float* xyz, const float* nxyz, size_t n,
                 float d_dist);
// keys of all n*n ordered pairs of a cloud held as float4 device arrays
void pair_keys_device(Context& ctx, const float4* pts, const float4* nrm, uint32_t n,
                      uint32_t ref_df, float d_dist, uint32_t* keys);
// upload n x 3 floats (host or device) into a float4 device array
void upload_points(Context& ctx, const float* xyz, size_t n, DevBuf& dst);
// Device memory of `device` or managed memory: true; host memory: false.
// Device memory of another GPU raises PPF_ERR_INVALID_ARGUMENT.
bool is_device_pointer(const void* p, int device);
// Device or managed memory of any GPU.
bool is_any_device_pointer(const void* p);

// ---- voting (vote.cu)
struct VoteResult {
  uint32_t max_count = 0;
  uint64_t n_votes = 0, n_matched = 0, n_exact = 0;
  uint64_t n_cand = 0;
  uint32_t n_redo = 0;  // items emitted by a second launch after the buffer grew
  uint64_t n_needed = 0;  // cells the first launch's items asked for (sizes the next buffer)
  float vote_ms = 0;
};
// Runs the vote pass.  emit_all: emit every nonzero cell (no threshold);
// floor >= 0 forces the emission floor.  Candidates land in
// ctx.cand_codes / ctx.cand_counts.
VoteResult run_votes(Context& ctx, const Model& m, const SceneData& s, bool emit_all, float floor);
// One request of a batched vote pass: its candidate cells land in its own
// buffers (cap cells, grown if they do not fit).
struct BatchVote {
  const Model* m = nullptr;
  const SceneData* s = nullptr;
  size_t cap = 0;
  DevBuf codes, counts;
  VoteResult r;
};
// The vote passes of all requests in one persistent launch (threshold x
// running maximum emission, as run_votes with emit_all = false).
void run_votes_batch(Context& ctx, std::vector<BatchVote>& reqs);
void pair_vote_counts(Context& ctx, const Model& m, const SceneData& s, uint64_t* out_dev);
// The vote pass with no device allocation: scene and outputs are the
// caller's device arrays, everything else lives in a static device array of
// vote.cu (ppf_model_vote_cells_noalloc).
void vote_cells_noalloc(Context& ctx, const Model& m, const float* xyz, const float* nxyz,
                        uint64_t n, uint32_t ref_df, float vote_floor, uint64_t* codes,
                        uint32_t* counts, uint64_t capacity, uint64_t* n_out, uint32_t* max_out);

// Default log2 segment length of the vote pass and the tuner's candidates.
constexpr uint32_t kSegShiftDefault = 12;
// Chooses the vote pass's segment length for model m on its first lookup
// (per model signature, cached in the context): short vote launches over a
// sample of the work items of (m, s), counting only, one per candidate.
void tune_vote_segments(Context& ctx, Model& m, const SceneData& s, uint64_t signature);
uint64_t model_signature(const Model& m);

// ---- poses and clustering (pose.cu)
// Filters the candidates to the kept votes and orders them (count desc,
// code asc); returns U.
size_t select_votes(Context& ctx, const Model& m, const SceneData& s, LookupState& st,
                    const unsigned long long* cand_code, const uint32_t* cand_count, size_t n_cand,
                    float min_votecount, uint32_t max_count);
// Orders arbitrary (code, count) pairs by code ascending (all-votes dump).
void sort_by_code(Context& ctx, LookupState& st, size_t n);
void compute_poses(Context& ctx, const Model& m, const SceneData& s, LookupState& st);
// GPU clustering + argmax; writes the best pose into st.best and returns the index.
size_t cluster_poses_gpu(Context& ctx, const Model& m, LookupState& st, float* best_score);

// ---- driver preprocessing (preprocess.cu)
// per-axis min / max over finite points (false when there is none)
bool cloud_extent(Context& ctx, const float* xyz_dev, size_t n, float lo[3], float hi[3]);
// pcl::VoxelGrid centroids of an n x 3 cloud; returns the voxel count
size_t voxel_downsample(Context& ctx, const float* xyz_dev, const float* nxyz_dev, size_t n, float leaf,
                        DevBuf& out_xyz, DevBuf& out_nxyz);

// ---- PLY files (ply.cpp)
ppf_status ply_read(const char* path, float* xyz, float* nxyz, uint64_t cap, uint64_t* n_out, std::string* err);
ppf_status ply_write(const char* path, const float* xyz, const float* nxyz, uint64_t n);

// ---- lookups (capi.cu)
struct LookupOut {
  ppf_status status = PPF_OK;
  float pose[16] = {0};
  ppf_stats stats{};
  size_t cand_hint = 0;  // candidate cells to provide for the next pass of this model
};
void init_context(Context& c, int device);
// Lookups of (models[i], scenes[i]) with one batched vote pass.  states:
// per-request lookup state (nullptr: each model's own `last`); caps:
// per-request candidate capacity hints (nullptr: the models' last passes).
std::vector<LookupOut> lookup_batch(Context& ctx, const std::vector<Model*>& models,
                                    const std::vector<const SceneData*>& scenes, LookupState* states,
                                    const size_t* caps);

// ---- request loop (serve.cu)
struct Server;
Server* server_create(int device, const std::vector<Model*>& models, size_t memory_budget,
                      uint32_t n_workers, uint32_t max_batch);
uint64_t server_submit(Server* srv, const float* xyz, const float* nxyz, uint64_t n, uint32_t ref_df,
                       const uint32_t* model_ids, uint64_t n_ids);
ppf_status server_wait(Server* srv, uint64_t ticket, float* poses, ppf_stats* stats, double* latency_ms,
                       std::string* error);
void server_destroy(Server* srv);

// ---- greedy clustering of the cpu_clustering path on the device (greedy.cu)
int cluster_poses_greedy_gpu(Context& ctx, const float* transforms_dev, const uint32_t* votes_dev, size_t U,
                             float trans_thresh, float rot_thresh, float out_poses[3 * 16], uint32_t out_votes[3]);

int cluster_poses_sorted_gpu(Context& ctx, const float* transforms_dev, const uint32_t* votes_dev, size_t U,
                             float trans_thresh, float rot_thresh, float out_poses[3 * 16], uint32_t out_votes[3]);

}  // namespace ppf

// Handles are reference-counted: the caller's handle is one reference, and
// every model, scene and server made on a context holds one on it (a server
// also holds one on each library model).  A destroy call drops the caller's
// reference; the object goes when the last one does, so handles can be
// destroyed in any order.
struct ppf_context_s {
  ppf::Context c;
  std::atomic<int> refs{1};
};
struct ppf_model_s {
  ppf::Model m;
  ppf_context_s* owner = nullptr;
  std::atomic<int> refs{1};
};
struct ppf_scene_s {
  ppf::Context* ctx = nullptr;
  ppf_context_s* owner = nullptr;
  ppf::SceneData s;
};
struct ppf_server_s {
  ppf::Server* srv = nullptr;
  std::vector<ppf_model_s*> library;
};
