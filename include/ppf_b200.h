/*
 * ppf_b200 -- C ABI of the B200 point pair feature (PPF) registration engine.
 *
 * Drop-in boundary for the reference's registration path
 * (nicolasavru/ppf-registration-spatial-hashing).  The reference exposes only
 * C++ (include/ppf.h, include/model.h, include/scene.h); every entry point
 * below names the reference interface it replaces.  Plain pointers and sizes,
 * no C++ or framework types.  Nothing here exits the process or resets the
 * device: failures return a status and ppf_last_error() describes them.
 *
 * Pointers: point/normal inputs may be host or device memory (detected per
 * call).  Clouds are n x 3 float32 arrays (x, y, z per point), normals unit
 * length.  Poses are 4x4 float32 row-major and map model coordinates into
 * scene coordinates.
 */
#ifndef PPF_B200_H
#define PPF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PPF_B200_ABI_VERSION 3

typedef enum ppf_status {
  PPF_OK = 0,
  PPF_ERR_INVALID_ARGUMENT = 1, /* bad sizes, null pointers, out-of-range knobs */
  PPF_ERR_CUDA = 2,             /* a CUDA runtime call failed */
  PPF_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed */
  PPF_ERR_NO_VOTES = 4,         /* no scene pair matched the model: no pose */
  PPF_ERR_TIMEOUT = 5,          /* a bounded device-side wait gave up */
  PPF_ERR_INTERNAL = 6
} ppf_status;
#define PPF_ERR_OOM PPF_ERR_OUT_OF_MEMORY

typedef struct ppf_context_s* ppf_context_t; /* device + stream + workspace */
typedef struct ppf_model_s* ppf_model_t;     /* resident model hash array */
typedef struct ppf_scene_s* ppf_scene_t;     /* resident scene cloud */
typedef struct ppf_server_s* ppf_server_t;   /* request loop over a model library */

/* Per-lookup statistics (the reference logs these at debug level,
 * src/cuda/model.cu:122,152,161-168,280). */
typedef struct ppf_stats {
  uint64_t n_votes;          /* V: votes cast (sum of matched run lengths) */
  uint64_t n_matched_pairs;  /* scene pairs whose key matched a model run */
  uint32_t max_vote_count;   /* largest (s_r, m_r, alpha) vote count */
  float min_votecount;       /* vote_count_threshold * max_vote_count */
  uint64_t n_kept;           /* U: vote codes above the threshold */
  uint64_t max_idx;          /* index of the chosen pose among the U */
  float best_score;          /* its clustering score */
  uint64_t n_candidates;     /* cells emitted by the vote pass (>= U) */
  uint64_t n_exact_bins;     /* votes binned by the exact-atan2 path */
  float vote_ms;             /* device time of the vote pass */
  float total_ms;            /* device time of the whole lookup */
  uint32_t gpu_launches;     /* kernels launched by the lookup */
  uint32_t n_redo_items;     /* vote items emitted again after the candidate buffer grew */
  uint32_t cluster_path;     /* clustering that ran: 0 none, 1 ordered sums per cell tile,
                                2 per-pose neighbour lists, 3 split exact sums, 4 greedy */
  uint32_t vote_segment;     /* entries per warp segment of the vote pass: chosen per model
                                by timing sample vote launches on the model's first lookup
                                (the same choice for every later lookup of a model with the
                                same points count, d_dist and threshold on this context) */
} ppf_stats;

/* Error text of the last failing call on this thread ("" if none). */
const char* ppf_last_error(void);
int ppf_abi_version(void);

/* Device selection as ppf_registration's devUse: device min(count-1, device)
 * (src/cuda/ppf.cu:37-49).  The context owns a CUDA stream and a workspace;
 * it never resets the device (the reference calls cudaDeviceReset at the end
 * of ppf_registration, src/cuda/ppf.cu:103).  Models and scenes keep using
 * the context that made them; each holds a reference on it, and a server
 * holds one on each of its library models.  Handles may be destroyed in any
 * order: ppf_context_destroy and ppf_model_destroy drop the caller's
 * reference, and the context or model goes (after its stream finishes) when
 * the last model, scene or server using it is destroyed. */
ppf_status ppf_context_create(int device, ppf_context_t* out);
ppf_status ppf_context_destroy(ppf_context_t ctx);
ppf_status ppf_context_synchronize(ppf_context_t ctx);
/* The stream all work of this context is ordered on (a cudaStream_t). */
void* ppf_context_stream(ppf_context_t ctx);
/* Kernels this context has launched so far (running total). */
uint64_t ppf_context_kernel_launches(ppf_context_t ctx);
/* The CUDA device index the context runs on (-1 for a null context). */
int ppf_context_device(ppf_context_t ctx);

/* Model::Model(cloud, d_dist, vote_count_threshold, cpu_clustering,
 * use_l1_norm, use_averaged_clusters) (include/model.h:17-19,
 * src/cuda/model.cu:43-82): PPFs of all ordered model pairs, their keys and
 * the sorted hash array, kept resident for any number of lookups.
 * n must be in [2, 65535]. */
ppf_status ppf_model_create(ppf_context_t ctx, const float* xyz, const float* nxyz, uint64_t n,
                            float d_dist, float vote_count_threshold, int cpu_clustering,
                            int use_l1_norm, int use_averaged_clusters, ppf_model_t* out);
/* Model::SetModelPointVoteWeights (src/cuda/model.cu:91-93): n weights, one
 * per model point (default 1.0); host or device pointer. */
ppf_status ppf_model_set_point_vote_weights(ppf_model_t m, const float* w, uint64_t n);
ppf_status ppf_model_destroy(ppf_model_t m);
uint64_t ppf_model_num_points(ppf_model_t m);
uint64_t ppf_model_num_keys(ppf_model_t m); /* unique feature keys K */
/* Chunks of model reference points the vote pass splits the model into: one
 * chunk's (m_r, alpha) counters fill one block's shared memory, so a scene
 * reference point is one work item per chunk.  No counterpart in the
 * reference, which keeps every vote in global memory. */
uint64_t ppf_model_num_chunks(ppf_model_t m);

/* Scene::Scene(cloud, d_dist, ref_point_downsample_factor)
 * (include/scene.h:15-16, src/cuda/scene.cu:24-55).  Scene pair features are
 * streamed during lookup, never materialised.  n must be >= 1 and < 2^31. */
ppf_status ppf_scene_create(ppf_context_t ctx, const float* xyz, const float* nxyz, uint64_t n,
                            float d_dist, uint32_t ref_point_df, ppf_scene_t* out);
ppf_status ppf_scene_destroy(ppf_scene_t s);

/* Model::ppf_lookup(scene) (src/cuda/model.cu:269-306) followed by the pose
 * extraction of ppf_registration (src/cuda/ppf.cu:74-93): votes, threshold,
 * poses, GPU pose clustering (or the greedy CPU clustering when the model was
 * created with cpu_clustering) and the best pose, row-major into pose_out
 * (host or device).  stats may be NULL.  The scene must have been created
 * with the model's d_dist. */
ppf_status ppf_model_lookup(ppf_model_t m, ppf_scene_t s, float* pose_out, ppf_stats* stats);

/* n lookups, request i = (models[i], scenes[i]), with one batched vote pass:
 * the loop of Model::ppf_lookup calls in ppf_registration
 * (src/cuda/ppf.cu:57-96, src/cuda/model.cu:269-306) over resident models.
 * All work items of all requests share one persistent launch; the threshold,
 * poses and clustering then run per request.  Each pose and stats record is
 * the one ppf_model_lookup gives for the same request.  poses_out: n x 16
 * (host or device); stats_out: n records or NULL (vote_ms is the batch's
 * vote time split by work items).  Returns PPF_ERR_NO_VOTES when any request
 * had no vote above the threshold (its pose is zero).  A model may appear in
 * several requests; its inspection getters then show its last request. */
ppf_status ppf_lookup_batch(ppf_context_t ctx, uint64_t n, const ppf_model_t* models,
                            const ppf_scene_t* scenes, float* poses_out, ppf_stats* stats_out);

/* clusterPoses (src/transformation_clustering.cpp:62-123), the greedy
 * clustering of the cpu_clustering path, on the device: poses (n row-major
 * 4x4, host or device) sorted by votes descending (stable: equal votes keep
 * their input order; the reference's std::sort leaves them unspecified),
 * each joining the first cluster whose first pose is within trans_thresh and
 * rot_thresh radians, else starting one; the (at most) three clusters with
 * most votes, averaged (translations, and quaternions in 4-D renormalised),
 * go to out_poses (3 x 16, host) and their vote totals to out_votes. */
ppf_status ppf_cluster_poses(ppf_context_t ctx, const float* transforms, const uint32_t* votes, uint64_t n,
                             float trans_thresh, float rot_thresh, float* out_poses, uint32_t* out_votes,
                             uint32_t* n_clusters);

/* pcl::io::loadPLYFile<pcl::PointNormal> as the alignment driver loads its
 * scene and model files (src/alignment.cpp:212,241): the vertex element's x,
 * y, z and nx, ny, nz (or normal_x, normal_y, normal_z), any scalar type,
 * ascii or binary files; other elements are skipped.  xyz, nxyz: host arrays
 * of cap x 3 floats.  With cap = 0 and null arrays only *n_out is set. */
ppf_status ppf_ply_read(const char* path, float* xyz, float* nxyz, uint64_t cap, uint64_t* n_out);
/* Writes a binary_little_endian PLY of float x y z nx ny nz (host arrays). */
ppf_status ppf_ply_write(const char* path, const float* xyz, const float* nxyz, uint64_t n);

/* pcl::getMinMax3D of a cloud as the alignment driver uses it
 * (src/alignment.cpp:246-253): per-axis minimum and maximum over the finite
 * points of n x 3 xyz (host or device).  The driver's model d_dist is
 * tau_d * max(max - min).  PPF_ERR_INVALID_ARGUMENT when no point is finite. */
ppf_status ppf_cloud_extent(ppf_context_t ctx, const float* xyz, uint64_t n, float* min_out,
                            float* max_out);

/* voxelGridDownsample (src/alignment.cpp:79-87): pcl::VoxelGrid<PointNormal>
 * (PCL 1.8) with cubic leaf size `leaf`.  Non-empty voxels in the grid's
 * linear index order (x fastest), each the mean of its points' coordinates
 * and normals (normals are not renormalised); the input is returned
 * unchanged when the grid would exceed 2^31 - 1 cells, as PCL does.  Inputs
 * and outputs host or device; outputs need room for *n_out <= n points
 * (cap); PPF_ERR_INVALID_ARGUMENT with *n_out set when cap is smaller. */
ppf_status ppf_voxel_downsample(ppf_context_t ctx, const float* xyz, const float* nxyz, uint64_t n,
                                float leaf, float* out_xyz, float* out_nxyz, uint64_t cap,
                                uint64_t* n_out);

/* Request loop over a resident model library: a serving form of
 * ppf_registration (src/cuda/ppf.cu:29-106), which instead rebuilds every
 * model for every call.  The server holds a reference on each library
 * model until ppf_server_destroy, so the caller may destroy its model handles
 * earlier.  n_workers threads, each with its own context on
 * `device`, take queued requests in arrival order and admit them while their
 * estimated device memory (scene, candidate cells, lookup state) fits
 * memory_budget bytes; up to max_batch admitted requests share one batched
 * vote pass.  Workers run concurrently, so requests that arrive while others
 * are on the GPU are admitted as memory frees and overlap them.  A request
 * larger than the whole budget runs alone. */
ppf_status ppf_server_create(int device, uint64_t n_models, const ppf_model_t* models,
                             uint64_t memory_budget, uint32_t n_workers, uint32_t max_batch,
                             ppf_server_t* out);
/* Queues one scene (host memory, n x 3 points and normals, copied before the
 * call returns) for registration against the library models model_ids[0..
 * n_targets), each with its own d_dist as ppf_registration does.
 * Thread-safe. */
ppf_status ppf_server_submit(ppf_server_t srv, const float* xyz, const float* nxyz, uint64_t n,
                             uint32_t ref_point_df, uint64_t n_targets, const uint32_t* model_ids,
                             uint64_t* ticket);
/* Waits for a request and collects it (a ticket is collected once):
 * poses_out n_targets x 16 (host), stats_out n_targets records or NULL,
 * latency_ms (may be NULL) from submission to completion.  Each pose equals
 * ppf_model_lookup of the same (model, scene).  PPF_ERR_NO_VOTES when a
 * target had no vote above the threshold (its pose is zero). */
ppf_status ppf_server_wait(ppf_server_t srv, uint64_t ticket, float* poses_out, ppf_stats* stats_out,
                           double* latency_ms);
/* Finishes every queued request, then stops the workers. */
ppf_status ppf_server_destroy(ppf_server_t srv);

/* ppf_registration(scene_clouds, model_clouds, model_d_dists,
 * ref_point_downsample_factor, vote_count_threshold, cpu_clustering,
 * use_l1_norm, use_averaged_clusters, devUse, model_weights)
 * (include/ppf.h:9-15, src/cuda/ppf.cu:29-106): every scene against every
 * model; poses_out receives n_scenes * n_models row-major 4x4 poses, indexed
 * [scene][model] as the reference's result vector.  model_weights is accepted
 * and ignored, as in the reference (src/cuda/ppf.cu:35); per-point weights go
 * through ppf_model_set_point_vote_weights.  Each model's hash array is built
 * once and reused for all scenes (the reference rebuilds it per scene with
 * identical results).  A (scene, model) pair with no votes yields an all-zero
 * pose and the call returns PPF_ERR_NO_VOTES after finishing the others. */
ppf_status ppf_registration(ppf_context_t ctx, uint64_t n_scenes, const float* const* scene_xyz,
                            const float* const* scene_nxyz, const uint64_t* scene_n,
                            uint64_t n_models, const float* const* model_xyz,
                            const float* const* model_nxyz, const uint64_t* model_n,
                            const float* model_d_dists, uint32_t ref_point_df,
                            float vote_count_threshold, int cpu_clustering, int use_l1_norm,
                            int use_averaged_clusters, int dev_use, const float* model_weights,
                            float* poses_out, ppf_stats* stats_out /* n_scenes*n_models or NULL */);

/* ---- inspection of the last lookup (the reference's public Model members,
 *      include/model.h:61-113); host output buffers, *n receives the count.
 *      A NULL buffer or too small a capacity only reports *n. ---- */

/* votes / voteCounts after the threshold, ordered by count descending then
 * code ascending (src/cuda/model.cu:155-170); code = s_r<<32 | m_r<<6 | alpha. */
ppf_status ppf_model_get_votes(ppf_model_t m, uint64_t* codes, uint32_t* counts, uint64_t cap,
                               uint64_t* n);
/* transformations (src/cuda/model.cu:191-200), U x 16 row-major. */
ppf_status ppf_model_get_transformations(ppf_model_t m, float* T, uint64_t cap, uint64_t* n);
/* transformation_trans (after clustering), transformation_rots, vote_counts_out
 * (src/cuda/model.cu:202-244): U x 3, U x 4 (w,x,y,z), U. */
ppf_status ppf_model_get_cluster_state(ppf_model_t m, float* trans, float* quats, float* scores,
                                       uint64_t cap, uint64_t* n);
/* ParallelHashArray of the model (include/impl/parallel_hash_array.hpp:16-47):
 * unique keys, counts, first offsets (K each) and the key-sorted pair index
 * map (P = n*n entries; pair = row*n + col). */
ppf_status ppf_model_get_hash_array(ppf_model_t m, uint32_t* keys, uint32_t* counts,
                                    uint32_t* first, uint64_t cap_k, uint32_t* map, uint64_t cap_p,
                                    uint64_t* K, uint64_t* P);

/* Keys of all n*n ordered pairs of a cloud, as Scene::initPPFs +
 * ppf_hash_kernel produce them (src/cuda/scene.cu:64-99,
 * src/cuda/kernel.cu:404-477): rows with index % ref_point_df != 0 and self
 * pairs give 0.  keys is host or device memory of n*n uint32. */
ppf_status ppf_pair_keys(ppf_context_t ctx, const float* xyz, const float* nxyz, uint64_t n,
                         float d_dist, uint32_t ref_point_df, uint32_t* keys);

/* Every nonzero (s_r, m_r, alpha) vote cell of a lookup in code order with its
 * count: the reference's unique votes before the threshold
 * (src/cuda/model.cu:148-151).  Runs the vote pass with no threshold; meant
 * for small inputs. */
ppf_status ppf_model_all_votes(ppf_model_t m, ppf_scene_t s, uint64_t* codes, uint32_t* counts,
                               uint64_t cap, uint64_t* n);

/* Per-scene-pair vote counts of ppf_vote_count_kernel
 * (src/cuda/kernel.cu:480-501): counts[r*n_s + i] = model run length when
 * scene pair (r, i) matches, else 0.  counts: host or device, n_s*n_s uint64. */
ppf_status ppf_model_pair_vote_counts(ppf_model_t m, ppf_scene_t s, uint64_t* counts);

/* Allocation-free vote pass.  No counterpart in the reference: the
 * reference allocates its vote buffers on every lookup
 * (src/cuda/model.cu:95-171).
 *
 * For callers that must not allocate device memory while they run: a serving
 * process whose device-memory budget was reserved at start-up (its own pool
 * holds the rest of the device, so a cudaMalloc fails or takes memory the
 * budget does not have), and latency-bound loops that cannot take the latency
 * of cudaMalloc/cudaFree or the device-wide synchronisation cudaFree implies.
 * This call allocates no device memory; the model must already exist.
 *
 * Runs the vote pass of ppf_model_lookup for one scene whose points and
 * normals (n_scene x 3 float32 each) are device memory, with the model's
 * d_dist as ppf_registration uses, and writes vote cells (code = s_r<<32 |
 * m_r<<6 | alpha, as ppf_model_all_votes) and their counts to the caller's
 * device arrays codes / counts (capacity entries each), in no particular
 * order.  vote_floor >= 0: every cell whose count exceeds vote_floor (0 gives
 * the nonzero cells ppf_model_all_votes returns).  vote_floor < 0: the
 * lookup's candidates, every cell whose count exceeds the model's
 * vote_count_threshold x the running maximum when its work item finished, a
 * superset of the cells the lookup keeps (count >= threshold x *max_count),
 * whose size varies from call to call.  *n_out: cells written;
 * *max_count (may be NULL): the largest count.
 *
 * Scratch: counters, the work items that did not fit and the scene packed to
 * float4 live in one static device array of 3 MiB + 256 B in the library,
 * which every GPU that loads the library holds until the process exits.
 * Limits: n_scene <= 65536 points and ceil(n_scene / ref_point_df) x
 * ppf_model_num_chunks(m) <= 262144 work items; larger inputs return
 * PPF_ERR_INVALID_ARGUMENT before any GPU work.  The call zeroes the scratch's 256-byte counter header on the
 * context's stream before its kernels; nothing the caller passes needs to
 * start at zero.  Output too small: PPF_ERR_OUT_OF_MEMORY, *n_out = the cells
 * this call needed (the cells of the work items that fit were written).
 *
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls on one device share the array:
 * calls that overlap in time (other threads, contexts or streams on the same
 * device) race on it, so the caller serialises them.  Each call sets the
 * vote kernel's shared-memory attribute, reads its counters back into host
 * memory and waits for the context's stream (cudaStreamSynchronize) before
 * it returns. */
ppf_status ppf_model_vote_cells_noalloc(ppf_model_t m, const float* scene_xyz,
                                        const float* scene_nxyz, uint64_t n_scene,
                                        uint32_t ref_point_df, float vote_floor, uint64_t* codes,
                                        uint32_t* counts, uint64_t capacity, uint64_t* n_out,
                                        uint32_t* max_count);

#ifdef __cplusplus
}
#endif
#endif /* PPF_B200_H */
