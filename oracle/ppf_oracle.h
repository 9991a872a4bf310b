/*
 * CPU oracle for the PPF registration path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's algorithm (nicolasavru/
 * ppf-registration-spatial-hashing, src/cuda/kernel.cu, src/cuda/model.cu,
 * include/impl/parallel_hash_array.hpp, src/transformation_clustering.cpp),
 * used by the tests as the checker and by bench.py as the timed CPU baseline.
 * Nothing in the product library links or calls this code.
 *
 * Arithmetic: float32 with the host C library (compiled with
 * -ffp-contract=off), which reproduces the reference's own __host__ build of
 * the same helpers bit for bit (pinned by tests/test_oracle_pins.py against
 * oracle/_ref/libppfref_host.so).  The GPU path is compiled with fast-math
 * division/sqrt and CUDA's acosf/atan2f, so CPU and GPU integer outputs agree
 * except at quantisation boundaries; the tests state that flip rate.  The
 * bit-exact GPU oracle is the reference's own kernels (oracle/refharness.cu).
 */
#ifndef PPF_ORACLE_H
#define PPF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- single-item helpers (pinned against the reference's host build) ---- */

/* kernel.cu:23-30 */
uint32_t orc_fnv1a(const void* data, int n, uint32_t seed);
/* kernel.cu:109-122 + 94-100: discretised feature of one ordered pair */
void orc_pair_feature(const float* p1, const float* n1, const float* p2, const float* n2,
                      float d_dist, float out[4]);
/* kernel.cu:460-477: key of a discretised feature (0 when f.x is NaN) */
uint32_t orc_feature_key(const float f[4]);
/* kernel.cu:302-349: alpha bin of one vote, literal 4x4 restatement */
uint32_t orc_trans_model_scene(const float* m_r, const float* n_r_m, const float* m_i,
                               const float* s_r, const float* n_r_s, const float* s_i);
/* kernel.cu:352-401: pose of a vote, row-major T[16] */
void orc_vote_pose(uint32_t angle_idx, const float* m_r, const float* n_r_m, const float* s_r,
                   const float* n_r_s, float T[16]);
/* the same pose in float64 (for error statements) */
void orc_vote_pose_f64(uint32_t angle_idx, const float* m_r, const float* n_r_m,
                       const float* s_r, const float* n_r_s, double T[16]);
/* kernel.cu:128-144: quaternion (w,x,y,z) normalised by sqrt(|q|) */
void orc_hrotmat2quat(const float T[16], float q[4]);
/* kernel.cu:663-699: cell key and the 27 neighbour keys (centre = 0) */
uint32_t orc_trans_cell_keys(const float t[3], float d_dist, uint32_t adj[27]);

/* ---- whole-array stages ---- */

/* ppf_kernel + ppf_hash_kernel (kernel.cu:404-477): keys of all n*n ordered
 * pairs, rows with idx % ref_df != 0 and self pairs get key 0. */
void orc_pair_keys(const float* pts, const float* nrm, int64_t n, uint32_t ref_df, float d_dist,
                   uint32_t* keys, int n_threads);

/* ParallelHashArray constructor (parallel_hash_array.hpp:55-77): stable sort
 * of keys with their positions, unique keys, counts, first offsets.
 * Returns the number of unique keys K. sorted_keys/map have n entries,
 * uniq/counts/first need room for n entries. */
int64_t orc_hash_array(const uint32_t* keys, int64_t n, uint32_t* sorted_keys, uint32_t* map,
                       uint32_t* uniq, uint32_t* counts, uint32_t* first);

/* ---- full registration of one scene against one model ---- */

typedef struct orc_result {
  uint64_t n_votes;        /* V: total votes cast (model.cu:121) */
  uint64_t n_unique;       /* unique vote codes before the threshold */
  uint32_t max_count;      /* largest vote count */
  float min_votecount;     /* threshold * max_count (model.cu:164) */
  uint64_t n_kept;         /* U: codes with count > min_votecount */
  uint64_t* codes;         /* [n_kept] (s_r<<32 | m_r<<6 | alpha), count desc, code asc */
  uint32_t* counts;        /* [n_kept] */
  float* weighted;         /* [n_kept] weight[m_r] * count (kernel.cu:766-782) */
  float* transforms;       /* [n_kept*16] row-major poses (kernel.cu:605-645) */
  float* trans;            /* [n_kept*3] translations after clustering */
  float* quats;            /* [n_kept*4] */
  uint32_t* cell_keys;     /* [n_kept] */
  float* scores;           /* [n_kept] clustering scores (kernel.cu:702-763) */
  uint64_t max_idx;        /* first index of the largest score (model.cu:293-295) */
  float pose[16];          /* final pose (ppf.cu:74-93 / :75-76 with cpu_clustering) */
  int status;              /* 0 ok, 1 no votes, 2 out of memory */
  /* greedy CPU clustering (transformation_clustering.cpp:62-123) */
  int n_clusters;
  float cpu_poses[3 * 16];
  uint32_t cpu_votes[3];
  double t_build;          /* seconds spent building the model hash array */
  double t_vote;           /* seconds spent in the vote loop */
  uint64_t n_refs;         /* scene reference points processed */
} orc_result;

typedef struct orc_params {
  float d_dist;
  uint32_t ref_point_df;
  float vote_count_threshold;
  int cpu_clustering;
  int use_l1_norm;
  int use_averaged_clusters;
  int n_threads;
  /* restrict the scene reference points to [sr_begin, sr_end) (by index);
   * sr_end < 0 means all.  Used for bounded CPU baseline samples. */
  int64_t sr_begin, sr_end;
  /* step between processed reference points; 0 means ref_point_df */
  int64_t sr_step;
  /* nonzero: stop after the threshold (codes and counts only; no poses or
   * clustering).  With vote_count_threshold 0 this gives every nonzero cell. */
  int votes_only;
} orc_params;

/* Model::Model + Model::ppf_lookup + pose extraction for one (scene, model). */
orc_result* orc_register(const float* m_pts, const float* m_nrm, int64_t n_m,
                         const float* s_pts, const float* s_nrm, int64_t n_s,
                         const float* model_weights, const orc_params* prm);
void orc_result_free(orc_result* r);

/* Per-scene-pair vote counts (ppf_vote_count_kernel, kernel.cu:480-501) given
 * model run tables: counts[i] = run length if the scene key matches. */
void orc_vote_counts(const uint32_t* scene_keys, int64_t n, const uint32_t* uniq,
                     const uint32_t* run_counts, int64_t K, uint64_t* counts);

/* Greedy clustering of poses (transformation_clustering.cpp:62-123) on
 * row-major float poses with integer votes; returns the number of clusters
 * reported (<= 3) and writes averaged poses and vote totals. */
int orc_cluster_poses(const float* poses, const uint32_t* votes, int64_t n, float trans_thresh,
                      float rot_thresh, float out_poses[3 * 16], uint32_t out_votes[3]);

/* ---- driver preprocessing (src/alignment.cpp:79-87, 246-253) ---- */

/* pcl::getMinMax3D over the finite points; returns 0 when there is none. */
int orc_cloud_extent(const float* xyz, int64_t n, float lo[3], float hi[3]);

/* pcl::VoxelGrid<PointNormal> (PCL 1.8, restated from its published
 * algorithm) with leaf size `leaf`: voxel means of points and normals in
 * linear voxel order, each voxel summed in input order; out arrays need room
 * for n points.  Returns the number of voxels (n, with the input copied, when
 * the grid exceeds 2^31 - 1 cells). */
int64_t orc_voxel_downsample(const float* xyz, const float* nxyz, int64_t n, float leaf, float* out_xyz,
                             float* out_nxyz);

#ifdef __cplusplus
}
#endif
#endif
