// TEST INFRASTRUCTURE ONLY.  Host build of the reference's own arithmetic
// helpers, compiled in place from the reference sources (src/cuda/kernel.cu,
// src/cuda/vector_ops.cu) so the CPU oracle can be pinned against them bit for
// bit on a machine without a GPU.  kernel.cu's device-only helpers
// (trans_model_scene, compute_rot_angles, compute_transforms) are made
// host-callable by widening the __device__ execution-space macro for that one
// translation unit; every other declaration keeps its meaning.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <cuda_runtime.h>
#include <math_constants.h>
#include <vector_types.h>

#include "kernel.h"
#include "vector_ops.h"

#undef __device__
#define __device__ __location__(host) __location__(device)
#include "kernel.cu"
#undef __device__
#define __device__ __location__(device)

extern "C" {

uint32_t ref_hash(const void* p, int n) { return hash((void*)p, n); }

void ref_pair_feature(const float* p1, const float* n1, const float* p2, const float* n2,
                      float d_dist, float out[4]) {
  float3 a = make_float3(p1[0], p1[1], p1[2]), na = make_float3(n1[0], n1[1], n1[2]);
  float3 b = make_float3(p2[0], p2[1], p2[2]), nb = make_float3(n2[0], n2[1], n2[2]);
  float4 f = disc_feature(compute_ppf(a, na, b, nb), d_dist, D_ANGLE0);
  out[0] = f.x;
  out[1] = f.y;
  out[2] = f.z;
  out[3] = f.w;
}

uint32_t ref_feature_key(const float f[4]) {
  float4 v = make_float4(f[0], f[1], f[2], f[3]);
  if (isnan(v.x)) return 0;
  return hash(&v, sizeof(float4));
}

uint32_t ref_trans_model_scene(const float* m_r, const float* n_r_m, const float* m_i,
                               const float* s_r, const float* n_r_s, const float* s_i) {
  unsigned int a = 0;
  trans_model_scene(make_float3(m_r[0], m_r[1], m_r[2]), make_float3(n_r_m[0], n_r_m[1], n_r_m[2]),
                    make_float3(m_i[0], m_i[1], m_i[2]), make_float3(s_r[0], s_r[1], s_r[2]),
                    make_float3(n_r_s[0], n_r_s[1], n_r_s[2]), make_float3(s_i[0], s_i[1], s_i[2]),
                    0.f, a);
  return a;
}

void ref_vote_pose(uint32_t angle_idx, const float* m_r, const float* n_r_m, const float* s_r,
                   const float* n_r_s, float T[16]) {
  float mry, mrz, sry, srz;
  compute_rot_angles(make_float3(n_r_m[0], n_r_m[1], n_r_m[2]),
                     make_float3(n_r_s[0], n_r_s[1], n_r_s[2]), &mry, &mrz, &sry, &srz);
  compute_transforms(angle_idx, make_float3(m_r[0], m_r[1], m_r[2]), mry, mrz,
                     make_float3(s_r[0], s_r[1], s_r[2]), sry, srz, T);
}

void ref_hrotmat2quat(const float T[16], float q[4]) {
  float M[4][4];
  memcpy(M, T, sizeof(M));
  float4 r = hrotmat2quat(M);
  q[0] = r.x;
  q[1] = r.y;
  q[2] = r.z;
  q[3] = r.w;
}

// The host-side arithmetic of trans2idx_kernel (kernel.cu:675-694) for one
// translation, from the reference's own discretize() and hash().
uint32_t ref_trans_cell_keys(const float t[3], float d_dist, uint32_t adj[27]) {
  float3 disc = discretize(make_float3(t[0], t[1], t[2]), d_dist);
  int3 c;
  c.x = (int)(disc.x / d_dist);
  c.y = (int)(disc.y / d_dist);
  c.z = (int)(disc.z / d_dist);
  uint32_t key = hash(&c, sizeof(int3));
  int idx = 0;
  for (int i = -1; i < 2; i++)
    for (int j = -1; j < 2; j++)
      for (int k = -1; k < 2; k++, idx++) {
        if (i == 0 && j == 0 && k == 0) {
          adj[idx] = 0;
          continue;
        }
        int3 a = make_int3(c.x + i, c.y + j, c.z + k);
        adj[idx] = hash(&a, sizeof(int3));
      }
  return key;
}

}  // extern "C"
