// CPU oracle for the PPF registration path -- TEST INFRASTRUCTURE ONLY.
// See ppf_oracle.h.  Every function cites the reference lines it restates
// (paths relative to the reference project root).  Built with
// -ffp-contract=off so float expressions round exactly as written.
#include "ppf_oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// include/kernel.h:15-17
const float kPi = 3.141592654f;  // CUDART_PI_F
const float kD = (2.0f * kPi) / float(30);
const float kRotThresh = 2 * kD;

struct F3 {
  float x, y, z;
};
struct F4 {
  float x, y, z, w;
};
typedef float M4[4][4];

inline F3 ld3(const float* p) { return F3{p[0], p[1], p[2]}; }

// kernel.cu:51-65
inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot4(F4 a, F4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float norm3(F3 a) { return sqrtf(dot3(a, a)); }
inline float norm4(F4 a) { return sqrtf(dot4(a, a)); }
// kernel.cu:90-92
inline float quant_downf(float x, float y) { return x - fmodf(x, y); }

// kernel.cu:32-49, 170-223
void zero4(M4 T) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) T[i][j] = 0;
}
void trans4(F3 v, M4 T) {
  zero4(T);
  T[0][0] = 1;
  T[1][1] = 1;
  T[2][2] = 1;
  T[3][3] = 1;
  T[0][3] = v.x;
  T[1][3] = v.y;
  T[2][3] = v.z;
}
void rotx(float th, M4 T) {
  zero4(T);
  T[0][0] = 1;
  T[1][1] = cosf(th);
  T[2][1] = sinf(th);
  T[1][2] = -1 * T[2][1];
  T[2][2] = T[1][1];
  T[3][3] = 1;
}
void roty(float th, M4 T) {
  zero4(T);
  T[0][0] = cosf(th);
  T[0][2] = sinf(th);
  T[1][1] = 1;
  T[2][0] = -1 * T[0][2];
  T[2][2] = T[0][0];
  T[3][3] = 1;
}
void rotz(float th, M4 T) {
  zero4(T);
  T[0][0] = cosf(th);
  T[1][0] = sinf(th);
  T[0][1] = -1 * T[1][0];
  T[1][1] = T[0][0];
  T[2][2] = 1;
  T[3][3] = 1;
}
// kernel.cu:211-223
void mul4(const M4 A, const M4 B, M4 C) {
  zero4(C);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) C[i][j] += A[i][k] * B[k][j];
}
inline F4 row4(const M4 A, int i) { return F4{A[i][0], A[i][1], A[i][2], A[i][3]}; }
// kernel.cu:234-242
inline F4 vmul4(const M4 A, F4 b) {
  return F4{dot4(row4(A, 0), b), dot4(row4(A, 1), b), dot4(row4(A, 2), b), dot4(row4(A, 3), b)};
}
// kernel.cu:254-299
void invht(const M4 T, M4 Ti) {
  Ti[0][0] = T[0][0];
  Ti[0][1] = T[1][0];
  Ti[0][2] = T[2][0];
  Ti[1][0] = T[0][1];
  Ti[1][1] = T[1][1];
  Ti[1][2] = T[2][1];
  Ti[2][0] = T[0][2];
  Ti[2][1] = T[1][2];
  Ti[2][2] = T[2][2];
  F3 r0{-Ti[0][0], -Ti[0][1], -Ti[0][2]};
  F3 r1{-Ti[1][0], -Ti[1][1], -Ti[1][2]};
  F3 r2{-Ti[2][0], -Ti[2][1], -Ti[2][2]};
  F3 t{T[0][3], T[1][3], T[2][3]};
  Ti[0][3] = dot3(r0, t);
  Ti[1][3] = dot3(r1, t);
  Ti[2][3] = dot3(r2, t);
  Ti[3][0] = 0;
  Ti[3][1] = 0;
  Ti[3][2] = 0;
  Ti[3][3] = 1;
}

// Frame of a reference point: kernel.cu:310-318 (model) / :320-327 (scene).
void frame(F3 p, F3 n, M4 Tg) {
  M4 tr, ry, rz, tmp;
  F3 np{-1 * p.x, -1 * p.y, -1 * p.z};
  trans4(np, tr);
  roty(atan2f(n.z, n.x), ry);
  F4 nt = vmul4(ry, F4{n.x, n.y, n.z, 1});
  rotz(-1 * atan2f(nt.y, nt.x), rz);
  mul4(rz, ry, tmp);
  mul4(tmp, tr, Tg);
}

// kernel.cu:338-342
inline uint32_t alpha_bin(F3 u, F3 v) {
  u.x = 0;
  v.x = 0;
  float cx = u.y * v.z - u.z * v.y;
  float alpha = atan2f(cx, dot3(u, v));
  alpha = quant_downf(alpha + kPi, kD);
  return (uint32_t)lrintf(alpha / kD);
}

inline F3 frame_apply(const M4 T, F3 q) {
  F4 h = vmul4(T, F4{q.x, q.y, q.z, 1});
  return F3{h.x, h.y, h.z};
}

// kernel.cu:352-369 (one half)
void rot_angles(F3 n, float* ry_out, float* rz_out) {
  M4 ry;
  *ry_out = atan2f(n.z, n.x);
  roty(*ry_out, ry);
  F4 nt = vmul4(ry, F4{n.x, n.y, n.z, 1});
  *rz_out = -1 * atan2f(nt.y, nt.x);
}

// kernel.cu:372-401
void transforms(uint32_t angle_idx, F3 m_r, float m_roty, float m_rotz, F3 s_r, float s_roty,
                float s_rotz, float* T) {
  M4 tr, rx, ry, rz, tmp, tmp2, Tm, Ts;
  F3 nm{-1 * m_r.x, -1 * m_r.y, -1 * m_r.z};
  trans4(nm, tr);
  roty(m_roty, ry);
  rotz(m_rotz, rz);
  mul4(rz, ry, tmp);
  mul4(tmp, tr, Tm);
  F3 ns{-1 * s_r.x, -1 * s_r.y, -1 * s_r.z};
  trans4(ns, tr);
  roty(s_roty, ry);
  rotz(s_rotz, rz);
  mul4(rz, ry, tmp);
  mul4(tmp, tr, Ts);
  rotx(angle_idx * kD - kPi, rx);
  invht(Ts, tmp);
  mul4(tmp, rx, tmp2);
  M4 out;
  mul4(tmp2, Tm, out);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) T[i * 4 + j] = out[i][j];
}

// ------------------------------------------------------------- float64 --
typedef double D4[4][4];
void zero4d(D4 T) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) T[i][j] = 0;
}
void mul4d(const D4 A, const D4 B, D4 C) {
  zero4d(C);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) C[i][j] += A[i][k] * B[k][j];
}
void frame_d(const float* p, const float* n, D4 Tg) {
  double ay = atan2((double)n[2], (double)n[0]);
  D4 ry, rz, tr, tmp;
  zero4d(ry);
  ry[0][0] = cos(ay);
  ry[0][2] = sin(ay);
  ry[1][1] = 1;
  ry[2][0] = -ry[0][2];
  ry[2][2] = ry[0][0];
  ry[3][3] = 1;
  double ntx = ry[0][0] * n[0] + ry[0][2] * n[2];
  double nty = (double)n[1];
  double az = -atan2(nty, ntx);
  zero4d(rz);
  rz[0][0] = cos(az);
  rz[1][0] = sin(az);
  rz[0][1] = -rz[1][0];
  rz[1][1] = rz[0][0];
  rz[2][2] = 1;
  rz[3][3] = 1;
  zero4d(tr);
  for (int i = 0; i < 4; ++i) tr[i][i] = 1;
  tr[0][3] = -(double)p[0];
  tr[1][3] = -(double)p[1];
  tr[2][3] = -(double)p[2];
  mul4d(rz, ry, tmp);
  mul4d(tmp, tr, Tg);
}

// ------------------------------------------------------ hash array helpers
struct HashArray {
  std::vector<uint32_t> uniq, counts, first, map;
};

// Stable LSD radix sort of 64-bit (key << 32 | position) words by the key.
void radix_sort_keys(std::vector<uint64_t>& kv) {
  std::vector<uint64_t> tmp(kv.size());
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 32 + 8 * pass;
    size_t cnt[257] = {0};
    for (uint64_t v : kv) cnt[((v >> shift) & 0xff) + 1]++;
    for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
    for (uint64_t v : kv) tmp[cnt[(v >> shift) & 0xff]++] = v;
    kv.swap(tmp);
  }
}

// parallel_hash_array.hpp:55-77 (stable sort by key, positions as values)
void build_hash_array(const uint32_t* keys, int64_t n, HashArray& H) {
  std::vector<uint64_t> kv(n);
  for (int64_t i = 0; i < n; ++i) kv[i] = ((uint64_t)keys[i] << 32) | (uint64_t)i;
  radix_sort_keys(kv);
  H.map.resize(n);
  H.uniq.clear();
  H.counts.clear();
  H.first.clear();
  for (int64_t i = 0; i < n; ++i) {
    uint32_t k = (uint32_t)(kv[i] >> 32);
    H.map[i] = (uint32_t)(kv[i] & 0xffffffffu);
    if (i == 0 || k != H.uniq.back()) {
      H.uniq.push_back(k);
      H.counts.push_back(1);
      H.first.push_back((uint32_t)i);
    } else {
      H.counts.back()++;
    }
  }
}

// lower_bound + hash-only compare (parallel_hash_array.hpp:80-92,
// kernel.cu:488-496): run index or -1.
inline int64_t find_run(const HashArray& H, uint32_t key) {
  if (key == 0) return -1;
  auto it = std::lower_bound(H.uniq.begin(), H.uniq.end(), key);
  if (it == H.uniq.end() || *it != key) return -1;
  return it - H.uniq.begin();
}

inline uint32_t fnv(const void* f, int n, uint32_t h) {
  const signed char* s = (const signed char*)f;
  while (n--) {
    h ^= (uint32_t)(int32_t)*s++;
    h *= 16777619u;
  }
  return h;
}

inline uint32_t key_of(const float f[4]) {
  if (std::isnan(f[0])) return 0;
  return fnv(f, 16, 2166136261u);
}

void pair_feature(F3 p1, F3 n1, F3 p2, F3 n2, float d_dist, float out[4]) {
  F3 d{p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
  float f0 = norm3(d);
  float f1 = acosf(dot3(n1, d) / (norm3(n1) * norm3(d)));
  float f2 = acosf(dot3(n2, d) / (norm3(n2) * norm3(d)));
  float f3 = acosf(dot3(n1, n2) / (norm3(n1) * norm3(n2)));
  out[0] = quant_downf(f0, d_dist);
  out[1] = quant_downf(f1, kD);
  out[2] = quant_downf(f2, kD);
  out[3] = quant_downf(f3, kD);
}

// hrotmat2quat (kernel.cu:128-144); T row-major
void quat_of(const float* T, float q[4]) {
  float t, r;
  t = T[0] + T[5] + T[10];
  r = sqrtf(1 + t);
  float qx = 0.5 * r;
  float qy = copysignf(0.5 * sqrtf(1 + T[0] - T[5] - T[10]), T[9] - T[6]);
  float qz = copysignf(0.5 * sqrtf(1 - T[0] + T[5] - T[10]), T[2] - T[8]);
  float qw = copysignf(0.5 * sqrtf(1 - T[0] - T[5] + T[10]), T[4] - T[1]);
  F4 qq{qx, qy, qz, qw};
  float n = sqrtf(norm4(qq));
  q[0] = qx / n;
  q[1] = qy / n;
  q[2] = qz / n;
  q[3] = qw / n;
}

// trans2idx_kernel (kernel.cu:663-699)
uint32_t cell_keys(const float* t, float d, uint32_t adj[27]) {
  float q0 = quant_downf(t[0], d), q1 = quant_downf(t[1], d), q2 = quant_downf(t[2], d);
  int c[3] = {(int)(q0 / d), (int)(q1 / d), (int)(q2 / d)};
  uint32_t key = fnv(c, 12, 2166136261u);
  int idx = 0;
  for (int i = -1; i < 2; ++i)
    for (int j = -1; j < 2; ++j)
      for (int k = -1; k < 2; ++k, ++idx) {
        if (i == 0 && j == 0 && k == 0) {
          adj[idx] = 0;
          continue;
        }
        int a[3] = {c[0] + i, c[1] + j, c[2] + k};
        adj[idx] = fnv(a, 12, 2166136261u);
      }
  return key;
}

// ---- Eigen-equivalent rotation helpers for the greedy CPU clustering ----
// Quaternion (x, y, z, w) from a 3x3 rotation (Eigen's published
// trace/largest-diagonal method), row-major m[9].
void mat_to_quat_xyzw(const float* m, float q[4]) {
  float t = m[0] + m[4] + m[8];
  if (t > 0.f) {
    t = sqrtf(t + 1.0f);
    q[3] = 0.5f * t;
    t = 0.5f / t;
    q[0] = (m[7] - m[5]) * t;
    q[1] = (m[2] - m[6]) * t;
    q[2] = (m[3] - m[1]) * t;
  } else {
    int i = 0;
    if (m[4] > m[0]) i = 1;
    if (m[8] > m[i * 3 + i]) i = 2;
    int j = (i + 1) % 3, k = (j + 1) % 3;
    t = sqrtf(m[i * 3 + i] - m[j * 3 + j] - m[k * 3 + k] + 1.0f);
    q[i] = 0.5f * t;
    t = 0.5f / t;
    q[3] = (m[k * 3 + j] - m[j * 3 + k]) * t;
    q[j] = (m[j * 3 + i] + m[i * 3 + j]) * t;
    q[k] = (m[k * 3 + i] + m[i * 3 + k]) * t;
  }
}

// Rotation part of an affine pose (row-major 4x4) as a 3x3: the linear block,
// or the identity when the block is all zero (the polar factor of 0).
void rotation_of(const float* T, float R[9]) {
  bool zero = true;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      R[i * 3 + j] = T[i * 4 + j];
      if (R[i * 3 + j] != 0.f) zero = false;
    }
  if (zero) {
    for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.f : 0.f;
  }
}

// posesWithinErrorBounds (transformation_clustering.cpp:127-137)
bool within_bounds(const float* T1, const float* T2, float trans_thresh, float rot_thresh) {
  float dx = T1[3] - T2[3], dy = T1[7] - T2[7], dz = T1[11] - T2[11];
  float pos = sqrtf(dx * dx + dy * dy + dz * dz);
  float R1[9], R2[9], M[9];
  rotation_of(T1, R1);
  rotation_of(T2, R2);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float s = 0;
      for (int k = 0; k < 3; ++k) s += R1[k * 3 + i] * R2[k * 3 + j];  // R1^T R2
      M[i * 3 + j] = s;
    }
  float q[4];
  mat_to_quat_xyzw(M, q);
  float nv = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  float ang = (nv != 0.f) ? 2.f * atan2f(nv, fabsf(q[3])) : 0.f;
  return pos < trans_thresh && fabsf(ang) < rot_thresh;
}

}  // namespace

// =========================================================== public API ==
extern "C" {

uint32_t orc_fnv1a(const void* data, int n, uint32_t seed) { return fnv(data, n, seed); }

void orc_pair_feature(const float* p1, const float* n1, const float* p2, const float* n2,
                      float d_dist, float out[4]) {
  pair_feature(ld3(p1), ld3(n1), ld3(p2), ld3(n2), d_dist, out);
}

uint32_t orc_feature_key(const float f[4]) { return key_of(f); }

uint32_t orc_trans_model_scene(const float* m_r, const float* n_r_m, const float* m_i,
                               const float* s_r, const float* n_r_s, const float* s_i) {
  M4 Tm, Ts;
  frame(ld3(m_r), ld3(n_r_m), Tm);
  frame(ld3(s_r), ld3(n_r_s), Ts);
  F3 u = frame_apply(Tm, ld3(m_i));
  F3 v = frame_apply(Ts, ld3(s_i));
  return alpha_bin(u, v);
}

void orc_vote_pose(uint32_t angle_idx, const float* m_r, const float* n_r_m, const float* s_r,
                   const float* n_r_s, float T[16]) {
  float mry, mrz, sry, srz;
  rot_angles(ld3(n_r_m), &mry, &mrz);
  rot_angles(ld3(n_r_s), &sry, &srz);
  transforms(angle_idx, ld3(m_r), mry, mrz, ld3(s_r), sry, srz, T);
}

void orc_vote_pose_f64(uint32_t angle_idx, const float* m_r, const float* n_r_m,
                       const float* s_r, const float* n_r_s, double T[16]) {
  D4 Tm, Ts, Tsi, rx, tmp, out;
  frame_d(m_r, n_r_m, Tm);
  frame_d(s_r, n_r_s, Ts);
  double a = (double)angle_idx * (2.0 * M_PI / 30.0) - M_PI;
  zero4d(rx);
  rx[0][0] = 1;
  rx[1][1] = cos(a);
  rx[2][1] = sin(a);
  rx[1][2] = -rx[2][1];
  rx[2][2] = rx[1][1];
  rx[3][3] = 1;
  zero4d(Tsi);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Tsi[i][j] = Ts[j][i];
  for (int i = 0; i < 3; ++i) {
    double s = 0;
    for (int k = 0; k < 3; ++k) s -= Tsi[i][k] * Ts[k][3];
    Tsi[i][3] = s;
  }
  Tsi[3][3] = 1;
  mul4d(Tsi, rx, tmp);
  mul4d(tmp, Tm, out);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) T[i * 4 + j] = out[i][j];
}

void orc_hrotmat2quat(const float T[16], float q[4]) { quat_of(T, q); }

uint32_t orc_trans_cell_keys(const float t[3], float d_dist, uint32_t adj[27]) {
  return cell_keys(t, d_dist, adj);
}

void orc_pair_keys(const float* pts, const float* nrm, int64_t n, uint32_t ref_df, float d_dist,
                   uint32_t* keys, int n_threads) {
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
  for (int64_t r = 0; r < n; ++r) {
    uint32_t* row = keys + r * n;
    if (n <= 1 || r % ref_df != 0) {
      for (int64_t i = 0; i < n; ++i) row[i] = 0;
      continue;
    }
    F3 pr = ld3(pts + 3 * r), nr = ld3(nrm + 3 * r);
    for (int64_t i = 0; i < n; ++i) {
      if (i == r) {
        row[i] = 0;
        continue;
      }
      float f[4];
      pair_feature(pr, nr, ld3(pts + 3 * i), ld3(nrm + 3 * i), d_dist, f);
      row[i] = key_of(f);
    }
  }
}

int64_t orc_hash_array(const uint32_t* keys, int64_t n, uint32_t* sorted_keys, uint32_t* map,
                       uint32_t* uniq, uint32_t* counts, uint32_t* first) {
  HashArray H;
  build_hash_array(keys, n, H);
  for (int64_t i = 0; i < n; ++i) {
    map[i] = H.map[i];
    sorted_keys[i] = keys[H.map[i]];
  }
  for (size_t k = 0; k < H.uniq.size(); ++k) {
    uniq[k] = H.uniq[k];
    counts[k] = H.counts[k];
    first[k] = H.first[k];
  }
  return (int64_t)H.uniq.size();
}

void orc_vote_counts(const uint32_t* scene_keys, int64_t n, const uint32_t* uniq,
                     const uint32_t* run_counts, int64_t K, uint64_t* counts) {
  for (int64_t i = 0; i < n; ++i) {
    uint32_t k = scene_keys[i];
    const uint32_t* it = std::lower_bound(uniq, uniq + K, k);
    counts[i] = (k != 0 && it != uniq + K && *it == k) ? run_counts[it - uniq] : 0;
  }
}

int orc_cluster_poses(const float* poses, const uint32_t* votes, int64_t n, float trans_thresh,
                      float rot_thresh, float out_poses[3 * 16], uint32_t out_votes[3]) {
  // transformation_clustering.cpp:62-123
  struct PV {
    const float* T;
    uint32_t votes;
  };
  std::vector<PV> pv(n);
  for (int64_t i = 0; i < n; ++i) pv[i] = PV{poses + 16 * i, votes[i]};
  // The reference sorts with std::sort (transformation_clustering.cpp:66),
  // which leaves equal vote counts in an unspecified order; a stable sort
  // keeps them in input order (for lookups: vote code order).
  std::stable_sort(pv.begin(), pv.end(), [](const PV& a, const PV& b) { return a.votes > b.votes; });
  std::vector<std::vector<PV>> clusters;
  std::vector<std::pair<size_t, unsigned int>> cluster_votes;
  for (int64_t p = 0; p < n; ++p) {
    bool found = false;
    for (size_t c = 0; c < clusters.size(); ++c) {
      if (within_bounds(pv[p].T, clusters[c].front().T, trans_thresh, rot_thresh)) {
        found = true;
        clusters[c].push_back(pv[p]);
        cluster_votes[c].second += pv[p].votes;
        break;
      }
    }
    if (!found) {
      clusters.push_back(std::vector<PV>{pv[p]});
      cluster_votes.push_back(std::pair<size_t, unsigned int>(clusters.size() - 1, pv[p].votes));
    }
  }
  std::stable_sort(cluster_votes.begin(), cluster_votes.end(),
            [](const std::pair<size_t, unsigned int>& a, const std::pair<size_t, unsigned int>& b) {
              return a.second > b.second;
            });
  int nc = (int)std::min<size_t>(clusters.size(), 3);
  for (int c = 0; c < nc; ++c) {
    const std::vector<PV>& cl = clusters[cluster_votes[c].first];
    float ta[3] = {0, 0, 0}, qa[4] = {0, 0, 0, 0};
    for (const PV& e : cl) {
      ta[0] += e.T[3];
      ta[1] += e.T[7];
      ta[2] += e.T[11];
      float R[9], q[4];
      rotation_of(e.T, R);
      mat_to_quat_xyzw(R, q);
      for (int k = 0; k < 4; ++k) qa[k] += q[k];
    }
    float sz = (float)cl.size();
    for (int k = 0; k < 3; ++k) ta[k] /= sz;
    for (int k = 0; k < 4; ++k) qa[k] /= sz;
    float qn = sqrtf(qa[0] * qa[0] + qa[1] * qa[1] + qa[2] * qa[2] + qa[3] * qa[3]);
    float x = qa[0] / qn, y = qa[1] / qn, z = qa[2] / qn, w = qa[3] / qn;
    float tx = 2 * x, ty = 2 * y, tz = 2 * z;
    float twx = tx * w, twy = ty * w, twz = tz * w;
    float txx = tx * x, txy = ty * x, txz = tz * x;
    float tyy = ty * y, tyz = tz * y, tzz = tz * z;
    float* O = out_poses + 16 * c;
    O[0] = 1 - (tyy + tzz);
    O[1] = txy - twz;
    O[2] = txz + twy;
    O[4] = txy + twz;
    O[5] = 1 - (txx + tzz);
    O[6] = tyz - twx;
    O[8] = txz - twy;
    O[9] = tyz + twx;
    O[10] = 1 - (txx + tyy);
    O[3] = ta[0];
    O[7] = ta[1];
    O[11] = ta[2];
    O[12] = 0;
    O[13] = 0;
    O[14] = 0;
    O[15] = 1;
    out_votes[c] = cluster_votes[c].second;
  }
  return nc;
}

orc_result* orc_register(const float* m_pts, const float* m_nrm, int64_t n_m, const float* s_pts,
                         const float* s_nrm, int64_t n_s, const float* model_weights,
                         const orc_params* prm) {
  orc_result* R = (orc_result*)calloc(1, sizeof(orc_result));
  if (n_m > 65536) {  // m_r is kept in 16 bits per model pair below
    R->status = -2;
    return R;
  }
  typedef std::chrono::steady_clock Clk;
  const Clk::time_point t0 = Clk::now();
  const float d = prm->d_dist;
  const uint32_t df = prm->ref_point_df ? prm->ref_point_df : 1;
#ifdef _OPENMP
  if (prm->n_threads > 0) omp_set_num_threads(prm->n_threads);
#endif
  // ---- Model::Model (model.cu:43-82): model keys + hash array ----------
  std::vector<uint32_t> mkeys((size_t)n_m * n_m);
  orc_pair_keys(m_pts, m_nrm, n_m, 1, d, mkeys.data(), prm->n_threads);
  HashArray H;
  build_hash_array(mkeys.data(), (int64_t)mkeys.size(), H);
  mkeys.clear();
  mkeys.shrink_to_fit();
  // Model frames, once per model reference point (same bits as recomputing
  // them per vote in trans_model_scene, kernel.cu:310-318).
  std::vector<float> mframe((size_t)n_m * 16);
  for (int64_t r = 0; r < n_m; ++r) {
    M4 T;
    frame(ld3(m_pts + 3 * r), ld3(m_nrm + 3 * r), T);
    memcpy(&mframe[16 * r], T, sizeof(T));
  }
  // u = m_i in the frame of m_r for every entry of the hash array, in hash
  // array order (only its y and z enter alpha, kernel.cu:338-342), and the
  // entry's m_r: the same bits trans_model_scene recomputes per vote
  // (kernel.cu:329-336), computed once per model pair.
  const size_t n_pairs = H.map.size();
  std::vector<float> u_yz(2 * n_pairs);
  std::vector<uint16_t> u_mr(n_pairs);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int64_t j = 0; j < (int64_t)n_pairs; ++j) {
    const uint32_t pair = H.map[j];
    const uint32_t mr = pair / (uint32_t)n_m, mi = pair - mr * (uint32_t)n_m;
    M4 Tm;
    memcpy(Tm, &mframe[16 * mr], sizeof(Tm));
    const F3 u = frame_apply(Tm, ld3(m_pts + 3 * mi));
    u_yz[2 * j] = u.y;
    u_yz[2 * j + 1] = u.z;
    u_mr[j] = (uint16_t)mr;
  }
  const Clk::time_point t1 = Clk::now();
  R->t_build = std::chrono::duration<double>(t1 - t0).count();
  // ---- ComputeUniqueVotes (model.cu:95-171) -----------------------------
  const int64_t sr_step = prm->sr_step > 0 ? prm->sr_step : (int64_t)df;
  const int64_t sr_lo = std::max<int64_t>(prm->sr_begin, 0);
  const int64_t sr_hi = prm->sr_end < 0 ? n_s : std::min<int64_t>(prm->sr_end, n_s);
  const int nb = 31;  // alpha bins 0..30
  std::atomic<uint32_t> gmax(0);
  std::atomic<uint64_t> gvotes(0), guniq(0);
  struct Cand {
    uint64_t code;
    uint32_t count;
  };
  std::vector<std::vector<Cand>> per_sr((size_t)std::max<int64_t>(sr_hi - sr_lo, 0));
  const float thr = prm->vote_count_threshold;
  bool scene_ok = n_s > 1 && n_m > 1;
  if (scene_ok) {
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
      std::vector<uint32_t> acc((size_t)n_m * nb);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
      for (int64_t sr = sr_lo; sr < sr_hi; ++sr) {
        if (sr % df != 0 || (sr - sr_lo) % sr_step != 0) continue;
        std::fill(acc.begin(), acc.end(), 0u);
        F3 pr = ld3(s_pts + 3 * sr), nr = ld3(s_nrm + 3 * sr);
        M4 Ts;
        frame(pr, nr, Ts);
        uint64_t nv = 0;
        for (int64_t si = 0; si < n_s; ++si) {
          if (si == sr) continue;
          float f[4];
          pair_feature(pr, nr, ld3(s_pts + 3 * si), ld3(s_nrm + 3 * si), d, f);
          int64_t run = find_run(H, key_of(f));
          if (run < 0) continue;
          F3 v = frame_apply(Ts, ld3(s_pts + 3 * si));
          uint32_t first = H.first[run], cnt = H.counts[run];
          nv += cnt;
          for (uint32_t e = first; e < first + cnt; ++e) {
            const F3 u{0.f, u_yz[2 * (size_t)e], u_yz[2 * (size_t)e + 1]};
            uint32_t bin = alpha_bin(u, v);
            acc[(size_t)u_mr[e] * nb + bin]++;
          }
        }
        uint32_t lmax = 0;
        uint64_t lu = 0;
        for (size_t c = 0; c < acc.size(); ++c) {
          if (acc[c]) {
            ++lu;
            lmax = std::max(lmax, acc[c]);
          }
        }
        uint32_t g = gmax.load();
        while (lmax > g && !gmax.compare_exchange_weak(g, lmax)) {
        }
        float floor_v = thr * (float)std::max(g, lmax);
        std::vector<Cand>& out = per_sr[sr - sr_lo];
        for (size_t c = 0; c < acc.size(); ++c) {
          uint32_t cnt = acc[c];
          if (cnt && (float)cnt > floor_v) {
            uint32_t mr = (uint32_t)(c / nb), bin = (uint32_t)(c % nb);
            out.push_back(Cand{((uint64_t)sr << 32) | ((uint64_t)mr << 6) | bin, cnt});
          }
        }
        gvotes += nv;
        guniq += lu;
      }
    }
  }
  R->t_vote = std::chrono::duration<double>(Clk::now() - t1).count();
  for (int64_t sr = sr_lo; sr < sr_hi; ++sr)
    if (sr % df == 0 && (sr - sr_lo) % sr_step == 0) R->n_refs++;
  R->n_votes = gvotes.load();
  R->n_unique = guniq.load();
  R->max_count = gmax.load();
  R->min_votecount = thr * (float)R->max_count;
  std::vector<Cand> kept;
  for (auto& v : per_sr)
    for (auto& c : v)
      if ((float)c.count > R->min_votecount) kept.push_back(c);
  // codes are already ascending; order by count descending, ties by code
  std::stable_sort(kept.begin(), kept.end(),
                   [](const Cand& a, const Cand& b) { return a.count > b.count; });
  const size_t U = kept.size();
  R->n_kept = U;
  if (U == 0) {
    R->status = 1;
    return R;
  }
  R->codes = (uint64_t*)malloc(U * 8);
  R->counts = (uint32_t*)malloc(U * 4);
  R->weighted = (float*)calloc(U, 4);
  R->transforms = (float*)calloc(U * 16, 4);
  R->trans = (float*)calloc(U * 3, 4);
  R->quats = (float*)calloc(U * 4, 4);
  R->cell_keys = (uint32_t*)calloc(U, 4);
  R->scores = (float*)calloc(U, 4);
  for (size_t i = 0; i < U; ++i) {
    R->codes[i] = kept[i].code;
    R->counts[i] = kept[i].count;
  }
  if (prm->votes_only) return R;
  // Every per-vote kernel returns early for count <= 1 (kernel.cu:609 etc.),
  // so a single kept vote leaves all derived arrays at zero.
  const bool run_kernels = U > 1;
  // ---- ComputeTransformations (model.cu:191-200, kernel.cu:605-645) ------
  if (run_kernels) {
    for (size_t i = 0; i < U; ++i) {
      uint64_t v = R->codes[i];
      uint32_t sr = (uint32_t)(v >> 32), mc = (uint32_t)(v & 0xffffffffu);
      uint32_t mr = mc >> 6, ai = mc & 63u;
      if (sr == 0 && mr == 0 && ai == 0) continue;
      orc_vote_pose(ai, m_pts + 3 * mr, m_nrm + 3 * mr, s_pts + 3 * sr, s_nrm + 3 * sr,
                    R->transforms + 16 * i);
    }
    // ComputeWeightedVoteCounts (model.cu:173-189, kernel.cu:766-782)
    for (size_t i = 0; i < U; ++i) {
      uint32_t mr = ((uint32_t)(R->codes[i] & 0xffffffffu)) >> 6;
      float w = model_weights ? model_weights[mr] : 1.0f;
      R->weighted[i] = w * (float)R->counts[i];
    }
  }
  if (prm->cpu_clustering) {
    // ClusterTransformationsCPU (model.cu:246-266)
    R->n_clusters = orc_cluster_poses(R->transforms, R->counts, (int64_t)U, d, kD, R->cpu_poses,
                                      R->cpu_votes);
    memcpy(R->pose, R->cpu_poses, 16 * sizeof(float));
    return R;
  }
  // ---- ClusterTransformations (model.cu:202-244) -------------------------
  std::vector<uint32_t> adj(U * 27, 0u);
  if (run_kernels) {
    for (size_t i = 0; i < U; ++i) {
      const float* T = R->transforms + 16 * i;
      R->trans[3 * i + 0] = T[3];
      R->trans[3 * i + 1] = T[7];
      R->trans[3 * i + 2] = T[11];
      quat_of(T, R->quats + 4 * i);
      R->cell_keys[i] = cell_keys(R->trans + 3 * i, d, &adj[27 * i]);
    }
  }
  HashArray P;
  build_hash_array(R->cell_keys, (int64_t)U, P);
  if (run_kernels) {
    std::vector<float> t0(R->trans, R->trans + 3 * U);  // snapshot (see header)
    const float rot_sq = kRotThresh * kRotThresh;
    for (size_t i = 0; i < U; ++i) {
      F3 t{t0[3 * i], t0[3 * i + 1], t0[3 * i + 2]};
      F4 q{R->quats[4 * i], R->quats[4 * i + 1], R->quats[4 * i + 2], R->quats[4 * i + 3]};
      float c = 1;
      F3 to = t;
      for (int b = 0; b < 27; ++b) {
        int64_t run = find_run(P, adj[27 * i + b]);
        if (run < 0) continue;
        for (uint32_t e = 0; e < P.counts[run]; ++e) {
          uint32_t j = P.map[P.first[run] + e];
          float w = R->weighted[j];
          F4 qj{R->quats[4 * j], R->quats[4 * j + 1], R->quats[4 * j + 2], R->quats[4 * j + 3]};
          float qd = fabsf(8 * (1 - dot4(q, qj)));
          if (qd < rot_sq) {
            F3 tj{t0[3 * j], t0[3 * j + 1], t0[3 * j + 2]};
            if (!prm->use_l1_norm) {
              F3 df3{t.x - tj.x, t.y - tj.y, t.z - tj.z};
              if (!(norm3(df3) < d)) continue;
            }
            if (prm->use_averaged_clusters) {
              F3 a{c * to.x, c * to.y, c * to.z};
              F3 b2{w * tj.x, w * tj.y, w * tj.z};
              F3 s{a.x + b2.x, a.y + b2.y, a.z + b2.z};
              float inv = 1 / (c + w);
              to = F3{inv * s.x, inv * s.y, inv * s.z};
            }
            c += w;
          }
        }
      }
      R->scores[i] = c;
      R->trans[3 * i] = to.x;
      R->trans[3 * i + 1] = to.y;
      R->trans[3 * i + 2] = to.z;
    }
  }
  size_t best = 0;
  for (size_t i = 1; i < U; ++i)
    if (R->scores[i] > R->scores[best]) best = i;
  R->max_idx = best;
  // ppf.cu:78-93
  memcpy(R->pose, R->transforms + 16 * best, 16 * sizeof(float));
  R->pose[3] = R->trans[3 * best];
  R->pose[7] = R->trans[3 * best + 1];
  R->pose[11] = R->trans[3 * best + 2];
  return R;
}

void orc_result_free(orc_result* r) {
  if (!r) return;
  free(r->codes);
  free(r->counts);
  free(r->weighted);
  free(r->transforms);
  free(r->trans);
  free(r->quats);
  free(r->cell_keys);
  free(r->scores);
  free(r);
}

}  // extern "C"

/* ---- driver preprocessing ---- */

int orc_cloud_extent(const float* xyz, int64_t n, float lo[3], float hi[3]) {
  int any = 0;
  for (int64_t i = 0; i < n; ++i) {
    const float* p = xyz + 3 * i;
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) continue;
    for (int k = 0; k < 3; ++k) {
      if (!any || p[k] < lo[k]) lo[k] = p[k];
      if (!any || p[k] > hi[k]) hi[k] = p[k];
    }
    any = 1;
  }
  return any;
}

/* pcl::VoxelGrid<PointT>::applyFilter (PCL 1.8) as the alignment driver
 * calls it (src/alignment.cpp:79-87): min/max bounding box in leaf units,
 * linear index per finite point, sort by index, mean of each voxel. */
int64_t orc_voxel_downsample(const float* xyz, const float* nxyz, int64_t n, float leaf, float* out_xyz,
                             float* out_nxyz) {
  float lo[3], hi[3];
  if (!orc_cloud_extent(xyz, n, lo, hi)) return 0;
  const float inv = 1.0f / leaf;
  long long d[3];
  for (int k = 0; k < 3; ++k) d[k] = (long long)((hi[k] - lo[k]) * inv) + 1;
  if (d[0] * d[1] * d[2] > (long long)INT32_MAX) {
    std::memcpy(out_xyz, xyz, (size_t)n * 12);
    std::memcpy(out_nxyz, nxyz, (size_t)n * 12);
    return n;
  }
  int min_b[3], max_b[3];
  for (int k = 0; k < 3; ++k) {
    min_b[k] = (int)std::floor(lo[k] * inv);
    max_b[k] = (int)std::floor(hi[k] * inv);
  }
  const long long dx = max_b[0] - min_b[0] + 1, dy = max_b[1] - min_b[1] + 1;
  std::vector<std::pair<uint32_t, int64_t>> iv;
  iv.reserve((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const float* p = xyz + 3 * i;
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) continue;
    int ijk[3];
    for (int k = 0; k < 3; ++k) ijk[k] = (int)(std::floor(p[k] * inv) - (float)min_b[k]);
    iv.push_back({(uint32_t)(ijk[0] + ijk[1] * (int)dx + ijk[2] * (int)(dx * dy)), i});
  }
  std::stable_sort(iv.begin(), iv.end(),
                   [](const std::pair<uint32_t, int64_t>& a, const std::pair<uint32_t, int64_t>& b) {
                     return a.first < b.first;
                   });
  int64_t K = 0;
  for (size_t a = 0; a < iv.size();) {
    size_t b = a;
    float s[6] = {0, 0, 0, 0, 0, 0};
    while (b < iv.size() && iv[b].first == iv[a].first) {
      const int64_t p = iv[b].second;
      for (int k = 0; k < 3; ++k) {
        s[k] += xyz[3 * p + k];
        s[3 + k] += nxyz[3 * p + k];
      }
      ++b;
    }
    const float c = (float)(b - a);
    for (int k = 0; k < 3; ++k) {
      out_xyz[3 * K + k] = s[k] / c;
      out_nxyz[3 * K + k] = s[3 + k] / c;
    }
    ++K;
    a = b;
  }
  return K;
}
