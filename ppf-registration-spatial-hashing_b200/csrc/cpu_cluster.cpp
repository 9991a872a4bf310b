// Greedy pose clustering on the host: the reference's cpu_clustering path
// (Model::ClusterTransformationsCPU, src/cuda/model.cu:246-266, and
// clusterPoses / posesWithinErrorBounds,
// src/transformation_clustering.cpp:62-137).  The reference does this with
// Eigen; the rotation arithmetic Eigen performs (quaternion from a rotation
// matrix by the trace / largest-diagonal method, axis-angle angle
// 2*atan2(|v|, |w|), quaternion to matrix) is written out here in float.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <utility>
#include <vector>

namespace ppf {
namespace {

// Rotation block of a row-major 4x4 pose; an all-zero block (a vote whose
// pose was never computed) is taken as the identity, the polar factor Eigen
// returns for it.
void rotation_block(const float* T, float R[9]) {
  bool zero = true;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      R[3 * i + j] = T[4 * i + j];
      zero = zero && R[3 * i + j] == 0.f;
    }
  if (zero)
    for (int k = 0; k < 9; ++k) R[k] = (k % 4 == 0) ? 1.f : 0.f;
}

// Quaternion (x, y, z, w) of a rotation matrix.
void quat_xyzw(const float* m, float q[4]) {
  float tr = m[0] + m[4] + m[8];
  if (tr > 0.f) {
    float s = std::sqrt(tr + 1.0f);
    q[3] = 0.5f * s;
    s = 0.5f / s;
    q[0] = (m[7] - m[5]) * s;
    q[1] = (m[2] - m[6]) * s;
    q[2] = (m[3] - m[1]) * s;
    return;
  }
  int i = 0;
  if (m[4] > m[0]) i = 1;
  if (m[8] > m[4 * i]) i = 2;
  const int j = (i + 1) % 3, k = (j + 1) % 3;
  float s = std::sqrt(m[4 * i] - m[4 * j] - m[4 * k] + 1.0f);
  q[i] = 0.5f * s;
  s = 0.5f / s;
  q[3] = (m[3 * k + j] - m[3 * j + k]) * s;
  q[j] = (m[3 * j + i] + m[3 * i + j]) * s;
  q[k] = (m[3 * k + i] + m[3 * i + k]) * s;
}

bool close_enough(const float* A, const float* B, float trans_thresh, float rot_thresh) {
  float dx = A[3] - B[3], dy = A[7] - B[7], dz = A[11] - B[11];
  float dist = std::sqrt(dx * dx + dy * dy + dz * dz);
  float Ra[9], Rb[9], M[9];
  rotation_block(A, Ra);
  rotation_block(B, Rb);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float s = 0.f;
      for (int k = 0; k < 3; ++k) s += Ra[3 * k + i] * Rb[3 * k + j];
      M[3 * i + j] = s;
    }
  float q[4];
  quat_xyzw(M, q);
  float nv = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  float angle = nv != 0.f ? 2.f * std::atan2(nv, std::fabs(q[3])) : 0.f;
  return dist < trans_thresh && std::fabs(angle) < rot_thresh;
}

}  // namespace

int cluster_poses_cpu(const float* poses, const uint32_t* votes, size_t n, float trans_thresh,
                      float rot_thresh, float out_poses[3 * 16], uint32_t out_votes[3]) {
  struct Item {
    const float* T;
    uint32_t votes;
  };
  std::vector<Item> items(n);
  for (size_t i = 0; i < n; ++i) items[i] = Item{poses + 16 * i, votes[i]};
  // The reference sorts with std::sort (src/transformation_clustering.cpp:66),
  // which leaves equal vote counts in an unspecified order; the stable sort
  // keeps them in input order, the vote code order of the kept votes.
  std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.votes > b.votes; });
  std::vector<std::vector<Item>> clusters;
  std::vector<std::pair<size_t, unsigned int>> totals;
  for (const Item& it : items) {
    bool placed = false;
    for (size_t c = 0; c < clusters.size() && !placed; ++c) {
      if (close_enough(it.T, clusters[c].front().T, trans_thresh, rot_thresh)) {
        clusters[c].push_back(it);
        totals[c].second += it.votes;
        placed = true;
      }
    }
    if (!placed) {
      clusters.push_back(std::vector<Item>(1, it));
      totals.emplace_back(clusters.size() - 1, it.votes);
    }
  }
  std::stable_sort(totals.begin(), totals.end(),
            [](const std::pair<size_t, unsigned int>& a, const std::pair<size_t, unsigned int>& b) {
              return a.second > b.second;
            });
  const int nc = (int)std::min<size_t>(clusters.size(), 3);
  for (int c = 0; c < nc; ++c) {
    const std::vector<Item>& cl = clusters[totals[c].first];
    float t[3] = {0.f, 0.f, 0.f}, qs[4] = {0.f, 0.f, 0.f, 0.f};
    for (const Item& it : cl) {
      t[0] += it.T[3];
      t[1] += it.T[7];
      t[2] += it.T[11];
      float R[9], q[4];
      rotation_block(it.T, R);
      quat_xyzw(R, q);
      for (int k = 0; k < 4; ++k) qs[k] += q[k];
    }
    const float sz = (float)cl.size();
    for (int k = 0; k < 3; ++k) t[k] /= sz;
    for (int k = 0; k < 4; ++k) qs[k] /= sz;
    float qn = std::sqrt(qs[0] * qs[0] + qs[1] * qs[1] + qs[2] * qs[2] + qs[3] * qs[3]);
    float x = qs[0] / qn, y = qs[1] / qn, z = qs[2] / qn, w = qs[3] / qn;
    float tx = 2 * x, ty = 2 * y, tz = 2 * z;
    float* O = out_poses + 16 * c;
    O[0] = 1 - (ty * y + tz * z);
    O[1] = ty * x - tz * w;
    O[2] = tz * x + ty * w;
    O[3] = t[0];
    O[4] = ty * x + tz * w;
    O[5] = 1 - (tx * x + tz * z);
    O[6] = tz * y - tx * w;
    O[7] = t[1];
    O[8] = tz * x - ty * w;
    O[9] = tz * y + tx * w;
    O[10] = 1 - (tx * x + ty * y);
    O[11] = t[2];
    O[12] = 0;
    O[13] = 0;
    O[14] = 0;
    O[15] = 1;
    out_votes[c] = totals[c].second;
  }
  return nc;
}

}  // namespace ppf
