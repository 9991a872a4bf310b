/*
 * ppf_b200.hpp -- C++ facade of the C ABI (ppf_b200.h) with the reference's
 * class and function names: ppf::Scene, ppf::Model and ppf::ppf_registration
 * (include/scene.h:10-16, include/model.h:14-35, include/ppf.h:9-15 of
 * nicolasavru/ppf-registration-spatial-hashing).  PCL is not needed: a cloud
 * is a std::vector of ppf::PointNormal (the x, y, z and normal_x, normal_y,
 * normal_z fields of pcl::PointNormal), and poses are row-major 4x4 float
 * arrays in place of Eigen::Matrix4f.  Header-only; link with -lppf_b200.
 *
 * Differences a caller sees: failures throw ppf::Error (status and message)
 * instead of exiting the process, and objects take an optional
 * ppf::Context (device + stream); without one they share a default context
 * on device 0.  Nothing here resets the device.
 */
#ifndef PPF_B200_HPP
#define PPF_B200_HPP

#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "ppf_b200.h"

namespace ppf {

struct PointNormal {
  float x, y, z;
  float normal_x, normal_y, normal_z;
};
typedef std::vector<PointNormal> PointCloud;
typedef std::array<float, 16> Matrix4f;  // row-major

class Error : public std::runtime_error {
 public:
  Error(ppf_status s, const std::string& what) : std::runtime_error(what), status(s) {}
  ppf_status status;
};

inline void check(ppf_status s) {
  if (s != PPF_OK) throw Error(s, ppf_last_error());
}

namespace detail {
// n x 3 point and normal arrays of a cloud (the C ABI's layout).
struct Soa {
  std::vector<float> xyz, nxyz;
  explicit Soa(const PointCloud& c) : xyz(3 * c.size()), nxyz(3 * c.size()) {
    for (size_t i = 0; i < c.size(); ++i) {
      xyz[3 * i] = c[i].x;
      xyz[3 * i + 1] = c[i].y;
      xyz[3 * i + 2] = c[i].z;
      nxyz[3 * i] = c[i].normal_x;
      nxyz[3 * i + 1] = c[i].normal_y;
      nxyz[3 * i + 2] = c[i].normal_z;
    }
  }
};
}  // namespace detail

class Context {
 public:
  explicit Context(int device = 0) { check(ppf_context_create(device, &h_)); }
  ~Context() { ppf_context_destroy(h_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  ppf_context_t handle() const { return h_; }
  void synchronize() const { check(ppf_context_synchronize(h_)); }

  static Context& default_context() {
    static Context c(0);
    return c;
  }

 private:
  ppf_context_t h_ = nullptr;
};

// Scene(cloud, d_dist, ref_point_downsample_factor) (include/scene.h:15-16).
class Scene {
 public:
  Scene(const PointCloud* cloud, float d_dist, unsigned int ref_point_downsample_factor = 1,
        Context* ctx = nullptr)
      : n_(cloud->size()) {
    detail::Soa s(*cloud);
    check(ppf_scene_create((ctx ? *ctx : Context::default_context()).handle(), s.xyz.data(), s.nxyz.data(),
                           cloud->size(), d_dist, ref_point_downsample_factor, &h_));
  }
  ~Scene() { ppf_scene_destroy(h_); }
  Scene(const Scene&) = delete;
  Scene& operator=(const Scene&) = delete;
  int numPoints() const { return (int)n_; }
  ppf_scene_t handle() const { return h_; }

 private:
  ppf_scene_t h_ = nullptr;
  size_t n_;
};

// Model(cloud, d_dist, vote_count_threshold, cpu_clustering, use_l1_norm,
// use_averaged_clusters) (include/model.h:17-19) with ppf_lookup and the
// inspection members of include/model.h:61-113 as getters.
class Model {
 public:
  Model(const PointCloud* cloud, float d_dist, float vote_count_threshold, bool cpu_clustering,
        bool use_l1_norm, bool use_averaged_clusters, Context* ctx = nullptr) {
    detail::Soa s(*cloud);
    check(ppf_model_create((ctx ? *ctx : Context::default_context()).handle(), s.xyz.data(), s.nxyz.data(),
                           cloud->size(), d_dist, vote_count_threshold, cpu_clustering, use_l1_norm,
                           use_averaged_clusters, &h_));
  }
  ~Model() { ppf_model_destroy(h_); }
  Model(const Model&) = delete;
  Model& operator=(const Model&) = delete;

  // Model::SetModelPointVoteWeights (src/cuda/model.cu:91-93)
  void SetModelPointVoteWeights(const std::vector<float>& w) {
    check(ppf_model_set_point_vote_weights(h_, w.data(), w.size()));
  }
  // Model::ppf_lookup (src/cuda/model.cu:269-306) and the pose of
  // ppf_registration (src/cuda/ppf.cu:74-93); PPF_ERR_NO_VOTES leaves a zero
  // pose and returns false.
  bool ppf_lookup(Scene* scene) {
    ppf_status s = ppf_model_lookup(h_, scene->handle(), pose_.data(), &stats_);
    if (s == PPF_ERR_NO_VOTES) return false;
    check(s);
    return true;
  }
  const Matrix4f& pose() const { return pose_; }
  const ppf_stats& stats() const { return stats_; }
  uint64_t max_idx() const { return stats_.max_idx; }
  // votes / voteCounts after the threshold (src/cuda/model.cu:155-170)
  void getVotes(std::vector<uint64_t>* votes, std::vector<uint32_t>* counts) const {
    uint64_t n = 0;
    check(ppf_model_get_votes(h_, nullptr, nullptr, 0, &n));
    votes->resize(n);
    counts->resize(n);
    check(ppf_model_get_votes(h_, votes->data(), counts->data(), n, &n));
  }
  // transformations (src/cuda/model.cu:191-200), U x 16 row-major
  std::vector<float> getTransformations() const {
    uint64_t n = 0;
    check(ppf_model_get_transformations(h_, nullptr, 0, &n));
    std::vector<float> T(16 * n);
    check(ppf_model_get_transformations(h_, T.data(), n, &n));
    return T;
  }
  ppf_model_t handle() const { return h_; }

 private:
  ppf_model_t h_ = nullptr;
  Matrix4f pose_{};
  ppf_stats stats_{};
};

// ppf_registration (include/ppf.h:9-15, src/cuda/ppf.cu:29-106): result
// [scene][model].  model_weights is accepted and ignored, as in the
// reference (src/cuda/ppf.cu:35).  Pairs with no votes keep a zero pose.
inline std::vector<std::vector<Matrix4f>> ppf_registration(
    const std::vector<const PointCloud*>& scene_clouds, const std::vector<const PointCloud*>& model_clouds,
    const std::vector<float>& model_d_dists, unsigned int ref_point_downsample_factor,
    float vote_count_threshold, bool cpu_clustering, bool use_l1_norm, bool use_averaged_clusters, int devUse,
    float* model_weights, Context* ctx = nullptr) {
  if (model_d_dists.size() != model_clouds.size())
    throw Error(PPF_ERR_INVALID_ARGUMENT, "one d_dist per model is required");
  std::vector<detail::Soa> scenes, models;
  std::vector<const float*> sx, sn, mx, mn;
  std::vector<uint64_t> sc, mc;
  for (const PointCloud* c : scene_clouds) scenes.emplace_back(*c);
  for (const PointCloud* c : model_clouds) models.emplace_back(*c);
  for (size_t i = 0; i < scenes.size(); ++i) {
    sx.push_back(scenes[i].xyz.data());
    sn.push_back(scenes[i].nxyz.data());
    sc.push_back(scene_clouds[i]->size());
  }
  for (size_t j = 0; j < models.size(); ++j) {
    mx.push_back(models[j].xyz.data());
    mn.push_back(models[j].nxyz.data());
    mc.push_back(model_clouds[j]->size());
  }
  std::vector<float> poses(16 * scenes.size() * models.size());
  ppf_status s = ::ppf_registration(ctx ? ctx->handle() : nullptr, scenes.size(), sx.data(), sn.data(), sc.data(),
                                    models.size(), mx.data(), mn.data(), mc.data(), model_d_dists.data(),
                                    ref_point_downsample_factor, vote_count_threshold, cpu_clustering,
                                    use_l1_norm, use_averaged_clusters, devUse, model_weights, poses.data(),
                                    nullptr);
  if (s != PPF_ERR_NO_VOTES) check(s);
  std::vector<std::vector<Matrix4f>> out(scenes.size(), std::vector<Matrix4f>(models.size()));
  for (size_t i = 0; i < scenes.size(); ++i)
    for (size_t j = 0; j < models.size(); ++j)
      for (int k = 0; k < 16; ++k) out[i][j][k] = poses[16 * (i * models.size() + j) + k];
  return out;
}

// pcl::io::loadPLYFile<PointNormal> (src/alignment.cpp:212,241).
inline PointCloud load_ply(const std::string& path) {
  uint64_t n = 0;
  check(ppf_ply_read(path.c_str(), nullptr, nullptr, 0, &n));
  std::vector<float> xyz(3 * n), nxyz(3 * n);
  check(ppf_ply_read(path.c_str(), xyz.data(), nxyz.data(), n, &n));
  PointCloud c(n);
  for (uint64_t i = 0; i < n; ++i)
    c[i] = PointNormal{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], nxyz[3 * i], nxyz[3 * i + 1], nxyz[3 * i + 2]};
  return c;
}

}  // namespace ppf

#endif /* PPF_B200_HPP */
