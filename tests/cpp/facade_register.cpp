// Registers a scene PLY against a model PLY through the C++ facade
// (include/ppf_b200.hpp) the way the reference's driver calls
// ppf_registration (src/alignment.cpp:290-298), then once more through
// ppf::Model / ppf::Scene, and prints both poses (16 floats each, row-major,
// as hex bit patterns so the caller can compare them exactly).
//   facade_register model.ply scene.ply d_dist ref_point_df threshold
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ppf_b200.hpp"

static void print_pose(const char* tag, const float* p) {
  std::printf("%s", tag);
  for (int k = 0; k < 16; ++k) {
    unsigned u;
    std::memcpy(&u, &p[k], 4);
    std::printf(" %08x", u);
  }
  std::printf("\n");
}

int main(int argc, char** argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s model.ply scene.ply d_dist ref_point_df threshold\n", argv[0]);
    return 2;
  }
  try {
    ppf::PointCloud model = ppf::load_ply(argv[1]);
    ppf::PointCloud scene = ppf::load_ply(argv[2]);
    const float d = std::strtof(argv[3], nullptr);
    const unsigned df = (unsigned)std::strtoul(argv[4], nullptr, 10);
    const float thr = std::strtof(argv[5], nullptr);
    auto poses = ppf::ppf_registration({&scene}, {&model}, {d}, df, thr, false, false, false, 0, nullptr);
    print_pose("registration", poses[0][0].data());
    ppf::Context ctx(0);
    ppf::Model m(&model, d, thr, false, false, false, &ctx);
    ppf::Scene s(&scene, d, df, &ctx);
    m.ppf_lookup(&s);
    print_pose("lookup", m.pose().data());
    std::printf("votes %llu kept %llu points %d\n", (unsigned long long)m.stats().n_votes,
                (unsigned long long)m.stats().n_kept, s.numPoints());
  } catch (const ppf::Error& e) {
    std::fprintf(stderr, "ppf error %d: %s\n", (int)e.status, e.what());
    return 1;
  }
  return 0;
}
