// PLY clouds with normals, as the alignment driver loads them with
// pcl::io::loadPLYFile<pcl::PointNormal> (src/alignment.cpp:212,241): the
// "vertex" element's x, y, z and nx, ny, nz (or normal_x, normal_y,
// normal_z) properties, of any scalar type, in ascii, binary_little_endian or
// binary_big_endian files.  Other elements (faces and the like) are skipped.
// Writing produces binary_little_endian float x y z nx ny nz.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ppf_b200.h"

namespace {

enum class Fmt { Ascii, Le, Be };

struct Prop {
  std::string name;
  int type = 0;        // bytes of a scalar (1, 2, 4, 8); 0: list
  bool is_float = false, is_signed = false;
  int count_type = 0;  // list: bytes of the count
  int item_type = 0;   // list: bytes of an item
};

struct Element {
  std::string name;
  uint64_t count = 0;
  std::vector<Prop> props;
};

bool scalar_type(const std::string& t, int& bytes, bool& fl, bool& sg) {
  static const struct { const char* n; int b; bool f, s; } tbl[] = {
      {"char", 1, false, true},    {"int8", 1, false, true},     {"uchar", 1, false, false},
      {"uint8", 1, false, false},  {"short", 2, false, true},    {"int16", 2, false, true},
      {"ushort", 2, false, false}, {"uint16", 2, false, false},  {"int", 4, false, true},
      {"int32", 4, false, true},   {"uint", 4, false, false},    {"uint32", 4, false, false},
      {"float", 4, true, true},    {"float32", 4, true, true},   {"double", 8, true, true},
      {"float64", 8, true, true}};
  for (const auto& e : tbl)
    if (t == e.n) {
      bytes = e.b;
      fl = e.f;
      sg = e.s;
      return true;
    }
  return false;
}

struct Reader {
  std::ifstream in;
  Fmt fmt = Fmt::Ascii;
  std::vector<Element> elems;
  std::string err;

  bool header(const char* path) {
    in.open(path, std::ios::binary);
    if (!in) return fail(std::string("cannot open ") + path);
    std::string line;
    if (!std::getline(in, line) || line.compare(0, 3, "ply") != 0) return fail("not a PLY file");
    while (std::getline(in, line)) {
      if (!line.empty() && line.back() == '\r') line.pop_back();
      std::istringstream ss(line);
      std::string kw;
      ss >> kw;
      if (kw == "format") {
        std::string f;
        ss >> f;
        if (f == "ascii") fmt = Fmt::Ascii;
        else if (f == "binary_little_endian") fmt = Fmt::Le;
        else if (f == "binary_big_endian") fmt = Fmt::Be;
        else return fail("unknown PLY format " + f);
      } else if (kw == "element") {
        Element e;
        ss >> e.name >> e.count;
        elems.push_back(e);
      } else if (kw == "property") {
        if (elems.empty()) return fail("property before any element");
        Prop p;
        std::string t;
        ss >> t;
        if (t == "list") {
          std::string ct, it;
          ss >> ct >> it >> p.name;
          bool f, s;
          if (!scalar_type(ct, p.count_type, f, s) || !scalar_type(it, p.item_type, f, s))
            return fail("unknown list type in PLY header");
        } else {
          ss >> p.name;
          if (!scalar_type(t, p.type, p.is_float, p.is_signed)) return fail("unknown property type " + t);
        }
        elems.back().props.push_back(p);
      } else if (kw == "end_header") {
        return true;
      }
    }
    return fail("PLY header without end_header");
  }

  bool fail(const std::string& m) {
    err = m;
    return false;
  }

  // one binary scalar of `bytes` as double
  bool read_bin(int bytes, bool fl, bool sg, double& v) {
    unsigned char b[8];
    if (!in.read(reinterpret_cast<char*>(b), bytes)) return false;
    if (fmt == Fmt::Be)
      for (int i = 0; i < bytes / 2; ++i) std::swap(b[i], b[bytes - 1 - i]);
    if (fl) {
      if (bytes == 4) {
        float f;
        std::memcpy(&f, b, 4);
        v = f;
      } else {
        std::memcpy(&v, b, 8);
      }
    } else {
      uint64_t u = 0;
      std::memcpy(&u, b, bytes);
      if (sg && bytes < 8 && (u >> (8 * bytes - 1)) & 1) u |= ~uint64_t(0) << (8 * bytes);
      v = sg ? (double)(int64_t)u : (double)u;
    }
    return true;
  }
};

int find(const Element& e, const char* a, const char* b) {
  for (size_t i = 0; i < e.props.size(); ++i)
    if (e.props[i].name == a || (b && e.props[i].name == b)) return (int)i;
  return -1;
}

}  // namespace

namespace ppf {

ppf_status ply_read(const char* path, float* xyz, float* nxyz, uint64_t cap, uint64_t* n_out, std::string* err) {
  auto error = [&](const std::string& m) {
    if (err) *err = m;
    return PPF_ERR_INVALID_ARGUMENT;
  };
  if (!path || !n_out) return error("null path or count");
  Reader r;
  if (!r.header(path)) return error(r.err);
  int vi = -1;
  for (size_t i = 0; i < r.elems.size(); ++i)
    if (r.elems[i].name == "vertex") vi = (int)i;
  if (vi < 0) return error("PLY file without a vertex element");
  const Element& ve = r.elems[vi];
  const int col[6] = {find(ve, "x", nullptr),        find(ve, "y", nullptr),        find(ve, "z", nullptr),
                      find(ve, "nx", "normal_x"), find(ve, "ny", "normal_y"), find(ve, "nz", "normal_z")};
  for (int k = 0; k < 3; ++k)
    if (col[k] < 0) return error("PLY vertex element without x, y and z");
  for (int k = 3; k < 6; ++k)
    if (col[k] < 0) return error("PLY vertex element without normals (nx, ny, nz)");
  *n_out = ve.count;
  if (cap == 0 && !xyz && !nxyz) return PPF_OK;  // size query
  if (cap < ve.count) return error("output capacity below the vertex count");
  if (!xyz || !nxyz) return error("null output arrays");
  std::vector<double> vals;
  for (size_t ei = 0; ei < r.elems.size(); ++ei) {
    const Element& e = r.elems[ei];
    const bool is_v = (int)ei == vi;
    for (uint64_t row = 0; row < e.count; ++row) {
      vals.assign(e.props.size(), 0.0);
      if (r.fmt == Fmt::Ascii) {
        std::string line;
        do {
          if (!std::getline(r.in, line)) return error("PLY file ends early");
        } while (line.find_first_not_of(" \t\r") == std::string::npos);
        std::istringstream ss(line);
        for (size_t p = 0; p < e.props.size(); ++p) {
          if (e.props[p].type == 0) {
            double c;
            ss >> c;
            for (uint64_t k = 0; k < (uint64_t)c; ++k) {
              double d;
              ss >> d;
            }
          } else if (!(ss >> vals[p])) {
            return error("malformed PLY ascii row");
          }
        }
      } else {
        for (size_t p = 0; p < e.props.size(); ++p) {
          const Prop& pr = e.props[p];
          if (pr.type == 0) {
            double c;
            if (!r.read_bin(pr.count_type, false, false, c)) return error("PLY file ends early");
            r.in.seekg((std::streamoff)((uint64_t)c * pr.item_type), std::ios::cur);
          } else if (!r.read_bin(pr.type, pr.is_float, pr.is_signed, vals[p])) {
            return error("PLY file ends early");
          }
        }
      }
      if (is_v)
        for (int k = 0; k < 3; ++k) {
          xyz[3 * row + k] = (float)vals[col[k]];
          nxyz[3 * row + k] = (float)vals[col[3 + k]];
        }
    }
    if (is_v) break;  // elements after the vertices are not needed
  }
  return PPF_OK;
}

ppf_status ply_write(const char* path, const float* xyz, const float* nxyz, uint64_t n) {
  if (!path || (n && (!xyz || !nxyz))) return PPF_ERR_INVALID_ARGUMENT;
  std::ofstream out(path, std::ios::binary);
  if (!out) return PPF_ERR_INVALID_ARGUMENT;
  out << "ply\nformat binary_little_endian 1.0\nelement vertex " << n
      << "\nproperty float x\nproperty float y\nproperty float z\nproperty float nx\nproperty float ny\n"
         "property float nz\nend_header\n";
  const uint16_t probe = 1;
  const bool little = *reinterpret_cast<const uint8_t*>(&probe) == 1;
  for (uint64_t i = 0; i < n; ++i) {
    float row[6] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], nxyz[3 * i], nxyz[3 * i + 1], nxyz[3 * i + 2]};
    if (!little)
      for (float& f : row) {
        unsigned char b[4];
        std::memcpy(b, &f, 4);
        std::swap(b[0], b[3]);
        std::swap(b[1], b[2]);
        std::memcpy(&f, b, 4);
      }
    out.write(reinterpret_cast<const char*>(row), sizeof(row));
  }
  return out ? PPF_OK : PPF_ERR_INVALID_ARGUMENT;
}

}  // namespace ppf
