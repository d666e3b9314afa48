// OpenVDB file export of the velocity field (host only, no OpenVDB needed).
//
// The reference's VDB export (src/main.cpp:1767-1790) reads velocity_image
// back as rgba16f, converts each half to float (half_to_float, :320-337) and
// calls gpusims::vdb::writeVec3Grid (common/common-cpp/src/vdb_writer.cpp:
// 96-141) for vdb_export/velocity_%06u.vdb: a Vec3SGrid named "velocity",
// grid class staggered, a linear transform of voxel size 1, every voxel of
// the Nx x Ny x Nz box set through an accessor (so every voxel is active and
// stored in a leaf, zeros included; no tiles).  That writer needs OpenVDB;
// this one writes the same grid in the OpenVDB file layout directly.
//
// File layout written (format version 224, little-endian):
//   header   int64 magic 0x56444220, uint32 file version, uint32 library
//            major / minor, uint8 has-grid-offsets = 1, 36-char UUID
//   file metadata: int32 count (0)
//   int32 grid count (1)
//   grid     name, type "Tree_vec3s_5_4_3", instance parent "" (uint32
//            length-prefixed strings); int64 grid / block / end positions;
//            uint32 compression flags (0: raw values); grid metadata (count,
//            then name, type name, uint32 size, value, sorted by name);
//            transform: map type name and its Vec3d fields;
//            topology: int32 buffer count 1, root (background Vec3f, uint32
//            tile count 0, uint32 child count, per child its int32[3] origin
//            and the 32^3 internal node), internal nodes (child mask, value
//            mask, one metadata byte 6 = all values follow, then every value
//            of the node, then the children in index order), leaf topology =
//            its 8^3 value mask;
//            buffers: per leaf in the same order, value mask, metadata byte
//            6 and its 512 Vec3f values.
//   Node indices put x slowest and z fastest: offset = (x' << 2L) | (y' << L)
//   | z' in each node of log2 size L.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "lbm_internal.h"

namespace {

thread_local std::string g_vdb_err = "no error";

int vdb_fail(int code, const std::string& msg) {
  g_vdb_err = msg;
  return code;
}

// Node sizes of the standard 5-4-3 tree.
constexpr int kLeafLog2 = 3, kInt1Log2 = 4, kInt2Log2 = 5;
constexpr int kLeafDim = 1 << kLeafLog2;                       // 8 voxels
constexpr int kInt1Span = 1 << (kInt1Log2 + kLeafLog2);        // 128 voxels
constexpr int kInt2Span = 1 << (kInt2Log2 + kInt1Log2 + kLeafLog2);  // 4096 voxels
constexpr uint32_t kFileVersion = 224;
constexpr uint32_t kLibMajor = 9, kLibMinor = 0;  // the OpenVDB release line that writes version 224
constexpr uint8_t kAllValues = 6;                 // compressed-values metadata: no mask, all values

class Writer {
 public:
  explicit Writer(FILE* f) : f_(f) {}
  bool ok() const { return ok_; }
  uint64_t pos() const { return pos_; }
  void raw(const void* p, size_t n) {
    if (ok_ && n && std::fwrite(p, 1, n, f_) != n) ok_ = false;
    pos_ += n;
  }
  template <class T>
  void pod(T v) { raw(&v, sizeof v); }
  void str(const std::string& s) {
    pod<uint32_t>((uint32_t)s.size());
    raw(s.data(), s.size());
  }
  void zeros(size_t n) {
    static const char z[4096] = {};
    while (n) {
      const size_t k = n < sizeof z ? n : sizeof z;
      raw(z, k);
      n -= k;
    }
  }
  bool patch(uint64_t at, const void* p, size_t n) {
    if (!ok_) return false;
    if (std::fseek(f_, (long)at, SEEK_SET) != 0 || std::fwrite(p, 1, n, f_) != n ||
        std::fseek(f_, 0, SEEK_END) != 0)
      ok_ = false;
    return ok_;
  }

 private:
  FILE* f_;
  uint64_t pos_ = 0;
  bool ok_ = true;
};

// A node mask of 2^(3L) bits as 64-bit words.
struct Mask {
  std::vector<uint64_t> w;
  explicit Mask(int log2) : w(((size_t)1 << (3 * log2)) / 64, 0) {}
  void set(size_t i) { w[i >> 6] |= uint64_t(1) << (i & 63); }
  void save(Writer& o) const { o.raw(w.data(), w.size() * 8); }
};

struct Box {
  int32_t nx, ny, nz;
};

// Index of the child (or voxel) at (x, y, z) inside a node of log2 size L
// whose children span 2^C voxels.
inline size_t node_index(int x, int y, int z, int L, int C) {
  const int m = (1 << (L + C)) - 1;
  return ((size_t)((x & m) >> C) << (2 * L)) | ((size_t)((y & m) >> C) << L) | (size_t)((z & m) >> C);
}

// The children of an internal node at origin o (span S, child span s) that
// intersect the box, in index order (x slowest).
std::vector<std::array<int, 3>> children(const Box& b, const std::array<int, 3>& o, int S, int s) {
  std::vector<std::array<int, 3>> out;
  for (int x = o[0]; x < o[0] + S && x < b.nx; x += s)
    for (int y = o[1]; y < o[1] + S && y < b.ny; y += s)
      for (int z = o[2]; z < o[2] + S && z < b.nz; z += s) out.push_back({x, y, z});
  return out;
}

Mask leaf_mask(const Box& b, const std::array<int, 3>& o) {
  Mask m(kLeafLog2);
  for (int i = 0; i < kLeafDim; ++i)
    for (int j = 0; j < kLeafDim; ++j)
      for (int k = 0; k < kLeafDim; ++k)
        if (o[0] + i < b.nx && o[1] + j < b.ny && o[2] + k < b.nz) m.set((size_t)(i << 6 | j << 3 | k));
  return m;
}

template <int L, int C>
Mask child_mask(const std::vector<std::array<int, 3>>& kids) {
  Mask m(L);
  for (const auto& c : kids) m.set(node_index(c[0], c[1], c[2], L, C));
  return m;
}

void write_internal_values(Writer& o, int log2) {
  // inactive background tiles everywhere (child slots also write zero)
  o.pod<uint8_t>(kAllValues);
  o.zeros(((size_t)1 << (3 * log2)) * 12);
}

void meta_string(Writer& o, const char* name, const std::string& v) {
  o.str(name);
  o.str("string");
  o.str(v);
}

}  // namespace

extern "C" {

int lbm_vdb_write_vec3(const char* path, const float* xyz, int32_t nx, int32_t ny, int32_t nz,
                       float voxel_size, const float origin[3], const char* grid_name) {
  if (!path || !xyz) return vdb_fail(LBM_ERR_INVALID_ARG, "path and data must not be NULL");
  if (nx <= 0 || ny <= 0 || nz <= 0) return vdb_fail(LBM_ERR_INVALID_ARG, "dimensions must be positive");
  if (!(voxel_size > 0.f) || !std::isfinite(voxel_size))
    return vdb_fail(LBM_ERR_INVALID_ARG, "voxel_size must be finite and > 0");
  const double org[3] = {origin ? origin[0] : 0.0, origin ? origin[1] : 0.0, origin ? origin[2] : 0.0};
  const Box box{nx, ny, nz};
  FILE* f = std::fopen(path, "wb");
  if (!f) return vdb_fail(LBM_ERR_IO, std::string("cannot open ") + path);
  Writer o(f);

  // header
  o.pod<int64_t>(0x56444220);
  o.pod<uint32_t>(kFileVersion);
  o.pod<uint32_t>(kLibMajor);
  o.pod<uint32_t>(kLibMinor);
  o.pod<uint8_t>(1);
  {
    std::random_device rd;
    std::mt19937_64 gen(((uint64_t)rd() << 32) ^ rd());
    uint8_t u[16];
    for (int i = 0; i < 16; i += 8) {
      const uint64_t v = gen();
      std::memcpy(u + i, &v, 8);
    }
    u[6] = (uint8_t)((u[6] & 0x0f) | 0x40);  // version 4 (random)
    u[8] = (uint8_t)((u[8] & 0x3f) | 0x80);  // RFC 4122 variant
    char s[37];
    std::snprintf(s, sizeof s, "%02x%02x%02x%02x-%02x%02x-%02x%02x-%02x%02x-%02x%02x%02x%02x%02x%02x",
                  u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], u[8], u[9], u[10], u[11], u[12], u[13],
                  u[14], u[15]);
    o.raw(s, 36);
  }
  o.pod<uint32_t>(0);  // file metadata: none
  o.pod<int32_t>(1);   // one grid

  // grid descriptor
  o.str(grid_name && *grid_name ? grid_name : "velocity");
  o.str("Tree_vec3s_5_4_3");
  o.str("");
  const uint64_t offsets_at = o.pos();
  int64_t pos3[3] = {0, 0, 0};
  o.raw(pos3, sizeof pos3);
  pos3[0] = (int64_t)o.pos();
  o.pod<uint32_t>(0);  // compression: none

  // grid metadata, sorted by name
  {
    o.pod<uint32_t>(6);
    meta_string(o, "class", "staggered");
    o.str("file_bbox_max");
    o.str("vec3i");
    o.pod<uint32_t>(12);
    o.pod<int32_t>(nx - 1);
    o.pod<int32_t>(ny - 1);
    o.pod<int32_t>(nz - 1);
    o.str("file_bbox_min");
    o.str("vec3i");
    o.pod<uint32_t>(12);
    o.zeros(12);
    o.str("file_voxel_count");
    o.str("int64");
    o.pod<uint32_t>(8);
    o.pod<int64_t>((int64_t)nx * ny * nz);
    o.str("is_saved_as_half_float");
    o.str("bool");
    o.pod<uint32_t>(1);
    o.pod<uint8_t>(0);
    meta_string(o, "name", grid_name && *grid_name ? grid_name : "velocity");
  }

  // transform: a uniform scale, with the origin as a translation if nonzero
  {
    const double s = voxel_size;
    const double vals[5][3] = {{s, s, s}, {s, s, s}, {1 / s, 1 / s, 1 / s},
                               {1 / (s * s), 1 / (s * s), 1 / (s * s)},
                               {0.5 / s, 0.5 / s, 0.5 / s}};
    if (org[0] != 0.0 || org[1] != 0.0 || org[2] != 0.0) {
      o.str("UniformScaleTranslateMap");
      o.raw(org, sizeof org);
    } else {
      o.str("UniformScaleMap");
    }
    o.raw(vals, sizeof vals);
  }

  // topology
  const std::array<int, 3> zero{0, 0, 0};
  const auto roots = children(box, zero, 1 << 30, kInt2Span);
  o.pod<int32_t>(1);     // buffer count
  o.zeros(12);           // background (0, 0, 0)
  o.pod<uint32_t>(0);    // tiles
  o.pod<uint32_t>((uint32_t)roots.size());
  // leaves in file order, for the buffer pass
  std::vector<std::array<int, 3>> leaves;
  for (const auto& r : roots) {
    o.raw(r.data(), 12);
    const auto n1s = children(box, r, kInt2Span, kInt1Span);
    child_mask<kInt2Log2, kInt1Log2 + kLeafLog2>(n1s).save(o);
    Mask(kInt2Log2).save(o);  // no active tiles
    write_internal_values(o, kInt2Log2);
    for (const auto& n1 : n1s) {
      const auto ls = children(box, n1, kInt1Span, kLeafDim);
      child_mask<kInt1Log2, kLeafLog2>(ls).save(o);
      Mask(kInt1Log2).save(o);
      write_internal_values(o, kInt1Log2);
      for (const auto& l : ls) {
        leaf_mask(box, l).save(o);
        leaves.push_back(l);
      }
    }
  }
  pos3[1] = (int64_t)o.pos();

  // buffers: the 512 values of each leaf, z fastest; inactive voxels 0
  std::vector<float> buf(512 * 3);
  for (const auto& l : leaves) {
    leaf_mask(box, l).save(o);
    o.pod<uint8_t>(kAllValues);
    std::fill(buf.begin(), buf.end(), 0.f);
    const int xe = std::min(kLeafDim, nx - l[0]), ye = std::min(kLeafDim, ny - l[1]),
              ze = std::min(kLeafDim, nz - l[2]);
    for (int i = 0; i < xe; ++i)
      for (int j = 0; j < ye; ++j)
        for (int k = 0; k < ze; ++k) {
          const size_t src = ((size_t)(l[0] + i) + (size_t)nx * ((size_t)(l[1] + j) + (size_t)ny * (l[2] + k))) * 3;
          std::memcpy(&buf[(size_t)(i << 6 | j << 3 | k) * 3], xyz + src, 12);
        }
    o.raw(buf.data(), buf.size() * 4);
  }
  pos3[2] = (int64_t)o.pos();
  const bool ok = o.ok() && o.patch(offsets_at, pos3, sizeof pos3);
  const bool closed = std::fclose(f) == 0;
  if (!ok || !closed) return vdb_fail(LBM_ERR_IO, std::string("write failed: ") + path);
  return LBM_OK;
}

int lbm_vdb_export(lbm_ctx* ctx, const char* dir, uint32_t frame_idx, int flags) {
  if (!ctx || !dir) return vdb_fail(LBM_ERR_INVALID_ARG, "ctx and dir must not be NULL");
  if (flags & ~LBM_VDB_F32) return vdb_fail(LBM_ERR_INVALID_ARG, "unknown flags");
  lbm_desc d;
  d.struct_size = sizeof d;
  if (int rc = lbm_get_desc(ctx, &d)) return vdb_fail(rc, lbm_last_error(ctx));
  const size_t n = (size_t)d.nx * d.ny * d.nz;
  std::vector<float> xyz(3 * n);
  if (flags & LBM_VDB_F32) {
    if (int rc = lbm_read_moments(ctx, nullptr, xyz.data(), LBM_U_F32X3)) return vdb_fail(rc, lbm_last_error(ctx));
  } else {
    // as the reference: rgba16f readback, then half -> float of x, y, z
    std::vector<uint16_t> h(4 * n);
    if (int rc = lbm_read_moments(ctx, nullptr, h.data(), LBM_U_F16X4)) return vdb_fail(rc, lbm_last_error(ctx));
    std::vector<uint16_t> h3(3 * n);
    for (size_t i = 0; i < n; ++i) {
      h3[3 * i] = h[4 * i];
      h3[3 * i + 1] = h[4 * i + 1];
      h3[3 * i + 2] = h[4 * i + 2];
    }
    lbm_half_to_float(h3.data(), xyz.data(), 3 * n);
  }
  char name[64];
  std::snprintf(name, sizeof name, "/velocity_%06u.vdb", frame_idx);
  const std::string path = std::string(dir) + name;
  return lbm_vdb_write_vec3(path.c_str(), xyz.data(), d.nx, d.ny, d.nz, 1.0f, nullptr, "velocity");
}

const char* lbm_vdb_last_error(void) { return g_vdb_err.c_str(); }

}  // extern "C"
