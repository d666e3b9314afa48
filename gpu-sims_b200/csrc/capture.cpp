// Capture directories in the layout of GPU-Sims' StateWriter / StateReader
// (common/common-cpp/src/state_writer.cpp:26-85, state_reader.cpp:12-85) and
// of the lattice-Boltzmann F5/F9 handlers (volumetric-grid/lattice-boltzmann/
// src/main.cpp:1267-1390): <root>/capture_%04u/state.json plus one raw
// `<name>.bin` per buffer.  The lattice writes `density` (r32f),
// `velocity` (rgba16f), `obstacle_mask` (r8uint, frame_invariant) and, for a
// full-state checkpoint, `populations` (r32f, 19 values per node,
// direction-major): the f-state the reference does not capture, so that a
// load resumes the run exactly.
//
// state.json is written as the reference's nlohmann dump(2) writes it (keys
// sorted, two-space indent); the caller's meta object is embedded under
// "latticeBoltzmann" with its number tokens kept verbatim.  Reading accepts
// any RFC 8259 JSON.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "lbm_internal.h"

namespace fs = std::filesystem;

namespace {

// ---- a small JSON value, parser and nlohmann-style printer -----------------
struct JVal {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } k = Null;
  bool b = false;
  std::string s;                        // string value, or the number token
  std::vector<JVal> a;
  std::map<std::string, JVal> o;        // sorted keys, as nlohmann::json
  const JVal* get(const std::string& key) const {
    if (k != Obj) return nullptr;
    auto it = o.find(key);
    return it == o.end() ? nullptr : &it->second;
  }
  double num() const { return k == Num ? std::strtod(s.c_str(), nullptr) : 0.0; }
};

class Parser {
 public:
  Parser(const char* p, const char* e) : p_(p), e_(e) {}
  bool parse(JVal& v) {
    ws();
    if (!value(v, 0)) return false;
    ws();
    return p_ == e_;
  }

 private:
  const char* p_;
  const char* e_;
  void ws() {
    while (p_ < e_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) ++p_;
  }
  bool lit(const char* w) {
    const size_t n = std::strlen(w);
    if ((size_t)(e_ - p_) < n || std::strncmp(p_, w, n) != 0) return false;
    p_ += n;
    return true;
  }
  static void utf8(std::string& out, unsigned cp) {
    if (cp < 0x80) {
      out += (char)cp;
    } else if (cp < 0x800) {
      out += (char)(0xC0 | (cp >> 6));
      out += (char)(0x80 | (cp & 0x3F));
    } else if (cp < 0x10000) {
      out += (char)(0xE0 | (cp >> 12));
      out += (char)(0x80 | ((cp >> 6) & 0x3F));
      out += (char)(0x80 | (cp & 0x3F));
    } else {
      out += (char)(0xF0 | (cp >> 18));
      out += (char)(0x80 | ((cp >> 12) & 0x3F));
      out += (char)(0x80 | ((cp >> 6) & 0x3F));
      out += (char)(0x80 | (cp & 0x3F));
    }
  }
  bool hex4(unsigned& v) {
    if (e_ - p_ < 4) return false;
    v = 0;
    for (int i = 0; i < 4; ++i) {
      const char c = *p_++;
      v <<= 4;
      if (c >= '0' && c <= '9') v |= (unsigned)(c - '0');
      else if (c >= 'a' && c <= 'f') v |= (unsigned)(c - 'a' + 10);
      else if (c >= 'A' && c <= 'F') v |= (unsigned)(c - 'A' + 10);
      else return false;
    }
    return true;
  }
  bool string(std::string& out) {
    if (p_ >= e_ || *p_ != '"') return false;
    ++p_;
    while (p_ < e_ && *p_ != '"') {
      const unsigned char c = (unsigned char)*p_++;
      if (c < 0x20) return false;
      if (c != '\\') {
        out += (char)c;
        continue;
      }
      if (p_ >= e_) return false;
      const char esc = *p_++;
      switch (esc) {
        case '"': out += '"'; break;
        case '\\': out += '\\'; break;
        case '/': out += '/'; break;
        case 'b': out += '\b'; break;
        case 'f': out += '\f'; break;
        case 'n': out += '\n'; break;
        case 'r': out += '\r'; break;
        case 't': out += '\t'; break;
        case 'u': {
          unsigned cp;
          if (!hex4(cp)) return false;
          if (cp >= 0xD800 && cp < 0xDC00) {  // surrogate pair
            unsigned lo;
            if (!lit("\\u") || !hex4(lo) || lo < 0xDC00 || lo >= 0xE000) return false;
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          } else if (cp >= 0xDC00 && cp < 0xE000) {
            return false;
          }
          utf8(out, cp);
          break;
        }
        default: return false;
      }
    }
    if (p_ >= e_) return false;
    ++p_;
    return true;
  }
  bool number(std::string& tok) {
    const char* s = p_;
    if (p_ < e_ && *p_ == '-') ++p_;
    if (p_ >= e_) return false;
    if (*p_ == '0') {
      ++p_;
    } else if (*p_ >= '1' && *p_ <= '9') {
      while (p_ < e_ && *p_ >= '0' && *p_ <= '9') ++p_;
    } else {
      return false;
    }
    if (p_ < e_ && *p_ == '.') {
      ++p_;
      if (p_ >= e_ || *p_ < '0' || *p_ > '9') return false;
      while (p_ < e_ && *p_ >= '0' && *p_ <= '9') ++p_;
    }
    if (p_ < e_ && (*p_ == 'e' || *p_ == 'E')) {
      ++p_;
      if (p_ < e_ && (*p_ == '+' || *p_ == '-')) ++p_;
      if (p_ >= e_ || *p_ < '0' || *p_ > '9') return false;
      while (p_ < e_ && *p_ >= '0' && *p_ <= '9') ++p_;
    }
    tok.assign(s, p_);
    return true;
  }
  bool value(JVal& v, int depth) {
    if (depth > 64 || p_ >= e_) return false;
    const char c = *p_;
    if (c == '{') {
      ++p_;
      v.k = JVal::Obj;
      ws();
      if (p_ < e_ && *p_ == '}') { ++p_; return true; }
      for (;;) {
        ws();
        std::string key;
        if (!string(key)) return false;
        ws();
        if (p_ >= e_ || *p_ != ':') return false;
        ++p_;
        ws();
        JVal child;
        if (!value(child, depth + 1)) return false;
        v.o[key] = std::move(child);
        ws();
        if (p_ < e_ && *p_ == ',') { ++p_; continue; }
        if (p_ < e_ && *p_ == '}') { ++p_; return true; }
        return false;
      }
    }
    if (c == '[') {
      ++p_;
      v.k = JVal::Arr;
      ws();
      if (p_ < e_ && *p_ == ']') { ++p_; return true; }
      for (;;) {
        ws();
        JVal child;
        if (!value(child, depth + 1)) return false;
        v.a.push_back(std::move(child));
        ws();
        if (p_ < e_ && *p_ == ',') { ++p_; continue; }
        if (p_ < e_ && *p_ == ']') { ++p_; return true; }
        return false;
      }
    }
    if (c == '"') { v.k = JVal::Str; return string(v.s); }
    if (lit("true")) { v.k = JVal::Bool; v.b = true; return true; }
    if (lit("false")) { v.k = JVal::Bool; v.b = false; return true; }
    if (lit("null")) { v.k = JVal::Null; return true; }
    v.k = JVal::Num;
    return number(v.s);
  }
};

void dump_str(std::string& out, const std::string& s) {
  out += '"';
  for (unsigned char c : s) {
    switch (c) {
      case '"': out += "\\\""; break;
      case '\\': out += "\\\\"; break;
      case '\b': out += "\\b"; break;
      case '\f': out += "\\f"; break;
      case '\n': out += "\\n"; break;
      case '\r': out += "\\r"; break;
      case '\t': out += "\\t"; break;
      default:
        if (c < 0x20) {
          char b[8];
          std::snprintf(b, sizeof(b), "\\u%04x", c);
          out += b;
        } else {
          out += (char)c;
        }
    }
  }
  out += '"';
}

// nlohmann::json::dump(2) layout
void dump(std::string& out, const JVal& v, int ind) {
  const std::string pad((size_t)ind + 2, ' '), end((size_t)ind, ' ');
  switch (v.k) {
    case JVal::Null: out += "null"; break;
    case JVal::Bool: out += v.b ? "true" : "false"; break;
    case JVal::Num: out += v.s; break;
    case JVal::Str: dump_str(out, v.s); break;
    case JVal::Arr:
      if (v.a.empty()) { out += "[]"; break; }
      out += "[\n";
      for (size_t i = 0; i < v.a.size(); ++i) {
        out += pad;
        dump(out, v.a[i], ind + 2);
        out += i + 1 < v.a.size() ? ",\n" : "\n";
      }
      out += end + "]";
      break;
    case JVal::Obj: {
      if (v.o.empty()) { out += "{}"; break; }
      out += "{\n";
      size_t i = 0;
      for (const auto& kv : v.o) {
        out += pad;
        dump_str(out, kv.first);
        out += ": ";
        dump(out, kv.second, ind + 2);
        out += ++i < v.o.size() ? ",\n" : "\n";
      }
      out += end + "}";
      break;
    }
  }
}

JVal jnum(double x) {
  JVal v;
  v.k = JVal::Num;
  char b[40];
  if (std::floor(x) == x && std::fabs(x) < 9.007199254740992e15) {
    std::snprintf(b, sizeof(b), "%.0f", x);
  } else {
    std::snprintf(b, sizeof(b), "%.17g", x);
  }
  v.s = b;
  return v;
}
JVal jstr(const std::string& s) {
  JVal v;
  v.k = JVal::Str;
  v.s = s;
  return v;
}
JVal jbool(bool b) {
  JVal v;
  v.k = JVal::Bool;
  v.b = b;
  return v;
}
JVal jshape(int nx, int ny, int nz) {
  JVal v;
  v.k = JVal::Arr;
  v.a = {jnum(nx), jnum(ny), jnum(nz)};
  return v;
}

thread_local std::string g_cap_err = "no error";

int cfail(int code, const std::string& msg) {
  g_cap_err = msg;
  lbm::set_thread_error(msg.c_str());
  return code;
}

bool write_file(const fs::path& p, const void* data, size_t bytes) {
  std::ofstream out(p, std::ios::binary | std::ios::trunc);
  if (!out) return false;
  out.write(static_cast<const char*>(data), (std::streamsize)bytes);
  return out.good();
}

bool read_file(const fs::path& p, std::vector<char>& out) {
  std::ifstream in(p, std::ios::binary | std::ios::ate);
  if (!in) return false;
  const std::streamsize n = in.tellg();
  if (n < 0) return false;
  out.resize((size_t)n);
  in.seekg(0);
  return n == 0 || (bool)in.read(out.data(), n);
}

struct Capture {
  JVal state;
  fs::path dir;
  int nx = 0, ny = 0, nz = 0;
  uint32_t frame = 0;
  uint64_t iteration = 0;
  const JVal* buffer(const std::string& name) const {
    const JVal* b = state.get("buffers");
    if (!b || b->k != JVal::Arr) return nullptr;
    for (const auto& e : b->a) {
      const JVal* n = e.get("name");
      if (n && n->k == JVal::Str && n->s == name) return &e;
    }
    return nullptr;
  }
};

// Parses state.json and the lattice meta; checks that every buffer the
// lattice reads has the size its descriptor states.
int open_capture(const char* dir, Capture& c) {
  if (!dir) return cfail(LBM_ERR_INVALID_ARG, "capture: directory is NULL");
  c.dir = fs::path(dir);
  std::vector<char> text;
  if (!read_file(c.dir / "state.json", text))
    return cfail(LBM_ERR_IO, "capture: cannot read " + (c.dir / "state.json").string());
  Parser ps(text.data(), text.data() + text.size());
  if (!ps.parse(c.state) || c.state.k != JVal::Obj)
    return cfail(LBM_ERR_IO, "capture: state.json is not valid JSON");
  const JVal* fr = c.state.get("frame");
  c.frame = fr && fr->k == JVal::Num ? (uint32_t)fr->num() : 0u;
  const JVal* meta = c.state.get("meta");
  const JVal* lm = meta ? meta->get("latticeBoltzmann") : nullptr;
  if (!lm || lm->k != JVal::Obj) return cfail(LBM_ERR_IO, "capture: no latticeBoltzmann meta");
  const JVal* it = lm->get("iteration");
  c.iteration = it && it->k == JVal::Num ? (uint64_t)it->num() : 0u;
  // dimensions: the meta's Nx/Ny/Nz, else the density buffer's shape
  const JVal *jx = lm->get("Nx"), *jy = lm->get("Ny"), *jz = lm->get("Nz");
  if (jx && jy && jz && jx->k == JVal::Num && jy->k == JVal::Num && jz->k == JVal::Num) {
    c.nx = (int)jx->num(); c.ny = (int)jy->num(); c.nz = (int)jz->num();
  } else if (const JVal* d = c.buffer("density")) {
    const JVal* sh = d->get("shape");
    if (sh && sh->k == JVal::Arr && sh->a.size() == 3) {
      c.nx = (int)sh->a[0].num(); c.ny = (int)sh->a[1].num(); c.nz = (int)sh->a[2].num();
    }
  }
  if (c.nx < 1 || c.ny < 1 || c.nz < 1) return cfail(LBM_ERR_IO, "capture: no lattice dimensions");
  return LBM_OK;
}

// Reads buffer `name` into dst (bytes_expected bytes): LBM_OK, 1 if the
// buffer is absent, or an error.
int read_buffer(const Capture& c, const char* name, void* dst, size_t bytes_expected) {
  const JVal* b = c.buffer(name);
  if (!b) return 1;
  const JVal* f = b->get("file");
  const std::string file = f && f->k == JVal::Str ? f->s : std::string(name) + ".bin";
  std::vector<char> data;
  if (!read_file(c.dir / file, data)) return cfail(LBM_ERR_IO, "capture: cannot read " + file);
  if (data.size() != bytes_expected)
    return cfail(LBM_ERR_IO, "capture: " + file + " has " + std::to_string(data.size()) +
                                 " bytes, expected " + std::to_string(bytes_expected));
  if (dst) std::memcpy(dst, data.data(), bytes_expected);
  return LBM_OK;
}

JVal default_meta(int nx, int ny, int nz, uint64_t iteration, double tau) {
  JVal m;
  m.k = JVal::Obj;
  m.o["schemaVersion"] = jnum(1);
  m.o["Nx"] = jnum(nx);
  m.o["Ny"] = jnum(ny);
  m.o["Nz"] = jnum(nz);
  m.o["iteration"] = jnum((double)iteration);
  m.o["substeps"] = jnum(1);
  if (tau > 0) m.o["tau"] = jnum(tau);
  return m;
}

int write_capture(const char* root, uint32_t frame, const char* meta_json, int32_t nx, int32_t ny,
                  int32_t nz, const float* rho, const uint16_t* vel, const uint8_t* mask, const float* pops,
                  bool shifted);

}  // namespace

extern "C" {

int lbm_capture_write(const char* root, uint32_t frame, const char* meta_json, int32_t nx, int32_t ny,
                      int32_t nz, const float* rho, const uint16_t* vel, const uint8_t* mask,
                      const float* pops) {
  return write_capture(root, frame, meta_json, nx, ny, nz, rho, vel, mask, pops, false);
}

}  // extern "C"

namespace {

int write_capture(const char* root, uint32_t frame, const char* meta_json, int32_t nx, int32_t ny,
                  int32_t nz, const float* rho, const uint16_t* vel, const uint8_t* mask, const float* pops,
                  bool shifted) {
  if (!root || !rho || !vel || !mask) return cfail(LBM_ERR_INVALID_ARG, "capture write: NULL argument");
  if (nx < 1 || ny < 1 || nz < 1) return cfail(LBM_ERR_INVALID_ARG, "capture write: bad dimensions");
  const size_t N = (size_t)nx * ny * nz;
  JVal meta;
  if (meta_json) {
    Parser ps(meta_json, meta_json + std::strlen(meta_json));
    if (!ps.parse(meta) || meta.k != JVal::Obj)
      return cfail(LBM_ERR_INVALID_ARG, "capture write: meta is not a JSON object");
  } else {
    meta = default_meta(nx, ny, nz, 0, 0.0);
  }
  char dname[32];
  std::snprintf(dname, sizeof(dname), "capture_%04u", frame);
  const fs::path dir = fs::path(root) / dname;
  std::error_code ec;
  fs::create_directories(dir, ec);
  if (ec) return cfail(LBM_ERR_IO, "capture write: cannot create " + dir.string() + ": " + ec.message());
  JVal state;
  state.k = JVal::Obj;
  state.o["frame"] = jnum(frame);
  JVal m;
  m.k = JVal::Obj;
  m.o["latticeBoltzmann"] = meta;
  state.o["meta"] = m;
  JVal bufs;
  bufs.k = JVal::Arr;
  struct B { const char* name; const void* data; size_t bytes; size_t count; int stride; const char* fmt; };
  std::vector<B> list = {{"density", rho, N * 4, N, 4, "r32f"},
                         {"velocity", vel, N * 8, N, 8, "rgba16f"},
                         {"obstacle_mask", mask, N, N, 1, "r8uint"}};
  if (pops) list.push_back({"populations", pops, N * 19 * 4, N * 19, 4, "r32f"});
  for (const B& b : list) {
    const std::string file = std::string(b.name) + ".bin";
    if (!write_file(dir / file, b.data, b.bytes)) return cfail(LBM_ERR_IO, "capture write: cannot write " + file);
    JVal d;
    d.k = JVal::Obj;
    d.o["count"] = jnum((double)b.count);
    d.o["stride"] = jnum(b.stride);
    d.o["format"] = jstr(b.fmt);
    d.o["shape"] = jshape(nx, ny, nz);
    d.o["name"] = jstr(b.name);
    d.o["file"] = jstr(file);
    d.o["bytes"] = jnum((double)b.bytes);
    if (std::strcmp(b.name, "obstacle_mask") == 0) d.o["frame_invariant"] = jbool(true);
    if (std::strcmp(b.name, "populations") == 0) {
      d.o["shape"].a.insert(d.o["shape"].a.begin(), jnum(19));
      d.o["components"] = jnum(19);
      d.o["layout"] = jstr("direction-major f[19][Nx*Ny*Nz], x fastest, post-collision");
      if (shifted) d.o["values"] = jstr("f - w");
    }
    bufs.a.push_back(std::move(d));
  }
  state.o["buffers"] = bufs;
  std::string text;
  dump(text, state, 0);
  if (!write_file(dir / "state.json", text.data(), text.size()))
    return cfail(LBM_ERR_IO, "capture write: cannot write state.json");
  return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_capture_read(const char* dir, lbm_capture_info* info, float* rho, uint16_t* vel, uint8_t* mask,
                     float* pops) {
  if (!info) return cfail(LBM_ERR_INVALID_ARG, "capture read: info is NULL");
  if (info->struct_size != sizeof(lbm_capture_info))
    return cfail(LBM_ERR_INVALID_ARG, "capture read: lbm_capture_info struct_size");
  Capture c;
  if (int rc = open_capture(dir, c)) return rc;
  const size_t N = (size_t)c.nx * c.ny * c.nz;
  info->nx = c.nx;
  info->ny = c.ny;
  info->nz = c.nz;
  info->frame = c.frame;
  info->iteration = c.iteration;
  info->has_populations = c.buffer("populations") != nullptr;
  info->mask_frame_invariant = 0;
  if (const JVal* mb = c.buffer("obstacle_mask"))
    if (const JVal* fi = mb->get("frame_invariant")) info->mask_frame_invariant = fi->k == JVal::Bool && fi->b;
  struct R { const char* name; void* dst; size_t bytes; bool required; };
  const R rs[] = {{"density", rho, N * 4, true},
                  {"velocity", vel, N * 8, true},
                  {"obstacle_mask", mask, N, false},
                  {"populations", pops, N * 19 * 4, false}};
  for (const R& r : rs) {
    const int rc = read_buffer(c, r.name, r.dst, r.bytes);
    if (rc < 0) return rc;
    if (rc == 1 && (r.required || r.dst))
      return cfail(LBM_ERR_IO, std::string("capture read: no ") + r.name + " buffer");
  }
  return LBM_OK;
}

int lbm_capture_latest(const char* root, char* out, size_t cap) {
  if (!root || !out || cap == 0) return cfail(LBM_ERR_INVALID_ARG, "capture latest: bad argument");
  std::error_code ec;
  if (!fs::is_directory(root, ec)) return cfail(LBM_ERR_IO, std::string("capture latest: no directory ") + root);
  std::vector<fs::path> found;
  for (const auto& e : fs::directory_iterator(root, ec)) {
    if (ec) break;
    if (!e.is_directory()) continue;
    if (e.path().filename().string().rfind("capture_", 0) == 0) found.push_back(e.path());
  }
  if (found.empty()) return cfail(LBM_ERR_IO, std::string("capture latest: no capture under ") + root);
  std::sort(found.begin(), found.end());
  const std::string s = found.back().string();
  if (s.size() + 1 > cap) return cfail(LBM_ERR_INVALID_ARG, "capture latest: output buffer too small");
  std::memcpy(out, s.c_str(), s.size() + 1);
  return LBM_OK;
}

int lbm_capture_save(lbm_ctx* ctx, const char* root, uint32_t frame, const char* meta_json, int full_state) {
  if (!ctx) return cfail(LBM_ERR_INVALID_ARG, "capture save: ctx is NULL");
  lbm_info inf{};
  inf.struct_size = sizeof(inf);
  if (int rc = lbm_get_info(ctx, &inf)) return rc;
  const size_t N = (size_t)inf.nx * inf.ny * inf.nz;
  std::vector<float> rho(N);
  std::vector<uint16_t> vel(4 * N);
  std::vector<uint8_t> mask(N);
  std::vector<float> pops;
  if (int rc = lbm_read_moments(ctx, rho.data(), vel.data(), LBM_U_F16X4)) return rc;
  if (int rc = lbm_read_mask(ctx, mask.data(), N)) return rc;
  const bool shifted = full_state && inf.mode == LBM_MODE_PHYSICS;
  if (full_state) {
    pops.resize(19 * N);
    const int rc = shifted ? lbm_read_populations_shifted(ctx, pops.data(), 19 * N)
                           : lbm_read_populations(ctx, pops.data(), 19 * N);
    if (rc) return rc;
  }
  std::string meta;
  if (!meta_json) {
    lbm_desc d{};
    d.struct_size = sizeof(d);
    lbm_get_desc(ctx, &d);
    std::string text;
    dump(text, default_meta(inf.nx, inf.ny, inf.nz, inf.iteration, d.tau), 0);
    meta = text;
  }
  return write_capture(root, frame, meta_json ? meta_json : meta.c_str(), inf.nx, inf.ny, inf.nz, rho.data(),
                       vel.data(), mask.data(), full_state ? pops.data() : nullptr, shifted);
}

int lbm_capture_load(lbm_ctx* ctx, const char* dir, int flags) {
  if (!ctx) return cfail(LBM_ERR_INVALID_ARG, "capture load: ctx is NULL");
  if (flags & ~(LBM_CAPTURE_LOAD_MASK | LBM_CAPTURE_MOMENTS_ONLY))
    return cfail(LBM_ERR_INVALID_ARG, "capture load: unknown flag");
  lbm_capture_info ci{};
  ci.struct_size = sizeof(ci);
  if (int rc = lbm_capture_read(dir, &ci, nullptr, nullptr, nullptr, nullptr)) return rc;
  lbm_info inf{};
  inf.struct_size = sizeof(inf);
  if (int rc = lbm_get_info(ctx, &inf)) return rc;
  if (ci.nx != inf.nx || ci.ny != inf.ny || ci.nz != inf.nz)
    return cfail(LBM_ERR_INVALID_ARG, "capture load: capture and lattice dimensions differ");
  const size_t N = (size_t)ci.nx * ci.ny * ci.nz;
  const bool pops = ci.has_populations && !(flags & LBM_CAPTURE_MOMENTS_ONLY);
  std::vector<float> rho(N), f(pops ? 19 * N : 0);
  std::vector<uint16_t> vel(4 * N);
  std::vector<uint8_t> mask((flags & LBM_CAPTURE_LOAD_MASK) ? N : 0);
  if (int rc = lbm_capture_read(dir, &ci, rho.data(), vel.data(), mask.empty() ? nullptr : mask.data(),
                                pops ? f.data() : nullptr))
    return rc;
  if (!mask.empty())
    if (int rc = lbm_set_flags(ctx, mask.data(), N)) return rc;
  if (int rc = lbm_init_from_moments(ctx, rho.data(), vel.data(), LBM_U_F16X4)) return rc;
  if (pops) {
    // f - w as stored by a physics-mode lattice, or plain f
    Capture c;
    if (int rc = open_capture(dir, c)) return rc;
    const JVal* vals = c.buffer("populations")->get("values");
    const bool shifted = vals && vals->k == JVal::Str && vals->s == "f - w";
    int rc;
    if (shifted && inf.mode == LBM_MODE_PHYSICS) {
      rc = lbm_write_populations_shifted(ctx, f.data(), 19 * N);
    } else {
      if (shifted)  // f - w into a reference-mode lattice: add w back on the host
        for (size_t i = 0; i < 19; ++i) {
          const float wi = i == 0 ? 1.0f / 3.0f : (i <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f);
          for (size_t k = 0; k < N; ++k) f[i * N + k] += wi;
        }
      rc = lbm_write_populations(ctx, f.data(), 19 * N);
    }
    if (rc) return rc;
  }
  return lbm_set_iteration(ctx, ci.iteration);
}

const char* lbm_capture_last_error(void) { return g_cap_err.c_str(); }

}  // extern "C"
