// Host-side helpers of the C ABI that need no GPU: the lattice tables, the
// NACA obstacle-mask producer and the binary16 decoder used by the readback.
//
// Compiled with -ffp-contract=off so the voxeliser's float arithmetic rounds
// after every operation, as the reference's C++ does on x86-64 without FMA.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/lbm.h"
#include "d3q19.cuh"
#include "lbm_internal.h"

namespace {

struct Naca {
  float m, p, t;  // max camber, its chord position, thickness (fractions)
};

bool parse_naca(const char* s, Naca* out) {
  if (!s || std::strlen(s) != 4) return false;
  for (int i = 0; i < 4; ++i)
    if (s[i] < '0' || s[i] > '9') return false;
  out->m = float(s[0] - '0') / 100.0f;
  out->p = float(s[1] - '0') / 10.0f;
  out->t = float((s[2] - '0') * 10 + (s[3] - '0')) / 100.0f;
  return true;
}

// NACA 4-digit half thickness (NACA Report 460), chord = 1.
float half_thickness(float x, float t) {
  const float poly = 0.2969f * std::sqrt(x) - 0.1260f * x - 0.3516f * x * x +
                     0.2843f * x * x * x - 0.1015f * x * x * x * x;
  return 5.0f * t * poly;
}

// Mean camber line y_c(x) and its slope.
void camber(float x, float m, float p, float* yc, float* slope) {
  if (m <= 0.0f) {
    *yc = 0.0f;
    *slope = 0.0f;
    return;
  }
  if (x <= p) {
    const float k = m / (p * p);
    *yc = k * (2.0f * p * x - x * x);
    *slope = k * (2.0f * p - 2.0f * x);
  } else {
    const float k = 1.0f / ((1.0f - p) * (1.0f - p));
    *yc = m * k * ((1.0f - 2.0f * p) + 2.0f * p * x - x * x);
    *slope = m * k * (2.0f * p - 2.0f * x);
  }
}

struct P2 {
  float x, y;
};

// Upper and lower surface points at chord station x (thickness applied
// perpendicular to the camber line).
void surface(float x, const Naca& a, P2* up, P2* lo) {
  const float yt = half_thickness(x, a.t);
  float yc, dyc;
  camber(x, a.m, a.p, &yc, &dyc);
  const float th = std::atan(dyc);
  const float s = std::sin(th), c = std::cos(th);
  *up = {x - yt * s, yc + yt * c};
  *lo = {x + yt * s, yc - yt * c};
}

// Winding number of a closed polygon around (px, py), crossing rule with the
// signed edge test (upward crossing with the point left of the edge counts
// +1, downward crossing with the point right of it counts -1).
int winding(const std::vector<P2>& poly, float px, float py) {
  int wn = 0;
  const size_t n = poly.size();
  for (size_t i = 0; i < n; ++i) {
    const P2 a = poly[i];
    const P2 b = poly[(i + 1) % n];
    const float side = (b.x - a.x) * (py - a.y) - (px - a.x) * (b.y - a.y);
    if (a.y <= py) {
      if (b.y > py && side > 0.0f) ++wn;
    } else {
      if (b.y <= py && side < 0.0f) --wn;
    }
  }
  return wn;
}

}  // namespace

namespace lbm {

bool naca_perimeter(const char* designation, int32_t nx, int32_t ny, float chord_frac, float center_x_frac,
                    float angle_of_attack_deg, std::vector<float>* xy) {
  Naca a;
  if (!parse_naca(designation, &a) || nx < 1 || ny < 1) return false;
  // Preset geometry (src/main.cpp:1180-1190): chord in pixels, leading edge
  // half a chord upstream of the chord centre, on the domain's mid-height.
  const float chord = chord_frac * float(nx);
  const float le_x = center_x_frac * float(nx) - chord * 0.5f;
  const float le_y = float(ny) * 0.5f;
  const float alpha = angle_of_attack_deg * 0.01745329251994329576923690768489f;

  // Closed perimeter: 256 upper-surface samples leading -> trailing edge,
  // then 256 lower-surface samples back to the leading edge.
  constexpr int kSamples = 256;
  std::vector<P2> poly;
  poly.reserve(2 * kSamples);
  std::vector<P2> lower(kSamples);
  for (int i = 0; i < kSamples; ++i) {
    const float x = float(i) / float(kSamples - 1);
    P2 up, lo;
    surface(x, a, &up, &lo);
    poly.push_back(up);
    lower[i] = lo;
  }
  for (int i = kSamples - 1; i >= 0; --i) poly.push_back(lower[i]);
  const float ca = std::cos(alpha), sa = std::sin(alpha);
  xy->resize(2 * poly.size());
  for (size_t i = 0; i < poly.size(); ++i) {
    const float xp = poly[i].x * chord, yp = poly[i].y * chord;
    const float xr = ca * xp - sa * yp;
    const float yr = sa * xp + ca * yp;
    (*xy)[2 * i] = xr + le_x;
    (*xy)[2 * i + 1] = yr + le_y;
  }
  return true;
}

}  // namespace lbm

extern "C" {

int lbm_lattice_tables(int32_t* c, float* w, int32_t* opp) {
  for (int i = 0; i < 19; ++i) {
    if (c) {
      c[3 * i + 0] = lbm::cx(i);
      c[3 * i + 1] = lbm::cy(i);
      c[3 * i + 2] = lbm::cz(i);
    }
    if (w) w[i] = lbm::wf(i);
    if (opp) opp[i] = lbm::opp(i);
  }
  return LBM_OK;
}

int lbm_voxelize_naca(const char* designation, int32_t nx, int32_t ny, int32_t nz, float chord_frac,
                      float center_x_frac, float angle_of_attack_deg, uint8_t* mask, size_t n) {
  if (nx < 1 || ny < 1 || nz < 1 || !mask) return LBM_ERR_INVALID_ARG;
  if (n != (size_t)nx * (size_t)ny * (size_t)nz) return LBM_ERR_INVALID_ARG;
  std::vector<float> xy;
  if (!lbm::naca_perimeter(designation, nx, ny, chord_frac, center_x_frac, angle_of_attack_deg, &xy))
    return LBM_ERR_INVALID_ARG;
  std::vector<P2> poly(xy.size() / 2);
  for (size_t i = 0; i < poly.size(); ++i) poly[i] = {xy[2 * i], xy[2 * i + 1]};
  std::memset(mask, 0, n);
  for (int32_t y = 0; y < ny; ++y)
    for (int32_t x = 0; x < nx; ++x) {
      if (winding(poly, float(x) + 0.5f, float(y) + 0.5f) == 0) continue;
      for (int32_t z = 0; z < nz; ++z) mask[(size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z)] = 1;
    }
  return LBM_OK;
}

// IEEE 754 binary16 -> binary32.  Normal numbers re-bias the exponent
// (15 -> 127); subnormals are normalised by shifting the mantissa until its
// leading one reaches the implicit-bit position; Inf/NaN keep their payload.
int lbm_half_to_float(const uint16_t* h, float* f, size_t n) {
  if ((!h || !f) && n) return LBM_ERR_INVALID_ARG;
  for (size_t i = 0; i < n; ++i) {
    const uint32_t v = h[i];
    const uint32_t sign = (v & 0x8000u) << 16;
    int32_t exp = (int32_t)((v >> 10) & 0x1Fu);
    uint32_t man = v & 0x3FFu;
    uint32_t bits;
    if (exp == 0x1F) {
      bits = sign | 0x7F800000u | (man << 13);
    } else if (exp == 0) {
      if (man == 0) {
        bits = sign;
      } else {
        int32_t e = -14;
        while (!(man & 0x400u)) {
          man <<= 1;
          --e;
        }
        man &= 0x3FFu;
        bits = sign | ((uint32_t)(e + 127) << 23) | (man << 13);
      }
    } else {
      bits = sign | ((uint32_t)(exp - 15 + 127) << 23) | (man << 13);
    }
    std::memcpy(&f[i], &bits, sizeof(float));
  }
  return LBM_OK;
}

const char* lbm_build_info(void) {
  return "lbm_b200 abi=" "1" " arch=sm_100a"
#ifdef LBM_BUILD_TAG
         " " LBM_BUILD_TAG
#endif
      ;
}

}  // extern "C"

// Colour LUT of the velocity-magnitude pass, rgba8 [4][256][4], rows equal:
// the cool-to-warm ramp of src/main.cpp:529-563 (dark blue, cyan, green,
// yellow, red over four quarter ranges of t = i / 255), channels truncated
// to bytes.
extern "C" int lbm_colormap_lut(uint8_t* out) {
  if (!out) return LBM_ERR_INVALID_ARG;
  auto clamp01 = [](float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); };
  for (int i = 0; i < 256; ++i) {
    const float t = (float)i / 255.0f;
    float r, g, b;
    if (t < 0.25f) {
      const float f = t / 0.25f;
      r = 0.05f; g = 0.05f + 0.6f * f; b = 0.4f + 0.6f * f;
    } else if (t < 0.5f) {
      const float f = (t - 0.25f) / 0.25f;
      r = 0.05f; g = 0.65f + 0.3f * f; b = 1.0f - 0.7f * f;
    } else if (t < 0.75f) {
      const float f = (t - 0.5f) / 0.25f;
      r = 0.05f + 0.95f * f; g = 0.95f - 0.05f * f; b = 0.3f - 0.25f * f;
    } else {
      const float f = (t - 0.75f) / 0.25f;
      r = 1.0f; g = 0.9f - 0.7f * f; b = 0.05f;
    }
    const uint8_t rgb[3] = {(uint8_t)(clamp01(r) * 255.0f), (uint8_t)(clamp01(g) * 255.0f),
                            (uint8_t)(clamp01(b) * 255.0f)};
    for (int row = 0; row < 4; ++row) {
      uint8_t* o = out + 4 * (row * 256 + i);
      o[0] = rgb[0]; o[1] = rgb[1]; o[2] = rgb[2]; o[3] = 255;
    }
  }
  return LBM_OK;
}

// Jitter LUT, r8 [256][256]: the top byte of successive states of the LCG
// s' = 1664525 s + 1013904223 from s = 0x9E3779B9 (src/main.cpp:565-573).
extern "C" int lbm_jitter_lut(uint8_t* out) {
  if (!out) return LBM_ERR_INVALID_ARG;
  uint32_t s = 0x9E3779B9u;
  for (int i = 0; i < 256 * 256; ++i) {
    s = s * 1664525u + 1013904223u;
    out[i] = (uint8_t)((s >> 24) & 0xFFu);
  }
  return LBM_OK;
}

