// CPU oracle for the D3Q19 step.  TEST INFRASTRUCTURE ONLY: the product
// (gpu-sims_b200/) never links, loads or calls this code.  Tests, the smoke
// check and bench.py's CPU-baseline leg use it as the checker.
//
// RefStep<T> restates the reference's four compute passes literally, one
// pass at a time, exactly as the shaders are written:
//   lattice constants  volumetric-grid/lattice-boltzmann/shaders/lattice_constants.glsl:23-93
//   init               shaders/init_equilibrium.comp.glsl:35-47
//   collide            shaders/collide.comp.glsl:39-61
//   stream             shaders/stream.comp.glsl:29-47
//   boundaries         shaders/apply_boundaries.comp.glsl:52-169
//   moments            shaders/compute_moments.comp.glsl:29-50
//   step order         src/main.cpp:1523-1591 (uniforms :1523-1541)
// with two reading choices the GPU source leaves open:
//   * the u image is rgba16f (src/main.cpp:843): u is rounded to binary16
//     (round-to-nearest-even by default, RTZ selectable) before the collide
//     that reads it;
//   * the outlet (apply_boundaries.comp.glsl:103-125) reads x = Nx-2 from
//     the post-stream state before any boundary write (the GPU reference
//     races with that node's own boundary writes).
//
// ExtStep<T> is the textbook stream-collide the physics mode implements and
// the reference lacks: pull streaming with periodic wrap or half-way
// bounce-back, momentum-corrected moving walls, BGK/TRT, Smagorinsky and Guo
// forcing.  It works on plain populations f (not f - w), so it shares no
// arithmetic shortcut with the GPU kernels.
//
// Build: oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off); each float
// operation rounds on its own, in source order.
#include <omp.h>

#include "ext_step.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// shaders/lattice_constants.glsl:23-43
const int C[19][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},   {0, -1, 0},
                      {0, 0, 1},  {0, 0, -1}, {1, 1, 0},  {1, -1, 0},  {-1, 1, 0},
                      {-1, -1, 0}, {1, 0, 1}, {1, 0, -1}, {-1, 0, 1},  {-1, 0, -1},
                      {0, 1, 1},  {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};
// shaders/lattice_constants.glsl:55-75
const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};

template <class T> T weight(int i) {
  // 1.0/3.0, 1.0/18.0, 1.0/36.0 evaluated in the working precision
  // (shaders/lattice_constants.glsl:46-52).
  return i == 0 ? T(1) / T(3) : (i <= 6 ? T(1) / T(18) : T(1) / T(36));
}

// feq_i (shaders/lattice_constants.glsl:86-93), canonical form, written
// exactly as the GLSL expression.
template <class T> T feq_i(int i, T rho, T ux, T uy, T uz) {
  const T cx = T(C[i][0]), cy = T(C[i][1]), cz = T(C[i][2]);
  const T cdotu = cx * ux + cy * uy + cz * uz;
  const T udotu = ux * ux + uy * uy + uz * uz;
  return weight<T>(i) * rho * (T(1) + T(3) * cdotu + T(4.5) * cdotu * cdotu - T(1.5) * udotu);
}

// binary32 -> binary16 -> binary32 with round-to-nearest-even (mode 1) or
// round-toward-zero (mode 2), from the IEEE 754 definition: the result is
// a multiple of the binary16 quantum of x's binade (2^(e-10), or 2^-24 for
// subnormals); overflow goes to Inf (RTE) or the largest finite (RTZ).
float round_f16(float v, int mode) {
  if (mode == 0 || std::isnan(v) || v == 0.0f) return v;
  const double a = std::fabs((double)v);
  const double s = v < 0 ? -1.0 : 1.0;
  if (std::isinf(v)) return v;
  int e;
  std::frexp(a, &e);          // a = m * 2^e, m in [0.5, 1)  -> binade exponent e-1
  int qexp = (e - 1) - 10;    // quantum exponent for a normal binary16
  if (e - 1 < -14) qexp = -24; // subnormal binary16 range
  const double q = std::ldexp(1.0, qexp);
  double r = a / q;           // exact (power-of-two scaling)
  r = (mode == 1) ? std::nearbyint(r) : std::trunc(r);  // default FP env: ties-to-even
  double out = r * q;
  if (out > 65504.0) out = (mode == 1) ? INFINITY : 65504.0;
  return (float)(s * out);
}

inline size_t idx(int nx, int ny, int x, int y, int z) {
  return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * (size_t)z);
}

struct RefP {
  int nx, ny, nz;
  float tau;
  float u_inf[3];
  float rho0;
  int inlet_outlet, free_slip, u_round;
};

inline unsigned mask_at(const RefP& p, const uint8_t* mask, int x, int y, int z) {
  // shaders/apply_boundaries.comp.glsl:52-55
  if (x < 0 || y < 0 || z < 0 || x >= p.nx || y >= p.ny || z >= p.nz) return 1u;
  return mask[idx(p.nx, p.ny, x, y, z)];
}

// collide (shaders/collide.comp.glsl:39-61), in place.  rho from the r32f
// image, u from the rgba16f image; tau_inv/omtau_inv as src/main.cpp:1524-1526.
void ref_collide(const RefP& p, float* f, const float* rho, const float* u) {
  const size_t N = (size_t)p.nx * p.ny * p.nz;
  const float tau_inv = 1.0f / p.tau;
  const float omtau_inv = 1.0f - tau_inv;
#pragma omp parallel for schedule(static)
  for (long long n = 0; n < (long long)N; ++n) {
    const float r = rho[n];
    const float ux = round_f16(u[n], p.u_round), uy = round_f16(u[N + n], p.u_round),
                uz = round_f16(u[2 * N + n], p.u_round);
    for (int i = 0; i < 19; ++i) {
      const float fi = f[i * N + n];
      const float fe = feq_i<float>(i, r, ux, uy, uz);
      f[i * N + n] = omtau_inv * fi + tau_inv * fe;
    }
  }
}

// stream (shaders/stream.comp.glsl:29-47): pull, sampler clamps to edge.
void ref_stream(const RefP& p, const float* fin, float* fout) {
  const size_t N = (size_t)p.nx * p.ny * p.nz;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < p.nz; ++z)
    for (int y = 0; y < p.ny; ++y)
      for (int x = 0; x < p.nx; ++x) {
        const size_t n = idx(p.nx, p.ny, x, y, z);
        fout[n] = fin[n];
        for (int i = 1; i < 19; ++i) {
          int xs = x - C[i][0], ys = y - C[i][1], zs = z - C[i][2];
          xs = xs < 0 ? 0 : (xs >= p.nx ? p.nx - 1 : xs);
          ys = ys < 0 ? 0 : (ys >= p.ny ? p.ny - 1 : ys);
          zs = zs < 0 ? 0 : (zs >= p.nz ? p.nz - 1 : zs);
          fout[i * N + n] = fin[i * N + idx(p.nx, p.ny, xs, ys, zs)];
        }
      }
}

// compute_moments body (shaders/compute_moments.comp.glsl:37-47) on one
// node's 19 values; also the outlet's upstream moments (:112-119).
void moments_of(const float* v, float& rho, float& rx, float& ry, float& rz) {
  rho = v[0];
  rx = ry = rz = 0.0f;
  for (int i = 1; i < 19; ++i) {
    const float fi = v[i];
    rho += fi;
    rx += fi * float(C[i][0]);
    ry += fi * float(C[i][1]);
    rz += fi * float(C[i][2]);
  }
}

// apply_boundaries (shaders/apply_boundaries.comp.glsl:57-169) in place on
// the post-stream state f; snap is that state before this pass.
void ref_boundaries(const RefP& p, const uint8_t* mask, float* f, const float* snap) {
  const size_t N = (size_t)p.nx * p.ny * p.nz;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < p.nz; ++z)
    for (int y = 0; y < p.ny; ++y)
      for (int x = 0; x < p.nx; ++x) {
        const size_t n = idx(p.nx, p.ny, x, y, z);
        auto F = [&](int i) -> float& { return f[i * N + n]; };
        if (mask_at(p, mask, x, y, z) == 1u) {  // (1)
          for (int i = 0; i < 19; ++i) F(i) = 0.0f;
          continue;
        }
        for (int i = 1; i < 19; ++i)  // (2)
          if (mask_at(p, mask, x + C[i][0], y + C[i][1], z + C[i][2]) == 1u) F(OPP[i]) = F(i);
        const float rho0 = p.rho0;
        if (p.inlet_outlet) {
          if (x == 0) {  // (3a)
            for (int i = 0; i < 19; ++i) F(i) = feq_i<float>(i, rho0, p.u_inf[0], p.u_inf[1], p.u_inf[2]);
          }
          if (x == p.nx - 1) {  // (3b)
            float u[3];
            if (mask_at(p, mask, x - 1, y, z) == 1u) {
              u[0] = p.u_inf[0]; u[1] = p.u_inf[1]; u[2] = p.u_inf[2];
            } else {
              float v[19];
              const size_t up = idx(p.nx, p.ny, x - 1, y, z);
              for (int i = 0; i < 19; ++i) v[i] = snap[i * N + up];
              float rl, rx, ry, rz;
              moments_of(v, rl, rx, ry, rz);
              if (rl > 1e-12f) { u[0] = rx / rl; u[1] = ry / rl; u[2] = rz / rl; }
              else { u[0] = p.u_inf[0]; u[1] = p.u_inf[1]; u[2] = p.u_inf[2]; }
            }
            for (int i = 0; i < 19; ++i) F(i) = feq_i<float>(i, rho0, u[0], u[1], u[2]);
          }
        }
        if (p.free_slip) {  // (4)
          if (y == 0) { F(4) = F(3); F(8) = F(7); F(10) = F(9); F(17) = F(15); F(18) = F(16); }
          if (y == p.ny - 1) { F(3) = F(4); F(7) = F(8); F(9) = F(10); F(15) = F(17); F(16) = F(18); }
          if (z == 0) { F(6) = F(5); F(12) = F(11); F(14) = F(13); F(16) = F(15); F(18) = F(17); }
          if (z == p.nz - 1) { F(5) = F(6); F(11) = F(12); F(13) = F(14); F(15) = F(16); F(17) = F(18); }
        }
      }
}

// compute_moments (shaders/compute_moments.comp.glsl:29-50).
void ref_moments(const RefP& p, const float* f, float* rho, float* u) {
  const size_t N = (size_t)p.nx * p.ny * p.nz;
#pragma omp parallel for schedule(static)
  for (long long n = 0; n < (long long)N; ++n) {
    float v[19];
    for (int i = 0; i < 19; ++i) v[i] = f[i * N + n];
    float r, rx, ry, rz;
    moments_of(v, r, rx, ry, rz);
    float ux = 0.0f, uy = 0.0f, uz = 0.0f;
    if (r > 1e-12f) { ux = rx / r; uy = ry / r; uz = rz / r; }
    rho[n] = r;
    u[n] = ux; u[N + n] = uy; u[2 * N + n] = uz;
  }
}

static RefP make_ref(const int* ip, const float* fp) {
  RefP p;
  p.nx = ip[0]; p.ny = ip[1]; p.nz = ip[2];
  p.inlet_outlet = ip[3]; p.free_slip = ip[4]; p.u_round = ip[5];
  p.tau = fp[0];
  p.u_inf[0] = fp[1]; p.u_inf[1] = fp[2]; p.u_inf[2] = fp[3];
  p.rho0 = fp[4];
  return p;
}

// ---------------------------------------------------------------------------
// ExtStep drivers (node update in ext_step.h, shared with the FP64 GPU copy).
// ---------------------------------------------------------------------------
using ox::ExtP;
using ox::make_ext;

template <class T>
static void ext_init_t(const int* ip, const double* dp, const uint8_t* mask, const T* rho,
                       const T* u, T* f) {
  const ExtP p = make_ext(ip, dp);
  const size_t N = (size_t)p.nx * p.ny * p.nz;
#pragma omp parallel for schedule(static)
  for (long long n = 0; n < (long long)N; ++n) {
    const bool solid = mask[n] == 1;
    for (int i = 0; i < 19; ++i)
      f[i * N + n] = solid ? T(0) : ox::feq_i<T>(i, rho[n], u[n], u[N + n], u[2 * N + n]);
  }
}

template <class T>
static void ext_step_t(const int* ip, const double* dp, const uint8_t* mask, T* f, int nsteps,
                       T* rho_o, T* u_o) {
  const ExtP p = make_ext(ip, dp);
  const size_t N = (size_t)p.nx * p.ny * p.nz;
  std::vector<T> g(19 * N);
  for (int s = 0; s < nsteps; ++s) {
    const bool last = s == nsteps - 1;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < p.nz; ++z)
      for (int y = 0; y < p.ny; ++y)
        for (int x = 0; x < p.nx; ++x) {
          const size_t n = idx(p.nx, p.ny, x, y, z);
          if (mask[n] == 1) {
            for (int i = 0; i < 19; ++i) g[i * N + n] = T(0);
            if (last && rho_o) { rho_o[n] = 0; u_o[n] = u_o[N + n] = u_o[2 * N + n] = 0; }
            continue;
          }
          T v[19];
          for (int i = 0; i < 19; ++i) v[i] = ox::incoming<T>(p, mask, f, x, y, z, i, N);
          ox::open_face<T>(p, v, x);
          T r, ux, uy, uz;
          ox::ext_collide_node<T>(p, v, r, ux, uy, uz);
          for (int i = 0; i < 19; ++i) g[i * N + n] = v[i];
          if (last && rho_o) { rho_o[n] = r; u_o[n] = ux; u_o[N + n] = uy; u_o[2 * N + n] = uz; }
        }
    std::memcpy(f, g.data(), 19 * N * sizeof(T));
  }
}

}  // namespace

extern "C" {

void oracle_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int oracle_max_threads(void) { return omp_get_max_threads(); }

void oracle_tables(int* c, double* w, int* opp) {
  for (int i = 0; i < 19; ++i) {
    for (int a = 0; a < 3; ++a) c[3 * i + a] = C[i][a];
    w[i] = weight<double>(i);
    opp[i] = OPP[i];
  }
}

void oracle_feq_f64(double rho, double ux, double uy, double uz, double* out) {
  for (int i = 0; i < 19; ++i) out[i] = feq_i<double>(i, rho, ux, uy, uz);
}
void oracle_feq_f32(float rho, float ux, float uy, float uz, float* out) {
  for (int i = 0; i < 19; ++i) out[i] = feq_i<float>(i, rho, ux, uy, uz);
}

float oracle_round_f16(float v, int mode) { return round_f16(v, mode); }

// Classification word per node: bit 0 solid, bit i solid-or-outside at
// x + c_i (periodic axes wrap).
void oracle_classify(int nx, int ny, int nz, const int* periodic, const uint8_t* mask, uint32_t* out) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        uint32_t L = mask[idx(nx, ny, x, y, z)] == 1 ? 1u : 0u;
        for (int i = 1; i < 19; ++i) {
          int p[3] = {x + C[i][0], y + C[i][1], z + C[i][2]};
          const int d[3] = {nx, ny, nz};
          bool s = false;
          for (int a = 0; a < 3; ++a)
            if (p[a] < 0 || p[a] >= d[a]) {
              if (periodic[a]) p[a] = (p[a] + d[a]) % d[a];
              else s = true;
            }
          if (!s) s = mask[idx(nx, ny, p[0], p[1], p[2])] == 1;
          if (s) L |= 1u << i;
        }
        out[idx(nx, ny, x, y, z)] = L;
      }
}

// --- RefStep ---------------------------------------------------------------
// params: nx ny nz as ints; floats: tau, u_inf[3], rho0; ints: inlet_outlet,
// free_slip, u_round.  State: f float[19][N] (the ping images after the
// last step), rho float[N], u float[3][N] (moment images; u unrounded).

// init_equilibrium (shaders/init_equilibrium.comp.glsl:35-47): f = feq(rho, u)
// at every node, moment images = (rho, u).  rho_in/u_in may be NULL for the
// uniform (rho0_init, u0) state.
void oracle_ref_init(const int* ip, const float* fp, const float* rho_in, const float* u_in,
                     float rho0_init, const float* u0, float* f, float* rho, float* u) {
  const RefP p = make_ref(ip, fp);
  const size_t N = (size_t)p.nx * p.ny * p.nz;
#pragma omp parallel for schedule(static)
  for (long long n = 0; n < (long long)N; ++n) {
    const float r = rho_in ? rho_in[n] : rho0_init;
    const float ux = u_in ? u_in[n] : u0[0], uy = u_in ? u_in[N + n] : u0[1],
                uz = u_in ? u_in[2 * N + n] : u0[2];
    for (int i = 0; i < 19; ++i) f[i * N + n] = feq_i<float>(i, r, ux, uy, uz);
    rho[n] = r;
    u[n] = ux; u[N + n] = uy; u[2 * N + n] = uz;
  }
}

// nsteps of collide -> stream -> boundaries -> moments (src/main.cpp:1554-1591).
void oracle_ref_step(const int* ip, const float* fp, const uint8_t* mask, float* f, float* rho,
                     float* u, int nsteps) {
  const RefP p = make_ref(ip, fp);
  const size_t N = (size_t)p.nx * p.ny * p.nz;
  std::vector<float> g(19 * N), snap(19 * N);
  for (int s = 0; s < nsteps; ++s) {
    ref_collide(p, f, rho, u);
    ref_stream(p, f, g.data());
    std::memcpy(snap.data(), g.data(), 19 * N * sizeof(float));
    ref_boundaries(p, mask, g.data(), snap.data());
    ref_moments(p, g.data(), rho, u);
    std::memcpy(f, g.data(), 19 * N * sizeof(float));
  }
}

// The collide of the next step applied to the current state, i.e. the
// post-collision populations the fused GPU step stores between launches.
void oracle_ref_collided(const int* ip, const float* fp, const float* f, const float* rho,
                         const float* u, float* out) {
  const RefP p = make_ref(ip, fp);
  const size_t N = (size_t)p.nx * p.ny * p.nz;
  std::memcpy(out, f, 19 * N * sizeof(float));
  ref_collide(p, out, rho, u);
}

void oracle_ext_init_f64(const int* ip, const double* dp, const uint8_t* mask, const double* rho,
                         const double* u, double* f) { ext_init_t<double>(ip, dp, mask, rho, u, f); }
void oracle_ext_init_f32(const int* ip, const double* dp, const uint8_t* mask, const float* rho,
                         const float* u, float* f) { ext_init_t<float>(ip, dp, mask, rho, u, f); }
void oracle_ext_step_f64(const int* ip, const double* dp, const uint8_t* mask, double* f, int nsteps,
                         double* rho, double* u) { ext_step_t<double>(ip, dp, mask, f, nsteps, rho, u); }
void oracle_ext_step_f32(const int* ip, const double* dp, const uint8_t* mask, float* f, int nsteps,
                         float* rho, float* u) { ext_step_t<float>(ip, dp, mask, f, nsteps, rho, u); }

// --- NACA voxeliser (src/main.cpp:200-312, preset geometry :1180-1190) ------
static void naca_pt(float x, float M, float P, float T, float* ux, float* uy, float* lx, float* ly) {
  const float yt = 5.0f * T * (0.2969f * std::sqrt(x) - 0.1260f * x - 0.3516f * x * x +
                               0.2843f * x * x * x - 0.1015f * x * x * x * x);
  float yc = 0.0f, dyc = 0.0f;
  if (M > 0.0f) {
    if (x <= P) {
      yc = (M / (P * P)) * (2.0f * P * x - x * x);
      dyc = (M / (P * P)) * (2.0f * P - 2.0f * x);
    } else {
      const float inv = 1.0f / ((1.0f - P) * (1.0f - P));
      yc = M * inv * ((1.0f - 2.0f * P) + 2.0f * P * x - x * x);
      dyc = M * inv * (2.0f * P - 2.0f * x);
    }
  }
  const float th = std::atan(dyc);
  *ux = x - yt * std::sin(th); *uy = yc + yt * std::cos(th);
  *lx = x + yt * std::sin(th); *ly = yc - yt * std::cos(th);
}

int oracle_voxelize_naca(const char* d, int nx, int ny, int nz, float chord_frac, float cx_frac,
                         float aoa_deg, uint8_t* mask) {
  const float M = float(d[0] - '0') / 100.0f, P = float(d[1] - '0') / 10.0f,
              T = float((d[2] - '0') * 10 + (d[3] - '0')) / 100.0f;
  const float chord = chord_frac * float(nx);
  const float lex = cx_frac * float(nx) - chord * 0.5f, ley = float(ny) * 0.5f;
  const float alpha = aoa_deg * 0.01745329251994329576923690768489f;
  std::vector<float> px, py;
  std::vector<float> lo_x(256), lo_y(256);
  for (int i = 0; i < 256; ++i) {
    const float x = float(i) / float(255);
    float a, b, c, e;
    naca_pt(x, M, P, T, &a, &b, &c, &e);
    px.push_back(a); py.push_back(b); lo_x[i] = c; lo_y[i] = e;
  }
  for (int i = 255; i >= 0; --i) { px.push_back(lo_x[i]); py.push_back(lo_y[i]); }
  const float c = std::cos(alpha), s = std::sin(alpha);
  for (size_t k = 0; k < px.size(); ++k) {
    const float xp = px[k] * chord, yp = py[k] * chord;
    const float xr = c * xp - s * yp, yr = s * xp + c * yp;
    px[k] = xr + lex; py[k] = yr + ley;
  }
  std::memset(mask, 0, (size_t)nx * ny * nz);
  const size_t m = px.size();
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
      const float qx = float(x) + 0.5f, qy = float(y) + 0.5f;
      int wn = 0;
      for (size_t k = 0; k < m; ++k) {
        const size_t j = (k + 1) % m;
        const float cr = (px[j] - px[k]) * (qy - py[k]) - (qx - px[k]) * (py[j] - py[k]);
        if (py[k] <= qy) { if (py[j] > qy && cr > 0.0f) ++wn; }
        else if (py[j] <= qy && cr < 0.0f) --wn;
      }
      if (wn != 0)
        for (int z = 0; z < nz; ++z) mask[idx(nx, ny, x, y, z)] = 1;
    }
  return 0;
}

}  // extern "C"
