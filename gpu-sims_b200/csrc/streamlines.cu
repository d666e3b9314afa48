// Streamline advection on the device velocity field: one thread per
// streamline, an RK2 step with trilinearly sampled velocity, a ring buffer of
// (x, y, z, age) positions per streamline, and reseeding of aged-out or
// escaped streamlines into the inlet slab.  Restates the reference's
// streamline_advect compute pass (volumetric-grid/lattice-boltzmann/shaders/
// streamline_advect.comp.glsl:34-91, dispatched from src/main.cpp:1596-1623)
// and its host seeding (src/main.cpp:1126-1152).
//
// The reference samples the rgba16f velocity image through a hardware
// trilinear sampler (clamp to edge).  Here the sample is computed in fp32
// with every operation explicitly rounded, from the u planes of the moment
// fields (optionally rounded to binary16 first, as the image stores them):
// texel centres at i + 1/2, u = ctr * N - 1/2, i0 = floor(u), weights
// u - i0, indices clamped to [0, N-1].  The oracle evaluates the same
// operations in the same order, so positions agree bit for bit; a hardware
// sampler's reduced-precision weights do not enter.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <random>
#include <string>

#include "lbm_internal.h"

namespace lbm {
namespace {

struct Field {
  const float* u;  // [3][n] planes
  int nx, ny, nz;
  size_t n;
  int round_f16;
};

__device__ __forceinline__ float texel(const Field& F, int c, int i, int j, int k) {
  const float v = F.u[(size_t)c * F.n + (size_t)i + (size_t)F.nx * ((size_t)j + (size_t)F.ny * (size_t)k)];
  return F.round_f16 ? __half2float(__float2half_rn(v)) : v;
}

__device__ __forceinline__ void axis(float ctr, int N, int& i0, int& i1, float& a) {
  const float u = __fsub_rn(__fmul_rn(ctr, (float)N), 0.5f);
  const float f = floorf(u);
  a = __fsub_rn(u, f);
  int lo = (int)f;
  int hi = lo + 1;
  i0 = lo < 0 ? 0 : (lo > N - 1 ? N - 1 : lo);
  i1 = hi < 0 ? 0 : (hi > N - 1 ? N - 1 : hi);
}

__device__ __forceinline__ float lerp_rn(float a, float b, float t) {
  return __fadd_rn(a, __fmul_rn(t, __fsub_rn(b, a)));
}

// Trilinear sample at normalised coordinate ctr (clamp to edge).
__device__ void sample(const Field& F, float cx, float cy, float cz, float out[3]) {
  int x0, x1, y0, y1, z0, z1;
  float ax, ay, az;
  axis(cx, F.nx, x0, x1, ax);
  axis(cy, F.ny, y0, y1, ay);
  axis(cz, F.nz, z0, z1, az);
  for (int c = 0; c < 3; ++c) {
    const float c00 = lerp_rn(texel(F, c, x0, y0, z0), texel(F, c, x1, y0, z0), ax);
    const float c10 = lerp_rn(texel(F, c, x0, y1, z0), texel(F, c, x1, y1, z0), ax);
    const float c01 = lerp_rn(texel(F, c, x0, y0, z1), texel(F, c, x1, y0, z1), ax);
    const float c11 = lerp_rn(texel(F, c, x0, y1, z1), texel(F, c, x1, y1, z1), ax);
    const float c0 = lerp_rn(c00, c10, ay);
    const float c1 = lerp_rn(c01, c11, ay);
    out[c] = lerp_rn(c0, c1, az);
  }
}

__device__ __forceinline__ uint32_t xorshift(uint32_t& s) {
  s ^= s << 13;
  s ^= s >> 17;
  s ^= s << 5;
  return s;
}
__device__ __forceinline__ float rng01(uint32_t& s) {
  return (float)(xorshift(s) & 0x00FFFFFFu) / 16777216.0f;  // exact: power-of-two divisor
}

struct Advect {
  uint32_t count, history, head, frame, reseed_age;
  float dt;
};

__global__ void k_streamline_advect(Field F, float4* __restrict__ pos_hist, Advect A) {
  const uint32_t sid = blockIdx.x * blockDim.x + threadIdx.x;
  if (sid >= A.count) return;
  const float dmax[3] = {(float)F.nx, (float)F.ny, (float)F.nz};
  const uint32_t prev_head = (A.head + A.history - 1u) % A.history;
  const float4 prev = pos_hist[(size_t)sid * A.history + prev_head];
  float p[3] = {prev.x, prev.y, prev.z};
  float age = prev.w;
  bool out = false;
  for (int c = 0; c < 3; ++c) out |= (p[c] < 0.0f) || (p[c] > dmax[c]);
  bool reseed = false;
  if (age >= (float)A.reseed_age || out) {
    uint32_t st = (sid * 2654435761u) ^ (A.frame * 1597334677u);
    const float r0 = rng01(st);
    p[0] = __fadd_rn(0.0f, __fmul_rn(__fmul_rn(__fsub_rn(dmax[0], 0.0f), 0.0625f), __fadd_rn(1.0f, r0)));
    const float r1 = rng01(st);
    p[1] = __fadd_rn(0.0f, __fmul_rn(__fsub_rn(dmax[1], 0.0f), r1));
    const float r2 = rng01(st);
    p[2] = __fadd_rn(0.0f, __fmul_rn(__fsub_rn(dmax[2], 0.0f), r2));
    age = 0.0f;
    reseed = true;
  } else {
    float u1[3], u2[3], mid[3];
    sample(F, __fdiv_rn(p[0], dmax[0]), __fdiv_rn(p[1], dmax[1]), __fdiv_rn(p[2], dmax[2]), u1);
    const float h = __fmul_rn(0.5f, A.dt);
    for (int c = 0; c < 3; ++c) mid[c] = __fadd_rn(p[c], __fmul_rn(h, u1[c]));
    sample(F, __fdiv_rn(mid[0], dmax[0]), __fdiv_rn(mid[1], dmax[1]), __fdiv_rn(mid[2], dmax[2]), u2);
    for (int c = 0; c < 3; ++c) p[c] = __fadd_rn(p[c], __fmul_rn(A.dt, u2[c]));
    age = __fadd_rn(age, 1.0f);
  }
  const float4 v = make_float4(p[0], p[1], p[2], age);
  if (reseed) {
    for (uint32_t hh = 0; hh < A.history; ++hh) pos_hist[(size_t)sid * A.history + hh] = v;
  } else {
    pos_hist[(size_t)sid * A.history + A.head] = v;
  }
}

}  // namespace
}  // namespace lbm

extern "C" {

int lbm_streamline_seed(float* positions, uint32_t count, uint32_t history, int32_t nx, int32_t ny,
                        int32_t nz, uint32_t seed, uint32_t reseed_age) {
  if (!positions || count == 0 || history == 0 || nx < 1 || ny < 1 || nz < 1) {
    lbm::set_thread_error("streamline seed: bad argument");
    return LBM_ERR_INVALID_ARG;
  }
  // the reference's seed_streamlines: one mt19937 stream, per streamline an
  // initial age then x, y, z, drawn by std::uniform_real_distribution<float>
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> ud(0.0f, 1.0f);
  const float x_lo = (float)nx * 0.0625f, x_hi = (float)nx * 0.125f;
  for (uint32_t i = 0; i < count; ++i) {
    const float initial_age = ud(rng) * (float)reseed_age;
    const float px = x_lo + (x_hi - x_lo) * ud(rng);
    const float py = ud(rng) * (float)ny;
    const float pz = ud(rng) * (float)nz;
    for (uint32_t h = 0; h < history; ++h) {
      float* v = positions + 4 * ((size_t)i * history + h);
      v[0] = px; v[1] = py; v[2] = pz; v[3] = initial_age;
    }
  }
  return LBM_OK;
}

int lbm_streamline_advect(const float* d_u, int32_t nx, int32_t ny, int32_t nz, float* d_positions,
                          uint32_t count, uint32_t history, uint32_t head_index, uint32_t frame_count,
                          float dt_render, uint32_t reseed_age, int32_t round_f16, void* stream) {
  if (!d_u || !d_positions || count == 0 || history == 0 || head_index >= history || nx < 1 || ny < 1 ||
      nz < 1 || !(dt_render >= 0.0f)) {
    lbm::set_thread_error("streamline advect: bad argument");
    return LBM_ERR_INVALID_ARG;
  }
  if ((reinterpret_cast<uintptr_t>(d_positions) & 15u) != 0) {
    lbm::set_thread_error("streamline advect: positions must be 16-byte aligned (float4)");
    return LBM_ERR_INVALID_ARG;
  }
  lbm::Field F{d_u, nx, ny, nz, (size_t)nx * ny * nz, round_f16 ? 1 : 0};
  lbm::Advect A{count, history, head_index, frame_count, reseed_age, dt_render};
  lbm::k_streamline_advect<<<(count + 63) / 64, 64, 0, static_cast<cudaStream_t>(stream)>>>(
      F, reinterpret_cast<float4*>(d_positions), A);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    lbm::set_thread_error((std::string("streamline advect: ") + cudaGetErrorString(e)).c_str());
    return LBM_ERR_CUDA;
  }
  return LBM_OK;
}

}  // extern "C"
