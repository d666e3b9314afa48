// Velocity-magnitude volume raymarch into a headless RGBA buffer: one thread
// per pixel.  Restates the reference's velmag fragment pass (volumetric-grid/
// lattice-boltzmann/shaders/velmag.frag.glsl:44-96, uniforms from
// src/main.cpp:1720-1731, LUTs src/main.cpp:529-573, full-screen triangle
// shaders/fullscreen.vert.glsl) without a graphics API: no swapchain,
// window or sampler objects; the image lands in device memory.
//
// Pixel (px, py), row py from the top, is the fragment at
// v_uv = ((px + 1/2) / W, (py + 1/2) / H).  The three samplers are evaluated
// in fp32 with every operation rounded on its own: the velocity field
// trilinear with clamp to edge (texel centres at i + 1/2, u rounded to
// binary16 first when round_f16, as the rgba16f image holds it), the colour
// LUT linear along t (its rows are equal), the 256 x 256 jitter LUT at texel
// centres with clamp to edge (so pixels beyond 255 repeat the edge, as the
// reference's clamp-to-edge sampler does).  exp is this file's own
// (Cody-Waite reduction, degree-7 Taylor polynomial, exact power-of-two
// scale), so the oracle can evaluate the same operations and the images
// agree bit for bit.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <string>

#include "lbm_internal.h"

namespace lbm {
namespace {

struct RenderArgs {
  float m[16];        // inverse view-projection, column-major (m[4*col + row])
  float cam[3];
  float vmin[3], vmax[3];
  int steps;
  float absorption, mag_min, mag_max, exposure;
  int round_f16;
  int width, height;
  unsigned char lut[256][3];  // colour LUT row (rgb bytes)
};

__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float dv(float a, float b) { return __fdiv_rn(a, b); }

// e^x for x <= 0: x = n ln2 + r (ln2 split in a 16-bit head and a tail),
// e^r by its Taylor series to r^7 in Horner form, times 2^n built from bits.
__device__ float exp_neg(float x) {
  if (!(x > -87.0f)) return 0.0f;
  const float n = rintf(mul(x, 1.44269502f));
  const float r = sub(sub(x, mul(n, 0.693145751953125f)), mul(n, 1.42860677e-06f));
  float p = 1.0f / 5040.0f;
  p = add(mul(p, r), 1.0f / 720.0f);
  p = add(mul(p, r), 1.0f / 120.0f);
  p = add(mul(p, r), 1.0f / 24.0f);
  p = add(mul(p, r), 1.0f / 6.0f);
  p = add(mul(p, r), 0.5f);
  p = add(mul(p, r), 1.0f);
  p = add(mul(p, r), 1.0f);
  return mul(p, __int_as_float(((int)n + 127) << 23));
}

// jitter LUT byte k: the (k+1)-th state of the LCG s' = 1664525 s + 1013904223
// from s = 0x9E3779B9, top byte; the k+1 steps composed by squaring.
__device__ unsigned jitter_byte(unsigned k) {
  unsigned A = 1u, C = 0u;              // accumulated map s -> A s + C
  unsigned a = 1664525u, c = 1013904223u;
  unsigned e = k + 1u;
  while (e) {
    if (e & 1u) { C = a * C + c; A = a * A; }
    c = a * c + c;
    a = a * a;
    e >>= 1;
  }
  return ((A * 0x9E3779B9u + C) >> 24) & 0xFFu;
}

__device__ __forceinline__ float lerp_rn(float a, float b, float t) { return add(a, mul(t, sub(b, a))); }

struct Vol {
  const float* u;
  int nx, ny, nz;
  size_t n;
  int round_f16;
};

__device__ __forceinline__ float texel(const Vol& V, int c, int i, int j, int k) {
  const float v = V.u[(size_t)c * V.n + (size_t)i + (size_t)V.nx * ((size_t)j + (size_t)V.ny * (size_t)k)];
  return V.round_f16 ? __half2float(__float2half_rn(v)) : v;
}

__device__ __forceinline__ void axis(float ctr, int N, int& i0, int& i1, float& a) {
  const float u = sub(mul(ctr, (float)N), 0.5f);
  const float f = floorf(u);
  a = sub(u, f);
  const int lo = (int)f, hi = lo + 1;
  i0 = lo < 0 ? 0 : (lo > N - 1 ? N - 1 : lo);
  i1 = hi < 0 ? 0 : (hi > N - 1 ? N - 1 : hi);
}

__device__ void sample_u(const Vol& V, float cx, float cy, float cz, float out[3]) {
  int x0, x1, y0, y1, z0, z1;
  float ax, ay, az;
  axis(cx, V.nx, x0, x1, ax);
  axis(cy, V.ny, y0, y1, ay);
  axis(cz, V.nz, z0, z1, az);
  for (int c = 0; c < 3; ++c) {
    const float c00 = lerp_rn(texel(V, c, x0, y0, z0), texel(V, c, x1, y0, z0), ax);
    const float c10 = lerp_rn(texel(V, c, x0, y1, z0), texel(V, c, x1, y1, z0), ax);
    const float c01 = lerp_rn(texel(V, c, x0, y0, z1), texel(V, c, x1, y0, z1), ax);
    const float c11 = lerp_rn(texel(V, c, x0, y1, z1), texel(V, c, x1, y1, z1), ax);
    out[c] = lerp_rn(lerp_rn(c00, c10, ay), lerp_rn(c01, c11, ay), az);
  }
}

__global__ void __launch_bounds__(256) k_velmag(Vol V, const __grid_constant__ RenderArgs R,
                                                float4* __restrict__ out) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= R.width || py >= R.height) return;
  // ray through the fragment's far-plane point
  const float ndc[4] = {sub(mul(dv(add((float)px, 0.5f), (float)R.width), 2.0f), 1.0f),
                        sub(mul(dv(add((float)py, 0.5f), (float)R.height), 2.0f), 1.0f), 1.0f, 1.0f};
  float w4[4];
  for (int r = 0; r < 4; ++r)
    w4[r] = add(add(add(mul(R.m[r], ndc[0]), mul(R.m[4 + r], ndc[1])), mul(R.m[8 + r], ndc[2])),
                mul(R.m[12 + r], ndc[3]));
  float rd[3];
  for (int c = 0; c < 3; ++c) rd[c] = sub(dv(w4[c], w4[3]), R.cam[c]);
  const float len = __fsqrt_rn(add(add(mul(rd[0], rd[0]), mul(rd[1], rd[1])), mul(rd[2], rd[2])));
  for (int c = 0; c < 3; ++c) rd[c] = dv(rd[c], len);
  // slab intersection
  float te = -INFINITY, tx = INFINITY;
  for (int c = 0; c < 3; ++c) {
    const float inv = dv(1.0f, rd[c]);
    const float t0 = mul(sub(R.vmin[c], R.cam[c]), inv);
    const float t1 = mul(sub(R.vmax[c], R.cam[c]), inv);
    te = fmaxf(te, fminf(t0, t1));
    tx = fminf(tx, fmaxf(t0, t1));
  }
  float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
  if (!(tx < te || tx < 0.0f)) {
    const float t0 = fmaxf(te, 0.0f);
    const float ray = sub(tx, t0);
    const unsigned jx = px > 255 ? 255u : (unsigned)px, jy = py > 255 ? 255u : (unsigned)py;
    const float jitter = dv((float)jitter_byte(jy * 256u + jx), 255.0f);
    const float dt = dv(ray, (float)R.steps);
    float t = add(t0, mul(jitter, dt));
    float col[3] = {0.f, 0.f, 0.f};
    float trans = 1.0f;
    float ext[3];
    for (int c = 0; c < 3; ++c) ext[c] = sub(R.vmax[c], R.vmin[c]);
    const float range = fmaxf(sub(R.mag_max, R.mag_min), 1e-6f);
    for (int i = 0; i < R.steps && trans > 0.01f; ++i) {
      float uvw[3];
      bool inside = true;
      for (int c = 0; c < 3; ++c) {
        uvw[c] = dv(sub(add(R.cam[c], mul(rd[c], t)), R.vmin[c]), ext[c]);
        inside &= uvw[c] >= 0.0f && uvw[c] <= 1.0f;
      }
      if (inside) {
        float u[3];
        sample_u(V, uvw[0], uvw[1], uvw[2], u);
        const float mag = __fsqrt_rn(add(add(mul(u[0], u[0]), mul(u[1], u[1])), mul(u[2], u[2])));
        const float t01 = fminf(fmaxf(dv(sub(mag, R.mag_min), range), 0.0f), 1.0f);
        // colour LUT: linear filter along the 256 texels, clamp to edge
        const float lu = sub(mul(t01, 256.0f), 0.5f);
        const float lf = floorf(lu);
        const float la = sub(lu, lf);
        const int l0 = lf < 0.f ? 0 : ((int)lf > 255 ? 255 : (int)lf);
        const int l1 = (int)lf + 1 < 0 ? 0 : ((int)lf + 1 > 255 ? 255 : (int)lf + 1);
        const float abs_step = mul(mul(R.absorption, dt), t01);
        for (int c = 0; c < 3; ++c) {
          const float cc = lerp_rn(dv((float)R.lut[l0][c], 255.0f), dv((float)R.lut[l1][c], 255.0f), la);
          col[c] = add(col[c], mul(mul(mul(trans, cc), abs_step), R.exposure));
        }
        trans = mul(trans, exp_neg(-abs_step));
      }
      t = add(t, dt);
    }
    o = make_float4(col[0], col[1], col[2], sub(1.0f, trans));
  }
  out[(size_t)py * R.width + px] = o;
}

}  // namespace
}  // namespace lbm

extern "C" {

int lbm_velmag_params_default(lbm_velmag_params* p) {
  if (!p) return LBM_ERR_INVALID_ARG;
  *p = lbm_velmag_params{};
  p->struct_size = sizeof(lbm_velmag_params);
  for (int i = 0; i < 16; ++i) p->inv_view_proj[i] = (i % 5 == 0) ? 1.0f : 0.0f;
  p->steps = 128;
  p->absorption = 4.0f;
  p->velmag_min = 0.0f;
  p->velmag_max = 0.1f;
  p->exposure = 1.5f;
  p->round_f16 = 1;
  p->volume_max[0] = p->volume_max[1] = p->volume_max[2] = -1.0f;  // = (Nx, Ny, Nz)
  return LBM_OK;
}

int lbm_render_velmag(const float* d_u, int32_t nx, int32_t ny, int32_t nz, const lbm_velmag_params* p,
                      int32_t width, int32_t height, float* d_rgba, void* stream) {
  if (!d_u || !p || !d_rgba || nx < 1 || ny < 1 || nz < 1 || width < 1 || height < 1) {
    lbm::set_thread_error("render velmag: bad argument");
    return LBM_ERR_INVALID_ARG;
  }
  if (p->struct_size != sizeof(lbm_velmag_params) || p->steps < 1 || p->steps > 4096) {
    lbm::set_thread_error("render velmag: bad parameters (struct_size, steps in [1, 4096])");
    return LBM_ERR_INVALID_ARG;
  }
  if ((reinterpret_cast<uintptr_t>(d_rgba) & 15u) != 0) {
    lbm::set_thread_error("render velmag: output must be 16-byte aligned (float4)");
    return LBM_ERR_INVALID_ARG;
  }
  lbm::RenderArgs R{};
  for (int i = 0; i < 16; ++i) R.m[i] = p->inv_view_proj[i];
  const float dims[3] = {(float)nx, (float)ny, (float)nz};
  for (int c = 0; c < 3; ++c) {
    R.cam[c] = p->camera_pos[c];
    R.vmin[c] = p->volume_min[c];
    R.vmax[c] = p->volume_max[c] < 0.0f ? dims[c] : p->volume_max[c];
  }
  R.steps = p->steps;
  R.absorption = p->absorption;
  R.mag_min = p->velmag_min;
  R.mag_max = p->velmag_max;
  R.exposure = p->exposure;
  R.round_f16 = p->round_f16 ? 1 : 0;
  R.width = width;
  R.height = height;
  unsigned char lut[256 * 4 * 4];
  lbm_colormap_lut(lut);
  for (int i = 0; i < 256; ++i)
    for (int c = 0; c < 3; ++c) R.lut[i][c] = lut[4 * i + c];  // row 0 (all rows equal)
  lbm::Vol V{d_u, nx, ny, nz, (size_t)nx * ny * nz, R.round_f16};
  const dim3 blk(16, 16);
  const dim3 grd((width + 15) / 16, (height + 15) / 16);
  lbm::k_velmag<<<grd, blk, 0, static_cast<cudaStream_t>(stream)>>>(V, R, reinterpret_cast<float4*>(d_rgba));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    lbm::set_thread_error((std::string("render velmag: ") + cudaGetErrorString(e)).c_str());
    return LBM_ERR_CUDA;
  }
  return LBM_OK;
}

}  // extern "C"
