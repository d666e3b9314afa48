// Device code shared by the single-domain and batched physics-mode kernels:
// storage traits, padded-grid addressing, the pair-form collision and the
// per-row esoteric-pull step.  The layout and the step are described in
// phys_kernels.cu.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "d3q19.cuh"
#include "lbm_internal.h"

namespace lbm {

constexpr float F16_SCALE = 4096.0f;
constexpr float F16_INV_SCALE = 1.0f / 4096.0f;

// Storage traits.  The step kernel works in "storage units" v = SC * g
// (SC = 1 for fp32 and bf16, 2^12 for fp16) so that loads and stores need no
// rescaling; ld/st convert to plain g for init and population transfer.
template <int PREC> struct Store;
template <> struct Store<LBM_PREC_F32> {
  using T = float;
  static constexpr float SC = 1.0f, INV = 1.0f;
  static __device__ __forceinline__ float raw_ld(const T* p, uint32_t i) { return p[i]; }
  static __device__ __forceinline__ void raw_st(T* p, uint32_t i, float v) { p[i] = v; }
  static __device__ __forceinline__ float ld(const T* p, size_t i) { return p[i]; }
  static __device__ __forceinline__ void st(T* p, size_t i, float v) { p[i] = v; }
};
template <> struct Store<LBM_PREC_F16S> {
  using T = __half;
  static constexpr float SC = F16_SCALE, INV = F16_INV_SCALE;
  static __device__ __forceinline__ float raw_ld(const T* p, uint32_t i) { return __half2float(p[i]); }
  static __device__ __forceinline__ void raw_st(T* p, uint32_t i, float v) { p[i] = __float2half_rn(v); }
  static __device__ __forceinline__ float ld(const T* p, size_t i) {
    return __half2float(p[i]) * F16_INV_SCALE;
  }
  static __device__ __forceinline__ void st(T* p, size_t i, float v) {
    p[i] = __float2half_rn(v * F16_SCALE);
  }
};
template <> struct Store<LBM_PREC_BF16S> {
  using T = __nv_bfloat16;
  static constexpr float SC = 1.0f, INV = 1.0f;
  static __device__ __forceinline__ float raw_ld(const T* p, uint32_t i) { return __bfloat162float(p[i]); }
  static __device__ __forceinline__ void raw_st(T* p, uint32_t i, float v) { p[i] = __float2bfloat16_rn(v); }
  static __device__ __forceinline__ float ld(const T* p, size_t i) { return __bfloat162float(p[i]); }
  static __device__ __forceinline__ void st(T* p, size_t i, float v) { p[i] = __float2bfloat16_rn(v); }
};

namespace {

__device__ __forceinline__ size_t lin(const PhysGeom& g, int x, int y, int z) {
  return (size_t)x + (size_t)g.px * ((size_t)(y + g.gy) + (size_t)g.py * (size_t)(z + g.gz));
}

// Padded index of n + d: periodic axes wrap, others step into the ghost layer.
template <int DX, int DY, int DZ>
__device__ __forceinline__ size_t lin_fwd(const PhysGeom& g, int x, int y, int z) {
  int xn = x + DX, yn = y + DY, zn = z + DZ;
  if (DX != 0 && g.per[0]) xn = xn >= g.nx ? xn - g.nx : xn;
  if (DY != 0 && g.per[1]) yn = yn >= g.ny ? yn - g.ny : (yn < 0 ? yn + g.ny : yn);
  if (DZ != 0 && g.per[2]) zn = zn >= g.nz ? zn - g.nz : (zn < 0 ? zn + g.nz : zn);
  return lin(g, xn, yn, zn);
}

// Moving-wall term for the population arriving in direction J after
// reflecting off the wall crossed by the link n -> n + c_opp(J).  A link that
// leaves the box through a z face takes that face's velocity, then y, then x
// (so lid edges move with the lid); a link into an interior solid sees a
// resting wall.
template <int J>
__device__ __forceinline__ float wall_term(const PhysParams& p, int x, int y, int z) {
  constexpr int K = opp(J);
  const int tx = x + cx(K), ty = y + cy(K), tz = z + cz(K);
  const PhysGeom& g = p.g;
  int face = -1;
  if (!g.per[2] && (tz < 0 || tz >= g.nz)) face = tz < 0 ? LBM_FACE_ZM : LBM_FACE_ZP;
  else if (!g.per[1] && (ty < 0 || ty >= g.ny)) face = ty < 0 ? LBM_FACE_YM : LBM_FACE_YP;
  else if (!g.per[0] && (tx < 0 || tx >= g.nx)) face = tx < 0 ? LBM_FACE_XM : LBM_FACE_XP;
  if (face < 0) return 0.0f;
  const float cu = cx(J) * p.wall[face][0] + cy(J) * p.wall[face][1] + cz(J) * p.wall[face][2];
  return 6.0f * wf(J) * cu;
}

// Collision on shifted populations in storage units v = SC (f - w), in
// place, written per opposite pair (a, b): with cu = c_a . u the equilibrium
// splits into an even part  w (drho + rho (4.5 cu^2 - 1.5 u.u))  shared by a
// and b and an odd part  3 w rho cu  with opposite signs; the Guo source
// splits into  w rho (9 cu (c_a.g) - 3 u.g)  and  3 w rho (c_a.g)  (g the
// body acceleration, F = rho g).  BGK relaxes both parts with omega; TRT the
// odd part with omega-, from Lambda = (1/omega - 1/2)(1/omega- - 1/2):
//   v_a' = (1 - h) v_a - k v_b + E + O,   v_b' = (1 - h) v_b - k v_a + E - O
// with h = (omega + omega-)/2, k = (omega - omega-)/2, E = omega even +
// (1 - omega/2) even source, O = omega- odd + (1 - omega-/2) odd source.
// Returns rho and the force-shifted velocity u = (sum c f + F/2) / rho.
template <int COLL, bool SMAG, bool FORCE, int PREC>
__device__ __forceinline__ void collide(const PhysParams& p, float (&g)[Q], float& rho_out,
                                        float& ux, float& uy, float& uz) {
  constexpr float SC = Store<PREC>::SC, INV = Store<PREC>::INV;
  constexpr float WF = 1.0f / 18.0f, WE = 1.0f / 36.0f, W0 = 1.0f / 3.0f;
  float drs = g[0], jx = 0.0f, jy = 0.0f, jz = 0.0f;  // sums in storage units
  static_for<0, 9>([&](auto PI) {
    constexpr int a = pair_a(decltype(PI)::value), b = pair_b(decltype(PI)::value);
    const float d = g[a] - g[b];
    drs += g[a] + g[b];
    if (cx(a)) jx += cx(a) * d;
    if (cy(a)) jy += cy(a) * d;
    if (cz(a)) jz += cz(a) * d;
  });
  const float rho = fmaf(drs, INV, 1.0f);
  const float js = INV / rho;
  ux = jx * js;
  uy = jy * js;
  uz = jz * js;
  if (FORCE) {
    ux = fmaf(0.5f, p.accel[0], ux);
    uy = fmaf(0.5f, p.accel[1], uy);
    uz = fmaf(0.5f, p.accel[2], uz);
  }
  rho_out = rho;
  const float uu15 = 1.5f * (ux * ux + uy * uy + uz * uz);
  const float sr = SC * rho;

  float omega = p.omega;
  if (SMAG) {
    // Pi = sum c c (f - feq) (even in c: pair sums suffice); Hou et al. (1996)
    //   tau_eff = (tau + sqrt(tau^2 + 18 sqrt(2) Cs^2 |Pi| / rho)) / 2.
    float pxx = 0.f, pyy = 0.f, pzz = 0.f, pxy = 0.f, pxz = 0.f, pyz = 0.f;
    static_for<0, 9>([&](auto PI) {
      constexpr int a = pair_a(decltype(PI)::value), b = pair_b(decltype(PI)::value);
      constexpr float w = wf(a);
      const float cu = cx(a) * ux + cy(a) * uy + cz(a) * uz;
      const float even = fmaf(w * sr, fmaf(4.5f * cu, cu, -uu15), w * drs);
      const float ne = (g[a] + g[b]) - 2.0f * even;
      if (cx(a)) pxx += ne;
      if (cy(a)) pyy += ne;
      if (cz(a)) pzz += ne;
      if (cx(a) * cy(a)) pxy += cx(a) * cy(a) * ne;
      if (cx(a) * cz(a)) pxz += cx(a) * cz(a) * ne;
      if (cy(a) * cz(a)) pyz += cy(a) * cz(a) * ne;
    });
    const float pn = INV * sqrtf(pxx * pxx + pyy * pyy + pzz * pzz +
                                 2.0f * (pxy * pxy + pxz * pxz + pyz * pyz));
    const float cs2 = p.smag_cs * p.smag_cs;
    const float tau_eff = 0.5f * (p.tau + sqrtf(fmaf(p.tau, p.tau, 25.455844f * cs2 * pn / rho)));
    omega = 1.0f / tau_eff;
  }
  const float omega_m =
      COLL == LBM_COLL_BGK ? omega : 1.0f / (p.trt_magic / (1.0f / omega - 0.5f) + 0.5f);
  const float h = 0.5f * (omega + omega_m), k = 0.5f * (omega - omega_m);
  const float c1 = 1.0f - h;
  // per weight class: omega w SC rho, omega w drs, 3 omega- w SC rho, source factors
  const float erF = omega * WF * sr, erE = omega * WE * sr;
  const float edF = omega * WF * drs, edE = omega * WE * drs;
  const float orF = 3.0f * omega_m * WF * sr, orE = 3.0f * omega_m * WE * sr;
  float ua3 = 0.f, ksF = 0.f, ksE = 0.f, kaF = 0.f, kaE = 0.f;
  if (FORCE) {
    ua3 = 3.0f * (ux * p.accel[0] + uy * p.accel[1] + uz * p.accel[2]);
    const float fp = 1.0f - 0.5f * omega, fm = 1.0f - 0.5f * omega_m;
    ksF = fp * WF * sr;
    ksE = fp * WE * sr;
    kaF = 3.0f * fm * WF * sr;
    kaE = 3.0f * fm * WE * sr;
  }
  {
    float e0 = fmaf(-omega * W0 * sr, uu15, omega * W0 * drs);
    if (FORCE) e0 = fmaf(-(1.0f - 0.5f * omega) * W0 * sr, ua3, e0);
    g[0] = fmaf(1.0f - omega, g[0], e0);
  }
  static_for<0, 9>([&](auto PI) {
    constexpr int a = pair_a(decltype(PI)::value), b = pair_b(decltype(PI)::value);
    constexpr bool face = (a <= 6);
    const float cu = cx(a) * ux + cy(a) * uy + cz(a) * uz;
    const float t = fmaf(4.5f * cu, cu, -uu15);
    float E = fmaf(face ? erF : erE, t, face ? edF : edE);
    float O = (face ? orF : orE) * cu;
    if (FORCE) {
      const float ca = cx(a) * p.accel[0] + cy(a) * p.accel[1] + cz(a) * p.accel[2];
      E = fmaf(face ? ksF : ksE, fmaf(9.0f * ca, cu, -ua3), E);
      O = fmaf(face ? kaF : kaE, ca, O);
    }
    const float ga = g[a], gb = g[b];
    if (COLL == LBM_COLL_BGK) {
      g[a] = fmaf(c1, ga, E + O);
      g[b] = fmaf(c1, gb, E - O);
    } else {
      g[a] = fmaf(c1, ga, fmaf(-k, gb, E + O));
      g[b] = fmaf(c1, gb, fmaf(-k, ga, E - O));
    }
  });
}

// Launch shape of the step kernel: a block is 32 x STEP_BY nodes of one
// z-plane, so every warp covers 32 consecutive x of one row.
#ifndef LBM_STEP_BY
#define LBM_STEP_BY 4
#endif
#ifndef LBM_STEP_MINB
#define LBM_STEP_MINB 6
#endif
constexpr int STEP_BY = LBM_STEP_BY;
constexpr int STEP_THREADS = 32 * STEP_BY;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t lin32(const PhysGeom& g, int x, int y, int z) {
  return (uint32_t)x + (uint32_t)g.px * ((uint32_t)(y + g.gy) + (uint32_t)g.py * (uint32_t)(z + g.gz));
}

template <int DX, int DY, int DZ>
__device__ __forceinline__ uint32_t lin32_fwd(const PhysGeom& g, int x, int y, int z) {
  int xn = x + DX, yn = y + DY, zn = z + DZ;
  if (DX != 0 && g.per[0]) xn = xn >= g.nx ? xn - g.nx : xn;
  if (DY != 0 && g.per[1]) yn = yn >= g.ny ? yn - g.ny : (yn < 0 ? yn + g.ny : yn);
  if (DZ != 0 && g.per[2]) zn = zn >= g.nz ? zn - g.nz : (zn < 0 ? zn + g.nz : zn);
  return lin32(g, xn, yn, zn);
}

// Padded-index offset of n + (0, DY, DZ) (X == 0) or n + (DX, DY, DZ)
// (X == 1) from n, periodic wrap included; w* are the per-node wrap terms.
struct Wrap {
  uint32_t wx, wyp, wym, wzp, wzm;
};

__device__ __forceinline__ Wrap wrap_terms(const PhysGeom& G, int x, int y, int z) {
  Wrap w;
  w.wx = (G.per[0] && x == G.nx - 1) ? (uint32_t)(-G.nx) : 0u;
  w.wyp = (G.per[1] && y == G.ny - 1) ? (uint32_t)0 - (uint32_t)G.ny * (uint32_t)G.px : 0u;
  w.wym = (G.per[1] && y == 0) ? (uint32_t)G.ny * (uint32_t)G.px : 0u;
  w.wzp = (G.per[2] && z == G.nz - 1) ? (uint32_t)0 - (uint32_t)G.nz * G.pxy : 0u;
  w.wzm = (G.per[2] && z == 0) ? (uint32_t)G.nz * G.pxy : 0u;
  return w;
}

template <int DX, int DY, int DZ>
__device__ __forceinline__ uint32_t offs(const PhysGeom& G, const Wrap& w) {
  uint32_t o = (uint32_t)DX + (uint32_t)(DY * G.px) + (uint32_t)DZ * G.pxy;
  if (DX > 0) o += w.wx;
  if (DY > 0) o += w.wyp;
  if (DY < 0) o += w.wym;
  if (DZ > 0) o += w.wzp;
  if (DZ < 0) o += w.wzm;
  return o;
}

// One fused stream+collide launch.  All lanes of a warp stay converged:
//  * the 19 slots of the streaming pattern are loaded before the flag byte
//    is known (a solid node's slots exist, so the loads are in bounds), so a
//    node costs one memory round trip, not two;
//  * the five pairs whose forward vector has cx = +1 read and write slot
//    Y at x+1.  Instead of a 4-byte-shifted warp access, every lane accesses
//    its own aligned x and the values move one lane by warp shuffle; the
//    last lane of a warp (or of a row) touches x+1 directly;
//  * boundary nodes (flag bit) then re-read the bounce-back slots.
// One warp updates nodes x0 .. x0+31 of row (y, z); y < ny (the caller's
// test is uniform over the warp).  Used by the single-domain kernel and by
// the batched kernels (phys_batch.cu).
template <int PREC, int COLL, bool SMAG, bool FORCE, bool WRITE_MOMENTS, int P>
__device__ __forceinline__ void step_row(const PhysParams& p, void* __restrict__ pop_v,
                                         const uint8_t* __restrict__ flags,
                                         const uint32_t* __restrict__ links,
                                         float* __restrict__ rho_o, float* __restrict__ u_o,
                                         unsigned* __restrict__ status, const int x0, const int y,
                                         const int z) {
  using S = Store<PREC>;
  using T = typename S::T;
  const PhysGeom& G = p.g;
  const int lane = threadIdx.x & 31;
  const int x = x0 + lane;
  const bool valid = x < G.nx;
  const int xc = valid ? x : G.nx - 1;  // in-bounds address for idle lanes
  const bool edge = (lane == 31) || (x >= G.nx - 1);  // touches x+1 itself
  const uint32_t N = (uint32_t)G.n;
  const uint32_t nid = (uint32_t)xc + (uint32_t)G.nx * ((uint32_t)y + (uint32_t)G.ny * (uint32_t)z);
  T* pop = reinterpret_cast<T*>(pop_v);
  const size_t SS = G.slot_stride;
  const uint32_t ln = lin32(G, xc, y, z);
  const Wrap w = wrap_terms(G, xc, y, z);

  // Faces of non-periodic axes at this node: links across them are half-way
  // bounce-back links known from the coordinates, so their slots are read in
  // the first batch of loads (the y and z parts are uniform over the warp).
  const bool xlo = !G.per[0] && xc == 0, xhi = !G.per[0] && xc == G.nx - 1;
  const bool ylo = !G.per[1] && y == 0, yhi = !G.per[1] && y == G.ny - 1;
  const bool zlo = !G.per[2] && z == 0, zhi = !G.per[2] && z == G.nz - 1;
  const bool moving = p.any_moving_wall;

  const uint8_t fl = valid ? flags[nid] : FLAG_SOLID;
  float g[Q];
  g[0] = S::raw_ld(pop, ln);
  static_for<0, 9>([&](auto PI) {
    constexpr int pi = decltype(PI)::value;
    constexpr int a = pair_a(pi), b = pair_b(pi);
    constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
    const T* s0 = pop + (size_t)(1 + 2 * pi) * SS;
    const T* sP = P ? s0 + SS : s0;
    const T* sQ = P ? s0 : s0 + SS;
    // n + d (forward) or n - d (backward) beyond a wall face
    const bool fyz = (DY > 0 && yhi) || (DY < 0 && ylo) || (DZ > 0 && zhi) || (DZ < 0 && zlo);
    const bool fwd_wall = fyz || (DX > 0 && xhi);
    const bool bwd_wall =
        (DX > 0 && xlo) || (DY > 0 && ylo) || (DY < 0 && yhi) || (DZ > 0 && zlo) || (DZ < 0 && zhi);
    // f_a from X = S[1-P](n), or f*_b(n) from S[P](n) across a wall
    g[a] = S::raw_ld(bwd_wall ? sP : sQ, ln);
    // f_b from Y = S[P](n+d), or f*_a(n) from S[1-P](n+d) across a wall
    if (DX == 0) {
      g[b] = S::raw_ld(fwd_wall ? sQ : sP, ln + offs<0, DY, DZ>(G, w));
    } else {
      const float own = S::raw_ld(fyz ? sQ : sP, ln + offs<0, DY, DZ>(G, w));
      float nb = __shfl_down_sync(FULL, own, 1);
      if (edge) nb = S::raw_ld(fwd_wall ? sQ : sP, ln + offs<1, DY, DZ>(G, w));
      g[b] = nb;
    }
  });
  // Moving-wall momentum terms, in a pass of their own: inside the load loop
  // even a predicated-off add would wait for its load and serialise them.
  if (moving) {
    static_for<0, 9>([&](auto PI) {
      constexpr int pi = decltype(PI)::value;
      constexpr int a = pair_a(pi), b = pair_b(pi);
      constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
      const bool fwd_wall = (DX > 0 && xhi) || (DY > 0 && yhi) || (DY < 0 && ylo) || (DZ > 0 && zhi) ||
                            (DZ < 0 && zlo);
      const bool bwd_wall =
          (DX > 0 && xlo) || (DY > 0 && ylo) || (DY < 0 && yhi) || (DZ > 0 && zlo) || (DZ < 0 && zhi);
      if (bwd_wall) g[a] = fmaf(S::SC, wall_term<a>(p, x, y, z), g[a]);
      if (fwd_wall) g[b] = fmaf(S::SC, wall_term<b>(p, x, y, z), g[b]);
    });
  }

  const bool fluid = valid && !(fl & FLAG_SOLID);
  // Links into interior solid nodes (resting walls) need the classification
  // word: a second, rare round trip.
  if (fluid && (fl & FLAG_SOLID_LINK)) {
    const uint32_t L = links[nid];
    static_for<0, 9>([&](auto PI) {
      constexpr int pi = decltype(PI)::value;
      constexpr int a = pair_a(pi), b = pair_b(pi);
      constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
      const T* s0 = pop + (size_t)(1 + 2 * pi) * SS;
      const T* sP = P ? s0 + SS : s0;
      const T* sQ = P ? s0 : s0 + SS;
      const bool fwd_wall = (DX > 0 && xhi) || (DY > 0 && yhi) || (DY < 0 && ylo) || (DZ > 0 && zhi) ||
                            (DZ < 0 && zlo);
      const bool bwd_wall =
          (DX > 0 && xlo) || (DY > 0 && ylo) || (DY < 0 && yhi) || (DZ > 0 && zlo) || (DZ < 0 && zhi);
      if (((L >> b) & 1u) && !bwd_wall) g[a] = S::raw_ld(sP, ln);
      if (((L >> a) & 1u) && !fwd_wall) g[b] = S::raw_ld(sQ, ln + offs<DX, DY, DZ>(G, w));
    });
  }

  float rho, ux, uy, uz;
  collide<COLL, SMAG, FORCE, PREC>(p, g, rho, ux, uy, uz);

  if (WRITE_MOMENTS && valid) {
    const bool s = !fluid;
    rho_o[nid] = s ? 0.0f : rho;
    u_o[nid] = s ? 0.0f : ux;
    u_o[N + nid] = s ? 0.0f : uy;
    u_o[2 * N + nid] = s ? 0.0f : uz;
    if (fluid && (!(rho > 0.0f) || !isfinite(rho) || !isfinite(ux) || !isfinite(uy) || !isfinite(uz)))
      atomicOr(status, 1u);
  }

  if (fluid) S::raw_st(pop, ln, g[0]);
  const bool pass = fluid && !edge;  // this lane's Y value is stored by lane+1
  static_for<0, 9>([&](auto PI) {
    constexpr int pi = decltype(PI)::value;
    constexpr int a = pair_a(pi), b = pair_b(pi);
    constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
    T* s0 = pop + (size_t)(1 + 2 * pi) * SS;
    T* sP = P ? s0 + SS : s0;
    T* sQ = P ? s0 : s0 + SS;
    if (fluid) S::raw_st(sQ, ln, g[b]);  // f*_b -> X = S[1-P](n)
    if (DX == 0) {
      if (fluid) S::raw_st(sP, ln + offs<0, DY, DZ>(G, w), g[a]);  // f*_a -> Y = S[P](n+d)
    } else {
      const float from_left = __shfl_up_sync(FULL, g[a], 1);
      const bool left_ok = __shfl_up_sync(FULL, pass, 1) && lane > 0;
      if (left_ok) S::raw_st(sP, ln + offs<0, DY, DZ>(G, w), from_left);
      if (fluid && edge) S::raw_st(sP, ln + offs<1, DY, DZ>(G, w), g[a]);
    }
  });
}

}  // namespace
}  // namespace lbm
