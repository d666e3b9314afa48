// Device code shared by the single-domain and batched physics-mode kernels:
// storage traits, padded-grid addressing, the pair-form collision and the
// per-row esoteric-pull step.  The layout and the step are described in
// phys_kernels.cu.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "d3q19.cuh"
#include "closure.cuh"
#include "fops.cuh"
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

// Open x face (Zou & He 1997; D3Q19 form of Hecht & Harting 2010): the five
// populations entering through the face, c_x = SX (+1 at x = 0, -1 at
// x = nx-1), rebuilt from the streamed ones before the collision:
//   rho (1 - SX u_x) = S0 + 2 Sk      (S0: c_x = 0 sum, Sk: c_x = -SX sum)
//   f_a = f_opp(a) + 6 w_a rho (c_a.u) - c_ay N_y - c_az N_z,
//   N_t = (1/2) sum_{c_x = 0} f_i c_it - rho u_t / 3,
// which returns exactly rho and rho u as the node's moments.  A VELOCITY face
// knows u and solves for rho, a PRESSURE face knows rho (u_y = u_z = 0) and
// solves for u_x.  On shifted storage v = SC (f - w) the weights cancel:
// S0 + 2 Sk = 1 + (V0 + 2 Vk) / SC and the c_t-weighted sums of w vanish.
// at(i) is the node's value of direction i.
template <int SX, class At>
__device__ __forceinline__ void zou_he(const PhysParams& p, float sc, float inv_sc, At&& at) {
  constexpr int side = SX > 0 ? 0 : 1;
  float v0 = 0.0f, vk = 0.0f, my = 0.0f, mz = 0.0f;
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    if constexpr (cx(i) == 0) {
      v0 += at(i);
      if constexpr (cy(i) != 0) my += float(cy(i)) * at(i);
      if constexpr (cz(i) != 0) mz += float(cz(i)) * at(i);
    } else if constexpr (cx(i) == -SX) {
      vk += at(i);
    }
  });
  const float dm = (v0 + 2.0f * vk) * inv_sc;  // S0 + 2 Sk - 1
  float rho, ux, uy, uz;
  if (p.open[side] == LBM_OPEN_VELOCITY) {
    ux = p.wall[side][0];
    uy = p.wall[side][1];
    uz = p.wall[side][2];
    rho = (1.0f + dm) / (1.0f - float(SX) * ux);
  } else {
    // u_x = SX (1 - (1 + dm) / rho) in deviation form: rho - 1 is exact for
    // rho in [0.5, 2], so a small u_x does not come from cancelling ~1 terms
    rho = p.open_rho[side];
    ux = float(SX) * (((rho - 1.0f) - dm) / rho);
    uy = 0.0f;
    uz = 0.0f;
  }
  const float ny = 0.5f * my - sc * rho * uy * (1.0f / 3.0f);
  const float nz = 0.5f * mz - sc * rho * uz * (1.0f / 3.0f);
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    if constexpr (cx(i) == SX) {
      const float cu = float(SX) * ux + float(cy(i)) * uy + float(cz(i)) * uz;
      at(i) = at(opp(i)) + sc * (6.0f * wf(i)) * rho * cu - float(cy(i)) * ny - float(cz(i)) * nz;
    }
  });
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
// O is Ops1 (one node) or Ops2 (two nodes in the .x/.y lanes).
template <class O, int COLL, int SGS, bool FORCE, int PREC>
__device__ __forceinline__ void collide_t(const PhysParams& p, const CloNet<SGS>& net,
                                          typename O::F (&g)[Q],
                                          typename O::F& rho_out, typename O::F& ux,
                                          typename O::F& uy, typename O::F& uz) {
  using F = typename O::F;
  constexpr float SC = Store<PREC>::SC, INV = Store<PREC>::INV;
  constexpr float WF = 1.0f / 18.0f, WE = 1.0f / 36.0f, W0 = 1.0f / 3.0f;
  F drs = g[0], jx = O::splat(0.f), jy = O::splat(0.f), jz = O::splat(0.f);
  static_for<0, 9>([&](auto PI) {
    constexpr int a = pair_a(decltype(PI)::value), b = pair_b(decltype(PI)::value);
    const F d = O::sub(g[a], g[b]);
    drs = O::add(drs, O::add(g[a], g[b]));
    if (cx(a) > 0) jx = O::add(jx, d);
    if (cy(a) > 0) jy = O::add(jy, d);
    if (cy(a) < 0) jy = O::sub(jy, d);
    if (cz(a) > 0) jz = O::add(jz, d);
    if (cz(a) < 0) jz = O::sub(jz, d);
  });
  const F rho = O::fma(drs, O::splat(INV), O::splat(1.0f));
  // 1/rho: to about 2 ulp for the 2-byte formats (far inside their error
  // against FP64; measured on B200 with fp16 storage, lid cavity 96^3 33.7 ->
  // 35.8 GLUPS, 160^3 43.1 -> 44.1, ensemble 34.8 -> 35.3); correctly rounded
  // for fp32, where the shorter division changed the register allocation at
  // the 80-register bound (spills 0-68 -> 32-272 bytes) and the channel fell
  // from 39.3 to 31.2 GLUPS
  const F js = PREC == LBM_PREC_F32 ? O::div(O::splat(INV), rho) : O::div_fast(O::splat(INV), rho);
  ux = O::mul(jx, js);
  uy = O::mul(jy, js);
  uz = O::mul(jz, js);
  if (FORCE) {
    ux = O::add(ux, O::splat(0.5f * p.accel[0]));
    uy = O::add(uy, O::splat(0.5f * p.accel[1]));
    uz = O::add(uz, O::splat(0.5f * p.accel[2]));
  }
  rho_out = rho;
  const F uu15 = O::mul(O::splat(1.5f), O::fma(ux, ux, O::fma(uy, uy, O::mul(uz, uz))));
  const F sr = O::mul(O::splat(SC), rho);

  F omega = O::splat(p.omega);
  if (SGS) {
    // Pi = sum c c (f - feq) (even in c: pair sums suffice); Hou et al. (1996)
    //   tau_eff = (tau + sqrt(tau^2 + 18 sqrt(2) Cs^2 |Pi| / rho)) / 2.
    F pxx = O::splat(0.f), pyy = pxx, pzz = pxx, pxy = pxx, pxz = pxx, pyz = pxx;
    static_for<0, 9>([&](auto PI) {
      constexpr int a = pair_a(decltype(PI)::value), b = pair_b(decltype(PI)::value);
      constexpr float w = wf(a);
      F cu = O::splat(0.f);
      if (cx(a)) cu = ux;
      if (cy(a) > 0) cu = cx(a) ? O::add(cu, uy) : uy;
      if (cy(a) < 0) cu = cx(a) ? O::sub(cu, uy) : O::sub(O::splat(0.f), uy);
      if (cz(a) > 0) cu = (cx(a) || cy(a)) ? O::add(cu, uz) : uz;
      if (cz(a) < 0) cu = (cx(a) || cy(a)) ? O::sub(cu, uz) : O::sub(O::splat(0.f), uz);
      const F t = O::fma(O::mul(O::splat(4.5f), cu), cu, O::sub(O::splat(0.f), uu15));
      const F even = O::fma(O::mul(O::splat(w), sr), t, O::mul(O::splat(w), drs));
      const F ne = O::fma(O::splat(-2.0f), even, O::add(g[a], g[b]));
      if (cx(a)) pxx = O::add(pxx, ne);
      if (cy(a)) pyy = O::add(pyy, ne);
      if (cz(a)) pzz = O::add(pzz, ne);
      if (cx(a) * cy(a) > 0) pxy = O::add(pxy, ne);
      if (cx(a) * cy(a) < 0) pxy = O::sub(pxy, ne);
      if (cx(a) * cz(a) > 0) pxz = O::add(pxz, ne);
      if (cx(a) * cz(a) < 0) pxz = O::sub(pxz, ne);
      if (cy(a) * cz(a) > 0) pyz = O::add(pyz, ne);
      if (cy(a) * cz(a) < 0) pyz = O::sub(pyz, ne);
    });
    const F off = O::fma(pxy, pxy, O::fma(pxz, pxz, O::mul(pyz, pyz)));
    const F q = O::fma(pxx, pxx, O::fma(pyy, pyy, O::fma(pzz, pzz, O::mul(O::splat(2.f), off))));
    const F pn = O::mul(O::splat(INV), O::sqrt(q));
    const float cs2 = p.smag_cs * p.smag_cs;
    F k2 = O::splat(25.455844f * cs2);
    if constexpr (SGS >= 2) {
      // learned closure: Cs^2 = Cs0^2 r(features of Pi, rho)
      const F P[6] = {O::mul(O::splat(INV), pxx), O::mul(O::splat(INV), pyy),
                      O::mul(O::splat(INV), pzz), O::mul(O::splat(INV), pxy),
                      O::mul(O::splat(INV), pxz), O::mul(O::splat(INV), pyz)};
      F xin[CLO_IN];
      closure_features<O>(P, rho, xin);
      if constexpr (SGS == 2) k2 = O::mul(k2, closure_mlp<O>(net, xin));
      else k2 = O::mul(k2, closure_mlp_tc(net, xin));  // one node per thread (Ops1)
    }
    const F arg = O::fma(O::splat(p.tau), O::splat(p.tau), O::div(O::mul(k2, pn), rho));
    const F tau_eff = O::mul(O::splat(0.5f), O::add(O::splat(p.tau), O::sqrt(arg)));
    omega = O::div(O::splat(1.0f), tau_eff);
  }
  F omega_m = omega;
  if (COLL == LBM_COLL_TRT && SGS == 0)
    omega_m = O::splat(p.omega_m);  // the same operations, done once on the host
  else if (COLL == LBM_COLL_TRT)
    omega_m = O::div(O::splat(1.0f),
                     O::add(O::div(O::splat(p.trt_magic),
                                   O::sub(O::div(O::splat(1.0f), omega), O::splat(0.5f))),
                            O::splat(0.5f)));
  const F h = O::mul(O::splat(0.5f), O::add(omega, omega_m));
  const F k = O::mul(O::splat(0.5f), O::sub(omega, omega_m));
  const F c1 = O::sub(O::splat(1.0f), h);
  // per weight class: omega w SC rho, omega w drs, 3 omega- w SC rho
  const F osr = O::mul(omega, sr), ods = O::mul(omega, drs), omsr = O::mul(omega_m, sr);
  const F erF = O::mul(O::splat(WF), osr), erE = O::mul(O::splat(WE), osr);
  const F edF = O::mul(O::splat(WF), ods), edE = O::mul(O::splat(WE), ods);
  const F orF = O::mul(O::splat(3.0f * WF), omsr), orE = O::mul(O::splat(3.0f * WE), omsr);
  F ua3 = O::splat(0.f), ksF = ua3, ksE = ua3, kaF = ua3, kaE = ua3;
  if (FORCE) {
    ua3 = O::mul(O::splat(3.0f),
                 O::fma(ux, O::splat(p.accel[0]), O::fma(uy, O::splat(p.accel[1]),
                                                        O::mul(uz, O::splat(p.accel[2])))));
    const F fpsr = O::mul(O::fma(O::splat(-0.5f), omega, O::splat(1.0f)), sr);
    const F fmsr = O::mul(O::fma(O::splat(-0.5f), omega_m, O::splat(1.0f)), sr);
    ksF = O::mul(O::splat(WF), fpsr);
    ksE = O::mul(O::splat(WE), fpsr);
    kaF = O::mul(O::splat(3.0f * WF), fmsr);
    kaE = O::mul(O::splat(3.0f * WE), fmsr);
  }
  {
    F e0 = O::fma(O::sub(O::splat(0.f), O::mul(O::splat(W0), osr)), uu15, O::mul(O::splat(W0), ods));
    if (FORCE)
      e0 = O::fma(O::sub(O::splat(0.f), O::mul(O::splat(W0), O::mul(O::fma(O::splat(-0.5f), omega,
                                                                          O::splat(1.0f)), sr))),
                  ua3, e0);
    g[0] = O::fma(O::sub(O::splat(1.0f), omega), g[0], e0);
  }
  static_for<0, 9>([&](auto PI) {
    constexpr int a = pair_a(decltype(PI)::value), b = pair_b(decltype(PI)::value);
    constexpr bool face = (a <= 6);
    F cu = O::splat(0.f);
    if (cx(a)) cu = ux;
    if (cy(a) > 0) cu = cx(a) ? O::add(cu, uy) : uy;
    if (cy(a) < 0) cu = cx(a) ? O::sub(cu, uy) : O::sub(O::splat(0.f), uy);
    if (cz(a) > 0) cu = (cx(a) || cy(a)) ? O::add(cu, uz) : uz;
    if (cz(a) < 0) cu = (cx(a) || cy(a)) ? O::sub(cu, uz) : O::sub(O::splat(0.f), uz);
    const F t = O::fma(O::mul(O::splat(4.5f), cu), cu, O::sub(O::splat(0.f), uu15));
    F E = O::fma(face ? erF : erE, t, face ? edF : edE);
    F Od = O::mul(face ? orF : orE, cu);
    if (FORCE) {
      const float ca = cx(a) * p.accel[0] + cy(a) * p.accel[1] + cz(a) * p.accel[2];
      E = O::fma(face ? ksF : ksE, O::fma(O::splat(9.0f * ca), cu, O::sub(O::splat(0.f), ua3)), E);
      Od = O::fma(face ? kaF : kaE, O::splat(ca), Od);
    }
    const F ga = g[a], gb = g[b];
    if (COLL == LBM_COLL_BGK) {
      g[a] = O::fma(c1, ga, O::add(E, Od));
      g[b] = O::fma(c1, gb, O::sub(E, Od));
    } else {
      const F mk = O::sub(O::splat(0.f), k);
      g[a] = O::fma(c1, ga, O::fma(mk, gb, O::add(E, Od)));
      g[b] = O::fma(c1, gb, O::fma(mk, ga, O::sub(E, Od)));
    }
  });
}

template <int COLL, int SGS, bool FORCE, int PREC>
__device__ __forceinline__ void collide(const PhysParams& p, const CloNet<SGS>& net, float (&g)[Q],
                                        float& rho_out, float& ux, float& uy, float& uz) {
  collide_t<Ops1, COLL, SGS, FORCE, PREC>(p, net, g, rho_out, ux, uy, uz);
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

// Moving-wall pass gate: a node gets momentum terms only through a link that
// leaves through a moving face, so only nodes on such a face run the pass
// (p.any_moving_wall holds bit f for each moving face f).  x_lo / x_hi are
// the node group's first and last x.
__device__ __forceinline__ bool near_moving(const PhysParams& p, int x_lo, int x_hi, int y, int z) {
  const int m = p.any_moving_wall;
  const PhysGeom& G = p.g;
  return ((m & (1 << LBM_FACE_XM)) && !G.per[0] && x_lo == 0) ||
         ((m & (1 << LBM_FACE_XP)) && !G.per[0] && x_hi == G.nx - 1) ||
         ((m & (1 << LBM_FACE_YM)) && !G.per[1] && y == 0) ||
         ((m & (1 << LBM_FACE_YP)) && !G.per[1] && y == G.ny - 1) ||
         ((m & (1 << LBM_FACE_ZM)) && !G.per[2] && z == 0) ||
         ((m & (1 << LBM_FACE_ZP)) && !G.per[2] && z == G.nz - 1);
}

// Index of pair pi among the five pairs with c_x = +1 (pairs 0, 3, 4, 5, 6).
__host__ __device__ constexpr int xpair_slot(int pi) {
  int k = 0;
  for (int q = 0; q < pi; ++q) k += cx(pair_a(q)) > 0 ? 1 : 0;
  return k;
}
static_assert(xpair_slot(8) == 5 && cx(pair_a(6)) > 0 && xpair_slot(6) == 4, "five c_x = +1 pairs");

// A node of step_row between its two phases: the raw stored values of its
// 19 slots (not yet converted, shuffled or used, so the loads can still be in
// flight), the raw values an edge lane loads at x+1 for the five c_x = +1
// pairs, and the node's addressing.
template <int PREC>
struct RowNode {
  using T = typename Store<PREC>::T;
  T raw[Q];
  T edge_raw[5];
  uint8_t fl;
  bool valid, edge;
  int x, xc;
  uint32_t nid, ln;
  Wrap w;
};

// Load phase of step_row: the flag byte and every slot of the node's
// streaming pattern, nothing that consumes a loaded value.  A caller may
// issue the loads of the next plane before it finishes this one (each slot
// is read and written by exactly one node per launch, so the two planes'
// accesses never overlap).
template <int PREC, int P, bool FACE>
__device__ __forceinline__ void row_load(const PhysParams& p, bool row_ok, const void* __restrict__ pop_v,
                                         const uint8_t* __restrict__ flags, const int x0, const int y,
                                         const int z, const bool lane_ok, RowNode<PREC>& r) {
  using T = typename Store<PREC>::T;
  const PhysGeom& G = p.g;
  const int lane = threadIdx.x & 31;
  r.x = FACE ? x0 : x0 + lane;
  r.valid = FACE ? lane_ok : r.x < G.nx && row_ok;
  r.xc = r.x < G.nx ? r.x : G.nx - 1;  // in-bounds address for idle lanes
  r.edge = FACE || (lane == 31) || (r.x >= G.nx - 1);  // touches x+1 itself
  r.nid = (uint32_t)r.xc + (uint32_t)G.nx * ((uint32_t)y + (uint32_t)G.ny * (uint32_t)z);
  const T* pop = reinterpret_cast<const T*>(pop_v);
  const size_t SS = G.slot_stride;
  r.ln = lin32(G, r.xc, y, z);
  r.w = wrap_terms(G, r.xc, y, z);
  const uint32_t ln = r.ln;
  const Wrap& w = r.w;
  // Faces of non-periodic axes at this node: links across them are half-way
  // bounce-back links known from the coordinates, so their slots are read in
  // the first batch of loads (the y and z parts are uniform over the warp).
  const bool xlo = !G.per[0] && r.xc == 0, xhi = !G.per[0] && r.xc == G.nx - 1;
  const bool ylo = !G.per[1] && y == 0, yhi = !G.per[1] && y == G.ny - 1;
  const bool zlo = !G.per[2] && z == 0, zhi = !G.per[2] && z == G.nz - 1;
  r.fl = r.valid ? flags[r.nid] : FLAG_SOLID;
  r.raw[0] = pop[ln];
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
    r.raw[a] = (bwd_wall ? sP : sQ)[ln];
    // f_b from Y = S[P](n+d), or f*_a(n) from S[1-P](n+d) across a wall; the
    // c_x = +1 pairs read their own x here (the next lane's value arrives by
    // shuffle in the second phase) and an edge lane reads x+1 as well
    if (DX == 0) {
      r.raw[b] = (fwd_wall ? sQ : sP)[ln + offs<0, DY, DZ>(G, w)];
    } else {
      constexpr int k = xpair_slot(pi);
      r.raw[b] = (fyz ? sQ : sP)[ln + offs<0, DY, DZ>(G, w)];
      if (r.edge) r.edge_raw[k] = (fwd_wall ? sQ : sP)[ln + offs<1, DY, DZ>(G, w)];
    }
  });
}

// The raw values of a deferred load (row_load) in float storage units, with
// the c_x = +1 pairs' x+1 values shuffled in from the next lane.
template <int PREC>
__device__ __forceinline__ void row_convert(const RowNode<PREC>& r, float (&g)[Q]) {
  using T = typename Store<PREC>::T;
  auto cvt = [](T v) -> float {
    if constexpr (PREC == LBM_PREC_F32) return v;
    else if constexpr (PREC == LBM_PREC_F16S) return __half2float(v);
    else return __bfloat162float(v);
  };
  g[0] = cvt(r.raw[0]);
  static_for<0, 9>([&](auto PI) {
    constexpr int pi = decltype(PI)::value;
    constexpr int a = pair_a(pi), b = pair_b(pi);
    g[a] = cvt(r.raw[a]);
    if constexpr (cx(a) == 0) {
      g[b] = cvt(r.raw[b]);
    } else {
      constexpr int k = xpair_slot(pi);
      float nb = __shfl_down_sync(FULL, cvt(r.raw[b]), 1);
      if (r.edge) nb = cvt(r.edge_raw[k]);
      g[b] = nb;
    }
  });
}

// Second phase of a node's step, from its streamed values g (float storage
// units): the moving-wall and solid-link corrections, the Zou-He faces, the
// collision, the moments and the stores.  r supplies the addressing (its
// raw values are not used).
template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P, bool FACE>
__device__ __forceinline__ void row_finish(const PhysParams& p, const CloNet<SGS>& net,
                                           void* __restrict__ pop_v,
                                           const uint32_t* __restrict__ links,
                                           float* __restrict__ rho_o, float* __restrict__ u_o,
                                           unsigned* __restrict__ status, const int y, const int z,
                                           const RowNode<PREC>& r, float (&g)[Q]) {
  using S = Store<PREC>;
  using T = typename S::T;
  const PhysGeom& G = p.g;
  const int lane = threadIdx.x & 31;
  const int x = r.x, xc = r.xc;
  const bool valid = r.valid, edge = r.edge;
  const uint32_t N = (uint32_t)G.n;
  const uint32_t nid = r.nid, ln = r.ln;
  const Wrap& w = r.w;
  const uint8_t fl = r.fl;
  T* pop = reinterpret_cast<T*>(pop_v);
  const size_t SS = G.slot_stride;
  const bool xlo = !G.per[0] && xc == 0, xhi = !G.per[0] && xc == G.nx - 1;
  const bool ylo = !G.per[1] && y == 0, yhi = !G.per[1] && y == G.ny - 1;
  const bool zlo = !G.per[2] && z == 0, zhi = !G.per[2] && z == G.nz - 1;
  const bool moving = p.any_moving_wall;

  // Moving-wall momentum terms, in a pass of their own: inside the load loop
  // even a predicated-off add would wait for its load and serialise them.
  if (moving && near_moving(p, xc, xc, y, z)) {
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

  const bool fluid = valid && !(fl & (FACE ? FLAG_SOLID : FLAG_SKIP));
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

  if constexpr (FACE) {
    if (fluid && xlo && p.open[0] != LBM_OPEN_NONE)
      zou_he<1>(p, S::SC, S::INV, [&](int i) -> float& { return g[i]; });
    if (fluid && xhi && p.open[1] != LBM_OPEN_NONE)
      zou_he<-1>(p, S::SC, S::INV, [&](int i) -> float& { return g[i]; });
  }

  float rho, ux, uy, uz;
  collide<COLL, SGS, FORCE, PREC>(p, net, g, rho, ux, uy, uz);

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
//
// FACE: the open-face variant.  Each lane updates its own node (x0, y, z)
// with every neighbour slot accessed directly (no shuffles), lane_ok false
// for idle lanes, and the Zou-He reconstruction before the collision.  The
// row kernels skip these nodes (FLAG_OPEN); the two sets of nodes read and
// write disjoint slots, so the face kernel may run after them.
template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P, bool FACE = false>
__device__ __forceinline__ void step_row(const PhysParams& p, const CloNet<SGS>& net,
                                         void* __restrict__ pop_v,
                                         const uint8_t* __restrict__ flags,
                                         const uint32_t* __restrict__ links,
                                         float* __restrict__ rho_o, float* __restrict__ u_o,
                                         unsigned* __restrict__ status, const int x0, const int y,
                                         const int z, const bool lane_ok = true) {
  using S = Store<PREC>;
  using T = typename S::T;
  const PhysGeom& G = p.g;
  const int lane = threadIdx.x & 31;
  bool row_ok = true;  // y < ny; only the tensor-core closure runs rows beyond
  if constexpr (SGS == 3) row_ok = net.row_ok;
  RowNode<PREC> r;
  r.x = FACE ? x0 : x0 + lane;
  r.valid = FACE ? lane_ok : r.x < G.nx && row_ok;
  r.xc = r.x < G.nx ? r.x : G.nx - 1;  // in-bounds address for idle lanes
  r.edge = FACE || (lane == 31) || (r.x >= G.nx - 1);  // touches x+1 itself
  r.nid = (uint32_t)r.xc + (uint32_t)G.nx * ((uint32_t)y + (uint32_t)G.ny * (uint32_t)z);
  T* pop = reinterpret_cast<T*>(pop_v);
  const size_t SS = G.slot_stride;
  r.ln = lin32(G, r.xc, y, z);
  r.w = wrap_terms(G, r.xc, y, z);
  const uint32_t ln = r.ln;
  const Wrap& w = r.w;
  const bool edge = r.edge;

  // Faces of non-periodic axes at this node: links across them are half-way
  // bounce-back links known from the coordinates, so their slots are read in
  // the first batch of loads (the y and z parts are uniform over the warp).
  const bool xlo = !G.per[0] && r.xc == 0, xhi = !G.per[0] && r.xc == G.nx - 1;
  const bool ylo = !G.per[1] && y == 0, yhi = !G.per[1] && y == G.ny - 1;
  const bool zlo = !G.per[2] && z == 0, zhi = !G.per[2] && z == G.nz - 1;

  r.fl = r.valid ? flags[r.nid] : FLAG_SOLID;
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
  row_finish<PREC, COLL, SGS, FORCE, WRITE_MOMENTS, P, FACE>(p, net, pop_v, links, rho_o, u_o, status, y,
                                                             z, r, g);
}

// Two nodes per thread (step_row2) need an even row length, so that pairs
// never straddle a row and vector accesses stay aligned, and pay off when the
// rows fill the 64-wide warps: measured on B200 a two-node lane does the work
// of about 1.25 one-node lanes, so pairs are used when
// 1.25 * nx / (64 ceil(nx/64)) >= nx / (32 ceil(nx/32)).
__host__ __device__ inline bool step_pairs(int nx) {
#ifdef LBM_NO_PAIRS
  return false;
#else
  if (nx % 2) return false;
  const int w64 = 64 * ((nx + 63) / 64), w32 = 32 * ((nx + 31) / 32);
  return 5 * w32 >= 4 * w64;
#endif
}

// Four nodes per thread (step_row4, 2-byte formats) need nx % 4 == 0.  They
// are not chosen automatically: measured on B200 on the 512 x 128 x 128
// channel, fp16 runs at 46.8 GLUPS with four nodes per thread (167 registers,
// three 128-thread blocks per SM) against 50.2 with two, so the automatic
// choice stays at two; lbm_set_step_variant(ctx, 4) selects them.
__host__ __device__ inline bool step_quads(int nx) {
#ifdef LBM_AUTO_QUADS
  return nx % 4 == 0;
#else
  (void)nx;
  return false;
#endif
}

// Vector access to two x-adjacent slots (x even, so 8- or 4-byte aligned).
template <int PREC> struct Vec2;
template <> struct Vec2<LBM_PREC_F32> {
  using V = float2;
  static __device__ __forceinline__ V ld(const float* p, uint32_t i) { return *reinterpret_cast<const float2*>(p + i); }
  static __device__ __forceinline__ void st(float* p, uint32_t i, float a, float b) {
    *reinterpret_cast<float2*>(p + i) = make_float2(a, b);
  }
  static __device__ __forceinline__ float lo(V v) { return v.x; }
  static __device__ __forceinline__ float hi(V v) { return v.y; }
};
template <> struct Vec2<LBM_PREC_F16S> {
  using V = __half2;
  static __device__ __forceinline__ V ld(const __half* p, uint32_t i) { return *reinterpret_cast<const __half2*>(p + i); }
  static __device__ __forceinline__ void st(__half* p, uint32_t i, float a, float b) {
    *reinterpret_cast<__half2*>(p + i) = __floats2half2_rn(a, b);
  }
  static __device__ __forceinline__ float lo(V v) { return __low2float(v); }
  static __device__ __forceinline__ float hi(V v) { return __high2float(v); }
};
template <> struct Vec2<LBM_PREC_BF16S> {
  using V = __nv_bfloat162;
  static __device__ __forceinline__ V ld(const __nv_bfloat16* p, uint32_t i) {
    return *reinterpret_cast<const __nv_bfloat162*>(p + i);
  }
  static __device__ __forceinline__ void st(__nv_bfloat16* p, uint32_t i, float a, float b) {
    *reinterpret_cast<__nv_bfloat162*>(p + i) = __floats2bfloat162_rn(a, b);
  }
  static __device__ __forceinline__ float lo(V v) { return __low2float(v); }
  static __device__ __forceinline__ float hi(V v) { return __high2float(v); }
};

// The step of step_row for two nodes per thread: lane l of the warp updates
// x = x0 + 2l (node A) and x + 1 (node B) (nx even, so both exist or neither
// does); a warp covers 64 consecutive x.  Every slot pair (x, x+1) moves as
// one vector access; the slots at x+1 / x+2 of the c_x = +1 pairs come from
// the lane's own vector and the next lane's by shuffle, the row's last pair
// touching x+2 itself.  The two nodes collide together in the lanes of
// packed fp32 instructions (Ops2).  Solid nodes are never written (their
// slots hold neighbours' bounce-back values), so a pair with a solid node
// stores element-wise.
template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P>
__device__ __forceinline__ void step_row2(const PhysParams& p, const CloNet<SGS>& net,
                                          void* __restrict__ pop_v,
                                          const uint8_t* __restrict__ flags,
                                          const uint32_t* __restrict__ links,
                                          float* __restrict__ rho_o, float* __restrict__ u_o,
                                          unsigned* __restrict__ status, const int x0, const int y,
                                          const int z) {
  using S = Store<PREC>;
  using V2 = Vec2<PREC>;
  using T = typename S::T;
  const PhysGeom& G = p.g;
  const int lane = threadIdx.x & 31;
  const int xa = x0 + 2 * lane;
  const bool valid = xa < G.nx;
  const int xc = valid ? xa : G.nx - 2;
  const bool edge = (lane == 31) || (xa + 2 >= G.nx);  // its node B touches x+2 itself
  const uint32_t N = (uint32_t)G.n;
  const uint32_t nid = (uint32_t)xc + (uint32_t)G.nx * ((uint32_t)y + (uint32_t)G.ny * (uint32_t)z);
  T* pop = reinterpret_cast<T*>(pop_v);
  const size_t SS = G.slot_stride;
  const uint32_t lnA = lin32(G, xc, y, z);
  const uint32_t lnB = lnA + 1;
  const Wrap w = wrap_terms(G, xc, y, z);       // y/z terms; node A is never at x = nx-1
  const Wrap wB = wrap_terms(G, xc + 1, y, z);  // x term of node B
  const bool xloA = !G.per[0] && xc == 0, xhiB = !G.per[0] && xc + 1 == G.nx - 1;
  const bool ylo = !G.per[1] && y == 0, yhi = !G.per[1] && y == G.ny - 1;
  const bool zlo = !G.per[2] && z == 0, zhi = !G.per[2] && z == G.nz - 1;
  const bool moving = p.any_moving_wall;

  const uint16_t fl2 = valid ? *reinterpret_cast<const uint16_t*>(flags + nid) : (uint16_t)0x0101u;
  const uint8_t flA = (uint8_t)(fl2 & 0xffu), flB = (uint8_t)(fl2 >> 8);
  float2 g2[Q];  // .x = node A, .y = node B
  {
    const typename V2::V r = V2::ld(pop, lnA);
    g2[0] = make_float2(V2::lo(r), V2::hi(r));
  }
  static_for<0, 9>([&](auto PI) {
    constexpr int pi = decltype(PI)::value;
    constexpr int a = pair_a(pi), b = pair_b(pi);
    constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
    const T* s0 = pop + (size_t)(1 + 2 * pi) * SS;
    const T* sP = P ? s0 + SS : s0;
    const T* sQ = P ? s0 : s0 + SS;
    const bool yz_fwd = (DY > 0 && yhi) || (DY < 0 && ylo) || (DZ > 0 && zhi) || (DZ < 0 && zlo);
    const bool yz_bwd = (DY > 0 && ylo) || (DY < 0 && yhi) || (DZ > 0 && zlo) || (DZ < 0 && zhi);
    // f_a of both nodes from X = S[1-P](x, x+1); S[P] across a wall
    const typename V2::V xv = V2::ld(yz_bwd ? sP : sQ, lnA);
    g2[a] = make_float2(V2::lo(xv), V2::hi(xv));
    if (DX > 0 && xloA) g2[a].x = S::raw_ld(sP, lnA);  // node A at the -x wall
    // f_b from Y = S[P](n + d); S[1-P] across a wall
    const typename V2::V yv = V2::ld(yz_fwd ? sQ : sP, lnA + offs<0, DY, DZ>(G, w));
    if (DX == 0) {
      g2[b] = make_float2(V2::lo(yv), V2::hi(yv));
    } else {
      float nxt = __shfl_down_sync(FULL, V2::lo(yv), 1);  // x + 2
      if (edge) nxt = S::raw_ld((yz_fwd || xhiB) ? sQ : sP, lnB + offs<1, DY, DZ>(G, wB));
      g2[b] = make_float2(V2::hi(yv), nxt);  // x + 1, x + 2
    }
  });
  if (moving && near_moving(p, xc, xc + 1, y, z)) {
    static_for<0, 9>([&](auto PI) {
      constexpr int pi = decltype(PI)::value;
      constexpr int a = pair_a(pi), b = pair_b(pi);
      constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
      const bool yz_fwd = (DY > 0 && yhi) || (DY < 0 && ylo) || (DZ > 0 && zhi) || (DZ < 0 && zlo);
      const bool yz_bwd = (DY > 0 && ylo) || (DY < 0 && yhi) || (DZ > 0 && zlo) || (DZ < 0 && zhi);
      if (yz_bwd || (DX > 0 && xloA)) g2[a].x = fmaf(S::SC, wall_term<a>(p, xc, y, z), g2[a].x);
      if (yz_fwd) g2[b].x = fmaf(S::SC, wall_term<b>(p, xc, y, z), g2[b].x);
      if (yz_bwd) g2[a].y = fmaf(S::SC, wall_term<a>(p, xc + 1, y, z), g2[a].y);
      if (yz_fwd || (DX > 0 && xhiB)) g2[b].y = fmaf(S::SC, wall_term<b>(p, xc + 1, y, z), g2[b].y);
    });
  }
  const bool fluidA = valid && !(flA & FLAG_SKIP);
  const bool fluidB = valid && !(flB & FLAG_SKIP);
  auto solid_fix = [&](auto lane_sel, uint32_t nidn, uint32_t ln, const Wrap& wn, bool xlo, bool xhi) {
    constexpr bool B = decltype(lane_sel)::value != 0;
    auto at = [&](int i) -> float& { return B ? g2[i].y : g2[i].x; };
    const uint32_t L = links[nidn];
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
      if (((L >> b) & 1u) && !bwd_wall) at(a) = S::raw_ld(sP, ln);
      if (((L >> a) & 1u) && !fwd_wall) at(b) = S::raw_ld(sQ, ln + offs<DX, DY, DZ>(G, wn));
    });
  };
  if (fluidA && (flA & FLAG_SOLID_LINK)) solid_fix(IC<0>{}, nid, lnA, w, xloA, false);
  if (fluidB && (flB & FLAG_SOLID_LINK)) solid_fix(IC<1>{}, nid + 1, lnB, wB, false, xhiB);

  float2 r2, ux2, uy2, uz2;
  collide_t<Ops2, COLL, SGS, FORCE, PREC>(p, net, g2, r2, ux2, uy2, uz2);

  if (WRITE_MOMENTS && valid) {
    *reinterpret_cast<float2*>(rho_o + nid) = make_float2(fluidA ? r2.x : 0.f, fluidB ? r2.y : 0.f);
    *reinterpret_cast<float2*>(u_o + nid) = make_float2(fluidA ? ux2.x : 0.f, fluidB ? ux2.y : 0.f);
    *reinterpret_cast<float2*>(u_o + N + nid) = make_float2(fluidA ? uy2.x : 0.f, fluidB ? uy2.y : 0.f);
    *reinterpret_cast<float2*>(u_o + 2 * N + nid) = make_float2(fluidA ? uz2.x : 0.f, fluidB ? uz2.y : 0.f);
    const bool badA = fluidA && (!(r2.x > 0.f) || !isfinite(r2.x) || !isfinite(ux2.x) ||
                                 !isfinite(uy2.x) || !isfinite(uz2.x));
    const bool badB = fluidB && (!(r2.y > 0.f) || !isfinite(r2.y) || !isfinite(ux2.y) ||
                                 !isfinite(uy2.y) || !isfinite(uz2.y));
    if (badA || badB) atomicOr(status, 1u);
  }

  const bool both = fluidA && fluidB;
  const bool passB = fluidB && !edge;  // node B's Y value at x+2 is stored by lane+1
  // The store phase is compiled twice: FAST for warps whose every pair stores
  // both nodes (a warp-uniform vote), with plain vector stores, and the
  // general form for the rest (measured on B200, channel 512x128x128: fp32
  // 37.4 GLUPS against 36.2; fp16 with one-warp blocks 53.7 against 52.0).
  auto stores = [&](auto fast_tag) {
    constexpr bool FAST = decltype(fast_tag)::value != 0;
    // store node A / node B values at slot positions i (A) and i+1 (B)
    auto st2 = [&](T* arr, uint32_t i, float va, float vb) {
      if (FAST || both) V2::st(arr, i, va, vb);
      else {
        if (fluidA) S::raw_st(arr, i, va);
        if (fluidB) S::raw_st(arr, i + 1, vb);
      }
    };
    st2(pop, lnA, g2[0].x, g2[0].y);
    static_for<0, 9>([&](auto PI) {
      constexpr int pi = decltype(PI)::value;
      constexpr int a = pair_a(pi), b = pair_b(pi);
      constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
      T* s0 = pop + (size_t)(1 + 2 * pi) * SS;
      T* sP = P ? s0 + SS : s0;
      T* sQ = P ? s0 : s0 + SS;
      st2(sQ, lnA, g2[b].x, g2[b].y);  // f*_b -> X = S[1-P](n)
      if (DX == 0) {
        st2(sP, lnA + offs<0, DY, DZ>(G, w), g2[a].x, g2[a].y);  // f*_a -> Y = S[P](n+d)
      } else {
        const float from_left = __shfl_up_sync(FULL, g2[a].y, 1);
        const bool left_ok = __shfl_up_sync(FULL, passB, 1) && lane > 0;
        const uint32_t i = lnA + offs<0, DY, DZ>(G, w);
        if (left_ok && fluidA) V2::st(sP, i, from_left, g2[a].x);
        else {
          if (left_ok) S::raw_st(sP, i, from_left);
          if (fluidA) S::raw_st(sP, i + 1, g2[a].x);
        }
        if (fluidB && edge) S::raw_st(sP, lnB + offs<1, DY, DZ>(G, wB), g2[a].y);
      }
    });
  };
#ifndef LBM_VOTE_STORES16
#define LBM_VOTE_STORES16 1
#endif
  if constexpr (PREC == LBM_PREC_F32 || LBM_VOTE_STORES16) {
    if (__all_sync(FULL, both)) stores(IC<1>{});
    else stores(IC<0>{});
  } else {
    stores(IC<0>{});
  }
}


// Four x-adjacent 2-byte slots as one 8-byte access (x a multiple of 4).
template <int PREC> struct Vec4;
template <> struct Vec4<LBM_PREC_F32> {  // one 16-byte access per slot quad
  using T = float;
  static __device__ __forceinline__ float4 ld(const T* p, uint32_t i) {
    return *reinterpret_cast<const float4*>(p + i);
  }
  static __device__ __forceinline__ float2 lo(float4 v) { return make_float2(v.x, v.y); }
  static __device__ __forceinline__ float2 hi(float4 v) { return make_float2(v.z, v.w); }
  static __device__ __forceinline__ void st(T* p, uint32_t i, float2 l, float2 h) {
    *reinterpret_cast<float4*>(p + i) = make_float4(l.x, l.y, h.x, h.y);
  }
};
template <> struct Vec4<LBM_PREC_F16S> {
  using T = __half;
  static __device__ __forceinline__ uint2 ld(const T* p, uint32_t i) { return *reinterpret_cast<const uint2*>(p + i); }
  static __device__ __forceinline__ float2 lo(uint2 v) { return __half22float2(*reinterpret_cast<const __half2*>(&v.x)); }
  static __device__ __forceinline__ float2 hi(uint2 v) { return __half22float2(*reinterpret_cast<const __half2*>(&v.y)); }
  static __device__ __forceinline__ uint32_t pack(float2 f) {
    const __half2 h = __float22half2_rn(f);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
  static __device__ __forceinline__ void st(T* p, uint32_t i, float2 l, float2 h) {
    *reinterpret_cast<uint2*>(p + i) = make_uint2(pack(l), pack(h));
  }
};
template <> struct Vec4<LBM_PREC_BF16S> {
  using T = __nv_bfloat16;
  static __device__ __forceinline__ uint2 ld(const T* p, uint32_t i) { return *reinterpret_cast<const uint2*>(p + i); }
  static __device__ __forceinline__ float2 lo(uint2 v) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.x));
  }
  static __device__ __forceinline__ float2 hi(uint2 v) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.y));
  }
  static __device__ __forceinline__ uint32_t pack(float2 f) {
    const __nv_bfloat162 h = __float22bfloat162_rn(f);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
  static __device__ __forceinline__ void st(T* p, uint32_t i, float2 l, float2 h) {
    *reinterpret_cast<uint2*>(p + i) = make_uint2(pack(l), pack(h));
  }
};

// Four nodes per thread, nx a multiple of 4: lane l updates x = x0 + 4l ..
// x + 3 (nodes A, B, C, D); a warp covers 128 consecutive x.  The same scheme
// as step_row2 with 8-byte (2-byte formats) or 16-byte (fp32) accesses:
// every slot quad moves as one access (x = 4l and rows padded to multiples of
// 8 slots keep it aligned), the slots at
// x+1 .. x+4 of the c_x = +1 pairs come from the lane's own vector and the
// next lane's first element by one shuffle, the row's last quad touching
// x+4 itself; A+B and C+D collide as two packed pairs (Ops2), so results are
// bit-identical to the one- and two-node kernels.  Per node, the address,
// flag and wall arithmetic is shared four ways instead of two, which is what
// the issue-bound 2-byte kernel needs.
template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P>
__device__ __forceinline__ void step_row4(const PhysParams& p, const CloNet<SGS>& net,
                                          void* __restrict__ pop_v,
                                          const uint8_t* __restrict__ flags,
                                          const uint32_t* __restrict__ links,
                                          float* __restrict__ rho_o, float* __restrict__ u_o,
                                          unsigned* __restrict__ status, const int x0, const int y,
                                          const int z) {
  using S = Store<PREC>;
  using V4 = Vec4<PREC>;
  using T = typename S::T;
  const PhysGeom& G = p.g;
  const int lane = threadIdx.x & 31;
  const int xa = x0 + 4 * lane;
  const bool valid = xa < G.nx;
  const int xc = valid ? xa : G.nx - 4;
  const bool edge = (lane == 31) || (xa + 4 >= G.nx);  // its node D touches x+4 itself
  const uint32_t N = (uint32_t)G.n;
  const uint32_t nid = (uint32_t)xc + (uint32_t)G.nx * ((uint32_t)y + (uint32_t)G.ny * (uint32_t)z);
  T* pop = reinterpret_cast<T*>(pop_v);
  const size_t SS = G.slot_stride;
  const uint32_t lnA = lin32(G, xc, y, z);
  const uint32_t lnD = lnA + 3;
  const Wrap w = wrap_terms(G, xc, y, z);       // y/z terms; nodes A..C never at x = nx-1
  const Wrap wD = wrap_terms(G, xc + 3, y, z);  // x term of node D
  const bool xloA = !G.per[0] && xc == 0, xhiD = !G.per[0] && xc + 3 == G.nx - 1;
  const bool ylo = !G.per[1] && y == 0, yhi = !G.per[1] && y == G.ny - 1;
  const bool zlo = !G.per[2] && z == 0, zhi = !G.per[2] && z == G.nz - 1;
  const bool moving = p.any_moving_wall;

  const uint32_t fl4 = valid ? *reinterpret_cast<const uint32_t*>(flags + nid) : 0x01010101u;
  float2 gl[Q], gh[Q];  // gl: .x = A, .y = B;  gh: .x = C, .y = D
  {
    const auto r = V4::ld(pop, lnA);
    gl[0] = V4::lo(r);
    gh[0] = V4::hi(r);
  }
  static_for<0, 9>([&](auto PI) {
    constexpr int pi = decltype(PI)::value;
    constexpr int a = pair_a(pi), b = pair_b(pi);
    constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
    const T* s0 = pop + (size_t)(1 + 2 * pi) * SS;
    const T* sP = P ? s0 + SS : s0;
    const T* sQ = P ? s0 : s0 + SS;
    const bool yz_fwd = (DY > 0 && yhi) || (DY < 0 && ylo) || (DZ > 0 && zhi) || (DZ < 0 && zlo);
    const bool yz_bwd = (DY > 0 && ylo) || (DY < 0 && yhi) || (DZ > 0 && zlo) || (DZ < 0 && zhi);
    // f_a of the four nodes from X = S[1-P](x..x+3); S[P] across a wall
    const auto xv = V4::ld(yz_bwd ? sP : sQ, lnA);
    gl[a] = V4::lo(xv);
    gh[a] = V4::hi(xv);
    if (DX > 0 && xloA) gl[a].x = S::raw_ld(sP, lnA);  // node A at the -x wall
    // f_b from Y = S[P](n + d); S[1-P] across a wall
    const auto yv = V4::ld(yz_fwd ? sQ : sP, lnA + offs<0, DY, DZ>(G, w));
    const float2 ylo2 = V4::lo(yv), yhi2 = V4::hi(yv);
    if (DX == 0) {
      gl[b] = ylo2;
      gh[b] = yhi2;
    } else {
      float nxt = __shfl_down_sync(FULL, ylo2.x, 1);  // x + 4
      if (edge) nxt = S::raw_ld((yz_fwd || xhiD) ? sQ : sP, lnD + offs<1, DY, DZ>(G, wD));
      gl[b] = make_float2(ylo2.y, yhi2.x);  // x + 1, x + 2
      gh[b] = make_float2(yhi2.y, nxt);     // x + 3, x + 4
    }
  });
  if (moving && near_moving(p, xc, xc + 3, y, z)) {
    static_for<0, 9>([&](auto PI) {
      constexpr int pi = decltype(PI)::value;
      constexpr int a = pair_a(pi), b = pair_b(pi);
      constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
      const bool yz_fwd = (DY > 0 && yhi) || (DY < 0 && ylo) || (DZ > 0 && zhi) || (DZ < 0 && zlo);
      const bool yz_bwd = (DY > 0 && ylo) || (DY < 0 && yhi) || (DZ > 0 && zlo) || (DZ < 0 && zhi);
      if (yz_bwd || (DX > 0 && xloA)) gl[a].x = fmaf(S::SC, wall_term<a>(p, xc, y, z), gl[a].x);
      if (yz_bwd) {
        gl[a].y = fmaf(S::SC, wall_term<a>(p, xc + 1, y, z), gl[a].y);
        gh[a].x = fmaf(S::SC, wall_term<a>(p, xc + 2, y, z), gh[a].x);
        gh[a].y = fmaf(S::SC, wall_term<a>(p, xc + 3, y, z), gh[a].y);
      }
      if (yz_fwd) {
        gl[b].x = fmaf(S::SC, wall_term<b>(p, xc, y, z), gl[b].x);
        gl[b].y = fmaf(S::SC, wall_term<b>(p, xc + 1, y, z), gl[b].y);
        gh[b].x = fmaf(S::SC, wall_term<b>(p, xc + 2, y, z), gh[b].x);
      }
      if (yz_fwd || (DX > 0 && xhiD)) gh[b].y = fmaf(S::SC, wall_term<b>(p, xc + 3, y, z), gh[b].y);
    });
  }
  const uint8_t fl[4] = {(uint8_t)(fl4 & 0xffu), (uint8_t)((fl4 >> 8) & 0xffu), (uint8_t)((fl4 >> 16) & 0xffu),
                         (uint8_t)(fl4 >> 24)};
  bool fluid[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) fluid[k] = valid && !(fl[k] & FLAG_SKIP);
  // links into interior solids, per node (rare)
  auto solid_fix = [&](auto kk, const Wrap& wn, bool xlo, bool xhi) {
    constexpr int k = decltype(kk)::value;
    auto at = [&](int i) -> float& {
      return k == 0 ? gl[i].x : (k == 1 ? gl[i].y : (k == 2 ? gh[i].x : gh[i].y));
    };
    const uint32_t L = links[nid + k];
    const uint32_t ln = lnA + k;
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
      if (((L >> b) & 1u) && !bwd_wall) at(a) = S::raw_ld(sP, ln);
      if (((L >> a) & 1u) && !fwd_wall) at(b) = S::raw_ld(sQ, ln + offs<DX, DY, DZ>(G, wn));
    });
  };
  if (fluid[0] && (fl[0] & FLAG_SOLID_LINK)) solid_fix(IC<0>{}, w, xloA, false);
  if (fluid[1] && (fl[1] & FLAG_SOLID_LINK)) solid_fix(IC<1>{}, w, false, false);
  if (fluid[2] && (fl[2] & FLAG_SOLID_LINK)) solid_fix(IC<2>{}, w, false, false);
  if (fluid[3] && (fl[3] & FLAG_SOLID_LINK)) solid_fix(IC<3>{}, wD, false, xhiD);

  float2 rl, uxl, uyl, uzl, rh, uxh, uyh, uzh;
  collide_t<Ops2, COLL, SGS, FORCE, PREC>(p, net, gl, rl, uxl, uyl, uzl);
  collide_t<Ops2, COLL, SGS, FORCE, PREC>(p, net, gh, rh, uxh, uyh, uzh);

  if (WRITE_MOMENTS && valid) {
    auto m4 = [&](float* dst, float2 l, float2 h) {
      *reinterpret_cast<float4*>(dst) = make_float4(fluid[0] ? l.x : 0.f, fluid[1] ? l.y : 0.f,
                                                    fluid[2] ? h.x : 0.f, fluid[3] ? h.y : 0.f);
    };
    m4(rho_o + nid, rl, rh);
    m4(u_o + nid, uxl, uxh);
    m4(u_o + N + nid, uyl, uyh);
    m4(u_o + 2 * N + nid, uzl, uzh);
    auto bad = [](bool f, float r, float ux, float uy, float uz) {
      return f && (!(r > 0.f) || !isfinite(r) || !isfinite(ux) || !isfinite(uy) || !isfinite(uz));
    };
    if (bad(fluid[0], rl.x, uxl.x, uyl.x, uzl.x) || bad(fluid[1], rl.y, uxl.y, uyl.y, uzl.y) ||
        bad(fluid[2], rh.x, uxh.x, uyh.x, uzh.x) || bad(fluid[3], rh.y, uxh.y, uyh.y, uzh.y))
      atomicOr(status, 1u);
  }

  const bool all4 = fluid[0] && fluid[1] && fluid[2] && fluid[3];
  // store the four nodes' values at slot positions i .. i+3
  auto st4 = [&](T* arr, uint32_t i, float2 l, float2 h) {
    if (all4) V4::st(arr, i, l, h);
    else {
      if (fluid[0]) S::raw_st(arr, i, l.x);
      if (fluid[1]) S::raw_st(arr, i + 1, l.y);
      if (fluid[2]) S::raw_st(arr, i + 2, h.x);
      if (fluid[3]) S::raw_st(arr, i + 3, h.y);
    }
  };
  st4(pop, lnA, gl[0], gh[0]);
  const bool passD = fluid[3] && !edge;  // node D's Y value at x+4 is stored by lane+1
  static_for<0, 9>([&](auto PI) {
    constexpr int pi = decltype(PI)::value;
    constexpr int a = pair_a(pi), b = pair_b(pi);
    constexpr int DX = cx(a), DY = cy(a), DZ = cz(a);
    T* s0 = pop + (size_t)(1 + 2 * pi) * SS;
    T* sP = P ? s0 + SS : s0;
    T* sQ = P ? s0 : s0 + SS;
    st4(sQ, lnA, gl[b], gh[b]);  // f*_b -> X = S[1-P](n)
    if (DX == 0) {
      st4(sP, lnA + offs<0, DY, DZ>(G, w), gl[a], gh[a]);  // f*_a -> Y = S[P](n+d)
    } else {
      // aligned quad (x .. x+3) of row (y+dy, z+dz): x from lane-1's node D,
      // x+1 .. x+3 from nodes A, B, C
      const float from_left = __shfl_up_sync(FULL, gh[a].y, 1);
      const bool left_ok = __shfl_up_sync(FULL, passD, 1) && lane > 0;
      const uint32_t i = lnA + offs<0, DY, DZ>(G, w);
      if (left_ok && fluid[0] && fluid[1] && fluid[2]) {
        V4::st(sP, i, make_float2(from_left, gl[a].x), make_float2(gl[a].y, gh[a].x));
      } else {
        if (left_ok) S::raw_st(sP, i, from_left);
        if (fluid[0]) S::raw_st(sP, i + 1, gl[a].x);
        if (fluid[1]) S::raw_st(sP, i + 2, gl[a].y);
        if (fluid[2]) S::raw_st(sP, i + 3, gh[a].x);
      }
      if (fluid[3] && edge) S::raw_st(sP, lnD + offs<1, DY, DZ>(G, wD), gh[a].y);
    }
  });
}

}  // namespace
}  // namespace lbm
