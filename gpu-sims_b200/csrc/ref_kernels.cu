// Reference-mode kernels: the reference's four-pass step fused into one
// two-buffer pull kernel per step.
//
// One launch computes, for every node, the tail of step t and the head of
// step t+1:
//   stream_t (shaders/stream.comp.glsl:29-47)          pull with clamp-to-edge
//   apply_boundaries_t (shaders/apply_boundaries.comp.glsl:57-169)
//   compute_moments_t (shaders/compute_moments.comp.glsl:29-50)
//   collide_{t+1} (shaders/collide.comp.glsl:39-61)      with rho and half(u)
// so the stored state between launches is the post-collision population of
// the next step, and the moments of step t are available in registers to the
// collide that needs them (the reference keeps them in the rho/velocity
// images between dispatches, src/main.cpp:1554-1591).
//
// Two buffers, not an in-place scheme: clamp-to-edge streaming reads the
// same direction at a clamped neighbour, and the outlet reads all 19
// post-stream populations of x = Nx-2; both gather from locations that other
// threads overwrite in an in-place layout.
#include <cuda_fp16.h>

#include "d3q19.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace {

__device__ __forceinline__ float round_u(float v, int mode) {
  if (mode == LBM_UROUND_RTE) return __half2float(__float2half_rn(v));
  if (mode == LBM_UROUND_RTZ) return __half2float(__float2half_rz(v));
  return v;
}

__device__ __forceinline__ int clamp_edge(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

// Post-stream value of direction I at (x,y,z): f_in[clamp(x - c_I)][I]
// (shaders/stream.comp.glsl:43-46; the sampler clamps to edge).
template <int I>
__device__ __forceinline__ float pull(const RefParams& p, const float* __restrict__ fin, int x, int y,
                                      int z) {
  int xs = x - cx(I), ys = y - cy(I), zs = z - cz(I);
  if (cx(I) != 0) xs = clamp_edge(xs, p.nx - 1);
  if (cy(I) != 0) ys = clamp_edge(ys, p.ny - 1);
  if (cz(I) != 0) zs = clamp_edge(zs, p.nz - 1);
  const size_t src = (size_t)xs + (size_t)p.nx * ((size_t)ys + (size_t)p.ny * (size_t)zs);
  return __ldg(fin + (size_t)I * p.n + src);
}

// The 19 pulls of a node.  Away from the y and z faces every source lies in
// a row at a constant offset from the node's row, so only x is clamped (the
// x faces fall inside ordinary warps, which then do not diverge); nodes on a
// y or z face take the fully clamped path.
__device__ __forceinline__ void pull_all(const RefParams& p, const float* __restrict__ fin, int x, int y,
                                         int z, size_t nid, float (&g)[Q]) {
  if (y > 0 && y < p.ny - 1 && z > 0 && z < p.nz - 1) {
    const ptrdiff_t sy = p.nx, sz = (ptrdiff_t)p.nx * p.ny;
    const float* row = fin + (nid - (size_t)x);  // (0, y, z)
    static_for<0, Q>([&](auto I) {
      constexpr int i = decltype(I)::value;
      const int xs = cx(i) == 0 ? x : clamp_edge(x - cx(i), p.nx - 1);
      g[i] = __ldg(row + (size_t)i * p.n + (-(cy(i) * sy + cz(i) * sz) + xs));
    });
  } else {
    static_for<0, Q>([&](auto I) { g[I.value] = pull<decltype(I)::value>(p, fin, x, y, z); });
  }
}

// compute_moments (shaders/compute_moments.comp.glsl:37-47): rho summed in
// direction order, rho*u as signed sums, u = rho*u / rho guarded by 1e-12.
// Also the outlet's upstream velocity (apply_boundaries.comp.glsl:112-119),
// which differs only in the fallback value.
__device__ __forceinline__ void moments(const float (&g)[Q], float& rho, float& jx, float& jy,
                                        float& jz) {
  rho = g[0];
  static_for<1, Q>([&](auto I) { rho = rl_add(rho, g[I.value]); });
  jx = 0.0f;
  jy = 0.0f;
  jz = 0.0f;
  static_for<1, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    if (cx(i) > 0) jx = rl_add(jx, g[i]);
    if (cx(i) < 0) jx = rl_sub(jx, g[i]);
    if (cy(i) > 0) jy = rl_add(jy, g[i]);
    if (cy(i) < 0) jy = rl_sub(jy, g[i]);
    if (cz(i) > 0) jz = rl_add(jz, g[i]);
    if (cz(i) < 0) jz = rl_sub(jz, g[i]);
  });
}

__device__ __forceinline__ void set_equilibrium(float (&g)[Q], float rho, float ux, float uy,
                                                float uz) {
  const float uu = rl_udotu(ux, uy, uz);
  static_for<0, Q>([&](auto I) { g[I.value] = rl_feq<decltype(I)::value>(rho, ux, uy, uz, uu); });
}

// LBM_REF_WARPS warps per block side by side along x, the row (y, z) from
// blockIdx: the row terms of the pulls are warp-uniform to the compiler
// (uniform datapath).
#ifndef LBM_REF_WARPS
#define LBM_REF_WARPS 1
#endif
#ifndef LBM_REF_MINB
#define LBM_REF_MINB (32 / LBM_REF_WARPS)
#endif
template <bool WRITE_MOMENTS>
__global__ void __launch_bounds__(32 * LBM_REF_WARPS, LBM_REF_MINB)
    k_ref_step(RefParams p, const float* __restrict__ fin, float* __restrict__ fout,
               const uint8_t* __restrict__ flags, const uint32_t* __restrict__ links,
               float* __restrict__ rho_o, float* __restrict__ u_o, unsigned* __restrict__ status) {
  const int x = (blockIdx.x * LBM_REF_WARPS + threadIdx.y) * 32 + threadIdx.x;
  const int y = blockIdx.y;
  const int z = blockIdx.z;
  if (x >= p.nx || y >= p.ny || z >= p.nz) return;
  const size_t N = p.n;
  const size_t nid = (size_t)x + (size_t)p.nx * ((size_t)y + (size_t)p.ny * (size_t)z);
  const uint8_t fl = flags[nid];
  // the pulls are issued before the flag is known (every source is in the
  // grid), so a node costs one memory round trip, not two
  float g[Q];
  pull_all(p, fin, x, y, z, nid, g);

  if (fl & FLAG_SOLID) {
    // (1) solid: populations zeroed (apply_boundaries.comp.glsl:62-66); the
    // moments pass reads rho = 0 -> u = 0; collide of a zero state is zero.
    static_for<0, Q>([&](auto I) { fout[(size_t)I.value * N + nid] = 0.0f; });
    if (WRITE_MOMENTS) {
      rho_o[nid] = 0.0f;
      u_o[nid] = 0.0f;
      u_o[N + nid] = 0.0f;
      u_o[2 * N + nid] = 0.0f;
    }
    return;
  }

  // (2) post-stream bounce-back, sequential in i (apply_boundaries.comp.glsl:76-82):
  // if mask(x + c_i) (out of bounds = solid): f[opp i] := f[i].
  if (fl & FLAG_BOUNDARY) {
    const uint32_t L = links[nid];
    static_for<1, Q>([&](auto I) {
      constexpr int i = decltype(I)::value;
      if (L & (1u << i)) g[opp(i)] = g[i];
    });
  }

  if (p.inlet_outlet) {
    // (3a) x = 0 equilibrium inlet (apply_boundaries.comp.glsl:91-97).
    if (x == 0) set_equilibrium(g, p.rho0, p.u_inf[0], p.u_inf[1], p.u_inf[2]);
    // (3b) x = Nx-1 equilibrium outlet with the upstream node's velocity
    // (apply_boundaries.comp.glsl:103-125).  The reference reads x = Nx-2
    // from the buffer its neighbour threads are rewriting in the same
    // dispatch; here it is read from the post-stream state before any
    // boundary write, which is deterministic.
    if (x == p.nx - 1) {
      float vx = p.u_inf[0], vy = p.u_inf[1], vz = p.u_inf[2];
      const bool up_solid = (x < 1) || (flags[nid - 1] & FLAG_SOLID);
      if (!up_solid) {
        float h[Q];
        static_for<0, Q>([&](auto I) { h[I.value] = pull<decltype(I)::value>(p, fin, x - 1, y, z); });
        float rl, jx, jy, jz;
        moments(h, rl, jx, jy, jz);
        if (rl > 1e-12f) {
          vx = __fdiv_rn(jx, rl);
          vy = __fdiv_rn(jy, rl);
          vz = __fdiv_rn(jz, rl);
        }
      }
      set_equilibrium(g, p.rho0, vx, vy, vz);
    }
  }

  if (p.free_slip) {
    // (4) free-slip swaps, in source order (apply_boundaries.comp.glsl:136-169).
    if (y == 0) { g[4] = g[3]; g[8] = g[7]; g[10] = g[9]; g[17] = g[15]; g[18] = g[16]; }
    if (y == p.ny - 1) { g[3] = g[4]; g[7] = g[8]; g[9] = g[10]; g[15] = g[17]; g[16] = g[18]; }
    if (z == 0) { g[6] = g[5]; g[12] = g[11]; g[14] = g[13]; g[16] = g[15]; g[18] = g[17]; }
    if (z == p.nz - 1) { g[5] = g[6]; g[11] = g[12]; g[13] = g[14]; g[15] = g[16]; g[17] = g[18]; }
  }

  float rho, jx, jy, jz;
  moments(g, rho, jx, jy, jz);
  float ux = 0.0f, uy = 0.0f, uz = 0.0f;
  if (rho > 1e-12f) {
    ux = __fdiv_rn(jx, rho);
    uy = __fdiv_rn(jy, rho);
    uz = __fdiv_rn(jz, rho);
  }
  if (WRITE_MOMENTS) {
    rho_o[nid] = rho;
    u_o[nid] = ux;
    u_o[N + nid] = uy;
    u_o[2 * N + nid] = uz;
    if (!(rho > 0.0f) || !isfinite(rho) || !isfinite(ux) || !isfinite(uy) || !isfinite(uz))
      atomicOr(status, 1u);
  }

  // collide of the next step: rho from the r32f image, u through the rgba16f
  // image (collide.comp.glsl:44-45; src/main.cpp:843).
  const float qx = round_u(ux, p.u_round), qy = round_u(uy, p.u_round), qz = round_u(uz, p.u_round);
  const float uu = rl_udotu(qx, qy, qz);
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    const float feq = rl_feq<i>(rho, qx, qy, qz, uu);
    fout[(size_t)i * N + nid] = rl_add(rl_mul(p.omtau_inv, g[i]), rl_mul(p.tau_inv, feq));
  });
}

// init_equilibrium (shaders/init_equilibrium.comp.glsl:35-47) followed by the
// first collide, which reads rho = 1 and the fp16-stored u_inf.  With host
// moment fields the same is done per node from (rho(x), u(x)).
__global__ void __launch_bounds__(256)
    k_ref_init(RefParams p, const float* __restrict__ rho_in, const float* __restrict__ u_in,
               float rho0, float u0x, float u0y, float u0z, float* __restrict__ fout,
               float* rho_o, float* u_o) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= p.nx || y >= p.ny || z >= p.nz) return;
  const size_t N = p.n;
  const size_t nid = (size_t)x + (size_t)p.nx * ((size_t)y + (size_t)p.ny * (size_t)z);
  float r = rho0, vx = u0x, vy = u0y, vz = u0z;
  if (rho_in) r = rho_in[nid];
  if (u_in) {
    vx = u_in[nid];
    vy = u_in[N + nid];
    vz = u_in[2 * N + nid];
  }
  const float uu = rl_udotu(vx, vy, vz);
  const float qx = round_u(vx, p.u_round), qy = round_u(vy, p.u_round), qz = round_u(vz, p.u_round);
  const float qq = rl_udotu(qx, qy, qz);
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    const float f = rl_feq<i>(r, vx, vy, vz, uu);
    const float feq = rl_feq<i>(r, qx, qy, qz, qq);
    fout[(size_t)i * N + nid] = rl_add(rl_mul(p.omtau_inv, f), rl_mul(p.tau_inv, feq));
  });
  if (rho_o) {
    rho_o[nid] = r;
    u_o[nid] = vx;
    u_o[N + nid] = vy;
    u_o[2 * N + nid] = vz;
  }
}

dim3 ref_block() { return dim3(32, 4, 2); }
dim3 ref_grid(const RefParams& p) {
  const dim3 b = ref_block();
  return dim3((p.nx + b.x - 1) / b.x, (p.ny + b.y - 1) / b.y, (p.nz + b.z - 1) / b.z);
}
// k_ref_step: LBM_REF_WARPS warps of 32 x per block, a block per (x tile, y, z)
dim3 row_grid(const RefParams& p) {
  return dim3((p.nx + 32 * LBM_REF_WARPS - 1) / (32 * LBM_REF_WARPS), p.ny, p.nz);
}
dim3 row_block() { return dim3(32, LBM_REF_WARPS, 1); }

}  // namespace

cudaError_t ref_init(const Ctx& c, const float* rho, const float* u3, float rho0, const float* u0,
                     cudaStream_t s, bool write_moments) {
  const float zero[3] = {0.f, 0.f, 0.f};
  if (!u0) u0 = zero;
  k_ref_init<<<ref_grid(c.rp), ref_block(), 0, s>>>(c.rp, rho, u3, rho0, u0[0], u0[1], u0[2],
                                                    c.fbuf[c.cur], write_moments ? c.rho : nullptr,
                                                    write_moments ? c.u : nullptr);
  return cudaGetLastError();
}

cudaError_t ref_step_with(const Ctx& c, const RefParams& p, const float* fin, float* fout,
                          bool write_moments, cudaStream_t s) {
  if (write_moments)
    k_ref_step<true><<<row_grid(p), row_block(), 0, s>>>(p, fin, fout, c.flags, c.links, c.rho, c.u, c.status);
  else
    k_ref_step<false><<<row_grid(p), row_block(), 0, s>>>(p, fin, fout, c.flags, c.links, c.rho, c.u, c.status);
  return cudaGetLastError();
}

cudaError_t ref_step(const Ctx& c, const float* fin, float* fout, bool write_moments,
                     cudaStream_t s) {
  return ref_step_with(c, c.rp, fin, fout, write_moments, s);
}

}  // namespace lbm
