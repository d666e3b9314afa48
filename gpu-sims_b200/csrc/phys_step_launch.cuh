// Launchers of the physics-mode step kernels, instantiated once per storage
// precision by phys_step_{f32,f16,bf16}.cu and, for the learned closure, by
// phys_step_clo_{f32,f16,bf16}.cu (split so the six compile in parallel).  The kernels wrap step_row / step_row2 (phys_step.cuh).
#pragma once
#include "phys_step.cuh"

namespace lbm {
namespace {

// Residency of the pair kernel, x STEP_BY one-warp blocks per SM.  fp32
// without Smagorinsky: 24 blocks (80 registers, up to ~100 bytes spilled in
// the forced / moment-writing forms) against 20 (94 registers, no spills),
// measured on B200: channel 512x128x128 39.3 vs 38.4 GLUPS, periodic TRT
// 256^3 40.4 vs 37.7, lid cavity 192^3 38.8 vs 36.7; 28 blocks (72 registers,
// 12-168 bytes spilled) fall back: 37.5 / 40.6 / 37.8 against 39.4 / 42.1 /
// 38.1 on one box.  With Smagorinsky the
// same bound spills 280-340 bytes and loses (128^3: 28.3 vs 32.8), so the
// Smagorinsky forms have their own bound: fp32 20 blocks (128^3 / 256^3 BGK /
// 256^3 TRT: 32.7 / 34.7 / 32.6 GLUPS against 30.2 / 31.7 / 31.0 at 16); fp16
// storage 20 blocks (128^3 BGK / 256^3 TRT: 45.2 / 41.5 against 43.0 / 38.9
// at 24 and 47.1 / 35.0 at 16).
#ifndef LBM_STEP2_MINB
#define LBM_STEP2_MINB 6
#endif
#ifndef LBM_STEP2_MINB_SMAG
#define LBM_STEP2_MINB_SMAG 5
#endif
// the 2-byte formats are issue-bound rather than memory-bound: their
// residency bounds are tuned separately
#ifndef LBM_STEP2_MINB16
#define LBM_STEP2_MINB16 6
#endif
#ifndef LBM_STEP2_MINB16_SMAG
#define LBM_STEP2_MINB16_SMAG 5
#endif
// Residency bounds of the learned-closure kernels (the MLP's hidden layer
// stays in registers: two nodes' worth in the pair kernel).
#ifndef LBM_CLO_MINB
#define LBM_CLO_MINB 3
#endif
// The pair kernel with the CUDA-core MLP, 128^3: fp32 storage at three
// blocks per SM (168 registers, 32-124 bytes spilled) 11.3 GLUPS against 10.5
// at two (208-220 registers, no spills); the 2-byte formats 11.7 against 11.9,
// so they keep two.
#ifndef LBM_CLO2_MINB
#define LBM_CLO2_MINB 2
#endif
#ifndef LBM_CLO2_MINB32
#define LBM_CLO2_MINB32 3
#endif

// Rows per block of the pair kernel.  One-warp blocks whose row is
// blockIdx.y: y is then warp-uniform to the compiler, which moves the row's
// wall predicates, wrap terms and slot selection to the uniform datapath
// (measured on B200, channel 512x128x128: fp32 36.55 GLUPS against 35.74 with
// four-row blocks; fp16 52.0 against 51.1, and 53.7 with the vote-based store
// phase of step_row2, which alone on four-row blocks ran 50.2).  The 2-byte
// kernel fits its 102-register bound (20 one-warp blocks per SM) without
// spills; an earlier form of it spilled there.
#ifndef LBM_STEP2_ROWS16
#define LBM_STEP2_ROWS16 1
#endif
template <int PREC, int SGS>
constexpr int step2_rows() {
  return SGS == 2 ? STEP_BY : (PREC == LBM_PREC_F32 ? 1 : LBM_STEP2_ROWS16);
}

// Two nodes per thread (step_pairs(nx)): a warp covers 64 consecutive x.
// SGS: 0 none, 1 Smagorinsky, 2 learned closure (net = the network).
template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P>
__global__ void __launch_bounds__(32 * step2_rows<PREC, SGS>(),
                                  SGS == 2 ? (PREC == LBM_PREC_F32 ? LBM_CLO2_MINB32 : LBM_CLO2_MINB)
                                  : PREC == LBM_PREC_F32
                                      ? (SGS == 1 ? LBM_STEP2_MINB_SMAG : LBM_STEP2_MINB) * STEP_BY
                                      : (SGS == 1 ? LBM_STEP2_MINB16_SMAG : LBM_STEP2_MINB16) * STEP_BY /
                                            LBM_STEP2_ROWS16)
    k_phys_step2(PhysParams p, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                 const uint32_t* __restrict__ links, float* __restrict__ rho_o,
                 float* __restrict__ u_o, unsigned* __restrict__ status,
                 const __grid_constant__ CloNet<SGS> net) {
  constexpr int R = step2_rows<PREC, SGS>();
  const int y = R == 1 ? (int)blockIdx.y : (int)(blockIdx.y * R + threadIdx.y);
  if (y >= p.g.ny) return;  // uniform over the warp
  step_row2<PREC, COLL, SGS, FORCE, WRITE_MOMENTS, P>(p, net, pop_v, flags, links, rho_o, u_o,
                                                      status, blockIdx.x * 64, y, blockIdx.z);
}

// Rows per block of the one-node kernel (1: one-warp blocks, row = blockIdx.y).
#ifndef LBM_STEP1_ROWS
#define LBM_STEP1_ROWS STEP_BY
#endif
template <int SGS>
constexpr int step1_rows() {
  return SGS == 2 ? STEP_BY : LBM_STEP1_ROWS;
}

template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P>
__global__ void __launch_bounds__(32 * step1_rows<SGS>(),
                                  SGS == 2 ? LBM_CLO_MINB : LBM_STEP_MINB * STEP_BY / step1_rows<SGS>())
    k_phys_step(PhysParams p, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                const uint32_t* __restrict__ links, float* __restrict__ rho_o,
                float* __restrict__ u_o, unsigned* __restrict__ status,
                const __grid_constant__ CloNet<SGS> net) {
  constexpr int R = step1_rows<SGS>();
  const int y = R == 1 ? (int)blockIdx.y : (int)(blockIdx.y * R + threadIdx.y);
  if (y >= p.g.ny) return;  // uniform over the warp
  step_row<PREC, COLL, SGS, FORCE, WRITE_MOMENTS, P>(p, net, pop_v, flags, links, rho_o, u_o,
                                                     status, blockIdx.x * 32, y, blockIdx.z);
}

// Open x faces: one thread per face node, lanes over (y, z), blockIdx.y
// the side (0: x = 0, 1: x = nx-1).  Runs after the row kernel of the same
// step, which leaves these nodes alone (FLAG_OPEN).
template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P>
__global__ void __launch_bounds__(128)
    k_phys_face(PhysParams p, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                const uint32_t* __restrict__ links, float* __restrict__ rho_o,
                float* __restrict__ u_o, unsigned* __restrict__ status,
                const __grid_constant__ CloNet<SGS> net) {
  const int side = blockIdx.y;
  if (p.open[side] == LBM_OPEN_NONE) return;  // uniform over the block
  const int nyz = p.g.ny * p.g.nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int tc = t < nyz ? t : nyz - 1;  // idle lanes take part in the shuffles
  step_row<PREC, COLL, SGS, FORCE, WRITE_MOMENTS, P, true>(p, net, pop_v, flags, links, rho_o, u_o,
                                                          status, side ? p.g.nx - 1 : 0, tc % p.g.ny,
                                                          tc / p.g.ny, t < nyz);
}

#ifndef LBM_STEP4_MINB
#define LBM_STEP4_MINB 4  // x STEP_BY / LBM_STEP4_ROWS blocks per SM
#endif
// fp32 storage (16-byte slot quads), channel 512x128x128 with a body force,
// against 38.4 GLUPS for the two-node kernel: 16 blocks per SM 37.9 GLUPS
// (128 registers, 124 bytes spilled in the forced kernel), 12 blocks 36.6 (168,
// no spills), 8 blocks 27.8.  The automatic choice stays at two nodes.
#ifndef LBM_STEP4_MINB32
#define LBM_STEP4_MINB32 4
#endif

// Four nodes per thread (nx % 4 == 0): a warp covers 128 x, in one-warp
// blocks (row = blockIdx.y, warp-uniform).  2-byte storage: 16 per SM (127
// registers, no spills).  Measured on B200, channel 512x128x128 fp16: 53.8
// GLUPS against 47.6 with four-row blocks and 49.9 with 12 one-warp blocks per
// SM (which spilled 36 bytes); the two-node kernel runs 54.1.
#ifndef LBM_STEP4_ROWS
#define LBM_STEP4_ROWS 1
#endif
template <int PREC>
constexpr int step4_minb() {
  return (PREC == LBM_PREC_F32 ? LBM_STEP4_MINB32 : LBM_STEP4_MINB) * STEP_BY / LBM_STEP4_ROWS;
}
template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P>
__global__ void __launch_bounds__(32 * LBM_STEP4_ROWS, step4_minb<PREC>())
    k_phys_step4(PhysParams p, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                 const uint32_t* __restrict__ links, float* __restrict__ rho_o,
                 float* __restrict__ u_o, unsigned* __restrict__ status,
                 const __grid_constant__ CloNet<SGS> net) {
  constexpr int R = LBM_STEP4_ROWS;
  const int y = R == 1 ? (int)blockIdx.y : (int)(blockIdx.y * R + threadIdx.y);
  if (y >= p.g.ny) return;  // uniform over the warp
  step_row4<PREC, COLL, SGS, FORCE, WRITE_MOMENTS, P>(p, net, pop_v, flags, links, rho_o, u_o,
                                                      status, blockIdx.x * 128, y, blockIdx.z);
}

// Learned closure with the hidden layer on the tensor cores (CloNet<3>): one
// node per thread, a CTA of 128 threads is one M = 128 MMA per z-plane, and
// walks LBM_TC_ZPB planes so that its set-up (the 32-column TMEM allocation,
// the bf16 W2 tile, the mbarrier) is paid once per several MMAs.  Rows
// beyond ny run on the last row without storing, so every thread reaches the
// CTA-wide barriers.  At four CTAs per SM, 128^3: 16 planes 14.5 / 15.8
// GLUPS (fp32 / fp16 storage), 8 planes 14.3 / 15.6, 4 planes 13.6 / 14.8.
#ifndef LBM_TC_ZPB
#define LBM_TC_ZPB 16
#endif
// Four CTAs per SM (124 registers, no spills): 14.3 / 15.5 GLUPS (fp32 /
// fp16 storage, 128^3) against 12.5 / 14.1 with the three CTAs that 149
// registers allow.  The kernel is bound by dependent-instruction latency
// (MMA waits, barriers, the feature chain) at a few warps per scheduler, so
// residency pays more than instruction count.  (Before the first layer moved
// to the tensor cores the kernel needed 168 registers and spilled at three.)
#ifndef LBM_TC_MINB
#define LBM_TC_MINB 4
#endif
template <int PREC, int COLL, bool WRITE_MOMENTS, int P>
__global__ void __launch_bounds__(STEP_THREADS, LBM_TC_MINB)
    k_phys_step_tc(PhysParams p, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                   const uint32_t* __restrict__ links, float* __restrict__ rho_o,
                   float* __restrict__ u_o, unsigned* __restrict__ status,
                   const __grid_constant__ CloNet<2> net, uint32_t wait_polls) {
  static_assert(STEP_THREADS == 128, "one MMA row per thread");
  __shared__ __align__(1024) uint8_t sA[2 * CLO_TILE_A_BYTES];
  __shared__ __align__(1024) uint8_t sB[CLO_HID * 64];
  __shared__ __align__(1024) uint8_t sB1[CLO_HID * 64];  // W1 as a 32 x 32 tile, k >= 9 zero
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ uint32_t gave_up[STEP_THREADS / 32];
  __shared__ uint32_t last_phase;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  if (tid < STEP_THREADS / 32) gave_up[tid] = 0u;
  if (tid == 0) last_phase = 0u;
  for (int e = tid; e < CLO_HID * CLO_HID; e += STEP_THREADS) {
    const int n = e / CLO_HID, k = e % CLO_HID;
    *reinterpret_cast<__nv_bfloat16*>(sB + clo_tile_off(n, k)) = __float2bfloat16_rn(net.v[CLO_W2 + e]);
    *reinterpret_cast<__nv_bfloat16*>(sB1 + clo_tile_off(n, k)) =
        __float2bfloat16_rn(k < CLO_IN ? net.v[CLO_W1 + n * CLO_IN + k] : 0.0f);
  }
  const uint32_t mbar_addr = (uint32_t)__cvta_generic_to_shared(&mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(mbar_addr), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.y == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"((uint32_t)__cvta_generic_to_shared(&tslot)), "r"(32) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int y = blockIdx.y * STEP_BY + threadIdx.y;
  CloNet<3> c;
  c.net = &net;
  c.sA = sA;
  c.sA_addr = (uint32_t)__cvta_generic_to_shared(sA);
  c.sB_addr = (uint32_t)__cvta_generic_to_shared(sB);
  c.sB1_addr = (uint32_t)__cvta_generic_to_shared(sB1);
  c.mbar_addr = mbar_addr;
  c.tmem = tslot;
  c.status = status;
  c.gave_up = gave_up;
  c.last_phase = &last_phase;
  c.wait_limit = wait_polls;
  c.row_ok = y < p.g.ny;
  const int z0 = blockIdx.z * LBM_TC_ZPB;
  const int z1 = min(p.g.nz, z0 + LBM_TC_ZPB);  // uniform over the CTA
  const int yr = c.row_ok ? y : p.g.ny - 1;
  const int x0 = blockIdx.x * 32;
  // Software pipeline over the planes: the loads of plane z+1 are issued
  // before plane z's collision, whose MMA wait and arithmetic then hide their
  // latency (each slot belongs to one node, so the two planes never touch
  // the same slot).
  RowNode<PREC> cur, nxt;
  row_load<PREC, P, false>(p, c.row_ok, pop_v, flags, x0, yr, z0, true, cur);
  for (int z = z0; z < z1; ++z) {
    c.phase = (uint32_t)((z - z0) & 1);
    float g[Q];
    row_convert(cur, g);  // waits for plane z's loads
    if (z + 1 < z1) row_load<PREC, P, false>(p, c.row_ok, pop_v, flags, x0, yr, z + 1, true, nxt);
    row_finish<PREC, COLL, 3, false, WRITE_MOMENTS, P, false>(p, c, pop_v, links, rho_o, u_o, status, yr, z,
                                                              cur, g);
    cur = nxt;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  const bool aborted = __syncthreads_or(gave_up[threadIdx.y] != 0);
  if (threadIdx.y == 0) {
    if (aborted) {
      // the last MMA whose wait ran out may still run: wait for its commit
      // (bounded, always by the default limit, whatever the per-plane
      // bound) before its tensor memory is freed
      uint32_t done = 0;
      for (int it = 0; it < LBM_CLO_WAIT_LIMIT && !done; ++it)
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done) : "r"(mbar_addr), "r"(last_phase) : "memory");
      __syncwarp();
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(c.tmem), "r"(32) : "memory");
  }
}

template <int SGS> CloNet<SGS> net_of(const Ctx&) { return CloNet<SGS>{}; }
template <> CloNet<2> net_of<2>(const Ctx& c) {
  CloNet<2> n;
  for (int k = 0; k < CLO_FLOATS; ++k) n.v[k] = c.clo[k];
  return n;
}

// Nodes per thread: the context's choice (lbm_set_step_variant) or, by
// default, four when step_quads(nx) (a build option), two when
// step_pairs(nx), else one.
inline bool use_quads(const Ctx& c) {
  const int nx = c.pp.g.nx;
  if (c.closure || c.pp.any_open || nx % 4) return false;
  return c.step_variant == 4 || (c.step_variant == 0 && step_quads(nx));
}
inline bool use_pairs(const Ctx& c) {
  const int nx = c.pp.g.nx;
  if (nx % 2 || c.step_variant == 1 || c.step_variant == 8) return false;
  return c.step_variant == 2 || c.step_variant == 4 || step_pairs(nx);
}

template <int PREC, int COLL, int SGS, bool FORCE>
cudaError_t launch_rows(const Ctx& c, int P, bool wm, cudaStream_t s) {
  const PhysGeom& G = c.pp.g;
  const CloNet<SGS> net = net_of<SGS>(c);
  const dim3 blk(32, STEP_BY, 1);
  if constexpr (SGS != 2) {
    if (use_quads(c)) {
      constexpr int R4 = LBM_STEP4_ROWS;
      const dim3 grd((G.nx + 127) / 128, (G.ny + R4 - 1) / R4, G.nz), blk4(32, R4, 1);
#define LBM_STEP_LAUNCH(WM, PAR)                                          \
  k_phys_step4<PREC, COLL, SGS, FORCE, WM, PAR><<<grd, blk4, 0, s>>>(     \
      c.pp, c.pop, c.flags, c.links, c.rho, c.u, c.status, net)
      if (wm) {
        if (P) LBM_STEP_LAUNCH(true, 1); else LBM_STEP_LAUNCH(true, 0);
      } else {
        if (P) LBM_STEP_LAUNCH(false, 1); else LBM_STEP_LAUNCH(false, 0);
      }
#undef LBM_STEP_LAUNCH
      return cudaGetLastError();
    }
  }
  if (use_pairs(c)) {
    constexpr int R = step2_rows<PREC, SGS>();
    const dim3 grd((G.nx + 63) / 64, (G.ny + R - 1) / R, G.nz), blk2(32, R, 1);
#define LBM_STEP_LAUNCH(WM, PAR)                                          \
  k_phys_step2<PREC, COLL, SGS, FORCE, WM, PAR><<<grd, blk2, 0, s>>>(     \
      c.pp, c.pop, c.flags, c.links, c.rho, c.u, c.status, net)
    if (wm) {
      if (P) LBM_STEP_LAUNCH(true, 1); else LBM_STEP_LAUNCH(true, 0);
    } else {
      if (P) LBM_STEP_LAUNCH(false, 1); else LBM_STEP_LAUNCH(false, 0);
    }
#undef LBM_STEP_LAUNCH
    return cudaGetLastError();
  }
  constexpr int R1 = step1_rows<SGS>();
  const dim3 grd((G.nx + 31) / 32, (G.ny + R1 - 1) / R1, G.nz), blk1(32, R1, 1);
#define LBM_STEP_LAUNCH(WM, PAR)                                          \
  k_phys_step<PREC, COLL, SGS, FORCE, WM, PAR><<<grd, blk1, 0, s>>>(      \
      c.pp, c.pop, c.flags, c.links, c.rho, c.u, c.status, net)
  if (wm) {
    if (P) LBM_STEP_LAUNCH(true, 1); else LBM_STEP_LAUNCH(true, 0);
  } else {
    if (P) LBM_STEP_LAUNCH(false, 1); else LBM_STEP_LAUNCH(false, 0);
  }
#undef LBM_STEP_LAUNCH
  return cudaGetLastError();
}

// One step: the row kernel, then (open x faces only) the face kernel.
template <int PREC, int COLL, int SGS, bool FORCE>
cudaError_t launch_step(const Ctx& c, int P, bool wm, cudaStream_t s) {
  const cudaError_t e = launch_rows<PREC, COLL, SGS, FORCE>(c, P, wm, s);
  if (e != cudaSuccess || !c.pp.any_open) return e;
  const CloNet<SGS> net = net_of<SGS>(c);
  const dim3 grd((c.pp.g.ny * c.pp.g.nz + 127) / 128, 2, 1);
#define LBM_FACE_LAUNCH(WM, PAR)                                          \
  k_phys_face<PREC, COLL, SGS, FORCE, WM, PAR><<<grd, 128, 0, s>>>(       \
      c.pp, c.pop, c.flags, c.links, c.rho, c.u, c.status, net)
  if (wm) {
    if (P) LBM_FACE_LAUNCH(true, 1); else LBM_FACE_LAUNCH(true, 0);
  } else {
    if (P) LBM_FACE_LAUNCH(false, 1); else LBM_FACE_LAUNCH(false, 0);
  }
#undef LBM_FACE_LAUNCH
  return cudaGetLastError();
}

template <int PREC, int COLL, int SGS>
cudaError_t dispatch_force(const Ctx& c, int P, bool wm, cudaStream_t s) {
  const bool force = c.pp.accel[0] != 0.f || c.pp.accel[1] != 0.f || c.pp.accel[2] != 0.f;
  return force ? launch_step<PREC, COLL, SGS, true>(c, P, wm, s)
               : launch_step<PREC, COLL, SGS, false>(c, P, wm, s);
}

template <int PREC, int COLL>
cudaError_t launch_step_tc(const Ctx& c, int P, bool wm, cudaStream_t s) {
  const PhysGeom& G = c.pp.g;
  const CloNet<2> net = net_of<2>(c);
  const dim3 blk(32, STEP_BY, 1);
  const dim3 grd((G.nx + 31) / 32, (G.ny + STEP_BY - 1) / STEP_BY, (G.nz + LBM_TC_ZPB - 1) / LBM_TC_ZPB);
#define LBM_STEP_LAUNCH(WM, PAR)                                          \
  k_phys_step_tc<PREC, COLL, WM, PAR><<<grd, blk, 0, s>>>(                \
      c.pp, c.pop, c.flags, c.links, c.rho, c.u, c.status, net, polls)
  const uint32_t polls = c.clo_wait_polls;
  if (wm) {
    if (P) LBM_STEP_LAUNCH(true, 1); else LBM_STEP_LAUNCH(true, 0);
  } else {
    if (P) LBM_STEP_LAUNCH(false, 1); else LBM_STEP_LAUNCH(false, 0);
  }
#undef LBM_STEP_LAUNCH
  return cudaGetLastError();
}

// CLOSURE: the learned-closure kernels (compiled in their own files; no body
// force, which lbm_set_closure enforces): the CUDA-core MLP (one or two
// nodes per thread, fp32 activations) by default, the tensor-core MLP (bf16
// hidden activations) for variant 8.  Measured on B200 at 128^3: CUDA-core
// pair kernel 11.3 / 11.9 GLUPS (fp32 / fp16 storage), tensor-core kernel
// 14.5 / 15.8.
template <int PREC, int COLL, bool CLOSURE>
cudaError_t dispatch_smag(const Ctx& c, int P, bool wm, cudaStream_t s) {
  if constexpr (CLOSURE) {
    if (c.step_variant == 8) return launch_step_tc<PREC, COLL>(c, P, wm, s);
    return launch_step<PREC, COLL, 2, false>(c, P, wm, s);
  } else {
    return c.pp.smag_cs > 0.f ? dispatch_force<PREC, COLL, 1>(c, P, wm, s)
                              : dispatch_force<PREC, COLL, 0>(c, P, wm, s);
  }
}

template <int PREC, bool CLOSURE>
cudaError_t dispatch_coll(const Ctx& c, int P, bool wm, cudaStream_t s) {
  return c.d.collision == LBM_COLL_TRT ? dispatch_smag<PREC, LBM_COLL_TRT, CLOSURE>(c, P, wm, s)
                                       : dispatch_smag<PREC, LBM_COLL_BGK, CLOSURE>(c, P, wm, s);
}

}  // namespace
}  // namespace lbm

#define LBM_DEFINE_PHYS_STEP(NAME, PREC, CLOSURE)                                  \
  namespace lbm {                                                                  \
  cudaError_t NAME(const Ctx& c, int parity, bool write_moments, cudaStream_t s) { \
    return dispatch_coll<PREC, CLOSURE>(c, parity, write_moments, s);              \
  }                                                                                \
  }
