// Learned sub-grid closure: the per-node feature map and the MLP, shared by
// the training kernels (closure.cu) and the collide of the physics step
// (phys_step.cuh), so the network sees the same inputs, evaluated by the same
// code, in both places.
//
// Inputs (9) come from the non-equilibrium momentum flux Pi = sum c c (f -
// feq) of the node (physical units) and its density: the direction Pi / |Pi|
// (6 components xx yy zz xy xz yz), log |Pi|, the invariant tr((Pi/|Pi|)^3)
// and rho - 1.  The output r >= 0 scales the Smagorinsky constant,
// Cs^2 = Cs0^2 r, which then sets the node's relaxation time by the Hou et
// al. (1996) relation.
#pragma once
#include <cstdint>

#include <cuda_bf16.h>

#include "fops.cuh"
#include "lbm_internal.h"

namespace lbm {

// Network handed to a step kernel by value: in the kernel's parameter space
// every weight is a constant-bank operand of its FMA.  Kernels without the
// closure take the one-float placeholder.
template <int SGS> struct CloNet {
  float v[1];
  __device__ __forceinline__ float operator[](int) const { return 0.0f; }
};
template <> struct CloNet<2> {
  float v[CLO_FLOATS];
  __device__ __forceinline__ float operator[](int k) const { return v[k]; }
};

// SGS 3: the same network with its hidden layer on the tensor cores.  One
// CTA of 128 threads, one node per thread, evaluates its 128 nodes' 32 x 32
// hidden layer as one tcgen05 MMA (M = 128, N = 32, K = 32 in two K = 16
// steps; bf16 operands in shared memory, fp32 accumulator in tensor memory):
// each thread writes its node's first-layer activations (bf16) as row r of
// A, thread 0 issues the MMAs, every thread reads its row of D back from
// tensor memory (warp w owns TMEM lanes 32w .. 32w+31) and finishes the
// output layer on CUDA cores.  The first layer (9 -> 32) stays on CUDA
// cores.  Built by k_phys_step_tc (phys_step_launch.cuh), which owns the
// shared tiles, the mbarrier and the TMEM columns.
//
// A wait for an MMA that runs out (wait_limit polls) must not leave
// the tensor core reading a tile that the CTA goes on to rewrite.  So the A
// tile is double-buffered by phase, a warp that gives up marks its entry of
// `gave_up` (shared, sticky), and every later evaluation starts with a
// __syncthreads_or over those marks: from then on the whole CTA issues no
// MMA and falls back to r = 1, and the kernel drains the last commit (again
// bounded) before it frees its tensor memory.
template <> struct CloNet<3> {
  const CloNet<2>* net;     // parameters (kernel parameter space)
  uint8_t* sA;              // two A tiles: 128 rows x 32 bf16 each, canonical K-major layout
  uint32_t sA_addr, sB_addr, mbar_addr;  // shared-window addresses
  uint32_t sB1_addr;        // W1 tile (first layer on the tensor cores)
  uint32_t tmem;            // TMEM base (lane 0, first column)
  unsigned* status;
  uint32_t* gave_up;        // shared, one word per warp: that warp's wait ran out
  uint32_t* last_phase;     // shared: phase of the last MMA commit issued
  uint32_t wait_limit;      // polls per MMA wait before the CTA gives up
  bool row_ok;              // this thread's row exists (y < ny)
  uint32_t phase;           // mbarrier phase of this evaluation (alternates per use)
  __device__ __forceinline__ float operator[](int k) const { return net->v[k]; }
};
constexpr int CLO_TILE_A_BYTES = 128 * 64;
// First layer (9 -> 32) on the tensor cores as well: one K = 16 MMA of the
// bf16 standardised features (zero-padded) against W1, before the 32 x 32
// layer.  0: the first layer on the CUDA cores in fp32.
#ifndef LBM_TC_LAYER1
#define LBM_TC_LAYER1 1
#endif

// Shared-memory matrix descriptor of a K-major tile without swizzle: 8-row x
// 16-byte core matrices, rows 16 B apart, K-adjacent core matrices `lbo`
// bytes apart, M/N-adjacent ones `sbo` bytes apart (tcgen05 descriptor
// format: start >> 4 in bits 0-13, lbo >> 4 in 16-29, sbo >> 4 in 32-45,
// version 1 in 46-47, layout 0 = no swizzle in 61-63).
__host__ __device__ constexpr uint64_t clo_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}
// Instruction descriptor of kind::f16: D f32 (bit 4), A and B bf16 (bits 7,
// 10), both K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28.
constexpr uint32_t CLO_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
// byte offset of element (row, k) in a canonical K-major tile of 32 columns
__host__ __device__ constexpr uint32_t clo_tile_off(int row, int k) {
  return (uint32_t)((row >> 3) * 512 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

namespace {

// Features of a node from its non-equilibrium flux P (xx, yy, zz, xy, xz,
// yz; physical units) and density.
template <class O>
__device__ __forceinline__ void closure_features(const typename O::F (&P)[6], typename O::F rho,
                                                 typename O::F (&x)[CLO_IN]) {
  using F = typename O::F;
  const F off = O::fma(P[3], P[3], O::fma(P[4], P[4], O::mul(P[5], P[5])));
  const F n2 = O::fma(P[0], P[0], O::fma(P[1], P[1], O::fma(P[2], P[2], O::mul(O::splat(2.0f), off))));
  const F n = O::add(O::sqrt(n2), O::splat(1e-30f));
  const F in = O::div(O::splat(1.0f), n);
  F p[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) p[k] = O::mul(P[k], in);
  // tr(p^3) of [[xx,xy,xz],[xy,yy,yz],[xz,yz,zz]]
  const F d3 = O::fma(O::mul(p[0], p[0]), p[0],
                      O::fma(O::mul(p[1], p[1]), p[1], O::mul(O::mul(p[2], p[2]), p[2])));
  const F m3 = O::fma(O::mul(p[3], p[3]), O::add(p[0], p[1]),
                      O::fma(O::mul(p[4], p[4]), O::add(p[0], p[2]),
                             O::mul(O::mul(p[5], p[5]), O::add(p[1], p[2]))));
  const F t3 = O::fma(O::splat(6.0f), O::mul(O::mul(p[3], p[4]), p[5]),
                      O::fma(O::splat(3.0f), m3, d3));
#pragma unroll
  for (int k = 0; k < 6; ++k) x[k] = p[k];
  x[6] = O::log(n);
  x[7] = t3;
  x[8] = O::sub(rho, O::splat(1.0f));
}

// Forward pass: standardised inputs -> ReLU(32) -> ReLU(32) -> softplus.
// w[k] reads parameter k (a CloNet<2> in parameter space, or shared memory).
template <class O, class W>
__device__ __forceinline__ typename O::F closure_mlp(const W& w, const typename O::F (&xr)[CLO_IN]) {
  using F = typename O::F;
  F x[CLO_IN];
#pragma unroll
  for (int j = 0; j < CLO_IN; ++j)
    x[j] = O::mul(O::sub(xr[j], O::splat(w[CLO_MEAN + j])), O::splat(w[CLO_ISCALE + j]));
  F h1[CLO_HID];
#pragma unroll
  for (int i = 0; i < CLO_HID; ++i) {
    F a = O::splat(w[CLO_B1 + i]);
#pragma unroll
    for (int j = 0; j < CLO_IN; ++j) a = O::fma(O::splat(w[CLO_W1 + i * CLO_IN + j]), x[j], a);
    h1[i] = O::relu(a);
  }
  F z = O::splat(w[CLO_B3]);
#pragma unroll
  for (int i = 0; i < CLO_HID; ++i) {
    F a = O::splat(w[CLO_B2 + i]);
#pragma unroll
    for (int j = 0; j < CLO_HID; ++j) a = O::fma(O::splat(w[CLO_W2 + i * CLO_HID + j]), h1[j], a);
    z = O::fma(O::splat(w[CLO_W3 + i]), O::relu(a), z);
  }
  return O::softplus(z);
}

// The tensor-core evaluation of CloNet<3> (see there); every thread of the
// CTA calls it once, with its own node's raw inputs.
// Bounded wait for the mbarrier phase of the given parity: true when it
// completed, per warp (the tensor-memory load after it is warp-collective).
__device__ __forceinline__ bool clo_wait(const CloNet<3>& c, uint32_t parity) {
  uint32_t done = 0;
  for (uint32_t it = 0; it < c.wait_limit && !done; ++it)
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done) : "r"(c.mbar_addr), "r"(parity) : "memory");
  return __all_sync(0xffffffffu, done != 0);
}

// The warp's 32 accumulator columns (its 32 TMEM lanes) into registers.
__device__ __forceinline__ void clo_tmem_ld(const CloNet<3>& c, uint32_t (&v)[CLO_HID]) {
  const uint32_t ta = c.tmem + ((uint32_t)(threadIdx.y * 32) << 16);
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(ta));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// One MMA of K = 16 (kk: which K half of the 32-column tiles) into the
// accumulator; accumulate = 0 overwrites it.
__device__ __forceinline__ void clo_mma(const CloNet<3>& c, uint32_t a_addr, uint32_t b_addr, int accumulate) {
  const uint64_t da = clo_smem_desc(a_addr, 128, 512);
  const uint64_t db = clo_smem_desc(b_addr, 128, 512);
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :: "r"(c.tmem), "l"(da), "l"(db), "r"(CLO_IDESC), "r"(accumulate) : "memory");
}

__device__ __forceinline__ void clo_commit(const CloNet<3>& c, uint32_t parity) {
  *c.last_phase = parity;
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(c.mbar_addr) : "memory");
}

// The A tile is visible to the tensor core and every thread has finished its
// tensor-memory loads; true (uniform) when any warp has given up a wait in
// this launch, in which case every warp marks itself so that none writes an
// A tile again.
__device__ __forceinline__ bool clo_barrier_abort(const CloNet<3>& c, bool warp_gave_up) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  const bool abort = __syncthreads_or(warp_gave_up);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (abort && threadIdx.x == 0) c.gave_up[threadIdx.y] = 1u;
  __syncwarp();
  return abort;
}

__device__ __forceinline__ void clo_give_up(const CloNet<3>& c) {
  if (threadIdx.x == 0) {
    c.gave_up[threadIdx.y] = 1u;
    atomicOr(c.status, 2u);
  }
  __syncwarp();
}

// The tensor-core evaluation of CloNet<3> (see there); every thread of the
// CTA calls it once, with its own node's raw inputs.  With LBM_TC_LAYER1 the
// mbarrier completes twice per evaluation (parities 0 and 1), else once (the
// evaluation's parity).
__device__ __forceinline__ float closure_mlp_tc(const CloNet<3>& c, const float (&xr)[CLO_IN]) {
  const CloNet<2>& w = *c.net;
  const int r = threadIdx.y * 32 + threadIdx.x;
  float x[CLO_IN];
#pragma unroll
  for (int j = 0; j < CLO_IN; ++j) x[j] = __fmul_rn(__fsub_rn(xr[j], w.v[CLO_MEAN + j]), w.v[CLO_ISCALE + j]);
  // this warp's own mark (only it writes it): the same value in every lane
  const bool warp_gave_up = c.gave_up[threadIdx.y] != 0;
  const uint32_t buf = c.phase * CLO_TILE_A_BYTES;
  uint8_t* row = c.sA + buf + clo_tile_off(r, 0);
  uint32_t hp[CLO_HID / 2];
  uint32_t parity2 = c.phase;  // parity of the hidden layer's commit
  if constexpr (LBM_TC_LAYER1) {
    // A = the features in bf16, k < 9, zeros to k = 16
    uint32_t xp[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float lo = 2 * q < CLO_IN ? x[2 * q] : 0.f, hi = 2 * q + 1 < CLO_IN ? x[2 * q + 1] : 0.f;
      const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
      xp[q] = *reinterpret_cast<const uint32_t*>(&h);
    }
    if (!warp_gave_up) {
      *reinterpret_cast<uint4*>(row) = make_uint4(xp[0], xp[1], xp[2], xp[3]);
      *reinterpret_cast<uint4*>(row + 128) = make_uint4(xp[4], xp[5], xp[6], xp[7]);
    }
    if (clo_barrier_abort(c, warp_gave_up)) return 1.0f;
    if (r == 0) {
      clo_mma(c, c.sA_addr + buf, c.sB1_addr, 0);
      clo_commit(c, 0u);
    }
    bool mine = !warp_gave_up;
    if (!clo_wait(c, 0u)) {  // gave up: r = 1 after the next barrier
      clo_give_up(c);
      mine = false;
    }
    if (mine) {
      __syncwarp();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t d[CLO_HID];
      clo_tmem_ld(c, d);
#pragma unroll
      for (int i = 0; i < CLO_HID; i += 2) {
        const float a0 = __fadd_rn(__uint_as_float(d[i]), w.v[CLO_B1 + i]);
        const float a1 = __fadd_rn(__uint_as_float(d[i + 1]), w.v[CLO_B1 + i + 1]);
        const __nv_bfloat162 h = __floats2bfloat162_rn(fmaxf(a0, 0.f), fmaxf(a1, 0.f));
        hp[i / 2] = *reinterpret_cast<const uint32_t*>(&h);
      }
      // the first MMA has completed: its A tile may be overwritten
#pragma unroll
      for (int q = 0; q < 4; ++q)
        *reinterpret_cast<uint4*>(row + q * 128) =
            make_uint4(hp[4 * q], hp[4 * q + 1], hp[4 * q + 2], hp[4 * q + 3]);
    }
    parity2 = 1u;
    if (clo_barrier_abort(c, c.gave_up[threadIdx.y] != 0)) return 1.0f;
  } else {
#pragma unroll
    for (int i = 0; i < CLO_HID; i += 2) {
      float a0 = w.v[CLO_B1 + i], a1 = w.v[CLO_B1 + i + 1];
#pragma unroll
      for (int j = 0; j < CLO_IN; ++j) {
        a0 = __fmaf_rn(w.v[CLO_W1 + i * CLO_IN + j], x[j], a0);
        a1 = __fmaf_rn(w.v[CLO_W1 + (i + 1) * CLO_IN + j], x[j], a1);
      }
      const __nv_bfloat162 h = __floats2bfloat162_rn(fmaxf(a0, 0.f), fmaxf(a1, 0.f));
      hp[i / 2] = *reinterpret_cast<const uint32_t*>(&h);
    }
    if (!warp_gave_up) {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        *reinterpret_cast<uint4*>(row + q * 128) =
            make_uint4(hp[4 * q], hp[4 * q + 1], hp[4 * q + 2], hp[4 * q + 3]);
    }
    if (clo_barrier_abort(c, warp_gave_up)) return 1.0f;  // no more MMAs
  }
  if (r == 0) {
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) clo_mma(c, c.sA_addr + buf + kk * 256, c.sB_addr + kk * 256, kk);
    clo_commit(c, parity2);
  }
  if (!clo_wait(c, parity2)) {  // gave up: plain Smagorinsky, error reported at sync
    clo_give_up(c);
    return 1.0f;
  }
  __syncwarp();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  uint32_t v[CLO_HID];
  clo_tmem_ld(c, v);
  float z = w.v[CLO_B3];
#pragma unroll
  for (int i = 0; i < CLO_HID; ++i)
    z = __fmaf_rn(w.v[CLO_W3 + i], fmaxf(__fadd_rn(__uint_as_float(v[i]), w.v[CLO_B2 + i]), 0.f), z);
  return Ops1::softplus(z);
}

}  // namespace
}  // namespace lbm
