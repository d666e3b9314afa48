// Batched physics-mode step: many independent domains of uneven size, one
// launch per step (graph mode) or one cooperative launch for many steps
// (persistent mode).
//
// Work list.  Every domain is cut into tiles of 32 (64 when a thread takes two
// nodes) x R x Z nodes (R rows per block, Z z-planes per thread, chosen by the
// schedule/autotuner); tiles are
// numbered domain after domain; a table gives each tile's domain and its
// index within the domain, and the block copies that domain's parameters
// into shared memory.  The node update is the single-domain step_row / step_row2
// (phys_step.cuh) chosen by the same rule, so a domain advanced in a batch is
// bit-identical to the same domain advanced alone.
//
// Persistent mode.  A grid of co-resident blocks (cooperative launch) walks
// the tile list grid-stride, then meets at a grid barrier before the next
// step.  The barrier wait is bounded: after spin_limit cycles a block records
// BATCH_STATUS_TIMEOUT and returns, so a barrier that can never complete ends
// the kernel with an error status instead of a hang.
#include <cuda_runtime.h>

#include "batch_internal.h"
#include "phys_step.cuh"

namespace lbm {
namespace {

__device__ __forceinline__ void load_tile(const BatchDomain* __restrict__ dp,
                                          const uint2* __restrict__ tiles, uint32_t t,
                                          BatchDomain& sD, uint32_t& s_local) {
  __shared__ uint32_t s_dom;
  const int tid = threadIdx.x + 32 * threadIdx.y;
  if (tid == 0) {
    const uint2 e = tiles[t];
    s_dom = e.x;
    s_local = e.y;
  }
  __syncthreads();
  const uint32_t* src = reinterpret_cast<const uint32_t*>(dp + s_dom);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&sD);
  constexpr int W = sizeof(BatchDomain) / 4;
  for (int i = tid; i < W; i += blockDim.x * blockDim.y) dst[i] = src[i];
  __syncthreads();
}

template <int PREC, int COLL, bool WM, int P>
__device__ __forceinline__ void batch_tile(const BatchDomain& D, uint32_t local, int nzt,
                                           unsigned* __restrict__ status) {
  const int tx = (int)(local % (uint32_t)D.tiles_x);
  const uint32_t r = local / (uint32_t)D.tiles_x;
  const int ty = (int)(r % (uint32_t)D.tiles_y);
  const int tz = (int)(r / (uint32_t)D.tiles_y);
  const int y = ty * (int)blockDim.y + (int)threadIdx.y;
  if (y >= D.p.g.ny) return;  // uniform over the warp
  for (int k = 0; k < nzt; ++k) {
    const int z = tz * nzt + k;
    if (z >= D.p.g.nz) break;
    if (LBM_BATCH_PAIRS && D.pairs)  // uniform over the block
      step_row2<PREC, COLL, 0, false, WM, P>(D.p, CloNet<0>{}, D.pop, D.flags, D.links, D.rho, D.u,
                                             status, tx * 64, y, z);
    else
      step_row<PREC, COLL, 0, false, WM, P>(D.p, CloNet<0>{}, D.pop, D.flags, D.links, D.rho, D.u,
                                            status, tx * 32, y, z);
  }
}

#ifndef LBM_BATCH_MINB
#define LBM_BATCH_MINB 4
#endif
#ifndef LBM_BATCH_PMINB
#define LBM_BATCH_PMINB 2
#endif

template <int PREC, int COLL, bool WM, int P>
__global__ void __launch_bounds__(256, LBM_BATCH_MINB)
    k_batch_step(const BatchDomain* __restrict__ dp, const uint2* __restrict__ tiles, int nzt,
                 unsigned* status) {
  __shared__ BatchDomain sD;
  __shared__ uint32_t s_local;
  load_tile(dp, tiles, blockIdx.x, sD, s_local);
  batch_tile<PREC, COLL, WM, P>(sD, s_local, nzt, status);
}

// Grid barrier with a bounded wait.  bar[0] counts arrivals, bar[1] is the
// generation.  The last arriver resets the count, then bumps the generation.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned expected, long long spin,
                                             unsigned* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    volatile unsigned* vgen = bar + 1;
    const unsigned gen = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u) + 1u;
    int ok = 1;
    if (arrived == expected) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const long long t0 = clock64();
      while (*vgen == gen) {
        if (clock64() - t0 > spin) {
          ok = 0;
          atomicOr(status, BATCH_STATUS_TIMEOUT);
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  __threadfence();
  return s_ok != 0;
}

// write_last: the last step writes the moments (0 for the chunks a CUDA
// graph replays before the call's final launch).  A launch that finds the
// timeout bit already set (an earlier barrier gave up; the state needs a new
// init) returns at once, so replayed chunks after a timeout cost nothing.
template <int PREC, int COLL>
__global__ void __launch_bounds__(256, LBM_BATCH_PMINB)
    k_batch_persistent(const BatchDomain* __restrict__ dp, const uint2* __restrict__ tiles,
                       uint32_t ntiles, int nzt,
                       int nsteps, int P0, int write_last, unsigned* bar, unsigned expected,
                       long long spin, unsigned* status) {
  __shared__ BatchDomain sD;
  __shared__ uint32_t s_local;
  if (*reinterpret_cast<volatile unsigned*>(status) & BATCH_STATUS_TIMEOUT) return;  // same for every block
  // one tile loop per (parity, moment write) variant, chosen once per step
  auto tiles_of_step = [&](auto wm_tag, auto p_tag) {
    constexpr bool WM = decltype(wm_tag)::value != 0;
    constexpr int P = decltype(p_tag)::value;
#pragma unroll 1
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
      load_tile(dp, tiles, t, sD, s_local);
      batch_tile<PREC, COLL, WM, P>(sD, s_local, nzt, status);
      __syncthreads();  // sD is rewritten by the next tile
    }
  };
#pragma unroll 1
  for (int st = 0; st < nsteps; ++st) {
    const int P = (P0 + st) & 1;
    const bool wm = write_last && st == nsteps - 1;
    if (P) {
      if (wm) tiles_of_step(IC<1>{}, IC<1>{});
      else tiles_of_step(IC<0>{}, IC<1>{});
    } else {
      if (wm) tiles_of_step(IC<1>{}, IC<0>{});
      else tiles_of_step(IC<0>{}, IC<0>{});
    }
    if (st + 1 < nsteps && !grid_barrier(bar, expected, spin, status)) return;
  }
}

template <int PREC, int COLL>
cudaError_t step_launch(const BatchLaunch& L, int P, bool wm, cudaStream_t s) {
  const dim3 blk(32, L.rows, 1);
#define LBM_BATCH_LAUNCH(WM, PAR) \
  k_batch_step<PREC, COLL, WM, PAR><<<L.ntiles, blk, 0, s>>>(L.dom, L.tiles, L.nzt, L.status)
  if (wm) {
    if (P) LBM_BATCH_LAUNCH(true, 1); else LBM_BATCH_LAUNCH(true, 0);
  } else {
    if (P) LBM_BATCH_LAUNCH(false, 1); else LBM_BATCH_LAUNCH(false, 0);
  }
#undef LBM_BATCH_LAUNCH
  return cudaGetLastError();
}

template <int PREC, int COLL>
void* persistent_fn() {
  return reinterpret_cast<void*>(&k_batch_persistent<PREC, COLL>);
}

void* pick_persistent(int prec, int coll) {
  if (prec == LBM_PREC_F32) return coll ? persistent_fn<LBM_PREC_F32, 1>() : persistent_fn<LBM_PREC_F32, 0>();
  if (prec == LBM_PREC_F16S) return coll ? persistent_fn<LBM_PREC_F16S, 1>() : persistent_fn<LBM_PREC_F16S, 0>();
  return coll ? persistent_fn<LBM_PREC_BF16S, 1>() : persistent_fn<LBM_PREC_BF16S, 0>();
}

}  // namespace

cudaError_t batch_step(const BatchLaunch& L, int P, bool wm, cudaStream_t s) {
  const bool trt = L.collision == LBM_COLL_TRT;
  switch (L.precision) {
    case LBM_PREC_F32: return trt ? step_launch<LBM_PREC_F32, 1>(L, P, wm, s) : step_launch<LBM_PREC_F32, 0>(L, P, wm, s);
    case LBM_PREC_F16S: return trt ? step_launch<LBM_PREC_F16S, 1>(L, P, wm, s) : step_launch<LBM_PREC_F16S, 0>(L, P, wm, s);
    default: return trt ? step_launch<LBM_PREC_BF16S, 1>(L, P, wm, s) : step_launch<LBM_PREC_BF16S, 0>(L, P, wm, s);
  }
}

cudaError_t batch_persistent_grid(const BatchLaunch& L, int* grid) {
  int per_sm = 0, dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pick_persistent(L.precision, L.collision),
                                                      32 * L.rows, 0);
  if (e != cudaSuccess) return e;
  long long g = (long long)per_sm * sms;
  if (g > (long long)L.ntiles) g = L.ntiles;
  *grid = (int)(g < 1 ? 1 : g);
  return per_sm > 0 ? cudaSuccess : cudaErrorInvalidConfiguration;
}

cudaError_t batch_persistent(const BatchLaunch& L, int nsteps, int P0, int grid, cudaStream_t s,
                             bool write_last) {
  // the barrier state is reset by a memset node before every launch, so a
  // captured launch starts from zero at each replay
  cudaError_t e = cudaMemsetAsync(L.bar, 0, 2 * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  const unsigned expected = (unsigned)grid + (unsigned)L.missing_blocks;
  long long spin = L.spin_limit;
  BatchDomain* dom = L.dom;
  const uint2* tiles = L.tiles;
  int nzt = L.nzt;
  uint32_t ntiles = L.ntiles;
  int wl = write_last ? 1 : 0;
  unsigned* bar = L.bar;
  unsigned* status = L.status;
  void* args[] = {&dom, (void*)&tiles, &ntiles, &nzt, &nsteps, &P0, &wl, &bar, (void*)&expected, &spin, &status};
  // a cooperative launch through cudaLaunchKernelExC, which stream capture
  // records as a cooperative kernel node
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(32, L.rows, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, pick_persistent(L.precision, L.collision), args);
}

}  // namespace lbm
