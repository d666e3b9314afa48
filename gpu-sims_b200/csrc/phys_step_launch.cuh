// Launchers of the physics-mode step kernels, instantiated once per storage
// precision by phys_step_{f32,f16,bf16}.cu (split so the three compile in
// parallel).  The kernels wrap step_row / step_row2 (phys_step.cuh).
#pragma once
#include "phys_step.cuh"

namespace lbm {
namespace {

#ifndef LBM_STEP2_MINB
#define LBM_STEP2_MINB 5
#endif

// Two nodes per thread (step_pairs(nx)): a warp covers 64 consecutive x.
template <int PREC, int COLL, bool SMAG, bool FORCE, bool WRITE_MOMENTS, int P>
__global__ void __launch_bounds__(STEP_THREADS, LBM_STEP2_MINB)
    k_phys_step2(PhysParams p, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                 const uint32_t* __restrict__ links, float* __restrict__ rho_o,
                 float* __restrict__ u_o, unsigned* __restrict__ status) {
  const int y = blockIdx.y * STEP_BY + threadIdx.y;
  if (y >= p.g.ny) return;  // uniform over the warp
  step_row2<PREC, COLL, SMAG, FORCE, WRITE_MOMENTS, P>(p, pop_v, flags, links, rho_o, u_o, status,
                                                       blockIdx.x * 64, y, blockIdx.z);
}

template <int PREC, int COLL, bool SMAG, bool FORCE, bool WRITE_MOMENTS, int P>
__global__ void __launch_bounds__(STEP_THREADS, LBM_STEP_MINB)
    k_phys_step(PhysParams p, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                const uint32_t* __restrict__ links, float* __restrict__ rho_o,
                float* __restrict__ u_o, unsigned* __restrict__ status) {
  const int y = blockIdx.y * STEP_BY + threadIdx.y;
  if (y >= p.g.ny) return;  // uniform over the warp
  step_row<PREC, COLL, SMAG, FORCE, WRITE_MOMENTS, P>(p, pop_v, flags, links, rho_o, u_o, status,
                                                      blockIdx.x * 32, y, blockIdx.z);
}

template <int PREC, int COLL, bool SMAG, bool FORCE>
cudaError_t launch_step(const Ctx& c, int P, bool wm, cudaStream_t s) {
  const PhysGeom& G = c.pp.g;
  const dim3 blk(32, STEP_BY, 1);
  if (step_pairs(G.nx)) {
    const dim3 grd((G.nx + 63) / 64, (G.ny + STEP_BY - 1) / STEP_BY, G.nz);
#define LBM_STEP_LAUNCH(WM, PAR)                                          \
  k_phys_step2<PREC, COLL, SMAG, FORCE, WM, PAR><<<grd, blk, 0, s>>>(     \
      c.pp, c.pop, c.flags, c.links, c.rho, c.u, c.status)
    if (wm) {
      if (P) LBM_STEP_LAUNCH(true, 1); else LBM_STEP_LAUNCH(true, 0);
    } else {
      if (P) LBM_STEP_LAUNCH(false, 1); else LBM_STEP_LAUNCH(false, 0);
    }
#undef LBM_STEP_LAUNCH
    return cudaGetLastError();
  }
  const dim3 grd((G.nx + 31) / 32, (G.ny + STEP_BY - 1) / STEP_BY, G.nz);
#define LBM_STEP_LAUNCH(WM, PAR)                                          \
  k_phys_step<PREC, COLL, SMAG, FORCE, WM, PAR><<<grd, blk, 0, s>>>(      \
      c.pp, c.pop, c.flags, c.links, c.rho, c.u, c.status)
  if (wm) {
    if (P) LBM_STEP_LAUNCH(true, 1); else LBM_STEP_LAUNCH(true, 0);
  } else {
    if (P) LBM_STEP_LAUNCH(false, 1); else LBM_STEP_LAUNCH(false, 0);
  }
#undef LBM_STEP_LAUNCH
  return cudaGetLastError();
}

template <int PREC, int COLL, bool SMAG>
cudaError_t dispatch_force(const Ctx& c, int P, bool wm, cudaStream_t s) {
  const bool force = c.pp.accel[0] != 0.f || c.pp.accel[1] != 0.f || c.pp.accel[2] != 0.f;
  return force ? launch_step<PREC, COLL, SMAG, true>(c, P, wm, s)
               : launch_step<PREC, COLL, SMAG, false>(c, P, wm, s);
}

template <int PREC, int COLL>
cudaError_t dispatch_smag(const Ctx& c, int P, bool wm, cudaStream_t s) {
  return c.pp.smag_cs > 0.f ? dispatch_force<PREC, COLL, true>(c, P, wm, s)
                            : dispatch_force<PREC, COLL, false>(c, P, wm, s);
}

template <int PREC>
cudaError_t dispatch_coll(const Ctx& c, int P, bool wm, cudaStream_t s) {
  return c.d.collision == LBM_COLL_TRT ? dispatch_smag<PREC, LBM_COLL_TRT>(c, P, wm, s)
                                       : dispatch_smag<PREC, LBM_COLL_BGK>(c, P, wm, s);
}

}  // namespace
}  // namespace lbm

#define LBM_DEFINE_PHYS_STEP(NAME, PREC)                                           \
  namespace lbm {                                                                  \
  cudaError_t NAME(const Ctx& c, int parity, bool write_moments, cudaStream_t s) { \
    return dispatch_coll<PREC>(c, parity, write_moments, s);                       \
  }                                                                                \
  }
