// Launchers of the physics-mode step kernels, instantiated once per storage
// precision by phys_step_{f32,f16,bf16}.cu and, for the learned closure, by
// phys_step_clo_{f32,f16,bf16}.cu (split so the six compile in parallel).  The kernels wrap step_row / step_row2 (phys_step.cuh).
#pragma once
#include "phys_step.cuh"

namespace lbm {
namespace {

#ifndef LBM_STEP2_MINB
#define LBM_STEP2_MINB 5
#endif
// Residency bounds of the learned-closure kernels (the MLP's hidden layer
// stays in registers: two nodes' worth in the pair kernel).
#ifndef LBM_CLO_MINB
#define LBM_CLO_MINB 3
#endif
#ifndef LBM_CLO2_MINB
#define LBM_CLO2_MINB 2
#endif

// Two nodes per thread (step_pairs(nx)): a warp covers 64 consecutive x.
// SGS: 0 none, 1 Smagorinsky, 2 learned closure (net = the network).
template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P>
__global__ void __launch_bounds__(STEP_THREADS, SGS == 2 ? LBM_CLO2_MINB : LBM_STEP2_MINB)
    k_phys_step2(PhysParams p, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                 const uint32_t* __restrict__ links, float* __restrict__ rho_o,
                 float* __restrict__ u_o, unsigned* __restrict__ status,
                 const __grid_constant__ CloNet<SGS> net) {
  const int y = blockIdx.y * STEP_BY + threadIdx.y;
  if (y >= p.g.ny) return;  // uniform over the warp
  step_row2<PREC, COLL, SGS, FORCE, WRITE_MOMENTS, P>(p, net, pop_v, flags, links, rho_o, u_o,
                                                      status, blockIdx.x * 64, y, blockIdx.z);
}

template <int PREC, int COLL, int SGS, bool FORCE, bool WRITE_MOMENTS, int P>
__global__ void __launch_bounds__(STEP_THREADS, SGS == 2 ? LBM_CLO_MINB : LBM_STEP_MINB)
    k_phys_step(PhysParams p, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                const uint32_t* __restrict__ links, float* __restrict__ rho_o,
                float* __restrict__ u_o, unsigned* __restrict__ status,
                const __grid_constant__ CloNet<SGS> net) {
  const int y = blockIdx.y * STEP_BY + threadIdx.y;
  if (y >= p.g.ny) return;  // uniform over the warp
  step_row<PREC, COLL, SGS, FORCE, WRITE_MOMENTS, P>(p, net, pop_v, flags, links, rho_o, u_o,
                                                     status, blockIdx.x * 32, y, blockIdx.z);
}

template <int SGS> CloNet<SGS> net_of(const Ctx&) { return CloNet<SGS>{}; }
template <> CloNet<2> net_of<2>(const Ctx& c) {
  CloNet<2> n;
  for (int k = 0; k < CLO_FLOATS; ++k) n.v[k] = c.clo[k];
  return n;
}

template <int PREC, int COLL, int SGS, bool FORCE>
cudaError_t launch_step(const Ctx& c, int P, bool wm, cudaStream_t s) {
  const PhysGeom& G = c.pp.g;
  const CloNet<SGS> net = net_of<SGS>(c);
  const dim3 blk(32, STEP_BY, 1);
  if (step_pairs(G.nx)) {
    const dim3 grd((G.nx + 63) / 64, (G.ny + STEP_BY - 1) / STEP_BY, G.nz);
#define LBM_STEP_LAUNCH(WM, PAR)                                          \
  k_phys_step2<PREC, COLL, SGS, FORCE, WM, PAR><<<grd, blk, 0, s>>>(      \
      c.pp, c.pop, c.flags, c.links, c.rho, c.u, c.status, net)
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
  k_phys_step<PREC, COLL, SGS, FORCE, WM, PAR><<<grd, blk, 0, s>>>(       \
      c.pp, c.pop, c.flags, c.links, c.rho, c.u, c.status, net)
  if (wm) {
    if (P) LBM_STEP_LAUNCH(true, 1); else LBM_STEP_LAUNCH(true, 0);
  } else {
    if (P) LBM_STEP_LAUNCH(false, 1); else LBM_STEP_LAUNCH(false, 0);
  }
#undef LBM_STEP_LAUNCH
  return cudaGetLastError();
}

template <int PREC, int COLL, int SGS>
cudaError_t dispatch_force(const Ctx& c, int P, bool wm, cudaStream_t s) {
  const bool force = c.pp.accel[0] != 0.f || c.pp.accel[1] != 0.f || c.pp.accel[2] != 0.f;
  return force ? launch_step<PREC, COLL, SGS, true>(c, P, wm, s)
               : launch_step<PREC, COLL, SGS, false>(c, P, wm, s);
}

// CLOSURE: the learned-closure kernels (compiled in their own files; no body
// force, which lbm_set_closure enforces).
template <int PREC, int COLL, bool CLOSURE>
cudaError_t dispatch_smag(const Ctx& c, int P, bool wm, cudaStream_t s) {
  if constexpr (CLOSURE) {
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
