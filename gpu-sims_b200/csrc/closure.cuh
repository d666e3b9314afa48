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

}  // namespace
}  // namespace lbm
