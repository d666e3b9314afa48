// Arithmetic policies of the collision and the closure MLP: one node per
// thread (Ops1) or two nodes per thread in the lanes of Blackwell's packed
// fp32 instructions (Ops2).
#pragma once
#include <cuda_runtime.h>

namespace lbm {
namespace {

// Arithmetic policies for the collision.  Every operation is an explicitly
// rounded intrinsic, so the one-node policy and the two-node policy built on
// Blackwell's packed fp32 instructions (FADD2/FMUL2/FFMA2: one instruction
// for two lanes' values) evaluate the same operation graph.  The scalar
// intrinsics are never contracted; ptxas does merge a packed multiply into a
// packed add that consumes it (even when both carry an explicit .rn, and
// with ptxas contraction switched off), so the two policies agree bit for
// bit where the code is fma-shaped, and otherwise to within an ulp per
// merged pair.
struct Ops1 {
  using F = float;
  static __device__ __forceinline__ F splat(float c) { return c; }
  static __device__ __forceinline__ F add(F a, F b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ F sub(F a, F b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ F mul(F a, F b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ F fma(F a, F b, F c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ F div(F a, F b) { return __fdiv_rn(a, b); }
  // a / b to about 2 ulp (CUDA's fast division; b of order 1 here)
  static __device__ __forceinline__ F div_fast(F a, F b) { return __fdividef(a, b); }
  static __device__ __forceinline__ F sqrt(F a) { return __fsqrt_rn(a); }
  static __device__ __forceinline__ F log(F a) { return logf(a); }
  static __device__ __forceinline__ F relu(F a) { return fmaxf(a, 0.0f); }
  // log(1 + e^z), = z above 20 where the difference is below fp32 resolution
  static __device__ __forceinline__ F softplus(F z) { return z > 20.0f ? z : log1pf(expf(z)); }
};
struct Ops2 {
  using F = float2;
  static __device__ __forceinline__ F splat(float c) { return make_float2(c, c); }
  static __device__ __forceinline__ F add(F a, F b) { return __fadd2_rn(a, b); }
  // a - b as b * (-1) + a: the product is exact, so the single rounding
  // equals that of a - b.
  static __device__ __forceinline__ F sub(F a, F b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
  static __device__ __forceinline__ F mul(F a, F b) { return __fmul2_rn(a, b); }
  static __device__ __forceinline__ F fma(F a, F b, F c) { return __ffma2_rn(a, b, c); }
  static __device__ __forceinline__ F div(F a, F b) {
    return make_float2(__fdiv_rn(a.x, b.x), __fdiv_rn(a.y, b.y));
  }
  static __device__ __forceinline__ F div_fast(F a, F b) {
    return make_float2(__fdividef(a.x, b.x), __fdividef(a.y, b.y));
  }
  static __device__ __forceinline__ F sqrt(F a) { return make_float2(__fsqrt_rn(a.x), __fsqrt_rn(a.y)); }
  static __device__ __forceinline__ F log(F a) { return make_float2(Ops1::log(a.x), Ops1::log(a.y)); }
  static __device__ __forceinline__ F relu(F a) { return make_float2(fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f)); }
  static __device__ __forceinline__ F softplus(F z) {
    return make_float2(Ops1::softplus(z.x), Ops1::softplus(z.y));
  }
};
}  // namespace
}  // namespace lbm
