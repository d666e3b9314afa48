// D3Q19 lattice tables and the two equilibrium forms used by the kernels.
//
// Direction order is the reference's (shaders/lattice_constants.glsl:23-43):
//   0 rest, 1..6 faces (+x,-x,+y,-y,+z,-z), 7..10 xy edges (++,+-,-+,--),
//   11..14 xz edges, 15..18 yz edges; opposite table :55-75.
// Every accessor is a constexpr function so that, inside fully unrolled
// loops, directions resolve at compile time and no table lives in memory.
#pragma once
#include <cstdint>

namespace lbm {

constexpr int Q = 19;

__host__ __device__ constexpr int cx(int i) {
  return (i == 1 || i == 7 || i == 8 || i == 11 || i == 12) ? 1
       : (i == 2 || i == 9 || i == 10 || i == 13 || i == 14) ? -1 : 0;
}
__host__ __device__ constexpr int cy(int i) {
  return (i == 3 || i == 7 || i == 9 || i == 15 || i == 16) ? 1
       : (i == 4 || i == 8 || i == 10 || i == 17 || i == 18) ? -1 : 0;
}
__host__ __device__ constexpr int cz(int i) {
  return (i == 5 || i == 11 || i == 13 || i == 15 || i == 17) ? 1
       : (i == 6 || i == 12 || i == 14 || i == 16 || i == 18) ? -1 : 0;
}
__host__ __device__ constexpr int opp(int i) {
  return i == 0 ? 0
       : i <= 6 ? ((i & 1) ? i + 1 : i - 1)
       : (i == 7) ? 10 : (i == 8) ? 9 : (i == 9) ? 8 : (i == 10) ? 7
       : (i == 11) ? 14 : (i == 12) ? 13 : (i == 13) ? 12 : (i == 14) ? 11
       : (i == 15) ? 18 : (i == 16) ? 17 : (i == 17) ? 16 : 15;
}
// Weights in fp32, each the correctly rounded value of 1/3, 1/18, 1/36
// (shaders/lattice_constants.glsl:46-52 evaluates 1.0/3.0 etc. in float).
__host__ __device__ constexpr float wf(int i) {
  return i == 0 ? 1.0f / 3.0f : (i <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f);
}

// Opposite pairs (a, b = opp(a)), a < b.  The esoteric-pull layout keeps two
// slots per pair; the "forward" direction of a pair is c_a.
__host__ __device__ constexpr int pair_a(int p) {
  return p == 0 ? 1 : p == 1 ? 3 : p == 2 ? 5 : p == 3 ? 7 : p == 4 ? 8
       : p == 5 ? 11 : p == 6 ? 12 : p == 7 ? 15 : 16;
}
__host__ __device__ constexpr int pair_b(int p) { return opp(pair_a(p)); }

// Node-classification bits (flag byte per node).
constexpr uint8_t FLAG_SOLID = 1u;     // mask value 1
constexpr uint8_t FLAG_BOUNDARY = 2u;  // fluid node with a blocked link
constexpr uint8_t FLAG_SOLID_LINK = 4u;  // ... of which one ends at a solid node of the grid
// Fluid node on an open x face (physics mode): the row kernels leave it to
// the face kernel, as they leave solid nodes alone.
constexpr uint8_t FLAG_OPEN = 8u;
constexpr uint8_t FLAG_SKIP = FLAG_SOLID | FLAG_OPEN;

// ---------------------------------------------------------------------------
// Reference-literal arithmetic.  Each operation is a separately rounded fp32
// op (no contraction into FMA), in the evaluation order of the GLSL source,
// so that the GPU result equals the CPU restatement bit for bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float rl_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rl_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rl_sub(float a, float b) { return __fsub_rn(a, b); }

// dot(vec3(C_I[i]), u): products with components in {-1,0,1} are exact and
// adding a signed zero leaves a value unchanged, so the dot product reduces
// to the signed sum of the non-zero components, x then y then z.
template <int I>
__device__ __forceinline__ float rl_cdotu(float ux, float uy, float uz) {
  constexpr int X = cx(I), Y = cy(I), Z = cz(I);
  float s = 0.0f;
  bool first = true;
  if (X != 0) { s = X > 0 ? ux : -ux; first = false; }
  if (Y != 0) { s = first ? (Y > 0 ? uy : -uy) : (Y > 0 ? rl_add(s, uy) : rl_sub(s, uy)); first = false; }
  if (Z != 0) { s = first ? (Z > 0 ? uz : -uz) : (Z > 0 ? rl_add(s, uz) : rl_sub(s, uz)); }
  return s;
}

// feq_i (shaders/lattice_constants.glsl:86-93):
//   W_I[i] * rho * (1.0 + 3*cu + 4.5*cu*cu - 1.5*uu)
template <int I>
__device__ __forceinline__ float rl_feq(float rho, float ux, float uy, float uz, float uu) {
  float t;
  if (I == 0) {
    t = rl_sub(1.0f, rl_mul(1.5f, uu));
  } else {
    const float cu = rl_cdotu<I>(ux, uy, uz);
    t = rl_sub(rl_add(rl_add(1.0f, rl_mul(3.0f, cu)), rl_mul(rl_mul(4.5f, cu), cu)),
               rl_mul(1.5f, uu));
  }
  return rl_mul(rl_mul(wf(I), rho), t);
}

__device__ __forceinline__ float rl_udotu(float ux, float uy, float uz) {
  return rl_add(rl_add(rl_mul(ux, ux), rl_mul(uy, uy)), rl_mul(uz, uz));
}

// Compile-time loop helper: calls f(std::integral_constant-like tag) for
// I = 0..N-1 without relying on the optimiser to unroll.
template <int I> struct IC { static constexpr int value = I; };
template <int B, int E, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (B < E) {
    f(IC<B>{});
    static_for<B + 1, E>(f);
  }
}

}  // namespace lbm
