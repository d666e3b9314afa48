// Physics-mode kernels: one fused stream+collide launch per step on a single
// in-place population store (esoteric pull).
//
// Layout.  Each opposite pair (a, b = opp a) with forward vector d = c_a owns
// two slot arrays S0, S1; the rest population owns one.  A launch of parity P
// touches, for node n, exactly two slots of each pair,
//     X = S[1-P](n)      and      Y = S[P](n + d),
// reads the streamed-in f_a from X and f_b from Y, and writes the new
// post-collision f*_b to X and f*_a to Y.  Between launches this means
//     before parity 0:  S0(m) = f*_b(m),      S1(m) = f*_a(m - d)
//     before parity 1:  S0(m) = f*_a(m - d),  S1(m) = f*_b(m)
// so every launch streams and collides with no second buffer and no two
// threads touching one slot.
//
// Half-way bounce-back.  If n + d is a wall, f_b(n) arrives as the f*_a(n)
// that n itself wrote at the previous launch, which sits in the other slot of
// the same location: S[1-P](n + d).  If n - d is a wall, f_a(n) arrives as
// f*_b(n) from S[P](n).  Nobody else touches those slots (the node beyond is
// a solid that never runs, or a ghost).  Non-periodic faces therefore carry
// one ghost layer; periodic axes wrap.  Moving walls add the momentum term
// 6 w_i rho_w (c_i . u_w), rho_w = 1.
//
// Populations are stored shifted, g_i = f_i - w_i, in fp32, fp16 (scaled by
// 2^12) or bf16; all arithmetic is fp32.
#include "phys_step.cuh"

namespace lbm {
namespace {

// Places post-collision populations (shifted) of node n where the next
// launch of parity P expects them: f*_a(n) -> S[1-P](n + d), f*_b(n) ->
// S[P](n), rest -> R(n).  Used by init and by lbm_write_populations.
template <int PREC>
__device__ __forceinline__ void place(const PhysGeom& G, int P, typename Store<PREC>::T* pop,
                                      int x, int y, int z, const float (&g)[Q]) {
  using S = Store<PREC>;
  const size_t SS = G.slot_stride;
  const size_t ln = lin(G, x, y, z);
  S::st(pop, ln, g[0]);
  static_for<0, 9>([&](auto PI) {
    constexpr int pi = decltype(PI)::value;
    constexpr int a = pair_a(pi), b = pair_b(pi);
    auto* s0 = pop + (size_t)(1 + 2 * pi) * SS;
    auto* s1 = s0 + SS;
    S::st(P ? s0 : s1, lin_fwd<cx(a), cy(a), cz(a)>(G, x, y, z), g[a]);
    S::st(P ? s1 : s0, ln, g[b]);
  });
}

template <int PREC>
__device__ __forceinline__ void fetch(const PhysGeom& G, int P, const typename Store<PREC>::T* pop,
                                      int x, int y, int z, float (&g)[Q]) {
  using S = Store<PREC>;
  const size_t SS = G.slot_stride;
  const size_t ln = lin(G, x, y, z);
  g[0] = S::ld(pop, ln);
  static_for<0, 9>([&](auto PI) {
    constexpr int pi = decltype(PI)::value;
    constexpr int a = pair_a(pi), b = pair_b(pi);
    const auto* s0 = pop + (size_t)(1 + 2 * pi) * SS;
    const auto* s1 = s0 + SS;
    g[a] = S::ld(P ? s0 : s1, lin_fwd<cx(a), cy(a), cz(a)>(G, x, y, z));
    g[b] = S::ld(P ? s1 : s0, ln);
  });
}

// f = feq(rho, u) at every fluid node, stored for a launch of parity P.
template <int PREC>
__global__ void __launch_bounds__(256)
    k_phys_init(PhysGeom G, int P, const float* __restrict__ rho_in, const float* __restrict__ u_in,
                float rho0, float u0x, float u0y, float u0z, void* __restrict__ pop_v,
                const uint8_t* __restrict__ flags, float* __restrict__ rho_o,
                float* __restrict__ u_o) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= G.nx || y >= G.ny || z >= G.nz) return;
  const size_t N = G.n;
  const size_t nid = (size_t)x + (size_t)G.nx * ((size_t)y + (size_t)G.ny * (size_t)z);
  if (flags[nid] & FLAG_SOLID) {
    rho_o[nid] = 0.0f;
    u_o[nid] = u_o[N + nid] = u_o[2 * N + nid] = 0.0f;
    return;
  }
  float r = rho0, vx = u0x, vy = u0y, vz = u0z;
  if (rho_in) r = rho_in[nid];
  if (u_in) {
    vx = u_in[nid];
    vy = u_in[N + nid];
    vz = u_in[2 * N + nid];
  }
  const float drho = r - 1.0f;
  const float uu15 = 1.5f * (vx * vx + vy * vy + vz * vz);
  float g[Q];
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    const float cu = cx(i) * vx + cy(i) * vy + cz(i) * vz;
    g[i] = wf(i) * (drho + r * (3.0f * cu + 4.5f * cu * cu - uu15));
  });
  place<PREC>(G, P, reinterpret_cast<typename Store<PREC>::T*>(pop_v), x, y, z, g);
  rho_o[nid] = r;
  u_o[nid] = vx;
  u_o[N + nid] = vy;
  u_o[2 * N + nid] = vz;
}

template <int PREC>
__global__ void __launch_bounds__(256)
    k_phys_read(PhysGeom G, int P, const void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                float* __restrict__ out, int shifted) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= G.nx || y >= G.ny || z >= G.nz) return;
  const size_t nid = (size_t)x + (size_t)G.nx * ((size_t)y + (size_t)G.ny * (size_t)z);
  float g[Q];
  if (flags[nid] & FLAG_SOLID) {
    static_for<0, Q>([&](auto I) { out[(size_t)I.value * G.n + nid] = 0.0f; });
    return;
  }
  fetch<PREC>(G, P, reinterpret_cast<const typename Store<PREC>::T*>(pop_v), x, y, z, g);
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    out[(size_t)i * G.n + nid] = shifted ? g[i] : g[i] + wf(i);
  });
}

template <int PREC>
__global__ void __launch_bounds__(256)
    k_phys_write(PhysGeom G, int P, void* __restrict__ pop_v, const uint8_t* __restrict__ flags,
                 const float* __restrict__ in, int shifted) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= G.nx || y >= G.ny || z >= G.nz) return;
  const size_t nid = (size_t)x + (size_t)G.nx * ((size_t)y + (size_t)G.ny * (size_t)z);
  if (flags[nid] & FLAG_SOLID) return;
  float g[Q];
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    g[i] = shifted ? in[(size_t)i * G.n + nid] : in[(size_t)i * G.n + nid] - wf(i);
  });
  place<PREC>(G, P, reinterpret_cast<typename Store<PREC>::T*>(pop_v), x, y, z, g);
}

dim3 phys_block() { return dim3(32, 4, 2); }
dim3 phys_grid(const PhysGeom& g) {
  const dim3 b = phys_block();
  return dim3((g.nx + b.x - 1) / b.x, (g.ny + b.y - 1) / b.y, (g.nz + b.z - 1) / b.z);
}

}  // namespace

bool step_pairs_host(int nx) { return step_pairs(nx); }

// The step kernels of each storage precision are compiled in their own
// translation unit (phys_step_f32.cu, phys_step_f16.cu, phys_step_bf16.cu),
// and so are their learned-closure variants (phys_step_clo_*.cu).
cudaError_t phys_step(const Ctx& c, int parity, bool write_moments, cudaStream_t s) {
  if (c.closure) {
    switch (c.d.precision) {
      case LBM_PREC_F32: return phys_step_clo_f32(c, parity, write_moments, s);
      case LBM_PREC_F16S: return phys_step_clo_f16(c, parity, write_moments, s);
      default: return phys_step_clo_bf16(c, parity, write_moments, s);
    }
  }
  switch (c.d.precision) {
    case LBM_PREC_F32: return phys_step_f32(c, parity, write_moments, s);
    case LBM_PREC_F16S: return phys_step_f16(c, parity, write_moments, s);
    default: return phys_step_bf16(c, parity, write_moments, s);
  }
}

cudaError_t phys_init(const Ctx& c, const float* rho, const float* u3, float rho0, const float* u0,
                      cudaStream_t s) {
  const float zero[3] = {0.f, 0.f, 0.f};
  if (!u0) u0 = zero;
  const PhysGeom& G = c.pp.g;
  switch (c.d.precision) {
    case LBM_PREC_F32:
      k_phys_init<LBM_PREC_F32><<<phys_grid(G), phys_block(), 0, s>>>(
          G, c.parity, rho, u3, rho0, u0[0], u0[1], u0[2], c.pop, c.flags, c.rho, c.u);
      break;
    case LBM_PREC_F16S:
      k_phys_init<LBM_PREC_F16S><<<phys_grid(G), phys_block(), 0, s>>>(
          G, c.parity, rho, u3, rho0, u0[0], u0[1], u0[2], c.pop, c.flags, c.rho, c.u);
      break;
    default:
      k_phys_init<LBM_PREC_BF16S><<<phys_grid(G), phys_block(), 0, s>>>(
          G, c.parity, rho, u3, rho0, u0[0], u0[1], u0[2], c.pop, c.flags, c.rho, c.u);
  }
  return cudaGetLastError();
}

cudaError_t phys_read_pops(const Ctx& c, float* out, cudaStream_t s, bool shifted) {
  const PhysGeom& G = c.pp.g;
  switch (c.d.precision) {
    case LBM_PREC_F32:
      k_phys_read<LBM_PREC_F32><<<phys_grid(G), phys_block(), 0, s>>>(G, c.parity, c.pop, c.flags, out, shifted ? 1 : 0);
      break;
    case LBM_PREC_F16S:
      k_phys_read<LBM_PREC_F16S><<<phys_grid(G), phys_block(), 0, s>>>(G, c.parity, c.pop, c.flags, out, shifted ? 1 : 0);
      break;
    default:
      k_phys_read<LBM_PREC_BF16S><<<phys_grid(G), phys_block(), 0, s>>>(G, c.parity, c.pop, c.flags, out, shifted ? 1 : 0);
  }
  return cudaGetLastError();
}

cudaError_t phys_write_pops(const Ctx& c, const float* in, cudaStream_t s, bool shifted) {
  const PhysGeom& G = c.pp.g;
  switch (c.d.precision) {
    case LBM_PREC_F32:
      k_phys_write<LBM_PREC_F32><<<phys_grid(G), phys_block(), 0, s>>>(G, c.parity, c.pop, c.flags, in, shifted ? 1 : 0);
      break;
    case LBM_PREC_F16S:
      k_phys_write<LBM_PREC_F16S><<<phys_grid(G), phys_block(), 0, s>>>(G, c.parity, c.pop, c.flags, in, shifted ? 1 : 0);
      break;
    default:
      k_phys_write<LBM_PREC_BF16S><<<phys_grid(G), phys_block(), 0, s>>>(G, c.parity, c.pop, c.flags, in, shifted ? 1 : 0);
  }
  return cudaGetLastError();
}

}  // namespace lbm
