// Node classification, conservation reduction and host-format conversion.
#include <cuda_fp16.h>

#include "d3q19.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace {

// Per node: bit 0 = the node is solid (mask value 1); bit i = the node at
// x + c_i is solid, where a neighbour outside the box counts as solid on a
// non-periodic axis (mask_at, shaders/apply_boundaries.comp.glsl:52-55) and
// wraps on a periodic one.  FLAG_BOUNDARY marks fluid nodes with any link
// bit (the reference-mode step reads the word there); FLAG_OPEN fluid nodes on
// an open x face; FLAG_SOLID_LINK those
// with a link to a solid node of the grid (the physics-mode step derives
// wall links from the coordinates and reads the word only there).
__global__ void __launch_bounds__(256)
    k_classify(int nx, int ny, int nz, int px, int py, int pz, int open_lo, int open_hi,
               const uint8_t* __restrict__ mask, uint8_t* __restrict__ flags, uint32_t* __restrict__ links) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= nx || y >= ny || z >= nz) return;
  const size_t nid = (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * (size_t)z);
  const bool solid = mask[nid] == 1;
  uint32_t L = solid ? 1u : 0u;
  bool to_solid = false;
  static_for<1, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    int xn = x + cx(i), yn = y + cy(i), zn = z + cz(i);
    bool oob = false;
    if (xn < 0 || xn >= nx) { if (px) xn = (xn + nx) % nx; else oob = true; }
    if (yn < 0 || yn >= ny) { if (py) yn = (yn + ny) % ny; else oob = true; }
    if (zn < 0 || zn >= nz) { if (pz) zn = (zn + nz) % nz; else oob = true; }
    bool s = oob;
    if (!oob) {
      s = mask[(size_t)xn + (size_t)nx * ((size_t)yn + (size_t)ny * (size_t)zn)] == 1;
      to_solid = to_solid || s;
    }
    if (s) L |= 1u << i;
  });
  links[nid] = L;
  const bool open = (x == 0 && open_lo) || (x == nx - 1 && open_hi);
  flags[nid] = solid ? FLAG_SOLID
                     : (uint8_t)(((L >> 1) ? FLAG_BOUNDARY : 0) | (to_solid ? FLAG_SOLID_LINK : 0) |
                                 (open ? FLAG_OPEN : 0));
}

}  // namespace

// Conservation sums in fp64: each block reduces with warp shuffles, writes
// its partials; a single block then adds the partials in a fixed order, so
// the result does not depend on scheduling.
constexpr int CONS_THREADS = 256;

__global__ void __launch_bounds__(CONS_THREADS)
    k_cons_partials(size_t n, const float* __restrict__ rho, const float* __restrict__ u,
                    double* __restrict__ partials, int nblk) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double r = rho[i];
    s[0] += r;
    s[1] += r * (double)u[i];
    s[2] += r * (double)u[n + i];
    s[3] += r * (double)u[2 * n + i];
  }
  __shared__ double sh[4][CONS_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double v = s[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int w = 0; w < CONS_THREADS / 32; ++w) v += sh[threadIdx.x][w];
    partials[(size_t)threadIdx.x * nblk + blockIdx.x] = v;
  }
}

__global__ void k_cons_final(const double* __restrict__ partials, int nblk, double* __restrict__ out) {
  const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= 4) return;
  double v = 0.0;
  for (int b = lane; b < nblk; b += 32) v += partials[(size_t)k * nblk + b];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) out[k] = v;
}

namespace {

__global__ void k_planes_to_fmt(const float* __restrict__ u, size_t n, int fmt, void* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float x = u[i], y = u[n + i], z = u[2 * n + i];
    if (fmt == LBM_U_F32X3) {
      float* o = reinterpret_cast<float*>(out) + 3 * i;
      o[0] = x; o[1] = y; o[2] = z;
    } else if (fmt == LBM_U_F32X4) {
      reinterpret_cast<float4*>(out)[i] = make_float4(x, y, z, 0.0f);
    } else {
      // rgba16f, as the velocity image stores it (round to nearest even).
      __half* o = reinterpret_cast<__half*>(out) + 4 * i;
      o[0] = __float2half_rn(x); o[1] = __float2half_rn(y);
      o[2] = __float2half_rn(z); o[3] = __float2half_rn(0.0f);
    }
  }
}

__global__ void k_fmt_to_planes(const void* __restrict__ in, size_t n, int fmt, float* __restrict__ u) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float x, y, z;
    if (fmt == LBM_U_F32X3) {
      const float* p = reinterpret_cast<const float*>(in) + 3 * i;
      x = p[0]; y = p[1]; z = p[2];
    } else if (fmt == LBM_U_F32X4) {
      const float4 v = reinterpret_cast<const float4*>(in)[i];
      x = v.x; y = v.y; z = v.z;
    } else {
      const __half* p = reinterpret_cast<const __half*>(in) + 4 * i;
      x = __half2float(p[0]); y = __half2float(p[1]); z = __half2float(p[2]);
    }
    u[i] = x; u[n + i] = y; u[2 * n + i] = z;
  }
}

int grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

}  // namespace

int cons_blocks(size_t n) { return grid_for(n, CONS_THREADS); }

cudaError_t classify(const Ctx& c, const int per[3], cudaStream_t s) {
  const dim3 b(32, 4, 2);
  const dim3 g((c.d.nx + 31) / 32, (c.d.ny + 3) / 4, (c.d.nz + 1) / 2);
  const bool phys = c.d.mode == LBM_MODE_PHYSICS;
  k_classify<<<g, b, 0, s>>>(c.d.nx, c.d.ny, c.d.nz, per[0], per[1], per[2],
                             phys && c.d.open_x[0] != LBM_OPEN_NONE, phys && c.d.open_x[1] != LBM_OPEN_NONE,
                             c.mask, c.flags, c.links);
  return cudaGetLastError();
}

cudaError_t conservation_partials(const Ctx& c, cudaStream_t s) {
  k_cons_partials<<<c.nblk_cons, CONS_THREADS, 0, s>>>(c.n, c.rho, c.u, c.partials, c.nblk_cons);
  k_cons_final<<<1, 128, 0, s>>>(c.partials, c.nblk_cons, c.sums);
  return cudaGetLastError();
}

cudaError_t u_planes_to_format(const float* u, size_t n, int fmt, void* out, cudaStream_t s) {
  k_planes_to_fmt<<<grid_for(n, 256), 256, 0, s>>>(u, n, fmt, out);
  return cudaGetLastError();
}

cudaError_t u_format_to_planes(const void* in, size_t n, int fmt, float* u, cudaStream_t s) {
  k_fmt_to_planes<<<grid_for(n, 256), 256, 0, s>>>(in, n, fmt, u);
  return cudaGetLastError();
}

}  // namespace lbm

// ---------------------------------------------------------------------------
// Conservation sums without any allocation.
//
// For callers that must not allocate device memory: a viewer's frame loop
// that cannot afford the device-wide synchronisation cudaMalloc/cudaFree
// imply, or a host application whose memory arena already owns the whole
// device budget.  The two reduction kernels above are reused unchanged; their
// block partials and the four sums live in a file-scope __device__ array that
// every GPU loading this library holds until the process exits.
//
// In host code `g_noalloc_scratch` names a host-side shadow, not device
// memory, so every call looks its device address up with
// cudaGetSymbolAddress (with the caller's device current; the lookup
// allocates nothing) and the kernels receive that address.  Looking it up on
// every call, rather than caching it, keeps the address right for whichever
// context is current, also after a cudaDeviceReset reloaded the module.
// ---------------------------------------------------------------------------
namespace lbm {
void set_thread_error(const char* msg);
}

namespace {
constexpr int kNoAllocMaxBlocks = 4096;                 // partial-sum slots per quantity
constexpr size_t kNoAllocNodesPerBlock = 8192;          // 256 threads x 32 nodes
constexpr size_t kNoAllocMaxNodes = kNoAllocMaxBlocks * kNoAllocNodesPerBlock;  // 33,554,432
// 4 x 4096 partials + 4 sums, fp64: 131,104 bytes per device.
static __device__ __align__(256) double g_noalloc_scratch[4 * kNoAllocMaxBlocks + 4];
}  // namespace

extern "C" LBM_API int lbm_conservation_noalloc(const float* d_rho, const float* d_u, size_t n,
                                                double out[4], void* stream) {
  if (!d_rho || !d_u || !out || n == 0) {
    lbm::set_thread_error("lbm_conservation_noalloc: d_rho, d_u and out must be non-NULL and n > 0");
    return LBM_ERR_INVALID_ARG;
  }
  if (n > kNoAllocMaxNodes) {
    lbm::set_thread_error("lbm_conservation_noalloc: n exceeds the 33554432-node limit of its static "
                          "scratch; use lbm_conservation");
    return LBM_ERR_INVALID_ARG;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    lbm::set_thread_error("lbm_conservation_noalloc: no current CUDA device");
    return LBM_ERR_NO_DEVICE;
  }
  void* p = nullptr;
  const cudaError_t ea = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (ea != cudaSuccess || !p) {
    cudaGetLastError();
    lbm::set_thread_error("lbm_conservation_noalloc: cudaGetSymbolAddress failed");
    return LBM_ERR_CUDA;
  }
  double* scratch = static_cast<double*>(p);
  // Every partial the final kernel reads is written first by its block, and
  // the sums are overwritten, so nothing needs clearing between calls.
  const int nblk = (int)((n + kNoAllocNodesPerBlock - 1) / kNoAllocNodesPerBlock);
  double* sums = scratch + 4 * kNoAllocMaxBlocks;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  lbm::k_cons_partials<<<nblk, lbm::CONS_THREADS, 0, s>>>(n, d_rho, d_u, scratch, nblk);
  lbm::k_cons_final<<<1, 128, 0, s>>>(scratch, nblk, sums);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, sums, 4 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    lbm::set_thread_error(cudaGetErrorString(e));
    return LBM_ERR_CUDA;
  }
  return LBM_OK;
}
