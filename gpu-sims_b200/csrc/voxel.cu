// NACA obstacle mask on the device: the perimeter that lbm_voxelize_naca
// builds on the host (host_tools.cpp), then the winding-number test of every
// (x, y) column in a kernel, extruded in z.  Replaces naca::voxelize_into
// (src/main.cpp:254-312) for masks that go straight to the device.
//
// The perimeter travels as a __grid_constant__ kernel parameter (4 KB): every
// thread of a warp walks the same edge at the same time, so the reads are
// uniform constant-bank loads.  The edge test rounds after every operation
// (__fsub_rn / __fmul_rn are never contracted into FMAs), as the host
// voxeliser does, so both give the same mask bit for bit.
#include <vector>

#include "lbm_internal.h"

namespace lbm {
namespace {

constexpr int kMaxPerimeter = 512;

struct NacaPoly {
  int n;
  float x[kMaxPerimeter];
  float y[kMaxPerimeter];
};

__global__ void __launch_bounds__(256) k_naca_mask(const __grid_constant__ NacaPoly poly, int nx, int ny,
                                                   int nz, uint8_t* __restrict__ mask) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * 8 + threadIdx.y;
  if (x >= nx || y >= ny) return;
  const float px = float(x) + 0.5f, py = float(y) + 0.5f;
  int wn = 0;
  float ax = poly.x[0], ay = poly.y[0];
  for (int i = 0; i < poly.n; ++i) {
    const int j = i + 1 == poly.n ? 0 : i + 1;
    const float bx = poly.x[j], by = poly.y[j];
    // (b.x - a.x)(py - a.y) - (px - a.x)(b.y - a.y), each operation rounded
    const float side = __fsub_rn(__fmul_rn(__fsub_rn(bx, ax), __fsub_rn(py, ay)),
                                 __fmul_rn(__fsub_rn(px, ax), __fsub_rn(by, ay)));
    if (ay <= py) {
      if (by > py && side > 0.0f) ++wn;
    } else {
      if (by <= py && side < 0.0f) --wn;
    }
    ax = bx;
    ay = by;
  }
  const uint8_t v = wn != 0 ? 1 : 0;
  const size_t plane = (size_t)nx * (size_t)ny;
  uint8_t* m = mask + (size_t)x + (size_t)nx * (size_t)y;
  for (int z = 0; z < nz; ++z) m[(size_t)z * plane] = v;
}

}  // namespace

cudaError_t naca_mask_device(const char* designation, int32_t nx, int32_t ny, int32_t nz, float chord_frac,
                             float center_x_frac, float angle_of_attack_deg, uint8_t* d_mask,
                             cudaStream_t s, bool* bad_designation) {
  std::vector<float> xy;
  *bad_designation = false;
  if (!naca_perimeter(designation, nx, ny, chord_frac, center_x_frac, angle_of_attack_deg, &xy)) {
    *bad_designation = true;
    return cudaSuccess;
  }
  NacaPoly poly;
  poly.n = (int)(xy.size() / 2);
  if (poly.n > kMaxPerimeter) {
    *bad_designation = true;
    return cudaSuccess;
  }
  for (int i = 0; i < poly.n; ++i) {
    poly.x[i] = xy[2 * i];
    poly.y[i] = xy[2 * i + 1];
  }
  const dim3 blk(32, 8), grid((nx + 31) / 32, (ny + 7) / 8);
  k_naca_mask<<<grid, blk, 0, s>>>(poly, nx, ny, nz, d_mask);
  return cudaGetLastError();
}

}  // namespace lbm

extern "C" {

int lbm_voxelize_naca_device(const char* designation, int32_t nx, int32_t ny, int32_t nz, float chord_frac,
                             float center_x_frac, float angle_of_attack_deg, uint8_t* d_mask, size_t n,
                             void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !d_mask) {
    lbm::set_thread_error("voxelize_naca_device: sizes must be >= 1 and d_mask non-NULL");
    return LBM_ERR_INVALID_ARG;
  }
  if (n != (size_t)nx * (size_t)ny * (size_t)nz) {
    lbm::set_thread_error("voxelize_naca_device: n must be Nx*Ny*Nz");
    return LBM_ERR_INVALID_ARG;
  }
  if ((size_t)ny > 65535u * 8u) {
    lbm::set_thread_error("voxelize_naca_device: Ny above 524280");
    return LBM_ERR_UNSUPPORTED;
  }
  bool bad = false;
  const cudaError_t e = lbm::naca_mask_device(designation, nx, ny, nz, chord_frac, center_x_frac,
                                              angle_of_attack_deg, d_mask,
                                              reinterpret_cast<cudaStream_t>(stream), &bad);
  if (bad) {
    lbm::set_thread_error("voxelize_naca_device: designation must be four digits");
    return LBM_ERR_INVALID_ARG;
  }
  if (e != cudaSuccess) {
    lbm::set_thread_error(cudaGetErrorString(e));
    return LBM_ERR_CUDA;
  }
  return LBM_OK;
}

}  // extern "C"
