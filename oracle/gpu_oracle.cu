// FP64 copy of the oracle's ExtStep on the GPU, for full-size reference runs.
// TEST INFRASTRUCTURE ONLY: tests and the experiment runner use it as the
// checker; the product never loads it.  Two-buffer pull, one thread per node,
// the node update of ext_step.h compiled with -fmad=false so it equals the
// CPU oracle bit for bit.  All pointers are device pointers.
#include <cuda_runtime.h>

#include "ext_step.h"

namespace {

__global__ void k_init(ox::ExtP p, const uint8_t* mask, const double* rho, const double* u, double* f) {
  const size_t N = (size_t)p.nx * p.ny * p.nz;
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const bool solid = mask[n] == 1;
  for (int i = 0; i < 19; ++i)
    f[i * N + n] = solid ? 0.0 : ox::feq_i<double>(i, rho[n], u[n], u[N + n], u[2 * N + n]);
}

__global__ void k_step(ox::ExtP p, const uint8_t* mask, const double* fin, double* fout, double* rho,
                       double* u, int write_moments) {
  const size_t N = (size_t)p.nx * p.ny * p.nz;
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int x = (int)(n % p.nx), y = (int)((n / p.nx) % p.ny), z = (int)(n / ((size_t)p.nx * p.ny));
  if (mask[n] == 1) {
    for (int i = 0; i < 19; ++i) fout[i * N + n] = 0.0;
    if (write_moments) { rho[n] = 0.0; u[n] = u[N + n] = u[2 * N + n] = 0.0; }
    return;
  }
  double v[19];
  for (int i = 0; i < 19; ++i) v[i] = ox::incoming<double>(p, mask, fin, x, y, z, i, N);
  ox::open_face<double>(p, v, x);
  double r, ux, uy, uz;
  ox::ext_collide_node<double>(p, v, r, ux, uy, uz);
  for (int i = 0; i < 19; ++i) fout[i * N + n] = v[i];
  if (write_moments) { rho[n] = r; u[n] = ux; u[N + n] = uy; u[2 * N + n] = uz; }
}

}  // namespace

extern "C" {

int oracle_gpu_ext_init_f64(const int* ip, const double* dp, const uint8_t* mask, const double* rho,
                            const double* u, double* f) {
  const ox::ExtP p = ox::make_ext(ip, dp);
  const size_t N = (size_t)p.nx * p.ny * p.nz;
  k_init<<<(unsigned)((N + 255) / 256), 256>>>(p, mask, rho, u, f);
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : (int)e;
}

// nsteps steps; tmp is a second population buffer; the result is in f and
// the moments of the last step in rho/u.
int oracle_gpu_ext_step_f64(const int* ip, const double* dp, const uint8_t* mask, double* f,
                            double* tmp, int nsteps, double* rho, double* u) {
  const ox::ExtP p = ox::make_ext(ip, dp);
  const size_t N = (size_t)p.nx * p.ny * p.nz;
  double* a = f;
  double* b = tmp;
  for (int s = 0; s < nsteps; ++s) {
    k_step<<<(unsigned)((N + 255) / 256), 256>>>(p, mask, a, b, rho, u, s == nsteps - 1);
    double* t = a; a = b; b = t;
  }
  if (a != f) cudaMemcpy(f, a, 19 * N * sizeof(double), cudaMemcpyDeviceToDevice);
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"
