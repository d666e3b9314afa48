// Shared declarations of the batched step (phys_batch.cu, batch_api.cpp).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "lbm_internal.h"

namespace lbm {

// Whether batched domains may use the two-nodes-per-thread row update.  Off:
// with both row updates in one kernel the batch ran slower on B200 (fp16
// ensemble 20.3 vs 25.2 GLUPS), the domains being small.
#ifndef LBM_BATCH_PAIRS
#define LBM_BATCH_PAIRS 0
#endif

constexpr unsigned BATCH_STATUS_NONFINITE = 1u;  // same bit the single-domain step sets
constexpr unsigned BATCH_STATUS_TIMEOUT = 2u;    // a grid-barrier wait gave up

// One domain as the batched kernels see it (copied to shared memory per tile).
struct BatchDomain {
  PhysParams p;
  void* pop;
  const uint8_t* flags;
  const uint32_t* links;
  float* rho;
  float* u;
  int tiles_x, tiles_y;   // ceil(nx / (32 or 64)), ceil(ny / rows)
  uint32_t tile_begin;    // index of this domain's first tile
  uint32_t pairs;         // 1: two nodes per thread (tiles 64 wide)
};
static_assert(sizeof(BatchDomain) % 4 == 0, "copied as 32-bit words");

struct BatchLaunch {
  BatchDomain* dom;       // device array [ndom]
  const uint2* tiles;     // per tile: (domain, tile index within the domain)
  int ndom;
  uint32_t ntiles;
  int rows, nzt;          // block = 32 x rows threads; z-planes per thread
  int precision, collision;
  unsigned* status;
  unsigned* bar;          // [2] grid-barrier state
  long long spin_limit;   // cycles a barrier wait may take
  int missing_blocks;     // testing: blocks the barrier waits for in addition
};

cudaError_t batch_step(const BatchLaunch& L, int P, bool wm, cudaStream_t s);
cudaError_t batch_persistent_grid(const BatchLaunch& L, int* grid);
// One cooperative launch of nsteps steps from parity P0 (after a memset of
// the barrier state); write_last: its last step writes the moments.
cudaError_t batch_persistent(const BatchLaunch& L, int nsteps, int P0, int grid, cudaStream_t s,
                             bool write_last);

}  // namespace lbm
