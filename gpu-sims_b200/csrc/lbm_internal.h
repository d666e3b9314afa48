// Internal declarations shared by the host runtime and the kernel files.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/lbm.h"
#include "../../include/lbm_closure.h"

namespace lbm {

// Layout of a learned-closure network (lbm_closure.h).
constexpr int CLO_IN = 9, CLO_HID = 32;
// Parameter offsets in the packed float layout (also the gradient layout).
constexpr int CLO_W1 = 0;                          // [32][9]
constexpr int CLO_B1 = CLO_W1 + CLO_HID * CLO_IN;  // [32]
constexpr int CLO_W2 = CLO_B1 + CLO_HID;           // [32][32]
constexpr int CLO_B2 = CLO_W2 + CLO_HID * CLO_HID; // [32]
constexpr int CLO_W3 = CLO_B2 + CLO_HID;           // [32]
constexpr int CLO_B3 = CLO_W3 + CLO_HID;           // [1]
constexpr int CLO_NPARAM = CLO_B3 + 1;             // 1409
// A network: parameters (weights holding bf16 values), then the input mean
// and inverse scale.
constexpr int CLO_MEAN = CLO_NPARAM;
constexpr int CLO_ISCALE = CLO_MEAN + CLO_IN;
constexpr int CLO_FLOATS = CLO_ISCALE + CLO_IN;    // 1427

constexpr bool clo_is_weight(int k) {
  return (k >= CLO_W1 && k < CLO_B1) || (k >= CLO_W2 && k < CLO_B2) || (k >= CLO_W3 && k < CLO_B3);
}

static_assert(CLO_NPARAM == LBM_CLOSURE_PARAMS && CLO_FLOATS == LBM_CLOSURE_FLOATS,
              "closure layout");

// Launch-time parameters of the reference-mode (two-buffer) kernels.
struct RefParams {
  int nx, ny, nz;
  size_t n;            // nx*ny*nz; stride between direction planes
  float tau_inv;       // 1.0f / tau          (src/main.cpp:1525)
  float omtau_inv;     // 1.0f - tau_inv      (src/main.cpp:1526)
  float u_inf[3];
  float rho0;
  int inlet_outlet;
  int free_slip;
  int u_round;         // enum lbm_u_round
};

// Geometry of the padded esoteric-pull population store (physics mode).
// Slot arrays: 0 = rest; pair p owns arrays 1+2p and 2+2p.  Node (x,y,z)
// lives at  x + px*((y+gy) + py*(z+gz));  non-periodic axes carry one ghost
// layer (x: only at x = nx, since every pair's forward vector has cx >= 0).
struct PhysGeom {
  int nx, ny, nz;
  int px, py, pz;      // padded extents
  int gy, gz;          // ghost offsets (0 or 1)
  uint32_t pxy;        // px * py
  int per[3];          // periodic flags
  size_t n;            // natural node count
  size_t slot_stride;  // elements per slot array
};

// default bound of the tensor-core closure's wait for its MMA (lbm_set_closure_wait_limit sets
// another): the kernel reports LBM_ERR_TIMEOUT past it
#ifndef LBM_CLO_WAIT_LIMIT
#define LBM_CLO_WAIT_LIMIT (1 << 22)
#endif

struct PhysParams {
  PhysGeom g;
  float omega;         // 1/tau
  // TRT antisymmetric rate 1 / (trt_magic / (1/omega - 1/2) + 1/2) for that
  // omega, evaluated once on the host with the step's own float operations
  // (steps with Smagorinsky compute it per node from their local omega)
  float omega_m;
  float tau;
  float trt_magic;
  float smag_cs;
  float accel[3];
  float wall[6][3];
  int any_moving_wall;  // bit f: face f (enum lbm_face) moves
  // open x faces (enum lbm_open; [0] = x-, [1] = x+): a VELOCITY face takes
  // its velocity from wall[0] / wall[1]
  int open[2];
  float open_rho[2];
  int any_open;
};

struct Ctx;

// Whether the physics step runs two nodes per thread for this row length
// (the rule lives with the step, phys_step.cuh).
bool step_pairs_host(int nx);

// reference-mode kernels (ref_kernels.cu)
// ref_init with write_moments = false leaves the moment fields alone (the
// recomputation of the first collision from them after a tau change).
cudaError_t ref_init(const Ctx& c, const float* rho, const float* u3, float rho0,
                     const float* u0, cudaStream_t s, bool write_moments = true);
cudaError_t ref_step(const Ctx& c, const float* fin, float* fout, bool write_moments,
                     cudaStream_t s);
// ref_step with explicit parameters (the boundaries of an earlier launch
// with a new collision tau).
cudaError_t ref_step_with(const Ctx& c, const RefParams& p, const float* fin, float* fout,
                          bool write_moments, cudaStream_t s);

// physics-mode kernels (phys_kernels.cu)
cudaError_t phys_init(const Ctx& c, const float* rho, const float* u3, float rho0,
                      const float* u0, cudaStream_t s);
cudaError_t phys_step(const Ctx& c, int parity, bool write_moments, cudaStream_t s);
cudaError_t phys_step_f32(const Ctx& c, int parity, bool write_moments, cudaStream_t s);
cudaError_t phys_step_f16(const Ctx& c, int parity, bool write_moments, cudaStream_t s);
cudaError_t phys_step_bf16(const Ctx& c, int parity, bool write_moments, cudaStream_t s);
cudaError_t phys_step_clo_f32(const Ctx& c, int parity, bool write_moments, cudaStream_t s);
cudaError_t phys_step_clo_f16(const Ctx& c, int parity, bool write_moments, cudaStream_t s);
cudaError_t phys_step_clo_bf16(const Ctx& c, int parity, bool write_moments, cudaStream_t s);
// Populations in natural layout [19][N]: f = g + w, or with `shifted` the
// stored g = f - w itself (lossless for every storage precision).
cudaError_t phys_read_pops(const Ctx& c, float* out, cudaStream_t s, bool shifted = false);
cudaError_t phys_write_pops(const Ctx& c, const float* in, cudaStream_t s, bool shifted = false);

// shared utilities (util_kernels.cu)
cudaError_t classify(const Ctx& c, const int per[3], cudaStream_t s);
int cons_blocks(size_t n);
cudaError_t conservation_partials(const Ctx& c, cudaStream_t s);
cudaError_t u_planes_to_format(const float* u, size_t n, int fmt, void* out, cudaStream_t s);
cudaError_t u_format_to_planes(const void* in, size_t n, int fmt, float* u, cudaStream_t s);

struct Ctx {
  lbm_desc d{};
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  size_t n = 0;
  // reference mode: two full population buffers, natural layout [19][n]
  float* fbuf[2] = {nullptr, nullptr};
  int cur = 0;
  RefParams rp{};
  // What lbm_set_params must recompute after a tau change: the stored
  // populations are the post-collision state of the next step, made by the
  // init kernel (REDO_INIT: its inputs are the moment fields) or by the last
  // step launch (REDO_STEP: its input is fbuf[cur ^ 1], its boundary
  // parameters rp_last); REDO_NONE after a population write or a new mask.
  enum { REDO_NONE = 0, REDO_INIT = 1, REDO_STEP = 2 };
  int redo = REDO_NONE;
  RefParams rp_last{};
  // physics mode: one esoteric-pull store
  void* pop = nullptr;
  int parity = 0;
  PhysParams pp{};
  // shared
  uint8_t* mask = nullptr;    // raw mask as uploaded
  uint8_t* flags = nullptr;   // classification byte
  uint32_t* links = nullptr;  // classification word
  float* rho = nullptr;       // [n]
  float* u = nullptr;         // [3][n]
  unsigned* status = nullptr; // device status word
  double* partials = nullptr; // conservation block partials [4][nblk]
  double* sums = nullptr;     // [4]
  int nblk_cons = 0;
  void* staging = nullptr;    // device staging for host format conversion
  size_t staging_bytes = 0;
  // CUDA graphs of kGraphSteps step launches (no moment write), one per
  // starting parity (reference mode: per current buffer), built on first use.
  static constexpr int kGraphSteps = 16;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  // learned closure (lbm_set_closure): the network the step kernels take by
  // value; weights already rounded to bf16
  bool closure = false;
  float clo[LBM_CLOSURE_FLOATS] = {};
  uint32_t clo_wait_polls = LBM_CLO_WAIT_LIMIT;  // polls per tensor-core MMA wait
  // nodes per thread of the physics step: 0 automatic, 1, 2 or 4
  int step_variant = 0;
  bool initialized = false;
  uint64_t iteration = 0;
  uint64_t dev_bytes = 0;
  std::string err;
};

size_t elem_bytes(int precision);
// bfloat16 rounding, nearest even (NaN kept), of one float: the weights of a
// closure network as the kernels use them.
float round_bf16(float v);
// Fills c.pp (padded geometry and physics parameters) from a physics-mode
// descriptor; false if a slot array would exceed 2^32 elements.
bool setup_physics(Ctx& c, const lbm_desc& d);
int validate_desc(const lbm_desc* d);
// NACA perimeter of lbm_voxelize_naca in lattice units (x0 y0 x1 y1 ...);
// false for a designation that is not four digits (host_tools.cpp).
bool naca_perimeter(const char* designation, int32_t nx, int32_t ny, float chord_frac, float center_x_frac,
                    float angle_of_attack_deg, std::vector<float>* xy);
// Device NACA mask into d_mask (voxel.cu); *bad_designation set instead of
// launching when the designation is invalid.
cudaError_t naca_mask_device(const char* designation, int32_t nx, int32_t ny, int32_t nz, float chord_frac,
                             float center_x_frac, float angle_of_attack_deg, uint8_t* d_mask,
                             cudaStream_t s, bool* bad_designation);  // LBM_OK or an LBM_ERR_* (message set)
void set_thread_error(const char* msg);
double bytes_per_node(const lbm_desc& d);

}  // namespace lbm

struct lbm_ctx : lbm::Ctx {};
