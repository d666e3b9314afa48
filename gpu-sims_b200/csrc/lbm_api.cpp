// Host runtime behind the C ABI (include/lbm.h): context lifetime, device
// memory, the step loop and the host<->device transfers.
//
// It replaces the parts of the reference sim host that drive the compute
// path: allocate_tier_images (src/main.cpp:835-846), obstacle_mask.upload
// (:1190), the init dispatch (:1193-1206), the substep chain (:1554-1591)
// and the moment readback (:1290-1296, :1771-1779).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "lbm_internal.h"

using lbm::Ctx;

namespace {

thread_local std::string g_thread_err = "no error";

int fail(Ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  g_thread_err = msg;
  return code;
}

int cuda_fail(Ctx* c, cudaError_t e, const char* what) {
  int code = LBM_ERR_CUDA;
  if (e == cudaErrorMemoryAllocation) code = LBM_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) code = LBM_ERR_NO_DEVICE;
  return fail(c, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(expr, what)                                  \
  do {                                                  \
    cudaError_t e_ = (expr);                            \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
  } while (0)

size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

int validate(const lbm_desc* d) {
  if (!d) return fail(nullptr, LBM_ERR_INVALID_ARG, "desc is NULL");
  if (d->struct_size != sizeof(lbm_desc))
    return fail(nullptr, LBM_ERR_INVALID_ARG, "desc.struct_size does not match this library's lbm_desc");
  // 65535: the largest grid y / z extent of a launch (rows and planes map to
  // blockIdx.y / blockIdx.z)
  const long long lim = 65535;
  if (d->nx < 2 || d->ny < 2 || d->nz < 2 || d->nx > lim || d->ny > lim || d->nz > lim)
    return fail(nullptr, LBM_ERR_INVALID_ARG, "grid extents must be in [2, 65535]");
  const double nodes = (double)d->nx * d->ny * d->nz;
  if (nodes > 4.0e9) return fail(nullptr, LBM_ERR_INVALID_ARG, "more than 4e9 nodes");
  if (d->mode != LBM_MODE_REFERENCE && d->mode != LBM_MODE_PHYSICS)
    return fail(nullptr, LBM_ERR_INVALID_ARG, "mode must be LBM_MODE_REFERENCE or LBM_MODE_PHYSICS");
  if (d->precision < LBM_PREC_F32 || d->precision > LBM_PREC_BF16S)
    return fail(nullptr, LBM_ERR_INVALID_ARG, "unknown precision");
  if (d->collision != LBM_COLL_BGK && d->collision != LBM_COLL_TRT)
    return fail(nullptr, LBM_ERR_INVALID_ARG, "unknown collision");
  if (!(d->tau > 0.5f) || !std::isfinite(d->tau))
    return fail(nullptr, LBM_ERR_INVALID_ARG, "tau must be finite and > 0.5");
  if (d->ref_u_round < LBM_UROUND_NONE || d->ref_u_round > LBM_UROUND_RTZ)
    return fail(nullptr, LBM_ERR_INVALID_ARG, "unknown ref_u_round");
  for (int a = 0; a < 3; ++a)
    if (d->periodic[a] != 0 && d->periodic[a] != 1)
      return fail(nullptr, LBM_ERR_INVALID_ARG, "periodic flags must be 0 or 1");
  if (d->mode == LBM_MODE_REFERENCE) {
    if (d->precision != LBM_PREC_F32)
      return fail(nullptr, LBM_ERR_UNSUPPORTED, "reference mode stores fp32 populations only");
    if (d->collision != LBM_COLL_BGK || d->smagorinsky_cs != 0.f)
      return fail(nullptr, LBM_ERR_UNSUPPORTED, "reference mode is BGK without Smagorinsky");
    if (d->periodic[0] || d->periodic[1] || d->periodic[2])
      return fail(nullptr, LBM_ERR_UNSUPPORTED, "reference mode has no periodic axes");
  } else {
    if (!(d->smagorinsky_cs >= 0.f) || !(d->trt_magic > 0.f))
      return fail(nullptr, LBM_ERR_INVALID_ARG, "smagorinsky_cs must be >= 0 and trt_magic > 0");
  }
  for (int s = 0; s < 2; ++s) {
    if (d->open_x[s] < LBM_OPEN_NONE || d->open_x[s] > LBM_OPEN_PRESSURE)
      return fail(nullptr, LBM_ERR_INVALID_ARG, "open_x must be LBM_OPEN_NONE, _VELOCITY or _PRESSURE");
    if (d->open_x[s] == LBM_OPEN_NONE) continue;
    if (d->mode != LBM_MODE_PHYSICS || d->periodic[0])
      return fail(nullptr, LBM_ERR_UNSUPPORTED, "open x faces need physics mode and a non-periodic x axis");
    if (d->open_x[s] == LBM_OPEN_PRESSURE && !(d->open_rho[s] > 0.f && std::isfinite(d->open_rho[s])))
      return fail(nullptr, LBM_ERR_INVALID_ARG, "open_rho of a pressure face must be finite and > 0");
    const float* u = d->wall_velocity[s];
    if (d->open_x[s] == LBM_OPEN_VELOCITY &&
        !(std::fabs(u[0]) < 0.5f && std::isfinite(u[1]) && std::isfinite(u[2])))
      return fail(nullptr, LBM_ERR_INVALID_ARG, "velocity of an open face must be finite with |u_x| < 0.5");
  }
  return LBM_OK;
}

template <class T>
int dev_alloc(Ctx* c, T** p, size_t count, const char* what) {
  const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
  void* v = nullptr;
  cudaError_t e = cudaMalloc(&v, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return cuda_fail(c, e, what);
  }
  *p = static_cast<T*>(v);
  c->dev_bytes += bytes;
  return LBM_OK;
}

int ensure_staging(Ctx* c, size_t bytes) {
  if (c->staging_bytes >= bytes) return LBM_OK;
  if (c->staging) {
    cudaFree(c->staging);
    c->dev_bytes -= c->staging_bytes;
    c->staging = nullptr;
    c->staging_bytes = 0;
  }
  void* p = nullptr;
  int rc = dev_alloc(c, reinterpret_cast<char**>(&p), bytes, "cudaMalloc(staging)");
  if (rc) return rc;
  c->staging = p;
  c->staging_bytes = bytes;
  return LBM_OK;
}

void free_all(Ctx* c) {
  for (auto& g : c->graph)
    if (g) cudaGraphExecDestroy(g);
  void* ptrs[] = {c->fbuf[0], c->fbuf[1], c->pop,      c->mask,     c->flags, c->links,
                  c->rho,     c->u,       c->status,   c->partials, c->sums,  c->staging};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
}

int check_ctx(Ctx* c) {
  if (!c) return fail(nullptr, LBM_ERR_INVALID_ARG, "ctx is NULL");
  return LBM_OK;
}

size_t u_bytes(int fmt) {
  return fmt == LBM_U_F32X3 ? 12 : fmt == LBM_U_F32X4 ? 16 : fmt == LBM_U_F16X4 ? 8 : 0;
}

}  // namespace

namespace lbm {

void set_thread_error(const char* msg) { g_thread_err = msg; }

bool setup_physics(Ctx& c, const lbm_desc& d) {
  auto& g = c.pp.g;
  g.nx = d.nx; g.ny = d.ny; g.nz = d.nz;
  g.n = (size_t)d.nx * d.ny * d.nz;
  for (int a = 0; a < 3; ++a) g.per[a] = d.periodic[a];
  g.px = g.per[0] ? g.nx : (int)round_up((size_t)g.nx + 1, 8);
  g.gy = g.per[1] ? 0 : 1;
  g.gz = g.per[2] ? 0 : 1;
  g.py = g.ny + 2 * g.gy;
  g.pz = g.nz + 2 * g.gz;
  g.pxy = (uint32_t)((size_t)g.px * g.py);
  g.slot_stride = round_up((size_t)g.px * g.py * g.pz, 64);
  if (g.slot_stride >= (size_t(1) << 32)) return false;
  auto& p = c.pp;
  p.tau = d.tau;
  p.omega = 1.0f / d.tau;
  p.trt_magic = d.trt_magic;
  p.omega_m = 1.0f / (p.trt_magic / (1.0f / p.omega - 0.5f) + 0.5f);
  p.smag_cs = d.smagorinsky_cs;
  for (int a = 0; a < 3; ++a) p.accel[a] = d.body_accel[a];
  p.any_moving_wall = 0;
  for (int f = 0; f < 6; ++f)
    for (int a = 0; a < 3; ++a) {
      p.wall[f][a] = d.wall_velocity[f][a];
      // an open face's velocity is the inlet's (the face kernel rebuilds
      // every link across it), not a moving wall's
      const bool open = f < 2 && d.open_x[f] != LBM_OPEN_NONE;
      if (d.wall_velocity[f][a] != 0.f && !open) p.any_moving_wall |= 1 << f;
    }
  p.any_open = 0;
  for (int s = 0; s < 2; ++s) {
    p.open[s] = d.open_x[s];
    p.open_rho[s] = d.open_rho[s];
    if (d.open_x[s] != LBM_OPEN_NONE) p.any_open = 1;
  }
  return true;
}

int validate_desc(const lbm_desc* d) { return validate(d); }

size_t elem_bytes(int precision) { return precision == LBM_PREC_F32 ? 4 : 2; }

double bytes_per_node(const lbm_desc& d) {
  // 19 population loads + 19 stores + 1 flag byte per node update.
  return 38.0 * (double)elem_bytes(d.precision) + 1.0;
}

}  // namespace lbm

extern "C" {

static void drop_graphs(lbm_ctx* c);
static int prepare_graphs(lbm_ctx* c);

int lbm_desc_default(lbm_desc* d) {
  if (!d) return fail(nullptr, LBM_ERR_INVALID_ARG, "desc is NULL");
  std::memset(d, 0, sizeof(*d));
  d->struct_size = sizeof(lbm_desc);
  d->nx = d->ny = d->nz = 64;
  d->mode = LBM_MODE_REFERENCE;
  d->precision = LBM_PREC_F32;
  d->collision = LBM_COLL_BGK;
  d->tau = 0.6f;          // TAU_DEFAULT (src/main.cpp:84)
  d->trt_magic = 3.0f / 16.0f;
  d->rho0 = 1.0f;         // RHO_0 (src/main.cpp:86)
  d->ref_inlet_outlet = 1;
  d->ref_free_slip = 1;
  d->ref_u_round = LBM_UROUND_RTE;
  return LBM_OK;
}

int lbm_create(const lbm_desc* desc, lbm_ctx** out) {
  if (!out) return fail(nullptr, LBM_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  int rc = validate(desc);
  if (rc) return rc;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(nullptr, LBM_ERR_NO_DEVICE,
                std::string("no CUDA device: ") + (e == cudaSuccess ? "count is 0" : cudaGetErrorString(e)));
  }
  lbm_ctx* c = new (std::nothrow) lbm_ctx();
  if (!c) return fail(nullptr, LBM_ERR_OUT_OF_MEMORY, "host allocation failed");
  c->d = *desc;
  cudaGetDevice(&c->device);
  const size_t n = (size_t)desc->nx * desc->ny * desc->nz;
  c->n = n;
  auto bail = [&](int code) {
    g_thread_err = c->err;
    free_all(c);
    delete c;
    return code;
  };
  if ((e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(cuda_fail(c, e, "cudaStreamCreate"));
  c->stream = c->own_stream;

  if (desc->mode == LBM_MODE_REFERENCE) {
    for (int k = 0; k < 2; ++k)
      if ((rc = dev_alloc(c, &c->fbuf[k], 19 * n, "cudaMalloc(populations)"))) return bail(rc);
    auto& p = c->rp;
    p.nx = desc->nx; p.ny = desc->ny; p.nz = desc->nz; p.n = n;
    // CollideUniforms as the host fills them (src/main.cpp:1524-1526).
    p.tau_inv = 1.0f / desc->tau;
    p.omtau_inv = 1.0f - p.tau_inv;
    for (int a = 0; a < 3; ++a) p.u_inf[a] = desc->u_inf[a];
    p.rho0 = desc->rho0;
    p.inlet_outlet = desc->ref_inlet_outlet;
    p.free_slip = desc->ref_free_slip;
    p.u_round = desc->ref_u_round;
  } else {
    if (!lbm::setup_physics(*c, *desc))
      return bail(fail(c, LBM_ERR_UNSUPPORTED, "padded grid exceeds 2^32 nodes per slot array"));
    const size_t eb = lbm::elem_bytes(desc->precision);
    if ((rc = dev_alloc(c, reinterpret_cast<char**>(&c->pop), 19 * c->pp.g.slot_stride * eb,
                        "cudaMalloc(populations)")))
      return bail(rc);
  }
  c->nblk_cons = lbm::cons_blocks(n);
  if ((rc = dev_alloc(c, &c->mask, n, "cudaMalloc(mask)")) ||
      (rc = dev_alloc(c, &c->flags, n, "cudaMalloc(flags)")) ||
      (rc = dev_alloc(c, &c->links, n, "cudaMalloc(links)")) ||
      (rc = dev_alloc(c, &c->rho, n, "cudaMalloc(rho)")) ||
      (rc = dev_alloc(c, &c->u, 3 * n, "cudaMalloc(u)")) ||
      (rc = dev_alloc(c, &c->status, 4, "cudaMalloc(status)")) ||
      (rc = dev_alloc(c, &c->partials, 4 * (size_t)c->nblk_cons, "cudaMalloc(partials)")) ||
      (rc = dev_alloc(c, &c->sums, 4, "cudaMalloc(sums)")))
    return bail(rc);

  cudaStream_t s = c->stream;
  if (c->fbuf[0]) {
    cudaMemsetAsync(c->fbuf[0], 0, 19 * n * sizeof(float), s);
    cudaMemsetAsync(c->fbuf[1], 0, 19 * n * sizeof(float), s);
  }
  if (c->pop) cudaMemsetAsync(c->pop, 0, 19 * c->pp.g.slot_stride * lbm::elem_bytes(desc->precision), s);
  cudaMemsetAsync(c->mask, 0, n, s);
  cudaMemsetAsync(c->rho, 0, n * sizeof(float), s);
  cudaMemsetAsync(c->u, 0, 3 * n * sizeof(float), s);
  cudaMemsetAsync(c->status, 0, 4 * sizeof(unsigned), s);
  const int per[3] = {desc->mode == LBM_MODE_PHYSICS ? desc->periodic[0] : 0,
                      desc->mode == LBM_MODE_PHYSICS ? desc->periodic[1] : 0,
                      desc->mode == LBM_MODE_PHYSICS ? desc->periodic[2] : 0};
  if ((e = lbm::classify(*c, per, s)) != cudaSuccess) return bail(cuda_fail(c, e, "classify"));
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return bail(cuda_fail(c, e, "create sync"));
  *out = c;
  return LBM_OK;
}

int lbm_destroy(lbm_ctx* c) {
  if (!c) return LBM_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_all(c);
  delete c;
  return LBM_OK;
}

int lbm_set_stream(lbm_ctx* c, void* stream) {
  if (int rc = check_ctx(c)) return rc;
  // Work already queued on the old stream must finish before the new one
  // touches the same buffers.
  CK(cudaStreamSynchronize(c->stream), "set_stream sync");
  c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
  return LBM_OK;
}

int lbm_set_step_variant(lbm_ctx* c, int nodes_per_thread) {
  if (int rc = check_ctx(c)) return rc;
  const int v = nodes_per_thread;
  if (v != 0 && v != 1 && v != 2 && v != 4 && v != 8)
    return fail(c, LBM_ERR_INVALID_ARG, "variant: 0, 1, 2, 4 or 8");
  if (c->d.mode != LBM_MODE_PHYSICS && v != 0)
    return fail(c, LBM_ERR_UNSUPPORTED, "step variants are physics-mode kernels");
  if (v == 2 && c->d.nx % 2) return fail(c, LBM_ERR_UNSUPPORTED, "two nodes per thread need an even nx");
  if (v == 4 && c->d.nx % 4) return fail(c, LBM_ERR_UNSUPPORTED, "four nodes per thread need nx % 4 == 0");
  if ((v == 4 || v == 8) && c->pp.any_open)
    return fail(c, LBM_ERR_UNSUPPORTED, "open x faces run with one or two nodes per thread");
  CK(cudaStreamSynchronize(c->stream), "set_step_variant sync");
  drop_graphs(c);
  c->step_variant = v;
  return c->initialized ? prepare_graphs(c) : LBM_OK;
}

int lbm_set_closure(lbm_ctx* c, const float* net) {
  if (int rc = check_ctx(c)) return rc;
  if (c->d.mode != LBM_MODE_PHYSICS) return fail(c, LBM_ERR_UNSUPPORTED, "the closure needs physics mode");
  if (net) {
    if (!(c->d.smagorinsky_cs > 0.f))
      return fail(c, LBM_ERR_INVALID_ARG, "the closure scales smagorinsky_cs, which must be > 0");
    if (c->pp.accel[0] != 0.f || c->pp.accel[1] != 0.f || c->pp.accel[2] != 0.f)
      return fail(c, LBM_ERR_UNSUPPORTED, "the closure kernels are built without a body force");
    for (int k = 0; k < LBM_CLOSURE_FLOATS; ++k)
      if (!std::isfinite(net[k])) return fail(c, LBM_ERR_INVALID_ARG, "closure network has a non-finite value");
  }
  // Captured step graphs hold the old network by value: rebuild them.
  CK(cudaStreamSynchronize(c->stream), "set_closure sync");
  drop_graphs(c);
  c->closure = net != nullptr;
  for (int k = 0; k < LBM_CLOSURE_FLOATS; ++k) {
    c->clo[k] = !net ? 0.f : lbm::clo_is_weight(k) ? lbm::round_bf16(net[k]) : net[k];
  }
  return c->initialized ? prepare_graphs(c) : LBM_OK;
}

int lbm_set_closure_wait_limit(lbm_ctx* c, int32_t polls) {
  if (int rc = check_ctx(c)) return rc;
  // the bound is a launch argument of the captured step graphs: rebuild them
  CK(cudaStreamSynchronize(c->stream), "set_closure_wait_limit sync");
  drop_graphs(c);
  c->clo_wait_polls = polls < 0 ? (uint32_t)LBM_CLO_WAIT_LIMIT : (uint32_t)polls;
  return c->initialized ? prepare_graphs(c) : LBM_OK;
}

// Classifies the mask already in c->mask (lbm_set_flags, lbm_set_flags_naca).
static int classify_mask(lbm_ctx* c) {
  const int per[3] = {c->d.mode == LBM_MODE_PHYSICS ? c->d.periodic[0] : 0,
                      c->d.mode == LBM_MODE_PHYSICS ? c->d.periodic[1] : 0,
                      c->d.mode == LBM_MODE_PHYSICS ? c->d.periodic[2] : 0};
  CK(lbm::classify(*c, per, c->stream), "classify");
  CK(cudaStreamSynchronize(c->stream), "set_flags sync");
  // Physics mode keeps no populations at solid nodes, so a new mask needs a
  // new init; the reference step zeroes solids itself and can continue.
  if (c->d.mode == LBM_MODE_PHYSICS) c->initialized = false;
  // the last step's boundaries used the old mask: it cannot be rerun
  if (c->redo == Ctx::REDO_STEP) c->redo = Ctx::REDO_NONE;
  return LBM_OK;
}

int lbm_set_flags(lbm_ctx* c, const uint8_t* mask, size_t n) {
  if (int rc = check_ctx(c)) return rc;
  if (!mask) return fail(c, LBM_ERR_INVALID_ARG, "mask is NULL");
  if (n != c->n) return fail(c, LBM_ERR_INVALID_ARG, "mask length must be Nx*Ny*Nz");
  CK(cudaMemcpyAsync(c->mask, mask, n, cudaMemcpyHostToDevice, c->stream), "upload mask");
  return classify_mask(c);
}

int lbm_set_flags_naca(lbm_ctx* c, const char* designation, float chord_frac, float center_x_frac,
                       float angle_of_attack_deg) {
  if (int rc = check_ctx(c)) return rc;
  if (c->d.ny > 65535 * 8) return fail(c, LBM_ERR_UNSUPPORTED, "Ny above 524280");
  bool bad = false;
  const cudaError_t e = lbm::naca_mask_device(designation, c->d.nx, c->d.ny, c->d.nz, chord_frac,
                                              center_x_frac, angle_of_attack_deg, c->mask, c->stream, &bad);
  if (bad) return fail(c, LBM_ERR_INVALID_ARG, "designation must be four digits");
  if (e != cudaSuccess) return cuda_fail(c, e, "voxelise");
  return classify_mask(c);
}

int lbm_read_classification(lbm_ctx* c, uint32_t* out, size_t n) {
  if (int rc = check_ctx(c)) return rc;
  if (!out || n != c->n) return fail(c, LBM_ERR_INVALID_ARG, "out must hold Nx*Ny*Nz words");
  CK(cudaMemcpyAsync(out, c->links, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream),
     "read classification");
  CK(cudaStreamSynchronize(c->stream), "read classification sync");
  return LBM_OK;
}

// One step launch on stream s; flips the parity / current buffer.
static cudaError_t launch_one(lbm_ctx* c, bool wm, cudaStream_t s) {
  cudaError_t e;
  if (c->d.mode == LBM_MODE_REFERENCE) {
    e = lbm::ref_step(*c, c->fbuf[c->cur], c->fbuf[c->cur ^ 1], wm, s);
    c->cur ^= 1;
  } else {
    e = lbm::phys_step(*c, c->parity, wm, s);
    c->parity ^= 1;
  }
  return e;
}

// Captures kGraphSteps plain step launches, starting from the current parity,
// on the context's own stream (a capture needs a non-legacy stream).  An even
// count leaves the parity as it found it.
static int build_graph(lbm_ctx* c, int slot) {
  // capture from the slot's parity (current buffer); the captured launches do
  // not run, and an even count brings the parity back, restored below anyway
  int& par = c->d.mode == LBM_MODE_REFERENCE ? c->cur : c->parity;
  const int saved = par;
  par = slot;
  struct Restore {
    int& p;
    int v;
    ~Restore() { p = v; }
  } restore{par, saved};
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(c->own_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < Ctx::kGraphSteps && e == cudaSuccess; ++i) e = launch_one(c, false, c->own_stream);
  cudaError_t e2 = cudaStreamEndCapture(c->own_stream, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cuda_fail(c, e != cudaSuccess ? e : e2, "capture step graph");
  }
  e = cudaGraphInstantiate(&c->graph[slot], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(c, e, "instantiate step graph");
  // upload now, so that its first launch does not pay for it inside a
  // caller's step loop
  CK(cudaGraphUpload(c->graph[slot], c->stream), "upload step graph");
  return LBM_OK;
}

static void drop_graphs(lbm_ctx* c) {
  for (auto& g : c->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

// Builds the step graphs of both starting parities that do not exist yet, so
// that no capture or instantiation falls inside a caller's step loop.
static int prepare_graphs(lbm_ctx* c) {
  for (int slot = 0; slot < 2; ++slot)
    if (!c->graph[slot])
      if (int rc = build_graph(c, slot)) return rc;
  return LBM_OK;
}

static int do_init(lbm_ctx* c, const float* d_rho, const float* d_u, float rho0, const float* u0) {
  cudaError_t e;
  if (c->d.mode == LBM_MODE_REFERENCE) {
    c->cur = 0;
    e = lbm::ref_init(*c, d_rho, d_u, rho0, u0, c->stream);
  } else {
    c->parity = 0;
    e = lbm::phys_init(*c, d_rho, d_u, rho0, u0, c->stream);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "init kernel");
  CK(cudaMemsetAsync(c->status, 0, sizeof(unsigned), c->stream), "reset status");
  c->iteration = 0;
  c->initialized = true;
  c->redo = Ctx::REDO_INIT;
  return prepare_graphs(c);
}

int lbm_init_equilibrium(lbm_ctx* c, float rho0, const float u0[3]) {
  if (int rc = check_ctx(c)) return rc;
  if (!u0) return fail(c, LBM_ERR_INVALID_ARG, "u0 is NULL");
  if (!std::isfinite(rho0) || !(rho0 >= 0.f))
    return fail(c, LBM_ERR_INVALID_ARG, "rho0 must be finite and >= 0");
  return do_init(c, nullptr, nullptr, rho0, u0);
}

int lbm_init_from_moments(lbm_ctx* c, const float* rho, const void* u, int u_fmt) {
  if (int rc = check_ctx(c)) return rc;
  if (!rho || !u) return fail(c, LBM_ERR_INVALID_ARG, "rho and u must not be NULL");
  const size_t ub = u_bytes(u_fmt);
  if (!ub) return fail(c, LBM_ERR_INVALID_ARG, "unknown u format");
  const size_t n = c->n;
  if (int rc = ensure_staging(c, n * (4 + 12 + ub))) return rc;
  float* d_rho = static_cast<float*>(c->staging);
  float* d_u = d_rho + n;
  void* d_raw = d_u + 3 * n;
  CK(cudaMemcpyAsync(d_rho, rho, n * sizeof(float), cudaMemcpyHostToDevice, c->stream), "upload rho");
  CK(cudaMemcpyAsync(d_raw, u, n * ub, cudaMemcpyHostToDevice, c->stream), "upload u");
  CK(lbm::u_format_to_planes(d_raw, n, u_fmt, d_u, c->stream), "convert u");
  const float zero[3] = {0.f, 0.f, 0.f};
  int rc = do_init(c, d_rho, d_u, 1.0f, zero);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream), "init sync");
  return LBM_OK;
}

int lbm_step(lbm_ctx* c, int nsteps) {
  if (int rc = check_ctx(c)) return rc;
  if (nsteps < 0) return fail(c, LBM_ERR_INVALID_ARG, "nsteps must be >= 0");
  if (!c->initialized) return fail(c, LBM_ERR_STATE, "lbm_step before lbm_init_*");
  int left = nsteps;
  // Whole graphs while more than kGraphSteps steps remain (the last launch
  // of the call must write the moments, so it is never inside a graph).
  if (left > Ctx::kGraphSteps)
    if (int rc = prepare_graphs(c)) return rc;
  while (left > Ctx::kGraphSteps) {
    const int slot = c->d.mode == LBM_MODE_REFERENCE ? c->cur : c->parity;
    CK(cudaGraphLaunch(c->graph[slot], c->stream), "graph launch");
    left -= Ctx::kGraphSteps;
  }
  for (int i = 0; i < left; ++i) {
    cudaError_t e = launch_one(c, i == left - 1, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "step kernel launch");
  }
  if (nsteps > 0) {
    c->redo = Ctx::REDO_STEP;
    c->rp_last = c->rp;
  }
  c->iteration += (uint64_t)nsteps;
  return LBM_OK;
}

int lbm_sync(lbm_ctx* c) {
  if (int rc = check_ctx(c)) return rc;
  unsigned st = 0;
  CK(cudaMemcpyAsync(&st, c->status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream), "read status");
  CK(cudaStreamSynchronize(c->stream), "sync");
  if (st) {
    CK(cudaMemsetAsync(c->status, 0, sizeof(unsigned), c->stream), "reset status");
    if (st & 2u)
      return fail(c, LBM_ERR_TIMEOUT, "the closure's tensor-core MMA wait gave up (nodes fell back to Smagorinsky)");
    return fail(c, LBM_ERR_NONFINITE, "non-finite value or rho <= 0 at a fluid node");
  }
  return LBM_OK;
}

int lbm_read_moments(lbm_ctx* c, float* rho, void* u, int u_fmt) {
  if (int rc = check_ctx(c)) return rc;
  if (!c->initialized) return fail(c, LBM_ERR_STATE, "read_moments before lbm_init_*");
  const size_t n = c->n;
  if (rho)
    CK(cudaMemcpyAsync(rho, c->rho, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "read rho");
  if (u) {
    const size_t ub = u_bytes(u_fmt);
    if (!ub) return fail(c, LBM_ERR_INVALID_ARG, "unknown u format");
    if (int rc = ensure_staging(c, n * ub)) return rc;
    CK(lbm::u_planes_to_format(c->u, n, u_fmt, c->staging, c->stream), "convert u");
    CK(cudaMemcpyAsync(u, c->staging, n * ub, cudaMemcpyDeviceToHost, c->stream), "read u");
  }
  CK(cudaStreamSynchronize(c->stream), "read_moments sync");
  return LBM_OK;
}

int lbm_device_moments(lbm_ctx* c, const float** d_rho, const float** d_u) {
  if (int rc = check_ctx(c)) return rc;
  if (d_rho) *d_rho = c->rho;
  if (d_u) *d_u = c->u;
  return LBM_OK;
}

int lbm_conservation(lbm_ctx* c, double out[4]) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return fail(c, LBM_ERR_INVALID_ARG, "out is NULL");
  if (!c->initialized) return fail(c, LBM_ERR_STATE, "conservation before lbm_init_*");
  CK(lbm::conservation_partials(*c, c->stream), "conservation kernels");
  CK(cudaMemcpyAsync(out, c->sums, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "read sums");
  CK(cudaStreamSynchronize(c->stream), "conservation sync");
  return LBM_OK;
}

int lbm_conservation_async(lbm_ctx* c, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return fail(c, LBM_ERR_INVALID_ARG, "out is NULL");
  if (!c->initialized) return fail(c, LBM_ERR_STATE, "conservation before lbm_init_*");
  CK(lbm::conservation_partials(*c, c->stream), "conservation kernels");
  CK(cudaMemcpyAsync(out, c->sums, 4 * sizeof(double), cudaMemcpyDefault, c->stream), "copy sums");
  return LBM_OK;
}

int lbm_read_populations(lbm_ctx* c, float* f, size_t n) {
  if (int rc = check_ctx(c)) return rc;
  if (!f || n != 19 * c->n) return fail(c, LBM_ERR_INVALID_ARG, "f must hold 19*Nx*Ny*Nz floats");
  if (!c->initialized) return fail(c, LBM_ERR_STATE, "read_populations before lbm_init_*");
  if (c->d.mode == LBM_MODE_REFERENCE) {
    CK(cudaMemcpyAsync(f, c->fbuf[c->cur], n * sizeof(float), cudaMemcpyDeviceToHost, c->stream),
       "read populations");
  } else {
    if (int rc = ensure_staging(c, n * sizeof(float))) return rc;
    CK(lbm::phys_read_pops(*c, static_cast<float*>(c->staging), c->stream), "gather populations");
    CK(cudaMemcpyAsync(f, c->staging, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream),
       "read populations");
  }
  CK(cudaStreamSynchronize(c->stream), "read_populations sync");
  return LBM_OK;
}

int lbm_write_populations(lbm_ctx* c, const float* f, size_t n) {
  if (int rc = check_ctx(c)) return rc;
  if (!f || n != 19 * c->n) return fail(c, LBM_ERR_INVALID_ARG, "f must hold 19*Nx*Ny*Nz floats");
  if (c->d.mode == LBM_MODE_REFERENCE) {
    CK(cudaMemcpyAsync(c->fbuf[c->cur], f, n * sizeof(float), cudaMemcpyHostToDevice, c->stream),
       "write populations");
  } else {
    if (int rc = ensure_staging(c, n * sizeof(float))) return rc;
    CK(cudaMemcpyAsync(c->staging, f, n * sizeof(float), cudaMemcpyHostToDevice, c->stream),
       "write populations");
    CK(lbm::phys_write_pops(*c, static_cast<const float*>(c->staging), c->stream), "scatter populations");
  }
  CK(cudaStreamSynchronize(c->stream), "write_populations sync");
  c->initialized = true;
  c->redo = Ctx::REDO_NONE;
  return prepare_graphs(c);
}

int lbm_read_populations_shifted(lbm_ctx* c, float* g, size_t n) {
  if (int rc = check_ctx(c)) return rc;
  if (!g || n != 19 * c->n) return fail(c, LBM_ERR_INVALID_ARG, "g must hold 19*Nx*Ny*Nz floats");
  if (c->d.mode != LBM_MODE_PHYSICS) return fail(c, LBM_ERR_UNSUPPORTED, "shifted populations need physics mode");
  if (!c->initialized) return fail(c, LBM_ERR_STATE, "read_populations_shifted before lbm_init_*");
  if (int rc = ensure_staging(c, n * sizeof(float))) return rc;
  CK(lbm::phys_read_pops(*c, static_cast<float*>(c->staging), c->stream, true), "gather populations");
  CK(cudaMemcpyAsync(g, c->staging, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "read populations");
  CK(cudaStreamSynchronize(c->stream), "read_populations_shifted sync");
  return LBM_OK;
}

int lbm_write_populations_shifted(lbm_ctx* c, const float* g, size_t n) {
  if (int rc = check_ctx(c)) return rc;
  if (!g || n != 19 * c->n) return fail(c, LBM_ERR_INVALID_ARG, "g must hold 19*Nx*Ny*Nz floats");
  if (c->d.mode != LBM_MODE_PHYSICS) return fail(c, LBM_ERR_UNSUPPORTED, "shifted populations need physics mode");
  if (int rc = ensure_staging(c, n * sizeof(float))) return rc;
  CK(cudaMemcpyAsync(c->staging, g, n * sizeof(float), cudaMemcpyHostToDevice, c->stream), "write populations");
  CK(lbm::phys_write_pops(*c, static_cast<const float*>(c->staging), c->stream, true), "scatter populations");
  CK(cudaStreamSynchronize(c->stream), "write_populations_shifted sync");
  c->initialized = true;
  c->redo = Ctx::REDO_NONE;
  return prepare_graphs(c);
}

int lbm_read_mask(lbm_ctx* c, uint8_t* mask, size_t n) {
  if (int rc = check_ctx(c)) return rc;
  if (!mask || n != c->n) return fail(c, LBM_ERR_INVALID_ARG, "mask must hold Nx*Ny*Nz bytes");
  CK(cudaMemcpyAsync(mask, c->mask, n, cudaMemcpyDeviceToHost, c->stream), "read mask");
  CK(cudaStreamSynchronize(c->stream), "read_mask sync");
  return LBM_OK;
}

int lbm_get_desc(lbm_ctx* c, lbm_desc* desc) {
  if (int rc = check_ctx(c)) return rc;
  if (!desc || desc->struct_size != sizeof(lbm_desc))
    return fail(c, LBM_ERR_INVALID_ARG, "desc is NULL or desc.struct_size is wrong");
  *desc = c->d;
  return LBM_OK;
}

int lbm_set_iteration(lbm_ctx* c, uint64_t iteration) {
  if (int rc = check_ctx(c)) return rc;
  c->iteration = iteration;
  return LBM_OK;
}

int lbm_get_info(lbm_ctx* c, lbm_info* info) {
  if (int rc = check_ctx(c)) return rc;
  if (!info || info->struct_size != sizeof(lbm_info))
    return fail(c, LBM_ERR_INVALID_ARG, "info is NULL or info.struct_size is wrong");
  info->nx = c->d.nx;
  info->ny = c->d.ny;
  info->nz = c->d.nz;
  info->mode = c->d.mode;
  info->precision = c->d.precision;
  info->iteration = c->iteration;
  info->device_bytes = c->dev_bytes;
  info->bytes_per_node = lbm::bytes_per_node(c->d);
  info->layout = c->d.mode == LBM_MODE_PHYSICS ? 1 : 0;
  info->device = c->device;
  return LBM_OK;
}

int lbm_get_params(lbm_ctx* c, lbm_params* p) {
  if (int rc = check_ctx(c)) return rc;
  if (!p || p->struct_size != sizeof(lbm_params))
    return fail(c, LBM_ERR_INVALID_ARG, "params is NULL or params.struct_size is wrong");
  const lbm_desc& d = c->d;
  p->tau = d.tau;
  std::memcpy(p->u_inf, d.u_inf, sizeof(p->u_inf));
  std::memcpy(p->body_accel, d.body_accel, sizeof(p->body_accel));
  std::memcpy(p->wall_velocity, d.wall_velocity, sizeof(p->wall_velocity));
  p->smagorinsky_cs = d.smagorinsky_cs;
  p->trt_magic = d.trt_magic;
  std::memcpy(p->open_rho, d.open_rho, sizeof(p->open_rho));
  return LBM_OK;
}

int lbm_set_params(lbm_ctx* c, const lbm_params* p) {
  if (int rc = check_ctx(c)) return rc;
  if (!p || p->struct_size != sizeof(lbm_params))
    return fail(c, LBM_ERR_INVALID_ARG, "params is NULL or params.struct_size is wrong");
  lbm_desc d = c->d;
  d.tau = p->tau;
  std::memcpy(d.u_inf, p->u_inf, sizeof(d.u_inf));
  std::memcpy(d.body_accel, p->body_accel, sizeof(d.body_accel));
  std::memcpy(d.wall_velocity, p->wall_velocity, sizeof(d.wall_velocity));
  d.smagorinsky_cs = p->smagorinsky_cs;
  d.trt_magic = p->trt_magic;
  std::memcpy(d.open_rho, p->open_rho, sizeof(d.open_rho));
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(d.u_inf[a]) || !std::isfinite(d.body_accel[a]))
      return fail(c, LBM_ERR_INVALID_ARG, "u_inf and body_accel must be finite");
  for (int f = 0; f < 6; ++f)
    for (int a = 0; a < 3; ++a)
      if (!std::isfinite(d.wall_velocity[f][a]))
        return fail(c, LBM_ERR_INVALID_ARG, "wall velocities must be finite");
  if (int rc = validate(&d)) return fail(c, rc, g_thread_err);
  if (c->d.mode == LBM_MODE_REFERENCE) {
    // The reference's uniforms carry tau and u_inf only (src/main.cpp:1523-1537).
    if (std::memcmp(d.body_accel, c->d.body_accel, sizeof(d.body_accel)) ||
        std::memcmp(d.wall_velocity, c->d.wall_velocity, sizeof(d.wall_velocity)) ||
        d.trt_magic != c->d.trt_magic || std::memcmp(d.open_rho, c->d.open_rho, sizeof(d.open_rho)))
      return fail(c, LBM_ERR_UNSUPPORTED, "reference mode takes tau and u_inf only");
  } else if (c->closure) {
    if (d.body_accel[0] != 0.f || d.body_accel[1] != 0.f || d.body_accel[2] != 0.f)
      return fail(c, LBM_ERR_UNSUPPORTED, "the closure kernels are built without a body force");
    if (!(d.smagorinsky_cs > 0.f))
      return fail(c, LBM_ERR_INVALID_ARG, "the closure scales smagorinsky_cs, which must be > 0");
  }
  // Captured graphs and queued launches hold the old parameters by value.
  CK(cudaStreamSynchronize(c->stream), "set_params sync");
  drop_graphs(c);
  const bool new_tau = d.tau != c->d.tau;
  c->d = d;
  if (d.mode == LBM_MODE_REFERENCE) {
    // CollideUniforms / BoundariesUniforms as the host fills them
    // (src/main.cpp:1524-1526, 1535).
    c->rp.tau_inv = 1.0f / d.tau;
    c->rp.omtau_inv = 1.0f - c->rp.tau_inv;
    for (int a = 0; a < 3; ++a) c->rp.u_inf[a] = d.u_inf[a];
    if (new_tau && c->initialized && c->redo != Ctx::REDO_NONE) {
      // Recompute the pending collision with the new tau.
      cudaError_t e;
      if (c->redo == Ctx::REDO_INIT) {
        // init's pre-collision state is feq of the moment fields it wrote
        e = lbm::ref_init(*c, c->rho, c->u, 1.0f, nullptr, c->stream, false);
      } else {
        // rerun the last launch from its untouched input: boundaries with the
        // parameters of that step, the collision with the new tau
        lbm::RefParams q = c->rp_last;
        q.tau_inv = c->rp.tau_inv;
        q.omtau_inv = c->rp.omtau_inv;
        e = lbm::ref_step_with(*c, q, c->fbuf[c->cur ^ 1], c->fbuf[c->cur], true, c->stream);
        c->rp_last.tau_inv = q.tau_inv;
        c->rp_last.omtau_inv = q.omtau_inv;
      }
      if (e != cudaSuccess) return cuda_fail(c, e, "recompute collision");
    }
  } else {
    lbm::setup_physics(*c, d);
  }
  return c->initialized ? prepare_graphs(c) : LBM_OK;
}

const char* lbm_last_error(lbm_ctx* c) { return c ? c->err.c_str() : g_thread_err.c_str(); }

}  // extern "C"
