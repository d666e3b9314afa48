// Host runtime of the batched ensemble (lbm_batch_* in include/lbm.h).
//
// All domains share one population pool and one auxiliary pool; each domain
// is described by a non-owning lbm::Ctx view into them, so initialisation,
// classification and readback reuse the single-domain kernels unchanged.
// The step runs as a CUDA graph of per-step launches or as one persistent
// cooperative launch (phys_batch.cu), with the tile shape picked by
// lbm_batch_autotune.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "batch_internal.h"

struct lbm_batch {
  std::vector<lbm::Ctx> dom;  // views into the pools; they own nothing
  std::vector<bool> ready;    // domain initialised since its last set_flags
  int precision = 0, collision = 0;
  lbm_batch_schedule sched{};
  std::vector<void*> allocs;
  lbm::BatchDomain* d_dom = nullptr;
  std::vector<lbm::BatchDomain> h_dom;
  uint2* d_tiles = nullptr;  // per tile: (domain, index within the domain)
  size_t tiles_cap = 0;
  unsigned* status = nullptr;
  unsigned* bar = nullptr;
  uint32_t ntiles = 0;
  int grid = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  static constexpr int kGraphSteps = 16;
  int parity = 0;
  uint64_t total_nodes = 0, iteration = 0, dev_bytes = 0;
  void* staging = nullptr;
  size_t staging_bytes = 0;
  size_t pop_bytes = 0;
  std::string err;
};

namespace {

int bfail(lbm_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  lbm::set_thread_error(msg.c_str());
  return code;
}

int bcuda(lbm_batch* b, cudaError_t e, const char* what) {
  cudaGetLastError();
  const int code = e == cudaErrorMemoryAllocation ? LBM_ERR_OUT_OF_MEMORY : LBM_ERR_CUDA;
  return bfail(b, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BCK(expr, what)                                    \
  do {                                                     \
    cudaError_t e_ = (expr);                               \
    if (e_ != cudaSuccess) return bcuda(b, e_, what);      \
  } while (0)

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

int balloc(lbm_batch* b, void** p, size_t bytes, const char* what) {
  cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 256));
  if (e != cudaSuccess) return bcuda(b, e, what);
  b->allocs.push_back(*p);
  b->dev_bytes += bytes;
  return LBM_OK;
}

void drop_graphs(lbm_batch* b) {
  for (auto& g : b->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

lbm::BatchLaunch launch_of(const lbm_batch* b) {
  lbm::BatchLaunch L{};
  L.dom = b->d_dom;
  L.tiles = b->d_tiles;
  L.ndom = (int)b->dom.size();
  L.ntiles = b->ntiles;
  L.rows = b->sched.rows_per_block;
  L.nzt = b->sched.z_per_thread;
  L.precision = b->precision;
  L.collision = b->collision;
  L.status = b->status;
  L.bar = b->bar;
  L.spin_limit = b->sched.spin_limit_cycles;
  L.missing_blocks = b->sched.test_missing_blocks;
  return L;
}

// Rebuilds the tile table for the current schedule and uploads it.
int build_tiles(lbm_batch* b) {
  const int R = b->sched.rows_per_block, Z = b->sched.z_per_thread;
  uint64_t t = 0;
  for (size_t i = 0; i < b->dom.size(); ++i) {
    const lbm::Ctx& v = b->dom[i];
    lbm::BatchDomain& D = b->h_dom[i];
    std::memset(&D, 0, sizeof(D));
    D.p = v.pp;
    D.pop = v.pop;
    D.flags = v.flags;
    D.links = v.links;
    D.rho = v.rho;
    D.u = v.u;
    D.pairs = (LBM_BATCH_PAIRS && lbm::step_pairs_host(v.d.nx)) ? 1u : 0u;
    D.tiles_x = D.pairs ? (v.d.nx + 63) / 64 : (v.d.nx + 31) / 32;
    D.tiles_y = (v.d.ny + R - 1) / R;
    D.tile_begin = (uint32_t)t;
    t += (uint64_t)D.tiles_x * D.tiles_y * ((v.d.nz + Z - 1) / Z);
  }
  if (t >= (1ull << 31)) return bfail(b, LBM_ERR_UNSUPPORTED, "more than 2^31 tiles");
  b->ntiles = (uint32_t)t;
  std::vector<uint2> table(t);
  for (size_t i = 0; i < b->dom.size(); ++i) {
    const uint32_t begin = b->h_dom[i].tile_begin;
    const uint32_t end = i + 1 < b->dom.size() ? b->h_dom[i + 1].tile_begin : (uint32_t)t;
    for (uint32_t k = begin; k < end; ++k) table[k] = make_uint2((unsigned)i, k - begin);
  }
  if (b->tiles_cap < t) {
    if (b->d_tiles) {
      cudaFree(b->d_tiles);
      b->allocs.erase(std::find(b->allocs.begin(), b->allocs.end(), (void*)b->d_tiles));
      b->d_tiles = nullptr;
    }
    void* p = nullptr;
    if (int rc = balloc(b, &p, t * sizeof(uint2), "cudaMalloc(tile table)")) return rc;
    b->d_tiles = static_cast<uint2*>(p);
    b->tiles_cap = t;
  }
  BCK(cudaMemcpyAsync(b->d_tiles, table.data(), t * sizeof(uint2), cudaMemcpyHostToDevice, b->stream),
      "upload tile list");
  BCK(cudaMemcpyAsync(b->d_dom, b->h_dom.data(), b->h_dom.size() * sizeof(lbm::BatchDomain),
                      cudaMemcpyHostToDevice, b->stream),
      "upload tile table");
  BCK(cudaStreamSynchronize(b->stream), "tile table sync");
  drop_graphs(b);
  b->grid = 0;
  if (b->sched.persistent) BCK(lbm::batch_persistent_grid(launch_of(b), &b->grid), "persistent grid");
  return LBM_OK;
}

int ensure_staging(lbm_batch* b, size_t bytes) {
  if (b->staging_bytes >= bytes) return LBM_OK;
  if (b->staging) {
    cudaFree(b->staging);
    b->allocs.erase(std::find(b->allocs.begin(), b->allocs.end(), b->staging));
    b->dev_bytes -= b->staging_bytes;
    b->staging = nullptr;
  }
  if (int rc = balloc(b, &b->staging, bytes, "cudaMalloc(staging)")) return rc;
  b->staging_bytes = bytes;
  return LBM_OK;
}

int check_domain(lbm_batch* b, int d) {
  if (!b) return bfail(nullptr, LBM_ERR_INVALID_ARG, "batch is NULL");
  if (d < 0 || d >= (int)b->dom.size()) return bfail(b, LBM_ERR_INVALID_ARG, "domain index out of range");
  return LBM_OK;
}

size_t u_bytes(int fmt) {
  return fmt == LBM_U_F32X3 ? 12 : fmt == LBM_U_F32X4 ? 16 : fmt == LBM_U_F16X4 ? 8 : 0;
}

bool valid_schedule(const lbm_batch_schedule& s) {
  const bool rows = s.rows_per_block == 1 || s.rows_per_block == 2 || s.rows_per_block == 4 ||
                    s.rows_per_block == 8;
  const bool z = s.z_per_thread >= 1 && s.z_per_thread <= 16;
  return rows && z && (s.persistent == 0 || s.persistent == 1) && s.spin_limit_cycles > 0 &&
         s.test_missing_blocks >= 0;
}

// Captures kGraphSteps steps from parity `slot`, without the moment write:
// kGraphSteps launches of the tile kernel, or in persistent mode one
// cooperative launch that takes all of them with grid barriers between.
int build_graph(lbm_batch* b, int slot) {
  const lbm::BatchLaunch L = launch_of(b);
  cudaGraph_t g = nullptr;
  BCK(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaError_t e = cudaSuccess;
  if (b->sched.persistent) {
    e = lbm::batch_persistent(L, lbm_batch::kGraphSteps, slot, b->grid, b->own, false);
  } else {
    int P = slot;
    for (int i = 0; i < lbm_batch::kGraphSteps && e == cudaSuccess; ++i, P ^= 1)
      e = lbm::batch_step(L, P, false, b->own);
  }
  const cudaError_t e2 = cudaStreamEndCapture(b->own, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return bcuda(b, e != cudaSuccess ? e : e2, "capture batch graph");
  }
  e = cudaGraphInstantiate(&b->graph[slot], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return bcuda(b, e, "instantiate batch graph");
  BCK(cudaGraphUpload(b->graph[slot], b->stream), "upload batch graph");
  return LBM_OK;
}

// Launches nsteps steps (the last one writes the moments): captured graphs
// of kGraphSteps steps while more remain (an even count keeps the parity),
// then the rest directly.
int run_steps(lbm_batch* b, int nsteps) {
  if (nsteps <= 0) return LBM_OK;
  const lbm::BatchLaunch L = launch_of(b);
  int left = nsteps;
  while (left > lbm_batch::kGraphSteps) {
    const int slot = b->parity;
    if (!b->graph[slot])
      if (int rc = build_graph(b, slot)) return rc;
    BCK(cudaGraphLaunch(b->graph[slot], b->stream), "batch graph launch");
    left -= lbm_batch::kGraphSteps;
  }
  if (b->sched.persistent) {
    BCK(lbm::batch_persistent(L, left, b->parity, b->grid, b->stream, true), "persistent launch");
    b->parity ^= (left & 1);
    return LBM_OK;
  }
  for (int i = 0; i < left; ++i) {
    BCK(lbm::batch_step(L, b->parity, i == left - 1, b->stream), "batch step launch");
    b->parity ^= 1;
  }
  return LBM_OK;
}

// Autotune results for this process, keyed by (precision, collision,
// log2 of total nodes, log2 of domain count); optionally persisted as text
// lines in $LBM_AUTOTUNE_CACHE.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, lbm_batch_schedule> g_tune;

std::tuple<int, int, int, int> tune_key(const lbm_batch* b) {
  return {b->precision, b->collision, (int)std::lround(std::log2((double)std::max<uint64_t>(b->total_nodes, 1))),
          (int)std::lround(std::log2((double)std::max<size_t>(b->dom.size(), 1)))};
}

void cache_load() {
  const char* path = std::getenv("LBM_AUTOTUNE_CACHE");
  if (!path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  int p, c, n, d, r, z, pe;
  while (std::fscanf(f, "%d %d %d %d %d %d %d", &p, &c, &n, &d, &r, &z, &pe) == 7) {
    lbm_batch_schedule s{};
    s.struct_size = sizeof(s);
    s.rows_per_block = r;
    s.z_per_thread = z;
    s.persistent = pe;
    s.spin_limit_cycles = 2000000000LL;
    if (valid_schedule(s)) g_tune[{p, c, n, d}] = s;
  }
  std::fclose(f);
}

void cache_store(const std::tuple<int, int, int, int>& k, const lbm_batch_schedule& s) {
  const char* path = std::getenv("LBM_AUTOTUNE_CACHE");
  if (!path) return;
  if (FILE* f = std::fopen(path, "a")) {
    std::fprintf(f, "%d %d %d %d %d %d %d\n", std::get<0>(k), std::get<1>(k), std::get<2>(k),
                 std::get<3>(k), s.rows_per_block, s.z_per_thread, s.persistent);
    std::fclose(f);
  }
}

}  // namespace

extern "C" {

int lbm_batch_schedule_default(lbm_batch_schedule* s) {
  if (!s) return bfail(nullptr, LBM_ERR_INVALID_ARG, "schedule is NULL");
  std::memset(s, 0, sizeof(*s));
  s->struct_size = sizeof(*s);
  s->rows_per_block = 4;
  s->z_per_thread = 1;
  s->persistent = 0;
  s->spin_limit_cycles = 2000000000LL;  // about one second at the B200's clocks
  s->test_missing_blocks = 0;
  return LBM_OK;
}

int lbm_batch_create(const lbm_desc* descs, int n, lbm_batch** out) {
  if (!out) return bfail(nullptr, LBM_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!descs || n < 1) return bfail(nullptr, LBM_ERR_INVALID_ARG, "need at least one descriptor");
  for (int i = 0; i < n; ++i) {
    if (int rc = lbm::validate_desc(&descs[i])) return rc;
    const lbm_desc& d = descs[i];
    if (d.mode != LBM_MODE_PHYSICS)
      return bfail(nullptr, LBM_ERR_UNSUPPORTED, "batched domains run the physics mode");
    if (d.precision != descs[0].precision || d.collision != descs[0].collision)
      return bfail(nullptr, LBM_ERR_UNSUPPORTED, "all batched domains share precision and collision");
    if (d.smagorinsky_cs != 0.f || d.body_accel[0] != 0.f || d.body_accel[1] != 0.f ||
        d.body_accel[2] != 0.f)
      return bfail(nullptr, LBM_ERR_UNSUPPORTED,
                   "batched domains have no Smagorinsky term and no body force (use lbm_create)");
    if (d.open_x[0] != LBM_OPEN_NONE || d.open_x[1] != LBM_OPEN_NONE)
      return bfail(nullptr, LBM_ERR_UNSUPPORTED, "batched domains have no open faces (use lbm_create)");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return bfail(nullptr, LBM_ERR_NO_DEVICE, "no CUDA device");
  }
  lbm_batch* b = new (std::nothrow) lbm_batch();
  if (!b) return bfail(nullptr, LBM_ERR_OUT_OF_MEMORY, "host allocation failed");
  auto bail = [&](int code) {
    lbm_batch_destroy(b);
    return code;
  };
  b->precision = descs[0].precision;
  b->collision = descs[0].collision;
  lbm_batch_schedule_default(&b->sched);
  if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess)
    return bail(bfail(b, LBM_ERR_CUDA, "cudaStreamCreate"));
  b->stream = b->own;
  int dev = 0;
  cudaGetDevice(&dev);
  b->dom.resize(n);
  b->ready.assign(n, false);
  b->h_dom.resize(n);
  // layout of the pools
  const size_t eb = lbm::elem_bytes(b->precision);
  std::vector<size_t> pop_off(n), aux_off(n);
  size_t pop_total = 0, aux_total = 0;
  for (int i = 0; i < n; ++i) {
    lbm::Ctx& v = b->dom[i];
    v.d = descs[i];
    v.device = dev;
    v.n = (size_t)descs[i].nx * descs[i].ny * descs[i].nz;
    if (!lbm::setup_physics(v, descs[i]))
      return bail(bfail(b, LBM_ERR_UNSUPPORTED, "a domain exceeds 2^32 nodes per slot array"));
    pop_off[i] = pop_total;
    pop_total += up256(19 * v.pp.g.slot_stride * eb);
    aux_off[i] = aux_total;
    aux_total += up256(v.n) * 2 + up256(4 * v.n) * 2 + up256(12 * v.n);
    b->total_nodes += v.n;
  }
  void *pop = nullptr, *aux = nullptr, *dd = nullptr, *st = nullptr;
  if (int rc = balloc(b, &pop, pop_total, "cudaMalloc(population pool)")) return bail(rc);
  if (int rc = balloc(b, &aux, aux_total, "cudaMalloc(aux pool)")) return bail(rc);
  if (int rc = balloc(b, &dd, n * sizeof(lbm::BatchDomain), "cudaMalloc(tile table)")) return bail(rc);
  if (int rc = balloc(b, &st, 256, "cudaMalloc(status)")) return bail(rc);
  b->pop_bytes = pop_total;
  b->d_dom = static_cast<lbm::BatchDomain*>(dd);
  b->status = static_cast<unsigned*>(st);
  b->bar = b->status + 8;
  BCK(cudaMemsetAsync(pop, 0, pop_total, b->stream), "clear pool");
  BCK(cudaMemsetAsync(aux, 0, aux_total, b->stream), "clear pool");
  BCK(cudaMemsetAsync(st, 0, 256, b->stream), "clear status");
  for (int i = 0; i < n; ++i) {
    lbm::Ctx& v = b->dom[i];
    char* a = static_cast<char*>(aux) + aux_off[i];
    v.pop = static_cast<char*>(pop) + pop_off[i];
    v.mask = reinterpret_cast<uint8_t*>(a);
    a += up256(v.n);
    v.flags = reinterpret_cast<uint8_t*>(a);
    a += up256(v.n);
    v.links = reinterpret_cast<uint32_t*>(a);
    a += up256(4 * v.n);
    v.rho = reinterpret_cast<float*>(a);
    a += up256(4 * v.n);
    v.u = reinterpret_cast<float*>(a);
    v.status = b->status;
    v.stream = b->stream;
    const int per[3] = {v.d.periodic[0], v.d.periodic[1], v.d.periodic[2]};
    if (cudaError_t e = lbm::classify(v, per, b->stream)) return bail(bcuda(b, e, "classify"));
  }
  if (int rc = build_tiles(b)) return bail(rc);
  *out = b;
  return LBM_OK;
}

int lbm_batch_destroy(lbm_batch* b) {
  if (!b) return LBM_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  for (void* p : b->allocs) cudaFree(p);
  if (b->own) cudaStreamDestroy(b->own);
  delete b;
  return LBM_OK;
}

int lbm_batch_set_stream(lbm_batch* b, void* stream) {
  if (!b) return bfail(nullptr, LBM_ERR_INVALID_ARG, "batch is NULL");
  BCK(cudaStreamSynchronize(b->stream), "set_stream sync");
  b->stream = stream ? static_cast<cudaStream_t>(stream) : b->own;
  for (auto& v : b->dom) v.stream = b->stream;
  return LBM_OK;
}

int lbm_batch_set_flags(lbm_batch* b, int d, const uint8_t* mask, size_t n) {
  if (int rc = check_domain(b, d)) return rc;
  lbm::Ctx& v = b->dom[d];
  if (!mask || n != v.n) return bfail(b, LBM_ERR_INVALID_ARG, "mask length must be Nx*Ny*Nz");
  BCK(cudaMemcpyAsync(v.mask, mask, n, cudaMemcpyHostToDevice, b->stream), "upload mask");
  const int per[3] = {v.d.periodic[0], v.d.periodic[1], v.d.periodic[2]};
  BCK(lbm::classify(v, per, b->stream), "classify");
  BCK(cudaStreamSynchronize(b->stream), "set_flags sync");
  b->ready[d] = false;
  return LBM_OK;
}

static int batch_init(lbm_batch* b, int d, const float* d_rho, const float* d_u, float rho0,
                      const float* u0) {
  lbm::Ctx& v = b->dom[d];
  v.parity = b->parity;
  BCK(lbm::phys_init(v, d_rho, d_u, rho0, u0, b->stream), "init kernel");
  b->ready[d] = true;
  return LBM_OK;
}

int lbm_batch_init_equilibrium(lbm_batch* b, int d, float rho0, const float u0[3]) {
  if (!b) return bfail(nullptr, LBM_ERR_INVALID_ARG, "batch is NULL");
  if (!u0 || !std::isfinite(rho0)) return bfail(b, LBM_ERR_INVALID_ARG, "bad rho0 or u0");
  if (d == -1) {
    for (int i = 0; i < (int)b->dom.size(); ++i)
      if (int rc = batch_init(b, i, nullptr, nullptr, rho0, u0)) return rc;
    return LBM_OK;
  }
  if (int rc = check_domain(b, d)) return rc;
  return batch_init(b, d, nullptr, nullptr, rho0, u0);
}

int lbm_batch_init_from_moments(lbm_batch* b, int d, const float* rho, const void* u, int u_fmt) {
  if (int rc = check_domain(b, d)) return rc;
  if (!rho || !u) return bfail(b, LBM_ERR_INVALID_ARG, "rho and u must not be NULL");
  const size_t ub = u_bytes(u_fmt);
  if (!ub) return bfail(b, LBM_ERR_INVALID_ARG, "unknown u format");
  const size_t n = b->dom[d].n;
  if (int rc = ensure_staging(b, n * (16 + ub))) return rc;
  float* d_rho = static_cast<float*>(b->staging);
  float* d_u = d_rho + n;
  void* d_raw = d_u + 3 * n;
  BCK(cudaMemcpyAsync(d_rho, rho, n * 4, cudaMemcpyHostToDevice, b->stream), "upload rho");
  BCK(cudaMemcpyAsync(d_raw, u, n * ub, cudaMemcpyHostToDevice, b->stream), "upload u");
  BCK(lbm::u_format_to_planes(d_raw, n, u_fmt, d_u, b->stream), "convert u");
  const float zero[3] = {0.f, 0.f, 0.f};
  if (int rc = batch_init(b, d, d_rho, d_u, 1.0f, zero)) return rc;
  BCK(cudaStreamSynchronize(b->stream), "init sync");
  return LBM_OK;
}

int lbm_batch_step(lbm_batch* b, int nsteps) {
  if (!b) return bfail(nullptr, LBM_ERR_INVALID_ARG, "batch is NULL");
  if (nsteps < 0) return bfail(b, LBM_ERR_INVALID_ARG, "nsteps must be >= 0");
  for (size_t i = 0; i < b->ready.size(); ++i)
    if (!b->ready[i]) return bfail(b, LBM_ERR_STATE, "lbm_batch_step before every domain was initialised");
  if (int rc = run_steps(b, nsteps)) return rc;
  b->iteration += (uint64_t)nsteps;
  for (auto& v : b->dom) v.parity = b->parity;
  return LBM_OK;
}

int lbm_batch_sync(lbm_batch* b) {
  if (!b) return bfail(nullptr, LBM_ERR_INVALID_ARG, "batch is NULL");
  unsigned st = 0;
  BCK(cudaMemcpyAsync(&st, b->status, sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream), "read status");
  BCK(cudaStreamSynchronize(b->stream), "sync");
  if (st) {
    BCK(cudaMemsetAsync(b->status, 0, sizeof(unsigned), b->stream), "reset status");
    BCK(cudaStreamSynchronize(b->stream), "sync");
    if (st & lbm::BATCH_STATUS_TIMEOUT) {
      // The persistent kernel stopped between steps; the state is not a
      // whole number of steps any more.
      for (size_t i = 0; i < b->ready.size(); ++i) b->ready[i] = false;
      return bfail(b, LBM_ERR_TIMEOUT, "a grid-barrier wait of the persistent step gave up");
    }
    return bfail(b, LBM_ERR_NONFINITE, "non-finite value or rho <= 0 at a fluid node");
  }
  return LBM_OK;
}

int lbm_batch_read_moments(lbm_batch* b, int d, float* rho, void* u, int u_fmt) {
  if (int rc = check_domain(b, d)) return rc;
  lbm::Ctx& v = b->dom[d];
  if (rho) BCK(cudaMemcpyAsync(rho, v.rho, v.n * 4, cudaMemcpyDeviceToHost, b->stream), "read rho");
  if (u) {
    const size_t ub = u_bytes(u_fmt);
    if (!ub) return bfail(b, LBM_ERR_INVALID_ARG, "unknown u format");
    if (int rc = ensure_staging(b, v.n * ub)) return rc;
    BCK(lbm::u_planes_to_format(v.u, v.n, u_fmt, b->staging, b->stream), "convert u");
    BCK(cudaMemcpyAsync(u, b->staging, v.n * ub, cudaMemcpyDeviceToHost, b->stream), "read u");
  }
  BCK(cudaStreamSynchronize(b->stream), "read sync");
  return LBM_OK;
}

int lbm_batch_read_populations(lbm_batch* b, int d, float* f, size_t n) {
  if (int rc = check_domain(b, d)) return rc;
  lbm::Ctx& v = b->dom[d];
  if (!f || n != 19 * v.n) return bfail(b, LBM_ERR_INVALID_ARG, "f must hold 19*Nx*Ny*Nz floats");
  if (int rc = ensure_staging(b, n * 4)) return rc;
  v.parity = b->parity;
  BCK(lbm::phys_read_pops(v, static_cast<float*>(b->staging), b->stream), "gather populations");
  BCK(cudaMemcpyAsync(f, b->staging, n * 4, cudaMemcpyDeviceToHost, b->stream), "read populations");
  BCK(cudaStreamSynchronize(b->stream), "read sync");
  return LBM_OK;
}

int lbm_batch_set_schedule(lbm_batch* b, const lbm_batch_schedule* s) {
  if (!b || !s) return bfail(b, LBM_ERR_INVALID_ARG, "NULL argument");
  if (s->struct_size != sizeof(lbm_batch_schedule) || !valid_schedule(*s))
    return bfail(b, LBM_ERR_INVALID_ARG, "schedule out of range (rows 1/2/4/8, z 1..16, persistent 0/1)");
  BCK(cudaStreamSynchronize(b->stream), "schedule sync");
  b->sched = *s;
  return build_tiles(b);
}

int lbm_batch_get_schedule(lbm_batch* b, lbm_batch_schedule* s) {
  if (!b || !s) return bfail(b, LBM_ERR_INVALID_ARG, "NULL argument");
  *s = b->sched;
  return LBM_OK;
}

int lbm_batch_autotune(lbm_batch* b, int trial_steps, lbm_batch_schedule* best_out) {
  if (!b) return bfail(nullptr, LBM_ERR_INVALID_ARG, "batch is NULL");
  if (trial_steps < 2) return bfail(b, LBM_ERR_INVALID_ARG, "trial_steps must be >= 2");
  for (size_t i = 0; i < b->ready.size(); ++i)
    if (!b->ready[i]) return bfail(b, LBM_ERR_STATE, "autotune needs every domain initialised");
  const auto key = tune_key(b);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    static bool loaded = false;
    if (!loaded) {
      cache_load();
      loaded = true;
    }
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      lbm_batch_schedule s = it->second;
      s.spin_limit_cycles = b->sched.spin_limit_cycles;
      if (int rc = lbm_batch_set_schedule(b, &s)) return rc;
      if (best_out) *best_out = b->sched;
      return LBM_OK;
    }
  }
  // The trials advance the state: keep a copy of the populations and put it
  // back afterwards (moments are rewritten by the next step anyway).
  void* snap = nullptr;
  BCK(cudaMalloc(&snap, b->pop_bytes), "cudaMalloc(autotune snapshot)");
  void* pool = b->dom[0].pop;
  const int parity0 = b->parity;
  cudaMemcpyAsync(snap, pool, b->pop_bytes, cudaMemcpyDeviceToDevice, b->stream);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  lbm_batch_schedule best = b->sched;
  float best_ms = 1e30f;
  int rc = LBM_OK;
  for (int pers = 0; pers <= 1 && rc == LBM_OK; ++pers)
    for (int rows : {2, 4, 8})
      for (int zt : {1, 2, 4, 8, 16}) {
        lbm_batch_schedule s = b->sched;
        s.rows_per_block = rows;
        s.z_per_thread = zt;
        s.persistent = pers;
        s.test_missing_blocks = 0;
        if ((rc = lbm_batch_set_schedule(b, &s))) break;
        if ((rc = run_steps(b, 2))) break;  // warm (and build graphs)
        cudaEventRecord(e0, b->stream);
        if ((rc = run_steps(b, trial_steps))) break;
        cudaEventRecord(e1, b->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
          best_ms = ms;
          best = s;
        }
      }
  cudaMemcpyAsync(pool, snap, b->pop_bytes, cudaMemcpyDeviceToDevice, b->stream);
  cudaStreamSynchronize(b->stream);
  cudaFree(snap);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->parity = parity0;
  for (auto& v : b->dom) v.parity = parity0;
  if (rc) return rc;
  if (int r2 = lbm_batch_set_schedule(b, &best)) return r2;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = best;
    cache_store(key, best);
  }
  if (best_out) *best_out = best;
  return LBM_OK;
}

int lbm_batch_get_info(lbm_batch* b, lbm_batch_info* info) {
  if (!b || !info || info->struct_size != sizeof(lbm_batch_info))
    return bfail(b, LBM_ERR_INVALID_ARG, "NULL argument or wrong struct_size");
  info->domains = (int32_t)b->dom.size();
  info->total_nodes = b->total_nodes;
  info->tiles = b->ntiles;
  info->grid = b->grid;
  info->iteration = b->iteration;
  info->device_bytes = b->dev_bytes;
  info->bytes_per_node = lbm::bytes_per_node(b->dom[0].d);
  return LBM_OK;
}

const char* lbm_batch_last_error(lbm_batch* b) { return b ? b->err.c_str() : lbm_last_error(nullptr); }

}  // extern "C"
