// Learned-closure training pipeline: box filter of fine moment fields,
// training samples from a filtered field, the fused forward/backward kernel
// of the MLP, the Adam update, prediction, and the trainer's C ABI
// (lbm_closure.h).  The network and its features are closure.cuh, shared
// with the collide of the step kernels.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "closure.cuh"
#include "lbm_internal.h"

namespace lbm {

float round_bf16(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) {  // Inf or NaN: truncate, keep NaN quiet
    if (u & 0x007fffffu) u |= 0x00400000u;
    u &= 0xffff0000u;
  } else {
    u += 0x7fffu + ((u >> 16) & 1u);  // nearest, ties to even
    u &= 0xffff0000u;
  }
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

namespace {

// ---------------------------------------------------------------------------
// Box filter: one thread per coarse node, Favre averages of factor^3 fine
// nodes accumulated in fp64.  Consecutive threads take consecutive coarse x,
// so a warp reads contiguous fine rows.
// ---------------------------------------------------------------------------
__global__ void k_box_filter(const float* __restrict__ rho, const float* __restrict__ u, int nx,
                             int ny, int nz, int f, float* __restrict__ out) {
  const int ncx = nx / f, ncy = ny / f, ncz = nz / f;
  const size_t nc = (size_t)ncx * ncy * ncz;
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int X = (int)(c % ncx);
  const size_t r = c / ncx;
  const int Y = (int)(r % ncy), Z = (int)(r / ncy);
  const size_t n = (size_t)nx * ny * nz;
  double sr = 0, jx = 0, jy = 0, jz = 0, xx = 0, yy = 0, zz = 0, xy = 0, xz = 0, yz = 0;
  for (int dz = 0; dz < f; ++dz)
    for (int dy = 0; dy < f; ++dy) {
      const size_t base = (size_t)X * f + (size_t)nx * ((size_t)Y * f + dy + (size_t)ny * ((size_t)Z * f + dz));
      for (int dx = 0; dx < f; ++dx) {
        const size_t i = base + dx;
        const double rh = rho[i], ux = u[i], uy = u[n + i], uz = u[2 * n + i];
        const double mx = rh * ux, my = rh * uy, mz = rh * uz;
        sr += rh;
        jx += mx; jy += my; jz += mz;
        xx += mx * ux; yy += my * uy; zz += mz * uz;
        xy += mx * uy; xz += mx * uz; yz += my * uz;
      }
    }
  float o[10] = {};
  if (sr > 0) {
    const double ux = jx / sr, uy = jy / sr, uz = jz / sr;
    o[0] = (float)(sr / ((double)f * f * f));
    o[1] = (float)ux; o[2] = (float)uy; o[3] = (float)uz;
    o[4] = (float)(xx / sr - ux * ux); o[5] = (float)(yy / sr - uy * uy); o[6] = (float)(zz / sr - uz * uz);
    o[7] = (float)(xy / sr - ux * uy); o[8] = (float)(xz / sr - ux * uz); o[9] = (float)(yz / sr - uy * uz);
  }
  for (int k = 0; k < 10; ++k) out[k * nc + c] = o[k];
}

// ---------------------------------------------------------------------------
// Training samples (see lbm_closure_samples).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void k_samples(const float* __restrict__ filt, int nx, int ny, int nz, float tau,
                          float cs0, uint64_t seed, int64_t ns, float* __restrict__ xo,
                          float* __restrict__ to, float* __restrict__ wo) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const size_t n = (size_t)nx * ny * nz;
  const size_t node = seed == 0 ? (size_t)i : (size_t)(mix64(seed * 0x9e3779b97f4a7c15ull + (uint64_t)i) % n);
  const int x = (int)(node % nx);
  const int y = (int)((node / nx) % ny), z = (int)(node / ((size_t)nx * ny));
  const int xp = x + 1 == nx ? 0 : x + 1, xm = x == 0 ? nx - 1 : x - 1;
  const int yp = y + 1 == ny ? 0 : y + 1, ym = y == 0 ? ny - 1 : y - 1;
  const int zp = z + 1 == nz ? 0 : z + 1, zm = z == 0 ? nz - 1 : z - 1;
  auto at = [&](int xx, int yy, int zz) { return (size_t)xx + (size_t)nx * ((size_t)yy + (size_t)ny * zz); };
  const size_t nb[3][2] = {{at(xp, y, z), at(xm, y, z)}, {at(x, yp, z), at(x, ym, z)}, {at(x, y, zp), at(x, y, zm)}};
  double G[3][3];  // G[a][b] = d u_a / d x_b, central differences
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      G[a][b] = 0.5 * ((double)filt[(1 + a) * n + nb[b][0]] - (double)filt[(1 + a) * n + nb[b][1]]);
  // S in the order xx yy zz xy xz yz
  const double S[6] = {G[0][0], G[1][1], G[2][2], 0.5 * (G[0][1] + G[1][0]),
                       0.5 * (G[0][2] + G[2][0]), 0.5 * (G[1][2] + G[2][1])};
  const double ss = S[0] * S[0] + S[1] * S[1] + S[2] * S[2] + 2.0 * (S[3] * S[3] + S[4] * S[4] + S[5] * S[5]);
  const double smag = sqrt(2.0 * ss);  // |S|
  double t[6];
  for (int k = 0; k < 6; ++k) t[k] = filt[(4 + k) * n + node];
  const double tr = (t[0] + t[1] + t[2]) / 3.0;
  const double tds = (t[0] - tr) * S[0] + (t[1] - tr) * S[1] + (t[2] - tr) * S[2] +
                     2.0 * (t[3] * S[3] + t[4] * S[4] + t[5] * S[5]);
  const double c2 = (double)cs0 * cs0;
  const double s3 = smag * smag * smag;
  const bool ok = s3 > 1e-300;
  const double rho = filt[node];
  const double taus = (double)tau + 3.0 * c2 * smag;
  float P[6];
  for (int k = 0; k < 6; ++k) P[k] = (float)(-(2.0 / 3.0) * rho * taus * S[k]);
  float xf[CLO_IN];
  closure_features<Ops1>(P, (float)rho, xf);
  for (int k = 0; k < CLO_IN; ++k) xo[(size_t)i * CLO_IN + k] = xf[k];
  to[i] = ok ? (float)(-tds / (c2 * s3)) : 0.0f;
  wo[i] = ok ? (float)s3 : 0.0f;
}

// ---------------------------------------------------------------------------
// Prediction: one thread per sample, network in shared memory.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_predict(const float* __restrict__ net,
                                                 const float* __restrict__ x, int64_t n,
                                                 float* __restrict__ r) {
  __shared__ float sw[CLO_FLOATS];
  for (int k = threadIdx.x; k < CLO_FLOATS; k += blockDim.x) sw[k] = net[k];
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float xi[CLO_IN];
  for (int k = 0; k < CLO_IN; ++k) xi[k] = x[(size_t)i * CLO_IN + k];
  const float* w = sw;
  r[i] = closure_mlp<Ops1>(w, xi);
}

// ---------------------------------------------------------------------------
// Fused forward/backward of one batch.
//
// A warp takes 32 samples at a time, lane = sample, for the forward pass
// and the backward pass through the activations; it leaves the per-sample
// activations (h1, h2), pre-activation gradients (d a1, d a2), standardised
// inputs and d z in shared memory.  The weight gradients are then
// accumulated with lane = hidden unit: lane i owns row i of dW2 and dW1 and
// entry i of db1, db2, dW3, so each sums its 32 samples with no atomics.
// At the end the block's warps are summed in a fixed order into the
// block's slot of `part` (one row of LBM_CLOSURE_PARAMS per block), which
// the Adam kernel sums over blocks, again in a fixed order: the gradient is
// deterministic.
// Sample j of the batch is dataset row (a * (start + j) + c) mod n.
// ---------------------------------------------------------------------------
constexpr int TR_WARPS = 4;
constexpr int TR_THREADS = 32 * TR_WARPS;
constexpr int TR_LD = 36;   // row stride of the per-warp [32][36] tiles: float4
                            // stores of 8 lanes hit 32 distinct banks
constexpr int TR_XLD = 12;  // row stride of the inputs tile
constexpr int TR_WARP_FLOATS = 4 * 32 * TR_LD + 32 * TR_XLD + 32;
constexpr int TR_MAX_BLOCKS = 296;
// the network copy is padded to a multiple of 4 floats so that every tile
// after it starts on a 16-byte boundary (float4 accesses)
constexpr int TR_NET = (CLO_FLOATS + 3) / 4 * 4;
constexpr size_t TR_SMEM = (size_t)(TR_NET + CLO_HID * CLO_HID + TR_WARPS * TR_WARP_FLOATS) * 4;
static_assert(TR_NET % 4 == 0 && (CLO_HID * CLO_HID) % 4 == 0 && TR_WARP_FLOATS % 4 == 0 &&
                  TR_LD % 4 == 0 && TR_XLD % 4 == 0 && CLO_W2 % 4 == 0,
              "16-byte alignment of the float4 tiles");

struct Batch {
  const float* x;
  const float* t;
  const float* w;
  int64_t n;       // dataset rows
  int64_t start;   // position of the batch in the epoch order
  int64_t nb;      // samples in the batch
  uint64_t a, c;   // affine order: row = (a * pos + c) mod n
  float wscale;    // loss = wscale * sum w (r - t)^2
};

__global__ void __launch_bounds__(TR_THREADS, 2)
    k_mlp_grad(const float* __restrict__ net, Batch B, float* __restrict__ part,
               double* __restrict__ loss_part) {
  extern __shared__ __align__(16) float sm[];
  float* sw = sm;                                       // network [CLO_FLOATS] (padded)
  float* sW2T = sm + TR_NET;                            // W2 transposed [j][i]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* wb = sW2T + CLO_HID * CLO_HID + warp * TR_WARP_FLOATS;
  float* sH1 = wb;                  // [32][TR_LD] h1 per sample
  float* sH2 = sH1 + 32 * TR_LD;    // h2
  float* sA1 = sH2 + 32 * TR_LD;    // d a1
  float* sA2 = sA1 + 32 * TR_LD;    // d a2
  float* sX = sA2 + 32 * TR_LD;     // [32][TR_XLD] standardised inputs
  float* sDZ = sX + 32 * TR_XLD;    // [32] d z

  for (int k = threadIdx.x; k < CLO_FLOATS; k += TR_THREADS) sw[k] = net[k];
  for (int k = threadIdx.x; k < CLO_HID * CLO_HID; k += TR_THREADS) {
    const int i = k / CLO_HID, j = k % CLO_HID;
    sW2T[j * CLO_HID + i] = net[CLO_W2 + k];
  }
  __syncthreads();

  float gW2[CLO_HID], gW1[CLO_IN];
#pragma unroll
  for (int j = 0; j < CLO_HID; ++j) gW2[j] = 0.f;
#pragma unroll
  for (int k = 0; k < CLO_IN; ++k) gW1[k] = 0.f;
  float gb1 = 0.f, gb2 = 0.f, gW3 = 0.f, gb3 = 0.f;
  double lsum = 0.0;

  const int64_t groups = (B.nb + 31) / 32;
  for (int64_t gi = (int64_t)blockIdx.x * TR_WARPS + warp; gi < groups;
       gi += (int64_t)gridDim.x * TR_WARPS) {
    // ---- forward and activation backward, lane = sample ----
    const int64_t j = gi * 32 + lane;
    const bool valid = j < B.nb;
    float xs[CLO_IN];
    float tgt = 0.f, wt = 0.f;
    if (valid) {
      const uint64_t pos = (uint64_t)(B.start + j);
      const size_t row = (size_t)((B.a * pos + B.c) % (uint64_t)B.n);
#pragma unroll
      for (int k = 0; k < CLO_IN; ++k)
        xs[k] = (B.x[row * CLO_IN + k] - sw[CLO_MEAN + k]) * sw[CLO_ISCALE + k];
      tgt = B.t[row];
      wt = B.w[row];
    } else {
#pragma unroll
      for (int k = 0; k < CLO_IN; ++k) xs[k] = 0.f;
    }
    float h1[CLO_HID];
#pragma unroll
    for (int i = 0; i < CLO_HID; ++i) {
      float a = sw[CLO_B1 + i];
#pragma unroll
      for (int k = 0; k < CLO_IN; ++k) a = fmaf(sw[CLO_W1 + i * CLO_IN + k], xs[k], a);
      h1[i] = fmaxf(a, 0.f);
    }
    float z = sw[CLO_B3];
    unsigned m2 = 0;
#pragma unroll
    for (int i = 0; i < CLO_HID; i += 4) {
      float h2v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float4* wr = reinterpret_cast<const float4*>(sw + CLO_W2 + (i + q) * CLO_HID);
        float a = sw[CLO_B2 + i + q];
#pragma unroll
        for (int jj = 0; jj < CLO_HID / 4; ++jj) {
          const float4 w4 = wr[jj];
          a = fmaf(w4.x, h1[4 * jj], a);
          a = fmaf(w4.y, h1[4 * jj + 1], a);
          a = fmaf(w4.z, h1[4 * jj + 2], a);
          a = fmaf(w4.w, h1[4 * jj + 3], a);
        }
        h2v[q] = fmaxf(a, 0.f);
        if (a > 0.f) m2 |= 1u << (i + q);
        z = fmaf(sw[CLO_W3 + i + q], h2v[q], z);
      }
      *reinterpret_cast<float4*>(sH2 + lane * TR_LD + i) = make_float4(h2v[0], h2v[1], h2v[2], h2v[3]);
    }
#pragma unroll
    for (int i = 0; i < CLO_HID; i += 4)
      *reinterpret_cast<float4*>(sH1 + lane * TR_LD + i) = make_float4(h1[i], h1[i + 1], h1[i + 2], h1[i + 3]);
    // softplus output and the weighted squared error
    const float r = z > 20.f ? z : log1pf(expf(z));
    const float sig = 1.f / (1.f + expf(-z));
    const float e = r - tgt;
    const float dz = valid ? 2.f * B.wscale * wt * e * sig : 0.f;
    if (valid) lsum += (double)B.wscale * (double)wt * (double)e * (double)e;
    float da2[CLO_HID];
#pragma unroll
    for (int i = 0; i < CLO_HID; ++i) da2[i] = (m2 >> i & 1u) ? sw[CLO_W3 + i] * dz : 0.f;
#pragma unroll
    for (int i = 0; i < CLO_HID; i += 4)
      *reinterpret_cast<float4*>(sA2 + lane * TR_LD + i) = make_float4(da2[i], da2[i + 1], da2[i + 2], da2[i + 3]);
    // d a1_j = [a1_j > 0] sum_i W2[i][j] d a2_i  (W2 transposed: row j contiguous)
#pragma unroll
    for (int jq = 0; jq < CLO_HID; jq += 4) {
      float d[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int jj = jq + q;
        const float4* wr = reinterpret_cast<const float4*>(sW2T + jj * CLO_HID);
        float a = 0.f;
#pragma unroll
        for (int i4 = 0; i4 < CLO_HID / 4; ++i4) {
          const float4 w4 = wr[i4];
          a = fmaf(w4.x, da2[4 * i4], a);
          a = fmaf(w4.y, da2[4 * i4 + 1], a);
          a = fmaf(w4.z, da2[4 * i4 + 2], a);
          a = fmaf(w4.w, da2[4 * i4 + 3], a);
        }
        d[q] = h1[jj] > 0.f ? a : 0.f;
      }
      *reinterpret_cast<float4*>(sA1 + lane * TR_LD + jq) = make_float4(d[0], d[1], d[2], d[3]);
    }
#pragma unroll
    for (int k = 0; k < CLO_IN; ++k) sX[lane * TR_XLD + k] = xs[k];
    sDZ[lane] = dz;
    __syncwarp();
    // ---- weight gradients, lane = hidden unit ----
    for (int s = 0; s < 32; ++s) {
      const float a2 = sA2[s * TR_LD + lane];
      const float a1 = sA1[s * TR_LD + lane];
      const float dzs = sDZ[s];
      const float4* h = reinterpret_cast<const float4*>(sH1 + s * TR_LD);
#pragma unroll
      for (int q = 0; q < CLO_HID / 4; ++q) {
        const float4 hv = h[q];
        gW2[4 * q] = fmaf(a2, hv.x, gW2[4 * q]);
        gW2[4 * q + 1] = fmaf(a2, hv.y, gW2[4 * q + 1]);
        gW2[4 * q + 2] = fmaf(a2, hv.z, gW2[4 * q + 2]);
        gW2[4 * q + 3] = fmaf(a2, hv.w, gW2[4 * q + 3]);
      }
#pragma unroll
      for (int k = 0; k < CLO_IN; ++k) gW1[k] = fmaf(a1, sX[s * TR_XLD + k], gW1[k]);
      gb1 += a1;
      gb2 += a2;
      gW3 = fmaf(dzs, sH2[s * TR_LD + lane], gW3);
      gb3 += dzs;
    }
    __syncwarp();
  }

  // ---- block reduction in a fixed order ----
  // loss: warp sum (butterfly, the same order on every run), then warps in order
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  __syncthreads();  // every warp is done with its tiles
  float* g = wb;    // this warp's gradient row, CLO_NPARAM floats (fits the tiles)
#pragma unroll
  for (int jj = 0; jj < CLO_HID; ++jj) g[CLO_W2 + lane * CLO_HID + jj] = gW2[jj];
#pragma unroll
  for (int k = 0; k < CLO_IN; ++k) g[CLO_W1 + lane * CLO_IN + k] = gW1[k];
  g[CLO_B1 + lane] = gb1;
  g[CLO_B2 + lane] = gb2;
  g[CLO_W3 + lane] = gW3;
  if (lane == 0) g[CLO_B3] = gb3;
  __shared__ double sl[TR_WARPS];
  if (lane == 0) sl[warp] = lsum;
  __syncthreads();
  const float* g0 = sW2T + CLO_HID * CLO_HID;
  for (int k = threadIdx.x; k < CLO_NPARAM; k += TR_THREADS) {
    float acc = g0[k];
#pragma unroll
    for (int w = 1; w < TR_WARPS; ++w) acc += g0[w * TR_WARP_FLOATS + k];
    part[(size_t)blockIdx.x * CLO_NPARAM + k] = acc;
  }
  if (threadIdx.x == 0) {
    double l = 0.0;
    for (int w = 0; w < TR_WARPS; ++w) l += sl[w];
    loss_part[blockIdx.x] = l;
  }
}

struct AdamArgs {
  float lr, b1, b2, eps, wd;
  float bc1, bc2;   // 1 - beta^t
  int apply;        // 0: only reduce the gradient
};

// Sums the block partials (fixed order), then optionally one Adam step of
// the fp32 master parameters; writes the network the kernels use (weights
// rounded to bf16).  Thread 0 adds the batch loss to loss_acc.
__global__ void k_adam(const float* __restrict__ part, int nblk, const double* __restrict__ loss_part,
                       double* __restrict__ loss_acc, float* __restrict__ grad,
                       float* __restrict__ theta, float* __restrict__ m, float* __restrict__ v,
                       float* __restrict__ net, AdamArgs A) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0) {
    double l = 0.0;
    for (int b = 0; b < nblk; ++b) l += loss_part[b];
    *loss_acc += l;
  }
  if (k >= CLO_NPARAM) return;
  float gk = 0.f;
  for (int b = 0; b < nblk; ++b) gk += part[(size_t)b * CLO_NPARAM + k];
  grad[k] = gk;
  if (!A.apply) return;
  const float mk = A.b1 * m[k] + (1.f - A.b1) * gk;
  const float vk = A.b2 * v[k] + (1.f - A.b2) * gk * gk;
  m[k] = mk;
  v[k] = vk;
  float th = theta[k];
  const bool wgt = clo_is_weight(k);
  if (wgt && A.wd > 0.f) th -= A.lr * A.wd * th;
  th -= A.lr * (mk / A.bc1) / (sqrtf(vk / A.bc2) + A.eps);
  theta[k] = th;
  net[k] = wgt ? __bfloat162float(__float2bfloat16_rn(th)) : th;
}

__global__ void k_wsum(const float* __restrict__ w, int64_t n, double* __restrict__ out) {
  __shared__ double s[256];
  double a = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a += w[i];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

}  // namespace
}  // namespace lbm

using namespace lbm;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct lbm_trainer {
  lbm_adam opt{};
  cudaStream_t stream = nullptr;
  float* theta = nullptr;   // fp32 master parameters [CLO_NPARAM]
  float* m = nullptr;
  float* v = nullptr;
  float* grad = nullptr;    // last reduced gradient
  float* net = nullptr;     // network the kernels use [CLO_FLOATS]
  float* part = nullptr;    // [TR_MAX_BLOCKS][CLO_NPARAM]
  double* loss_part = nullptr;
  double* loss_acc = nullptr;
  double* wpart = nullptr;  // [TR_MAX_BLOCKS]
  int64_t t = 0;            // Adam steps taken
  std::string err = "no error";
};

namespace {

thread_local std::string g_clo_err = "no error";

int tfail(lbm_trainer* t, int code, const std::string& msg) {
  if (t) t->err = msg;
  g_clo_err = msg;
  set_thread_error(msg.c_str());
  return code;
}

int tcuda(lbm_trainer* t, cudaError_t e, const char* what) {
  const int code = e == cudaErrorMemoryAllocation ? LBM_ERR_OUT_OF_MEMORY
                   : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? LBM_ERR_NO_DEVICE
                                                                                  : LBM_ERR_CUDA;
  return tfail(t, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define TCK(t, expr, what)                              \
  do {                                                  \
    cudaError_t e_ = (expr);                            \
    if (e_ != cudaSuccess) return tcuda(t, e_, what);   \
  } while (0)

bool grad_kernel_ready(cudaError_t* e) {
  static cudaError_t once = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)TR_SMEM);
  *e = once;
  return once == cudaSuccess;
}

int grid_for(int64_t nb) {
  const int64_t groups = (nb + 31) / 32;
  const int64_t blocks = (groups + TR_WARPS - 1) / TR_WARPS;
  return (int)(blocks < 1 ? 1 : blocks > TR_MAX_BLOCKS ? TR_MAX_BLOCKS : blocks);
}

int launch_grad(lbm_trainer* t, const Batch& B, int* nblk) {
  cudaError_t e;
  if (!grad_kernel_ready(&e)) return tcuda(t, e, "closure grad kernel attribute");
  const int g = grid_for(B.nb);
  k_mlp_grad<<<g, TR_THREADS, TR_SMEM, t->stream>>>(t->net, B, t->part, t->loss_part);
  TCK(t, cudaGetLastError(), "closure grad kernel");
  *nblk = g;
  return LBM_OK;
}

int launch_adam(lbm_trainer* t, int nblk, bool apply) {
  AdamArgs A{};
  A.lr = t->opt.lr;
  A.b1 = t->opt.beta1;
  A.b2 = t->opt.beta2;
  A.eps = t->opt.eps;
  A.wd = t->opt.weight_decay;
  A.apply = apply ? 1 : 0;
  if (apply) {
    t->t += 1;
    A.bc1 = (float)(1.0 - std::pow((double)A.b1, (double)t->t));
    A.bc2 = (float)(1.0 - std::pow((double)A.b2, (double)t->t));
  } else {
    A.bc1 = A.bc2 = 1.f;
  }
  k_adam<<<(CLO_NPARAM + 255) / 256, 256, 0, t->stream>>>(t->part, nblk, t->loss_part, t->loss_acc,
                                                          t->grad, t->theta, t->m, t->v, t->net, A);
  TCK(t, cudaGetLastError(), "closure adam kernel");
  return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_round_bf16(const float* in, float* out, size_t n) {
  if ((!in || !out) && n) return LBM_ERR_INVALID_ARG;
  for (size_t i = 0; i < n; ++i) out[i] = round_bf16(in[i]);
  return LBM_OK;
}

int lbm_box_filter(const float* d_rho, const float* d_u, int32_t nx, int32_t ny, int32_t nz,
                   int32_t factor, float* d_out, void* stream) {
  if (!d_rho || !d_u || !d_out) return tfail(nullptr, LBM_ERR_INVALID_ARG, "box filter: NULL pointer");
  if (factor < 1 || nx < factor || ny < factor || nz < factor || nx % factor || ny % factor || nz % factor)
    return tfail(nullptr, LBM_ERR_INVALID_ARG, "box filter: factor must divide nx, ny and nz");
  const size_t nc = (size_t)(nx / factor) * (ny / factor) * (nz / factor);
  k_box_filter<<<(unsigned)((nc + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_rho, d_u, nx, ny, nz, factor, d_out);
  TCK(nullptr, cudaGetLastError(), "box filter kernel");
  return LBM_OK;
}

int lbm_closure_samples(const float* d_filt, int32_t nx, int32_t ny, int32_t nz, float tau, float cs0,
                        uint64_t seed, int64_t n_samples, float* d_x, float* d_target, float* d_weight,
                        void* stream) {
  if (!d_filt || !d_x || !d_target || !d_weight)
    return tfail(nullptr, LBM_ERR_INVALID_ARG, "closure samples: NULL pointer");
  if (nx < 3 || ny < 3 || nz < 3) return tfail(nullptr, LBM_ERR_INVALID_ARG, "closure samples: grid below 3^3");
  if (!(cs0 > 0.f) || !(tau > 0.5f)) return tfail(nullptr, LBM_ERR_INVALID_ARG, "closure samples: need cs0 > 0, tau > 1/2");
  const int64_t n = (int64_t)nx * ny * nz;
  if (n_samples < 0 || (seed == 0 && n_samples > n))
    return tfail(nullptr, LBM_ERR_INVALID_ARG, "closure samples: bad sample count");
  if (n_samples == 0) return LBM_OK;
  k_samples<<<(unsigned)((n_samples + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_filt, nx, ny, nz, tau, cs0, seed, n_samples, d_x, d_target, d_weight);
  TCK(nullptr, cudaGetLastError(), "closure samples kernel");
  return LBM_OK;
}

int lbm_closure_predict(const float* net, const float* d_x, int64_t n, float* d_r, void* stream) {
  if (!net || !d_x || !d_r) return tfail(nullptr, LBM_ERR_INVALID_ARG, "closure predict: NULL pointer");
  if (n <= 0) return n == 0 ? LBM_OK : tfail(nullptr, LBM_ERR_INVALID_ARG, "closure predict: n < 0");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float h[CLO_FLOATS];
  for (int k = 0; k < CLO_FLOATS; ++k) h[k] = clo_is_weight(k) ? round_bf16(net[k]) : net[k];
  float* d_net = nullptr;
  TCK(nullptr, cudaMallocAsync(reinterpret_cast<void**>(&d_net), sizeof(h), s), "closure predict alloc");
  cudaError_t e = cudaMemcpyAsync(d_net, h, sizeof(h), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    k_predict<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_net, d_x, n, d_r);
    e = cudaGetLastError();
  }
  cudaError_t e2 = cudaFreeAsync(d_net, s);
  cudaError_t e3 = cudaStreamSynchronize(s);  // h is a stack buffer
  if (e != cudaSuccess) return tcuda(nullptr, e, "closure predict");
  if (e2 != cudaSuccess) return tcuda(nullptr, e2, "closure predict free");
  TCK(nullptr, e3, "closure predict sync");
  return LBM_OK;
}

int lbm_adam_default(lbm_adam* a) {
  if (!a) return LBM_ERR_INVALID_ARG;
  *a = lbm_adam{};
  a->struct_size = sizeof(lbm_adam);
  a->lr = 1e-3f;
  a->beta1 = 0.9f;
  a->beta2 = 0.999f;
  a->eps = 1e-8f;
  a->weight_decay = 0.f;
  return LBM_OK;
}

int lbm_trainer_create(const float* net, const lbm_adam* opt, lbm_trainer** out) {
  if (!net || !out) return tfail(nullptr, LBM_ERR_INVALID_ARG, "trainer: NULL pointer");
  *out = nullptr;
  lbm_adam o;
  lbm_adam_default(&o);
  if (opt) {
    if (opt->struct_size != sizeof(lbm_adam)) return tfail(nullptr, LBM_ERR_INVALID_ARG, "lbm_adam struct_size");
    o = *opt;
  }
  if (!(o.lr > 0.f) || !(o.beta1 >= 0.f && o.beta1 < 1.f) || !(o.beta2 >= 0.f && o.beta2 < 1.f) ||
      !(o.eps > 0.f) || !(o.weight_decay >= 0.f))
    return tfail(nullptr, LBM_ERR_INVALID_ARG, "trainer: bad Adam hyper-parameters");
  for (int k = 0; k < CLO_FLOATS; ++k)
    if (!std::isfinite(net[k])) return tfail(nullptr, LBM_ERR_INVALID_ARG, "trainer: non-finite network value");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return tfail(nullptr, LBM_ERR_NO_DEVICE, "trainer: no CUDA device");
  lbm_trainer* t = new (std::nothrow) lbm_trainer();
  if (!t) return tfail(nullptr, LBM_ERR_OUT_OF_MEMORY, "trainer: host allocation");
  t->opt = o;
  struct A { void** p; size_t bytes; } allocs[] = {
      {reinterpret_cast<void**>(&t->theta), CLO_NPARAM * 4}, {reinterpret_cast<void**>(&t->m), CLO_NPARAM * 4},
      {reinterpret_cast<void**>(&t->v), CLO_NPARAM * 4},     {reinterpret_cast<void**>(&t->grad), CLO_NPARAM * 4},
      {reinterpret_cast<void**>(&t->net), CLO_FLOATS * 4},
      {reinterpret_cast<void**>(&t->part), (size_t)TR_MAX_BLOCKS * CLO_NPARAM * 4},
      {reinterpret_cast<void**>(&t->loss_part), TR_MAX_BLOCKS * 8},
      {reinterpret_cast<void**>(&t->loss_acc), 8}, {reinterpret_cast<void**>(&t->wpart), TR_MAX_BLOCKS * 8}};
  for (auto& a : allocs) {
    cudaError_t e = cudaMalloc(a.p, a.bytes);
    if (e != cudaSuccess) {
      const int rc = tcuda(nullptr, e, "trainer: cudaMalloc");
      lbm_trainer_destroy(t);
      return rc;
    }
  }
  std::vector<float> h(CLO_FLOATS);
  for (int k = 0; k < CLO_FLOATS; ++k) h[k] = clo_is_weight(k) ? round_bf16(net[k]) : net[k];
  cudaError_t e = cudaMemcpy(t->theta, net, CLO_NPARAM * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->net, h.data(), CLO_FLOATS * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(t->m, 0, CLO_NPARAM * 4);
  if (e == cudaSuccess) e = cudaMemset(t->v, 0, CLO_NPARAM * 4);
  if (e == cudaSuccess) e = cudaMemset(t->grad, 0, CLO_NPARAM * 4);
  if (e != cudaSuccess) {
    const int rc = tcuda(nullptr, e, "trainer: initial upload");
    lbm_trainer_destroy(t);
    return rc;
  }
  *out = t;
  return LBM_OK;
}

int lbm_trainer_destroy(lbm_trainer* t) {
  if (!t) return LBM_OK;
  void* ptrs[] = {t->theta, t->m, t->v, t->grad, t->net, t->part, t->loss_part, t->loss_acc, t->wpart};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete t;
  return LBM_OK;
}

int lbm_trainer_set_stream(lbm_trainer* t, void* stream) {
  if (!t) return tfail(nullptr, LBM_ERR_INVALID_ARG, "trainer is NULL");
  TCK(t, cudaStreamSynchronize(t->stream), "trainer set_stream sync");
  t->stream = static_cast<cudaStream_t>(stream);
  return LBM_OK;
}

int lbm_trainer_grad(lbm_trainer* t, const float* d_x, const float* d_target, const float* d_weight,
                     int64_t n, float wscale, float* grad, double* loss) {
  if (!t) return tfail(nullptr, LBM_ERR_INVALID_ARG, "trainer is NULL");
  if (!d_x || !d_target || !d_weight || n <= 0) return tfail(t, LBM_ERR_INVALID_ARG, "trainer grad: bad batch");
  Batch B{d_x, d_target, d_weight, n, 0, n, 1, 0, wscale};
  int nblk = 0;
  TCK(t, cudaMemsetAsync(t->loss_acc, 0, 8, t->stream), "trainer grad: reset loss");
  if (int rc = launch_grad(t, B, &nblk)) return rc;
  if (int rc = launch_adam(t, nblk, false)) return rc;
  if (grad) TCK(t, cudaMemcpyAsync(grad, t->grad, CLO_NPARAM * 4, cudaMemcpyDeviceToHost, t->stream), "trainer grad: read");
  double l = 0.0;
  TCK(t, cudaMemcpyAsync(&l, t->loss_acc, 8, cudaMemcpyDeviceToHost, t->stream), "trainer grad: read loss");
  TCK(t, cudaStreamSynchronize(t->stream), "trainer grad: sync");
  if (loss) *loss = l;
  return LBM_OK;
}

int lbm_trainer_adam_step(lbm_trainer* t) {
  if (!t) return tfail(nullptr, LBM_ERR_INVALID_ARG, "trainer is NULL");
  // the reduced gradient of the last lbm_trainer_grad becomes the single
  // partial row that the Adam kernel sums
  TCK(t, cudaMemcpyAsync(t->part, t->grad, CLO_NPARAM * 4, cudaMemcpyDeviceToDevice, t->stream), "trainer adam: stage");
  TCK(t, cudaMemsetAsync(t->loss_part, 0, 8, t->stream), "trainer adam: loss");
  if (int rc = launch_adam(t, 1, true)) return rc;
  return LBM_OK;
}

int lbm_trainer_fit(lbm_trainer* t, const float* d_x, const float* d_target, const float* d_weight,
                    int64_t n, int32_t batch, int32_t epochs, uint64_t seed, double* epoch_loss) {
  if (!t) return tfail(nullptr, LBM_ERR_INVALID_ARG, "trainer is NULL");
  if (!d_x || !d_target || !d_weight || n <= 0 || batch <= 0 || epochs < 0)
    return tfail(t, LBM_ERR_INVALID_ARG, "trainer fit: bad arguments");
  // mean weight of the dataset
  const int wb = (int)std::min<int64_t>(TR_MAX_BLOCKS, (n + 255) / 256);
  k_wsum<<<wb, 256, 0, t->stream>>>(d_weight, n, t->wpart);
  TCK(t, cudaGetLastError(), "trainer fit: weight sum");
  std::vector<double> wp(wb);
  TCK(t, cudaMemcpyAsync(wp.data(), t->wpart, wb * 8, cudaMemcpyDeviceToHost, t->stream), "trainer fit: read weight sum");
  TCK(t, cudaStreamSynchronize(t->stream), "trainer fit: sync");
  double wsum = 0.0;
  for (double v : wp) wsum += v;
  if (!(wsum > 0.0) || !std::isfinite(wsum)) return tfail(t, LBM_ERR_INVALID_ARG, "trainer fit: weights sum to <= 0");
  const double wmean = wsum / (double)n;
  uint64_t rs = seed * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull;
  auto next = [&rs]() {  // splitmix64
    uint64_t z = (rs += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  };
  auto gcd = [](uint64_t a, uint64_t b) {
    while (b) { const uint64_t r = a % b; a = b; b = r; }
    return a;
  };
  for (int ep = 0; ep < epochs; ++ep) {
    uint64_t a = 1, c = 0;
    if (n > 1) {
      do { a = 1 + next() % (uint64_t)(n - 1); } while (gcd(a, (uint64_t)n) != 1);
      c = next() % (uint64_t)n;
    }
    TCK(t, cudaMemsetAsync(t->loss_acc, 0, 8, t->stream), "trainer fit: reset loss");
    int64_t nbatches = 0;
    for (int64_t s = 0; s < n; s += batch) {
      const int64_t nb = std::min<int64_t>(batch, n - s);
      Batch B{d_x, d_target, d_weight, n, s, nb, a, c, (float)(1.0 / (wmean * (double)nb))};
      int nblk = 0;
      if (int rc = launch_grad(t, B, &nblk)) return rc;
      if (int rc = launch_adam(t, nblk, true)) return rc;
      ++nbatches;
    }
    if (epoch_loss) {
      double l = 0.0;
      TCK(t, cudaMemcpyAsync(&l, t->loss_acc, 8, cudaMemcpyDeviceToHost, t->stream), "trainer fit: read loss");
      TCK(t, cudaStreamSynchronize(t->stream), "trainer fit: sync");
      epoch_loss[ep] = l / (double)nbatches;
    }
  }
  TCK(t, cudaStreamSynchronize(t->stream), "trainer fit: sync");
  return LBM_OK;
}

int lbm_trainer_get_net(lbm_trainer* t, float* net) {
  if (!t || !net) return tfail(t, LBM_ERR_INVALID_ARG, "trainer get_net: NULL pointer");
  TCK(t, cudaMemcpyAsync(net, t->net, CLO_FLOATS * 4, cudaMemcpyDeviceToHost, t->stream), "trainer get_net");
  TCK(t, cudaStreamSynchronize(t->stream), "trainer get_net: sync");
  return LBM_OK;
}

const char* lbm_trainer_last_error(lbm_trainer* t) { return t ? t->err.c_str() : g_clo_err.c_str(); }

}  // extern "C"
