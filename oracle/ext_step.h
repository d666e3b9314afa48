// ExtStep node update, shared by the CPU oracle (lbm_oracle.cpp) and its FP64
// GPU copy (gpu_oracle.cu).  TEST INFRASTRUCTURE ONLY.
//
// Textbook stream-collide on plain populations f: pull streaming with
// periodic wrap or half-way bounce-back, momentum-corrected moving walls
// (f_i = f*_opp(i) + 6 w_i rho_w (c_i . u_w), rho_w = 1; a link leaving the
// box through a z face takes that face's velocity, then y, then x), BGK or
// TRT, Smagorinsky (Hou et al. 1996), optionally with the learned closure
// (Cs^2 scaled per node by a network), and Guo forcing with F = rho g.  Both
// builds round every operation on its own (-ffp-contract=off / -fmad=false)
// in the same order, so CPU and GPU FP64 results agree bit for bit.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>

#ifdef __CUDACC__
#define OX_HD __host__ __device__
#else
#define OX_HD
#endif

namespace ox {

// volumetric-grid/lattice-boltzmann/shaders/lattice_constants.glsl:23-43, 55-75
#define OX_C_TABLE                                                                         \
  {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},   {0, -1, 0},  {0, 0, 1},  {0, 0, -1},   \
   {1, 1, 0},  {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1},   {1, 0, -1}, {-1, 0, 1},   \
   {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1},  {0, -1, -1}}
#define OX_OPP_TABLE {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15}

#ifdef __CUDACC__
__constant__ int d_C[19][3] = OX_C_TABLE;
__constant__ int d_OPP[19] = OX_OPP_TABLE;
#endif
static const int h_C[19][3] = OX_C_TABLE;
static const int h_OPP[19] = OX_OPP_TABLE;

OX_HD inline int cc(int i, int a) {
#ifdef __CUDA_ARCH__
  return d_C[i][a];
#else
  return h_C[i][a];
#endif
}
OX_HD inline int opp(int i) {
#ifdef __CUDA_ARCH__
  return d_OPP[i];
#else
  return h_OPP[i];
#endif
}

template <class T> OX_HD inline T weight(int i) {
  return i == 0 ? T(1) / T(3) : (i <= 6 ? T(1) / T(18) : T(1) / T(36));
}

// feq_i, canonical form (shaders/lattice_constants.glsl:86-93).
template <class T> OX_HD inline T feq_i(int i, T rho, T ux, T uy, T uz) {
  const T cx = T(cc(i, 0)), cy = T(cc(i, 1)), cz = T(cc(i, 2));
  const T cdotu = cx * ux + cy * uy + cz * uz;
  const T udotu = ux * ux + uy * uy + uz * uz;
  return weight<T>(i) * rho * (T(1) + T(3) * cdotu + T(4.5) * cdotu * cdotu - T(1.5) * udotu);
}

// Learned-closure network, layout of include/lbm_closure.h: W1[32][9] b1[32]
// W2[32][32] b2[32] W3[32] b3, input mean[9], input inverse scale[9].
constexpr int NET_FLOATS = 1427;

struct ExtP {
  int nx, ny, nz;
  int periodic[3];
  double tau;
  int collision;  // 0 BGK, 1 TRT
  double trt_magic;
  double smag_cs;
  double accel[3];
  double wall[6][3];
  int open[2];    // open x faces: 0 none, 1 velocity (u = wall[side]), 2 pressure
  double open_rho[2];
  int has_net;    // learned closure: Cs^2 = smag_cs^2 * r(Pi, rho)
  double net[NET_FLOATS];
};

// ip: nx ny nz px py pz collision open[2];
// dp: tau trt_magic smag_cs accel[3] wall[18] open_rho[2] has_net
//     [net[NET_FLOATS] if has_net]
inline ExtP make_ext(const int* ip, const double* dp) {
  ExtP p;
  p.nx = ip[0]; p.ny = ip[1]; p.nz = ip[2];
  p.periodic[0] = ip[3]; p.periodic[1] = ip[4]; p.periodic[2] = ip[5];
  p.collision = ip[6];
  p.open[0] = ip[7]; p.open[1] = ip[8];
  p.tau = dp[0]; p.trt_magic = dp[1]; p.smag_cs = dp[2];
  for (int a = 0; a < 3; ++a) p.accel[a] = dp[3 + a];
  for (int f = 0; f < 6; ++f)
    for (int a = 0; a < 3; ++a) p.wall[f][a] = dp[6 + 3 * f + a];
  p.open_rho[0] = dp[24]; p.open_rho[1] = dp[25];
  p.has_net = dp[26] != 0.0;
  for (int k = 0; k < NET_FLOATS; ++k) p.net[k] = p.has_net ? dp[27 + k] : 0.0;
  return p;
}

// Network output r for the flux P (xx yy zz xy xz yz) and density rho.
template <class T>
OX_HD inline T ext_closure_r(const ExtP& p, const T P[6], T rho) {
  const double* w = p.net;
  const T n = std::sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2] +
                        T(2) * (P[3] * P[3] + P[4] * P[4] + P[5] * P[5])) + T(1e-30);
  T q[6];
  for (int k = 0; k < 6; ++k) q[k] = P[k] / n;
  // tr(M^3) with M = [[xx,xy,xz],[xy,yy,yz],[xz,yz,zz]] by explicit products
  const T M[3][3] = {{q[0], q[3], q[4]}, {q[3], q[1], q[5]}, {q[4], q[5], q[2]}};
  T t3 = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) t3 += M[i][j] * M[j][k] * M[k][i];
  T x[9] = {q[0], q[1], q[2], q[3], q[4], q[5], std::log(n), t3, rho - T(1)};
  for (int j = 0; j < 9; ++j) x[j] = (x[j] - T(w[1409 + j])) * T(w[1418 + j]);
  T h1[32];
  for (int i = 0; i < 32; ++i) {
    T a = T(w[288 + i]);
    for (int j = 0; j < 9; ++j) a += T(w[i * 9 + j]) * x[j];
    h1[i] = a > T(0) ? a : T(0);
  }
  T z = T(w[1408]);
  for (int i = 0; i < 32; ++i) {
    T a = T(w[1344 + i]);
    for (int j = 0; j < 32; ++j) a += T(w[320 + i * 32 + j]) * h1[j];
    z += T(w[1376 + i]) * (a > T(0) ? a : T(0));
  }
  return z > T(20) ? z : std::log(T(1) + std::exp(z));
}

OX_HD inline size_t nidx(int nx, int ny, int x, int y, int z) {
  return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * (size_t)z);
}

// Population arriving at (x,y,z) in direction i: pulled from the node at
// -c_i; if that node is solid or outside a non-periodic face, the half-way
// bounce-back value f*_opp(i) of this node plus the moving-wall term.
template <class T>
OX_HD inline T incoming(const ExtP& p, const uint8_t* mask, const T* f, int x, int y, int z, int i,
                        size_t N) {
  int xs = x - cc(i, 0), ys = y - cc(i, 1), zs = z - cc(i, 2);
  int face = -1;
  bool out = false;
  if (zs < 0 || zs >= p.nz) { if (p.periodic[2]) zs = (zs + p.nz) % p.nz; else { out = true; face = zs < 0 ? 4 : 5; } }
  if (ys < 0 || ys >= p.ny) { if (p.periodic[1]) ys = (ys + p.ny) % p.ny; else { out = true; if (face < 0) face = ys < 0 ? 2 : 3; } }
  if (xs < 0 || xs >= p.nx) { if (p.periodic[0]) xs = (xs + p.nx) % p.nx; else { out = true; if (face < 0) face = xs < 0 ? 0 : 1; } }
  const size_t n = nidx(p.nx, p.ny, x, y, z);
  if (!out && mask[nidx(p.nx, p.ny, xs, ys, zs)] != 1) return f[i * N + nidx(p.nx, p.ny, xs, ys, zs)];
  T v = f[opp(i) * N + n];
  if (face >= 0) {
    const double cu = cc(i, 0) * p.wall[face][0] + cc(i, 1) * p.wall[face][1] + cc(i, 2) * p.wall[face][2];
    v += T(6.0 * weight<double>(i) * cu);
  }
  return v;
}

// Open x face: the populations entering through it (c_x = +1 at x = 0,
// -1 at x = nx-1) rebuilt from the streamed ones by the non-equilibrium
// bounce-back of Zou & He (1997), D3Q19 form (Hecht & Harting 2010):
//   rho (1 - s u_x) = sum_{c_x=0} f + 2 sum_{c_x=-s} f,
//   f_i = f_opp(i) + 6 w_i rho (c_i.u) - c_iy N_y - c_iz N_z,
//   N_t = 1/2 sum_{c_x=0} f c_t - rho u_t / 3.
// Velocity faces know u (wall[side]) and solve for rho; pressure faces know
// rho with u_y = u_z = 0 and solve for u_x.  Written from the definitions,
// independently of the kernels' shifted-storage form.
template <class T>
OX_HD inline void open_face(const ExtP& p, T* v, int x) {
  int side;
  if (x == 0 && p.open[0]) side = 0;
  else if (x == p.nx - 1 && p.open[1]) side = 1;
  else return;
  const int s = side == 0 ? 1 : -1;
  T s0 = 0, sk = 0, my = 0, mz = 0;
  for (int i = 0; i < 19; ++i) {
    if (cc(i, 0) == 0) {
      s0 += v[i];
      my += T(cc(i, 1)) * v[i];
      mz += T(cc(i, 2)) * v[i];
    } else if (cc(i, 0) == -s) {
      sk += v[i];
    }
  }
  T rho, u[3];
  if (p.open[side] == 1) {
    for (int a = 0; a < 3; ++a) u[a] = T(p.wall[side][a]);
    rho = (s0 + T(2) * sk) / (T(1) - T(s) * u[0]);
  } else {
    rho = T(p.open_rho[side]);
    u[0] = T(s) * (T(1) - (s0 + T(2) * sk) / rho);
    u[1] = u[2] = T(0);
  }
  const T Ny = my / T(2) - rho * u[1] / T(3), Nz = mz / T(2) - rho * u[2] / T(3);
  for (int i = 0; i < 19; ++i) {
    if (cc(i, 0) != s) continue;
    const T cu = T(cc(i, 0)) * u[0] + T(cc(i, 1)) * u[1] + T(cc(i, 2)) * u[2];
    v[i] = v[opp(i)] + T(6) * weight<T>(i) * rho * cu - T(cc(i, 1)) * Ny - T(cc(i, 2)) * Nz;
  }
}

// Moments (u with the Guo half-force shift) and the collision, in place.
template <class T>
OX_HD inline void ext_collide_node(const ExtP& p, T* v, T& rho_o, T& ux_o, T& uy_o, T& uz_o) {
  T rho = 0, jx = 0, jy = 0, jz = 0;
  for (int i = 0; i < 19; ++i) {
    rho += v[i];
    jx += v[i] * T(cc(i, 0));
    jy += v[i] * T(cc(i, 1));
    jz += v[i] * T(cc(i, 2));
  }
  const T ax = T(p.accel[0]), ay = T(p.accel[1]), az = T(p.accel[2]);
  const T ux = jx / rho + ax / T(2), uy = jy / rho + ay / T(2), uz = jz / rho + az / T(2);
  rho_o = rho; ux_o = ux; uy_o = uy; uz_o = uz;
  const T Fx = rho * ax, Fy = rho * ay, Fz = rho * az;
  T feq[19];
  for (int i = 0; i < 19; ++i) feq[i] = feq_i<T>(i, rho, ux, uy, uz);
  T tau = T(p.tau);
  if (p.smag_cs > 0) {
    T P[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int i = 0; i < 19; ++i)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) P[a][b] += T(cc(i, a) * cc(i, b)) * (v[i] - feq[i]);
    T q = 0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) q += P[a][b] * P[a][b];
    T cs2 = T(p.smag_cs * p.smag_cs);
    if (p.has_net) {
      const T Pv[6] = {P[0][0], P[1][1], P[2][2], P[0][1], P[0][2], P[1][2]};
      cs2 = cs2 * ext_closure_r<T>(p, Pv, rho);
    }
    tau = (tau + std::sqrt(tau * tau + T(18) * std::sqrt(T(2)) * cs2 * std::sqrt(q) / rho)) / T(2);
  }
  const T om = T(1) / tau;
  T src[19];
  for (int i = 0; i < 19; ++i) {
    const T cu = T(cc(i, 0)) * ux + T(cc(i, 1)) * uy + T(cc(i, 2)) * uz;
    const T cF = T(cc(i, 0)) * Fx + T(cc(i, 1)) * Fy + T(cc(i, 2)) * Fz;
    const T uF = ux * Fx + uy * Fy + uz * Fz;
    src[i] = weight<T>(i) * (T(3) * (cF - uF) + T(9) * cu * cF);  // Guo term without prefactor
  }
  if (p.collision == 0) {
    for (int i = 0; i < 19; ++i) v[i] = v[i] + om * (feq[i] - v[i]) + (T(1) - om / T(2)) * src[i];
  } else {
    const T om_m = T(1) / (T(p.trt_magic) / (tau - T(0.5)) + T(0.5));
    T out[19];
    for (int i = 0; i < 19; ++i) {
      const int j = opp(i);
      const T fp = (v[i] + v[j]) / T(2), fm = (v[i] - v[j]) / T(2);
      const T ep = (feq[i] + feq[j]) / T(2), em = (feq[i] - feq[j]) / T(2);
      const T sp = (src[i] + src[j]) / T(2), sm = (src[i] - src[j]) / T(2);
      out[i] = v[i] - om * (fp - ep) - om_m * (fm - em) + (T(1) - om / T(2)) * sp +
               (T(1) - om_m / T(2)) * sm;
    }
    for (int i = 0; i < 19; ++i) v[i] = out[i];
  }
}

}  // namespace ox
