"""FP64 numpy restatement of the learned-closure pipeline.  TEST
INFRASTRUCTURE ONLY: tests use it as the checker of the CUDA kernels; the
product never imports it.

The closure has no counterpart in the reference (its only collision is the
plain BGK of volumetric-grid/lattice-boltzmann/shaders/collide.comp.glsl:
39-61), so this is a restatement of the definitions the C ABI states
(include/lbm_closure.h), written independently of the kernels:
  * box filter: Favre averages over factor^3 blocks;
  * training samples: central-difference strain of the filtered velocity,
    target r* = -tau^d:S / (cs0^2 |S|^3), weight |S|^3, features of
    Pi = -(2/3) rho tau_s S, tau_s = tau + 3 cs0^2 |S|;
  * the MLP 9 -> 32 ReLU -> 32 ReLU -> 1 softplus, its loss
    wscale * sum w (r - t)^2, the gradient by reverse-mode differentiation
    (checked against central finite differences in the CPU tests), Adam.
The parameter layout is that of include/lbm_closure.h.
"""
from __future__ import annotations

import numpy as np

NIN, NH = 9, 32
W1, B1 = 0, 288
W2, B2 = 320, 1344
W3, B3 = 1376, 1408
NPARAM = 1409
MEAN, ISCALE = 1409, 1418
NFLOATS = 1427


def is_weight(k: np.ndarray) -> np.ndarray:
    return ((k >= W1) & (k < B1)) | ((k >= W2) & (k < B2)) | ((k >= W3) & (k < B3))


def round_bf16(a) -> np.ndarray:
    """Round to the nearest bfloat16 value, ties to even (finite inputs)."""
    x = np.ascontiguousarray(a, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def kernel_net(net) -> np.ndarray:
    """The network the kernels use: weights rounded to bf16."""
    w = np.array(net, np.float32).copy()
    k = np.arange(NFLOATS)
    m = is_weight(k)
    w[m] = round_bf16(w[m])
    return w


def unpack(net):
    w = np.asarray(net, np.float64)
    return (w[W1:B1].reshape(NH, NIN), w[B1:W2], w[W2:B2].reshape(NH, NH), w[B2:W3],
            w[W3:B3], w[B3], w[MEAN:ISCALE], w[ISCALE:NFLOATS])


def random_net(seed: int, mean=None, iscale=None) -> np.ndarray:
    """He-initialised network (float32 layout), zero biases but b3."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NFLOATS, np.float32)
    w[W1:B1] = rng.standard_normal(NH * NIN) * np.sqrt(2.0 / NIN)
    w[W2:B2] = rng.standard_normal(NH * NH) * np.sqrt(2.0 / NH)
    w[W3:B3] = rng.standard_normal(NH) * np.sqrt(1.0 / NH)
    w[B1:W2] = 0.05 * rng.standard_normal(NH)
    w[B2:W3] = 0.05 * rng.standard_normal(NH)
    w[B3] = np.log(np.e - 1.0)  # softplus(b3) = 1
    w[MEAN:ISCALE] = 0.0 if mean is None else mean
    w[ISCALE:NFLOATS] = 1.0 if iscale is None else iscale
    return w


def unit_net(mean=None, iscale=None) -> np.ndarray:
    """r = softplus(b3) = 1 everywhere: plain Smagorinsky."""
    w = np.zeros(NFLOATS, np.float32)
    w[B3] = np.log(np.e - 1.0)
    w[MEAN:ISCALE] = 0.0 if mean is None else mean
    w[ISCALE:NFLOATS] = 1.0 if iscale is None else iscale
    return w


def features(P: np.ndarray, rho: np.ndarray) -> np.ndarray:
    """P [..., 6] (xx yy zz xy xz yz), rho [...] -> x [..., 9]."""
    P = np.asarray(P, np.float64)
    n = np.sqrt(P[..., 0] ** 2 + P[..., 1] ** 2 + P[..., 2] ** 2 +
                2 * (P[..., 3] ** 2 + P[..., 4] ** 2 + P[..., 5] ** 2)) + 1e-30
    p = P / n[..., None]
    xx, yy, zz, xy, xz, yz = (p[..., k] for k in range(6))
    # tr(p^3) via the explicit matrix product
    M = np.stack([np.stack([xx, xy, xz], -1), np.stack([xy, yy, yz], -1), np.stack([xz, yz, zz], -1)], -2)
    t3 = np.einsum("...ij,...jk,...ki->...", M, M, M)
    return np.concatenate([p, np.log(n)[..., None], t3[..., None], (np.asarray(rho, np.float64) - 1)[..., None]], -1)


def softplus(z):
    return np.where(z > 20, z, np.log1p(np.exp(np.minimum(z, 20))))


def forward(net, X):
    """r and the activations for the backward pass; X [n, 9] raw inputs."""
    w1, b1, w2, b2, w3, b3, mean, isc = unpack(net)
    xs = (np.asarray(X, np.float64) - mean) * isc
    a1 = xs @ w1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w2.T + b2
    h2 = np.maximum(a2, 0)
    z = h2 @ w3 + b3
    return softplus(z), (xs, a1, h1, a2, h2, z)


def loss_and_grad(net, X, t, w, wscale):
    """L = wscale * sum w (r - t)^2 and dL/dparams (float64 [NPARAM])."""
    w1, b1, w2, b2, w3, b3, mean, isc = unpack(net)
    r, (xs, a1, h1, a2, h2, z) = forward(net, X)
    t = np.asarray(t, np.float64)
    w = np.asarray(w, np.float64)
    e = r - t
    L = wscale * np.sum(w * e * e)
    dz = 2 * wscale * w * e / (1 + np.exp(-z))
    g = np.zeros(NPARAM)
    g[W3:B3] = h2.T @ dz
    g[B3] = dz.sum()
    da2 = (dz[:, None] * w3[None, :]) * (a2 > 0)
    g[W2:B2] = (da2.T @ h1).reshape(-1)
    g[B2:W3] = da2.sum(0)
    da1 = (da2 @ w2) * (a1 > 0)
    g[W1:B1] = (da1.T @ xs).reshape(-1)
    g[B1:W2] = da1.sum(0)
    return L, g


def adam(theta, m, v, g, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    """One Adam update (decoupled weight decay on the weights); returns
    (theta, m, v, kernel network parameters)."""
    theta = np.asarray(theta, np.float64).copy()
    m = b1 * np.asarray(m, np.float64) + (1 - b1) * g
    v = b2 * np.asarray(v, np.float64) + (1 - b2) * g * g
    k = np.arange(NPARAM)
    if wd > 0:
        theta[is_weight(k)] -= lr * wd * theta[is_weight(k)]
    theta -= lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    out = theta.astype(np.float32)
    out[is_weight(k)] = round_bf16(out[is_weight(k)])
    return theta, m, v, out


def box_filter(rho, u, shape, f):
    """rho [n], u [3][n] (x-fastest) -> [10][nc] (rho_bar, u~ (3), tau (6))."""
    nx, ny, nz = shape
    r = np.asarray(rho, np.float64).reshape(nz // f, f, ny // f, f, nx // f, f)
    U = [np.asarray(u[a], np.float64).reshape(nz // f, f, ny // f, f, nx // f, f) for a in range(3)]
    ax = (1, 3, 5)
    sr = r.sum(ax)
    ut = [(r * U[a]).sum(ax) / sr for a in range(3)]
    out = [sr / f ** 3] + ut
    for a, b in ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)):
        out.append((r * U[a] * U[b]).sum(ax) / sr - ut[a] * ut[b])
    return np.stack([o.reshape(-1) for o in out])


def sample_nodes(seed: int, n_samples: int, n: int) -> np.ndarray:
    """Node of sample i: splitmix64 finaliser of seed * golden + i, mod n
    (seed 0: node i)."""
    i = np.arange(n_samples, dtype=np.uint64)
    if seed == 0:
        return i.astype(np.int64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + i
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z % np.uint64(n)).astype(np.int64)


def samples(filt, shape, tau, cs0, seed, n_samples):
    """Features, targets and weights of the training samples."""
    nx, ny, nz = shape
    F = np.asarray(filt, np.float64).reshape(10, nz, ny, nx)
    u = F[1:4]
    # G[a][b] = d u_a / d x_b (axis order of the arrays is z, y, x)
    axis = {0: 2, 1: 1, 2: 0}
    G = np.empty((3, 3, nz, ny, nx))
    for a in range(3):
        for b in range(3):
            G[a, b] = 0.5 * (np.roll(u[a], -1, axis[b]) - np.roll(u[a], 1, axis[b]))
    S = np.stack([G[0, 0], G[1, 1], G[2, 2], 0.5 * (G[0, 1] + G[1, 0]), 0.5 * (G[0, 2] + G[2, 0]),
                  0.5 * (G[1, 2] + G[2, 1])], -1).reshape(-1, 6)
    tau_sgs = np.moveaxis(F[4:10], 0, -1).reshape(-1, 6)
    rho = F[0].reshape(-1)
    nodes = sample_nodes(seed, n_samples, nx * ny * nz)
    S, T, rho = S[nodes], tau_sgs[nodes], rho[nodes]
    ss = (S[:, :3] ** 2).sum(1) + 2 * (S[:, 3:] ** 2).sum(1)
    smag = np.sqrt(2 * ss)
    tr = T[:, :3].sum(1) / 3
    Td = T.copy()
    Td[:, :3] -= tr[:, None]
    tds = (Td[:, :3] * S[:, :3]).sum(1) + 2 * (Td[:, 3:] * S[:, 3:]).sum(1)
    c2 = float(cs0) ** 2
    s3 = smag ** 3
    target = np.where(s3 > 0, -tds / (c2 * np.where(s3 > 0, s3, 1)), 0.0)
    taus = tau + 3 * c2 * smag
    P = -(2.0 / 3.0) * rho[:, None] * taus[:, None] * S
    return features(P, rho), target, s3
