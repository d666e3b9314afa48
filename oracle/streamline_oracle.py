"""Restatement of the reference's streamline advection and seeding in numpy
float32.  TEST INFRASTRUCTURE ONLY: tests use it as the checker of the CUDA
kernel; the product never imports it.

Follows volumetric-grid/lattice-boltzmann/shaders/streamline_advect.comp.glsl
:34-91 (xorshift32 reseed into the inlet slab, RK2 with trilinear
clamp-to-edge sampling, ring-buffer write) and the host seeding
src/main.cpp:1126-1152 (std::mt19937 and std::uniform_real_distribution
<float>, restated here from their published definitions: the MT19937
generator, and the canonical float of one 32-bit draw, x / 2^32 in float,
as libstdc++'s generate_canonical<float, 24> computes it).

Every float operation is a separate float32 operation in the kernel's order,
so the results are bit-identical to the kernel's.
"""
from __future__ import annotations

import numpy as np

F = np.float32


class MT19937:
    """The Mersenne Twister of Matsumoto and Nishimura (1998), 32-bit."""

    def __init__(self, seed: int):
        self.mt = [0] * 624
        self.mt[0] = seed & 0xFFFFFFFF
        for i in range(1, 624):
            self.mt[i] = (1812433253 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.idx = 624

    def _twist(self):
        mt = self.mt
        for i in range(624):
            y = (mt[i] & 0x80000000) | (mt[(i + 1) % 624] & 0x7FFFFFFF)
            mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ (0x9908B0DF if y & 1 else 0)
        self.idx = 0

    def __call__(self) -> int:
        if self.idx >= 624:
            self._twist()
        y = self.mt[self.idx]
        self.idx += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF


def canonical_float(rng: MT19937) -> np.float32:
    """Uniform float in [0, 1) from one 32-bit draw: float(x) / 2^32, and the
    largest float below 1 if that rounds up to 1."""
    v = F(rng()) / F(4294967296.0)
    if v >= F(1.0):
        v = np.nextafter(F(1.0), F(0.0), dtype=np.float32)
    return F(v)


def seed(count, history, shape, seed=12345, reseed_age=256) -> np.ndarray:
    nx, ny, nz = shape
    rng = MT19937(seed)
    out = np.empty((count, history, 4), np.float32)
    x_lo, x_hi = F(nx) * F(0.0625), F(nx) * F(0.125)
    for i in range(count):
        age = canonical_float(rng) * F(reseed_age)
        px = x_lo + (x_hi - x_lo) * canonical_float(rng)
        py = canonical_float(rng) * F(ny)
        pz = canonical_float(rng) * F(nz)
        out[i, :] = (px, py, pz, age)
    return out


def _xorshift(s):
    s = s ^ ((s << np.uint32(13)) & np.uint32(0xFFFFFFFF))
    s = s ^ (s >> np.uint32(17))
    s = s ^ ((s << np.uint32(5)) & np.uint32(0xFFFFFFFF))
    return s


def _rng01(s):
    s = _xorshift(s)
    return s, (s & np.uint32(0x00FFFFFF)).astype(np.float32) / F(16777216.0)


def _axis(ctr, N):
    u = ctr * F(N) - F(0.5)
    f = np.floor(u)
    a = u - f
    lo = f.astype(np.int64)
    return np.clip(lo, 0, N - 1), np.clip(lo + 1, 0, N - 1), a


def sample(u_planes, shape, cx, cy, cz, round_f16=True):
    """Trilinear, clamp-to-edge, per component; u_planes float32 [3][n]."""
    nx, ny, nz = shape
    U = u_planes.reshape(3, nz, ny, nx).astype(np.float32)
    if round_f16:
        U = U.astype(np.float16).astype(np.float32)
    x0, x1, ax = _axis(cx, nx)
    y0, y1, ay = _axis(cy, ny)
    z0, z1, az = _axis(cz, nz)

    def lerp(a, b, t):
        return a + t * (b - a)

    out = []
    for c in range(3):
        T = U[c]
        c00 = lerp(T[z0, y0, x0], T[z0, y0, x1], ax)
        c10 = lerp(T[z0, y1, x0], T[z0, y1, x1], ax)
        c01 = lerp(T[z1, y0, x0], T[z1, y0, x1], ax)
        c11 = lerp(T[z1, y1, x0], T[z1, y1, x1], ax)
        out.append(lerp(lerp(c00, c10, ay), lerp(c01, c11, ay), az))
    return out


def advect(u_planes, shape, ring, head, frame, dt, reseed_age=256, round_f16=True):
    """One advect pass on ring float32 [count][history][4] (in place)."""
    count, history, _ = ring.shape
    dmax = [F(shape[0]), F(shape[1]), F(shape[2])]
    prev = ring[:, (head + history - 1) % history, :].copy()
    p = [prev[:, 0].copy(), prev[:, 1].copy(), prev[:, 2].copy()]
    age = prev[:, 3].copy()
    out = np.zeros(count, bool)
    for c in range(3):
        out |= (p[c] < F(0)) | (p[c] > dmax[c])
    reseed = (age >= F(reseed_age)) | out
    sid = np.arange(count, dtype=np.uint64)
    st = ((sid * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)) ^ \
         ((np.uint64(frame) * np.uint64(1597334677)) & np.uint64(0xFFFFFFFF))
    st = st.astype(np.uint32)
    st, r0 = _rng01(st)
    st, r1 = _rng01(st)
    st, r2 = _rng01(st)
    sx = F(0) + ((dmax[0] - F(0)) * F(0.0625)) * (F(1) + r0)
    sy = F(0) + (dmax[1] - F(0)) * r1
    sz = F(0) + (dmax[2] - F(0)) * r2
    u1 = sample(u_planes, shape, p[0] / dmax[0], p[1] / dmax[1], p[2] / dmax[2], round_f16)
    h = F(0.5) * F(dt)
    mid = [p[c] + h * u1[c] for c in range(3)]
    u2 = sample(u_planes, shape, mid[0] / dmax[0], mid[1] / dmax[1], mid[2] / dmax[2], round_f16)
    adv = [p[c] + F(dt) * u2[c] for c in range(3)]
    new = np.stack([np.where(reseed, sx, adv[0]), np.where(reseed, sy, adv[1]),
                    np.where(reseed, sz, adv[2]), np.where(reseed, F(0), age + F(1))], -1).astype(np.float32)
    ring[~reseed, head, :] = new[~reseed]
    ring[reseed, :, :] = new[reseed][:, None, :]
    return ring
