"""Restatement of the reference's velocity-magnitude raymarch in numpy
float32.  TEST INFRASTRUCTURE ONLY: tests use it as the checker of the CUDA
kernel; the product never imports it.

Follows volumetric-grid/lattice-boltzmann/shaders/velmag.frag.glsl:44-96 with
the LUTs of src/main.cpp:529-573 and the full-screen triangle of
shaders/fullscreen.vert.glsl.  The samplers, sqrt and exp are the separately
rounded fp32 operations the kernel documents (gpu-sims_b200/csrc/render.cu),
evaluated here in the same order, so images agree bit for bit.
"""
from __future__ import annotations

import numpy as np

F = np.float32


def colormap_lut() -> np.ndarray:
    """rgba8 [4][256][4], the cool-to-warm ramp, channels truncated."""
    out = np.zeros((4, 256, 4), np.uint8)
    for i in range(256):
        t = F(i) / F(255.0)
        if t < F(0.25):
            f = t / F(0.25)
            r, g, b = F(0.05), F(0.05) + F(0.6) * f, F(0.4) + F(0.6) * f
        elif t < F(0.5):
            f = (t - F(0.25)) / F(0.25)
            r, g, b = F(0.05), F(0.65) + F(0.3) * f, F(1.0) - F(0.7) * f
        elif t < F(0.75):
            f = (t - F(0.5)) / F(0.25)
            r, g, b = F(0.05) + F(0.95) * f, F(0.95) - F(0.05) * f, F(0.3) - F(0.25) * f
        else:
            f = (t - F(0.75)) / F(0.25)
            r, g, b = F(1.0), F(0.9) - F(0.7) * f, F(0.05)
        rgb = [int(np.clip(v, F(0), F(1)) * F(255.0)) for v in (r, g, b)]
        out[:, i, :3] = rgb
        out[:, i, 3] = 255
    return out


def jitter_lut() -> np.ndarray:
    out = np.zeros(256 * 256, np.uint8)
    s = 0x9E3779B9
    for i in range(out.size):
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = (s >> 24) & 0xFF
    return out.reshape(256, 256)


def exp_neg(x):
    """e^x (x <= 0): Cody-Waite reduction by ln2, Taylor to r^7, 2^n from
    bits; float32 operations in the kernel's order."""
    x = np.asarray(x, np.float32)
    ok = x > F(-87.0)
    xs = np.where(ok, x, F(0))
    n = np.rint(xs * F(1.44269502))
    r = (xs - n * F(0.693145751953125)) - n * F(1.42860677e-06)
    p = F(1.0) / F(5040.0)
    for c in (F(1.0) / F(720.0), F(1.0) / F(120.0), F(1.0) / F(24.0), F(1.0) / F(6.0), F(0.5), F(1.0), F(1.0)):
        p = p * r + c
    two_n = ((n.astype(np.int32) + 127) << 23).astype(np.int32).view(np.float32)
    return np.where(ok, p * two_n, F(0)).astype(np.float32)


def _lerp(a, b, t):
    return a + t * (b - a)


def _axis(ctr, N):
    u = ctr * F(N) - F(0.5)
    f = np.floor(u)
    return np.clip(f.astype(np.int64), 0, N - 1), np.clip(f.astype(np.int64) + 1, 0, N - 1), u - f


def _sample(U, shape, cx, cy, cz):
    nx, ny, nz = shape
    x0, x1, ax = _axis(cx, nx)
    y0, y1, ay = _axis(cy, ny)
    z0, z1, az = _axis(cz, nz)
    out = []
    for c in range(3):
        T = U[c]
        c00 = _lerp(T[z0, y0, x0], T[z0, y0, x1], ax)
        c10 = _lerp(T[z0, y1, x0], T[z0, y1, x1], ax)
        c01 = _lerp(T[z1, y0, x0], T[z1, y0, x1], ax)
        c11 = _lerp(T[z1, y1, x0], T[z1, y1, x1], ax)
        out.append(_lerp(_lerp(c00, c10, ay), _lerp(c01, c11, ay), az))
    return out


def render(u_planes, shape, inv_view_proj, camera_pos, width, height, steps=128, absorption=4.0,
           vmin=0.0, vmax=0.1, exposure=1.5, round_f16=True, box_min=(0, 0, 0), box_max=None):
    """RGBA float32 [height][width][4]."""
    nx, ny, nz = shape
    U = np.asarray(u_planes, np.float32).reshape(3, nz, ny, nx)
    if round_f16:
        U = U.astype(np.float16).astype(np.float32)
    M = np.asarray(inv_view_proj, np.float32).reshape(4, 4)  # M[col][row]
    cam = [F(c) for c in camera_pos]
    bmin = [F(b) for b in box_min]
    bmax = [F(b) for b in (box_max if box_max is not None else (nx, ny, nz))]
    lut = colormap_lut()[0, :, :3]
    jit = jitter_lut()
    py, px = np.meshgrid(np.arange(height), np.arange(width), indexing="ij")
    px, py = px.reshape(-1), py.reshape(-1)
    ndc = [(px.astype(np.float32) + F(0.5)) / F(width) * F(2.0) - F(1.0),
           (py.astype(np.float32) + F(0.5)) / F(height) * F(2.0) - F(1.0), F(1.0), F(1.0)]
    w4 = [((M[0, r] * ndc[0] + M[1, r] * ndc[1]) + M[2, r] * ndc[2]) + M[3, r] * ndc[3] for r in range(4)]
    rd = [w4[c] / w4[3] - cam[c] for c in range(3)]
    ln = np.sqrt((rd[0] * rd[0] + rd[1] * rd[1]) + rd[2] * rd[2])
    rd = [rd[c] / ln for c in range(3)]
    te = np.full(px.size, -np.inf, np.float32)
    tx = np.full(px.size, np.inf, np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        for c in range(3):
            inv = F(1.0) / rd[c]
            t0 = (bmin[c] - cam[c]) * inv
            t1 = (bmax[c] - cam[c]) * inv
            te = np.fmax(te, np.fmin(t0, t1))
            tx = np.fmin(tx, np.fmax(t0, t1))
    hit = ~((tx < te) | (tx < F(0)))
    out = np.zeros((px.size, 4), np.float32)
    t0 = np.fmax(te, F(0))
    ray = tx - t0
    jitter = jit[np.minimum(py, 255), np.minimum(px, 255)].astype(np.float32) / F(255.0)
    dt = ray / F(steps)
    t = t0 + jitter * dt
    col = [np.zeros(px.size, np.float32) for _ in range(3)]
    trans = np.ones(px.size, np.float32)
    ext = [bmax[c] - bmin[c] for c in range(3)]
    rng_ = np.fmax(F(vmax) - F(vmin), F(1e-6))
    active = hit.copy()
    for _ in range(steps):
        active &= trans > F(0.01)
        if not active.any():
            break
        uvw = [((cam[c] + rd[c] * t) - bmin[c]) / ext[c] for c in range(3)]
        inside = active.copy()
        for c in range(3):
            inside &= (uvw[c] >= F(0)) & (uvw[c] <= F(1))
        idx = np.nonzero(inside)[0]
        if idx.size:
            u = _sample(U, shape, uvw[0][idx], uvw[1][idx], uvw[2][idx])
            mag = np.sqrt((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2])
            t01 = np.fmin(np.fmax((mag - F(vmin)) / rng_, F(0)), F(1))
            lu = t01 * F(256.0) - F(0.5)
            lf = np.floor(lu)
            la = lu - lf
            l0 = np.clip(lf.astype(np.int64), 0, 255)
            l1 = np.clip(lf.astype(np.int64) + 1, 0, 255)
            abs_step = (F(absorption) * dt[idx]) * t01
            for c in range(3):
                cc = _lerp(lut[l0, c].astype(np.float32) / F(255.0), lut[l1, c].astype(np.float32) / F(255.0), la)
                col[c][idx] = col[c][idx] + ((trans[idx] * cc) * abs_step) * F(exposure)
            trans[idx] = trans[idx] * exp_neg(-abs_step)
        t = np.where(active, t + dt, t)
    for c in range(3):
        out[:, c] = np.where(hit, col[c], F(0))
    out[:, 3] = np.where(hit, F(1) - trans, F(0))
    return out.reshape(height, width, 4)
