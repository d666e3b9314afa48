"""The BASELINE workloads against FP64 runs of the oracle on the GPU.

Each test runs the physics-mode step in fp32, fp16-shifted and bf16-shifted
storage and the FP64 oracle (ExtStep's GPU copy) on the same inputs, and
checks the errors against written bounds, at the full workload sizes:
cavity 64^3 x 1000, Taylor-Green 384^3 x 2000, channel 512x128x128 x 5000,
and the 256-cavity ensemble x 2000 (fp16 against fp32 storage per domain).
LBM_QUICK_CONFIGS=1 runs reduced sizes for quick iteration; with
LBM_RESULTS_DIR set, each result is written as JSON there.
"""
import json
import math
import os
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FULL = os.environ.get("LBM_QUICK_CONFIGS") != "1"
LID = 0.05


def record(name, data):
    d = os.environ.get("LBM_RESULTS_DIR")
    if d:
        Path(d).mkdir(parents=True, exist_ok=True)
        (Path(d) / f"{name}.json").write_text(json.dumps(data, indent=1))


class Timer:
    """CUDA-event timing on a dedicated stream the lattice runs on."""

    def __init__(self):
        import torch
        self.torch = torch
        self.stream = torch.cuda.Stream()

    def __call__(self, fn):
        t = self.torch
        e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        t.cuda.synchronize()
        e0.record(self.stream)
        fn()
        e1.record(self.stream)
        t.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3


def errors(u, ref_u, rho, ref_rho):
    du = u.T.astype(np.float64) - ref_u
    return {"rel_l2_velocity": float(np.linalg.norm(du) / max(np.linalg.norm(ref_u), 1e-300)),
            "max_abs_velocity_over_scale": float(np.abs(du).max() / max(np.abs(ref_u).max(), 1e-300)),
            "max_abs_rho": float(np.abs(rho.astype(np.float64) - ref_rho).max())}


def lattice(lbm, shape, timer, **kw):
    d = lbm.default_desc(nx=shape[0], ny=shape[1], nz=shape[2], mode=lbm.MODE_PHYSICS, **kw)
    lat = lbm.Lattice(d)
    lat.set_stream(timer.stream.cuda_stream)
    return lat


PRECS = (("f32", 0), ("f16s", 1), ("bf16s", 2))
# Written bounds on the relative L2 velocity error against FP64, per config.
# fp32 rounding in these near-steady flows repeats coherently from step to
# step, so it accumulates linearly (about 2e-4 after 5000 channel steps);
# fp16/bf16 rounding noise random-walks in the conserved momentum mode.
BOUNDS = {
    "cavity": {"f32": 1e-4, "f16s": 1e-3, "bf16s": 2e-2},
    "tgv": {"f32": 5e-4, "f16s": 1e-2, "bf16s": 5e-2},
    "channel": {"f32": 5e-4, "f16s": 1e-3, "bf16s": 1.5e-1},
}


def test_cavity_vs_fp64(gpu, oracle):
    """Config 1: lid-driven cavity, BGK tau 0.6 (Re = 96), lid 0.05 along +x
    on z = max, half-way bounce-back elsewhere, 1000 steps at 64^3."""
    L, steps, tau = (64, 1000, 0.6)
    timer = Timer()
    wall = np.zeros((6, 3))
    wall[gpu.FACE_ZP] = (LID, 0, 0)
    n = L ** 3
    ref = oracle.ExtStateGPU((L, L, L), tau=tau, wall=wall)
    ref.init(np.ones(n), np.zeros((3, n)))
    ref.step(steps)
    rr, ru = ref.moments()
    out = {"config": "cavity", "shape": [L] * 3, "steps": steps, "tau": tau,
           "Re": LID * L / ((tau - 0.5) / 3)}
    for name, prec in PRECS:
        lat = lattice(gpu, (L, L, L), timer, precision=prec, tau=tau, wall_velocity=wall)
        lat.init_equilibrium(1.0, (0, 0, 0))
        secs = timer(lambda: lat.step(steps))
        rho, u = lat.read_moments()
        out[name] = dict(errors(u, ru, rho, rr), mlups=n * steps / secs / 1e6)
        lat.close()
    record("cavity", out)
    for name, _ in PRECS:
        assert out[name]["rel_l2_velocity"] <= BOUNDS["cavity"][name], (name, out[name])


def test_taylor_green_vs_fp64(gpu, oracle):
    """Config 2: TRT Taylor-Green vortex at Re = 1600 (L = N / 2 pi), fp32 /
    fp16 / bf16 storage against FP64 on the same grid; kinetic energy sampled
    along the way; FP64 on a coarser grid at the same Re and t* gives the
    resolution reference for the decay."""
    from lbm import configs
    N, steps, Nref = (384, 2000, 128) if FULL else (96, 500, 32)
    u0, re = 0.05, 1600.0
    samples = 5
    timer = Timer()
    Lc = N / (2 * math.pi)
    tau = 0.5 + 3 * u0 * Lc / re
    rho0, u_init = configs.tgv_init(N, u0)
    n = N ** 3
    every = steps // samples

    def ke(u):
        u = np.asarray(u, np.float64)
        return 0.5 * float(np.mean(np.sum(u ** 2, axis=0 if u.shape[0] == 3 else 1)))

    ref = oracle.ExtStateGPU((N,) * 3, periodic=(1, 1, 1), tau=tau, collision=1)
    ref.init(rho0, u_init)
    ke_ref = [ke(u_init)]
    for _ in range(samples):
        ref.step(every)
        ke_ref.append(ke(ref.moments()[1]))
    rr, ru = ref.moments()
    del ref
    out = {"config": "tgv", "shape": [N] * 3, "steps": steps, "tau": tau, "Re": re,
           "t_star_end": steps * u0 / Lc, "f64_ke": ke_ref}
    for name, prec in PRECS:
        lat = lattice(gpu, (N,) * 3, timer, precision=prec, collision=1, periodic=(1, 1, 1), tau=tau)
        lat.init_from_moments(rho0.astype(np.float32), np.ascontiguousarray(u_init.T.astype(np.float32)))
        kes, secs = [ke(u_init)], 0.0
        for _ in range(samples):
            secs += timer(lambda: lat.step(every))
            kes.append(ke(lat.read_moments()[1]))
        rho, u = lat.read_moments()
        e = errors(u, ru, rho, rr)
        e.update(ke=kes, ke_rel_err_max=float(max(abs(a - b) / b for a, b in zip(kes, ke_ref))),
                 mlups=n * steps / secs / 1e6)
        out[name] = e
        lat.close()
    Lr = Nref / (2 * math.pi)
    tau_r = 0.5 + 3 * u0 * Lr / re
    steps_r = int(round(steps * Lr / Lc))
    rc, uc = configs.tgv_init(Nref, u0)
    cref = oracle.ExtStateGPU((Nref,) * 3, periodic=(1, 1, 1), tau=tau_r, collision=1)
    cref.init(rc, uc)
    ke_c = [ke(uc)]
    for _ in range(samples):
        cref.step(steps_r // samples)
        ke_c.append(ke(cref.moments()[1]))
    out["f64_coarse"] = {"shape": [Nref] * 3, "tau": tau_r, "steps": steps_r, "ke": ke_c}
    record("tgv", out)
    for name, _ in PRECS:
        assert out[name]["rel_l2_velocity"] <= BOUNDS["tgv"][name], (name, out[name]["rel_l2_velocity"])


def test_channel_vs_fp64(gpu, oracle):
    """Config 3 (the bench workload): x-periodic channel with body force and a
    sphere, BGK tau 0.55, seeded noise; full size 512x128x128 x 5000."""
    import bench
    if FULL:
        shape, steps, c, r = bench.SHAPE, 5000, bench.SPHERE_C, bench.SPHERE_R
        mask, rho, u = bench.make_inputs()
    else:
        shape, steps, c, r = (128, 32, 32), 1000, (32, 16, 16), 4
        nx, ny, nz = shape
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        mask = (((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) <= r * r).astype(np.uint8).reshape(-1)
        rng = np.random.Generator(np.random.Philox(bench.SEED))
        u = (bench.NOISE * rng.standard_normal((mask.size, 3))).astype(np.float32)
        u[mask == 1] = 0
        rho = np.ones(mask.size, np.float32)
    timer = Timer()
    n = mask.size
    ref = oracle.ExtStateGPU(shape, periodic=(1, 0, 0), tau=bench.TAU, collision=0, accel=bench.ACCEL,
                             mask=mask)
    ref.init(rho.astype(np.float64), u.T.astype(np.float64))
    ref.step(steps)
    rr, ru = ref.moments()
    del ref
    out = {"config": "channel", "shape": list(shape), "steps": steps,
           "mean_ux_f64": float(ru[0][mask == 0].mean())}
    for name, prec in PRECS:
        lat = lattice(gpu, shape, timer, precision=prec, periodic=(1, 0, 0), tau=bench.TAU,
                      body_accel=bench.ACCEL)
        lat.set_flags(mask)
        lat.init_from_moments(rho, u)
        secs = timer(lambda: lat.step(steps))
        r2, u2 = lat.read_moments()
        out[name] = dict(errors(u2, ru, r2, rr), mlups=n * steps / secs / 1e6)
        lat.close()
    record("channel", out)
    for name, _ in PRECS:
        assert out[name]["rel_l2_velocity"] <= BOUNDS["channel"][name], (name, out[name]["rel_l2_velocity"])


def test_ensemble_f16_vs_f32(gpu):
    """Config 4: 256 lid-driven cavities (edges from {32..96}, Re in
    [100, 1000], TRT) advanced together for 2000 steps in fp16-shifted and in
    fp32 storage; per domain, the relative L2 velocity error of the fp16 run
    against the fp32 run.  Bounds: median 1e-3, max 1e-2."""
    from lbm import configs
    n, steps = (256, 2000) if FULL else (32, 300)
    out = configs.run_ensemble(steps=steps, n=n, autotune=True)
    record("ensemble", out)
    e = out["f16s_vs_f32_rel_l2_velocity"]
    assert e["median"] <= 1e-3, e
    assert e["max"] <= 1e-2, e
