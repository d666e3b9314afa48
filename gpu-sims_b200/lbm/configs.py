"""Workload definitions of the benchmark configurations (lid-driven cavity,
Taylor-Green vortex, channel, cavity ensemble) and the voxel and duct runs.

    python -m lbm.configs ensemble [--steps 2000] [--domains 256] [--precision f16s]
                                   [--schedule rows,z,persistent]
    python -m lbm.configs voxel
    python -m lbm.configs duct [--steps 1000]
    python -m lbm.configs closure_step [--steps 200]

(run from gpu-sims_b200/, or with it on sys.path) prints one JSON line:
ensemble: the aggregate MLUPS of the 256-cavity ensemble in fp16 and fp32
storage and the per-domain fp16-vs-fp32 velocity error; voxel: host against
device NACA voxeliser at the capture tier; duct: the open-face channel
(Zou-He inlet / outlet) against the walled one.  All inputs are synthetic and seeded;
device time is measured with CUDA events on the library's stream.  The FP64
comparisons of the cavity, Taylor-Green and channel workloads are GPU tests
(tests/test_configs_gpu.py).
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

import lbm

EDGES = (32, 48, 64, 80, 96)
LID = 0.05


def _timer():
    import torch
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    def run(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    return stream, run


def ensemble_descs(n=256, seed=2024, precision=lbm.PREC_F16S, collision=lbm.COLL_TRT):
    """n lid-driven cavities: edge uniform from {32,48,64,80,96}, Re uniform in
    [100, 1000], tau = 0.5 + 3 nu with nu = U L / Re, lid U = 0.05 along +x on
    the z = max face, half-way bounce-back on the other five walls.  TRT by
    default: with BGK the 32- and 48-node cavities at tau below about 0.508
    (38 of the 256 for seed 2024) diverge in fp32 and fp16 alike."""
    rng = np.random.default_rng(seed)
    edges = rng.choice(EDGES, size=n)
    res = rng.uniform(100.0, 1000.0, size=n)
    descs = []
    for L, re in zip(edges, res):
        wall = np.zeros((6, 3))
        wall[lbm.FACE_ZP] = (LID, 0.0, 0.0)
        tau = 0.5 + 3.0 * LID * float(L) / float(re)
        descs.append(lbm.default_desc(nx=int(L), ny=int(L), nz=int(L), mode=lbm.MODE_PHYSICS,
                                      precision=precision, collision=collision, tau=tau,
                                      wall_velocity=wall))
    return descs, edges, res


def run_ensemble(steps=2000, n=256, seed=2024, autotune=True, compare=True, schedule=None,
                 precisions=("f16s", "f32")):
    """schedule: (rows, z, persistent) instead of the autotuner; precisions:
    which storage runs (the fp16-vs-fp32 error needs both)."""
    stream, timed = _timer()
    out = {"config": "ensemble", "domains": n, "steps": steps}
    fields = {}
    compare = compare and set(precisions) == {"f16s", "f32"}
    for name, prec in (("f16s", lbm.PREC_F16S), ("f32", lbm.PREC_F32)):
        if name not in precisions:
            continue
        descs, edges, res = ensemble_descs(n, seed, prec)
        b = lbm.Batch(descs)
        b.set_stream(stream.cuda_stream)
        b.init_equilibrium(-1, 1.0, (0.0, 0.0, 0.0))
        if schedule is not None:
            b.set_schedule(rows_per_block=schedule[0], z_per_thread=schedule[1], persistent=schedule[2])
            sched = b.schedule()
        else:
            sched = b.autotune(10) if autotune else b.schedule()
        info = b.info()
        b.init_equilibrium(-1, 1.0, (0.0, 0.0, 0.0))
        secs = timed(lambda: b.step(steps))
        b.sync()
        mlups = info.total_nodes * steps / secs / 1e6
        out[name] = {"mlups": mlups, "seconds": secs, "total_nodes": info.total_nodes,
                     "bytes_per_node": info.bytes_per_node,
                     "achieved_gbs": mlups * 1e6 * info.bytes_per_node / 1e9,
                     "schedule": {"rows_per_block": sched.rows_per_block,
                                  "z_per_thread": sched.z_per_thread,
                                  "persistent": sched.persistent},
                     "device_bytes": info.device_bytes}
        fields[name] = [b.read_moments(i)[1] for i in range(n)]
        b.close()
        out["edges_histogram"] = {int(e): int((edges == e).sum()) for e in EDGES}
    if compare:
        errs = np.array([np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
                         for a, b in zip(fields["f16s"], fields["f32"])])
        out["f16s_vs_f32_rel_l2_velocity"] = {"max": float(errs.max()), "median": float(np.median(errs)),
                                              "mean": float(errs.mean())}
        out["speedup_f16s_vs_f32"] = out["f16s"]["mlups"] / out["f32"]["mlups"]
    return out


def tgv_init(N, u0=0.05):
    """Taylor-Green vortex on an N^3 periodic box (wavelength N): velocity and
    the density carrying the analytic pressure rho = 1 + 3 p'."""
    k = 2.0 * math.pi / N
    x = np.arange(N)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    ux = u0 * np.sin(k * X) * np.cos(k * Y) * np.cos(k * Z)
    uy = -u0 * np.cos(k * X) * np.sin(k * Y) * np.cos(k * Z)
    p = u0 ** 2 / 16.0 * (np.cos(2 * k * X) + np.cos(2 * k * Y)) * (np.cos(2 * k * Z) + 2.0)
    rho = 1.0 + 3.0 * p
    u = np.stack([ux, uy, np.zeros_like(ux)]).reshape(3, -1)
    return rho.reshape(-1), u


def run_voxel(shape=(512, 256, 256), preset=2, reps=5):
    """The NACA mask of a preset at the capture tier: host voxeliser (one
    core) against the device voxeliser, and set_flags(host mask) against
    set_flags_naca (mask made on the device), each the median of reps."""
    import torch
    stream, timed = _timer()
    p = lbm.PRESETS[preset]
    nx, ny, nz = shape
    n = nx * ny * nz
    args = (lbm.AIRFOIL_CHORD_LENGTH_FRAC, lbm.AIRFOIL_CHORD_CENTER_X_FRAC, p.angle_of_attack_deg)
    host_s = []
    for _ in range(reps):
        t0 = time.perf_counter()
        mask = lbm.voxelize_naca(p.naca, nx, ny, nz, *args)
        host_s.append(time.perf_counter() - t0)
    d = torch.empty(n, dtype=torch.uint8, device="cuda")
    dev_s = [timed(lambda: lbm.voxelize_naca_device(p.naca, nx, ny, nz, d.data_ptr(), n, *args,
                                                    stream=stream.cuda_stream)) for _ in range(reps + 1)][1:]
    same = bool(np.array_equal(d.cpu().numpy(), mask))
    lat = lbm.Lattice(nx=nx, ny=ny, nz=nz)
    lat.set_stream(stream.cuda_stream)
    up_s, naca_s = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        lat.set_flags(mask)
        up_s.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        lat.set_flags_naca(p.naca, *args)
        naca_s.append(time.perf_counter() - t0)
    lat.close()
    med = lambda v: float(np.median(v))
    return {"config": "voxel", "shape": list(shape), "naca": p.naca, "mask_bytes": n,
            "host_voxelize_s": med(host_s), "device_voxelize_s": med(dev_s),
            "speedup": med(host_s) / med(dev_s), "same_mask": same,
            "set_flags_host_mask_s": med(up_s), "set_flags_naca_s": med(naca_s)}


def run_duct(steps=1000, shape=(512, 128, 128)):
    """Open-face channel: velocity inlet (u = 0.05) at x = 0, pressure outlet
    (rho = 1) at x = nx-1, half-way bounce-back y / z walls, sphere r = 16 at
    (128, 64, 64), tau = 0.55, BGK; MLUPS in fp32 and fp16 storage against the
    same channel with walls in place of the open faces."""
    stream, timed = _timer()
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    mask = (((x - 128) ** 2 + (y - 64) ** 2 + (z - 64) ** 2) <= 256).astype(np.uint8).reshape(-1)
    out = {"config": "duct", "shape": list(shape), "steps": steps}
    for name, prec in (("f32", lbm.PREC_F32), ("f16s", lbm.PREC_F16S)):
        for tag, kinds in (("open", (lbm.OPEN_VELOCITY, lbm.OPEN_PRESSURE)), ("walls", (0, 0))):
            wall = np.zeros((6, 3))
            if kinds[0]:
                wall[lbm.FACE_XM] = (0.05, 0.0, 0.0)
            d = lbm.default_desc(nx=nx, ny=ny, nz=nz, mode=lbm.MODE_PHYSICS, precision=prec, tau=0.55,
                                 wall_velocity=wall, open_x=kinds, open_rho=(0.0, 1.0 if kinds[1] else 0.0))
            lat = lbm.Lattice(d)
            lat.set_stream(stream.cuda_stream)
            lat.set_flags(mask)
            lat.init_equilibrium(1.0, (0.0, 0.0, 0.0))
            lat.step(20)
            secs = timed(lambda: lat.step(steps))
            lat.sync()
            rho, u = lat.read_moments()
            out[f"{name}_{tag}"] = {"mlups": nx * ny * nz * steps / secs / 1e6,
                                    "finite": bool(np.isfinite(u).all()),
                                    "outlet_mean_ux": float(u[:, 0].reshape(nz, ny, nx)[:, :, nx - 1].mean())}
            lat.close()
    return out


def run_closure_step(n=128, steps=200, variants=(0, 1, 8)):
    """The learned-closure step on an n^3 periodic box (tau 0.502, Cs0 0.1, a
    He-initialised network, seeded random velocity): MLUPS per step variant
    (0 automatic: CUDA-core MLP, two nodes per thread; 1 one node per
    thread; 8 tensor-core MLP) in fp32 and fp16 storage."""
    from lbm import closure as cl
    stream, timed = _timer()
    net = cl.init_net(5, np.zeros(lbm.CLOSURE_INPUTS), np.ones(lbm.CLOSURE_INPUTS))
    rng = np.random.default_rng(0)
    u = (0.02 * rng.standard_normal((n ** 3, 3))).astype(np.float32)
    out = {"config": "closure_step", "n": n, "steps": steps}
    for name, prec in (("f32", lbm.PREC_F32), ("f16s", lbm.PREC_F16S)):
        for v in variants:
            d = lbm.default_desc(nx=n, ny=n, nz=n, mode=lbm.MODE_PHYSICS, precision=prec, periodic=(1, 1, 1),
                                 tau=0.502, smagorinsky_cs=0.1)
            lat = lbm.Lattice(d)
            lat.set_stream(stream.cuda_stream)
            lat.set_closure(net)
            lat.init_from_moments(np.ones(n ** 3, np.float32), u)
            lat.set_step_variant(v)
            lat.step(20)
            secs = timed(lambda: lat.step(steps))
            lat.sync()
            out[f"{name}_variant{v}"] = n ** 3 * steps / secs / 1e6
            lat.close()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=["ensemble", "voxel", "duct", "closure_step"])
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--domains", type=int, default=256)
    ap.add_argument("--precision", choices=["both", "f16s", "f32"], default="both",
                    help="ensemble: storage precisions to run")
    ap.add_argument("--schedule", default=None,
                    help="ensemble: rows,z,persistent instead of the autotuner (e.g. 4,16,0)")
    a = ap.parse_args(argv)
    if a.config == "ensemble":
        sched = tuple(int(v) for v in a.schedule.split(",")) if a.schedule else None
        precs = ("f16s", "f32") if a.precision == "both" else (a.precision,)
        r = run_ensemble(steps=a.steps or 2000, n=a.domains, schedule=sched, precisions=precs)
    elif a.config == "voxel":
        r = run_voxel()
    elif a.config == "closure_step":
        r = run_closure_step(steps=a.steps or 200)
    else:
        r = run_duct(steps=a.steps or 1000)
    print(json.dumps(r), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
