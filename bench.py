#!/usr/bin/env python
"""D3Q19 step throughput (MLUPS) and HBM-roofline fraction.

Workload: the plain D3Q19 BGK channel, 512 x 128 x 128 nodes, x-periodic
with body force g = 1e-6 along x, half-way bounce-back at the y and z walls,
a solid sphere of radius 16 at (128, 64, 64), tau = 0.55, rho = 1 and u =
seeded Gaussian noise (sigma 1e-4, Philox seed 1234).  fp32 populations
(the headline) and fp16-shifted populations (a variant on the same line).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one fused stream+collide launch over the whole domain.  For N > 1
the script runs under torchrun, one independent replica per GPU (the path
has no exchange step), and reports the aggregate over ranks with the time
taken as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for p in (ROOT, ROOT / "gpu-sims_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

SHAPE = (512, 128, 128)
SPHERE_C, SPHERE_R = (128, 64, 64), 16
TAU, ACCEL, NOISE, SEED = 0.55, (1e-6, 0.0, 0.0), 1e-4, 1234
WORKLOAD = ("channel 512x128x128 D3Q19 BGK, x-periodic, body force g=1e-6 (x), half-way "
            "bounce-back y/z walls, sphere r=16 at (128,64,64), tau=0.55")
METRIC = "D3Q19 MLUPS (channel 512x128x128, fp32 BGK)"
REF_TIER = (256, 128, 128)
FALLBACK_HBM_GBS = 6650.0


def make_inputs():
    nx, ny, nz = SHAPE
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    mask = (((x - SPHERE_C[0]) ** 2 + (y - SPHERE_C[1]) ** 2 + (z - SPHERE_C[2]) ** 2)
            <= SPHERE_R ** 2).astype(np.uint8).reshape(-1)
    rng = np.random.Generator(np.random.Philox(SEED))
    n = nx * ny * nz
    u = (NOISE * rng.standard_normal((n, 3))).astype(np.float32)
    u[mask == 1] = 0.0
    rho = np.ones(n, np.float32)
    return mask, rho, u


def peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        v = float(json.loads(p.read_text())["hbm_gbs"])
        return v, "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(name: str):
    """DRAM read+write bytes per launch from a committed ncu summary, if any."""
    f = ROOT / "profiles" / f"{name}.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML while running."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    # polled as fast as NVML answers: a 20-step timed region lasts a few
    # milliseconds
    def __init__(self, index: int, period: float = 0.0005):
        self.index, self.period = index, period
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception as e:  # no NVML: report that, do not fail the run
            self.error = str(e)
        return self

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(self.period)

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != n_gpus:
        raise SystemExit(f"--gpus {n_gpus} but WORLD_SIZE={world}: launch N>1 with torchrun")
    return world, rank, local


def max_over_ranks(v: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's time (every rank takes part; one all-reduce)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_mlups(nodes_per_rank: int, steps: int, seconds_max: float, world: int) -> float:
    """Whole-job rate: every rank advances its own replica of nodes_per_rank
    nodes, so the job did world * nodes * steps updates in the slowest
    rank's time."""
    return world * nodes_per_rank * steps / seconds_max / 1e6


def bench_config(n: int, world: int) -> dict:
    """The workload description both arms print (the same dict, so the two
    lines name the same configuration)."""
    return {"workload": WORKLOAD, "nodes": n, "precision": "f32 populations (f - w)",
            "layout": "esoteric pull, one population store",
            "l2": "inputs larger than L2 (populations %.0f MB > 126 MB L2)" % (n * 76 / 1e6),
            "parallelism": f"replicas x{world}"}


CPU_KIND = ("the oracle's float restatement of the physics step (ExtStep<float>, the only CPU "
            "implementation of this workload: the reference's step is four Vulkan compute shaders "
            "with no CPU path), built -O3 -march=x86-64-v3 with FMA contraction, OpenMP over planes")


def run_reference_arm(args, world, rank):
    """The CPU implementation of the same step (the oracle's float port of
    the stream-collide), on all host threads, on the same workload."""
    if rank != 0:
        return 0
    from oracle import oracle
    oracle.build()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    mask, rho, u = make_inputs()
    st = oracle.ExtState(SHAPE, periodic=(1, 0, 0), tau=TAU, collision=0, accel=ACCEL, mask=mask,
                         dtype=np.float32, fast=True)
    st.init(rho, np.ascontiguousarray(u.T))
    n = mask.size
    for _ in range(max(args.warmup, 0)):
        st.step(1)
    t0 = time.perf_counter()
    st.step(1)
    t1 = time.perf_counter() - t0
    k = max(1, min(args.steps, int(150.0 / max(t1, 1e-6))))
    t0 = time.perf_counter()
    st.step(k)
    dt = time.perf_counter() - t0
    mlups = n * k / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": mlups, "unit": "MLUPS",
        "n_gpus": world, "steps": k, "warmup": args.warmup, "ms_per_step": dt / k * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": bench_config(n, world),
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": "port",
                         "what": CPU_KIND,
                         "sample": f"{k} full-domain steps of the workload (requested {args.steps})"},
        "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample():
    """The oracle's float port timed on a bounded sample (about 15 s)."""
    from oracle import oracle
    oracle.build()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    mask, rho, u = make_inputs()
    st = oracle.ExtState(SHAPE, periodic=(1, 0, 0), tau=TAU, collision=0, accel=ACCEL, mask=mask,
                         dtype=np.float32, fast=True)
    st.init(rho, np.ascontiguousarray(u.T))
    t0 = time.perf_counter()
    st.step(1)
    t1 = time.perf_counter() - t0
    k = max(1, min(20, int(15.0 / max(t1, 1e-6))))
    t0 = time.perf_counter()
    st.step(k)
    dt = time.perf_counter() - t0
    return {"value": mask.size * k / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "what": CPU_KIND, "sample": f"{k} full-domain steps of the workload after 1 untimed step"}


def run_ours(args, world, rank, local):
    import torch
    import torch.distributed as dist

    import lbm

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    # A dedicated stream: the library runs on it and the CUDA events are
    # recorded on it.  (The legacy default stream has handle 0, which
    # lbm_set_stream reads as "the context's own stream".)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def ranks_max(v: float) -> float:
        return max_over_ranks(v, world, "cuda")

    mask, rho, u = make_inputs()
    n = mask.size
    peak, peak_kind = peak_hbm()

    def make_phys(precision: int):
        d = lbm.default_desc(nx=SHAPE[0], ny=SHAPE[1], nz=SHAPE[2], mode=lbm.MODE_PHYSICS,
                             precision=precision, collision=lbm.COLL_BGK, periodic=(1, 0, 0),
                             tau=TAU, body_accel=ACCEL)
        lat = lbm.Lattice(d)
        lat.set_stream(stream.cuda_stream)
        lat.set_flags(mask)
        lat.init_from_moments(rho, u)
        return lat

    def make_ref_tier():
        """Reference mode on the reference's own desktop tier and default
        preset (256x128x128, NACA0012 at 4 deg, |u| 0.04, tau 0.6;
        src/main.cpp:103-135), through apply_preset."""
        lat = lbm.Lattice(lbm.preset_desc(0, *REF_TIER))
        lat.set_stream(stream.cuda_stream)
        lbm.apply_preset(lat, 0)
        return lat

    def device_run(make):
        """Device-timed steady state: the step graphs of both parities exist
        from the init on, so the timed lbm_step(K) only launches (K // 16
        graphs of 16 launches, the rest one by one); its last launch also
        writes the moments (16 B/node more, counted in the bytes)."""
        lat = make()
        nodes = lat.n
        bpn = lat.info().bytes_per_node
        lat.step(max(args.warmup, 3))
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            e0.record(stream)
            lat.step(args.steps)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = ranks_max(e0.elapsed_time(e1))
        lat.sync()
        lat.close()
        moment_bytes = 16.0 * nodes  # rho + u of the call's last launch
        achieved = (nodes * bpn * args.steps + moment_bytes) / (ms / 1e3) / 1e9
        return {"value": aggregate_mlups(nodes, args.steps, ms / 1e3, world), "unit": "MLUPS",
                "ms_per_step": ms / args.steps, "bytes_per_node": bpn,
                "achieved_gbs": achieved, "frac": achieved / peak, "clocks": clk.summary()}

    def e2e_run(precision: int):
        """Through the C ABI with host buffers: upload flags and initial
        moments from pinned memory, then per step one lbm_step and a read of
        the conservation sums (the step's metric), then the final moments."""
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
        m_h, r_h, u_h = pin(mask), pin(rho), pin(u)
        r_out = torch.empty(n, dtype=torch.float32).pin_memory().numpy()
        # the velocity as the reference's consumers read it back: rgba16f
        # (capture_save and the VDB export, src/main.cpp:1290-1296, 1771-1779)
        u_out = torch.empty((n, 4), dtype=torch.int16).pin_memory().numpy().view(np.uint16)
        d = lbm.default_desc(nx=SHAPE[0], ny=SHAPE[1], nz=SHAPE[2], mode=lbm.MODE_PHYSICS,
                             precision=precision, collision=lbm.COLL_BGK, periodic=(1, 0, 0),
                             tau=TAU, body_accel=ACCEL)
        lat = lbm.Lattice(d)
        lat.set_stream(stream.cuda_stream)
        lat.set_flags(m_h)
        lat.init_from_moments(r_h, u_h)
        lat.step(3)
        lat.conservation()
        sums = torch.zeros((args.steps, 4), dtype=torch.float64).pin_memory().numpy()
        lib = lbm.load()

        def timed(blocking: bool) -> float:
            barrier()
            t0 = time.perf_counter()
            lat.set_flags(m_h)
            lat.init_from_moments(r_h, u_h)
            for i in range(args.steps):
                lat.step(1)
                if blocking:
                    sums[i] = lat.conservation()
                else:
                    lat.conservation_async(sums[i].ctypes.data)
            rc = lib.lbm_read_moments(lat._h, r_out.ctypes.data, u_out.ctypes.data, lbm.U_F16X4)
            assert rc == 0
            torch.cuda.synchronize()
            return ranks_max(time.perf_counter() - t0)

        dt_block = timed(True)
        last = sums[-1].copy()
        dt = timed(False)
        # the queued reads landed: every step's sums, the last equal to the blocking run's
        assert np.isfinite(sums).all() and np.array_equal(sums[-1], last)
        lat.close()
        h2d = (m_h.nbytes + r_h.nbytes + u_h.nbytes) / args.steps
        d2h = 32 + (r_out.nbytes + u_out.nbytes) / args.steps
        return {"value": aggregate_mlups(n, args.steps, dt, world), "unit": "MLUPS",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "what": "flags + initial moments uploaded from pinned host memory, per step one "
                        "lbm_step(1) and a read of that step's fp64 conservation sums into pinned "
                        "host memory (lbm_conservation_async: no host wait per step), final rho (f32) "
                        "and u (rgba16f, as the reference's capture and VDB export read it) to pinned "
                        "host memory",
                "blocking": {"value": aggregate_mlups(n, args.steps, dt_block, world), "unit": "MLUPS",
                             "what": "the same with lbm_conservation (a host wait every step)"}}

    runs = {}
    want = args.variant
    if want in ("all", "f32"):
        runs["f32"] = device_run(lambda: make_phys(lbm.PREC_F32))
    if want in ("all", "f16s"):
        runs["f16s"] = device_run(lambda: make_phys(lbm.PREC_F16S))
    if want in ("all", "bf16s"):
        runs["bf16s"] = device_run(lambda: make_phys(lbm.PREC_BF16S))
    if want in ("all", "ref"):
        runs["reference_mode_desktop_tier"] = device_run(make_ref_tier)
    e2e = e2e_run(lbm.PREC_F32) if (want in ("all", "f32") and not args.no_e2e) else None
    cpu = cpu_baseline_sample() if (rank == 0 and world == 1 and not args.no_cpu) else None
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    head_key = "f32" if "f32" in runs else next(iter(runs))
    head = runs.pop(head_key)
    if "f32" == head_key:
        for k in ("f16s", "bf16s"):
            if k in runs:
                runs[k]["speedup_vs_f32"] = runs[k]["value"] / head["value"]
    traffic = ncu_traffic("lbm_step_channel_fp32") if head_key == "f32" else None
    line = {
        "metric": METRIC, "value": head["value"], "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": head["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if head_key == "f32" else head_key, "data": "synthetic",
        "config": bench_config(n, world),
        "roofline": {"bound": "hbm", "achieved": head["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": head["frac"], "traffic": traffic,
                     "bytes_per_node": head["bytes_per_node"],
                     "bytes_counted": "bytes_per_node per node update for every timed launch, plus "
                                      "16 B/node once for the moments the call's last launch writes",
                     "peak_kind": ("measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                                   else "fallback copy bandwidth (6650 GB/s, an earlier measurement on this pool; "
                                        "MEASURED_PEAKS.json absent)"),
                     "kernel": "k_phys_step2 (fused esoteric-pull stream+collide, two nodes per thread)"},
        "variants": runs,
        "e2e": e2e,
        "gpu_launches": args.steps,
        "clocks": head["clocks"],
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end C-ABI run")
    ap.add_argument("--variant", choices=["all", "f32", "f16s", "bf16s", "ref"], default="all",
                    help="which device runs to do (profiling uses one)")
    args = ap.parse_args()
    world, rank, local = dist_setup(args.gpus)
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
