"""The C++ host program (gpu-sims_b200/host/lbm_frame_loop.cpp) over the C
ABI: it builds with g++ against include/lbm.h and the library, and on the
GPU its frame loop -- the device-made NACA preset mask, the equilibrium
init, a tau / u_inf slider change between frames (lbm_set_params), substeps,
the per-frame fp64 sums, the VDB export -- gives the restated four-pass
reference step's moments bit for bit."""
import json
import math
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT


def _build(tmp_path, lbm_lib):
    sys.path.insert(0, str(ROOT / "gpu-sims_b200"))
    import build
    return build.build_host(lib=lbm_lib.LIB_PATH, out=tmp_path / "lbm_frame_loop")


def _u_inf(mag, aoa_deg):
    """update_u_inf_vector (src/main.cpp:1155-1160) in float."""
    a = np.float32(aoa_deg) * np.float32(0.01745329251994329576923690768489)
    return (float(np.float32(mag) * np.float32(math.cos(a))), float(np.float32(mag) * np.float32(math.sin(a))),
            0.0)


def test_host_program_builds_and_checks_its_arguments(lbm_lib, tmp_path):
    exe = _build(tmp_path, lbm_lib)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_host_frame_loop_matches_the_reference_step(gpu, oracle, tmp_path):
    from oracle import vdb_oracle
    exe = _build(tmp_path, gpu)
    shape, frames, substeps, change = (96, 48, 8), 12, 3, 5
    p = gpu.PRESETS[0]
    u1 = _u_inf(p.u_inf, p.angle_of_attack_deg)
    tau2, u2 = 0.7, _u_inf(0.05, 8.0)
    f9 = lambda v: "%.9g" % v  # noqa: E731  (float round trip)
    out = tmp_path / "run"
    vdb = tmp_path / "vdb"
    vdb.mkdir()
    args = [str(exe), *map(str, shape), p.naca, f9(p.angle_of_attack_deg), f9(p.tau), *map(f9, u1),
            str(frames), str(substeps), str(change), f9(tau2), *map(f9, u2), str(out), str(vdb)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["iteration"] == frames * substeps
    n = int(np.prod(shape))
    rho = np.fromfile(f"{out}.rho.bin", np.float32)
    u = np.fromfile(f"{out}.u.bin", np.float32).reshape(n, 3)
    mask = np.fromfile(f"{out}.mask.bin", np.uint8)
    # the device-made mask is the host voxeliser's
    assert np.array_equal(mask, gpu.voxelize_naca(p.naca, *shape, gpu.AIRFOIL_CHORD_LENGTH_FRAC,
                                                  gpu.AIRFOIL_CHORD_CENTER_X_FRAC, p.angle_of_attack_deg))
    st = oracle.RefState(shape, tau=p.tau, u_inf=u1, mask=mask)
    st.init(1.0, u1)
    st.step(change * substeps)
    st.set_params(tau=tau2, u_inf=u2)
    st.step((frames - change) * substeps)
    assert np.array_equal(rho, st.rho) and np.array_equal(u.T, st.u)
    # the last frame's fp64 sums are those of the moments read back
    fluid = mask != 1
    r64, u64 = rho.astype(np.float64), u.astype(np.float64)
    want = [r64[fluid].sum()] + [(r64 * u64[:, a])[fluid].sum() for a in range(3)]
    assert np.allclose(res["sums"][-1], want, rtol=1e-12, atol=1e-12)
    # the VDB export of the last frame holds the rgba16f velocity as floats
    g = vdb_oracle.read(str(vdb / f"velocity_{frames - 1:06d}.vdb"))["grids"][0]
    vals, act = vdb_oracle.dense(g, shape)
    h = np.ascontiguousarray(u, np.float16).astype(np.float32)  # round to binary16, nearest even
    assert act.all() and np.array_equal(vals, h)
