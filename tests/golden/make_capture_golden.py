"""Regenerates the capture-format fixtures under tests/golden/capture/.

Run where the reference tree is available, after building the library, giving its path
as the argument or in $GPU_SIMS_REFERENCE:

    python tests/golden/make_capture_golden.py <reference tree>

It writes a small capture (6x4x3 lattice, seeded moments, a mask and a
full-state population buffer) with this library's host-only writer
lbm_capture_write, then reads it back with the reference's own Python
StateReader (common/common-py/gpusims_common/state_reader.py) and records
what that reader sees: the meta block, every buffer's dtype, element count
and float64 sum, and the reshaped shapes.  The capture's state.json is kept
as `state.json`, and the reader's view as `reference_reader_view.json`.
Nothing here is needed at test time.
"""
from __future__ import annotations

import json
import os
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
def _reference_root() -> Path:
    """The reference tree: the first argument, else $GPU_SIMS_REFERENCE."""
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPU_SIMS_REFERENCE")
    if not arg:
        raise SystemExit("give the reference tree's path as the argument or in $GPU_SIMS_REFERENCE")
    return Path(arg)
OUT = HERE / "capture"

SHAPE = (6, 4, 3)
META = {"schemaVersion": 1, "tierIndex": 1, "presetIndex": 0, "Nx": 6, "Ny": 4, "Nz": 3,
        "tau": 0.6, "substeps": 1, "uInfMagnitude": 0.04, "angleOfAttackDeg": 4.0,
        "iteration": 4321, "camera": {"distance": 2.5, "pitch": 0.3, "yaw": -0.7}}


def sample_fields():
    """The seeded inputs of the fixture (also rebuilt by the tests)."""
    n = int(np.prod(SHAPE))
    rng = np.random.default_rng(2024)
    rho = (1 + 0.01 * rng.standard_normal(n)).astype(np.float32)
    vel = np.zeros((n, 4), np.float16)
    vel[:, :3] = (0.04 * rng.standard_normal((n, 3))).astype(np.float16)
    mask = (rng.random(n) < 0.2).astype(np.uint8)
    pops = rng.random((19, n)).astype(np.float32)
    return rho, vel, mask, pops


def main() -> int:
    REF = _reference_root()
    sys.path.insert(0, str(ROOT / "gpu-sims_b200"))
    import types
    import lbm
    # the package's __init__ pulls in the renderer (taichi); the reader and
    # its logger are loaded on their own under a bare package module
    pkg = types.ModuleType("gpusims_common")
    pkg.__path__ = [str(REF / "common" / "common-py" / "gpusims_common")]
    sys.modules["gpusims_common"] = pkg
    from gpusims_common.state_reader import StateReader

    tmp = Path(tempfile.mkdtemp())
    try:
        rho, vel, mask, pops = sample_fields()
        lbm.capture_write(str(tmp), 12, SHAPE, rho, vel, mask, pops, meta=META)
        reader = StateReader(tmp)
        cap = reader.find_latest()
        state = reader.load_meta(cap)
        view = {"frame": state["frame"], "meta": state["meta"], "buffers": {}}
        for b in state["buffers"]:
            arr = reader.load_buffer(cap, b["name"])
            shaped = reader.load_buffer_reshaped(cap, b["name"])
            view["buffers"][b["name"]] = {"dtype": str(arr.dtype), "size": int(arr.size),
                                          "sum": float(arr.astype(np.float64).sum()),
                                          "reshaped": list(shaped.shape)}
        OUT.mkdir(parents=True, exist_ok=True)
        shutil.copy(cap / "state.json", OUT / "state.json")
        (OUT / "reference_reader_view.json").write_text(json.dumps(view, indent=1, sort_keys=True) + "\n")
    finally:
        shutil.rmtree(tmp)
    print("wrote", OUT)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
