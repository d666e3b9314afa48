"""Capture directories on the CPU (host-only writer and reader): the
writer's state.json is pinned by the committed fixture, the files read back
through the reference's own Python StateReader as recorded by
tests/golden/make_capture_golden.py, and malformed captures are refused
with LBM_ERR_IO."""
import json
import os
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT

GOLD = ROOT / "tests" / "golden" / "capture"


def _fixture_inputs():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_capture_golden", ROOT / "tests" / "golden" / "make_capture_golden.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_state_json_matches_fixture(lbm_lib, tmp_path):
    g = _fixture_inputs()
    rho, vel, mask, pops = g.sample_fields()
    lbm_lib.capture_write(str(tmp_path), 12, g.SHAPE, rho, vel, mask, pops, meta=g.META)
    got = (tmp_path / "capture_0012" / "state.json").read_text()
    assert got == (GOLD / "state.json").read_text()


def test_reference_reader_view(lbm_lib, tmp_path):
    """What the reference's StateReader saw in the fixture capture (dtype by
    format, element counts, sums) equals what the same files give now."""
    g = _fixture_inputs()
    rho, vel, mask, pops = g.sample_fields()
    lbm_lib.capture_write(str(tmp_path), 12, g.SHAPE, rho, vel, mask, pops, meta=g.META)
    view = json.loads((GOLD / "reference_reader_view.json").read_text())
    cap = tmp_path / "capture_0012"
    state = json.loads((cap / "state.json").read_text())
    assert state["meta"] == view["meta"] and state["frame"] == view["frame"]
    fmt_dtype = {"r32f": np.float32, "rgba16f": np.float16}
    for b in state["buffers"]:
        v = view["buffers"][b["name"]]
        arr = np.fromfile(cap / b["file"], dtype=fmt_dtype.get(b["format"], np.float32))
        assert str(arr.dtype) == v["dtype"] and arr.size == v["size"]
        assert arr.astype(np.float64).sum() == pytest.approx(v["sum"], rel=1e-12, abs=1e-40)
    # the reader reshapes populations by its shape field
    assert view["buffers"]["populations"]["reshaped"] == [19, *g.SHAPE]


def test_roundtrip_and_latest(lbm_lib, tmp_path):
    shape = (5, 3, 2)
    n = 30
    rng = np.random.default_rng(1)
    rho = rng.random(n).astype(np.float32)
    vel = rng.standard_normal((n, 4)).astype(np.float16)
    mask = (rng.random(n) < 0.3).astype(np.uint8)
    meta = {"Nx": 5, "Ny": 3, "Nz": 2, "iteration": 99, "note": "quote \" slash \\ tab \t é ∑ 😀"}
    for frame in (3, 10, 7):
        lbm_lib.capture_write(str(tmp_path), frame, shape, rho * frame, vel, mask, meta=meta)
    latest = lbm_lib.capture_latest(str(tmp_path))
    assert latest.endswith("capture_0010")
    c = lbm_lib.capture_read(latest)
    assert c["shape"] == shape and c["frame"] == 10 and c["iteration"] == 99
    assert c["mask_frame_invariant"] and c["populations"] is None
    assert np.array_equal(c["density"], rho * 10)
    assert np.array_equal(c["velocity"], vel.view(np.uint16))
    assert np.array_equal(c["obstacle_mask"], mask)
    state = json.loads((Path(latest) / "state.json").read_text())
    assert state["meta"]["latticeBoltzmann"]["note"] == meta["note"]


def test_malformed_captures_are_io_errors(lbm_lib, tmp_path):
    shape = (4, 4, 4)
    n = 64
    lbm_lib.capture_write(str(tmp_path), 1, shape, np.ones(n), np.zeros((n, 4), np.float16),
                          np.zeros(n, np.uint8), meta={"Nx": 4, "Ny": 4, "Nz": 4})
    cap = tmp_path / "capture_0001"
    # truncated buffer
    data = (cap / "density.bin").read_bytes()
    (cap / "density.bin").write_bytes(data[:-4])
    with pytest.raises(lbm_lib.LbmError) as e:
        lbm_lib.capture_read(str(cap))
    assert e.value.code == lbm_lib.ERR_IO
    (cap / "density.bin").write_bytes(data)
    lbm_lib.capture_read(str(cap))
    # broken JSON, missing meta, missing directory
    text = (cap / "state.json").read_text()
    for bad in (text[:-3], text.replace('"latticeBoltzmann"', '"other"'), "[1, 2", ""):
        (cap / "state.json").write_text(bad)
        with pytest.raises(lbm_lib.LbmError) as e:
            lbm_lib.capture_read(str(cap))
        assert e.value.code == lbm_lib.ERR_IO
    with pytest.raises(lbm_lib.LbmError) as e:
        lbm_lib.capture_read(str(tmp_path / "nope"))
    assert e.value.code == lbm_lib.ERR_IO
    with pytest.raises(lbm_lib.LbmError) as e:
        lbm_lib.capture_latest(str(tmp_path / "empty_root_that_is_missing"))
    assert e.value.code == lbm_lib.ERR_IO
    # a meta that is not a JSON object is refused by the writer
    rc = lbm_lib.load().lbm_capture_write(str(tmp_path).encode(), 2, b"[1]", 4, 4, 4,
                                          np.ones(n, np.float32).ctypes.data,
                                          np.zeros(4 * n, np.uint16).ctypes.data,
                                          np.zeros(n, np.uint8).ctypes.data, None)
    assert rc == lbm_lib.ERR_INVALID_ARG
