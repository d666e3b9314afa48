"""Capture save / load through a lattice: a full-state capture resumes the
run bit for bit (both step modes), a moments-only load equals an
initialisation from the stored rgba16f moments (the reference's F9 intent),
and the mask and iteration counter come back."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lat(gpu, mode, shape=(24, 12, 10), precision=0):
    if mode == "physics":
        d = gpu.default_desc(nx=shape[0], ny=shape[1], nz=shape[2], mode=gpu.MODE_PHYSICS,
                             precision=precision, collision=gpu.COLL_TRT, periodic=(1, 0, 0),
                             tau=0.56, body_accel=(1e-5, 0, 0))
    else:
        d = gpu.default_desc(nx=shape[0], ny=shape[1], nz=shape[2], tau=0.6, u_inf=(0.04, 0.0, 0.0))
    return gpu.Lattice(d)


def _mask(shape):
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return (((x - 8) ** 2 + (y - 6) ** 2 + (z - 5) ** 2) <= 9).astype(np.uint8).reshape(-1)


@pytest.mark.parametrize("mode,precision", [("physics", 0), ("physics", 1), ("reference", 0)])
def test_full_state_capture_resumes_exactly(gpu, tmp_path, mode, precision):
    shape = (24, 12, 10)
    a = _lat(gpu, mode, shape, precision)
    mask = _mask(shape)
    a.set_flags(mask)
    a.init_equilibrium(1.0, (0.04, 0.0, 0.0) if mode == "reference" else (0.0, 0.0, 0.0))
    a.step(37)
    a.capture_save(str(tmp_path), 5, meta={"Nx": 24, "Ny": 12, "Nz": 10, "iteration": 37, "tau": 0.6},
                   full_state=True)
    b = _lat(gpu, mode, shape, precision)
    b.capture_load(gpu.capture_latest(str(tmp_path)), gpu.CAPTURE_LOAD_MASK)
    assert np.array_equal(b.read_mask(), mask)
    assert b.info().iteration == 37
    assert np.array_equal(a.read_populations(), b.read_populations())
    if mode == "physics":
        assert np.array_equal(a.read_populations_shifted(), b.read_populations_shifted())
    a.step(25)
    b.step(25)
    assert np.array_equal(a.read_populations(), b.read_populations())
    ra, ua = a.read_moments()
    rb, ub = b.read_moments()
    assert np.array_equal(ra, rb) and np.array_equal(ua, ub)
    a.close()
    b.close()


def test_moments_only_load_is_equilibrium_from_rgba16f(gpu, tmp_path):
    shape = (24, 12, 10)
    a = _lat(gpu, "physics", shape)
    a.set_flags(_mask(shape))
    a.init_equilibrium(1.0, (0.0, 0.0, 0.0))
    a.step(40)
    a.capture_save(str(tmp_path), 0, full_state=True)
    cap = gpu.capture_latest(str(tmp_path))
    b = _lat(gpu, "physics", shape)
    b.capture_load(cap, gpu.CAPTURE_LOAD_MASK | gpu.CAPTURE_MOMENTS_ONLY)
    c = _lat(gpu, "physics", shape)
    c.set_flags(_mask(shape))
    stored = gpu.capture_read(cap)
    c.init_from_moments(stored["density"], stored["velocity"], gpu.U_F16X4)
    assert np.array_equal(b.read_populations(), c.read_populations())
    # the default meta carries the iteration and the lattice's tau
    import json
    from pathlib import Path
    meta = json.loads((Path(cap) / "state.json").read_text())["meta"]["latticeBoltzmann"]
    assert meta["iteration"] == 40 and abs(meta["tau"] - 0.56) < 1e-6 and meta["Nx"] == 24
    for lat in (a, b, c):
        lat.close()


def test_load_refuses_other_dimensions(gpu, tmp_path):
    a = _lat(gpu, "physics", (24, 12, 10))
    a.init_equilibrium(1.0, (0.0, 0.0, 0.0))
    a.capture_save(str(tmp_path), 1)
    b = _lat(gpu, "physics", (24, 12, 12))
    with pytest.raises(gpu.LbmError) as e:
        b.capture_load(gpu.capture_latest(str(tmp_path)))
    assert e.value.code == gpu.ERR_INVALID_ARG
    with pytest.raises(gpu.LbmError):
        b.capture_load(gpu.capture_latest(str(tmp_path)), 8)  # unknown flag
    a.close()
    b.close()
