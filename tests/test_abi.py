"""The C ABI library on the CPU: it loads, exports every symbol the header
declares, validates arguments, and its host-only helpers are correct."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, cuda_available


def header_symbols():
    text = "".join(h.read_text() for h in sorted((ROOT / "include").glob("*.h")))
    return sorted(set(re.findall(r"LBM_API\s+[\w\s\*]+?\b(lbm_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(lbm_lib):
    lib = C.CDLL(str(lbm_lib.LIB_PATH))
    syms = header_symbols()
    assert len(syms) >= 50
    assert "lbm_trainer_fit" in syms and "lbm_set_closure" in syms
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # the Python layer binds every symbol too
    assert set(syms) <= set(lbm_lib._SIGS)


def test_build_info(lbm_lib):
    assert "sm_100a" in lbm_lib.build_info()


def test_tables_match_golden(lbm_lib, golden):
    c, w, opp = lbm_lib.lattice_tables()
    assert c.tolist() == golden["velocity_set"]
    assert opp.tolist() == golden["opposite_index"]
    assert np.array_equal(w, np.array(golden["weights"], np.float32))


def test_desc_validation_without_device(lbm_lib):
    bad = [dict(nx=1), dict(tau=0.5), dict(mode=7), dict(precision=9),
           dict(mode=lbm_lib.MODE_REFERENCE, precision=lbm_lib.PREC_F16S),
           dict(mode=lbm_lib.MODE_REFERENCE, periodic=(1, 0, 0)),
           dict(ref_u_round=5), dict(nx=65536), dict(ny=70000, nx=2), dict(nz=-3)]
    for kw in bad:
        with pytest.raises(lbm_lib.LbmError) as e:
            lbm_lib.Lattice(**kw)
        assert e.value.code in (lbm_lib.ERR_INVALID_ARG, lbm_lib.ERR_UNSUPPORTED), kw


def test_struct_size_checked(lbm_lib):
    d = lbm_lib.default_desc()
    d.struct_size = 12
    h = C.c_void_p()
    assert lbm_lib.load().lbm_create(C.byref(d), C.byref(h)) == lbm_lib.ERR_INVALID_ARG


@pytest.mark.skipif(cuda_available(), reason="checks the no-device error path")
def test_create_without_device_reports_no_device(lbm_lib):
    with pytest.raises(lbm_lib.LbmError) as e:
        lbm_lib.Lattice()
    assert e.value.code == lbm_lib.ERR_NO_DEVICE


def test_null_arguments(lbm_lib):
    lib = lbm_lib.load()
    assert lib.lbm_create(None, None) == lbm_lib.ERR_INVALID_ARG
    assert lib.lbm_step(None, 1) == lbm_lib.ERR_INVALID_ARG
    assert lib.lbm_destroy(None) == lbm_lib.OK
    assert lib.lbm_last_error(None)


def test_half_to_float_all_patterns(lbm_lib):
    h = np.arange(65536, dtype=np.uint32).astype(np.uint16)
    got = lbm_lib.half_to_float(h)
    want = h.view(np.float16).astype(np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)) or np.array_equal(got, want, equal_nan=True)
    finite = np.isfinite(want)
    assert np.array_equal(got[finite].view(np.uint32), want[finite].view(np.uint32))


@pytest.mark.parametrize("preset", [0, 1, 2])
@pytest.mark.parametrize("shape", [(128, 128, 2), (96, 40, 3)])
def test_voxeliser_matches_oracle(lbm_lib, oracle, preset, shape):
    p = lbm_lib.PRESETS[preset]
    got = lbm_lib.voxelize_naca(p.naca, *shape, 0.25, 0.25, p.angle_of_attack_deg)
    want = oracle.voxelize_naca(p.naca, *shape, 0.25, 0.25, p.angle_of_attack_deg)
    assert got.sum() > 0
    assert np.array_equal(got, want)
    # extruded in z
    m = got.reshape(shape[::-1])
    assert all(np.array_equal(m[0], m[k]) for k in range(shape[2]))


def test_voxeliser_rejects_bad_input(lbm_lib):
    with pytest.raises(lbm_lib.LbmError):
        lbm_lib.voxelize_naca("00x2", 8, 8, 1)


def test_round_bf16_nearest_even(lbm_lib):
    rng = np.random.default_rng(4)
    x = np.concatenate([rng.standard_normal(20000).astype(np.float32) * 10.0 ** rng.integers(-30, 30, 20000),
                        np.array([0.0, -0.0, 1.0, 3.4e38, -3.4e38, 1e-40, np.inf, -np.inf], np.float32)]).astype(np.float32)
    got = lbm_lib.round_bf16(x)
    # nearest-even on the upper 16 bits: the result is the closer of the two
    # bf16 neighbours, and on a tie the one with an even last bit
    b = x.view(np.uint32).astype(np.uint64)
    lo = (b & 0xFFFF0000).astype(np.uint32).view(np.float32).astype(np.float64)
    hi = ((b & 0xFFFF0000) + 0x10000).astype(np.uint32).view(np.float32).astype(np.float64)
    finite = np.isfinite(x) & np.isfinite(hi)
    xd = x.astype(np.float64)
    dl, dh = np.abs(xd - lo), np.abs(hi - xd)
    pick_hi = (dh < dl) | ((dh == dl) & (((b >> 16) & 1) == 1))
    want = np.where(pick_hi, hi, lo)
    assert np.array_equal(got[finite].astype(np.float64), want[finite])
    assert np.array_equal(got[~np.isfinite(x)], x[~np.isfinite(x)])


def test_closure_argument_checks_without_device(lbm_lib):
    lib = lbm_lib.load()
    assert lib.lbm_set_closure(None, None) == lbm_lib.ERR_INVALID_ARG
    assert lib.lbm_box_filter(None, None, 8, 8, 8, 2, None, None) == lbm_lib.ERR_INVALID_ARG
    assert lib.lbm_closure_predict(None, None, 1, None, None) == lbm_lib.ERR_INVALID_ARG
    assert lib.lbm_trainer_create(None, None, None) == lbm_lib.ERR_INVALID_ARG
    assert lib.lbm_trainer_destroy(None) == lbm_lib.OK
    assert lib.lbm_trainer_fit(None, None, None, None, 1, 1, 1, 0, None) == lbm_lib.ERR_INVALID_ARG
    assert lib.lbm_trainer_last_error(None)
    a = lbm_lib.adam_default()
    assert a.struct_size == C.sizeof(lbm_lib.Adam) and abs(a.lr - 1e-3) < 1e-9
    # a factor that does not divide the grid is refused before any launch
    p = C.c_void_p(16)
    assert lib.lbm_box_filter(p, p, 9, 8, 8, 2, p, None) == lbm_lib.ERR_INVALID_ARG
