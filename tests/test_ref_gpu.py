"""Reference-mode parity: the fused CUDA step against the CPU restatement of
the reference's four passes.  Both evaluate every float operation in the
same order with the same rounding, so the expected difference is zero; the
bar written in each test is bit equality (and at least 1e-5 relative)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ref_pair(lbm, oracle, shape, mask=None, tau=0.6, u_inf=(0.0, 0.0, 0.0), io=1, fs=1, ur=1,
              rho=None, u=None):
    d = lbm.default_desc(nx=shape[0], ny=shape[1], nz=shape[2], tau=tau, u_inf=u_inf,
                         ref_inlet_outlet=io, ref_free_slip=fs, ref_u_round=ur)
    lat = lbm.Lattice(d)
    st = oracle.RefState(shape, tau=tau, u_inf=u_inf, inlet_outlet=io, free_slip=fs, u_round=ur,
                         mask=mask)
    if mask is not None:
        lat.set_flags(mask)
    if rho is None:
        lat.init_equilibrium(1.0, u_inf)
        st.init(1.0, u_inf)
    else:
        lat.init_from_moments(rho, np.ascontiguousarray(u.T))
        st.init(rho=rho, u=u)
    return lat, st


def _assert_same(lat, st, label=""):
    rho, u = lat.read_moments()
    # the stated bar: 1e-5 relative on rho and u ...
    scale_u = max(np.abs(st.u).max(), 1e-30)
    assert np.max(np.abs(rho - st.rho)) <= 1e-5 * np.abs(st.rho).max(), label
    assert np.max(np.abs(u.T - st.u)) <= 1e-5 * scale_u, label
    # ... and in fact bit equality
    assert np.array_equal(rho, st.rho), label
    assert np.array_equal(u.T, st.u), label
    assert np.array_equal(lat.read_populations(), st.collided()), label


def _random_moments(n, seed, amp=0.03):
    rng = np.random.default_rng(seed)
    rho = (1 + 0.01 * rng.standard_normal(n)).astype(np.float32)
    u = (amp * rng.standard_normal((3, n))).astype(np.float32)
    return rho, u


@pytest.mark.parametrize("shape", [(8, 6, 5), (13, 7, 9)])
@pytest.mark.parametrize("io,fs", [(1, 1), (0, 0), (1, 0), (0, 1)])
def test_small_grids_all_regimes(gpu, oracle, shape, io, fs):
    n = int(np.prod(shape))
    rng = np.random.default_rng(n + 10 * io + fs)
    mask = (rng.random(n) < 0.12).astype(np.uint8)
    mask[rng.random(n) < 0.03] = 2  # not 1 -> fluid, as mask_at(c) == 1u
    rho, u = _random_moments(n, n)
    lat, st = _ref_pair(gpu, oracle, shape, mask, u_inf=(0.05, 0.01, -0.005), io=io, fs=fs,
                        rho=rho, u=u)
    _assert_same(lat, st, "init")
    for k in (1, 2, 7):
        lat.step(k)
        st.step(k)
        _assert_same(lat, st, f"after {k}")
    lat.close()


@pytest.mark.parametrize("ur", [0, 1, 2])
def test_u_rounding_modes(gpu, oracle, ur):
    shape = (10, 8, 6)
    rho, u = _random_moments(int(np.prod(shape)), 3)
    lat, st = _ref_pair(gpu, oracle, shape, u_inf=(0.04, 0.0, 0.0), ur=ur, rho=rho, u=u)
    lat.step(20)
    st.step(20)
    _assert_same(lat, st, f"u_round={ur}")
    lat.close()


def test_naca_preset_1000_steps(gpu, oracle):
    """Preset 0 (NACA0012, AoA 4 deg, |u| 0.04, tau 0.6; src/main.cpp:131)
    through apply_preset on a 96x48x8 tunnel, 1000 steps."""
    shape = (96, 48, 8)
    d = gpu.preset_desc(0, *shape)
    lat = gpu.Lattice(d)
    mask = gpu.apply_preset(lat, 0)
    assert mask.sum() > 0
    st = oracle.RefState(shape, tau=d.tau, u_inf=tuple(d.u_inf), mask=mask)
    st.init(1.0, tuple(d.u_inf))
    lat.step(1000)
    st.step(1000)
    _assert_same(lat, st, "naca 1000")
    lat.close()


def test_cavity_64_regimes_off_1000_steps(gpu, oracle):
    """64^3 box closed by the out-of-bounds-as-solid bounce-back (regimes 3 and
    4 off), started from a smooth vortex, 1000 steps."""
    shape = (64, 64, 64)
    n = 64 ** 3
    x = (np.arange(64) + 0.5) / 64
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = np.stack([0.05 * np.sin(np.pi * X) * np.cos(np.pi * Y) * np.sin(np.pi * Z),
                  -0.05 * np.cos(np.pi * X) * np.sin(np.pi * Y) * np.sin(np.pi * Z),
                  np.zeros_like(X)]).reshape(3, n).astype(np.float32)
    rho = np.ones(n, np.float32)
    lat, st = _ref_pair(gpu, oracle, shape, io=0, fs=0, rho=rho, u=u)
    lat.step(1000)
    st.step(1000)
    _assert_same(lat, st, "cavity 1000")
    lat.close()


def test_classification_bit_exact(gpu, oracle):
    shape = (33, 17, 9)
    n = int(np.prod(shape))
    rng = np.random.default_rng(1)
    mask = rng.integers(0, 3, n).astype(np.uint8)
    lat = gpu.Lattice(nx=shape[0], ny=shape[1], nz=shape[2])
    lat.set_flags(mask)
    assert np.array_equal(lat.read_classification(), oracle.classify(mask, shape))
    naca = gpu.voxelize_naca("4412", *shape, 0.25, 0.25, 6.0)
    lat.set_flags(naca)
    assert np.array_equal(lat.read_classification(), oracle.classify(naca, shape))
    lat.close()


def test_conservation_and_formats(gpu, oracle):
    shape = (16, 12, 10)
    n = int(np.prod(shape))
    rho, u = _random_moments(n, 9)
    lat, st = _ref_pair(gpu, oracle, shape, io=0, fs=0, rho=rho, u=u)
    lat.step(5)
    r32, u32 = lat.read_moments(gpu.U_F32X3)
    _, u4 = lat.read_moments(gpu.U_F32X4)
    _, h4 = lat.read_moments(gpu.U_F16X4)
    assert np.array_equal(u4[:, :3], u32) and np.all(u4[:, 3] == 0)
    assert np.array_equal(h4[:, :3].view(np.float16), u32.astype(np.float16))
    assert np.array_equal(gpu.half_to_float(h4[:, :3]), u32.astype(np.float16).astype(np.float32))
    s = lat.conservation()
    r64 = r32.astype(np.float64)
    want = [r64.sum()] + [(r64 * u32[:, a]).sum() for a in range(3)]
    assert np.allclose(s, want, rtol=1e-12, atol=1e-12)
    lat.close()


def test_resume_from_rgba16f_capture(gpu, oracle):
    """init_from_moments with the capture's rgba16f velocity buffer equals an
    init from the decoded floats (the resume the reference's F9 intends)."""
    shape = (12, 10, 8)
    n = int(np.prod(shape))
    rho, u = _random_moments(n, 21)
    h = np.zeros((n, 4), np.float16)
    h[:, :3] = u.T.astype(np.float16)
    a = gpu.Lattice(nx=12, ny=10, nz=8, u_inf=(0.03, 0, 0))
    a.init_from_moments(rho, h.view(np.uint16), gpu.U_F16X4)
    b = gpu.Lattice(nx=12, ny=10, nz=8, u_inf=(0.03, 0, 0))
    b.init_from_moments(rho, np.ascontiguousarray(h[:, :3].astype(np.float32)))
    a.step(3)
    b.step(3)
    assert np.array_equal(a.read_populations(), b.read_populations())
    a.close()
    b.close()


def test_errors_and_status(gpu):
    lat = gpu.Lattice(nx=8, ny=8, nz=8)
    with pytest.raises(gpu.LbmError) as e:
        lat.step(1)
    assert e.value.code == gpu.ERR_STATE
    with pytest.raises(gpu.LbmError):
        lat.set_flags(np.zeros(7, np.uint8))
    lat.init_equilibrium(1.0, (0.0, 0.0, 0.0))
    with pytest.raises(gpu.LbmError):
        lat.step(-1)
    # a non-finite density planted by the host is reported, not trapped
    rho = np.ones(512, np.float32)
    rho[100] = np.nan
    lat.init_from_moments(rho, np.zeros((512, 3), np.float32))
    lat.step(2)
    with pytest.raises(gpu.LbmError) as e:
        lat.sync()
    assert e.value.code == gpu.ERR_NONFINITE
    lat.sync()  # status cleared after it was reported
    lat.close()


def test_deterministic(gpu):
    outs = []
    for _ in range(2):
        lat = gpu.Lattice(gpu.preset_desc(1, 64, 32, 8))
        gpu.apply_preset(lat, 1)
        lat.step(50)
        outs.append(lat.read_populations())
        lat.close()
    assert np.array_equal(outs[0], outs[1])
