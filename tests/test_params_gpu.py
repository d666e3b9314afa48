"""Live solver parameters (lbm_set_params) between steps.

The reference re-uploads tau and u_inf as uniforms before every frame
(src/main.cpp:1523-1537) from its sliders (:1648, :1657-1661), so a change
takes effect at the next collide and the next boundary pass with the flow
state kept.  Reference mode must stay bit-identical to the restated four-pass
step with the same change made between frames; physics mode is held to the
FP64 oracle at the physics-mode bar (3e-5 of the velocity scale, 1e-5 in rho)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from test_phys_gpu import compare, make_pair, sphere_mask  # noqa: E402
from test_ref_gpu import _assert_same  # noqa: E402


def _naca_pair(lbm, oracle, shape=(96, 48, 8)):
    d = lbm.preset_desc(0, *shape)
    lat = lbm.Lattice(d)
    mask = lbm.apply_preset(lat, 0)
    st = oracle.RefState(shape, tau=d.tau, u_inf=tuple(d.u_inf), mask=mask)
    st.init(1.0, tuple(d.u_inf))
    return lat, st


def test_reference_mode_tau_and_u_inf_mid_run(gpu, oracle):
    """Two slider changes between frames of different lengths (graph and
    single launches), bit for bit against the restated step."""
    lat, st = _naca_pair(gpu, oracle)
    lat.step(37)
    st.step(37)
    _assert_same(lat, st, "before")
    lat.set_params(tau=0.7, u_inf=(0.03, 0.004, 0.0))
    st.set_params(tau=0.7, u_inf=(0.03, 0.004, 0.0))
    p = lat.params()
    assert p.tau == np.float32(0.7) and tuple(p.u_inf) == tuple(np.float32([0.03, 0.004, 0.0]))
    _assert_same(lat, st, "right after the change")
    lat.step(41)
    st.step(41)
    _assert_same(lat, st, "41 steps after the first change")
    # u_inf alone (no collision to recompute), then tau twice with no step between
    lat.set_params(u_inf=(0.045, -0.002, 0.001))
    st.set_params(u_inf=(0.045, -0.002, 0.001))
    lat.step(5)
    st.step(5)
    lat.set_params(tau=0.65)
    lat.set_params(tau=0.9)
    st.set_params(tau=0.9)
    lat.step(20)
    st.step(20)
    _assert_same(lat, st, "after the second and third change")
    lat.close()


def test_reference_mode_tau_change_before_first_step(gpu, oracle):
    """A change right after init recomputes the init's collision."""
    shape = (24, 12, 6)
    n = int(np.prod(shape))
    rng = np.random.default_rng(3)
    rho = (1 + 0.01 * rng.standard_normal(n)).astype(np.float32)
    u = (0.03 * rng.standard_normal((3, n))).astype(np.float32)
    d = gpu.default_desc(nx=shape[0], ny=shape[1], nz=shape[2], tau=0.6, u_inf=(0.04, 0, 0))
    lat = gpu.Lattice(d)
    st = oracle.RefState(shape, tau=0.6, u_inf=(0.04, 0, 0))
    lat.init_from_moments(rho, np.ascontiguousarray(u.T))
    st.init(rho=rho, u=u)
    lat.set_params(tau=0.55)
    st.set_params(tau=0.55)
    _assert_same(lat, st, "after init")
    lat.step(18)
    st.step(18)
    _assert_same(lat, st, "18 steps")
    lat.close()


def test_reference_mode_rejects_physics_fields(gpu):
    lat = gpu.Lattice(nx=8, ny=8, nz=8)
    lat.init_equilibrium(1.0, (0.0, 0.0, 0.0))
    with pytest.raises(gpu.LbmError) as e:
        lat.set_params(body_accel=(1e-5, 0, 0))
    assert e.value.code == gpu.ERR_UNSUPPORTED
    with pytest.raises(gpu.LbmError) as e:
        lat.set_params(tau=0.5)
    assert e.value.code == gpu.ERR_INVALID_ARG
    assert lat.params().tau == np.float32(0.6)  # a rejected call changes nothing
    lat.close()


@pytest.mark.parametrize("precision,tol_u", [(0, 3e-5), (1, None)])
def test_physics_mode_tau_force_and_lid_mid_run(gpu, oracle, precision, tol_u):
    """Channel with a sphere and a body force; tau, the force and a moving
    wall change between calls, against the FP64 oracle with the same
    changes."""
    shape = (48, 16, 16)
    mask = sphere_mask(shape, (16, 8, 8), 4)
    rng = np.random.default_rng(7)
    u = 1e-3 * rng.standard_normal((3, int(np.prod(shape))))
    lat, st = make_pair(gpu, oracle, shape, periodic=(1, 0, 0), tau=0.55, accel=(1e-5, 0, 0),
                        mask=mask, u=u, precision=precision)
    lat.step(60)
    st.step(60)
    wall = np.zeros((6, 3))
    wall[gpu.FACE_ZP] = (0.02, 0.0, 0.0)
    lat.set_params(tau=0.62, body_accel=(2e-5, 1e-6, 0.0), wall_velocity=wall)
    st.set_params(tau=0.62, accel=(2e-5, 1e-6, 0.0), wall=wall)
    lat.step(100)
    st.step(100)
    if tol_u is not None:
        compare(lat, st, tol_u=tol_u)
    else:
        rho, uu = lat.read_moments()
        err = np.linalg.norm(uu.T - st.u) / np.linalg.norm(st.u)
        assert err < 2e-3, err
    # a step at the old parameters would differ: the change did take effect
    lat2, st2 = make_pair(gpu, oracle, shape, periodic=(1, 0, 0), tau=0.55, accel=(1e-5, 0, 0),
                          mask=mask, u=u, precision=precision)
    lat2.step(160)
    _, u_old = lat2.read_moments()
    _, u_new = lat.read_moments()
    assert np.abs(u_old - u_new).max() > 1e-3
    lat.close()
    lat2.close()
