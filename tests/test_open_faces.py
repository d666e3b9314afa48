"""Open x faces (Zou-He velocity inlet / pressure outlet) in the FP64 oracle,
on the CPU: the rebuilt populations return the prescribed moments exactly,
a duct reaches a steady state whose mass flux is the same through every
x plane, and descriptors that cannot have open faces are refused before a
device is touched."""
import numpy as np
import pytest

U_IN = 0.04


def duct(oracle, shape, kinds=(1, 2), rho_out=1.0, rho_in=1.0, tau=0.8, periodic=(0, 0, 1), coll=0,
         mask=None, accel=(0.0, 0.0, 0.0)):
    wall = np.zeros((6, 3))
    if kinds[0] == 1:
        wall[0] = (U_IN, 0.0, 0.0)
    if kinds[1] == 1:
        wall[1] = (U_IN, 0.0, 0.0)
    open_rho = (rho_in if kinds[0] == 2 else 0.0, rho_out if kinds[1] == 2 else 0.0)
    st = oracle.ExtState(shape, periodic=periodic, tau=tau, collision=coll, wall=wall, mask=mask,
                         open_x=kinds, open_rho=open_rho, accel=accel)
    st.init(1.0, np.zeros(3))
    return st


def face_nodes(shape, x):
    nx, ny, nz = shape
    z, y = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
    return (x + nx * (y + ny * z)).reshape(-1)


def test_rebuilt_populations_carry_the_prescribed_moments(oracle):
    shape = (12, 6, 4)
    st = duct(oracle, shape, kinds=(1, 2), rho_out=0.995)
    rng = np.random.default_rng(3)
    for _ in range(3):
        st.f += 1e-4 * rng.standard_normal(st.f.shape)  # arbitrary incoming states
        st.step(1)
        inlet = face_nodes(shape, 0)
        outlet = face_nodes(shape, shape[0] - 1)
        # moments of the rebuilt (pre-collision) populations = those of the
        # collided ones (the collision conserves rho and rho u)
        assert np.allclose(st.u[0, inlet], U_IN, rtol=0, atol=1e-14)
        assert np.allclose(st.u[1:, inlet], 0.0, rtol=0, atol=1e-14)
        assert np.allclose(st.rho[outlet], 0.995, rtol=0, atol=1e-14)
        assert np.allclose(st.u[1:, outlet], 0.0, rtol=0, atol=1e-14)


def plane_flux(st, shape):
    nx, ny, nz = shape
    return (st.rho.reshape(nz, ny, nx) * st.u[0].reshape(nz, ny, nx)).sum(axis=(0, 1))


def two_step_flux(st, shape):
    """Mass flux sum rho u_x through every x plane, averaged over two
    consecutive steps, and the half difference.  The impulsive start excites
    the lattice's staggered momentum mode (u_x alternating in x and in t, the
    same at every y and z), which neither BGK nor TRT damps: it stays at about
    1 % of the flux.  The two-step average removes it."""
    a = plane_flux(st, shape)
    st.step(1)
    b = plane_flux(st, shape)
    return 0.5 * (a + b), 0.5 * (a - b)


@pytest.mark.parametrize("coll", [0, 1])
def test_duct_reaches_a_steady_mass_flux(oracle, coll):
    """Velocity inlet, pressure outlet, no-slip walls in y, periodic z: the
    mass flux through every x plane agrees at steady state (to 1e-6 of it),
    and the outflow profile is symmetric about the duct's axis and peaks
    there."""
    shape = (40, 12, 2)
    nx, ny, nz = shape
    st = duct(oracle, shape, coll=coll)
    st.step(6000)
    flux, stag = two_step_flux(st, shape)
    assert np.all(flux > 0)
    assert (flux.max() - flux.min()) / flux.mean() < 1e-6, flux
    # the inflow is rho u_in summed over the inlet plane
    inlet_rho = st.rho[face_nodes(shape, 0)].sum()
    assert np.isclose(flux.mean(), U_IN * inlet_rho, rtol=1e-5)
    prof = st.u[0].reshape(nz, ny, nx)[0, :, nx - 1]
    assert np.allclose(prof, prof[::-1], rtol=1e-9, atol=1e-15)
    assert prof[ny // 2] > prof[0]


def test_pressure_driven_duct(oracle):
    """Pressure at both faces: flow runs from high to low density with a
    linear density drop and a uniform mass flux."""
    shape = (32, 10, 2)
    nx, ny, nz = shape
    st = duct(oracle, shape, kinds=(2, 2), rho_in=1.003, rho_out=0.997)
    st.step(2000)
    flux, _ = two_step_flux(st, shape)
    assert np.all(flux > 0)
    assert (flux.max() - flux.min()) / flux.mean() < 1e-6
    assert np.allclose(st.rho[face_nodes(shape, 0)], 1.003, atol=1e-14)
    assert np.allclose(st.rho[face_nodes(shape, nx - 1)], 0.997, atol=1e-14)
    mean_rho = st.rho.reshape(nz, ny, nx).mean(axis=(0, 1))
    assert np.all(np.diff(mean_rho) < 0)


def test_open_face_descriptor_rules(lbm_lib):
    bad = [dict(mode=lbm_lib.MODE_PHYSICS, open_x=(3, 0)),
           dict(mode=lbm_lib.MODE_PHYSICS, open_x=(1, 0), periodic=(1, 0, 0)),
           dict(mode=lbm_lib.MODE_REFERENCE, open_x=(1, 0)),
           dict(mode=lbm_lib.MODE_PHYSICS, open_x=(0, 2), open_rho=(0.0, 0.0)),
           dict(mode=lbm_lib.MODE_PHYSICS, open_x=(0, 2), open_rho=(0.0, float("nan"))),
           dict(mode=lbm_lib.MODE_PHYSICS, open_x=(1, 0), wall_velocity=[(0.6, 0, 0)] + [(0, 0, 0)] * 5)]
    for kw in bad:
        with pytest.raises(lbm_lib.LbmError) as e:
            lbm_lib.Lattice(**kw)
        assert e.value.code in (lbm_lib.ERR_INVALID_ARG, lbm_lib.ERR_UNSUPPORTED), kw
    d = lbm_lib.default_desc(mode=lbm_lib.MODE_PHYSICS, nx=8, ny=8, nz=8, open_x=(1, 2), open_rho=(0.0, 1.0))
    with pytest.raises(lbm_lib.LbmError) as e:
        lbm_lib.Batch([d])
    assert e.value.code == lbm_lib.ERR_UNSUPPORTED
