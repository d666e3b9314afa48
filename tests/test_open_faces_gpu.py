"""Open x faces (Zou-He velocity inlet / pressure outlet) on the GPU against
the FP64 oracle.  The kernels compute in fp32 on shifted populations, so
the bar is the physics-mode one: after a few hundred steps |du| within 3e-5
of the velocity scale and |drho| within 1e-5 (fp32 storage); fp16 / bf16
storage is held to a relative L2 velocity error of 2e-3 / 3e-2."""
import numpy as np
import pytest

from test_phys_gpu import compare, sphere_mask

pytestmark = pytest.mark.gpu

U_IN = 0.04


def open_pair(lbm, oracle, shape, kinds=(1, 2), rho_in=1.002, rho_out=0.998, periodic=(0, 0, 0), tau=0.6,
              collision=0, accel=(0.0, 0.0, 0.0), mask=None, precision=0, u_in=(U_IN, 0.0, 0.0)):
    wall = np.zeros((6, 3))
    if kinds[0] == 1:
        wall[0] = u_in
    if kinds[1] == 1:
        wall[1] = u_in
    open_rho = (rho_in if kinds[0] == 2 else 0.0, rho_out if kinds[1] == 2 else 0.0)
    d = lbm.default_desc(nx=shape[0], ny=shape[1], nz=shape[2], mode=lbm.MODE_PHYSICS, precision=precision,
                         collision=collision, periodic=periodic, tau=tau, body_accel=accel,
                         wall_velocity=wall, open_x=kinds, open_rho=open_rho)
    lat = lbm.Lattice(d)
    st = oracle.ExtState(shape, periodic=periodic, tau=tau, collision=collision, accel=accel, wall=wall,
                         mask=mask, open_x=kinds, open_rho=open_rho)
    n = int(np.prod(shape))
    if mask is not None:
        lat.set_flags(mask)
    rho = np.ones(n, np.float32)
    u = np.zeros((3, n), np.float32)
    lat.init_from_moments(rho, np.ascontiguousarray(u.T))
    st.init(rho.astype(np.float64), u.astype(np.float64))
    return lat, st


@pytest.mark.parametrize("shape", [(48, 12, 10), (47, 12, 10)])  # two nodes per thread / one
@pytest.mark.parametrize("kinds", [(1, 2), (2, 2), (2, 1), (1, 1)])
def test_duct_matches_oracle(gpu, oracle, shape, kinds):
    """Walls on y and z (the faces' edges and corners included)."""
    lat, st = open_pair(gpu, oracle, shape, kinds=kinds)
    lat.step(300)
    st.step(300)
    compare(lat, st)
    lat.close()


@pytest.mark.parametrize("coll", [0, 1])
@pytest.mark.parametrize("variant", [1, 2])
def test_sphere_force_periodic_z(gpu, oracle, coll, variant):
    """A solid sphere, a body force, periodic z, TRT and BGK, the one-node
    and two-node row updates."""
    shape = (40, 16, 12)
    mask = sphere_mask(shape, (14, 8, 6), 4)
    lat, st = open_pair(gpu, oracle, shape, kinds=(1, 2), periodic=(0, 0, 1), tau=0.56, collision=coll,
                        accel=(2e-6, 1e-6, 0.0), mask=mask, u_in=(U_IN, 0.005, -0.003))
    lat.set_step_variant(variant)
    lat.step(250)
    st.step(250)
    compare(lat, st)
    lat.close()


def test_inlet_moments_are_prescribed(gpu, oracle):
    shape = (32, 10, 8)
    lat, st = open_pair(gpu, oracle, shape, kinds=(1, 2), rho_out=0.997)
    lat.step(17)
    rho, u = lat.read_moments()
    nx, ny, nz = shape
    r3 = rho.reshape(nz, ny, nx)
    u3 = u.T.reshape(3, nz, ny, nx)
    assert np.allclose(u3[0, :, :, 0], U_IN, rtol=0, atol=2e-7)
    assert np.allclose(u3[1:, :, :, 0], 0.0, rtol=0, atol=2e-7)
    assert np.allclose(r3[:, :, nx - 1], 0.997, rtol=0, atol=2e-7)
    assert np.allclose(u3[1:, :, :, nx - 1], 0.0, rtol=0, atol=2e-7)
    lat.close()


@pytest.mark.parametrize("prec,tol", [(1, 2e-3), (2, 3e-2)])
@pytest.mark.parametrize("nx", [64, 63])
def test_reduced_precision_storage(gpu, oracle, prec, tol, nx):
    shape = (nx, 16, 12)
    lat, st = open_pair(gpu, oracle, shape, kinds=(1, 2), periodic=(0, 0, 1), precision=prec)
    lat.step(300)
    st.step(300)
    _, ug = lat.read_moments()
    err = np.linalg.norm(ug.T - st.u) / np.linalg.norm(st.u)
    assert err <= tol, f"relative L2 velocity error {err:.3e}"
    lat.close()


def test_variants_without_open_faces_support_refused(gpu):
    d = gpu.default_desc(nx=64, ny=8, nz=8, mode=gpu.MODE_PHYSICS, precision=gpu.PREC_F16S,
                         open_x=(1, 2), open_rho=(0.0, 1.0), wall_velocity=[(U_IN, 0, 0)] + [(0, 0, 0)] * 5)
    lat = gpu.Lattice(d)
    for v in (4, 8):
        with pytest.raises(gpu.LbmError) as e:
            lat.set_step_variant(v)
        assert e.value.code == gpu.ERR_UNSUPPORTED
    lat.set_step_variant(2)
    lat.init_equilibrium(1.0, (0.0, 0.0, 0.0))
    lat.step(3)
    lat.sync()
    lat.close()
