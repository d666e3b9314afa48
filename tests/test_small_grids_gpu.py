"""The smallest grids each path accepts (2 nodes per axis and odd neighbours
of it), against the oracles: physics mode (one- and two-node rows, periodic
and walled, fp32 and fp16), an open-face duct of the same sizes, and
reference mode bit for bit."""
import numpy as np
import pytest

from test_phys_gpu import compare, make_pair

pytestmark = pytest.mark.gpu

SHAPES = [(2, 2, 2), (3, 2, 2), (2, 3, 5), (4, 2, 3), (65, 2, 2)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("periodic", [(1, 1, 1), (0, 0, 0), (1, 0, 1)])
def test_physics_small(gpu, oracle, shape, periodic):
    n = int(np.prod(shape))
    rng = np.random.default_rng(sum(shape))
    u = 0.01 * rng.standard_normal((3, n))
    wall = np.zeros((6, 3))
    wall[gpu.FACE_ZP] = (0.02, 0.0, 0.0) if not periodic[2] else (0.0, 0.0, 0.0)
    lat, st = make_pair(gpu, oracle, shape, periodic=periodic, tau=0.7, wall=wall, u=u)
    lat.step(40)
    st.step(40)
    compare(lat, st, tol_u=5e-5)
    lat.close()


@pytest.mark.parametrize("shape", SHAPES)
def test_physics_small_fp16(gpu, oracle, shape):
    n = int(np.prod(shape))
    u = 0.01 * np.random.default_rng(3).standard_normal((3, n))
    lat, st = make_pair(gpu, oracle, shape, periodic=(1, 1, 1), tau=0.7, u=u, precision=gpu.PREC_F16S)
    lat.step(20)
    st.step(20)
    _, ug = lat.read_moments()
    assert np.linalg.norm(ug.T - st.u) / np.linalg.norm(st.u) < 2e-3
    lat.close()


@pytest.mark.parametrize("shape", [(2, 2, 2), (3, 3, 2), (4, 2, 3)])
def test_open_faces_small(gpu, oracle, shape):
    from test_open_faces_gpu import open_pair
    lat, st = open_pair(gpu, oracle, shape, kinds=(1, 2))
    lat.step(30)
    st.step(30)
    compare(lat, st, tol_u=5e-5)
    lat.close()


@pytest.mark.parametrize("shape", SHAPES)
def test_reference_small_bit_exact(gpu, oracle, shape):
    from test_ref_gpu import _ref_pair, _assert_same
    lat, st = _ref_pair(gpu, oracle, shape, u_inf=(0.03, 0.0, 0.0))
    lat.step(15)
    st.step(15)
    _assert_same(lat, st, f"reference {shape}")
    lat.close()
