"""lbm_conservation (fp64 sums of rho and rho u over the moment arrays,
block partials reduced in a fixed order) against the fp64 sums of the
moments lbm_read_moments returns, to rounding (1e-12 relative), after the
steps of every path: two- and one-node rows, open faces (row and face
kernels), four nodes per thread, reference mode; and the same bits when
called twice."""
import numpy as np
import pytest

from test_phys_gpu import sphere_mask

pytestmark = pytest.mark.gpu


def sums_of_moments(lat):
    rho, u = lat.read_moments()
    r = rho.astype(np.float64)
    return np.array([r.sum()] + [(r * u[:, a].astype(np.float64)).sum() for a in range(3)])


def check(lat, label):
    got = lat.conservation()
    want = sums_of_moments(lat)
    scale = np.abs(want[0])
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * scale), (label, got, want)
    # deterministic: the same call twice gives the same bits
    assert np.array_equal(lat.conservation(), got), label


def flow(gpu, shape, prec=0, **kw):
    n = int(np.prod(shape))
    d = gpu.default_desc(nx=shape[0], ny=shape[1], nz=shape[2], mode=gpu.MODE_PHYSICS, precision=prec,
                         tau=0.6, **kw)
    lat = gpu.Lattice(d)
    lat.set_flags(sphere_mask(shape, (shape[0] // 3, shape[1] // 2, shape[2] // 2), 3))
    rng = np.random.default_rng(7)
    u = (0.02 * rng.standard_normal((n, 3))).astype(np.float32)
    lat.init_from_moments(np.ones(n, np.float32), u)
    return lat


@pytest.mark.parametrize("shape", [(64, 20, 12), (47, 20, 12), (130, 9, 7)])
@pytest.mark.parametrize("prec", [0, 1])
def test_fused_partials_match_the_moments(gpu, shape, prec):
    lat = flow(gpu, shape, prec, periodic=(1, 0, 1), body_accel=(1e-5, 0, 0))
    check(lat, "after init")
    for steps in (1, 5, 40):  # direct launches, and graphs before the last launch
        lat.step(steps)
        check(lat, f"after {steps} steps")
    lat.set_step_variant(1)
    lat.step(3)
    check(lat, "one node per thread")
    lat.close()


def test_open_faces_partials(gpu):
    wall = np.zeros((6, 3))
    wall[gpu.FACE_XM] = (0.03, 0.0, 0.0)
    lat = flow(gpu, (48, 16, 20), open_x=(gpu.OPEN_VELOCITY, gpu.OPEN_PRESSURE), open_rho=(0.0, 1.0),
               wall_velocity=wall)
    for steps in (1, 30):
        lat.step(steps)
        check(lat, f"open faces, {steps} steps")
    lat.close()


def test_fallback_paths(gpu):
    lat = flow(gpu, (64, 16, 8), prec=1)
    lat.set_step_variant(4)  # four nodes per thread
    lat.step(3)
    check(lat, "quads")
    lat.set_step_variant(2)
    lat.step(2)
    check(lat, "pairs again")
    lat.close()
    ref = gpu.Lattice(nx=24, ny=16, nz=8)  # reference mode
    ref.init_equilibrium(1.0, (0.02, 0.0, 0.0))
    ref.step(3)
    check(ref, "reference mode")
    ref.close()


def test_async_reads_equal_the_blocking_ones(gpu):
    import torch
    lat = flow(gpu, (64, 16, 12), periodic=(1, 0, 1), body_accel=(1e-5, 0, 0))
    want = []
    for _ in range(6):
        lat.step(2)
        want.append(lat.conservation())
    lat2 = flow(gpu, (64, 16, 12), periodic=(1, 0, 1), body_accel=(1e-5, 0, 0))
    host = torch.zeros((6, 4), dtype=torch.float64).pin_memory()
    dev = torch.zeros((6, 4), dtype=torch.float64, device="cuda")
    for i in range(6):
        lat2.step(2)
        lat2.conservation_async(host[i].data_ptr())
        lat2.conservation_async(dev[i].data_ptr())
    lat2.sync()
    assert np.array_equal(host.numpy(), np.array(want))
    assert np.array_equal(dev.cpu().numpy(), np.array(want))
    with pytest.raises(gpu.LbmError):
        lat2.conservation_async(0)
    lat.close()
    lat2.close()
