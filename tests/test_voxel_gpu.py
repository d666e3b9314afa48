"""The device NACA voxeliser against the host voxeliser (itself checked
against the oracle's restatement of naca::voxelize_into, src/main.cpp:254-312,
in test_abi.py): the same mask bit for bit, for every preset, odd and large
shapes, angles and chords; and lbm_set_flags_naca against lbm_set_flags of
the host mask (mask and classification)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def torch(gpu):
    import torch as t
    return t


def _device_mask(gpu, torch, naca, shape, chord, cx, aoa):
    n = int(np.prod(shape))
    d = torch.full((n,), 7, dtype=torch.uint8, device="cuda")  # every byte must be written
    gpu.voxelize_naca_device(naca, *shape, d.data_ptr(), n, chord, cx, aoa,
                             stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return d.cpu().numpy()


@pytest.mark.parametrize("preset", [0, 1, 2])
@pytest.mark.parametrize("shape", [(128, 128, 2), (96, 40, 3), (257, 131, 5), (33, 17, 1)])
def test_device_mask_matches_host(gpu, torch, preset, shape):
    p = gpu.PRESETS[preset]
    want = gpu.voxelize_naca(p.naca, *shape, 0.25, 0.25, p.angle_of_attack_deg)
    got = _device_mask(gpu, torch, p.naca, shape, 0.25, 0.25, p.angle_of_attack_deg)
    assert want.sum() > 0
    assert np.array_equal(got, want)


@pytest.mark.parametrize("naca,chord,cx,aoa", [("2412", 0.4, 0.5, -12.5), ("0030", 0.6, 0.45, 31.0),
                                               ("9999", 0.3, 0.3, 90.0), ("0001", 0.25, 0.25, 0.0)])
def test_device_mask_other_airfoils(gpu, torch, naca, chord, cx, aoa):
    shape = (200, 150, 2)
    want = gpu.voxelize_naca(naca, *shape, chord, cx, aoa)
    got = _device_mask(gpu, torch, naca, shape, chord, cx, aoa)
    assert np.array_equal(got, want)


def test_device_mask_capture_tier(gpu, torch):
    """The largest preset tier, 512 x 256 x 256 (33.5 MB of mask)."""
    shape = (512, 256, 256)
    p = gpu.PRESETS[2]
    want = gpu.voxelize_naca(p.naca, *shape, 0.25, 0.25, p.angle_of_attack_deg)
    got = _device_mask(gpu, torch, p.naca, shape, 0.25, 0.25, p.angle_of_attack_deg)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("mode", ["reference", "physics"])
def test_set_flags_naca_matches_host_upload(gpu, mode):
    shape = (96, 48, 6)
    p = gpu.PRESETS[2]
    if mode == "reference":
        d = gpu.default_desc(nx=shape[0], ny=shape[1], nz=shape[2])
    else:
        d = gpu.default_desc(nx=shape[0], ny=shape[1], nz=shape[2], mode=gpu.MODE_PHYSICS,
                             periodic=(1, 0, 1), tau=0.6)
    a, b = gpu.Lattice(d), gpu.Lattice(d)
    host = gpu.apply_preset(a, 2)
    dev = gpu.apply_preset(b, 2, device=True)
    assert np.array_equal(host, dev)
    assert np.array_equal(b.read_mask(), host)
    assert np.array_equal(a.read_classification(), b.read_classification())
    a.step(3)
    b.step(3)
    ra, ua = a.read_moments()
    rb, ub = b.read_moments()
    assert np.array_equal(ra, rb) and np.array_equal(ua, ub)
    a.close()
    b.close()


def test_device_voxeliser_rejects_bad_input(gpu, torch):
    d = torch.zeros(64, dtype=torch.uint8, device="cuda")
    with pytest.raises(gpu.LbmError):
        gpu.voxelize_naca_device("00x2", 4, 4, 4, d.data_ptr(), 64)
    with pytest.raises(gpu.LbmError):
        gpu.voxelize_naca_device("0012", 4, 4, 4, d.data_ptr(), 63)
    lat = gpu.Lattice(nx=8, ny=8, nz=2)
    with pytest.raises(gpu.LbmError):
        lat.set_flags_naca("12")
    lat.close()
