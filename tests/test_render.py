"""Velocity-magnitude raymarch: the host LUTs equal the oracle's restatement
and the oracle's exp is accurate (CPU); the CUDA image equals the oracle's
bit for bit for several cameras, and a headless image file is written (GPU)."""
import numpy as np
import pytest

from oracle import render_oracle as ro


def test_luts_match_restatement(lbm_lib):
    assert np.array_equal(lbm_lib.colormap_lut(), ro.colormap_lut())
    assert np.array_equal(lbm_lib.jitter_lut(), ro.jitter_lut())


def test_exp_restatement_accuracy():
    x = -np.concatenate([np.linspace(0, 20, 20001), np.geomspace(1e-8, 86, 5000)]).astype(np.float32)
    got = ro.exp_neg(x).astype(np.float64)
    want = np.exp(x.astype(np.float64))
    assert np.max(np.abs(got - want) / want) < 4e-7
    assert ro.exp_neg(np.float32([-90.0]))[0] == 0.0


def test_camera_sees_the_box(lbm_lib):
    m = lbm_lib.camera((-40, 30, 90), (32, 16, 12), aspect=1.5).reshape(4, 4)  # [col][row]
    inv = np.linalg.inv(m.T.astype(np.float64))  # view-projection
    p = inv @ np.array([32, 16, 12, 1.0])
    ndc = p[:3] / p[3]
    assert np.all(np.abs(ndc[:2]) < 1e-3) and 0 < ndc[2] < 1  # float32 matrix


def _field(shape, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.arange(nz) / nz, np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")
    u = np.zeros((3, nz, ny, nx))
    u[0] += 0.04
    for _ in range(5):
        k = rng.integers(1, 4, 3)
        u += (rng.standard_normal(3) * 0.02)[:, None, None, None] * np.sin(
            2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + rng.uniform(0, 6))
    return u.reshape(3, -1).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("eye,size,steps,f16", [((-40, 30, 90), (72, 48), 64, True),
                                                ((100, -20, -30), (50, 40), 128, False),
                                                ((32, 16, 6), (40, 300), 32, True)])
def test_render_matches_oracle(gpu, tmp_path, eye, size, steps, f16):
    import torch
    shape = (64, 32, 24)
    u = _field(shape, 5)
    w, h = size
    m = gpu.camera(eye, (32, 16, 12), aspect=w / h)
    p = gpu.velmag_params(inv_view_proj=m, camera_pos=eye, steps=steps, velmag_max=0.08, round_f16=int(f16))
    d_u = torch.from_numpy(u).cuda()
    out = torch.empty((h, w, 4), device="cuda")
    gpu.render_velmag(d_u.data_ptr(), shape, p, w, h, out.data_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    want = ro.render(u, shape, m, eye, w, h, steps=steps, vmax=0.08, round_f16=f16)
    assert np.array_equal(got, want)
    assert (got[..., 3] > 0).mean() > 0.05  # the volume is in view
    gpu.write_ppm(str(tmp_path / "velmag.ppm"), got)
    assert (tmp_path / "velmag.ppm").stat().st_size == 3 * w * h + len(f"P6 {w} {h} 255\n")
