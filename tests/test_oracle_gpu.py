"""The FP64 GPU copy of the oracle equals the CPU oracle bit for bit (same
node update, every operation rounded on its own on both sides)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["cavity", "channel", "tgv_smag_trt"])
def test_gpu_fp64_oracle_equals_cpu(gpu, oracle, case):
    rng = np.random.default_rng(3)
    if case == "cavity":
        wall = np.zeros((6, 3))
        wall[5] = (0.05, 0, 0)  # lid on the z = max face
        shape, kw = (14, 12, 10), dict(tau=0.6, wall=wall)
    elif case == "channel":
        shape = (20, 10, 12)
        n = int(np.prod(shape))
        kw = dict(periodic=(1, 0, 0), tau=0.55, accel=(1e-5, 0, 0),
                  mask=(rng.random(n) < 0.05).astype(np.uint8))
    else:
        shape, kw = (12, 12, 12), dict(periodic=(1, 1, 1), tau=0.52, collision=1, smag_cs=0.1)
    n = int(np.prod(shape))
    u = 0.02 * rng.standard_normal((3, n))
    rho = 1 + 0.01 * rng.standard_normal(n)
    cpu = oracle.ExtState(shape, **kw)
    gpu_ = oracle.ExtStateGPU(shape, **kw)
    cpu.init(rho, u)
    gpu_.init(rho, u)
    cpu.step(15)
    gpu_.step(15)
    r, uu = gpu_.moments()
    assert np.array_equal(gpu_.f.view(19, -1).cpu().numpy(), cpu.f)
    assert np.array_equal(r, cpu.rho) and np.array_equal(uu, cpu.u)
