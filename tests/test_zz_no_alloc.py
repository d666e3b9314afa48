"""The allocation-free conservation entry point against the allocating one.

lbm_conservation_noalloc serves callers that may not allocate device memory
(a frame loop that cannot stall on cudaMalloc's device-wide sync, or a host
whose arena owns the whole device budget).  It must give the same sums as
lbm_conservation, within the fp64 tolerance the other conservation tests use,
on consecutive calls, and refuse inputs larger than its static scratch.
This file is collected last so a failure here leaves every other result in
place.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_NODES = 33554432


def test_noalloc_conservation_matches_lbm_conservation(gpu):
    lib = gpu.load()
    n = 72 * 40 * 36
    rng = np.random.default_rng(2024)
    lat = gpu.Lattice(nx=72, ny=40, nz=36, mode=gpu.MODE_PHYSICS, periodic=(1, 1, 0), tau=0.7,
                      body_accel=(2e-6, 0, 0))
    rho = (1 + 0.01 * rng.standard_normal(n)).astype(np.float32)
    u = (0.03 + 0.02 * rng.standard_normal((n, 3))).astype(np.float32)
    lat.init_from_moments(rho, u)
    d_rho, d_u = lat.device_moments()
    out = (C.c_double * 4)()
    for _ in range(2):  # two calls in a row share the static scratch
        lat.step(4)
        want = lat.conservation()  # synchronises the lattice's stream
        rc = lib.lbm_conservation_noalloc(d_rho, d_u, n, out, None)
        assert rc == gpu.OK, lib.lbm_last_error(None).decode()
        got = np.array(out[:])
        assert np.allclose(got, want, rtol=1e-12, atol=1e-12), (got, want)
    lat.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    lib = gpu.load()
    lat = gpu.Lattice(nx=8, ny=8, nz=8, mode=gpu.MODE_PHYSICS)
    lat.init_equilibrium(1.0, (0, 0, 0))
    d_rho, d_u = lat.device_moments()
    out = (C.c_double * 4)()
    rc = lib.lbm_conservation_noalloc(d_rho, d_u, MAX_NODES + 1, out, None)
    assert rc == gpu.ERR_INVALID_ARG
    assert b"33554432" in lib.lbm_last_error(None)
    assert lib.lbm_conservation_noalloc(None, d_u, 512, out, None) == gpu.ERR_INVALID_ARG
    lat.close()


def test_noalloc_at_its_node_limit(gpu):
    """n = the limit uses every partial slot, and the sums sit right after
    them.  rho = 1 and a constant u of powers of two make every partial and
    total exact, so the sums are known: (n, n*ux, n*uy, n*uz)."""
    import torch
    lib = gpu.load()
    torch.cuda.set_device(0)
    u0 = (0.25, -0.125, 0.0625)
    d_rho = torch.ones(MAX_NODES, dtype=torch.float32, device="cuda")
    d_u = torch.empty((3, MAX_NODES), dtype=torch.float32, device="cuda")
    for a in range(3):
        d_u[a].fill_(u0[a])
    torch.cuda.synchronize()
    out = (C.c_double * 4)()
    for _ in range(2):
        rc = lib.lbm_conservation_noalloc(d_rho.data_ptr(), d_u.data_ptr(), MAX_NODES, out, None)
        assert rc == gpu.OK, lib.lbm_last_error(None).decode()
        assert list(out) == [float(MAX_NODES)] + [MAX_NODES * v for v in u0]
    del d_rho, d_u
    torch.cuda.empty_cache()
