"""Batched ensemble: a domain advanced in a batch equals the same domain
advanced alone, bit for bit, in graph and persistent modes and for every tile
shape; the persistent grid barrier gives up with LBM_ERR_TIMEOUT instead of
hanging; the autotuner leaves the state as it found it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def domain_descs(lbm, prec=0, coll=0):
    specs = [  # (shape, periodic, tau, lid)
        ((16, 12, 10), (0, 0, 0), 0.6, 0.05),
        ((8, 8, 8), (1, 1, 1), 0.8, 0.0),
        ((33, 17, 9), (0, 0, 0), 0.55, 0.03),
        ((40, 20, 12), (0, 1, 0), 0.7, 0.04),
        ((24, 24, 24), (0, 0, 0), 0.52, 0.05),
    ]
    descs = []
    for shape, per, tau, lid in specs:
        wall = np.zeros((6, 3))
        wall[lbm.FACE_ZP] = (lid, 0, 0)
        descs.append(lbm.default_desc(nx=shape[0], ny=shape[1], nz=shape[2], mode=lbm.MODE_PHYSICS,
                                      precision=prec, collision=coll, periodic=per, tau=tau,
                                      wall_velocity=wall))
    return descs


def initial_state(d, seed):
    n = d.nx * d.ny * d.nz
    rng = np.random.default_rng(seed)
    mask = (rng.random(n) < 0.05).astype(np.uint8)
    rho = (1 + 0.005 * rng.standard_normal(n)).astype(np.float32)
    u = (0.01 * rng.standard_normal((n, 3))).astype(np.float32)
    return mask, rho, u


def singles(lbm, descs, steps):
    out = []
    for i, d in enumerate(descs):
        mask, rho, u = initial_state(d, i)
        lat = lbm.Lattice(d)
        lat.set_flags(mask)
        lat.init_from_moments(rho, u)
        lat.step(steps)
        out.append((lat.read_populations(), lat.read_moments()))
        lat.close()
    return out


def batch_of(lbm, descs):
    b = lbm.Batch(descs)
    for i, d in enumerate(descs):
        mask, rho, u = initial_state(d, i)
        b.set_flags(i, mask)
        b.init_from_moments(i, rho, u)
    return b


@pytest.mark.parametrize("prec,coll", [(0, 0), (1, 1), (2, 0)])
def test_batch_equals_single_domains(gpu, prec, coll):
    descs = domain_descs(gpu, prec, coll)
    steps = 37
    want = singles(gpu, descs, steps)
    for persistent in (0, 1):
        for rows, zt in ((4, 1), (2, 2), (8, 4), (1, 3), (4, 8), (2, 16)):
            b = batch_of(gpu, descs)
            b.set_schedule(rows_per_block=rows, z_per_thread=zt, persistent=persistent)
            b.step(20)
            b.step(steps - 20)
            b.sync()
            for i in range(len(descs)):
                f = b.read_populations(i)
                rho, u = b.read_moments(i)
                assert np.array_equal(f, want[i][0]), (persistent, rows, zt, i)
                assert np.array_equal(rho, want[i][1][0]) and np.array_equal(u, want[i][1][1])
            b.close()


@pytest.mark.parametrize("persistent", [0, 1])
def test_batch_matches_fp64_oracle(gpu, oracle, persistent):
    """Every domain of a batch against the FP64 textbook step run alone
    (ExtStep), at the physics-mode bar: |du| <= 3e-5 of the velocity scale,
    |drho| <= 1e-5, after 120 steps (fp32 storage, BGK)."""
    descs = domain_descs(gpu, 0, 0)
    b = batch_of(gpu, descs)
    b.set_schedule(rows_per_block=4, z_per_thread=2, persistent=persistent)
    b.step(120)
    b.sync()
    for i, d in enumerate(descs):
        mask, rho, u = initial_state(d, i)
        shape = (d.nx, d.ny, d.nz)
        wall = np.array([[d.wall_velocity[f][a] for a in range(3)] for f in range(6)])
        st = oracle.ExtState(shape, periodic=tuple(d.periodic), tau=d.tau, collision=0, wall=wall, mask=mask)
        st.init(rho.astype(np.float64), u.T.astype(np.float64))
        st.step(120)
        r2, u2 = b.read_moments(i)
        scale = max(np.abs(st.u).max(), 1e-12)
        assert np.abs(u2.T - st.u).max() / scale <= 3e-5, i
        assert np.abs(r2 - st.rho).max() <= 1e-5, i
    b.close()


def test_persistent_barrier_timeout_is_reported(gpu):
    descs = domain_descs(gpu)
    b = batch_of(gpu, descs)
    # a barrier that waits for one block more than the grid has: every wait
    # runs out after ~1 ms of clock cycles and the kernel returns
    b.set_schedule(persistent=1, spin_limit_cycles=2_000_000, test_missing_blocks=1)
    b.step(6)
    with pytest.raises(gpu.LbmError) as e:
        b.sync()
    assert e.value.code == gpu.ERR_TIMEOUT
    with pytest.raises(gpu.LbmError) as e:  # state no longer whole: re-init required
        b.step(1)
    assert e.value.code == gpu.ERR_STATE
    # the device and the batch stay usable
    b.set_schedule(persistent=1, spin_limit_cycles=2_000_000_000, test_missing_blocks=0)
    for i, d in enumerate(descs):
        _, rho, u = initial_state(d, i)
        b.init_from_moments(i, rho, u)
    b.step(37)
    b.sync()
    want = singles(gpu, descs, 37)
    for i in range(len(descs)):
        assert np.array_equal(b.read_populations(i), want[i][0])
    b.close()


def test_persistent_graph_replays_after_a_timeout(gpu):
    """Persistent launches replayed from a captured graph (a call of more than
    16 steps): the first launch's barrier runs out, the replays after it find
    the timeout bit and return at once, and the call reports LBM_ERR_TIMEOUT
    in about the time of one bounded wait."""
    import time
    descs = domain_descs(gpu)
    b = batch_of(gpu, descs)
    b.set_schedule(persistent=1, spin_limit_cycles=2_000_000, test_missing_blocks=1)
    t0 = time.perf_counter()
    b.step(70)  # 4 graph replays of 16 steps, then 6 steps launched directly
    with pytest.raises(gpu.LbmError) as e:
        b.sync()
    assert e.value.code == gpu.ERR_TIMEOUT
    assert time.perf_counter() - t0 < 5.0
    b.close()


def test_persistent_graph_many_steps(gpu):
    """A long call in persistent mode (graph replays of one cooperative launch
    of 16 steps each, then the rest) equals the single-domain runs."""
    descs = domain_descs(gpu, 1, 1)
    steps = 16 * 5 + 3
    want = singles(gpu, descs, steps)
    b = batch_of(gpu, descs)
    b.set_schedule(rows_per_block=4, z_per_thread=4, persistent=1)
    b.step(steps)
    b.sync()
    for i in range(len(descs)):
        assert np.array_equal(b.read_populations(i), want[i][0]), i
    b.close()


def test_autotune_restores_state(gpu):
    descs = domain_descs(gpu, 1, 0)
    b = batch_of(gpu, descs)
    b.step(5)
    before = [b.read_populations(i) for i in range(len(descs))]
    s = b.autotune(4)
    assert s.rows_per_block in (2, 4, 8) and s.z_per_thread in (1, 2, 4, 8, 16)
    cur = b.schedule()
    assert (cur.rows_per_block, cur.z_per_thread, cur.persistent) == (s.rows_per_block, s.z_per_thread, s.persistent)
    for i in range(len(descs)):
        assert np.array_equal(b.read_populations(i), before[i])
    b.step(3)
    b.sync()
    b.close()


def test_batch_rejects_unsupported(gpu):
    d = gpu.default_desc(nx=8, ny=8, nz=8, mode=gpu.MODE_PHYSICS, body_accel=(1e-6, 0, 0))
    with pytest.raises(gpu.LbmError) as e:
        gpu.Batch([d])
    assert e.value.code == gpu.ERR_UNSUPPORTED
    with pytest.raises(gpu.LbmError):
        gpu.Batch([gpu.default_desc(nx=8, ny=8, nz=8)])  # reference mode
