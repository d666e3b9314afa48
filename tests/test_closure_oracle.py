"""CPU checks of the closure oracle itself: its analytic gradient against
central finite differences, its Adam step against a scalar restatement, the
box filter and samples against direct loops, and the ExtStep closure against
plain Smagorinsky for a network whose output is 1."""
import numpy as np
import pytest

from oracle import closure_oracle as co


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 9))
    t = rng.uniform(0.0, 3.0, n)
    w = rng.uniform(0.1, 2.0, n)
    return X, t, w


def test_gradient_matches_finite_differences():
    net = co.random_net(3, mean=np.full(9, 0.1), iscale=np.full(9, 0.9)).astype(np.float64)
    X, t, w = _data(64, 1)
    L, g = co.loss_and_grad(net, X, t, w, 0.01)
    h = 1e-6
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(co.NPARAM, 200, replace=False), [co.B3]])
    for k in idx:
        p, m = net.copy(), net.copy()
        p[k] += h
        m[k] -= h
        fd = (co.loss_and_grad(p, X, t, w, 0.01)[0] - co.loss_and_grad(m, X, t, w, 0.01)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g).max()), k
    assert L > 0


def test_adam_matches_scalar_restatement():
    rng = np.random.default_rng(2)
    theta = rng.standard_normal(co.NPARAM)
    m = 0.01 * rng.standard_normal(co.NPARAM)
    v = np.abs(0.01 * rng.standard_normal(co.NPARAM))
    g = rng.standard_normal(co.NPARAM)
    th2, m2, v2, net = co.adam(theta, m, v, g, 3, lr=0.01, wd=0.1)
    for k in (0, 290, 500, 1350, 1400, 1408):
        mk = 0.9 * m[k] + 0.1 * g[k]
        vk = 0.999 * v[k] + 0.001 * g[k] ** 2
        th = theta[k] * (1 - 0.01 * 0.1) if co.is_weight(np.array(k)) else theta[k]
        th -= 0.01 * (mk / (1 - 0.9 ** 3)) / (np.sqrt(vk / (1 - 0.999 ** 3)) + 1e-8)
        assert np.isclose(th2[k], th, rtol=1e-14, atol=1e-15)
        want = co.round_bf16(np.float32(th)) if co.is_weight(np.array(k)) else np.float32(th)
        assert net[k] == want


def test_box_filter_against_loop():
    shape = (8, 4, 6)
    rng = np.random.default_rng(5)
    n = int(np.prod(shape))
    rho = 1 + 0.05 * rng.standard_normal(n)
    u = 0.04 * rng.standard_normal((3, n))
    out = co.box_filter(rho, u, shape, 2)
    r3 = rho.reshape(6, 4, 8)
    u3 = u.reshape(3, 6, 4, 8)
    c = 0
    for Z in range(3):
        for Y in range(2):
            for X in range(4):
                sl = (slice(2 * Z, 2 * Z + 2), slice(2 * Y, 2 * Y + 2), slice(2 * X, 2 * X + 2))
                rr = r3[sl]
                ut = [(rr * u3[a][sl]).sum() / rr.sum() for a in range(3)]
                assert np.isclose(out[0, c], rr.mean())
                assert np.allclose(out[1:4, c], ut)
                k = 4
                for a, b in ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)):
                    want = (rr * u3[a][sl] * u3[b][sl]).sum() / rr.sum() - ut[a] * ut[b]
                    assert np.isclose(out[k, c], want, rtol=1e-10, atol=1e-16)
                    k += 1
                c += 1


def test_samples_targets_by_hand():
    shape = (6, 5, 4)
    n = int(np.prod(shape))
    rng = np.random.default_rng(8)
    filt = np.zeros((10, n))
    filt[0] = 1 + 0.01 * rng.standard_normal(n)
    filt[1:4] = 0.03 * rng.standard_normal((3, n))
    filt[4:] = 1e-4 * rng.standard_normal((6, n))
    x, t, w = co.samples(filt, shape, 0.51, 0.1, 0, n)
    node = 37
    X, Y, Z = node % 6, (node // 6) % 5, node // 30
    u = filt[1:4].reshape(3, 4, 5, 6)
    G = np.zeros((3, 3))
    for a in range(3):
        G[a, 0] = 0.5 * (u[a, Z, Y, (X + 1) % 6] - u[a, Z, Y, (X - 1) % 6])
        G[a, 1] = 0.5 * (u[a, Z, (Y + 1) % 5, X] - u[a, Z, (Y - 1) % 5, X])
        G[a, 2] = 0.5 * (u[a, (Z + 1) % 4, Y, X] - u[a, (Z - 1) % 4, Y, X])
    S = 0.5 * (G + G.T)
    smag = np.sqrt(2 * (S * S).sum())
    T = np.array([[filt[4, node], filt[7, node], filt[8, node]],
                  [filt[7, node], filt[5, node], filt[9, node]],
                  [filt[8, node], filt[9, node], filt[6, node]]])
    Td = T - np.trace(T) / 3 * np.eye(3)
    assert np.isclose(t[node], -(Td * S).sum() / (0.01 * smag ** 3))
    assert np.isclose(w[node], smag ** 3)
    P = -(2 / 3) * filt[0, node] * (0.51 + 3 * 0.01 * smag) * S
    q = P / np.sqrt((P * P).sum())
    assert np.allclose(x[node, :6], [q[0, 0], q[1, 1], q[2, 2], q[0, 1], q[0, 2], q[1, 2]])
    assert np.isclose(x[node, 6], np.log(np.sqrt((P * P).sum())))
    assert np.isclose(x[node, 7], np.trace(q @ q @ q))
    assert np.isclose(x[node, 8], filt[0, node] - 1)


def test_sample_nodes_hash_is_stable():
    a = co.sample_nodes(7, 1000, 4096)
    assert np.array_equal(a, co.sample_nodes(7, 1000, 4096))
    assert a.min() >= 0 and a.max() < 4096 and len(np.unique(a)) > 800
    assert np.array_equal(co.sample_nodes(0, 10, 4096), np.arange(10))


def test_unit_network_is_smagorinsky(oracle):
    shape = (8, 6, 5)
    n = int(np.prod(shape))
    u = 0.03 * np.random.default_rng(1).standard_normal((3, n))
    runs = []
    for net in (None, co.unit_net()):
        st = oracle.ExtState(shape, periodic=(1, 1, 1), tau=0.52, smag_cs=0.15, net=net)
        st.init(1.0, u)
        st.step(10)
        runs.append(st.f.copy())
    # b3 = log(e - 1) stored as float32 gives r = 1 - 4.5e-10, not exactly 1
    assert np.max(np.abs(runs[0] - runs[1])) < 1e-10


@pytest.mark.parametrize("scale", [0.5, 3.0])
def test_closure_changes_the_oracle_step(oracle, scale):
    """A network with r != 1 changes the step in the direction of its
    eddy viscosity: r > 1 dissipates more kinetic energy than r = 1."""
    shape = (10, 8, 6)
    n = int(np.prod(shape))
    u = 0.04 * np.random.default_rng(2).standard_normal((3, n))
    net = co.unit_net()
    net[co.B3] = np.log(np.expm1(scale))  # softplus(b3) = scale
    out = {}
    for tag, nn in (("unit", co.unit_net()), ("scaled", net)):
        st = oracle.ExtState(shape, periodic=(1, 1, 1), tau=0.51, smag_cs=0.2, net=nn)
        st.init(1.0, u)
        st.step(20)
        out[tag] = (st.u ** 2).sum()
    assert (out["scaled"] < out["unit"]) == (scale > 1)
