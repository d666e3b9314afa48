"""CPU checks of the oracle itself: the literal RefStep against an
independent scalar restatement, and ExtStep against analytic solutions."""
import math

import numpy as np
import pytest

F = np.float32
C = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0),
     (1, -1, 0), (-1, 1, 0), (-1, -1, 0), (1, 0, 1), (1, 0, -1), (-1, 0, 1), (-1, 0, -1), (0, 1, 1),
     (0, 1, -1), (0, -1, 1), (0, -1, -1)]
OPP = [0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15]
W = [F(1) / F(3)] + [F(1) / F(18)] * 6 + [F(1) / F(36)] * 12


def feq(i, rho, u):
    cu = F(C[i][0]) * u[0] + F(C[i][1]) * u[1] + F(C[i][2]) * u[2]
    uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2]
    return W[i] * rho * (F(1) + F(3) * cu + F(4.5) * cu * cu - F(1.5) * uu)


def ref_step_scalar(f, rho, u, mask, shape, tau, u_inf, io, fs):
    """Independent float32 scalar restatement of one reference substep:
    collide, stream, boundaries, moments (shaders/*.comp.glsl)."""
    nx, ny, nz = shape
    idx = lambda x, y, z: x + nx * (y + ny * z)  # noqa: E731
    N = nx * ny * nz
    ti = F(1) / F(tau)
    om = F(1) - ti
    f = f.copy()
    for n in range(N):
        uh = [F(np.float16(u[a][n])) for a in range(3)]
        for i in range(19):
            f[i][n] = om * f[i][n] + ti * feq(i, rho[n], uh)
    g = np.zeros_like(f)
    cl = lambda v, hi: 0 if v < 0 else (hi if v > hi else v)  # noqa: E731
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                for i in range(19):
                    g[i][idx(x, y, z)] = f[i][idx(cl(x - C[i][0], nx - 1), cl(y - C[i][1], ny - 1),
                                                  cl(z - C[i][2], nz - 1))]
    snap = g.copy()

    def m_at(x, y, z):
        if x < 0 or y < 0 or z < 0 or x >= nx or y >= ny or z >= nz:
            return 1
        return int(mask[idx(x, y, z)])

    def mom(v):
        r = v[0]
        ru = [F(0), F(0), F(0)]
        for i in range(1, 19):
            r = r + v[i]
            for a in range(3):
                ru[a] = ru[a] + v[i] * F(C[i][a])
        return r, ru

    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                n = idx(x, y, z)
                if m_at(x, y, z) == 1:
                    g[:, n] = 0
                    continue
                for i in range(1, 19):
                    if m_at(x + C[i][0], y + C[i][1], z + C[i][2]) == 1:
                        g[OPP[i]][n] = g[i][n]
                if io:
                    if x == 0:
                        for i in range(19):
                            g[i][n] = feq(i, F(1), [F(v) for v in u_inf])
                    if x == nx - 1:
                        if m_at(x - 1, y, z) == 1:
                            uo = [F(v) for v in u_inf]
                        else:
                            r, ru = mom(snap[:, idx(x - 1, y, z)])
                            uo = [ru[a] / r for a in range(3)] if r > F(1e-12) else [F(v) for v in u_inf]
                        for i in range(19):
                            g[i][n] = feq(i, F(1), uo)
                if fs:
                    for cond, pairs in (
                        (y == 0, ((4, 3), (8, 7), (10, 9), (17, 15), (18, 16))),
                        (y == ny - 1, ((3, 4), (7, 8), (9, 10), (15, 17), (16, 18))),
                        (z == 0, ((6, 5), (12, 11), (14, 13), (16, 15), (18, 17))),
                        (z == nz - 1, ((5, 6), (11, 12), (13, 14), (15, 16), (17, 18))),
                    ):
                        if cond:
                            for dst, src in pairs:
                                g[dst][n] = g[src][n]
    rho2 = np.zeros(N, F)
    u2 = np.zeros((3, N), F)
    for n in range(N):
        r, ru = mom(g[:, n])
        rho2[n] = r
        if r > F(1e-12):
            for a in range(3):
                u2[a][n] = ru[a] / r
    return g, rho2, u2


@pytest.mark.parametrize("io,fs", [(1, 1), (0, 0), (1, 0)])
def test_refstep_matches_scalar_restatement(oracle, io, fs):
    shape = (5, 4, 3)
    n = int(np.prod(shape))
    rng = np.random.default_rng(11)
    mask = np.zeros(n, np.uint8)
    mask[[7, 20, 33]] = 1
    u_inf = (0.04, 0.01, 0.0)
    st = oracle.RefState(shape, tau=0.6, u_inf=u_inf, inlet_outlet=io, free_slip=fs, mask=mask)
    rho0 = (1 + 0.01 * rng.standard_normal(n)).astype(np.float32)
    u0 = (0.03 * rng.standard_normal((3, n))).astype(np.float32)
    st.init(rho=rho0, u=u0)
    f, rho, u = st.f.copy(), st.rho.copy(), st.u.copy()
    for _ in range(3):
        f, rho, u = ref_step_scalar(f, rho, u, mask, shape, 0.6, u_inf, io, fs)
    st.step(3)
    assert np.array_equal(st.f, f)
    assert np.array_equal(st.rho, rho)
    assert np.array_equal(st.u, u)


def test_ext_equilibrium_invariance(oracle):
    st = oracle.ExtState((8, 6, 5), periodic=(1, 1, 1), tau=0.7)
    st.init(1.0, np.array([0.02, -0.01, 0.03]).reshape(3, 1))
    f0 = st.f.copy()
    st.step(20)
    assert np.max(np.abs(st.f - f0)) < 1e-14


@pytest.mark.parametrize("coll", [0, 1])
def test_ext_mass_conserved_in_closed_box(oracle, coll):
    shape = (10, 8, 6)
    n = int(np.prod(shape))
    rng = np.random.default_rng(5)
    mask = np.zeros(n, np.uint8)
    mask[rng.choice(n, 20, replace=False)] = 1
    st = oracle.ExtState(shape, tau=0.62, collision=coll, mask=mask)
    st.init(1.0, 0.02 * rng.standard_normal((3, n)))
    m0 = st.f.sum()
    st.step(50)
    assert abs(st.f.sum() - m0) / m0 < 1e-13


@pytest.mark.parametrize("coll,tol", [(1, 2e-4), (0, 6e-3)])
def test_ext_poiseuille(oracle, coll, tol):
    """Force-driven flow between half-way bounce-back walls at y = -1/2 and
    y = H - 1/2: u(y) = g/(2 nu) (y + 1/2)(H - y - 1/2).  TRT with
    Lambda = 3/16 places the wall exactly; BGK carries a tau-dependent slip."""
    H, tau, g = 16, 0.8, 1e-6
    st = oracle.ExtState((2, H, 2), periodic=(1, 0, 1), tau=tau, collision=coll, accel=(g, 0, 0))
    st.init(1.0, np.zeros((3, 1)))
    st.step(12000)
    nu = (tau - 0.5) / 3
    y = np.arange(H) + 0.5
    want = g / (2 * nu) * y * (H - y)
    got = st.u[0].reshape(2, H, 2)[0, :, 0]
    assert np.max(np.abs(got - want)) / want.max() < tol


def test_ext_taylor_green_decay(oracle):
    """2-D Taylor-Green vortex: kinetic energy decays as exp(-4 nu k^2 t)."""
    L, tau, u0 = 32, 0.8, 0.01
    nu = (tau - 0.5) / 3
    k = 2 * math.pi / L
    x = np.arange(L)
    X, Y = np.meshgrid(x, x, indexing="xy")
    ux = u0 * np.sin(k * X) * np.cos(k * Y)
    uy = -u0 * np.cos(k * X) * np.sin(k * Y)
    shape = (L, L, 2)
    u = np.zeros((3, L * L * 2))
    u[0] = np.tile(ux.reshape(-1), 2)
    u[1] = np.tile(uy.reshape(-1), 2)
    rho = 1 - 3 * u0 ** 2 / 4 * (np.cos(2 * k * X) + np.cos(2 * k * Y))
    st = oracle.ExtState(shape, periodic=(1, 1, 1), tau=tau)
    st.init(np.tile(rho.reshape(-1), 2), u)
    e0 = (u[:2] ** 2).sum()
    T = 400
    st.step(T)
    e = (st.u[:2] ** 2).sum()
    rate = -math.log(e / e0) / T
    assert abs(rate - 4 * nu * k * k) / (4 * nu * k * k) < 0.02
