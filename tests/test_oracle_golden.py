"""Pins the CPU oracle to the reference's golden vectors (CPU only).

The reference's only pinned numbers are its D3Q19 tables and equilibrium at
four test points (tools/integrity/integrity/cat3_numerical/
d3q19_equilibrium.expected.json, checked by the reference at 1e-12 abs,
d3q19_verify.py:24; fp32 shader evaluation is held to 1e-6 rel / 1e-9 abs,
tools/integrity/docs/algebraic/d3q19.md:182-187).
"""
import numpy as np
import pytest


def test_tables_match_golden(oracle, golden):
    c, w, opp = oracle.tables()
    assert c.tolist() == golden["velocity_set"]
    assert np.array_equal(opp, golden["opposite_index"])
    assert np.max(np.abs(w - np.array(golden["weights"]))) <= 1e-15


@pytest.mark.parametrize("k", range(4))
def test_feq_f64_matches_golden(oracle, golden, k):
    tp = golden["test_points"][k]
    f = oracle.feq_f64(tp["rho"], *tp["u"])
    assert np.max(np.abs(f - np.array(tp["feq"]))) <= golden["tolerance_abs"]
    c = np.array(golden["velocity_set"], np.float64)
    s = tp["sums"]
    assert abs(f.sum() - s["mass"]) <= 1e-12
    for a, key in enumerate(("mom_x", "mom_y", "mom_z")):
        assert abs((f * c[:, a]).sum() - s[key]) <= 1e-12


@pytest.mark.parametrize("k", range(4))
def test_feq_f32_within_shader_tolerance(oracle, golden, k):
    tp = golden["test_points"][k]
    f = oracle.feq_f32(tp["rho"], *tp["u"]).astype(np.float64)
    ref = np.array(tp["feq"])
    assert np.all(np.abs(f - ref) <= np.maximum(1e-6 * np.abs(ref), 1e-9))


def test_round_f16_rte_matches_ieee(oracle):
    rng = np.random.default_rng(7)
    vals = np.concatenate([
        rng.normal(0, 0.05, 4000), rng.uniform(-1, 1, 2000), rng.uniform(-1e-4, 1e-4, 2000),
        rng.uniform(-7e4, 7e4, 200), [0.0, -0.0, 65504.0, 65519.9, 65520.0, 6.1e-5, 5.96e-8, 2.98e-8],
    ]).astype(np.float32)
    got = np.array([oracle.round_f16(float(v), 1) for v in vals], np.float32)
    want = vals.astype(np.float16).astype(np.float32)
    assert np.array_equal(got, want, equal_nan=True)


def test_round_f16_rtz_truncates(oracle):
    rng = np.random.default_rng(8)
    vals = rng.normal(0, 0.05, 2000).astype(np.float32)
    for v in vals:
        r = oracle.round_f16(float(v), 2)
        h = np.float32(v).astype(np.float16).astype(np.float32)
        assert abs(r) <= abs(v)
        # RTZ differs from RTE by at most one binary16 ulp, towards zero
        assert r == h or abs(h) > abs(v)
        assert np.float32(r).astype(np.float16).astype(np.float32) == r


def test_classify_matches_numpy_restatement(oracle):
    rng = np.random.default_rng(3)
    shape = (7, 6, 5)
    mask = (rng.random(np.prod(shape)) < 0.2).astype(np.uint8)
    mask[rng.random(mask.size) < 0.05] = 2  # value 2 counts as fluid (== 1 test)
    c, _, _ = oracle.tables()
    for periodic in ((0, 0, 0), (1, 0, 1), (1, 1, 1)):
        got = oracle.classify(mask, shape, periodic)
        m3 = mask.reshape(shape[::-1])  # [z][y][x]
        want = np.zeros(mask.size, np.uint32)
        for z in range(shape[2]):
            for y in range(shape[1]):
                for x in range(shape[0]):
                    L = 1 if m3[z, y, x] == 1 else 0
                    for i in range(1, 19):
                        p = [x + c[i, 0], y + c[i, 1], z + c[i, 2]]
                        s = False
                        for a in range(3):
                            if p[a] < 0 or p[a] >= shape[a]:
                                if periodic[a]:
                                    p[a] %= shape[a]
                                else:
                                    s = True
                        if not s:
                            s = m3[p[2], p[1], p[0]] == 1
                        if s:
                            L |= 1 << i
                    want[x + shape[0] * (y + shape[1] * z)] = L
        assert np.array_equal(got, want)
