"""Pin the CPU oracle (oracle/ogx_oracle.c) to the reference before trusting it.

Every fixture under tests/golden/ was produced by the reference's own code
(tests/golden/make_golden.py).  The restatement must reproduce it: forces to
roundoff (bit-identical in practice), trees and all five interaction lists as
exact sets, and the published operator convergence table
(outputs/fmm3d_operator_convergence.csv) to the 6 digits it was printed with.
"""
import numpy as np
import pytest

from helpers import assert_same_tree, canonical_from_arrays, rel_err
from oracle_lib import canonical_tree

CASES = [
    ("plummer2000_s2", "fmm_p4", 4, 64, 0.0),
    ("plummer2000_s2", "fmm_p8", 8, 64, 0.0),
    ("cube1000_s1", "fmm_p8_t64", 8, 64, 0.0),
    ("cube1000_s1", "fmm_p8_t16", 8, 16, 0.0),
    ("clump", "fmm_p4_t16", 4, 16, 0.0),
    ("coincident", "fmm_p4_t4_eps", 4, 4, 0.01),
    ("disk4000", "fmm_p6_t32", 6, 32, 0.0),
]


@pytest.mark.parametrize("name,key,p,thr,eps", CASES)
def test_oracle_fmm_matches_reference(oracle, golden, name, key, p, thr, eps):
    d = golden(name)
    acc = oracle.adaptive_fmm(d["pos"], d["mass"], eps=eps, p=p, thr=thr, with_pot=False)
    mx, rms = rel_err(d[key], acc)
    assert mx <= 1e-13, (mx, rms)


@pytest.mark.parametrize("name,key,eps", [("plummer2000_s2", "direct", 0.0), ("cube1000_s1", "direct", 0.0),
                                          ("clump", "direct", 0.0), ("coincident", "direct_eps", 0.01),
                                          ("disk4000", "direct", 0.0)])
def test_oracle_direct_matches_reference(oracle, golden, name, key, eps):
    d = golden(name)
    acc = oracle.direct(d["pos"], d["mass"], eps=eps, with_pot=False)
    np.testing.assert_array_equal(acc, d[key])


@pytest.mark.parametrize("name,prefix,thr,eps", [("plummer2000_s2", "t64", 64, 0.0), ("plummer2000_s2", "t8", 8, 0.0),
                                                 ("cube1000_s1", "t64", 64, 0.0), ("cube1000_s1", "t16", 16, 0.0),
                                                 ("clump", "t16", 16, 0.0), ("coincident", "t4", 4, 0.0),
                                                 ("coincident", "t4eps", 4, 0.01), ("disk4000", "t32", 32, 0.0)])
def test_oracle_tree_matches_reference(oracle, golden, name, prefix, thr, eps):
    d = golden(name)
    t = canonical_tree(oracle.tree(d["pos"], thr, eps))
    assert_same_tree(t, canonical_from_arrays(d, prefix), f"{name}/{prefix}")


def test_oracle_small_cases(oracle, golden):
    d = golden("small")
    for n in (1, 2, 64, 65):
        acc = oracle.adaptive_fmm(d[f"n{n}_pos"], d[f"n{n}_mass"], p=4, thr=64, with_pot=False)
        np.testing.assert_allclose(acc, d[f"n{n}_fmm"], rtol=1e-13, atol=1e-300)
        t = canonical_tree(oracle.tree(d[f"n{n}_pos"], 64))
        assert_same_tree(t, canonical_from_arrays(d, f"n{n}"), f"small n={n}")


def test_oracle_cfg1_fp64(oracle, golden):
    """Config 1 (Plummer 16384, 20a truncation, p=8, thr=64): oracle == reference."""
    d = golden("cfg1_plummer16384")
    acc = oracle.adaptive_fmm(d["pos"], d["mass"], p=8, thr=64, with_pot=False)
    mx, _ = rel_err(d["fmm_p8_t64"], acc)
    assert mx <= 1e-13
    mx, rms = rel_err(d["direct"], d["fmm_p8_t64"])
    assert rms < 5e-5  # truncation level at p=8 (Gate B bound of adaptive_tests.cpp:122)


def test_harmonics_closed_forms(oracle):
    """fmm3d_tests.cpp:134-157: Y_n^m at theta=1.0, phi=0.7 against closed forms, < 1e-13."""
    th, ph = 1.0, 0.7
    v = (np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th))
    Y = oracle.harmonics(v, 2)
    c, s = np.cos(th), np.sin(th)
    e = lambda m: np.exp(1j * m * ph)  # noqa: E731
    refs = {(0, 0): 1, (1, 0): c, (1, 1): np.sqrt(0.5) * s * e(1), (2, 0): (3 * c * c - 1) / 2,
            (2, 1): np.sqrt(1 / 6) * 3 * c * s * e(1), (2, 2): np.sqrt(1 / 24) * 3 * s * s * e(2)}
    err = 0.0
    for (n, m), val in refs.items():
        err = max(err, abs(Y[n * n + n + m] - val), abs(Y[n * n + n - m] - np.conj(val)))
    assert err < 1e-13


def test_gradient_recurrences_vs_finite_differences(oracle):
    """fmm3d_tests.cpp:159-189: field of a random multipole (far) and local (near) vs central FD."""
    rng = np.random.default_rng(123)
    p, h = 6, 1e-5
    S = (p + 1) ** 2
    M = rng.standard_normal(S) + 1j * rng.standard_normal(S)
    L = rng.standard_normal(S) + 1j * rng.standard_normal(S)
    worst = 0.0
    for _ in range(20):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        for kind, coef, t in ((0, M, 5.0 * d), (1, L, 0.4 * d)):
            _, g = oracle.evaluate(kind, p, [0, 0, 0], coef, t[None, :])
            fd = np.zeros(3)
            for a in range(3):
                e = np.zeros(3)
                e[a] = h
                pp, _ = oracle.evaluate(kind, p, [0, 0, 0], coef, (t + e)[None, :])
                pm, _ = oracle.evaluate(kind, p, [0, 0, 0], coef, (t - e)[None, :])
                fd[a] = (pp[0] - pm[0]) / (2 * h)
            worst = max(worst, np.linalg.norm(g[0] - fd) / np.linalg.norm(g[0]))
    assert worst < 1e-6


def _op_err(oracle, d, op, p):
    def pot_acc_direct(src, q, tgt):
        diff = src[None, :, :] - tgt[:, None, :]
        r = np.linalg.norm(diff, axis=2)
        return (q[None, :] / r).sum(1), (q[None, :, None] * diff / r[:, :, None] ** 3).sum(1)

    def err(pt, at, pa, aa):
        return (np.sqrt(((pa - pt) ** 2).sum() / (pt ** 2).sum()),
                np.sqrt(((aa - at) ** 2).sum() / (at ** 2).sum()))

    if op == "P2M":
        src, q, tgt = d["p2m_src"], d["p2m_q"], d["p2m_tgt"]
        M = oracle.p2m(p, [0, 0, 0], src, q)
        pa, aa = oracle.evaluate(0, p, [0, 0, 0], M, tgt)
        return err(*pot_acc_direct(src, q, tgt), pa, aa)
    if op == "M2L":
        worst = (0.0, 0.0)
        for k in range(4):
            src, q, tgt, zl = d[f"m2l{k}_src"], d[f"m2l{k}_q"], d[f"m2l{k}_tgt"], d[f"m2l{k}_zl"]
            M = oracle.p2m(p, [0, 0, 0], src, q)
            L = oracle.translate(1, p, [0, 0, 0], zl, M)
            pa, aa = oracle.evaluate(1, p, zl, L, tgt)
            e = err(*pot_acc_direct(src, q, tgt), pa, aa)
            worst = (max(worst[0], e[0]), max(worst[1], e[1]))
        return worst
    if op == "M2M":
        src, q, tgt = d["m2m_src"], d["m2m_q"], d["m2m_tgt"]
        Mc = oracle.p2m(p, [0.5, 0.4, 0.3], src, q)
        Mp = oracle.translate(0, p, [0.5, 0.4, 0.3], [0, 0, 0], Mc)
        pa, aa = oracle.evaluate(0, p, [0, 0, 0], Mp, tgt)
        return err(*pot_acc_direct(src, q, tgt), pa, aa)
    src, q, tgt = d["l2l_src"], d["l2l_q"], d["l2l_tgt"]
    Lp = oracle.p2l(p, [0, 0, 0], src, q)
    Lc = oracle.translate(2, p, [0, 0, 0], [0.5, 0.4, 0.3], Lp)
    pa, aa = oracle.evaluate(1, p, [0.5, 0.4, 0.3], Lc, tgt)
    return err(*pot_acc_direct(src, q, tgt), pa, aa)


def test_operator_convergence_table(oracle, golden):
    """Reproduce outputs/fmm3d_operator_convergence.csv (printed with 6 significant digits)."""
    d = golden("operators")
    for op in ("P2M", "M2L", "M2M", "L2L"):
        for p in (2, 4, 6, 8, 10):
            pot, acc = _op_err(oracle, d, op, p)
            for qty, val in (("potential", pot), ("acceleration", acc)):
                sel = (d["csv_op"] == op) & (d["csv_qty"] == qty) & (d["csv_p"] == p)
                ref = float(d["csv_err"][sel][0])
                assert abs(val - ref) <= 6e-6 * ref, (op, qty, p, val, ref)
