"""GPU parity of the plain FP64 form, through the C ABI.

Bars (per the drop-in contract of src3d/ForceSolver3D.hpp):
  * trees and all five interaction lists equal the reference's as sets
    (AdaptiveOctree::build/buildLists, src3d/AdaptiveOctree.hpp:65-189);
  * accelerations match the reference AdaptiveFMM3D at the same p and leaf
    capacity to max_rel <= 1e-12 (metric of src3d/adaptive_tests.cpp:40-50);
  * the direct solver matches DirectSolver3D to max_rel <= 1e-12;
  * potentials (not produced by the reference) match the oracle's restatement.
"""
import numpy as np
import pytest

from helpers import assert_same_tree, canonical_from_arrays, canonical_from_tree, rel_err

pytestmark = pytest.mark.gpu

FMM_TOL = 1e-12

TREE_CASES = [("plummer2000_s2", "t64", 64, 0.0), ("plummer2000_s2", "t8", 8, 0.0), ("cube1000_s1", "t64", 64, 0.0),
              ("cube1000_s1", "t16", 16, 0.0), ("clump", "t16", 16, 0.0), ("coincident", "t4", 4, 0.0),
              ("coincident", "t4eps", 4, 0.01), ("disk4000", "t32", 32, 0.0)]


@pytest.mark.parametrize("name,prefix,thr,eps", TREE_CASES)
def test_tree_and_lists_match_reference(ogx, golden, name, prefix, thr, eps):
    d = golden(name)
    # eps=0 with exactly coincident bodies gives non-finite forces (as in the reference);
    # only the tree is compared there.
    with ogx.AdaptiveFMM3D(eps=eps, p=2, threshold=thr) as s:
        s.compute_accelerations(d["pos"], d["mass"])
        t = s.tree()
        st = s.stats()
    assert_same_tree(canonical_from_tree(t), canonical_from_arrays(d, prefix), f"{name}/{prefix}")
    assert st["adjacency_mismatch"] == 0
    assert st["num_boxes"] == len(d[f"{prefix}_keys"])


FMM_CASES = [("plummer2000_s2", "fmm_p4", 4, 64, 0.0), ("plummer2000_s2", "fmm_p8", 8, 64, 0.0),
             ("cube1000_s1", "fmm_p8_t64", 8, 64, 0.0), ("cube1000_s1", "fmm_p8_t16", 8, 16, 0.0),
             ("clump", "fmm_p4_t16", 4, 16, 0.0), ("coincident", "fmm_p4_t4_eps", 4, 4, 0.01),
             ("disk4000", "fmm_p6_t32", 6, 32, 0.0)]


@pytest.mark.parametrize("name,key,p,thr,eps", FMM_CASES)
def test_fmm_fp64_matches_reference(ogx, golden, name, key, p, thr, eps):
    d = golden(name)
    with ogx.AdaptiveFMM3D(eps=eps, p=p, threshold=thr) as s:
        acc = s.compute_accelerations(d["pos"], d["mass"])
    mx, rms = rel_err(d[key], acc)
    assert mx <= FMM_TOL, (mx, rms)


def test_cfg1_fp64_accelerations_and_potentials(ogx, oracle, golden):
    """Config 1: Plummer N=16384 (20a truncation), p=8, leaf capacity 64, FP64 acc + pot."""
    d = golden("cfg1_plummer16384")
    with ogx.AdaptiveFMM3D(p=8, threshold=64) as s:
        acc, pot = s.compute_accelerations(d["pos"], d["mass"], with_potential=True)
        st = s.stats()
    mx, rms = rel_err(d["fmm_p8_t64"], acc)
    assert mx <= FMM_TOL, (mx, rms)
    # against DirectSolver3D: p=8 truncation error (reference itself: same number)
    mx_d, rms_d = rel_err(d["direct"], acc)
    mx_r, rms_r = rel_err(d["direct"], d["fmm_p8_t64"])
    assert abs(rms_d - rms_r) <= 1e-9 * rms_r
    # potentials vs the oracle's FMM restatement and vs the direct sum
    _, pot_o = oracle.adaptive_fmm(d["pos"], d["mass"], p=8, thr=64)
    assert np.max(np.abs(pot - pot_o) / np.abs(pot_o)) <= FMM_TOL
    _, pot_dir = oracle.direct(d["pos"], d["mass"])
    assert np.sqrt(np.sum((pot - pot_dir) ** 2) / np.sum(pot_dir ** 2)) < 1e-6
    assert st["max_leaf_occupancy"] <= 64 and st["num_leaves"] > 0


def test_small_and_ragged_sizes(ogx, golden):
    d = golden("small")
    for n in (1, 2, 64, 65):
        with ogx.AdaptiveFMM3D(p=4, threshold=64) as s:
            acc = s.compute_accelerations(d[f"n{n}_pos"], d[f"n{n}_mass"])
            t = s.tree()
        np.testing.assert_allclose(acc, d[f"n{n}_fmm"], rtol=1e-12, atol=1e-300)
        assert_same_tree(canonical_from_tree(t), canonical_from_arrays(d, f"n{n}"), f"n={n}")
    with ogx.AdaptiveFMM3D() as s:
        acc = s.compute_accelerations(np.zeros((0, 3)), np.zeros(0))
        assert acc.shape == (0, 3)


@pytest.mark.parametrize("name,key,eps", [("plummer2000_s2", "direct", 0.0), ("clump", "direct", 0.0),
                                          ("coincident", "direct_eps", 0.01), ("disk4000", "direct", 0.0)])
def test_direct_fp64_matches_reference(ogx, oracle, golden, name, key, eps):
    d = golden(name)
    with ogx.DirectSolver3D(eps=eps) as s:
        acc, pot = s.compute_accelerations(d["pos"], d["mass"], with_potential=True)
    mx, rms = rel_err(d[key], acc)
    assert mx <= 1e-12, (mx, rms)
    _, pot_o = oracle.direct(d["pos"], d["mass"], eps=eps)
    assert np.max(np.abs(pot - pot_o) / np.abs(pot_o)) <= 1e-12


def test_direct_fp64_cfg1(ogx, golden):
    d = golden("cfg1_plummer16384")
    with ogx.DirectSolver3D() as s:
        acc = s.compute_accelerations(d["pos"], d["mass"])
    mx, rms = rel_err(d["direct"], acc)
    assert mx <= 1e-12, (mx, rms)


def test_p_range_converges(ogx, golden):
    """Gate B pattern (adaptive_tests.cpp:108-126): error vs direct falls monotonically with p."""
    d = golden("plummer2000_s2")
    prev = 1e300
    for p in (2, 4, 6, 8, 10, 12):
        with ogx.AdaptiveFMM3D(p=p, threshold=64) as s:
            _, rms = rel_err(d["direct"], s.compute_accelerations(d["pos"], d["mass"]))
        assert rms < prev
        prev = rms
    assert prev < 1e-6


def test_device_leapfrog_matches_host_loop(ogx, golden):
    """ogx_upload/ogx_step (device-resident VelocityVerlet3D) vs the same KDK on the host."""
    d = golden("plummer2000_s2")
    rng = np.random.default_rng(0)
    vel = 0.1 * rng.standard_normal(d["pos"].shape)
    dt, steps = 0.01, 3
    with ogx.AdaptiveFMM3D(p=6, threshold=64) as s:
        s.upload(d["pos"], vel, d["mass"])
        s.step(dt, steps)
        pos_d, vel_d, acc_d = s.download()
    with ogx.AdaptiveFMM3D(p=6, threshold=64) as s:
        x, v = d["pos"].copy(), vel.copy()
        a = s.compute_accelerations(x, d["mass"])
        for _ in range(steps):  # Integrator3D.hpp:23-40
            x = x + v * dt + a * (0.5 * dt * dt)
            an = s.compute_accelerations(x, d["mass"])
            v = v + (a + an) * (0.5 * dt)
            a = an
    np.testing.assert_allclose(pos_d, x, rtol=0, atol=1e-13)
    np.testing.assert_allclose(vel_d, v, rtol=0, atol=1e-12)
    np.testing.assert_allclose(acc_d, a, rtol=1e-12, atol=1e-12)


def test_repeated_evaluations_reuse_buffers(ogx, golden):
    """Steady-state calls allocate nothing new and give identical results."""
    d = golden("disk4000")
    with ogx.AdaptiveFMM3D(p=6, threshold=32) as s:
        a1 = s.compute_accelerations(d["pos"], d["mass"])
        a2 = s.compute_accelerations(d["pos"], d["mass"])
        small = golden("plummer2000_s2")
        s.compute_accelerations(small["pos"], small["mass"])
        a3 = s.compute_accelerations(d["pos"], d["mass"])
    np.testing.assert_array_equal(a1, a2)
    np.testing.assert_array_equal(a1, a3)
