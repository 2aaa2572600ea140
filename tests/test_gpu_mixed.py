"""GPU checks of the mixed-precision form (FP32 P2P, scaled FP16 hi/lo tensor-core M2L,
FP64 translations), through the C ABI.

Tolerances (stated per the precision design):
  * vs the FP64 form at the same p and leaf capacity: RMS <= 5e-6, max_rel <= 1e-3.
    The budget is set by the FP32 near field: leaf-centred FP32 positions carry an
    absolute error of 2^-24 x leaf size, so a pair at separation r gets a relative
    force error ~3e-8 x leaf/r (measured on CPU for Plummer N=2000: RMS 2.6e-6);
    the split M2L (three FP16 products of 11-bit halves, power-of-two scales,
    FP32 accumulation per combination) contributes ~2^-22 per product;
  * vs the FP64 direct oracle: RMS within 5e-6 of the FP64 form's own truncation error.
"""
import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("p", [2, 4, 6, 8, 9, 10, 11, 12])
def test_mixed_vs_fp64_form(ogx, golden, p):
    d = golden("plummer2000_s2")
    with ogx.AdaptiveFMM3D(p=p, threshold=64, precision=ogx.PREC_FP64) as s64:
        a64 = s64.compute_accelerations(d["pos"], d["mass"])
    with ogx.AdaptiveFMM3D(p=p, threshold=64, precision=ogx.PREC_MIXED) as sm:
        am = sm.compute_accelerations(d["pos"], d["mass"])
    mx, rms = rel_err(a64, am)
    assert rms <= 5e-6 and mx <= 1e-3, (p, mx, rms)


@pytest.mark.parametrize("name,thr", [("disk4000", 32), ("cube1000_s1", 16), ("clump", 16)])
def test_mixed_other_inputs(ogx, golden, name, thr):
    d = golden(name)
    with ogx.AdaptiveFMM3D(p=8, threshold=thr, precision=ogx.PREC_FP64) as s64:
        a64 = s64.compute_accelerations(d["pos"], d["mass"])
    with ogx.AdaptiveFMM3D(p=8, threshold=thr, precision=ogx.PREC_MIXED) as sm:
        am = sm.compute_accelerations(d["pos"], d["mass"])
    mx, rms = rel_err(a64, am)
    assert rms <= 5e-6, (name, mx, rms)


def test_mixed_cfg1_vs_direct_and_potentials(ogx, golden, oracle):
    d = golden("cfg1_plummer16384")
    with ogx.AdaptiveFMM3D(p=8, threshold=64, precision=ogx.PREC_MIXED) as sm:
        am, pm = sm.compute_accelerations(d["pos"], d["mass"], with_potential=True)
    _, rms_m = rel_err(d["direct"], am)
    _, rms_f = rel_err(d["direct"], d["fmm_p8_t64"])
    assert abs(rms_m - rms_f) <= 5e-6, (rms_m, rms_f)
    mx, rms = rel_err(d["fmm_p8_t64"], am)
    assert rms <= 5e-6, (mx, rms)
    _, pot_o = oracle.adaptive_fmm(d["pos"], d["mass"], p=8, thr=64)
    assert np.sqrt(np.sum((pm - pot_o) ** 2) / np.sum(pot_o ** 2)) <= 1e-6


def test_mixed_leapfrog_runs_and_tracks_fp64(ogx, golden):
    d = golden("plummer2000_s2")
    rng = np.random.default_rng(1)
    vel = 0.1 * rng.standard_normal(d["pos"].shape)
    out = []
    for prec in (ogx.PREC_FP64, ogx.PREC_MIXED):
        with ogx.AdaptiveFMM3D(p=8, threshold=64, precision=prec) as s:
            s.upload(d["pos"], vel, d["mass"])
            s.step(0.01, 5)
            out.append(s.download())
    np.testing.assert_allclose(out[1][0], out[0][0], rtol=0, atol=1e-9)
    assert rel_err(out[0][2], out[1][2])[1] <= 5e-6


def test_bounded_wait_runs_out_and_the_handle_stays_usable(ogx, golden):
    """The tensor-core pipeline's bounded mbarrier wait, given a barrier nothing arrives on,
    and the translation passes' bounded ready-flag wait, given a flag nothing sets, both give
    up after their poll limit and the host reports OGX_ERR_TIMEOUT (no copy or MMA is
    outstanding, so no GPU fault is involved); the same handle then evaluates as before."""
    d = golden("plummer2000_s2")
    with ogx.AdaptiveFMM3D(p=8, threshold=64, precision=ogx.PREC_MIXED) as s:
        a1 = s.compute_accelerations(d["pos"], d["mass"])
        for polls in (1, 1000):
            with pytest.raises(ogx.OgxError) as e:
                s.check_bounded_wait(polls)
            assert e.value.code == ogx.ERR_TIMEOUT
            s.synchronize()   # the error word was cleared when it was reported
        a2 = s.compute_accelerations(d["pos"], d["mass"])
    np.testing.assert_array_equal(a1, a2)


@pytest.mark.parametrize("units", [32, 64])
def test_every_tuning_choice_stays_within_the_mixed_tolerance(ogx, golden, units):
    """The autotuner's launch-shape knobs: the M2L batch width does not change any bit of the
    result, and every (batch width, near-field units) choice stays within the mixed form's
    tolerance of the FP64 form (RMS <= 5e-6, as above)."""
    d = golden("disk4000")
    with ogx.AdaptiveFMM3D(p=8, threshold=32, precision=ogx.PREC_FP64) as s64:
        a64 = s64.compute_accelerations(d["pos"], d["mass"])
    ref = None
    with ogx.AdaptiveFMM3D(p=8, threshold=32, precision=ogx.PREC_MIXED) as sm:
        for fill in (32, 64, 96, 128):
            sm.set_tuning(m2l_tile_targets=fill, near_units=units)
            assert sm.tuning() == {"m2l_tile_targets": fill, "near_units": units, "capture_steps": 0}
            am = sm.compute_accelerations(d["pos"], d["mass"])
            _, rms = rel_err(a64, am)
            assert rms <= 5e-6, (fill, units, rms)
            if ref is None:
                ref = am
            np.testing.assert_array_equal(am, ref)
        with pytest.raises(ogx.OgxError) as e:
            sm.set_tuning(m2l_tile_targets=48)
        assert e.value.code == ogx.ERR_INVALID


@pytest.mark.parametrize("softening", [0, 1])
def test_mixed_with_leaves_held_large_by_the_eps_floor(ogx, softening):
    """Disk+bulge galaxy of 100k bodies at eps = 0.05 (the reference's merger setting): the
    eps floor stops splitting in the bulge, so leaves hold more than the leaf capacity and the near
    field spreads each over many work items (chunks of 32 targets).  Mixed vs FP64 form,
    both with Plummer's kernel and with the spline."""
    from ogx_ic import disk_bulge
    pos, mass, _ = disk_bulge(100000, seed=4)
    kw = dict(eps=0.05, p=8, threshold=64, softening=softening)
    with ogx.AdaptiveFMM3D(precision=ogx.PREC_FP64, **kw) as s64:
        a64, p64 = s64.compute_accelerations(pos, mass, with_potential=True)
        st = s64.stats()
    with ogx.AdaptiveFMM3D(precision=ogx.PREC_MIXED, **kw) as sm:
        am, pm = sm.compute_accelerations(pos, mass, with_potential=True)
    assert st["max_leaf_occupancy"] > 64, st["max_leaf_occupancy"]   # above the leaf capacity: the floor acts
    mx, rms = rel_err(a64, am)
    assert rms <= 1e-6 and mx <= 1e-3, (mx, rms)
    assert float(np.sqrt(np.mean((pm - p64) ** 2) / np.mean(p64 ** 2))) <= 1e-6
