"""The third form, beyond the reference: FP64 with rotation-based M2L (OGX_PREC_FP64_ROT).

The reference translates with the dense O(p^4) formulas and defers an O(p^3) rotation
scheme (README.md:75 of the reference).  Here each M2L operator T_o is factored as
Q_o^-1 Z_|o| Q_o: a rotation taking the offset o to the z axis, the z-axis translation
(which couples only equal orders m) and the rotation back.  The factors are exact in exact
arithmetic, so this form differs from the plain one only by rounding; it is checked against
the reference's own AdaptiveFMM3D results (golden fixtures) with the plain form's bar,
max_rel <= 1e-12, and against the plain form directly, potentials included.
"""
import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu

CASES = [("plummer2000_s2", "fmm_p4", 4, 64, 0.0), ("plummer2000_s2", "fmm_p8", 8, 64, 0.0),
         ("cube1000_s1", "fmm_p8_t16", 8, 16, 0.0), ("clump", "fmm_p4_t16", 4, 16, 0.0),
         ("coincident", "fmm_p4_t4_eps", 4, 4, 0.01), ("disk4000", "fmm_p6_t32", 6, 32, 0.0)]


@pytest.mark.parametrize("name,key,p,thr,eps", CASES)
def test_rotation_form_matches_reference(ogx, golden, name, key, p, thr, eps):
    d = golden(name)
    with ogx.AdaptiveFMM3D(eps=eps, p=p, threshold=thr, precision=ogx.PREC_FP64_ROT) as s:
        acc = s.compute_accelerations(d["pos"], d["mass"])
        assert "rotation" in s.name()
    mx, rms = rel_err(d[key], acc)
    assert mx <= 1e-12, (mx, rms)


@pytest.mark.parametrize("p", [1, 2, 3, 5, 7, 8, 9, 10, 11, 12])
def test_rotation_form_equals_plain_form(ogx, golden, p):
    d = golden("disk4000")
    out = []
    for prec in (ogx.PREC_FP64, ogx.PREC_FP64_ROT):
        with ogx.AdaptiveFMM3D(p=p, threshold=32, precision=prec) as s:
            out.append(s.compute_accelerations(d["pos"], d["mass"], with_potential=True))
    (a0, p0), (a1, p1) = out
    mx, _ = rel_err(a0, a1)
    assert mx <= 1e-12, (p, mx)
    assert np.max(np.abs(p1 - p0) / np.abs(p0)) <= 1e-12


def test_rotation_form_on_a_large_clustered_system(ogx):
    """262,144 bodies of the disk+bulge galaxy, p = 8: the two FP64 forms agree."""
    import ogx_ic

    pos, mass, _ = ogx_ic.disk_bulge(262_144, seed=3)
    res = []
    for prec in (ogx.PREC_FP64, ogx.PREC_FP64_ROT):
        with ogx.AdaptiveFMM3D(p=8, threshold=64, precision=prec) as s:
            res.append(s.compute_accelerations(pos, mass))
    mx, rms = rel_err(res[0], res[1])
    assert mx <= 1e-11 and rms <= 1e-13, (mx, rms)
