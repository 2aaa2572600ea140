"""OGX_SOFT_SPLINE: the compact-support softening kernel with the far field corrected
within its support (an extension beyond the reference, which softens the P2P part only,
src3d/AdaptiveFMM3D.hpp:18, and names the resulting seam as its energy-drift cause,
README.md:73-75).

The kernel is the cubic spline of Monaghan & Lattanzio (1985) in the form GADGET-2 uses
(Springel 2005, MNRAS 364, 1105, eq. 4), support h = 2.8 eps.  It is exactly Newtonian
beyond h, so the expansions are exact for it there; the library corrects every pair the
far field takes closer than h.  Bars:
  * the kernel (numpy restatement below) has the published properties;
  * the GPU direct sum with the spline matches the numpy direct sum to 1e-12;
  * the adaptive FMM with the spline matches the spline direct sum at the expansion's
    truncation level, while with Plummer's kernel the FMM differs from the Plummer direct
    sum by the seam, an order of magnitude more;
  * the mixed form matches the FP64 form with the spline to 1e-6 RMS.
"""
import numpy as np
import pytest

from helpers import rel_err


def spline_gk(r2, h):
    """(g, k) of the spline: acceleration m g (r_j - r_i), potential -G m k."""
    r2 = np.asarray(r2, np.float64)
    r = np.sqrt(r2)
    g = np.empty_like(r)
    k = np.empty_like(r)
    far = r >= h
    with np.errstate(divide="ignore"):
        g[far] = r[far] ** -3
        k[far] = 1.0 / r[far]
    u = r / h
    a = (~far) & (u < 0.5)
    b = (~far) & (u >= 0.5)
    ua, ub = u[a], u[b]
    g[a] = (32.0 / 3.0 + ua ** 2 * (32.0 * ua - 38.4)) / h ** 3
    k[a] = (2.8 - ua ** 2 * (16.0 / 3.0 + ua ** 2 * (6.4 * ua - 9.6))) / h
    g[b] = (64.0 / 3.0 - 48.0 * ub + 38.4 * ub ** 2 - 32.0 / 3.0 * ub ** 3 - 1.0 / (15.0 * ub ** 3)) / h ** 3
    k[b] = (3.2 - 1.0 / (15.0 * ub) - ub ** 2 * (32.0 / 3.0 + ub * (-16.0 + ub * (9.6 - 32.0 / 15.0 * ub)))) / h
    return g, k


def direct_spline(pos, mass, eps, G=1.0):
    h = 2.8 * eps
    n = len(mass)
    acc = np.zeros((n, 3))
    pot = np.zeros(n)
    for i0 in range(0, n, 512):
        d = pos[None, :, :] - pos[i0:i0 + 512, None, :]
        r2 = np.sum(d * d, axis=2)
        g, k = spline_gk(np.where(r2 > 0, r2, 1.0), h)
        m = np.broadcast_to(mass[None, :], r2.shape).copy()
        idx = np.arange(i0, min(n, i0 + 512))
        m[idx - i0, idx] = 0.0
        acc[i0:i0 + 512] = G * np.einsum("ij,ijk->ik", m * g, d)
        pot[i0:i0 + 512] = -G * np.sum(m * k, axis=1)
    return acc, pot


def test_spline_kernel_properties():
    eps = 0.05
    h = 2.8 * eps
    # Plummer-equivalent at the centre: k(0) = 1 / eps
    g0, k0 = spline_gk(np.array([0.0]), h)
    assert abs(k0[0] - 1.0 / eps) < 1e-12 / eps
    assert abs(g0[0] - 32.0 / 3.0 / h ** 3) < 1e-9 / h ** 3
    # Newtonian from the support on
    r = np.array([h, 1.5 * h, 10 * h])
    g, k = spline_gk(r * r, h)
    assert np.allclose(g, r ** -3, rtol=1e-12) and np.allclose(k, 1.0 / r, rtol=1e-12)
    # continuous at u = 1/2 and u = 1 (value and force)
    for u in (0.5, 1.0):
        lo, hi = spline_gk(np.array([(u * h * (1 - 1e-12)) ** 2]), h), spline_gk(np.array([(u * h * (1 + 1e-12)) ** 2]), h)
        assert abs(lo[0][0] - hi[0][0]) < 1e-9 * abs(hi[0][0]) and abs(lo[1][0] - hi[1][0]) < 1e-9 * abs(hi[1][0])
    # the force is minus the potential's gradient: g = -(1/r) dk/dr
    for u in (0.1, 0.3, 0.49, 0.51, 0.7, 0.95, 1.2):
        r0, dr = u * h, 1e-6 * h
        kp = spline_gk(np.array([(r0 + dr) ** 2]), h)[1][0]
        km = spline_gk(np.array([(r0 - dr) ** 2]), h)[1][0]
        g = spline_gk(np.array([r0 * r0]), h)[0][0]
        assert abs(-(kp - km) / (2 * dr) / r0 - g) < 1e-6 * g, u


def _plummer(n, seed):
    from ogx_ic import plummer
    pos, _, mass = plummer(n, seed=seed)
    return pos, mass


@pytest.mark.gpu
def test_direct_spline_matches_numpy(ogx):
    pos, mass = _plummer(3000, 5)
    eps = 0.05
    ref_acc, ref_pot = direct_spline(pos, mass, eps)
    with ogx.DirectSolver3D(eps=eps, softening=ogx.SOFT_SPLINE) as s:
        acc, pot = s.compute_accelerations(pos, mass, with_potential=True)
    mx, _ = rel_err(ref_acc, acc)
    assert mx <= 1e-12, mx
    assert np.max(np.abs(pot - ref_pot) / np.abs(ref_pot)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("eps", [0.02, 0.2])
def test_fmm_spline_matches_spline_direct_without_the_seam(ogx, eps):
    """Plummer sphere N=16384, p=8, leaf capacity 64.  eps=0.02: the support is below the
    core's leaf edges, so no far-field pair needs a correction; eps=0.2: it reaches across
    leaves and the S lists carry the correction."""
    pos, mass = _plummer(16384, 11)
    res = {}
    for kind in (ogx.SOFT_PLUMMER, ogx.SOFT_SPLINE):
        with ogx.DirectSolver3D(eps=eps, softening=kind) as d:
            ref_acc, ref_pot = d.compute_accelerations(pos, mass, with_potential=True)
        with ogx.AdaptiveFMM3D(eps=eps, p=8, threshold=64, softening=kind) as s:
            acc, pot = s.compute_accelerations(pos, mass, with_potential=True)
            st = s.stats()
        _, rms = rel_err(ref_acc, acc)
        prms = float(np.sqrt(np.mean((pot - ref_pot) ** 2) / np.mean(ref_pot ** 2)))
        res[kind] = (rms, prms, st["list_s"])
    rms_p, prms_p, ls_p = res[ogx.SOFT_PLUMMER]
    rms_s, prms_s, ls_s = res[ogx.SOFT_SPLINE]
    assert ls_p == 0
    if eps >= 0.2:
        assert ls_s > 0
    # the spline FMM sits at the truncation level of p = 8 (1e-5 class on Plummer data)
    assert rms_s <= 3e-5, res
    assert prms_s <= 3e-6, res
    # the Plummer FMM carries the seam: at least ten times the spline's error
    assert rms_p >= 10 * rms_s, res


@pytest.mark.gpu
def test_mixed_spline_matches_fp64_spline(ogx):
    pos, mass = _plummer(16384, 12)
    eps = 0.2
    with ogx.AdaptiveFMM3D(eps=eps, p=8, threshold=64, softening=ogx.SOFT_SPLINE) as s:
        ref, ref_pot = s.compute_accelerations(pos, mass, with_potential=True)
    with ogx.AdaptiveFMM3D(eps=eps, p=8, threshold=64, precision=ogx.PREC_MIXED, softening=ogx.SOFT_SPLINE) as s:
        acc, pot = s.compute_accelerations(pos, mass, with_potential=True)
        assert s.stats()["list_s"] > 0
    _, rms = rel_err(ref, acc)
    assert rms <= 1e-6, rms
    assert float(np.sqrt(np.mean((pot - ref_pot) ** 2) / np.mean(ref_pot ** 2))) <= 1e-6


def test_softening_parameter_is_checked(ogx):
    with pytest.raises(ogx.OgxError) as ei:
        ogx.AdaptiveFMM3D(eps=0.1, softening=7)
    assert ei.value.code == 1   # OGX_ERR_INVALID, before any device is touched
