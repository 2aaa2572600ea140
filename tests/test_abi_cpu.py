"""C-ABI checks that need no GPU: the library loads, exports every entry point
of include/ogx.h, validates arguments, reports a missing device as a status
code, and its host-built translation matrices equal the oracle's operators."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ogx.h")


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ogx_[a-z_0-9]+)\s*\(", txt)))


def test_header_and_binding_agree(ogx):
    assert sorted(ogx.EXPORTS) == header_symbols()


def test_library_exports_every_symbol(ogx):
    lib = ogx.load()
    for sym in header_symbols():
        assert hasattr(lib, sym), sym


def test_strerror_names_every_status(ogx):
    lib = ogx.load()
    for code in range(8):
        assert lib.ogx_strerror(code).decode() not in ("", "unknown status")
    assert lib.ogx_strerror(99).decode() == "unknown status"


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.parametrize("kw", [dict(p=0), dict(p=13), dict(threshold=0), dict(eps=-1.0), dict(precision=7)])
def test_invalid_parameters_are_rejected(ogx, kw):
    with pytest.raises(ogx.OgxError) as e:
        ogx.AdaptiveFMM3D(**kw)
    assert e.value.code in (ogx.ERR_INVALID, ogx.ERR_NO_DEVICE)
    if not _cuda_available():
        # without a device the argument check still comes first
        assert e.value.code == ogx.ERR_INVALID


@pytest.mark.skipif(_cuda_available(), reason="a GPU is present")
def test_no_device_is_a_status_not_a_crash(ogx):
    with pytest.raises(ogx.OgxError) as e:
        ogx.AdaptiveFMM3D()
    assert e.value.code == ogx.ERR_NO_DEVICE


def _real(z, p):
    out = []
    for n in range(p + 1):
        out.append(z[n * n + n].real)
        for m in range(1, n + 1):
            out += [z[n * n + n + m].real, z[n * n + n + m].imag]
    return np.array(out)


def _scaled(z, p, s, power):
    z = z.copy()
    for n in range(p + 1):
        for m in range(-n, n + 1):
            z[n * n + n + m] *= s ** (power * n)
    return z


@pytest.mark.parametrize("p", [2, 5, 8, 12])
def test_translation_matrices_match_oracle_operators(ogx, oracle, p):
    """The level-independent matrices reproduce fmm::M2M / L2L / M2L (FmmExpansions3D.hpp:242-330)."""
    rng = np.random.default_rng(p)
    side, h = 0.37, 0.185
    pc = np.array([0.3, -0.2, 0.9])
    worst = 0.0
    for s in range(8):
        d = np.array([h / 2 if s & 1 else -h / 2, h / 2 if s & 2 else -h / 2, h / 2 if s & 4 else -h / 2])
        cc = pc + d
        pts, q = cc + rng.uniform(-h / 2, h / 2, (12, 3)), rng.uniform(0.5, 1.5, 12)
        Mc = oracle.p2m(p, cc, pts, q)
        got = ogx.operator_matrix(0, p, s) @ _real(_scaled(Mc, p, h, -1), p)
        ref = _real(_scaled(oracle.translate(0, p, cc, pc, Mc), p, side, -1), p)
        worst = max(worst, np.abs(got - ref).max() / np.abs(ref).max())
        src = pc + np.array([5.0, 1.0, -2.0]) + rng.uniform(-0.3, 0.3, (12, 3))
        Lp = oracle.p2l(p, pc, src, q)
        got = ogx.operator_matrix(1, p, s) @ _real(_scaled(Lp, p, side, 1), p)
        ref = _real(_scaled(oracle.translate(2, p, pc, cc, Lp), p, h, 1), p)
        worst = max(worst, np.abs(got - ref).max() / np.abs(ref).max())
    for idx in rng.choice([i for i in range(343) if max(abs(i % 7 - 3), abs(i // 7 % 7 - 3), abs(i // 49 - 3)) >= 2],
                          24, replace=False):
        o = np.array([idx % 7 - 3, (idx // 7) % 7 - 3, idx // 49 - 3])
        tc = np.array([0.1, 0.2, -0.4])
        sc = tc + side * o
        pts, q = sc + rng.uniform(-h, h, (10, 3)), rng.uniform(0.5, 1.5, 10)
        Ms = oracle.p2m(p, sc, pts, q)
        got = ogx.operator_matrix(2, p, int(idx)) @ _real(_scaled(Ms, p, side, -1), p) / side
        ref = _real(_scaled(oracle.translate(1, p, sc, tc, Ms), p, side, 1), p)
        worst = max(worst, np.abs(got - ref).max() / np.abs(ref).max())
    assert worst < 1e-13


def test_adjacent_offsets_have_no_m2l_matrix(ogx):
    assert np.all(ogx.operator_matrix(2, 4, 3 + 7 * 3 + 49 * 3) == 0.0)  # offset (0,0,0)
    assert np.all(ogx.operator_matrix(2, 4, 4 + 7 * 2 + 49 * 3) == 0.0)  # offset (1,-1,0)
    with pytest.raises(ogx.OgxError):
        ogx.operator_matrix(2, 4, 343)


@pytest.mark.parametrize("p", [1, 2, 5, 8, 12])
def test_rotation_factors_multiply_back_to_the_m2l_matrix(ogx, p):
    """Kind 3 returns Q^-1 Z Q, the rotation-based form's factors of M2L offset o multiplied
    out; it must equal the dense M2L matrix (kind 2) up to rounding, entry by entry."""
    for idx in range(0, 343, 7):
        ox, oy, oz = idx % 7 - 3, (idx // 7) % 7 - 3, idx // 49 - 3
        T = ogx.operator_matrix(2, p, idx)
        R = ogx.operator_matrix(3, p, idx)
        if max(abs(ox), abs(oy), abs(oz)) <= 1:
            assert not T.any() and not R.any()
            continue
        # each row's entries against that row's scale (rows of high degree are small)
        scale = np.abs(T).max(axis=1, keepdims=True)
        assert np.max(np.abs(R - T) / scale) <= 1e-13, (p, idx)


def test_python_params_struct_covers_the_c_struct(ogx):
    """ogx_params_default fills the whole C struct: the binding's mirror must be at least as
    large (a canary behind it must stay intact) and read back the documented defaults."""
    import ctypes as C

    class Guarded(C.Structure):
        _fields_ = [("prm", ogx.Params), ("canary", C.c_uint64 * 4)]

    g = Guarded()
    for i in range(4):
        g.canary[i] = 0x5A5A5A5A5A5A5A5A
    assert ogx.load().ogx_params_default(C.byref(g.prm)) == 0
    assert all(g.canary[i] == 0x5A5A5A5A5A5A5A5A for i in range(4))
    assert (g.prm.G, g.prm.eps, g.prm.p, g.prm.leaf_capacity) == (1.0, 0.0, 8, 64)
    assert g.prm.softening == ogx.SOFT_PLUMMER
