"""C++ drop-in boundary: the B200 solvers behind the reference's ForceSolver3D seam.

oracle/_ref/dropin_check is compiled from the reference's own headers
(src3d/AdaptiveFMM3D.hpp, DirectSolver3D.hpp, Integrator3D.hpp,
InitialConditions3D.hpp) plus on-galaxy_b200/cpp/ogx_force_solver.hpp, so these
tests exercise exactly the code a reference user would write: a
`const ForceSolver3D&` handed to VelocityVerlet3D.  The binary exists only where
the reference sources were present at build time; the tests skip without it.
"""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "dropin_check")


def _run(*args, timeout=600):
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/dropin_check not built (reference sources absent at build time)")
    r = subprocess.run([BIN, *map(str, args)], capture_output=True, text=True, timeout=timeout)
    line = r.stdout.strip().splitlines()[-1] if r.stdout.strip() else "{}"
    return r.returncode, json.loads(line)


def test_dropin_error_path_without_device():
    """No GPU: the adapter turns the C-ABI status into std::runtime_error (no exit())."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    rc, out = _run(500, 4, 32)
    assert rc == 3
    assert "no CUDA device" in out["error"]


@pytest.mark.gpu
@pytest.mark.parametrize("n,p,thr", [(4096, 6, 32), (3000, 8, 64)])
def test_dropin_matches_reference_solvers(n, p, thr):
    rc, out = _run(n, p, thr)
    assert rc == 0, out
    assert out["fmm_max_rel"] <= 1e-12
    assert out["direct_max_rel"] <= 1e-12
    assert out["verlet_max_rel"] <= 1e-12
    assert out["boxes_ogx"] == out["boxes_ref"]
    assert out["maxocc_ogx"] == out["maxocc_ref"]
    # mixed form vs the reference FMM: FP32 near field / split-FP16 M2L rounding only
    assert out["mixed_rms_rel"] <= 5e-6
