"""ogx_direct_eval_noalloc: the direct sum for callers that must not allocate device memory.

Such callers (latency-bound processes whose other streams a cudaMalloc/cudaFree could
stall, or processes that reserve all their device memory up front under a fixed
budget) get the FP64 direct sum with its staging in a fixed per-GPU array of the
library (at most 65536 bodies).  Its results must equal those of the ordinary direct
solver (ogx_eval on an OGX_SOLVER_DIRECT handle) within the direct-solver tolerance
of the other tests, call after call, since every call reuses the same array.

This file is named to be collected last, so a run that stops at the first failure
has run every other test before it.
"""
import numpy as np
import pytest

DIRECT_TOL = 1e-12


def _bodies(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.normal(size=(n, 3))
    mass = rng.uniform(0.5, 1.5, n) / n
    return pos, mass


def _max_rel(ref, got):
    a = np.linalg.norm(ref, axis=-1) if ref.ndim == 2 else np.abs(ref)
    e = np.linalg.norm(got - ref, axis=-1) if ref.ndim == 2 else np.abs(got - ref)
    return float(np.max(e / np.maximum(a, 1e-300)))


def test_noalloc_rejects_more_than_the_maximum(ogx):
    """Checked before any device work, so this runs without a GPU too."""
    n = ogx.NOALLOC_MAX_BODIES + 1
    pos, mass = np.zeros((n, 3)), np.ones(n)
    with pytest.raises(ogx.OgxError) as e:
        ogx.direct_eval_noalloc(pos, mass)
    assert e.value.code == ogx.ERR_INVALID
    assert "exceeds the no-alloc maximum" in str(e.value)


@pytest.mark.gpu
def test_noalloc_matches_direct_solver_on_consecutive_calls(ogx):
    G, eps = 1.0, 0.01
    # first call larger than the second and with potentials: stale contents of the
    # shared array must not leak into the later, smaller call
    cases = [(_bodies(5000, 1), True), (_bodies(3001, 2), False), (_bodies(ogx.NOALLOC_MAX_BODIES, 3), True)]
    for (pos, mass), with_pot in cases:
        with ogx.DirectSolver3D(G=G, eps=eps) as d:
            ref_acc, ref_pot = d.compute_accelerations(pos, mass, with_potential=True)
        got = ogx.direct_eval_noalloc(pos, mass, G=G, eps=eps, with_pot=with_pot)
        acc, pot = got if with_pot else (got, None)
        assert _max_rel(ref_acc, acc) <= DIRECT_TOL
        if with_pot:
            assert _max_rel(ref_pot, pot) <= DIRECT_TOL


@pytest.mark.gpu
def test_noalloc_on_a_caller_stream(ogx):
    """A caller's own (non-default) stream is honoured: the call returns with the results in
    place, twice in a row on the same stream."""
    import torch

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    for seed in (4, 5):
        pos, mass = _bodies(7000, seed)
        with ogx.DirectSolver3D(G=1.0, eps=0.0) as d:
            ref_acc = d.compute_accelerations(pos, mass)
        acc = ogx.direct_eval_noalloc(pos, mass, G=1.0, eps=0.0, stream=stream.cuda_stream)
        assert _max_rel(ref_acc, acc) <= DIRECT_TOL
