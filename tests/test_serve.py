"""The serving loop (on-galaxy_b200/cpp/ogx_serve.cpp): integration jobs from a seeded
Poisson stream, admitted under a device-memory budget, each running with its state resident
on the device while others run beside it.

The reference has no serving loop; what carries over is its integrator
(src3d/Integrator3D.hpp:23-40, one force evaluation per leapfrog step) and its initial
conditions (Plummer, src3d/InitialConditions3D.hpp; disk+bulge mergers,
src3d/gpu/GalaxyIC.hpp:43-125).  The property checked here is that a job's result does
not depend on what else runs: the final positions and velocities of every job are
bit-identical when it runs alone and when it shares the GPU.
"""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SERVE = os.path.join(ROOT, "on-galaxy_b200", "ogx_serve")


def _serve(*args, expect_rc=0):
    if not os.path.exists(SERVE):
        pytest.skip("ogx_serve not built")
    r = subprocess.run([SERVE, *map(str, args)], capture_output=True, text=True, timeout=900)
    assert r.returncode == expect_rc, r.stdout[-2000:] + r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


SMALL = ("--jobs", 8, "--rate", 400, "--nmin", 16384, "--nmax", 200000, "--smin", 3, "--smax", 8,
         "--orders", "6,8,12", "--seed", 7)


def test_serve_rejects_bad_arguments():
    if not os.path.exists(SERVE):
        pytest.skip("ogx_serve not built")
    r = subprocess.run([SERVE, "--jobs", "0"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
    r = subprocess.run([SERVE, "--nmin", "100", "--nmax", "10"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2


def test_serve_reports_missing_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    out = _serve("--jobs", 2, expect_rc=3)
    assert "error" in out


@pytest.mark.gpu
def test_jobs_give_the_same_bits_alone_and_in_the_mix():
    solo = _serve(*SMALL, "--solo")
    mixed = _serve(*SMALL)
    assert solo["failed"] == 0 and mixed["failed"] == 0
    assert solo["rejected"] == 0 and mixed["rejected"] == 0
    # jobs overlapped on the GPU
    assert mixed["peak_concurrent"] >= 2
    a = {j["id"]: j for j in solo["jobs_detail"]}
    b = {j["id"]: j for j in mixed["jobs_detail"]}
    assert a.keys() == b.keys()
    kinds = set()
    for k in a:
        assert (a[k]["n"], a[k]["p"], a[k]["steps"]) == (b[k]["n"], b[k]["p"], b[k]["steps"])
        assert a[k]["digest"] == b[k]["digest"], f"job {k} differs when run in the mix"
        kinds.add(a[k]["kind"])
    assert len(kinds) == 2
    assert solo["steps"] == mixed["steps"] == sum(j["steps"] for j in solo["jobs_detail"])
    assert 0 < mixed["p50_step_ms"] <= mixed["p99_step_ms"]
    # the admission estimate covers what each job used alone
    for j in solo["jobs_detail"]:
        assert j["peak_mb"] <= j["need_mb"], j


@pytest.mark.gpu
def test_jobs_above_the_budget_are_refused_and_the_rest_run():
    out = _serve("--jobs", 6, "--rate", 400, "--nmin", 16384, "--nmax", 1 << 20, "--smin", 2, "--smax", 3,
                 "--orders", "8", "--seed", 3, "--hbm-gb", 0.4)
    assert out["failed"] == 0
    refused = [j for j in out["jobs_detail"] if j["rejected"]]
    ran = [j for j in out["jobs_detail"] if not j["rejected"]]
    assert out["rejected"] == len(refused) >= 1 and len(ran) >= 1
    assert all(j["need_mb"] > 400 for j in refused)
    assert all(j["need_mb"] <= 400 and j["status"] == 0 for j in ran)
    assert out["steps"] == sum(j["steps"] for j in ran)


@pytest.mark.gpu
def test_fp64_jobs_give_the_same_bits_alone_and_in_the_mix():
    args = ("--jobs", 4, "--rate", 400, "--nmin", 16384, "--nmax", 65536, "--smin", 2, "--smax", 4,
            "--orders", "6,8", "--seed", 11, "--precision", "fp64")
    solo = _serve(*args, "--solo")
    mixed = _serve(*args)
    assert solo["precision"] == mixed["precision"] == "fp64"
    assert [j["digest"] for j in solo["jobs_detail"]] == [j["digest"] for j in mixed["jobs_detail"]]


@pytest.mark.gpu
def test_softened_jobs_give_the_same_bits_alone_and_in_the_mix():
    """Jobs with eps = 0.05 and the spline kernel (far field corrected inside its support):
    the same bits alone and in the mix, and different bits from the Plummer kernel."""
    args = ("--jobs", 4, "--rate", 400, "--nmin", 16384, "--nmax", 65536, "--smin", 2, "--smax", 4,
            "--orders", "6,8", "--seed", 13, "--eps", 0.05)
    solo = _serve(*args, "--softening", "spline", "--solo")
    mixed = _serve(*args, "--softening", "spline")
    plummer = _serve(*args, "--solo")
    assert solo["failed"] == mixed["failed"] == plummer["failed"] == 0
    digests = [j["digest"] for j in solo["jobs_detail"]]
    assert digests == [j["digest"] for j in mixed["jobs_detail"]]
    assert all(a != b for a, b in zip(digests, [j["digest"] for j in plummer["jobs_detail"]]))


@pytest.mark.gpu
def test_softened_ensemble_members_match_their_solo_runs():
    """Spline-softened systems step eagerly (their steps are never captured), so with --graph
    every lockstep step runs the members on the ensemble's host threads; each member still
    ends bit-identical to its solo run."""
    args = ("--ensemble", "--steps", 3, "--jobs", 10, "--nmin", 8192, "--nmax", 65536, "--orders", "6,8",
            "--seed", 17, "--eps", 0.05, "--softening", "spline")
    ens = _serve(*args, "--graph")
    solo = _serve(*args, "--solo")
    assert ens["failed"] == 0 and solo["failed"] == 0
    assert ens["graph_launch_steps"] == 0 and ens["member_by_member_steps"] == 3
    assert [j["digest"] for j in ens["jobs_detail"]] == [j["digest"] for j in solo["jobs_detail"]]


def test_serve_rejects_an_unknown_softening():
    if not os.path.exists(SERVE):
        pytest.skip("ogx_serve not built")
    r = subprocess.run([SERVE, "--softening", "gaussian"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2


ENS = ("--ensemble", "--steps", 4, "--jobs", 12, "--nmin", 8192, "--nmax", 131072, "--orders", "6,8", "--seed", 5)


@pytest.mark.gpu
def test_ensemble_members_match_their_solo_runs():
    ens = _serve(*ENS)
    solo = _serve(*ENS, "--solo")
    assert ens["mode"] == "ensemble" and ens["failed"] == 0 and ens["peak_concurrent"] == 12
    assert ens["steps"] == 12 * 4 == solo["steps"]
    assert 0 < ens["ensemble_step_ms_p50"] <= ens["ensemble_step_ms_p99"]
    assert [j["digest"] for j in ens["jobs_detail"]] == [j["digest"] for j in solo["jobs_detail"]]


@pytest.mark.gpu
def test_ensemble_in_one_graph_launch_per_step_matches_solo_runs():
    """--graph: after each system has captured its step, a lockstep step of all systems is
    one CUDA graph launch (ogx_ensemble_step); every system still ends bit-identical to its
    solo run."""
    args = ("--ensemble", "--steps", 6, "--jobs", 10, "--nmin", 8192, "--nmax", 131072, "--orders", "6,8",
            "--seed", 5)
    ens = _serve(*args, "--graph")
    solo = _serve(*args, "--solo")
    assert ens["graph"] is True and ens["failed"] == 0
    assert ens["graph_launch_steps"] >= 2 and ens["graph_launch_steps"] + ens["member_by_member_steps"] == 6
    assert [j["digest"] for j in ens["jobs_detail"]] == [j["digest"] for j in solo["jobs_detail"]]


@pytest.mark.gpu
def test_ensemble_autotune_picks_candidates_and_reuses_its_cache(tmp_path):
    """The tuner picks leaf capacity, M2L batch width and P2P tile shape from their candidate
    sets; its JSON cache is written after the run and, read by a second run, gives the same
    choices without a new search."""
    cache = tmp_path / "tune.json"
    args = ("--ensemble", "--steps", 2, "--jobs", 4, "--nmin", 8192, "--nmax", 65536, "--orders", "6,8",
            "--seed", 9, "--autotune", "--tune-cache", str(cache))
    out = _serve(*args)
    assert out["failed"] == 0 and out["autotune"] is True
    for j in out["jobs_detail"]:
        assert j["thr"] in (32, 48, 64, 96, 128)
        assert j["m2l_tile_targets"] in (32, 64, 96, 128)
        assert j["near_units"] in (32, 64)
    saved = json.loads(cache.read_text())
    assert saved and all(set(v) == {"leaf_capacity", "m2l_tile_targets", "near_units", "ms"} for v in saved.values())
    again = _serve(*args)
    assert all(j["tuned_from_cache"] for j in again["jobs_detail"])
    pick = lambda o: [(j["thr"], j["m2l_tile_targets"], j["near_units"]) for j in o["jobs_detail"]]  # noqa: E731
    assert pick(again) == pick(out)
