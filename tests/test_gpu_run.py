"""Running a simulation on the device: merger initial conditions, FP64 diagnostics,
float32 frames and the merger driver's output files.

References: makeDisk / setCircularVelocities / placeGalaxy (src3d/gpu/GalaxyIC.hpp:43-125),
computeDiagnostics (src3d/Diagnostics3D.hpp:20-38), comSep and the frames.bin /
species.bin writer (src3d/gpu/galaxy_sim.cu:179-226).
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SIM = os.path.join(ROOT, "on-galaxy_b200", "ogx_galaxy_sim")


def _run_sim(*args, cwd):
    if not os.path.exists(SIM):
        pytest.skip("ogx_galaxy_sim not built")
    return subprocess.run([SIM, *map(str, args)], capture_output=True, text=True, timeout=600, cwd=cwd)


def test_driver_reports_missing_device(tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    r = _run_sim("--N", 100, "--steps", 1, "--out", tmp_path / "x", cwd=tmp_path)
    assert r.returncode == 3
    assert "no CUDA device" in r.stderr


@pytest.mark.gpu
def test_ic_merger_is_deterministic_and_follows_the_profiles(ogx):
    n_per = 20000
    with ogx.AdaptiveFMM3D(p=6, threshold=32) as s:
        sp1 = s.ic_merger(n_per, seed=3)
        pos1, vel1, _ = s.download()
    with ogx.AdaptiveFMM3D(p=6, threshold=32) as s:
        sp2 = s.ic_merger(n_per, seed=3)
        pos2, vel2, _ = s.download()
    assert np.array_equal(pos1, pos2) and np.array_equal(vel1, vel2) and np.array_equal(sp1, sp2)
    assert (sp1[:n_per] == 0).all() and (sp1[n_per:] == 1).all()
    nd = n_per - round(0.2 * n_per)
    g0 = pos1[:nd] - np.array([-5.0, 0.0, 0.0])              # galaxy 0 disk, untilted
    R = np.hypot(g0[:, 0], g0[:, 1])
    assert abs(R.mean() - 2.0) < 0.04                         # <R> of the Gamma(2) profile, Rd = 1
    assert abs(g0[:, 2].std() - np.pi / np.sqrt(12.0) * 0.1) < 0.004   # sech^2, z0 = 0.1
    bul = np.linalg.norm(pos1[nd:n_per] - np.array([-5.0, 0.0, 0.0]), axis=1)
    s_half = np.sqrt(0.5) * 50.0 / 51.0                       # half-mass radius of the bulge cut at 50 a
    assert abs(np.median(bul) - 0.2 * s_half / (1.0 - s_half)) < 0.02
    # disk rotates counter-clockwise with v_c^2 = -a_R R of the galaxy's own field
    v = vel1[:nd] - np.array([0.25, 0.0, 0.0])
    vphi = (g0[:, 0] * v[:, 1] - g0[:, 1] * v[:, 0]) / np.maximum(R, 1e-9)
    assert np.median(vphi) > 0.3
    assert np.allclose(pos1[n_per:].mean(0), [5.0, 0.0, 0.0], atol=0.1)


@pytest.mark.gpu
def test_diagnostics_match_host_sums_and_direct_potential_energy(ogx, oracle):
    n_per = 3000
    with ogx.AdaptiveFMM3D(eps=0.0, p=8, threshold=32) as s:
        species = s.ic_merger(n_per, seed=5)
        pos, vel, _ = s.download()
        d = s.diagnostics()
        frame = s.download_frame()
    nd, nb = n_per - round(0.2 * n_per), round(0.2 * n_per)
    mass = np.concatenate([np.full(nd, 1.0 / nd), np.full(nb, 0.25 / nb)] * 2)
    ke = 0.5 * (mass * (vel * vel).sum(1)).sum()
    mom = (mass[:, None] * vel).sum(0)
    ang = (mass[:, None] * np.cross(pos, vel)).sum(0)
    c0 = (mass[species == 0, None] * pos[species == 0]).sum(0) / mass[species == 0].sum()
    c1 = (mass[species == 1, None] * pos[species == 1]).sum(0) / mass[species == 1].sum()
    assert d["kinetic"] == pytest.approx(ke, rel=1e-12)
    assert np.allclose([d["px"], d["py"], d["pz"]], mom, rtol=1e-12, atol=1e-14)
    assert np.allclose([d["lx"], d["ly"], d["lz"]], ang, rtol=1e-12, atol=1e-14)
    assert np.allclose([d["com0_x"], d["com0_y"], d["com0_z"]], c0, rtol=1e-12, atol=1e-13)
    assert d["sep"] == pytest.approx(np.linalg.norm(c0 - c1), rel=1e-12)
    _, pot = oracle.direct(pos, mass, eps=0.0, with_pot=True)
    pe = 0.5 * (mass * pot).sum()                            # sum_{i<j} -G m_i m_j / r
    assert d["potential"] == pytest.approx(pe, rel=1e-5)     # p = 8 FMM vs exact pair sum
    assert d["total"] == pytest.approx(d["kinetic"] + d["potential"], rel=1e-14)
    assert np.array_equal(frame, pos.astype(np.float32))


@pytest.mark.gpu
def test_merger_driver_writes_the_reference_formats(tmp_path):
    n_per, steps, stride = 3000, 20, 5
    r = _run_sim("--N", n_per, "--steps", steps, "--stride", stride, "--p", 6, "--thr", 32, "--eps", 0.05,
                 "--out", tmp_path / "m", cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "SEPARATION GATE" in r.stdout
    n, nframes = 2 * n_per, steps // stride + 1
    raw = (tmp_path / "m_frames.bin").read_bytes()
    assert np.frombuffer(raw[:8], np.int32).tolist() == [n, nframes]
    assert len(raw) == 8 + nframes * n * 12
    frames = np.frombuffer(raw[8:], np.float32).reshape(nframes, n, 3)
    species = np.frombuffer((tmp_path / "m_species.bin").read_bytes(), np.int8)
    assert species.shape == (n,) and (species[:n_per] == 0).all() and (species[n_per:] == 1).all()
    sep = np.loadtxt(tmp_path / "m_sep.csv", delimiter=",", skiprows=1)
    assert sep[:, 0].tolist() == [0, 5, 10, 15, 20]
    # centre-of-mass separation recomputed from the float32 frames agrees with sep.csv
    nd, nb = n_per - round(0.2 * n_per), round(0.2 * n_per)
    w = np.concatenate([np.full(nd, 1.0 / nd), np.full(nb, 0.25 / nb)] * 2)
    for row, f in zip(sep, frames):
        f = f.astype(np.float64)
        c0 = (w[species == 0, None] * f[species == 0]).sum(0) / w[species == 0].sum()
        c1 = (w[species == 1, None] * f[species == 1]).sum(0) / w[species == 1].sum()
        assert row[2] == pytest.approx(np.linalg.norm(c0 - c1), rel=1e-5)
    assert 9.0 < sep[0, 2] < 10.5 and sep[-1, 2] < sep[0, 2]   # galaxies at +-5 approaching
    en = np.loadtxt(tmp_path / "m_energy.csv", delimiter=",", skiprows=1)
    assert en.shape[0] == steps + 1 and np.abs(en[:, 3]).max() < 1e-2
