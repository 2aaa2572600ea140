"""Generate the golden fixtures in this directory from the REFERENCE itself.

Runs the reference's own CPU code (src3d headers, wrapped by
oracle/ref_wrapper.cpp into oracle/_ref/libogx_ref.so) on seeded inputs and
stores inputs + outputs as .npz files:

  plummer2000_s2.npz   makePlummerSphere(N=2000, seed 2) (Gate B input of
                       adaptive_tests.cpp:111): DirectSolver3D, AdaptiveFMM3D
                       p=4/8 thr=64, trees thr=64 and thr=8
  cube1000_s1.npz      makeUniformCube(1000, seed 1) (adaptive_tests.cpp:27-33):
                       DirectSolver3D, AdaptiveFMM3D p=8 thr=64/16, trees
  clump.npz            uniform cube + a 80-body clump inside a 1e-7 cube
                       (deep tree near the 24-level cap): direct, AdaptiveFMM3D
                       p=4 thr=16, tree thr=16
  coincident.npz       100 random bodies + 20 exact copies of one point: tree
                       thr=4 at eps=0 (depth cap) and AdaptiveFMM3D p=4 at
                       eps=0.01 (eps floor), direct at eps=0.01
  disk4000.npz         makeDisk(N=4000, seed 1) (GalaxyIC.hpp:43): AdaptiveFMM3D
                       p=6 thr=32 + tree
  small.npz            N = 1, 2, 64, 65 (thr=64) trees and forces
  cfg1_plummer16384.npz Plummer N=16384 seed 1 truncated at 20a (the FP64
                       parity configuration): AdaptiveFMM3D p=8 thr=64 and
                       DirectSolver3D
  operators.npz        the seeded point sets of fmm3d_tests.cpp (P2M/M2L/M2M/L2L
                       gates) and the published convergence table
                       outputs/fmm3d_operator_convergence.csv

Usage (needs a checkout of the reference, found through the environment variable
OGX_REFERENCE_DIR or else as a directory named `reference` beside this repository,
and `make -C oracle`):
    OGX_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py
"""
from __future__ import annotations

import csv
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "on-galaxy_b200"))

from oracle_lib import LISTS, Reference  # noqa: E402

import ogx_ic  # noqa: E402

REF_DIR = os.environ.get("OGX_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
REF_CSV = os.path.join(REF_DIR, "outputs", "fmm3d_operator_convergence.csv")


def tree_arrays(t, prefix):
    """Canonical arrays: box keys (level, ix, iy, iz), (leaf, pcount), list pairs as key indices."""
    b = t["boxes"]
    keys = b[:, :4].astype(np.int32)
    out = {f"{prefix}_keys": keys, f"{prefix}_info": np.stack([b[:, 5], b[:, 7]], 1).astype(np.int32)}
    for name in LISTS:
        off, idx = t["lists"][name]
        src = np.repeat(np.arange(len(keys)), np.diff(off))
        out[f"{prefix}_{name}"] = np.stack([src, idx], 1).astype(np.int32)
    return out


def main():
    ref = Reference()
    out_files = {}

    pos, vel, m = ref.plummer(2000, 2)
    d = dict(pos=pos, mass=m, direct=ref.direct(pos, m))
    for p in (4, 8):
        d[f"fmm_p{p}"] = ref.adaptive_fmm(pos, m, p=p, thr=64)
    d.update(tree_arrays(ref.tree(pos, 64), "t64"))
    d.update(tree_arrays(ref.tree(pos, 8), "t8"))
    out_files["plummer2000_s2"] = d

    pos, m = ref.uniform_cube(1000, 1)
    d = dict(pos=pos, mass=m, direct=ref.direct(pos, m), fmm_p8_t64=ref.adaptive_fmm(pos, m, p=8, thr=64),
             fmm_p8_t16=ref.adaptive_fmm(pos, m, p=8, thr=16))
    d.update(tree_arrays(ref.tree(pos, 64), "t64"))
    d.update(tree_arrays(ref.tree(pos, 16), "t16"))
    out_files["cube1000_s1"] = d

    rng = np.random.Generator(np.random.PCG64(7))
    base, mb = ref.uniform_cube(500, 3)
    clump = np.array([0.3, -0.2, 0.1]) + 1e-7 * rng.random((80, 3))
    pos = np.concatenate([base, clump])
    m = np.concatenate([mb, np.full(80, 0.01)])
    d = dict(pos=pos, mass=m, direct=ref.direct(pos, m), fmm_p4_t16=ref.adaptive_fmm(pos, m, p=4, thr=16))
    d.update(tree_arrays(ref.tree(pos, 16), "t16"))
    out_files["clump"] = d

    base, mb = ref.uniform_cube(100, 5)
    pos = np.concatenate([base, np.tile(np.array([[0.11, 0.22, -0.33]]), (20, 1))])
    m = np.concatenate([mb, np.full(20, 0.5)])
    d = dict(pos=pos, mass=m, direct_eps=ref.direct(pos, m, eps=0.01),
             fmm_p4_t4_eps=ref.adaptive_fmm(pos, m, eps=0.01, p=4, thr=4))
    d.update(tree_arrays(ref.tree(pos, 4, 0.0), "t4"))
    d.update(tree_arrays(ref.tree(pos, 4, 0.01), "t4eps"))
    out_files["coincident"] = d

    pos, m = ref.disk(4000, 1)
    d = dict(pos=pos, mass=m, fmm_p6_t32=ref.adaptive_fmm(pos, m, p=6, thr=32), direct=ref.direct(pos, m))
    d.update(tree_arrays(ref.tree(pos, 32), "t32"))
    out_files["disk4000"] = d

    d = {}
    for n in (1, 2, 64, 65):
        pos, m = ref.uniform_cube(n, 11 + n)
        d[f"n{n}_pos"], d[f"n{n}_mass"] = pos, m
        d[f"n{n}_fmm"] = ref.adaptive_fmm(pos, m, p=4, thr=64)
        d[f"n{n}_direct"] = ref.direct(pos, m)
        d.update(tree_arrays(ref.tree(pos, 64), f"n{n}"))
    out_files["small"] = d

    pos, vel, m = ogx_ic.plummer(16384, seed=1, rmax_a=20.0)
    out_files["cfg1_plummer16384"] = dict(pos=pos, mass=m, fmm_p8_t64=ref.adaptive_fmm(pos, m, p=8, thr=64),
                                          direct=ref.direct(pos, m))

    # operator gates of fmm3d_tests.cpp:196-288 (point sets from the same seeded generators)
    d = {}
    d["p2m_src"], d["p2m_q"] = ref.test_points(0, [0, 0, 0], 1.0, 0.0, 80, 11)
    d["p2m_tgt"], _ = ref.test_points(1, [0, 0, 0], 4.0, 8.0, 64, 99)
    for k, zl in enumerate(([6, 0, 0], [0, 6, 0], [0, 0, 6], [3.5, 3.5, 3.5])):
        d[f"m2l{k}_src"], d[f"m2l{k}_q"] = ref.test_points(0, [0, 0, 0], 0.9, 0.0, 80, 21)
        d[f"m2l{k}_tgt"], _ = ref.test_points(0, zl, 0.9, 0.0, 64, 77)
        d[f"m2l{k}_zl"] = np.array(zl, np.float64)
    d["m2m_src"], d["m2m_q"] = ref.test_points(0, [0.5, 0.4, 0.3], 0.4, 0.0, 80, 31)
    d["m2m_tgt"], _ = ref.test_points(1, [0, 0, 0], 5.0, 9.0, 64, 55)
    d["l2l_src"], d["l2l_q"] = ref.test_points(0, [-8, 3, 2], 1.0, 0.0, 80, 41)
    d["l2l_tgt"], _ = ref.test_points(0, [0.5, 0.4, 0.3], 0.4, 0.0, 64, 66)
    rows = list(csv.DictReader(open(REF_CSV)))
    d["csv_op"] = np.array([r["operator"] for r in rows])
    d["csv_qty"] = np.array([r["quantity"] for r in rows])
    d["csv_p"] = np.array([int(r["p"]) for r in rows])
    d["csv_err"] = np.array([float(r["rel_err"]) for r in rows])
    out_files["operators"] = d

    for name, arrs in out_files.items():
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **arrs)
        print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB)")


if __name__ == "__main__":
    main()
