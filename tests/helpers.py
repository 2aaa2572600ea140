"""Comparison helpers shared by the test files."""
import numpy as np

from oracle_lib import LISTS


def canonical_from_arrays(d, prefix):
    """Canonical tree (box key -> (leaf, pcount); list name -> set of key pairs) from fixture arrays."""
    keys = [tuple(int(v) for v in r) for r in d[f"{prefix}_keys"]]
    info = d[f"{prefix}_info"]
    out = {"boxes": {keys[i]: (int(info[i, 0]), int(info[i, 1])) for i in range(len(keys))}}
    for name in LISTS:
        pairs = d[f"{prefix}_{name}"]
        out[name] = {(keys[a], keys[b]) for a, b in pairs}
    return out


def canonical_from_tree(t):
    b = t["boxes"]
    keys = [tuple(int(v) for v in r[:4]) for r in b]
    out = {"boxes": {keys[i]: (int(b[i, 5]), int(b[i, 7])) for i in range(len(keys))}}
    for name in LISTS:
        off, idx = t["lists"][name]
        s = set()
        for i in range(len(keys)):
            for e in range(off[i], off[i + 1]):
                s.add((keys[i], keys[idx[e]]))
        out[name] = s
    return out


def assert_same_tree(a, b, what=""):
    assert a["boxes"] == b["boxes"], f"{what}: box sets differ ({len(a['boxes'])} vs {len(b['boxes'])})"
    for name in LISTS:
        assert a[name] == b[name], (f"{what}: list {name} differs: {len(a[name] - b[name])} extra, "
                                    f"{len(b[name] - a[name])} missing")


def rel_err(ref, got):
    """max_rel / rms_rel of src3d/adaptive_tests.cpp:40-50."""
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    a = np.linalg.norm(ref, axis=1)
    fl = 1e-30 + 1e-6 * (a.max() if a.size else 0.0)
    e = np.linalg.norm(got - ref, axis=1)
    mx = float(np.max(e / np.maximum(a, fl))) if a.size else 0.0
    den = float(np.sum(a * a))
    return mx, (float(np.sqrt(np.sum(e * e) / den)) if den > 0 else 0.0)
