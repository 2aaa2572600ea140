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


def canonical_rank(t):
    """Rank of every box in the order (level, ix, iy, iz): a numbering both trees share."""
    k = t["boxes"][:, :4].astype(np.int64)
    order = np.lexsort((k[:, 3], k[:, 2], k[:, 1], k[:, 0]))
    rank = np.empty(len(order), np.int64)
    rank[order] = np.arange(len(order))
    return order, rank


def assert_same_tree_arrays(a, b, what=""):
    """Vectorised form of assert_same_tree for large trees (millions of list pairs): box keys,
    leaf flags, body counts and FP64 centres (bit for bit) in the shared numbering, each of
    the five lists as a sorted array of (target, member) pairs, and the bodies of every
    leaf in their stored order."""
    oa, ra = canonical_rank(a)
    ob, rb = canonical_rank(b)
    ba, bb = a["boxes"][oa], b["boxes"][ob]
    assert ba.shape == bb.shape, f"{what}: {len(ba)} vs {len(bb)} boxes"
    np.testing.assert_array_equal(ba[:, :4], bb[:, :4], err_msg=f"{what}: box keys")
    np.testing.assert_array_equal(ba[:, 5], bb[:, 5], err_msg=f"{what}: leaf flags")
    np.testing.assert_array_equal(ba[:, 7], bb[:, 7], err_msg=f"{what}: body counts")
    np.testing.assert_array_equal(a["centers"][oa].view(np.int64), b["centers"][ob].view(np.int64),
                                  err_msg=f"{what}: box centres")
    nb = len(ba)
    for name in LISTS:
        codes = []
        for t, r in ((a, ra), (b, rb)):
            off, idx = t["lists"][name]
            src = np.repeat(np.arange(nb), np.diff(off))
            codes.append(np.sort(r[src] * nb + r[idx.astype(np.int64)]))
        assert codes[0].shape == codes[1].shape, f"{what}: list {name}: {len(codes[0])} vs {len(codes[1])} pairs"
        assert np.array_equal(codes[0], codes[1]), f"{what}: list {name} differs"

    def leaf_bodies(t, o):
        bx = t["boxes"][o]
        leaf = bx[:, 5] == 1
        starts, counts = bx[leaf, 6].astype(np.int64), bx[leaf, 7].astype(np.int64)
        pos = np.repeat(starts - np.concatenate(([0], np.cumsum(counts)[:-1])), counts) + np.arange(counts.sum())
        return t["perm"][pos]
    np.testing.assert_array_equal(leaf_bodies(a, oa), leaf_bodies(b, ob), err_msg=f"{what}: bodies of the leaves")
