"""ctypes bindings for the CPU parity checker (oracle/).

Test infrastructure: imported only by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``.  Two libraries are bound:

* ``oracle/libogx_oracle.so`` -- the C restatement of the reference path
  (always built by ``oracle/Makefile``);
* ``oracle/_ref/libogx_ref.so`` -- the reference's own ``src3d`` headers
  wrapped in C entry points (built only where the reference sources exist;
  it travels with the repository snapshot as a built file).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libogx_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libogx_ref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")

LISTS = ("colleague", "U", "V", "W", "X")


def _c(a, dt=np.float64):
    return np.ascontiguousarray(a, dtype=dt)


class _TreeLib:
    """Shared tree-export protocol of both libraries (prefix orc_ / ref_)."""

    def __init__(self, lib, prefix):
        self.lib, self.pre = lib, prefix
        f = lambda n: getattr(lib, prefix + n)  # noqa: E731
        f("tree_create").restype = C.c_void_p
        f("tree_create").argtypes = [C.c_long, _dp, C.c_int, C.c_double]
        f("tree_destroy").argtypes = [C.c_void_p]
        f("tree_sizes").argtypes = [C.c_void_p, _lp]
        f("tree_boxes").argtypes = [C.c_void_p, _ip, _dp, _ip]
        f("tree_list").argtypes = [C.c_void_p, C.c_int, _lp, _ip]

    def tree(self, pos, thr, eps_floor=0.0):
        """Return dict(boxes[nb,8] int, centers[nb,4], perm[n], lists{name: (off, idx)})."""
        pos = _c(pos)
        n = pos.shape[0]
        f = lambda name: getattr(self.lib, self.pre + name)  # noqa: E731
        h = f("tree_create")(n, pos.reshape(-1), int(thr), float(eps_floor))
        try:
            sizes = np.zeros(7, np.int64)
            f("tree_sizes")(h, sizes)
            nb = int(sizes[0])
            boxes = np.zeros((nb, 8), np.int32)
            centers = np.zeros((nb, 4), np.float64)
            perm = np.zeros(max(n, 1), np.int32)
            f("tree_boxes")(h, boxes.reshape(-1), centers.reshape(-1), perm)
            lists = {}
            for k, name in enumerate(LISTS):
                off = np.zeros(nb + 1, np.int64)
                idx = np.zeros(max(int(sizes[2 + k]), 1), np.int32)
                f("tree_list")(h, k, off, idx)
                lists[name] = (off, idx[: int(sizes[2 + k])])
            return dict(boxes=boxes, centers=centers, perm=perm[:n], lists=lists, nleaf=int(sizes[1]))
        finally:
            f("tree_destroy")(h)


class Oracle(_TreeLib):
    def __init__(self, path=ORACLE_SO):
        lib = C.CDLL(path)
        super().__init__(lib, "orc_")
        lib.orc_direct.argtypes = [C.c_long, _dp, _dp, C.c_double, C.c_double, _dp, C.c_void_p]
        lib.orc_direct_targets.argtypes = [C.c_long, _dp, _dp, C.c_double, C.c_double, C.c_long, _lp, _dp, C.c_void_p]
        lib.orc_adaptive_fmm.argtypes = [C.c_long, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_int, _dp, C.c_void_p]
        lib.orc_op_p2m.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp, _dp]
        lib.orc_op_p2l.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp, _dp]
        lib.orc_op_translate.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        lib.orc_op_eval.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _dp]
        lib.orc_op_harmonics.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, _dp]
        lib.orc_rel_err.argtypes = [C.c_long, _dp, _dp, _dp]

    def direct(self, pos, mass, G=1.0, eps=0.0, with_pot=True):
        pos, mass = _c(pos), _c(mass)
        n = mass.shape[0]
        acc = np.zeros((n, 3))
        pot = np.zeros(n) if with_pot else None
        self.lib.orc_direct(n, pos.reshape(-1), mass, G, eps, acc.reshape(-1),
                            pot.ctypes.data_as(C.c_void_p) if with_pot else None)
        return (acc, pot) if with_pot else acc

    def direct_targets(self, pos, mass, targets, G=1.0, eps=0.0):
        pos, mass = _c(pos), _c(mass)
        t = _c(targets, np.int64)
        acc = np.zeros((t.shape[0], 3))
        pot = np.zeros(t.shape[0])
        self.lib.orc_direct_targets(mass.shape[0], pos.reshape(-1), mass, G, eps, t.shape[0], t,
                                    acc.reshape(-1), pot.ctypes.data_as(C.c_void_p))
        return acc, pot

    def adaptive_fmm(self, pos, mass, G=1.0, eps=0.0, p=8, thr=64, with_pot=True):
        pos, mass = _c(pos), _c(mass)
        n = mass.shape[0]
        acc = np.zeros((n, 3))
        pot = np.zeros(max(n, 1))
        rc = self.lib.orc_adaptive_fmm(n, pos.reshape(-1), mass, G, eps, p, thr, acc.reshape(-1),
                                       pot.ctypes.data_as(C.c_void_p) if with_pot else None)
        if rc:
            raise ValueError(f"orc_adaptive_fmm rc={rc}")
        return (acc, pot[:n]) if with_pot else acc

    # --- single operators (complex coefficient arrays, (p+1)^2 entries) ---
    def p2m(self, p, c, pos, q):
        pos, q = _c(pos), _c(q)
        out = np.zeros(2 * (p + 1) ** 2)
        self.lib.orc_op_p2m(p, _c(c), q.shape[0], pos.reshape(-1), q, out)
        return out.view(np.complex128)

    def p2l(self, p, c, pos, q):
        pos, q = _c(pos), _c(q)
        out = np.zeros(2 * (p + 1) ** 2)
        self.lib.orc_op_p2l(p, _c(c), q.shape[0], pos.reshape(-1), q, out)
        return out.view(np.complex128)

    def translate(self, kind, p, c_from, c_to, coef):
        out = np.zeros(2 * (p + 1) ** 2)
        self.lib.orc_op_translate(kind, p, _c(c_from), _c(c_to), _c(np.asarray(coef, np.complex128).view(np.float64)), out)
        return out.view(np.complex128)

    def evaluate(self, kind, p, c, coef, tpos):
        tpos = _c(tpos)
        out = np.zeros((tpos.shape[0], 4))
        self.lib.orc_op_eval(kind, p, _c(c), _c(np.asarray(coef, np.complex128).view(np.float64)),
                             tpos.shape[0], tpos.reshape(-1), out.reshape(-1))
        return out[:, 0], out[:, 1:]

    def harmonics(self, v, L):
        out = np.zeros(2 * (L + 1) ** 2)
        self.lib.orc_op_harmonics(float(v[0]), float(v[1]), float(v[2]), L, out)
        return out.view(np.complex128)

    def rel_err(self, ref, got):
        out = np.zeros(2)
        self.lib.orc_rel_err(ref.shape[0], _c(ref).reshape(-1), _c(got).reshape(-1), out)
        return float(out[0]), float(out[1])


class Reference(_TreeLib):
    """The reference's own CPU code (src3d headers), wrapped."""

    def __init__(self, path=REF_SO):
        lib = C.CDLL(path)
        super().__init__(lib, "ref_")
        lib.ref_direct.argtypes = [C.c_long, _dp, _dp, C.c_double, C.c_double, _dp]
        lib.ref_adaptive_fmm.argtypes = [C.c_long, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_int, _dp, C.c_void_p]
        lib.ref_adaptive_fmm_batch.argtypes = [C.c_int, C.c_long, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_int,
                                               C.c_int, _dp]
        lib.ref_plummer.argtypes = [C.c_long, C.c_uint, C.c_double, _dp, _dp, _dp]
        lib.ref_uniform_cube.argtypes = [C.c_long, C.c_uint, _dp, _dp]
        lib.ref_disk.argtypes = [C.c_long, C.c_uint, _dp, _dp]
        lib.ref_test_points.argtypes = [C.c_int, _dp, C.c_double, C.c_double, C.c_int, C.c_uint, _dp, C.c_void_p]
        lib.ref_harmonics.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, _dp]
        lib.ref_p2m.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp, _dp]
        lib.ref_translate.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        lib.ref_eval.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _dp]

    def direct(self, pos, mass, G=1.0, eps=0.0):
        pos, mass = _c(pos), _c(mass)
        acc = np.zeros((mass.shape[0], 3))
        self.lib.ref_direct(mass.shape[0], pos.reshape(-1), mass, G, eps, acc.reshape(-1))
        return acc

    def adaptive_fmm(self, pos, mass, G=1.0, eps=0.0, p=8, thr=64):
        pos, mass = _c(pos), _c(mass)
        acc = np.zeros((mass.shape[0], 3))
        st = np.zeros(2, np.int32)
        self.lib.ref_adaptive_fmm(mass.shape[0], pos.reshape(-1), mass, G, eps, p, thr, acc.reshape(-1),
                                  st.ctypes.data_as(C.c_void_p))
        return acc

    def adaptive_fmm_batch(self, pos_stack, mass_stack, G, eps, p, thr, threads):
        pos_stack, mass_stack = _c(pos_stack), _c(mass_stack)
        nsys, n = mass_stack.shape
        acc = np.zeros((nsys, n, 3))
        self.lib.ref_adaptive_fmm_batch(nsys, n, pos_stack.reshape(-1), mass_stack.reshape(-1), G, eps, p, thr,
                                        threads, acc.reshape(-1))
        return acc

    def plummer(self, n, seed, a=1.0):
        pos, vel, mass = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
        self.lib.ref_plummer(n, seed, a, pos.reshape(-1), vel.reshape(-1), mass)
        return pos, vel, mass

    def uniform_cube(self, n, seed):
        pos, mass = np.zeros((n, 3)), np.zeros(n)
        self.lib.ref_uniform_cube(n, seed, pos.reshape(-1), mass)
        return pos, mass

    def disk(self, n, seed):
        pos, mass = np.zeros((n, 3)), np.zeros(n)
        self.lib.ref_disk(n, seed, pos.reshape(-1), mass)
        return pos, mass

    def test_points(self, kind, c, rad, rad2, n, seed):
        pos, q = np.zeros((n, 3)), np.zeros(n)
        self.lib.ref_test_points(kind, _c(c), rad, rad2, n, seed, pos.reshape(-1), q.ctypes.data_as(C.c_void_p))
        return pos, q

    def harmonics(self, v, L):
        out = np.zeros(2 * (L + 1) ** 2)
        self.lib.ref_harmonics(float(v[0]), float(v[1]), float(v[2]), L, out)
        return out.view(np.complex128)

    def p2m(self, p, c, pos, q):
        pos, q = _c(pos), _c(q)
        out = np.zeros(2 * (p + 1) ** 2)
        self.lib.ref_p2m(p, _c(c), q.shape[0], pos.reshape(-1), q, out)
        return out.view(np.complex128)

    def translate(self, kind, p, c_from, c_to, coef):
        out = np.zeros(2 * (p + 1) ** 2)
        self.lib.ref_translate(kind, p, _c(c_from), _c(c_to), _c(np.asarray(coef, np.complex128).view(np.float64)), out)
        return out.view(np.complex128)

    def evaluate(self, kind, p, c, coef, tpos):
        tpos = _c(tpos)
        out = np.zeros((tpos.shape[0], 4))
        self.lib.ref_eval(kind, p, _c(c), _c(np.asarray(coef, np.complex128).view(np.float64)), tpos.shape[0],
                          tpos.reshape(-1), out.reshape(-1))
        return out[:, 0], out[:, 1:]


def canonical_tree(t):
    """Box numbering-independent view: key (level, ix, iy, iz) per box, and
    every list as a set of (target key, member key) pairs."""
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


def rel_err(ref, got):
    """max_rel / rms_rel of src3d/adaptive_tests.cpp:40-50."""
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    a = np.linalg.norm(ref, axis=1)
    fl = 1e-30 + 1e-6 * (a.max() if a.size else 0.0)
    e = np.linalg.norm(got - ref, axis=1)
    mx = float(np.max(e / np.maximum(a, fl))) if a.size else 0.0
    den = float(np.sum(a * a))
    rms = float(np.sqrt(np.sum(e * e) / den)) if den > 0 else 0.0
    return mx, rms
