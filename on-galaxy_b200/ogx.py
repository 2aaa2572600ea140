"""Python host binding of libogx.so (the C ABI in include/ogx.h).

Mirrors the reference's solver interface (src3d/ForceSolver3D.hpp:20-28):

    AdaptiveFMM3D(KernelParams3D{G, eps}, p, threshold)   -> AdaptiveFMM3D(G, eps, p, threshold)
    DirectSolver3D(KernelParams3D{G, eps})                 -> DirectSolver3D(G, eps)
    solver.computeAccelerations(bodies)                     -> solver.compute_accelerations(pos, mass)
    solver.name()                                           -> solver.name()

with numpy (n, 3) float64 positions in the original body order, exactly the
memory of a ``std::vector<Vec3>``.  Every call goes through the compiled CUDA
library; there is no CPU path here: if libogx.so is missing or the call fails,
an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libogx.so")

OK, ERR_INVALID, ERR_CUDA, ERR_NO_DEVICE, ERR_OOM, ERR_UNSUPPORTED, ERR_TIMEOUT, ERR_STATE = range(8)
SOLVER_ADAPTIVE_FMM, SOLVER_DIRECT = 0, 1
PREC_FP64, PREC_MIXED, PREC_FP64_ROT = 0, 1, 2
SOFT_PLUMMER, SOFT_SPLINE = 0, 1

# Every entry point declared in include/ogx.h (checked by the ABI test).
EXPORTS = (
    "ogx_params_default", "ogx_create", "ogx_destroy", "ogx_eval", "ogx_eval_device", "ogx_synchronize",
    "ogx_name", "ogx_last_stats", "ogx_strerror", "ogx_last_error_message", "ogx_operator_matrix",
    "ogx_upload", "ogx_step", "ogx_download", "ogx_tree_sizes", "ogx_tree_boxes", "ogx_tree_list",
    "ogx_direct_eval_noalloc", "ogx_merger_params_default", "ogx_ic_merger", "ogx_set_species",
    "ogx_diagnostics", "ogx_download_frame", "ogx_check_bounded_wait", "ogx_set_tuning", "ogx_get_tuning",
    "ogx_ensemble_create", "ogx_ensemble_step", "ogx_ensemble_stats", "ogx_ensemble_destroy",
)


class Params(C.Structure):
    _fields_ = [("G", C.c_double), ("eps", C.c_double), ("p", C.c_int), ("leaf_capacity", C.c_int),
                ("solver", C.c_int), ("precision", C.c_int), ("device", C.c_int), ("stream", C.c_void_p),
                ("softening", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("n", C.c_int64), ("num_boxes", C.c_int32), ("num_leaves", C.c_int32),
                ("max_leaf_occupancy", C.c_int32), ("max_level", C.c_int32),
                ("list_u", C.c_int64), ("list_v", C.c_int64), ("list_w", C.c_int64), ("list_x", C.c_int64),
                ("p2p_pairs", C.c_int64), ("m2p_evals", C.c_int64), ("p2l_evals", C.c_int64),
                ("adjacency_mismatch", C.c_int64),
                ("ms_tree", C.c_double), ("ms_lists", C.c_double), ("ms_upward", C.c_double), ("ms_m2l", C.c_double),
                ("ms_p2l", C.c_double), ("ms_downward", C.c_double), ("ms_leaf", C.c_double), ("ms_total", C.c_double),
                ("ms_h2d", C.c_double), ("ms_d2h", C.c_double), ("launches", C.c_int64),
                ("graph_steps", C.c_int64), ("step_redos", C.c_int64), ("list_s", C.c_int64),
                ("graph_evals", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [("m2l_tile_targets", C.c_int), ("near_units", C.c_int), ("capture_steps", C.c_int)]


class MergerParams(C.Structure):
    _fields_ = [("n_per", C.c_int64), ("seed", C.c_uint64), ("sep", C.c_double), ("vrel", C.c_double),
                ("tilt_deg", C.c_double), ("disp_frac", C.c_double), ("Rd", C.c_double), ("z0", C.c_double),
                ("Md", C.c_double), ("ab", C.c_double), ("Mb", C.c_double), ("bulge_frac", C.c_double)]


DIAG_FIELDS = ("kinetic", "potential", "total", "px", "py", "pz", "lx", "ly", "lz",
               "com0_x", "com0_y", "com0_z", "com1_x", "com1_y", "com1_z", "sep")


class OgxError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        lib = load()
        msg = lib.ogx_strerror(code).decode()
        detail = lib.ogx_last_error_message().decode()
        super().__init__(f"{what}: {msg} ({code}) {detail}".strip())


_lib = None


def load(path: str = LIB_PATH):
    """Load libogx.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built (run `make -C on-galaxy_b200`)")
    lib = C.CDLL(path)
    vp, i64, dp, ip = C.c_void_p, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    lib.ogx_params_default.argtypes = [C.POINTER(Params)]
    lib.ogx_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
    lib.ogx_destroy.argtypes = [vp]
    lib.ogx_eval.argtypes = [vp, i64, vp, vp, vp, vp]
    lib.ogx_eval_device.argtypes = [vp, i64, vp, vp, vp, vp]
    lib.ogx_synchronize.argtypes = [vp]
    lib.ogx_name.argtypes = [vp]
    lib.ogx_name.restype = C.c_char_p
    lib.ogx_last_stats.argtypes = [vp, C.POINTER(Stats)]
    lib.ogx_strerror.argtypes = [C.c_int]
    lib.ogx_strerror.restype = C.c_char_p
    lib.ogx_last_error_message.argtypes = []
    lib.ogx_last_error_message.restype = C.c_char_p
    lib.ogx_operator_matrix.argtypes = [C.c_int, C.c_int, C.c_int, dp]
    lib.ogx_upload.argtypes = [vp, i64, vp, vp, vp]
    lib.ogx_step.argtypes = [vp, C.c_double, C.c_int]
    lib.ogx_download.argtypes = [vp, vp, vp, vp]
    lib.ogx_tree_sizes.argtypes = [vp, C.POINTER(C.c_int64)]
    lib.ogx_tree_boxes.argtypes = [vp, ip, dp, ip]
    lib.ogx_tree_list.argtypes = [vp, C.c_int, C.POINTER(C.c_int64), ip]
    lib.ogx_direct_eval_noalloc.argtypes = [i64, vp, vp, C.c_double, C.c_double, vp, vp, vp]
    lib.ogx_merger_params_default.argtypes = [C.POINTER(MergerParams)]
    lib.ogx_ic_merger.argtypes = [vp, C.POINTER(MergerParams), vp]
    lib.ogx_set_species.argtypes = [vp, vp]
    lib.ogx_diagnostics.argtypes = [vp, dp]
    lib.ogx_download_frame.argtypes = [vp, vp]
    lib.ogx_check_bounded_wait.argtypes = [vp, C.c_uint32]
    lib.ogx_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
    lib.ogx_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
    _lib = lib
    return lib


def _check(rc, what):
    if rc != OK:
        raise OgxError(rc, what)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def operator_matrix(kind: int, p: int, index: int) -> np.ndarray:
    """Host-side translation matrix (kind 0=M2M, 1=L2L, 2=M2L), K x K with K=(p+1)^2."""
    K = (p + 1) ** 2
    out = np.zeros(K * K)
    _check(load().ogx_operator_matrix(kind, p, index, out.ctypes.data_as(C.POINTER(C.c_double))),
           "ogx_operator_matrix")
    return out.reshape(K, K)


NOALLOC_MAX_BODIES = 65536


def direct_eval_noalloc(pos, mass, G=1.0, eps=0.0, with_pot=False, stream=None):
    """FP64 direct sum through ogx_direct_eval_noalloc: no device allocation, at most
    NOALLOC_MAX_BODIES bodies, host arrays in and out (see include/ogx.h)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    n = mass.shape[0]
    acc = np.zeros((n, 3))
    pot = np.zeros(n) if with_pot else None
    _check(load().ogx_direct_eval_noalloc(n, _ptr(pos), _ptr(mass), float(G), float(eps), _ptr(acc), _ptr(pot),
                                          stream), "ogx_direct_eval_noalloc")
    return (acc, pot) if with_pot else acc


class _Solver:
    def __init__(self, G=1.0, eps=0.0, p=8, threshold=64, solver=SOLVER_ADAPTIVE_FMM, precision=PREC_FP64,
                 device=0, stream=None, softening=SOFT_PLUMMER):
        lib = load()
        prm = Params()
        lib.ogx_params_default(C.byref(prm))
        prm.G, prm.eps, prm.p, prm.leaf_capacity = float(G), float(eps), int(p), int(threshold)
        prm.solver, prm.precision, prm.device = int(solver), int(precision), int(device)
        prm.stream = stream
        prm.softening = int(softening)
        h = C.c_void_p()
        _check(lib.ogx_create(C.byref(prm), C.byref(h)), "ogx_create")
        self._h = h
        self._lib = lib
        self.params = prm

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ogx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def name(self) -> str:
        return self._lib.ogx_name(self._h).decode()

    def compute_accelerations(self, pos, mass, with_potential=False):
        """ForceSolver3D::computeAccelerations on host arrays -> acc (n,3) [, pot (n,)]."""
        pos = np.ascontiguousarray(pos, np.float64)
        mass = np.ascontiguousarray(mass, np.float64)
        n = mass.shape[0]
        if pos.shape != (n, 3):
            raise ValueError("pos must be (n, 3)")
        acc = np.zeros((n, 3))
        pot = np.zeros(n) if with_potential else None
        _check(self._lib.ogx_eval(self._h, n, _ptr(pos), _ptr(mass), _ptr(acc), _ptr(pot)), "ogx_eval")
        return (acc, pot) if with_potential else acc

    # torch-tensor (device) path: plumbing only, the tensors are plain device buffers
    def compute_accelerations_device(self, pos_t, mass_t, acc_t, pot_t=None):
        n = mass_t.shape[0]
        _check(self._lib.ogx_eval_device(self._h, n, C.c_void_p(pos_t.data_ptr()), C.c_void_p(mass_t.data_ptr()),
                                         C.c_void_p(acc_t.data_ptr()),
                                         None if pot_t is None else C.c_void_p(pot_t.data_ptr())),
               "ogx_eval_device")

    def compute_accelerations_host_ptr(self, n, pos_p, mass_p, acc_p, pot_p=None):
        """Host-buffer call on raw pointers (pinned buffers from torch)."""
        _check(self._lib.ogx_eval(self._h, n, C.c_void_p(pos_p), C.c_void_p(mass_p), C.c_void_p(acc_p),
                                  None if pot_p is None else C.c_void_p(pot_p)), "ogx_eval")

    def synchronize(self):
        _check(self._lib.ogx_synchronize(self._h), "ogx_synchronize")

    def set_tuning(self, m2l_tile_targets=0, near_units=0, capture_steps=None):
        """Launch-shape knobs (0 keeps a size's default) and step capture (None keeps the
        current setting); see ogx_set_tuning."""
        if capture_steps is None:
            capture_steps = self.tuning()["capture_steps"]
        t = Tuning(int(m2l_tile_targets), int(near_units), int(bool(capture_steps)))
        _check(self._lib.ogx_set_tuning(self._h, C.byref(t)), "ogx_set_tuning")

    def tuning(self) -> dict:
        t = Tuning()
        _check(self._lib.ogx_get_tuning(self._h, C.byref(t)), "ogx_get_tuning")
        return {"m2l_tile_targets": t.m2l_tile_targets, "near_units": t.near_units, "capture_steps": t.capture_steps}

    def check_bounded_wait(self, polls=1000):
        """Run the pipeline's bounded device wait on a barrier nothing arrives on; raises
        OgxError(ERR_TIMEOUT) as an evaluation whose wait ran out would."""
        _check(self._lib.ogx_check_bounded_wait(self._h, int(polls)), "ogx_check_bounded_wait")

    def stats(self) -> dict:
        s = Stats()
        _check(self._lib.ogx_last_stats(self._h, C.byref(s)), "ogx_last_stats")
        return s.as_dict()

    # device-resident leapfrog (VelocityVerlet3D)
    def upload(self, pos, vel, mass):
        pos = np.ascontiguousarray(pos, np.float64)
        vel = np.ascontiguousarray(vel, np.float64)
        mass = np.ascontiguousarray(mass, np.float64)
        _check(self._lib.ogx_upload(self._h, mass.shape[0], _ptr(pos), _ptr(vel), _ptr(mass)), "ogx_upload")
        self._n = mass.shape[0]

    def step(self, dt, nsteps=1):
        _check(self._lib.ogx_step(self._h, float(dt), int(nsteps)), "ogx_step")

    def download(self):
        n = self._n
        pos, vel, acc = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        _check(self._lib.ogx_download(self._h, _ptr(pos), _ptr(vel), _ptr(acc)), "ogx_download")
        return pos, vel, acc

    # running a simulation on the device
    def ic_merger(self, n_per, seed=1, **kw):
        """Generate the two-galaxy merger on the device into the resident state; returns species (galaxy tags)."""
        mp = MergerParams()
        _check(self._lib.ogx_merger_params_default(C.byref(mp)), "ogx_merger_params_default")
        mp.n_per, mp.seed = int(n_per), int(seed)
        for k, v in kw.items():
            setattr(mp, k, v)
        species = np.zeros(2 * int(n_per), np.int8)
        _check(self._lib.ogx_ic_merger(self._h, C.byref(mp), _ptr(species)), "ogx_ic_merger")
        self._n = species.shape[0]
        return species

    def set_species(self, species):
        species = np.ascontiguousarray(species, np.int8)
        _check(self._lib.ogx_set_species(self._h, _ptr(species)), "ogx_set_species")

    def diagnostics(self) -> dict:
        out = np.zeros(len(DIAG_FIELDS))
        _check(self._lib.ogx_diagnostics(self._h, out.ctypes.data_as(C.POINTER(C.c_double))), "ogx_diagnostics")
        return dict(zip(DIAG_FIELDS, out.tolist()))

    def download_frame(self):
        frame = np.zeros((self._n, 3), np.float32)
        _check(self._lib.ogx_download_frame(self._h, _ptr(frame)), "ogx_download_frame")
        return frame

    def tree(self):
        """Tree of the last evaluation in the same layout as the oracle export."""
        lib = self._lib
        sizes = (C.c_int64 * 7)()
        _check(lib.ogx_tree_sizes(self._h, sizes), "ogx_tree_sizes")
        nb = int(sizes[0])
        boxes = np.zeros((nb, 8), np.int32)
        centers = np.zeros((nb, 4))
        n = self.stats()["n"]
        perm = np.zeros(max(n, 1), np.int32)
        _check(lib.ogx_tree_boxes(self._h, boxes.ctypes.data_as(C.POINTER(C.c_int32)),
                                  centers.ctypes.data_as(C.POINTER(C.c_double)),
                                  perm.ctypes.data_as(C.POINTER(C.c_int32))), "ogx_tree_boxes")
        lists = {}
        for k, name in enumerate(("colleague", "U", "V", "W", "X")):
            off = np.zeros(nb + 1, np.int64)
            idx = np.zeros(max(int(sizes[2 + k]), 1), np.int32)
            _check(lib.ogx_tree_list(self._h, k, off.ctypes.data_as(C.POINTER(C.c_int64)),
                                     idx.ctypes.data_as(C.POINTER(C.c_int32))), "ogx_tree_list")
            lists[name] = (off, idx[: int(sizes[2 + k])])
        return dict(boxes=boxes, centers=centers, perm=perm[:n], lists=lists, nleaf=int(sizes[1]))


class AdaptiveFMM3D(_Solver):
    """Drop-in for galaxy3d::AdaptiveFMM3D(KernelParams3D{G, eps}, p, threshold)."""

    def __init__(self, G=1.0, eps=0.0, p=8, threshold=64, precision=PREC_FP64, device=0, stream=None,
                 softening=SOFT_PLUMMER):
        super().__init__(G, eps, p, threshold, SOLVER_ADAPTIVE_FMM, precision, device, stream, softening)


class DirectSolver3D(_Solver):
    """Drop-in for galaxy3d::DirectSolver3D(KernelParams3D{G, eps})."""

    def __init__(self, G=1.0, eps=0.0, device=0, stream=None, softening=SOFT_PLUMMER):
        super().__init__(G, eps, 8, 64, SOLVER_DIRECT, PREC_FP64, device, stream, softening)
