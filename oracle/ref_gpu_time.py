"""Times the reference's own GPU adaptive FMM next to this library, on the same bodies.

MEASUREMENT INFRASTRUCTURE ONLY.  Runs oracle/_ref/ref_gpu_fmm (the reference's
galaxy3d::gpu::adaptiveFmm3dGpu, src3d/gpu/AdaptiveFMM3DGPU.cu:316-334, built by
oracle/Makefile) in FP64 and FP32 at p = 8, leaf capacity 64, on
  * the 1M-body two-galaxy merger of the benchmark (2 x 500,000 disk+bulge bodies), and
  * config 1, the 16,384-body Plummer sphere truncated at 20a (tests/golden fixture);
then this library's FP64 and mixed forms through ogx_eval (host buffers, copies
included) on the same bodies, and the RMS of the reference GPU's accelerations against
this library's FP64 form.  One JSON line per (workload, solver).

usage: python oracle/ref_gpu_time.py   (needs a GPU; prints JSON lines)
"""
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [os.path.join(ROOT, "on-galaxy_b200")]
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_fmm")


def rms(ref, got):
    a = np.linalg.norm(ref, axis=1)
    e = np.linalg.norm(got - ref, axis=1)
    return float(np.sqrt((e * e).sum() / (a * a).sum()))


def workloads():
    import ogx_ic
    pos, _, mass, _ = ogx_ic.merger(500_000, seed=1, accel_fn=None)
    yield "two-galaxy merger, 1000000 bodies", pos, mass, 2
    d = np.load(os.path.join(ROOT, "tests", "golden", "cfg1_plummer16384.npz"))
    yield "Plummer sphere, 16384 bodies (20a truncation)", d["pos"], d["mass"], 5


def main():
    import ogx
    for name, pos, mass, reps in workloads():
        n = mass.shape[0]
        with ogx.AdaptiveFMM3D(p=8, threshold=64, precision=ogx.PREC_FP64) as s:
            a64 = s.compute_accelerations(pos, mass)
        with tempfile.TemporaryDirectory() as td:
            bodies = os.path.join(td, "bodies.bin")
            with open(bodies, "wb") as f:
                np.array([n], np.int64).tofile(f)
                np.ascontiguousarray(pos, np.float64).tofile(f)
                np.ascontiguousarray(mass, np.float64).tofile(f)
            for prec in ("fp64", "fp32"):
                out = os.path.join(td, "acc.bin")
                r = subprocess.run([DRIVER, bodies, "8", "64", prec, str(reps), out], capture_output=True, text=True,
                                   timeout=1800)
                if r.returncode != 0:
                    print(json.dumps({"workload": name, "solver": f"reference GPU adaptiveFmm3dGpu<{prec}>",
                                      "failed": r.returncode, "stderr": r.stderr[-400:]}), flush=True)
                    continue
                line = json.loads(r.stdout.strip().splitlines()[-1])
                acc = np.fromfile(out, np.float64).reshape(n, 3)
                line.update({"workload": name, "solver": f"reference GPU adaptiveFmm3dGpu<{prec}>",
                             "bodies_per_s_total": n / line["total_s"],
                             "bodies_per_s_gpu_only": n / line["gpu_compute_s"],
                             "rms_vs_this_fp64_form": rms(a64, acc)})
                print(json.dumps(line), flush=True)
        for prec, pname in ((ogx.PREC_FP64, "fp64"), (ogx.PREC_MIXED, "mixed")):
            with ogx.AdaptiveFMM3D(p=8, threshold=64, precision=prec) as s:
                for _ in range(2):
                    s.compute_accelerations(pos, mass)
                best = 1e300
                for _ in range(reps):
                    t0 = time.perf_counter()
                    acc = s.compute_accelerations(pos, mass)
                    best = min(best, time.perf_counter() - t0)
                st = s.stats()
            print(json.dumps({"workload": name, "solver": f"this library, {pname} form (ogx_eval, host buffers)",
                              "n": n, "p": 8, "threshold": 64, "total_s": best, "bodies_per_s_total": n / best,
                              "device_ms": st["ms_total"], "rms_vs_this_fp64_form": rms(a64, acc)}), flush=True)


if __name__ == "__main__":
    main()
