"""Benchmark: adaptive-FMM force evaluation on the 1M-body two-galaxy merger.

Workload (the configuration the headline metric is quoted on): two disk+bulge
galaxies of 500,000 bodies each (80% exponential sech^2 disk, 20% Hernquist
bulge), placed at x = -/+5 with relative velocity 0.5 along x and the second
disk tilted by 30 degrees; velocities from the FP64 field (v_c^2 = -a_R R) plus
0.1 v_c dispersion; p = 8, leaf capacity 64, G = 1, eps = 0.  One step = one
device-resident leapfrog step with dt = 0.01 (drift, full force evaluation
including tree build and lists, kick), as VelocityVerlet3D::step
(src3d/Integrator3D.hpp:23-40).  Synthetic, seeded data.

value   : bodies/s = N / (device time of one step), inputs resident in HBM, L2
          flushed (256 MiB write) before every timed step, CUDA events per step.
e2e     : bodies/s through the C ABI call that replaces
          ForceSolver3D::computeAccelerations with host buffers (pinned), i.e.
          H2D pos+mass, evaluation, D2H accelerations, every step.
--impl reference : the reference's own CPU AdaptiveFMM3D (src3d headers compiled
          into oracle/_ref) on a bounded sample of the same workload, all host
          threads, one system per thread.
Multi-GPU: replicas only (one independent merger per rank, no collective on the
path); value = all ranks' bodies / max-over-ranks step time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "on-galaxy_b200")
sys.path.insert(0, PKG)

METRIC = "bodies/s, adaptive FMM 1M clustered @RMS err≤1e-5 vs FP64 form; p99 step ms"
N_PER = 500_000
P_ORDER = 8
THR = 64
DT = 0.01


# DRAM bytes per V-list pair of the tensor-core M2L launch: dram__bytes_read.sum +
# dram__bytes_write.sum of one k_m2l_tc<8> launch on the merger with 2 x 250,000 bodies
# (ncu --set full --clock-control none), (50.97 + 3.18) MB over its 3.42e6 V-list pairs.
# The bytes scale with the pairs a launch processes (sources gathered per pair, results
# per target), so the figure is applied to the measured workload's pair count.
M2L_DRAM_BYTES_PER_VPAIR = 15.82


def arm_config(n, n_per, world, eps=0.0, softening="plummer"):
    """The workload this arm is quoted on."""
    cfg = {"workload": f"two-galaxy merger, {n} bodies (2x{n_per} disk+bulge), one leapfrog step dt=0.01",
           "p": P_ORDER, "leaf_capacity": THR, "eps": eps, "parallelism": f"replicas x{world}",
           "l2": "flushed (256 MiB write) before every timed step"}
    if softening != "plummer":
        cfg["softening"] = softening
    return cfg


def reference_config(nsys, n_sys, n_per_full, world):
    """What the reference arm runs per step: a bounded sample of the merger workload, `nsys`
    independent mergers of n_sys bodies from the same generator, one per host thread (the
    reference's AdaptiveFMM3D is single-threaded and takes minutes for one full-size merger)."""
    return {"workload": f"{nsys} independent two-galaxy mergers of {n_sys} bodies each (2x{n_sys // 2} disk+bulge, "
                        f"same generator as the {2 * n_per_full}-body merger), one AdaptiveFMM3D evaluation each "
                        f"per step, one merger per host thread",
            "p": P_ORDER, "leaf_capacity": THR, "eps": 0.0, "parallelism": f"{nsys} host threads",
            "l2": "n/a (host)"}


def max_over_ranks(x, dist, device):
    """Max of a per-rank float over all ranks (the value itself without a process group).
    Works with NCCL (device "cuda") and gloo (device "cpu")."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(n_per_rank, world, ms_per_step):
    """Whole-job bodies/s of `world` independent replicas timed at the slowest rank's step."""
    return world * n_per_rank / (ms_per_step / 1e3)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "fp64rot"])
    ap.add_argument("--n-per", type=int, default=N_PER)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-capture", action="store_true", help="eager steps instead of replaying a captured CUDA graph")
    ap.add_argument("--no-serving", action="store_true", help="skip the ensemble (config 4) and serving (config 5) records")
    ap.add_argument("--eps", type=float, default=0.0, help="softening length of the timed workload (default 0)")
    ap.add_argument("--softening", default="plummer", choices=["plummer", "spline"],
                    help="softening kernel of the timed workload (spline: compact kernel, far field corrected)")
    return ap.parse_args()


# ---------------------------------------------------------------- reference arm
def cpu_sample_bodies(n_per, seed):
    import ogx_ic
    pos, _, mass, _ = ogx_ic.merger(n_per, seed=seed, accel_fn=None)
    return pos, mass


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import REF_SO, Oracle, Reference

    threads = os.cpu_count() or 1
    n_per = 4096  # 8,192-body merger per system, same generator as the workload
    kind = "reference" if os.path.exists(REF_SO) else "port"
    samples = [cpu_sample_bodies(n_per, seed=100 + s) for s in range(threads)]
    pos = np.stack([s[0] for s in samples])
    mass = np.stack([s[1] for s in samples])
    if kind == "reference":
        lib = Reference()
        run = lambda: lib.adaptive_fmm_batch(pos, mass, 1.0, 0.0, P_ORDER, THR, threads)  # noqa: E731
    else:
        orc = Oracle()
        run = lambda: [orc.adaptive_fmm(pos[s], mass[s], p=P_ORDER, thr=THR, with_pot=False)  # noqa: E731
                       for s in range(threads)]
    for _ in range(args.warmup):
        run()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    n_tot = pos.shape[0] * pos.shape[1]
    ms = 1e3 * float(np.mean(times))
    value = n_tot / (ms / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "bodies/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": reference_config(threads, pos.shape[1], args.n_per, args.gpus),
        "p50_step_ms": 1e3 * float(np.percentile(times, 50)), "p99_step_ms": 1e3 * float(np.percentile(times, 99)),
        "cpu_baseline": {"value": value, "unit": "bodies/s", "cores": threads, "kind": kind,
                         "sample": f"{threads} independent {pos.shape[1]}-body mergers per step (same generator, "
                                   f"2x{n_per} bodies each), one force evaluation of AdaptiveFMM3D p={P_ORDER} "
                                   f"thr={THR} per system, one system per host thread"},
        "e2e": {"value": value, "unit": "bodies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_single():
    """Reference CPU AdaptiveFMM3D on one core, bounded sample (16,384-body merger, one evaluation)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import REF_SO, Oracle, Reference
    pos, mass = cpu_sample_bodies(8192, seed=100)
    kind = "reference" if os.path.exists(REF_SO) else "port"
    t0 = time.perf_counter()
    if kind == "reference":
        Reference().adaptive_fmm(pos, mass, p=P_ORDER, thr=THR)
    else:
        Oracle().adaptive_fmm(pos, mass, p=P_ORDER, thr=THR, with_pot=False)
    sec = time.perf_counter() - t0
    return {"value": pos.shape[0] / sec, "unit": "bodies/s", "cores": 1, "kind": kind,
            "sample": f"one AdaptiveFMM3D evaluation of a {pos.shape[0]}-body merger (2x{pos.shape[0] // 2}, same "
                      f"generator), p={P_ORDER}, thr={THR}, {sec:.1f} s on 1 core; box has {os.cpu_count()} cores"}


# ---------------------------------------------------------------- configs 4 and 5
SERVE = os.path.join(PKG, "ogx_serve")
CONFIG4 = ["--ensemble", "--steps", "50", "--jobs", "64", "--nmin", "8192", "--nmax", "262144", "--orders", "6,8",
           "--seed", "3"]
CONFIG5 = ["--jobs", "24", "--rate", "20", "--nmin", "16384", "--nmax", "1048576", "--orders", "6,8,12", "--smin", "10",
           "--smax", "200", "--hbm-gb", "150", "--seed", "1"]


def serve_run(args, timeout=600):
    r = subprocess.run([SERVE, *args], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        return {"failed": r.returncode, "tail": (r.stdout + r.stderr)[-300:]}
    d = json.loads(r.stdout.strip().splitlines()[-1])
    d.pop("jobs_detail", None)
    return d


def serving_records():
    """Config 4 (64 resident systems, N log-uniform 8k-256k, p in {6, 8}, 50 lockstep steps)
    and config 5 (24 jobs arriving at 20/s, N 16k-1M, p in {6, 8, 12}, 10-200 steps, 150 GB
    budget) through the serving driver, mixed form: config 4 with eager steps on eight host
    threads and with every lockstep step as one graph launch; config 5 with every job
    replaying its captured step, and as the plain FP64 form run one job after another, eager
    (the comparison config 5 names).  Seeded synthetic jobs; wall-clock figures from the
    driver's own clock."""
    out = {}
    keep4 = ("bodies_steps_per_s", "steady_bodies_steps_per_s", "ensemble_step_ms_p50", "ensemble_step_ms_p99",
             "p50_step_ms", "p99_step_ms", "jobs", "failed", "rejected", "graph_launch_steps", "wall_s")
    keep5 = ("bodies_steps_per_s", "stepping_only_bodies_steps_per_s", "p50_step_ms", "p99_step_ms",
             "job_turnaround_s_p50", "job_turnaround_s_p99", "jobs", "failed", "rejected", "peak_concurrent", "wall_s")
    try:
        d = serve_run(CONFIG4)
        out["config4_ensemble_workers"] = {k: d.get(k) for k in keep4} if "failed" not in d or d["failed"] == 0 else d
        d = serve_run(CONFIG4 + ["--graph"])
        out["config4_ensemble_one_launch_per_step"] = {k: d.get(k) for k in keep4} if "failed" not in d or d["failed"] == 0 else d
        d = serve_run(CONFIG5 + ["--capture"])
        out["config5_served_mixed"] = {k: d.get(k) for k in keep5} if "failed" not in d or d["failed"] == 0 else d
        b = serve_run(CONFIG5 + ["--solo", "--precision", "fp64"], timeout=900)
        out["config5_fp64_sequential"] = {k: b.get(k) for k in keep5} if "failed" not in b or b["failed"] == 0 else b
        if d.get("bodies_steps_per_s") and b.get("bodies_steps_per_s"):
            out["config5_served_over_fp64_sequential"] = d["bodies_steps_per_s"] / b["bodies_steps_per_s"]
    except Exception as e:  # a failed record must not lose the headline line
        out["error"] = repr(e)[:300]
    out["note"] = "seeded synthetic jobs; bodies*steps/s over the driver's wall clock (set-up and arrivals included)"
    return out


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = os.path.join(tempfile.gettempdir(), f"ogx_clocks_{os.getpid()}_{index}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.out, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.out).read().strip().splitlines()]
            rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- our arm
def time_form(ogx, prec, p, pos, vel, mass, device, stream, flush, steps, warmup=2, eps=0.0, softening=0):
    """Step time of one more form on the same workload, measured like the headline (device
    resident, L2 flushed before every step, CUDA events on the library's stream)."""
    import torch
    with ogx.AdaptiveFMM3D(eps=eps, p=p, threshold=THR, precision=prec, device=device, stream=stream.cuda_stream,
                           softening=softening) as s:
        s.upload(pos, vel, mass)
        for _ in range(warmup):
            s.step(DT, 1)
        ms = []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s.step(DT, 1)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        st = s.stats()
    ms = np.array(ms)
    return {"p": p, "ms_per_step": float(ms.mean()), "bodies_per_s": mass.shape[0] / (float(ms.mean()) / 1e3),
            "p50_step_ms": float(np.percentile(ms, 50)), "p99_step_ms": float(np.percentile(ms, 99)),
            "steps": steps, "ms_m2l": st["ms_m2l"], "ms_leaf": st["ms_leaf"], "max_leaf_occupancy": st["max_leaf_occupancy"],
            "list_s": st["list_s"]}


def rms_max(ref, got):
    a = np.linalg.norm(ref, axis=1)
    e = np.linalg.norm(got - ref, axis=1)
    return float(np.sqrt((e * e).sum() / (a * a).sum())), float(np.max(e / np.maximum(a, 1e-6 * a.max())))


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import ogx
    import ogx_ic

    # a dedicated stream: the library and the timing events must share it (the legacy
    # default stream has handle 0, which the library would replace by its own stream)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    prec = {"mixed": ogx.PREC_MIXED, "fp64": ogx.PREC_FP64, "fp64rot": ogx.PREC_FP64_ROT}[args.precision]
    # ---- initial conditions (untimed): FP64 field for the circular velocities
    with ogx.AdaptiveFMM3D(p=P_ORDER, threshold=THR, precision=ogx.PREC_FP64, device=local) as ic_solver:
        pos, vel, mass, _ = ogx_ic.merger(args.n_per, seed=1, accel_fn=ic_solver.compute_accelerations)
    n = mass.shape[0]
    soft = ogx.SOFT_SPLINE if args.softening == "spline" else ogx.SOFT_PLUMMER
    solver = ogx.AdaptiveFMM3D(eps=args.eps, p=P_ORDER, threshold=THR, precision=prec, device=local,
                               stream=stream.cuda_stream, softening=soft)
    # each timed step replays a CUDA graph captured during the warm-up (no count read-back
    # in the middle of a step; a step that outgrows its capacities is redone eagerly)
    solver.set_tuning(capture_steps=0 if args.no_capture else 1)
    solver.upload(pos, vel, mass)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        solver.step(DT, 1)
    torch.cuda.synchronize()
    graph0 = solver.stats()["graph_steps"]
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    phase = []
    barrier()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.nvtx.range_push("ogx_step")
            starts[k].record(stream)
            solver.step(DT, 1)
            ends[k].record(stream)
            torch.cuda.nvtx.range_pop()
            phase.append(solver.stats())
        barrier()
    step_ms = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
    my_ms = float(step_ms.sum())
    tot_ms = max_over_ranks(my_ms, dist, "cuda")
    ms_per_step = tot_ms / args.steps
    value = replica_value(n, world, ms_per_step)
    st = phase[-1]

    # ---- e2e through the C ABI with pinned host buffers
    pos_h = torch.from_numpy(np.ascontiguousarray(pos)).pin_memory()
    mass_h = torch.from_numpy(np.ascontiguousarray(mass)).pin_memory()
    acc_h = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    for _ in range(2):
        solver.compute_accelerations_host_ptr(n, pos_h.data_ptr(), mass_h.data_ptr(), acc_h.data_ptr())
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        solver.compute_accelerations_host_ptr(n, pos_h.data_ptr(), mass_h.data_ptr(), acc_h.data_ptr())
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e_mean = max_over_ranks(float(np.mean(e2e_ms)), dist, "cuda")

    # ---- accuracy on the evaluated configuration (untimed)
    acc_info = {}
    if not args.no_accuracy and rank == 0:
        acc_form = acc_h.numpy().copy()
        with ogx.DirectSolver3D(eps=args.eps, device=local, softening=soft) as d:
            ref = d.compute_accelerations(pos, mass)
        with ogx.AdaptiveFMM3D(eps=args.eps, p=P_ORDER, threshold=THR, precision=ogx.PREC_FP64, device=local,
                               softening=soft) as f64:
            acc64 = f64.compute_accelerations(pos, mass)

        rms, mx = rms_max(ref, acc_form)
        rms64, mx64 = rms_max(ref, acc64)
        rmsf, _ = rms_max(acc64, acc_form)
        acc_info = {"rms_vs_fp64_direct": rms, "max_rel_vs_fp64_direct": mx, "rms_fp64_form_vs_direct": rms64,
                    "max_rel_fp64_form_vs_direct": mx64, "rms_vs_fp64_form": rmsf}

    # ---- the other forms on the same workload, same process (untimed in the headline):
    # the plain FP64 form at p = 8 (the mixed/plain speed-up), and both forms at p = 10,
    # the lowest order whose truncation error against the FP64 direct sum is below 1e-5
    forms = {}
    if (not args.no_accuracy and rank == 0 and prec == ogx.PREC_MIXED and args.eps == 0.0
            and args.softening == "plummer"):
        nf = max(3, min(args.steps, 5))
        forms["fp64_p8"] = time_form(ogx, ogx.PREC_FP64, P_ORDER, pos, vel, mass, local, stream, flush, nf)
        forms["fp64_p8"]["mixed_speedup"] = forms["fp64_p8"]["ms_per_step"] / ms_per_step
        forms["mixed_p10"] = time_form(ogx, ogx.PREC_MIXED, 10, pos, vel, mass, local, stream, flush, nf)
        forms["fp64_p10"] = time_form(ogx, ogx.PREC_FP64, 10, pos, vel, mass, local, stream, flush, nf)
        forms["mixed_p10"]["mixed_speedup"] = forms["fp64_p10"]["ms_per_step"] / forms["mixed_p10"]["ms_per_step"]
        with ogx.AdaptiveFMM3D(p=10, threshold=THR, precision=ogx.PREC_MIXED, device=local) as s10:
            am10 = s10.compute_accelerations(pos, mass)
        with ogx.AdaptiveFMM3D(p=10, threshold=THR, precision=ogx.PREC_FP64, device=local) as s10:
            a6410 = s10.compute_accelerations(pos, mass)
        r, m = rms_max(ref, am10)
        forms["mixed_p10"].update({"rms_vs_fp64_direct": r, "max_rel_vs_fp64_direct": m,
                                   "rms_vs_fp64_form": rms_max(a6410, am10)[0]})
        r, m = rms_max(ref, a6410)
        forms["fp64_p10"].update({"rms_vs_fp64_direct": r, "max_rel_vs_fp64_direct": m})
        # the same merger softened as the reference's own merger run (eps = 0.05): its Plummer
        # kernel, and the spline kernel with the far field corrected inside its support
        for kind, name in ((ogx.SOFT_PLUMMER, "mixed_eps0.05_plummer"), (ogx.SOFT_SPLINE, "mixed_eps0.05_spline")):
            forms[name] = time_form(ogx, ogx.PREC_MIXED, P_ORDER, pos, vel, mass, local, stream, flush, nf, eps=0.05,
                                    softening=kind)
        forms["note"] = ("same workload and timing as the headline (device-resident leapfrog step, L2 flushed); "
                         "mixed_speedup = FP64-form step time / mixed-form step time at the same p; "
                         "mixed_eps0.05_*: the same bodies softened with eps = 0.05 (list_s: leaf pairs the "
                         "spline's correction covers)")

    # ---- roofline of the dominant phase (CUDA events inside the library, same stream)
    phases = {k: float(np.mean([p[k] for p in phase])) for k in
              ("ms_tree", "ms_lists", "ms_upward", "ms_m2l", "ms_p2l", "ms_downward", "ms_leaf", "ms_total")}
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    tc_peak = peaks.get("bf16_tflops", 1590.0)
    K = (P_ORDER + 1) ** 2
    m2l_flops = 2.0 * K * K * st["list_v"] if st["list_v"] else 0.0
    traffic = M2L_DRAM_BYTES_PER_VPAIR * st["list_v"] if (M2L_DRAM_BYTES_PER_VPAIR and prec == ogx.PREC_MIXED) else None
    roofline = {"kernel": "m2l (k_m2l_tc, useful 2K^2 flops per V pair; split precision executes 3x)",
                "bound": "tensor",
                "achieved": (m2l_flops / (phases["ms_m2l"] / 1e3) / 1e12) if phases["ms_m2l"] > 0 else None,
                "peak": tc_peak, "unit": "TFLOP/s", "traffic": traffic,
                "peak_source": ("MEASURED_PEAKS.json bf16_tflops (of measured)" if peaks else
                                "fallback 1.59 PFLOP/s (of fallback)")}
    if roofline["achieved"] is not None:
        roofline["frac"] = roofline["achieved"] / roofline["peak"]

    line = {
        "metric": METRIC, "value": value, "unit": "bodies/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "mixed(f32 P2P, scaled 3xFP16 tensor-core M2L, f64 translations)" if prec == ogx.PREC_MIXED else ("f64 (rotation-based M2L)" if prec == ogx.PREC_FP64_ROT else "f64"),
        "data": "synthetic",
        "config": arm_config(n, args.n_per, world, args.eps, args.softening),
        "p50_step_ms": float(np.percentile(step_ms, 50)), "p99_step_ms": float(np.percentile(step_ms, 99)),
        "e2e": {"value": replica_value(n, world, e2e_mean), "unit": "bodies/s", "h2d_bytes_per_step": int(32 * n),
                "d2h_bytes_per_step": int(24 * n), "ms_per_step": e2e_mean},
        "step_capture": {"on": not args.no_capture, "graph_steps_timed": int(st["graph_steps"] - graph0),
                         "eager_redos": int(st["step_redos"])},
        "phases_ms": phases, "tree": {k: st[k] for k in ("num_boxes", "num_leaves", "max_level", "max_leaf_occupancy",
                                                          "list_u", "list_v", "list_w", "p2p_pairs", "m2p_evals")},
        "pair_interactions_per_s": st["p2p_pairs"] * world / (ms_per_step / 1e3),
        "roofline": roofline, "accuracy": acc_info, "forms": forms, "clocks": clk.summary(),
        "gpu_launches": int(st.get("launches", 0)) * args.steps,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_single()
    if rank == 0 and world == 1 and not args.no_serving and os.path.exists(SERVE):
        solver.close()
        line["configs_4_5"] = serving_records()
    solver.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
