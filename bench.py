"""Benchmark of the low-order frequency-domain BEM hot path on B200.

Workload (one step): the finite-depth cylinder of 4096 panels -- radius 1 m, draft 0.5 m, 64 x 32 side
and 64 x 32 bottom panels, depth h = 5 m, 40 wave periods evenly spaced 1.5-20 s, 4 headings
(0/30/60/90 deg) -- solved end to end: panel geometry and statics once, then for every frequency the
assembly of S and A, the right-hand sides of 6 radiation + 4 diffraction problems, the LU and
substitution, and the pressure integration to A, B, X.  Metric: frequency solves per second.
Inputs are synthetic (the reference's procedural mesh of that shape); every matrix (537 MB FP64 per
frequency) is larger than the 126 MB L2, so no L2 flush is needed between steps.

Arms:
  (default)         this library, through its C ABI (hbg_solve_batch), precision --precision
  --impl reference  the CPU restatement of the reference's path (oracle/, C + LAPACK) in its default
                    (production) arithmetic on all the host cores, every step one whole job.

Multi-GPU (torchrun): every rank solves its own copy of the job on its own GPU (independent
(body, frequency) units, no collective on the data path: weak scaling); the step time is the max
over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_PERIODS = 40
HEADINGS = [0.0, 30.0, 60.0, 90.0]
DEPTH = 5.0
WORKLOAD = "cylinder r=1 m d=0.5 m, 4096 panels (64x32 side + 64x32 bottom), h=5 m, 40 periods 1.5-20 s, 4 headings"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of a kernel family on the
# benchmark workload, from an ncu capture of the 8-frequency medium case scaled by 5 (every byte of
# the assembly scales with the frequencies of the launch).
DRAM_TRAFFIC = {("mixed", "assemble"): 32.5e9}

CASE_LABELS = {
    "c2": WORKLOAD,
    "c1": "cylinder r=1 m d=0.5 m, 512 panels (32x8 side + 32x8 bottom), infinite depth, 10 periods 2-11 s, "
          "heading 0 deg",
    "medium": "cylinder r=1 m d=0.5 m, 4096 panels, h=5 m, 8 periods 1.5-20 s, 4 headings (profiling cut)",
    "small": "cylinder r=1 m d=0.5 m, 2048 panels (32x16 side + 32x16 bottom), h=5 m, 4 periods 1.5-20 s, "
             "4 headings (profiling cut)",
    "tiny": "cylinder r=1 m d=0.5 m, 32 panels, h=5 m, 3 periods 1.5-20 s, 4 headings (host-logic tests)",
    "c3": "64 uneven bodies (seed 20261203: truncated cylinders or hemispheres, 840-5928 panels, 223044 in all), "
          "16 frequencies each (K r ~ U[0.1, 10]), headings 0 and 45 deg, infinite depth",
    "c4": "three cylinders r=1 m d=1 m 4 m apart (3 x 4096 panels, 18 interacting modes), 32 frequencies "
          "K a = 0.1-2, heading 0 deg, infinite depth",
    "c5": "barge 80 x 20 x 10 m: 16448 wetted + 2048 interior-lid panels, 100 frequencies K L ~ U[0.05, 8] "
          "(L = 80 m, seed 5), 8 headings, infinite depth",
}
# one-body cases: with N GPUs every rank solves its own copy of the job (weak scaling); the others are
# fixed workloads whose (body, frequency) units are split over the ranks (strong scaling)
SINGLE_BODY = ("c2", "c1", "medium", "small", "tiny")


def case_depth_headings():
    """(depth, headings in degrees) of a one-body case."""
    return (math.inf, [0.0]) if CASE == "c1" else (DEPTH, HEADINGS)


CASE = "c2"


def workload():
    """The benchmark body and frequencies; --case small is a 2048-panel, 4-frequency cut of the same
    family for profiler captures (each matrix 67 MB, the batch still larger than L2); --case medium
    the 4096-panel body at 8 of the periods (the benchmark's matrix shapes, a fifth of its batch)."""
    from hydrobem_b200 import meshes

    if CASE == "small":
        return meshes.cylinder(1.0, 0.5, 32, 16, 16), 2.0 * math.pi / np.linspace(1.5, 20.0, 4)
    if CASE == "medium":
        return meshes.cylinder(1.0, 0.5, 64, 32, 32), 2.0 * math.pi / np.linspace(1.5, 20.0, 8)
    if CASE == "tiny":
        return meshes.cylinder(1.0, 0.5, 8, 2, 2), 2.0 * math.pi / np.linspace(1.5, 20.0, 3)
    if CASE == "c1":
        return meshes.cylinder(1.0, 0.5, 32, 8, 8), 2.0 * math.pi / np.arange(2.0, 12.0)
    v = meshes.cylinder(1.0, 0.5, 64, 32, 32)
    periods = np.linspace(1.5, 20.0, N_PERIODS)
    return v, 2.0 * math.pi / periods


def case_problems():
    """The problems of the case as keyword dicts of native.Body, and the depth."""
    from hydrobem_b200 import meshes

    if CASE in SINGLE_BODY:
        v, omegas = workload()
        depth, heads = case_depth_headings()
        return [dict(vertices=v, omegas=omegas, headings_deg=heads)], depth
    if CASE == "c3":
        return [dict(vertices=v, omegas=om, headings_deg=[0.0, 45.0]) for v, om in meshes.uneven_bodies(64)], math.inf
    if CASE == "c4":
        v, pb, centers = meshes.cylinder_array()
        omegas = np.sqrt(np.linspace(0.1, 2.0, 32) * meshes.GRAVITY)
        return [dict(vertices=v, omegas=omegas, headings_deg=[0.0], panel_body=pb, rotation_centers=centers)], math.inf
    if CASE == "c5":
        v, kinds = meshes.barge()
        omegas = np.sqrt(np.random.default_rng(5).uniform(0.05, 8.0, 100) / 80.0 * meshes.GRAVITY)
        return [dict(vertices=v, omegas=omegas, headings_deg=list(np.arange(8) * 22.5), kinds=kinds)], math.inf
    raise ValueError(CASE)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, values, device="cpu"):
    """The element-wise maximum over ranks (the job's time is that of its slowest rank)."""
    if pg is None:
        return [float(x) for x in values]
    import torch

    t = torch.tensor([float(x) for x in values], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_cores():
    """The threads the CPU baseline uses: OMP_NUM_THREADS when set (the oracle's OpenMP and OpenBLAS
    follow it), else the cores this process may run on."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count()
    env = os.environ.get("OMP_NUM_THREADS", "")
    return min(n, int(env)) if env.isdigit() and int(env) > 0 else n


def cpu_job(production=True):
    """One whole job of the benchmark workload on the host cores by the CPU restatement of the reference
    (oracle/: C with OpenMP over rows, LAPACK ?gesv through scipy's threaded OpenBLAS): statics once, then
    every frequency -- no sampling.  production: the reference's default arithmetic (float32 Gauss tiers,
    direct wave-kernel tables, float32 static rows, complex64 matrices and LU); otherwise its diagnostic
    double path.  Returns (job seconds, statics seconds, mean seconds per frequency)."""
    from oracle import oracle as O

    v, omegas = workload()
    depth, heads_deg = case_depth_headings()
    heads = np.radians(heads_deg)
    O.lib()
    t0 = time.perf_counter()
    pan = O.make_panels(v)
    with O.ProductionMode(production):
        st = O.statics(pan, None, depth)
    t1 = time.perf_counter()
    for w in omegas:
        O.solve_frequency(pan, None, st, depth, w, heads, production=production)
    t2 = time.perf_counter()
    return t2 - t0, t1 - t0, (t2 - t1) / len(omegas)


def cpu_reference(args, world, rank, pg):
    """The reference's CPU path in its default (production) arithmetic, restated in oracle/, on all the
    host's cores: every step one whole job (statics + every frequency)."""
    if rank != 0:
        return None
    if CASE not in SINGLE_BODY:
        return {"impl": "reference", "unavailable": "the CPU reference arm times the one-body cases (c2, c1, medium, "
                                                    "small, tiny)"}
    cores = host_cores()
    for _ in range(min(args.warmup, 1)):
        cpu_job(True)
    times = [cpu_job(True) for _ in range(args.steps)]
    job = float(np.mean([t[0] for t in times]))
    F = len(workload()[1])
    value = F / job
    sample = (f"the whole job every step: statics ({np.mean([t[1] for t in times]):.2f} s) + all {F} frequencies "
              f"({np.mean([t[2] for t in times]):.3f} s each); {cores} threads on {cpu_model()}")
    line = {"metric": "freq solves/s at N=4096" if CASE == "c2" else "freq solves/s", "value": value, "unit": "freq solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": min(args.warmup, 1), "ms_per_step": job * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64+f32", "data": "synthetic",
            "config": {"workload": CASE_LABELS[CASE],
                       "form": "production (the reference's default path: float32 Gauss tiers, direct tables, "
                               "complex64 LU)",
                       "l2": "inputs larger than L2"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "freq solves/s", "cores": cores, "kind": "port",
                             "mode": "production", "cpu": cpu_model(), "sample": sample},
            "e2e": {"value": value, "unit": "freq solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def ours(args, world, rank, local, pg):
    import torch

    from hydrobem_b200 import native as nv

    from hydrobem_b200 import partition

    device = local if torch.cuda.is_available() else 0
    torch.cuda.set_device(device)
    probs, depth = case_problems()
    weak = CASE in SINGLE_BODY
    jobs = probs * world if weak else probs  # weak: one copy of the job per rank
    # this rank's (body, frequency) runs: the planner splits the units by their modelled cost
    runs = partition.plan([(len(p["vertices"]), len(p["omegas"])) for p in jobs], world)[rank]
    mine = [dict(jobs[r.body], omegas=np.asarray(jobs[r.body]["omegas"])[r.f0:r.f1]) for r in runs]
    precision = nv.HBG_MIXED if args.precision == "mixed" else nv.HBG_FP64
    bodies = [nv.Body(**m) for m in mine]
    arr = (nv.HbgProblem * max(len(bodies), 1))(*[b.problem() for b in bodies])
    opt = nv.default_options(precision=precision, depth=depth, device=device, concurrency=args.concurrency)
    import ctypes

    L = nv.lib()

    def step():
        if bodies:
            nv.check(L.hbg_solve_batch(arr, len(bodies), ctypes.byref(opt)))

    def barrier():
        if pg is not None:
            pg.barrier()

    for _ in range(args.warmup):
        step()
    # timed region: K steps bracketed by barrier + synchronize; device time by CUDA events
    nv.profile_kernels(False)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dev_ms, dev_phases = [], []
    with Clocks(device) as clk:
        e0.record()
        for _ in range(args.steps):
            step()
            ph = nv.last_profile()
            dev_ms.append(ph["total"])
            dev_phases.append([round(ph[k], 2) for k in ("statics", "assembly", "lu", "substitution", "forces")])
        e1.record()
        torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    step_ms = float(np.mean(dev_ms))
    step_ms, e2e_ms = reduce_max(pg, [step_ms, e2e_ms], f"cuda:{device}")
    launches = nv.last_launch_count()
    # one more step with kernel-family timing for the roofline (outside the timed region)
    nv.profile_kernels(True)
    step()
    prof = nv.kernel_profile()
    nv.profile_kernels(False)
    phases = nv.last_profile()
    ir = {"iterations": nv.last_ir_iterations(), "history": [float(f"{x:.3g}") for x in nv.last_ir_history()]} \
        if precision == nv.HBG_MIXED else None
    fallbacks = nv.last_fallback_count() if precision == nv.HBG_MIXED else None
    fallback_ms = nv.last_fallback_time() if precision == nv.HBG_MIXED else None
    pipe_peaks = nv.measure_peaks()  # FP64 FMA / FP64 MMA / TF32 tcgen05 of this device, measured here
    if rank != 0:
        return None
    F = sum(len(p["omegas"]) for p in jobs)  # frequency solves of the whole job over all ranks
    value = F / (step_ms * 1e-3)
    e2e = F / (e2e_ms * 1e-3)
    h2d = sum(b.vertices.nbytes + b.omegas.nbytes + b.headings.nbytes + (0 if b.kinds is None else b.kinds.nbytes)
              for b in bodies)
    d2h = sum(b.A.nbytes + b.B.nbytes + b.X.nbytes + b.FK.nbytes + b.SC.nbytes + b.HK.nbytes for b in bodies)
    peaks, peak_kind = measured_peaks()
    # the dominant kernel family by device time; in the mixed form the LU families run on concurrent
    # streams (their per-launch event times overlap one another), so the choice is among the others
    concurrent = {"lu_panel", "mixed_gemm", "mixed_convert"} if precision == nv.HBG_MIXED else set()
    fam, (ms, n, work) = max(((k, x) for k, x in prof.items() if k not in concurrent), key=lambda kv: kv[1][0])
    flops = fam in nv.FLOP_FAMILIES
    achieved = work / (ms * 1e-3) / (1e12 if flops else 1e9) if ms > 0 else None
    if flops:
        if fam == "mixed_gemm":
            peak = pipe_peaks["tf32_tcgen05"]
            pk = "tf32 tcgen05 dense (measured in this run by hbg_measure_peaks)"
        else:
            peak = pipe_peaks["fp64_fma"]
            pk = "fp64 FMA (measured in this run by hbg_measure_peaks)"
        bound, unit = "tensor", "TFLOP/s"
    else:
        peak, bound, unit, pk = peaks["hbm_gbs"], "hbm", "GB/s", f"hbm copy ({peak_kind})"
    traffic = DRAM_TRAFFIC.get((args.precision, fam)) if CASE == "c2" else None
    clocks = clk.summary()
    line = {"metric": "freq solves/s at N=4096" if CASE == "c2" else "freq solves/s", "value": value,
            "unit": "freq solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak" if weak else "strong", "vs_baseline": None,
            "dtype": "f64" if precision == nv.HBG_FP64 else "c64+tf32", "data": "synthetic",
            "config": {"workload": CASE_LABELS[CASE], "form": args.precision, "l2": "inputs larger than L2 (no flush)",
                       "parallelism": (f"one copy of the job per rank x{world}" if weak else
                                       f"(body, frequency) units split over {world} ranks by modelled cost")},
            "e2e": {"value": e2e, "unit": "freq solves/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches) * args.steps,
            "roofline": {"bound": bound, "kernel": fam, "achieved": achieved, "peak": peak, "unit": unit,
                         "frac": (achieved / peak) if (achieved and peak) else None, "traffic": traffic,
                         "peak_kind": pk, "launches": n, "ms": ms},
            "step_ms": [round(x, 2) for x in dev_ms],
            "step_phases_ms": {"order": ["statics", "assembly", "lu", "substitution", "forces"], "steps": dev_phases},
            "phases_ms": {k: round(x, 3) for k, x in phases.items()},
            "kernels_ms": {k: round(x[0], 3) for k, x in prof.items() if x[1]},
            "measured_peaks_tflops": {k: round(x, 1) for k, x in pipe_peaks.items()},
            "clocks": clocks}
    if ir is not None:
        line["refinement"] = ir
    if fallbacks is not None:
        line["fp64_fallback_frequencies"] = fallbacks
        # their FP64 solves' device time (of the kernel-timed step; summed over pipelines)
        line["fp64_fallback_ms"] = round(fallback_ms, 2)
    if precision == nv.HBG_FP64:  # over the timed steps' LU phase (the kernel-timed step's is inflated)
        line["lu"] = lu_rate(nv, {"lu": float(np.mean([p[2] for p in dev_phases]))}, pipe_peaks)
    if precision == nv.HBG_MIXED and not args.no_plain and bodies:
        line["plain_fp64"], plain = plain_comparison(nv, mine, bodies, depth, device, pipe_peaks)
    if precision == nv.HBG_MIXED and world == 1 and args.surrogate_steps > 0:
        line["surrogate"] = surrogate_comparison(nv, device, args.surrogate_steps)
    if world == 1 and not args.no_cpu_baseline and CASE in SINGLE_BODY:
        line["cpu_baseline"] = cpu_baseline_quick()
    return line


def lu_rate(nv, phases, pipe_peaks):
    """The FP64 form's factorizations of the last solve: real flops (the panel, triangular-solve and
    product launches' counted work), their rate over the LU phase, and that rate over the measured FP64
    peaks (FMA and warp MMA)."""
    prof = nv.kernel_profile()
    flops = sum(prof[k][2] for k in ("lu_panel", "lu_trsm", "lu_gemm"))
    ms = phases.get("lu", 0.0)
    tf = flops / (ms * 1e-3) / 1e12 if ms > 0 else None
    return {"flops": flops, "ms": round(ms, 2), "tflops": tf,
            "frac_of_fp64_fma": tf / pipe_peaks["fp64_fma"] if tf else None,
            "frac_of_fp64_mma": tf / pipe_peaks["fp64_mma"] if tf else None}


def plain_comparison(nv, mine, mixed_bodies, depth, device, pipe_peaks, max_solves=400):
    """The plain FP64 form of the same problems (the correctness oracle of the mixed form): its
    throughput, the speed-up of the mixed form, and the error of the mixed A, B, X against it (per entry,
    over the entry's largest modulus across frequencies, floor 1e-3 of the quantity's peak).  When the job
    has more than max_solves frequency solves the FP64 form runs on the first frequencies of each problem
    (the same count for each), and the comparison covers those."""
    import ctypes

    total = sum(len(m["omegas"]) for m in mine)
    keep = None if total <= max_solves else max(1, max_solves // len(mine))
    sub = [dict(m, omegas=np.asarray(m["omegas"])[:keep]) for m in mine]
    bodies = [nv.Body(**m) for m in sub]
    arr = (nv.HbgProblem * len(bodies))(*[b.problem() for b in bodies])
    opt = nv.default_options(precision=nv.HBG_FP64, depth=depth, device=device)
    L = nv.lib()
    nv.check(L.hbg_solve_batch(arr, len(bodies), ctypes.byref(opt)))  # warm-up
    ms = []
    for _ in range(2):
        nv.check(L.hbg_solve_batch(arr, len(bodies), ctypes.byref(opt)))
        ms.append(nv.last_profile()["total"])
    step = float(np.mean(ms))
    plain = [b.results() for b in bodies]
    mixed = [b.results() for b in mixed_bodies]
    nf = sum(len(m["omegas"]) for m in sub)
    err = {k: max(scaled_error(np.asarray(mx[k])[:len(pl[k])], pl[k]) for mx, pl in zip(mixed, plain))
           for k in ("A", "B", "X", "HK")}
    phases = nv.last_profile()
    out = {"value": nf / (step * 1e-3), "ms_per_step": step, "err_vs_fp64": err,
           "phases_ms": {k: round(x, 2) for k, x in phases.items()}, "lu": lu_rate(nv, phases, pipe_peaks)}
    if keep is not None:
        out["frequencies"] = f"the first {keep} of each problem ({nf} solves)"
    return out, plain


def scaled_error(got, ref):
    """Per entry |got - ref| over the entry's largest modulus across frequencies (floor 1e-3 of the
    quantity's peak), the largest over all entries."""
    ref = np.asarray(ref)
    peak = np.abs(ref).max()
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), 1e-3 * peak)
    return float((np.abs(np.asarray(got) - ref) / scale).max())


def surrogate_comparison(nv, device, train_steps):
    """The learned part measured against the table evaluation it would replace, on the three-cylinder
    array (3 x 4096 panels, infinite depth; three of its 32 frequencies): train the wave-term network on
    the device (its own kernels, 2^22 samples of the table and series evaluation over K R < 100,
    -K (z + zeta) < 50), solve the frequencies in the mixed form with the table and with the network as
    the wave term (tensor cores, tcgen05), and report each one's assembly time and A, B, X error against
    the FP64 form, the device time of one million evaluations of each, and the roofline bound of the
    network: its FLOPs per pair over the BF16 tensor peak, against the table's measured time per pair."""
    import ctypes

    from hydrobem_b200 import meshes

    samples = 1 << 22
    p, nm, rep = nv.surrogate_train(n_train=samples, batch=8192, steps=train_steps, lr=2e-3, seed=1,
                                    n_val=1 << 16)
    v, pb, centers = meshes.cylinder_array()
    omegas = np.sqrt(np.linspace(0.1, 2.0, 32) * meshes.GRAVITY)[[0, 15, 31]]
    N, F = len(v), len(omegas)
    kw = dict(panel_body=pb, rotation_centers=centers, device=device)
    ref = nv.solve(v, omegas, [0.0], precision=nv.HBG_FP64, **kw)
    out = {}
    for name, sg in (("table", None), ("network", nv.surrogate_blob(p, nm))):
        extra = {} if sg is None else {"surrogate": sg}
        nv.solve(v, omegas, [0.0], precision=nv.HBG_MIXED, **kw, **extra)  # warm-up
        got = nv.solve(v, omegas, [0.0], precision=nv.HBG_MIXED, **kw, **extra)
        prof = nv.last_profile()
        err = {k: scaled_error(got[k], ref[k]) for k in ("A", "B", "X")}
        out[name] = {"assembly_ms": round(prof["assembly"], 3), "job_ms": round(prof["total"], 3),
                     "pairs_from_network": int(nv.last_surrogate_pairs()), "err_vs_fp64": err,
                     "meets_1e-5": bool(max(err.values()) <= 1e-5)}
    rng = np.random.default_rng(5)
    u = rng.uniform(0.0, 1.0, (1 << 20, 2))
    xy = np.column_stack([np.expm1(u[:, 0] * np.log1p(100.0)), np.expm1(u[:, 1] * np.log1p(50.0))])
    _, _, (ms_net, ms_tab) = nv.surrogate_eval(p, nm, xy)
    pairs = F * N * (N + 1) // 2  # pair kernels of the assembly (one per unordered pair and frequency)
    flops = 2 * (3 * 128 + 3 * 128 * 128 + 128 * 6)
    peaks, kind = measured_peaks()
    return {"workload": f"three-cylinder array, {N} panels, {F} frequencies K a = 0.1, 1.05, 2, infinite depth",
            "table": out["table"], "network": out["network"],
            "train": {"steps": train_steps, "samples": samples, "device_ms": round(rep["train_ms"], 1),
                      "val_rms_over_spread": {k: round(x, 5) for k, x in rep["val_rms_over_spread"].items()}},
            "eval_ms_per_1M_points": {"network": round(ms_net, 3), "table": round(ms_tab, 3)},
            "roofline": {"network_flops_per_pair": flops, "bf16_peak_tflops": peaks["bf16_tflops"], "peak_kind": kind,
                         "network_bound_ps_per_pair": round(flops / (peaks["bf16_tflops"] * 1e12) * 1e12, 2),
                         "table_ps_per_pair": round(out["table"]["assembly_ms"] * 1e-3 / pairs * 1e12, 2),
                         "network_ps_per_pair": round(out["network"]["assembly_ms"] * 1e-3 / pairs * 1e12, 2)}}


def cpu_baseline_quick():
    """The CPU restatement of the reference on one whole job (no sampling) in its default production
    arithmetic, and beside it one whole job of its diagnostic double path (the FP64 form's semantics)."""
    cores = host_cores()
    job, st, per = cpu_job(True)
    djob, dst, dper = cpu_job(False)
    F = len(workload()[1])
    return {"value": F / job, "unit": "freq solves/s", "cores": cores, "kind": "port", "mode": "production",
            "cpu": cpu_model(),
            "sample": f"one whole job: statics ({st:.2f} s) + all {F} frequencies ({per:.3f} s each)",
            "diag_fp64": {"value": F / djob, "unit": "freq solves/s",
                          "sample": f"one whole job: statics ({dst:.2f} s) + all {F} frequencies ({dper:.3f} s each)"}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison of the mixed form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--surrogate-steps", type=int, default=4000,
                    help="training steps of the wave-term network measured beside the mixed form (0: skip)")
    ap.add_argument("--case", default="c2", choices=list(CASE_LABELS))
    ap.add_argument("--concurrency", type=int, default=0,
                    help="problems of the job solved at once (0: the library's tuner; 1: one after another)")
    args = ap.parse_args()
    global CASE
    CASE = args.case
    world, rank, local, pg = dist_setup()
    try:
        if args.impl == "reference":
            line = cpu_reference(args, world, rank, pg)
        else:
            line = ours(args, world, rank, local, pg)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
