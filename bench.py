"""Benchmark of the SBE propagation (one JSON line on stdout).

Workload (default): the 600x600 Haldane problem -- a0 = 1.44 A, t1 = 0.075,
t2 = t1/3, phi0 = 1.16, M = 2.54 t2, 3.2 um 8-cycle sin^2 pulse at
E0 = 0.0045 a.u., velocity gauge, dt = 0.1 a.u. (35 302 steps), RK4,
T2 = 220 a.u. -- run two ways: the mixed method (FP32 RK stages, FP64 sums;
the headline `value`) and the plain FP64 method.  A step is one complete
propagation of that problem.  Inputs are synthetic (no dataset exists for
this path).  Metric: k-point time steps per second (k.steps/s) and HHG
solves/hour.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own CPU implementation (the
unmodified reference sources built in oracle/_ref; the C oracle if that build
is absent) over all host cores on a bounded k-slice of the same workload.
Under torchrun (N > 1) each rank runs its own solves (independent solves:
weak scaling, no collective on the data path); rank 0 prints.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "HHG solves/hour & k·steps/s, batched FP32 vs plain FP64 at ≤1e-3 err; p99 lat"
UNIT = "k·steps/s"
FLOPS_PER_KSTEP = {4: 198.0, 5: 370.0}   # algorithmic flops per k-point step, 2-band velocity gauge


def wannier_flops_per_rhs(N: int, nR: int) -> float:
    """Algorithmic flops of one length-gauge RHS of an N-band Wannier model:
    Fourier synthesis of H0, D_x, D_y at k+A over the Hermitian half
    (3 nR N^2 8/2), the commutator (16 N^3) and the eigenbasis dephasing
    rotations (4 x 8 N^3).  The eigensolver is not counted."""
    return 3 * nR * N * N * 8 / 2 + 16 * N ** 3 + 4 * 8 * N ** 3
# Algorithmic flops per k-point step of the 2-band Haldane length gauge
# (FMA = 2): field terms of H0(k+A) at one stage time 44 (angle additions 27,
# B 10, |B|^2 5, 1/|B|^2 and (g2-g1)/|B|^2 2); right-hand side 30 (s.B 5,
# f 1, three components of 2 B x s + f B - g2 s at 8 each); currents and
# occupations 100 (cos of the b-vector angles 9, four j sums per axis 48,
# (s.B)/|B|^2 6, per axis interband and intraband 30, weights 1,
# occupations 6).  RK4: 4 RHS + 2 new stage times + 3 stage inputs and the
# final combination over 4 components (24 + 32) + currents = 364; Fehlberg
# RK5: 6 RHS + 5 new stage times + 15 stage-input and 5 final terms over 4
# components (120 + 40) + currents = 660.
LW_FLOPS_PER_KSTEP = {4: 364.0, 5: 660.0}
L2_FLUSH_BYTES = 512 << 20


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.proc, self.path = gpu, None, None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        busy = [s for s, _, _ in rows if s > 500] or [s for s, _, _ in rows]
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": rows[0][1], "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------- GPU arm
def bench_config(n: int, Nt: int, ncycles: float, env: str) -> dict:
    """The workload of one bench step, identical in both arms."""
    return {"workload": f"Haldane {n}x{n} velocity gauge, 3.2um {ncycles:g}-cycle {env} pulse (E0=0.0045), "
                        f"dt=0.1 ({Nt} steps), RK4, T2=220; one whole solve per step",
            "k_points": n * n, "time_steps": Nt, "precision": "fp64",
            "l2": "flushed (512 MiB write) between timed GPU steps; per-k state 69 MB > L2 per solve",
            "parallelism": "independent whole solves per device (weak scaling)"}


def run_ours(args):
    import torch

    # record the launch shapes the autotuner picks (reported in the JSON line)
    tune_file = tempfile.NamedTemporaryFile(prefix="sbe_tune_", suffix=".txt", delete=False).name
    os.environ.setdefault("SBE_TUNE_CACHE", tune_file)

    import antelope_b200 as ab
    from antelope_b200 import cfgtext, workloads
    from antelope_b200.api import Solver
    from antelope_b200.spectrum import per_harmonic_error

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    n = args.grid
    case = {p: workloads.haldane_case(n=n, precision=p, ncycles=args.ncycles, env=args.env)
            for p in ("mixed", "fp64")}
    probs = {p: ab.Problem.from_dict(c) for p, c in case.items()}
    dims = probs["fp64"].dims
    kst = float(dims.ntotal) * dims.Nt

    def timed(prec, k, w, profile):
        # solvers are created (tables uploaded, per-k set-up done) before timing
        solvers = [Solver(probs[prec], precision=prec, profile=profile, tile_k=args.tile_k,
                          k_per_thread=args.kpt, steps_per_launch=args.steps_per_launch) for _ in range(k + w)]
        for s in solvers[:w]:
            s.run(stream.cuda_stream)
        torch.cuda.synchronize()
        if profile:
            for s in solvers[:w]:
                s.kernel_times()
        times, launches, ktimes = [], 0, []
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for s in solvers[w:]:
            with torch.cuda.stream(stream):
                flush.zero_()                          # L2 flush between steps, outside the events
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                s.run(stream.cuda_stream)
                e1.record(stream)
            launches += s.launches
            times.append((e0, e1))
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ms = [a.elapsed_time(b) for a, b in times]
        if profile:
            ktimes = [s.kernel_times() for s in solvers[w:]]
        out = solvers[-1].get()
        for s in solvers:
            s.close()
        return ms, launches, ktimes, out

    from antelope_b200.dist import max_over_ranks

    # headline: the plain FP64 kernel, the reference's precision, on the
    # reference arm's workload; the mixed method follows as an extra section
    with ClockSampler(local) as clk:
        ms_fp64, launches, kt_fp64, out_fp64 = timed("fp64", args.steps, args.warmup, True)
        total_ms = max_over_ranks(sum(ms_fp64), dev)   # whole-job device time: max over ranks
        ms_mixed, launches_mixed, kt_mixed, out_mixed = timed("mixed", max(3, args.steps // 2), 2, True)
    clocks = clk.summary()
    value = world * args.steps * kst / (total_ms * 1e-3)
    mixed_value = kst / (statistics.mean(ms_mixed) * 1e-3)

    # per-harmonic spectral error of the mixed run against the FP64 run
    w0 = case["fp64"]["laser"]["pulses"][0]["w0"]
    spectral = {}
    for floor in (1e-6, 1e-8):
        orders, err, _ = per_harmonic_error({"inter": out_mixed.inter, "intra": out_mixed.intra},
                                            {"inter": out_fp64.inter, "intra": out_fp64.intra}, dims.dt, w0,
                                            floor=floor)
        spectral[f"max_floor_{floor:g}"] = float(err.max())
        spectral[f"harmonics_floor_{floor:g}"] = int(len(orders))

    # e2e through the C ABI from host inputs to host outputs, plain FP64
    e2e_s, phases = [], []
    text = cfgtext.dumps(case["fp64"])
    for i in range(max(3, args.steps // 2)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p = ab.Problem.from_text(text)
        t1 = time.perf_counter()
        s = Solver(p, precision="fp64")
        t2 = time.perf_counter()
        s.run(0)
        s.get()
        t3 = time.perf_counter()
        s.close()
        t4 = time.perf_counter()
        e2e_s.append(t4 - t0)
        phases.append((t1 - t0, t2 - t1, t3 - t2, t4 - t3))
    shapes_now = read_tune_cache()
    tile_k = args.tile_k or next((v["tile_k"] for k, v in shapes_now.items() if k.startswith("vg-fp64")), 128)
    ntiles = -(-dims.ntotal // tile_k)
    # the field table and per-k set-up are computed on the device from the
    # problem; what crosses to the device is the solve descriptor (with the
    # laser parameters) and the tile list, and back the per-step sums
    h2d = 512 + ntiles * 16
    d2h = dims.Nt * 8 * 8 + ntiles * 8 * 8       # per-step sums + per-tile constants
    # median over the samples: one host-side hiccup would dominate a mean
    e2e_value = kst / statistics.median(e2e_s)

    # roofline of the propagate kernels from their own launch events
    fp64_tf, fp32_tf, fp32x2_tf = ab.measure_fma_peaks(local)
    prop64 = sum(k["propagate_ms"] for k in kt_fp64)
    red64 = sum(k["reduce_ms"] for k in kt_fp64)
    achieved = FLOPS_PER_KSTEP[4] * kst * len(kt_fp64) / (prop64 * 1e-3) / 1e12
    propm = sum(k["propagate_ms"] for k in kt_mixed)
    redm = sum(k["reduce_ms"] for k in kt_mixed)
    ach_m = FLOPS_PER_KSTEP[4] * kst * len(kt_mixed) / (propm * 1e-3) / 1e12
    shapes = read_tune_cache()
    kpt_mixed = args.kpt or next((v["k_per_thread"] for k, v in shapes.items() if k.startswith("vg-mixed")), 2)
    kpt_fp64 = args.kpt or next((v["k_per_thread"] for k, v in shapes.items() if k.startswith("vg-fp64")), 1)
    mixed_kernel = "propagate_vg_x2<4> (2 k-points per thread, packed f32x2)" if kpt_mixed == 2 \
        else "propagate_vg<float,4,1>"

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(n, dims.Nt, args.ncycles, args.env),
        "solves_per_hour": value / kst * 3600.0,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "seconds_per_solve": statistics.median(e2e_s), "statistic": f"median of {len(e2e_s)} solves",
                "seconds_min_max": [min(e2e_s), max(e2e_s)],
                "phase_seconds": dict(zip(("parse", "create", "run_and_get", "destroy"),
                                          [statistics.mean(x) for x in zip(*phases)])),
                "path": "sbe_problem_from_string -> sbe_solver_create -> run -> sbe_solver_get (fp64)"},
        "roofline": {"bound": "fp64 FMA pipe", "achieved": achieved, "peak": fp64_tf, "unit": "TFLOP/s",
                     "frac": achieved / fp64_tf, "traffic": read_traffic("fp64"),
                     "peak_source": "measured FMA-chain microbenchmark on this GPU in this run "
                                    "(MEASURED_PEAKS.json has no FP64/FP32 figure)",
                     "flops_per_kstep": FLOPS_PER_KSTEP[4],
                     "kernel": f"propagate_vg<double,4,{kpt_fp64}>",
                     "kernel_share": prop64 / (prop64 + red64)},
        "mixed": {"value": mixed_value, "unit": UNIT, "dtype": "f32 stages / f64 state and sums",
                  "ms_per_solve": statistics.mean(ms_mixed), "solves_per_hour": mixed_value / kst * 3600.0,
                  "over_fp64": mixed_value / (value / world),
                  "spectral_error_vs_fp64": dict(spectral, floor="band power >= floor x the strongest"),
                  "roofline": {"bound": "fp32 FMA pipe", "achieved": ach_m, "peak": fp32_tf, "unit": "TFLOP/s",
                               "frac": ach_m / fp32_tf, "traffic": read_traffic("mixed"),
                               "kernel": mixed_kernel, "kernel_share": propm / (propm + redm)},
                  "launches": int(launches_mixed)},
        "fma_peaks_tflops": {"fp64": fp64_tf, "fp32": fp32_tf, "fp32x2": fp32x2_tf},
        "launch_shapes": shapes,
        "gpu_launches": int(launches) * 2,   # propagate + reduce per launch tick, timed steps only
        "clocks": clocks,
    }
    if args.lw_grid > 0 and world == 1:
        line["length_gauge"] = run_length_gauge(args, stream, fp64_tf, fp32_tf)
    if args.wannier_grid > 0 and world == 1:
        line["wannier"] = run_wannier(args, stream, fp64_tf)
    if args.scan_solves > 0:
        line["scan"] = run_scan(args, stream, rank, world)
    if args.serve_requests > 0 and world == 1:
        line["serving"] = run_serve(args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n, budget_s=args.cpu_seconds, ncycles=args.ncycles)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_length_gauge(args, stream, fp64_tf, fp32_tf):
    """The Haldane configuration (same model, pulse, dt, RK4, T2) in the
    length gauge, the reference's H0(k + A) form with eigenbasis dephasing,
    on its --lw-grid k-grid: plain FP64 and mixed, one solve each after a
    warm-up solve (launch shapes from the autotuner)."""
    import torch

    import antelope_b200 as ab
    from antelope_b200 import workloads
    from antelope_b200.api import Solver
    from antelope_b200.spectrum import per_harmonic_error

    n = args.lw_grid
    res, outs = {}, {}
    for prec in ("fp64", "mixed"):
        p = ab.Problem.from_dict(workloads.haldane_case(n=n, precision=prec, ncycles=args.ncycles,
                                                        gauge="Wannier"))
        kst = float(p.dims.ntotal) * p.dims.Nt
        ms = []
        for rep in range(2):   # the first solve is the warm-up
            s = Solver(p, precision=prec, profile=True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            s.run(stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
            kt = s.kernel_times()
            outs[prec] = s.get()
            s.close()
        t = ms[-1]
        tf = LW_FLOPS_PER_KSTEP[4] * kst / (kt["propagate_ms"] * 1e-3) / 1e12
        peak = fp64_tf if prec == "fp64" else fp32_tf
        res[prec] = {"ms_per_solve": t, "k_steps_per_s": kst / (t * 1e-3), "propagate_ms": kt["propagate_ms"],
                     "reduce_ms": kt["reduce_ms"], "achieved_tflops": tf, "roofline_frac": tf / peak,
                     "roofline_peak": "fp64 FMA pipe" if prec == "fp64" else "fp32 FMA pipe"}
    a, b = outs["fp64"], outs["mixed"]
    w0 = workloads.haldane_case(n=n)["laser"]["pulses"][0]["w0"]
    err = {}
    for floor in (1e-6, 1e-8):
        _, e, _ = per_harmonic_error({"inter": b.inter, "intra": b.intra}, {"inter": a.inter, "intra": a.intra},
                                     0.1, w0, floor=floor)
        err[f"max_floor_{floor:g}"] = float(e.max())
    return {"workload": f"Haldane {n}x{n} length gauge (H0(k+A), eigenbasis dephasing), 3.2um "
                        f"{args.ncycles:g}-cycle sin2, dt=0.1, RK4, T2=220",
            "fp64": res["fp64"], "mixed": res["mixed"],
            "mixed_over_fp64": res["fp64"]["ms_per_solve"] / res["mixed"]["ms_per_solve"],
            "flops_per_kstep": LW_FLOPS_PER_KSTEP[4],
            "spectral_error": dict(err, vs="fp64 run")}


def run_wannier(args, stream, fp64_tf):
    """The N = 6 Wannier configuration (triangular lattice, 37 lattice
    vectors, 3 valence bands, T2 = 220, 3.2 um sin2 pulse, Cash-Karp 4(5) at
    tol 1e-8 with one step size per solve) on its full k-grid: --wannier-seeds
    seeded models in one mixed-precision batch (sbe_batch_*: one attempt
    launch over all their k-points per iteration, each solve with its own
    controller, launches captured as CUDA graphs) against plain FP64 solves
    of the same models one at a time.  The pulse has --wannier-cycles cycles
    in place of 10 so that the run stays bounded: the work per step is the
    configuration's and the step count scales with the pulse length, so the
    10-cycle figures follow by the ratio of output steps (stated in the
    line).  k.steps count accepted steps; the roofline counts attempted ones."""
    import torch

    import antelope_b200 as ab
    from antelope_b200 import wannier
    from antelope_b200.api import Solver
    from antelope_b200.spectrum import per_harmonic_error

    n, nseeds = args.wannier_grid, args.wannier_seeds
    seeds = list(range(1, nseeds + 1))
    cases = [wannier.wannier_case(seed=s, n=n, ncycles=args.wannier_cycles, rk="cashkarp45", tol=1e-8)
             for s in seeds]
    group = cases[0]["SyntheticWannier"]
    N, nR = int(group["Nband"]), len(group["R"]) // 2
    probs = {prec: [ab.Problem.from_dict(dict(c, calc=dict(c["calc"], precision=prec))) for c in cases]
             for prec in ("fp64", "mixed")}
    nk = probs["fp64"][0].dims.ntotal
    Nt = probs["fp64"][0].dims.Nt
    full_steps = wannier.wannier_case(seed=1, n=4, ncycles=10.0)
    Nt_full = ab.Problem.from_dict(full_steps).dims.Nt

    def ev():
        return torch.cuda.Event(enable_timing=True)

    # plain FP64, one solve at a time (the first --wannier-fp64-seeds models)
    fp64_ms, fp64_out, fp64_st = [], [], []
    for p in probs["fp64"][:args.wannier_fp64_seeds]:
        s = Solver(p, precision="fp64")
        e0, e1 = ev(), ev()
        torch.cuda.synchronize()
        e0.record(stream)
        s.run(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        fp64_ms.append(e0.elapsed_time(e1))
        fp64_st.append(s.steps())
        fp64_out.append(s.get())
        s.close()
    # mixed, all seeds in one batch
    b = ab.Batch(probs["mixed"], precision="mixed", use_graph=True)
    e0, e1 = ev(), ev()
    torch.cuda.synchronize()
    e0.record(stream)
    b.run(stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1)
    mst = [b.steps(i) for i in range(nseeds)]
    errs6, errs8 = [], []
    w0 = cases[0]["laser"]["pulses"][0]["w0"]
    for i, a in enumerate(fp64_out):
        o = b.get(i)
        _, e6, _ = per_harmonic_error({"inter": o.inter, "intra": o.intra}, {"inter": a.inter, "intra": a.intra},
                                      0.1, w0, floor=1e-6)
        _, e8, _ = per_harmonic_error({"inter": o.inter, "intra": o.intra}, {"inter": a.inter, "intra": a.intra},
                                      0.1, w0, floor=1e-8)
        errs6.append(float(e6.max()))
        errs8.append(float(e8.max()))
    launches = b.launches
    b.close()
    rhs_flops = wannier_flops_per_rhs(N, nR) * 6 * nk
    fp64_att = sum(x["attempts"] for x in fp64_st)
    fp64_tflops = rhs_flops * fp64_att / (sum(fp64_ms) * 1e-3) / 1e12
    mixed_att = sum(x["attempts"] for x in mst)
    mixed_tflops = rhs_flops * mixed_att / (batch_ms * 1e-3) / 1e12
    sph_fp64 = len(fp64_ms) / (sum(fp64_ms) * 1e-3) * 3600.0
    sph_mixed = nseeds / (batch_ms * 1e-3) * 3600.0
    scale = Nt / Nt_full   # solves/hour of the 10-cycle pulse: step counts scale with its length
    out = {"workload": f"SyntheticWannier N={N}, {nR} R, {n}x{n} k, length gauge, Cash-Karp tol 1e-8, 3.2um sin2 "
                       f"pulse of {args.wannier_cycles:g} cycles ({Nt} output steps) in place of the "
                       f"configuration's 10 ({Nt_full} steps); {nseeds} seeds",
           "k_points": nk, "output_steps": Nt, "output_steps_10_cycles": Nt_full,
           "fp64": {"solves": len(fp64_ms), "ms_per_solve": statistics.mean(fp64_ms),
                    "k_steps_per_s": nk * sum(x["steps"] for x in fp64_st) / (sum(fp64_ms) * 1e-3),
                    "steps": fp64_st[0]["steps"], "attempts": fp64_st[0]["attempts"],
                    "solves_per_hour": sph_fp64, "solves_per_hour_10_cycles": sph_fp64 * scale,
                    "achieved_tflops": fp64_tflops, "roofline_frac_fp64": fp64_tflops / fp64_tf},
           "mixed_batch": {"solves": nseeds, "ms": batch_ms, "launches": launches, "graph": True,
                           "k_steps_per_s": nk * sum(x["steps"] for x in mst) / (batch_ms * 1e-3),
                           "solves_per_hour": sph_mixed, "solves_per_hour_10_cycles": sph_mixed * scale,
                           "achieved_tflops": mixed_tflops, "roofline_frac_fp64": mixed_tflops / fp64_tf},
           "batched_mixed_over_sequential_fp64": sph_mixed / sph_fp64,
           "flops_per_rhs": wannier_flops_per_rhs(N, nR), "rhs_per_attempt": 6,
           "spectral_error": {"max_floor_1e-6": max(errs6), "max_floor_1e-8": max(errs8),
                              "vs": f"fp64 solves of the first {len(fp64_out)} seeds"}}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = wannier_cpu_baseline(args.wannier_cycles, budget_s=args.cpu_seconds / 2,
                                                   grid=args.wannier_grid)
    return out


def wannier_cpu_baseline(ncycles: float, budget_s: float, grid: int = 300):
    """The reference's own propagation of the N = 6 model on all host cores:
    the harness build (the reference's SBEs/laser code with the
    SyntheticWannier material, oracle/make_harness.py) on ParaRange k-slices
    of the same grid, model and pulse, one emulated rank per core, sized to
    ~budget_s.  The reference has no adaptive integrator; its fixed-step
    Fehlberg-5 takes the same six stages per step as a Cash-Karp attempt, and
    at tol 1e-8 the Cash-Karp runs take one attempt per output step, so the
    work per k-point step is the same.  Without the harness build: the C
    oracle on a k-subgrid (kind "port")."""
    from antelope_b200 import cfgtext, wannier
    from oracle import pyoracle

    cores = os.cpu_count() or 1
    if os.path.exists(pyoracle.HARNESS_EXE):
        c = wannier.wannier_case(seed=1, n=grid, ncycles=ncycles, rk=None)
        c["calc"]["RKorder"] = 5
        del c["calc"]["precision"]
        per_kstep = 2.7e-4                      # single-core seconds per k-point step, N = 6, length gauge
        Nt_est = int(44129 * ncycles / 10.0) + 1
        ntot = grid * grid
        size = max(cores, int(ntot / max(1.0, budget_s / (Nt_est * per_kstep))))
        with tempfile.TemporaryDirectory() as d:
            with open(os.path.join(d, "inputParam.cfg"), "w") as f:
                f.write(cfgtext.dumps(c))
            t0 = time.perf_counter()
            procs = [subprocess.Popen([pyoracle.HARNESS_EXE], cwd=d, stdout=subprocess.DEVNULL,
                                      env=dict(os.environ, REF_RANK=str(r), REF_SIZE=str(size)))
                     for r in range(cores)]
            rc = [p.wait() for p in procs]
            wall = time.perf_counter() - t0
            with open(os.path.join(d, "outlaserdata.dat")) as f:
                Nt = sum(1 for line in f if line.strip())
        if any(rc):
            raise RuntimeError(f"reference harness run failed: {rc}")
        kdone = sum(ntot // size + (1 if ntot % size > r else 0) for r in range(cores))
        return {"value": kdone * Nt / wall, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": f"reference harness build (Fehlberg-5), {cores} processes x 1 emulated rank of {size} "
                          f"(ParaRange slices of the {grid}x{grid} grid, {kdone} k-points) x {Nt} steps"}

    def timed(g, cyc):
        c = wannier.wannier_case(seed=1, n=g, ncycles=cyc, rk="cashkarp45", tol=1e-8)
        t0 = time.perf_counter()
        r = pyoracle.run(c, nthreads=cores)
        return g * g * r["steps"] / (time.perf_counter() - t0), r["steps"]

    rate, _ = timed(8, 0.02)
    g = int(max(8, min(300, np.sqrt(rate * budget_s / 440.0 / max(ncycles, 0.05)))))
    rate, steps = timed(g, min(ncycles, 0.05))
    return {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"C oracle, same model, {g}x{g} k-subgrid, {steps} accepted steps, {cores} threads"}


def _fp64_sequential(problems, stream):
    """Plain FP64 solves one after another (device time per solve)."""
    import torch

    from antelope_b200.api import Solver

    total_ms, outs = 0.0, []
    for p in problems:
        s = Solver(p, precision="fp64")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.run(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        outs.append(s.get())
        s.close()
    return total_ms, outs


def run_scan(args, stream, rank, world):
    """The seeded 256-solve parameter scan: uneven grids 100^2..400^2, 4..12
    cycles, M/t2, phi0, ellipticity/helicity and CEP drawn per solve; mixed
    precision in one batch (all launches of the run in one CUDA graph),
    against the same solves run one by one in plain FP64 (every 4th solve)."""
    import torch

    import antelope_b200 as ab
    from antelope_b200 import workloads
    from antelope_b200.dist import max_over_ranks, para_range, sum_over_ranks
    from antelope_b200.spectrum import per_harmonic_error

    cases = workloads.scan_cases(n=args.scan_solves, precision="mixed")
    a, b = para_range(len(cases), world, rank)
    probs = [ab.Problem.from_dict(c) for c in cases[a:b]]
    kst = sum(float(p.dims.ntotal) * p.dims.Nt for p in probs)
    torch.cuda.synchronize()
    t_create = time.perf_counter()
    batch = ab.Batch(probs, precision="mixed", use_graph=True, steps_per_launch=256)
    torch.cuda.synchronize()
    t_create = time.perf_counter() - t_create
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.run(stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1))
    sub = list(range(0, len(probs), 4))
    fp64_ms, fp64_out = _fp64_sequential([probs[i] for i in sub], stream)
    errs = []
    for j, i in enumerate(sub[:8]):
        o = batch.get(i)
        w0 = cases[a + i]["laser"]["pulses"][0]["w0"]
        _, e, _ = per_harmonic_error({"inter": o.inter, "intra": o.intra},
                                     {"inter": fp64_out[j].inter, "intra": fp64_out[j].intra}, 0.1, w0)
        errs.append(float(e.max()))
    # harmonic band powers of every solve, on the GPU from the resident results
    t_h = time.perf_counter()
    for i in range(len(probs)):
        batch.harmonics(i, cases[a + i]["laser"]["pulses"][0]["w0"], 30)
    t_h = time.perf_counter() - t_h
    launches = batch.launches
    batch.close()
    nsolves = sum_over_ranks(len(probs))
    kst_all = sum_over_ranks(kst)
    sph = nsolves / (ms * 1e-3) * 3600.0
    sph64 = len(sub) / (fp64_ms * 1e-3) * 3600.0 * world
    return {"solves": int(nsolves), "k_steps": kst_all, "ms": ms, "k_steps_per_s": kst_all / (ms * 1e-3),
            "solves_per_hour": sph, "fp64_sequential_solves_per_hour": sph64,
            "batched_mixed_over_sequential_fp64": sph / sph64,
            "fp64_sequential_sample": f"{len(sub)} of {len(probs)} solves (every 4th)",
            "max_per_harmonic_error_vs_fp64": max(errs), "error_sample": f"{len(errs)} solves",
            "setup_s": t_create, "launches": launches, "graph": True, "steps_per_launch": 256,
            "harmonics_s_all_solves": t_h, "harmonics": "30 band powers per solve on the GPU (sbe_batch_harmonics)"}


def run_serve(args):
    """Poisson stream of Haldane and two-colour requests (64^2..512^2, 4..16
    cycles, 1.6..3.2 um, E0 in [0.002, 0.006]) into the continuous-batching
    server; p50/p99 latency from submit to result, and solves/hour against
    plain FP64 solves one after another on the same request distribution."""
    import concurrent.futures as cf

    import torch

    import antelope_b200 as ab
    from antelope_b200 import workloads

    arrivals, cases = workloads.serving_cases(n=args.serve_requests, rate_hz=args.serve_rate, precision="mixed")
    probs = [ab.Problem.from_dict(c) for c in cases]
    srv = ab.Server(precision="mixed", steps_per_launch=256)
    t0 = time.perf_counter()

    def submit(i):
        dt = t0 + arrivals[i] - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        return srv.submit(probs[i])

    # clients submit and wait from 16 threads each; a request's latency is
    # measured by the server (submit -> result available)
    with cf.ThreadPoolExecutor(max_workers=16) as pool:
        rids = list(pool.map(submit, range(len(probs))))
    with cf.ThreadPoolExecutor(max_workers=16) as pool:
        lat = [x[1] for x in pool.map(lambda r: srv.wait(r, timeout=600), rids)]
    wall = time.perf_counter() - t0
    stats = srv.stats()
    # capacity: the same requests submitted at once (saturated server)
    t1 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=16) as pool:
        rids2 = list(pool.map(srv.submit, probs))
    with cf.ThreadPoolExecutor(max_workers=16) as pool:
        lat_burst = np.array([x[1] for x in pool.map(lambda r: srv.wait(r, timeout=600), rids2)])
    wall_burst = time.perf_counter() - t1
    srv.close()
    kst = sum(float(p.dims.ntotal) * p.dims.Nt for p in probs)
    stream = torch.cuda.Stream()
    sub = list(range(0, len(probs), 20))
    fp64_ms, _ = _fp64_sequential([probs[i] for i in sub], stream)
    sph = len(probs) / wall * 3600.0
    sph64 = len(sub) / (fp64_ms * 1e-3) * 3600.0
    lat = np.array(lat)
    return {"requests": len(probs), "rate_hz": args.serve_rate, "wall_s": wall,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()), "solves_per_hour": sph, "k_steps_per_s": kst / wall,
            "fp64_sequential_solves_per_hour": sph64, "served_mixed_over_sequential_fp64": sph / sph64,
            "fp64_sequential_sample": f"{len(sub)} of {len(probs)} requests (every 20th)",
            "failed": stats["failed"], "launches": stats["launches"],
            "capacity_solves_per_hour": len(probs) / wall_burst * 3600.0,
            "capacity_k_steps_per_s": kst / wall_burst,
            "capacity_over_sequential_fp64": len(probs) / wall_burst * 3600.0 / sph64,
            "burst_p50_latency_s": float(np.percentile(lat_burst, 50)),
            "burst_p99_latency_s": float(np.percentile(lat_burst, 99)),
            "note": "Poisson stream at rate_hz: latency and solves/hour over the stream's wall time "
                    "(bounded by the offered load); capacity: the same requests submitted at once"}


def read_tune_cache():
    path = os.environ.get("SBE_TUNE_CACHE")
    out = {}
    try:
        for line in open(path):
            k, tile, kpt = line.split()
            out[k] = {"tile_k": int(tile), "k_per_thread": int(kpt)}
    except (OSError, TypeError, ValueError):
        pass
    return out


def read_traffic(kind: str):
    """DRAM bytes per propagate launch of the `kind` kernel (fp64 or mixed)
    from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "propagate_vg_dram_bytes.txt")
    try:
        for line in open(path):
            if line.startswith(f"bytes_per_launch_{kind} "):
                return float(line.split()[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------- CPU arms
def reference_case(n: int, ncycles: float) -> dict:
    """The bench workload as the unmodified reference reads it: its cos4
    envelope, no precision key."""
    from antelope_b200 import workloads

    case = workloads.haldane_case(n=n, env="cos4", ncycles=ncycles)
    del case["calc"]["precision"]
    return case


def cpu_baseline(n: int, budget_s: float = 15.0, samples: int = 1, ncycles: float = 8.0):
    """Time the reference on the host cores on a bounded k-slice of the
    n x n workload (each process = one emulated MPI rank of a large rank
    count; ParaRange, utility.h:104-115, gives it ~budget_s of work).  Nt is
    read from the reference's own outlaserdata.dat (rank 0 writes it), so this
    arm loads nothing of the product."""
    from antelope_b200 import cfgtext
    from oracle import pyoracle

    cores = os.cpu_count() or 1
    per_kstep = 2.4e-6                       # single-core seconds per k.step measured for this path
    Nt_est = int(35303 * ncycles / 8.0)
    kper = max(4, int(budget_s / (Nt_est * per_kstep)))
    ntot = n * n
    size = max(cores, ntot // kper)
    case = reference_case(n, ncycles)
    if os.path.exists(pyoracle.REF_EXE):
        kind, vals = "reference", []
        for _ in range(samples):
            with tempfile.TemporaryDirectory() as d:
                with open(os.path.join(d, "inputParam.cfg"), "w") as f:
                    f.write(cfgtext.dumps(case))
                t0 = time.perf_counter()
                procs = [subprocess.Popen([pyoracle.REF_EXE], cwd=d, stdout=subprocess.DEVNULL,
                                          env=dict(os.environ, REF_RANK=str(r), REF_SIZE=str(size)))
                         for r in range(cores)]
                rc = [p.wait() for p in procs]
                wall = time.perf_counter() - t0
                with open(os.path.join(d, "outlaserdata.dat")) as f:
                    Nt = sum(1 for line in f if line.strip())
            if any(rc):
                raise RuntimeError(f"reference run failed: {rc}")
            kdone = sum(ntot // size + (1 if ntot % size > r else 0) for r in range(cores))
            vals.append(kdone * Nt / wall)
        sample = (f"{cores} processes x 1 emulated rank of {size} (ParaRange slices of the {n}x{n} grid, "
                  f"{kdone} k-points) x {Nt} steps")
    else:
        kind = "port"
        g = max(2, int(np.sqrt(cores * kper)))
        c2 = reference_case(g, ncycles)
        vals = []
        for _ in range(samples):
            t0 = time.perf_counter()
            r = pyoracle.run(c2, nthreads=cores)
            wall = time.perf_counter() - t0
            Nt = r["dims"]["Nt"]
            vals.append(g * g * Nt / wall)
        sample = f"C oracle on a {g}x{g} grid x {Nt} steps, {cores} threads"
    v = float(statistics.median(vals))
    return {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
            "solves_per_hour": v / (ntot * Nt) * 3600.0, "time_steps": Nt}


def run_reference(args):
    """The reference arm: the reference's own CPU code on this host's cores
    (the unmodified sources built in oracle/_ref), on the same workload and
    metric as the GPU arm.  Under torchrun only rank 0 runs."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    for _ in range(args.warmup):
        cpu_baseline(args.grid, budget_s=args.ref_seconds, ncycles=args.ncycles)
    vals = [cpu_baseline(args.grid, budget_s=args.ref_seconds, ncycles=args.ncycles) for _ in range(args.steps)]
    v = statistics.median([x["value"] for x in vals])
    cb = dict(vals[-1])
    cb["value"] = v
    Nt = cb["time_steps"]
    ntot = args.grid * args.grid
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(args.grid, Nt, args.ncycles, "cos4"),
            "solves_per_hour": v / (ntot * Nt) * 3600.0,
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=600)
    ap.add_argument("--ncycles", type=float, default=8.0)
    ap.add_argument("--env", default="cos4", choices=["cos4", "sin2"],
                    help="pulse envelope; cos4 is the twin the unmodified reference can run (same duration)")
    ap.add_argument("--tile-k", dest="tile_k", type=int, default=0)
    ap.add_argument("--kpt", type=int, default=0)
    ap.add_argument("--steps-per-launch", dest="steps_per_launch", type=int, default=0)
    ap.add_argument("--cpu-seconds", dest="cpu_seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", dest="ref_seconds", type=float, default=6.0)
    ap.add_argument("--no-cpu-baseline", dest="no_cpu_baseline", action="store_true")
    ap.add_argument("--scan-solves", dest="scan_solves", type=int, default=256)
    ap.add_argument("--serve-requests", dest="serve_requests", type=int, default=2000)
    ap.add_argument("--serve-rate", dest="serve_rate", type=float, default=40.0)
    ap.add_argument("--lw-grid", dest="lw_grid", type=int, default=600)
    ap.add_argument("--wannier-grid", dest="wannier_grid", type=int, default=300)
    ap.add_argument("--wannier-cycles", dest="wannier_cycles", type=float, default=0.25)
    ap.add_argument("--wannier-seeds", dest="wannier_seeds", type=int, default=16)
    ap.add_argument("--wannier-fp64-seeds", dest="wannier_fp64_seeds", type=int, default=2)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
