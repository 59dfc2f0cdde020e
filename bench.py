"""Benchmark of the retarded-interaction time step on B200.

Workload (default): N = 4096 dots uniform in a centred 0.2 cube (seeded),
omega_0 ~ N(200, 0.5^2), T1 = T2 = 10, unit-random dipoles x 2e-3, Gaussian
pulse (15, 5, 1, 200, (200,0,0), (0,0,1)), c = 1, hbar = 1, mu0 = 1,
omega_L = 200, dt = 1e-3, 20000 steps, interpolation order 5, FP64 per-pair
coefficient table.  A "step" is one time step of the integrator: the pair sum
over all N(N-1)/2 pairs and 6 taps, then predictor + 11 evaluations + 10
corrections for every dot.

Metric: pair-updates/s = N^2 * steps / time (each ordered pair advanced one
step counts once; the reference evaluates the pair sum 11 times per step,
this implementation once plus the delay-0 terms per iteration, both credited
the same N^2 per step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload table|otf|batched|serving] [--precision fp64|mixed]

--workload otf: N = 65536 dots in a 0.5 cube (max delay ~860 steps), same
distributions, 5000-step run of which a bounded window is timed; the table
would need 215 GB, so the far-pair kernel computes the coefficients on the
fly.

For N > 1 (torchrun), every rank advances its own independent ensemble
(seed + rank) on its GPU: weak scaling, no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from quest_b200 import inputs as I  # noqa: E402

FALLBACK_HBM_GBS = 6650.0
TABLE_BYTES_PER_PAIR = lambda q: 4 + 16 * (q + 1)  # noqa: E731  int32 delay + (q+1) complex128
# FP64 flops of one on-the-fly coefficient evaluation (pair_coef_otf, q = 5):
# 6 reciprocals + node products and sums (~190), dyad scalars (~30), 6 taps
# of complex assembly (~90), sqrt / modf / sincos counted as ~40
OTF_COEF_FLOPS = 350
# Mixed precision (pair_coef_otf_mixed, q = 5): FP64 for the distance, the
# delay split, 1/r and the phase reduction (~80, sqrt and divisions counted
# as ~20 each); FP32 for the weights (6 nodes x (5 subtractions + 15 FMA of
# the symmetric-polynomial recurrence + 6 products) ~ 250), the dyad scalars
# (~35) and the 6 taps with their sum (~120)
OTF_COEF_FLOPS_MIXED = (80, 400)  # (FP64, FP32)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(name: str):
    """DRAM bytes per launch of the sweep kernel from the committed ncu
    summary (profiles/<name>.md, line 'traffic_bytes_per_launch: X')."""
    path = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"quest_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return None
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxs.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sms:
            return None
        return {"sm_mhz": float(np.median(sms)), "sm_max_mhz": float(max(maxs)), "reasons": sorted(reasons),
                "samples": len(sms)}


def workload(args, rank: int) -> I.Workload:
    if args.workload == "otf":
        return I.mixed_large(seed=3 + rank, n=args.n, steps=5000, pulse_delay=args.pulse_delay)
    wl = I.plain_table(seed=2 + rank, n=args.n, steps=args.warmup + args.steps, pulse_delay=args.pulse_delay)
    if args.dipole_scale != 1.0:
        wl.dots[:, 6:9] *= args.dipole_scale
    return wl


def fp64_peak_tflops(dtype="float64") -> float:
    """Dense throughput of this GPU in the given type, measured as the best
    of 5 cuBLAS GEMMs of 8192^3 (2 n^3 flops each), CUDA events; FP32 with
    TF32 disabled (CUDA-core FMA)."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    dt = torch.float64 if dtype == "float64" else torch.float32
    a = torch.randn(n, n, dtype=dt, device="cuda")
    b = torch.randn(n, n, dtype=dt, device="cuda")
    c = a @ b
    best = 1e30
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    torch.cuda.empty_cache()
    return 2 * n ** 3 / (best / 1e3) / 1e12


# far-pair kernel variants (qg_set_option "far_variant"; the first qg_run
# keeps the fastest of 0, 3, 5 and 6): kernel name and the ncu summary of
# its traffic
FAR_VARIANTS = {0: ("far_kernel<5,false>", "far_kernel_fp64_N4096"), 1: ("far_kernel_r4<5,false>", None),
                2: ("far_kernel_v2<5,false>", None), 3: ("far_kernel_async<5,false,0>", "far_kernel_async_fp64_N4096"),
                4: ("far_kernel_async<5,false,1>", None), 5: ("far_kernel_async<5,false,2>", None),
                6: ("far_kernel_async<5,false,3>", "far_kernel_async_pairs_fp64_N4096")}


def table_roofline(mixed, kname, variant, achieved, hbm, src, traffic, alg_bytes, pipe_tf, pipe_peak, flops, K,
                   avg_ms, pair_ms, ms, step_ms, launches, info):
    """Roofline of the far-pair table kernel.  Its two ceilings are the
    table stream (algorithmic bytes / HBM copy bandwidth) and the
    convolution's multiply-adds (flops / cuBLAS GEMM rate of the same type);
    the binding one (the larger ideal time) is reported as `bound`, the other
    beside it."""
    pipe = "fp32" if mixed else "fp64"
    t_hbm = alg_bytes / (hbm * 1e9)
    t_pipe = flops / (pipe_peak * 1e12)
    hbm_obj = {"achieved": achieved, "peak": hbm, "peak_source": src, "unit": "GB/s", "frac": achieved / hbm,
               "algorithmic_bytes_per_launch": alg_bytes}
    pipe_obj = {"achieved": pipe_tf, "peak": pipe_peak, "unit": "TFLOP/s", "frac": pipe_tf / pipe_peak,
                "flops_per_launch": flops,
                "peak_source": "measured here: best cuBLAS %s 8192^3" % ("SGEMM (no TF32)" if mixed else "DGEMM")}
    main = pipe_obj if t_pipe >= t_hbm else hbm_obj
    r = {"bound": pipe if t_pipe >= t_hbm else "hbm",
         "kernel": kname,
         "achieved": main["achieved"], "peak": main["peak"], "unit": main["unit"], "frac": main["frac"],
         "peak_source": main["peak_source"], "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
         "steps_per_launch": K, "avg_launch_ms": avg_ms,
         "share_of_timed_region": pair_ms / ms if ms > 0 else None,
         "step_kernels_ms_per_step": step_ms / max(launches * K, 1),
         "step_form": {0: "general (12 launches per step)", 1: "fused (1 launch per step)",
                       2: "block (1 cooperative launch per 16 steps)"}[info["fused_step"]],
         "far_variant": variant,
         "hbm": hbm_obj, pipe: pipe_obj}
    return r


def dist_setup(args, backend: str = "nccl"):
    """One process per GPU (torchrun): RANK / WORLD_SIZE / LOCAL_RANK from
    the environment; NCCL on GPUs, gloo for the CPU tests of this logic."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def _collective_device():
    import torch.distributed as dist
    return "cpu" if dist.get_backend() == "gloo" else "cuda"


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_collective_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, n: int, steps: int, ms_max: float) -> float:
    """Whole-job pair-updates/s: every rank advances its own N-dot ensemble
    `steps` steps; the job takes as long as the slowest rank."""
    return world * n * n * steps / (ms_max / 1e3)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(args, kind="port"):
    """The reference algorithm (faithful oracle: 11 full pair sweeps per step,
    single thread like the reference) on a bounded sample of the workload:
    `steps` steps from step t0 >= the largest delay on a synthetic history."""
    from oracle import oracle as O
    from quest_b200 import capi
    wl = I.plain_table(seed=2, n=args.n, steps=args.cpu_t0 + args.cpu_steps)
    c = wl.constants
    ps, cs, fc = capi.pc_weights()
    w = O.Weights(ps, cs, fc)
    delays, coefs = O.build_table(wl.dots, c)
    n = wl.n
    T = c.num_timesteps
    rng = np.random.default_rng(0)
    hist = np.zeros((n, T + O.WINDOW, 2, 2), dtype=np.complex128)
    hist[:, :, 0, 0] = 1.0
    hist[:, : args.cpu_t0 + O.WINDOW, 0, 1] = 1e-4 * (rng.normal(size=(n, args.cpu_t0 + O.WINDOW)) +
                                                     1j * rng.normal(size=(n, args.cpu_t0 + O.WINDOW)))
    t0 = time.perf_counter()
    done = O.faithful_steps(wl.dots, wl.pulse, c, w, T, delays, coefs, hist, args.cpu_t0, args.cpu_steps)
    dt = time.perf_counter() - t0
    value = n * n * done / dt
    return {"value": value, "unit": "pair-updates/s", "cores": 1, "kind": kind,
            "sample": f"N={n}, {done} faithful steps (11 full pair sweeps each) from step {args.cpu_t0} "
                      f"on a synthetic history, {dt:.2f} s; table build not timed"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    steps = max(1, min(args.steps, args.cpu_steps))
    a = argparse.Namespace(**vars(args))
    a.cpu_steps = steps
    if args.workload == "otf":
        # the reference needs the full table (215 GB at N = 65536): its CPU
        # rate is sampled on the table workload's size instead
        a.n = 4096
    base = cpu_baseline(a)
    line = {"impl": "reference", "metric": "pair-updates/s", "value": base["value"], "unit": "pair-updates/s",
            "n_gpus": world, "steps": steps, "warmup": 0, "ms_per_step": args.n * args.n / base["value"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict(args),
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "pair-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_dict(args):
    if args.workload == "otf":
        return {"workload": f"{args.precision}_otf_N{args.n}_T5000", "N": args.n, "steps_total": 5000,
                "steps_timed_window": [args.warmup, args.warmup + args.steps], "interpolation_order": 5,
                "side": 0.5, "dt": 1e-3, "c0": 1.0, "hbar": 1.0, "mu0": 1.0, "laser_frequency": 200.0,
                "pulse_delay": args.pulse_delay, "precision": args.precision, "coef_mode": "on_the_fly",
                "l2": "inputs larger than L2 (rho01 ring %.0f MB > 126 MB)" % (args.n * 906 * 16 / 1e6),
                "parallelism": "1 GPU"}
    return {"workload": f"{args.precision}_table_N{args.n}_T{args.warmup + args.steps}", "N": args.n,
            "steps_total": args.warmup + args.steps, "interpolation_order": 5, "side": 0.2,
            "dt": 1e-3, "c0": 1.0, "hbar": 1.0, "mu0": 1.0, "laser_frequency": 200.0,
            "pulse_delay": args.pulse_delay, "precision": args.precision, "coef_mode": "table",
            "l2": "inputs larger than L2 (coefficient table %.0f MB > 126 MB)" %
                  (args.n * (args.n - 1) / 2 * TABLE_BYTES_PER_PAIR(5) / 1e6),
            "parallelism": "independent ensemble per GPU" if int(os.environ.get("WORLD_SIZE", "1")) > 1
            else "1 GPU"}


def accuracy_vs_fp64(args, weights) -> dict:
    """Max relative error in rho of the mixed form against the FP64 form
    (which matches the oracle to 1e-10, tests/test_gpu_parity.py) on an
    excited, stable variant of the workload: dipoles x 0.1, pulse delay 0.3,
    700 steps (N = 4096 table) or 400 steps at N = 16384 in the 0.5 cube
    (on the fly).  max |d rho| / max |rho| per component."""
    from quest_b200 import capi
    otf = args.workload == "otf"
    if otf:
        wl = I.mixed_large(seed=3, n=16384, steps=400, pulse_delay=0.3)
        steps, cmode = 400, capi.COEF_ON_THE_FLY
    else:
        wl = I.plain_table(seed=2, n=args.n, steps=700, pulse_delay=0.3)
        steps, cmode = 700, capi.COEF_TABLE
    wl.dots[:, 6:9] *= 0.1
    out = {}
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=weights, precision=prec,
                             coef_mode=cmode) as sim:
            out[prec] = sim.run(steps)
    a, b = out[capi.PREC_FP64], out[capi.PREC_MIXED]
    err = [float(np.abs(a[..., k] - b[..., k]).max() / np.abs(a[..., k]).max()) for k in range(2)]
    return {"rho00": err[0], "rho01": err[1],
            "probe": f"N={wl.n}, {steps} steps, dipoles x0.1, pulse delay 0.3 ({'on the fly' if otf else 'table'})"}


def run_ours(args, world, rank, local):
    import torch

    from quest_b200 import capi
    torch.cuda.set_device(local)
    wl = workload(args, rank)
    n = wl.n
    total = args.warmup + args.steps
    weights = capi.pc_weights()

    # ---- device-resident throughput (value) and the sweep kernel's roofline
    nonfinite = None
    prec = capi.PREC_MIXED if args.precision == "mixed" else capi.PREC_FP64
    mixed_prec = args.precision == "mixed"
    otf = args.workload == "otf"
    cmode = capi.COEF_ON_THE_FLY if otf else capi.COEF_TABLE
    sim = capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=weights, precision=prec, coef_mode=cmode)
    info = sim.info()
    if args.far_variant is not None:
        sim.set_option("far_variant", args.far_variant)
    try:
        sim.run(args.warmup, record=False)
    except capi.NonFiniteError as e:
        nonfinite = e.step
    sim.set_option("profile", 1)
    sim.kernel_time(reset=True)
    stream = torch.cuda.ExternalStream(capi.lib().qg_stream(sim.h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        e0.record(stream)
        try:
            sim.run(args.steps, record=False)
        except capi.NonFiniteError as e:
            nonfinite = e.step if nonfinite is None else nonfinite
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    pair_ms, launches, step_ms, step_launches = sim.kernel_times()
    variant = sim.get_option("far_variant") if not (mixed_prec or otf) else None  # FP64 table only
    sim.close()
    ms_max = max_over_ranks(ms, world)
    value = job_throughput(world, n, args.steps, ms_max)

    # ---- end to end through the C ABI with host buffers: create (dots
    # upload + table build), every step's rho (N x 2 complex) copied back
    rho_host = np.empty((total, n, 2), dtype=np.complex128)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=weights, precision=prec,
                         coef_mode=cmode) as sim2:
        if args.far_variant is not None:
            sim2.set_option("far_variant", args.far_variant)
        try:
            sim2.run(total, out=rho_host)
        except capi.NonFiniteError:
            pass
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    e2e_value = world * n * n * total / e2e_s

    hbm, src = peaks()
    q = 5
    K = info["time_block"]
    mixed = args.precision == "mixed"
    # the table holds every ordered pair (each unordered pair twice) and one
    # launch streams it once for K steps; mixed: q+1 complex64 taps + their sum
    per_pair = (4 + 8 * (q + 2)) if mixed else TABLE_BYTES_PER_PAIR(q)
    alg_bytes = 2 * info["num_pairs"] * per_pair
    far_ordered = 2 * (info["num_pairs"] - info["mid_pairs"])
    flops = far_ordered * K * (q + 1) * 8  # complex multiply-add = 4 FMA = 8 flops
    avg_ms = pair_ms / max(launches, 1)
    achieved = alg_bytes / (avg_ms / 1e3) / 1e9
    fp64_tf = flops / (avg_ms / 1e3) / 1e12
    fp64_peak = fp64_peak_tflops("float32" if mixed else "float64")
    # ncu dram read + write per launch of the same kernel on the same workload
    kname, prof = (("far_kernel_mixed<5,false>", "far_kernel_mixed_N4096") if mixed else
                   FAR_VARIANTS[variant] if variant is not None else (None, None))
    traffic = profile_traffic(prof) if prof else None
    if otf:
        # compute-bound: every ordered pair's coefficients once per launch
        # (FP64; in mixed precision mostly FP32) plus the K-step convolution
        # (FP64, or FP32 in mixed)
        c64, c32 = OTF_COEF_FLOPS_MIXED if mixed else (OTF_COEF_FLOPS, 0)
        coef_flops = 2 * (info["num_pairs"]) * (c64 + c32)
        d_peak = fp64_peak if not mixed else fp64_peak_tflops("float64")
        t_s = avg_ms / 1e3
        # time-weighted peak: each kind of flop at its type's measured rate
        ideal_s = (2 * info["num_pairs"] * c64) / (d_peak * 1e12) + \
            (2 * info["num_pairs"] * c32 + flops) / (fp64_peak * 1e12)
        roof = {"bound": "fp64" if not mixed else "fp64+fp32", "kernel": "far_otf_kernel<5,false,%s>" %
                ("true" if mixed else "false"),
                "achieved": (coef_flops + flops) / t_s / 1e12, "unit": "TFLOP/s",
                "peak": (coef_flops + flops) / ideal_s / 1e12, "peak_source": "measured here: best cuBLAS "
                "DGEMM%s 8192^3" % (" and SGEMM (no TF32)" if mixed else ""),
                "frac": ideal_s / t_s, "traffic": None,
                "coef_flops_per_launch": coef_flops, "conv_flops_per_launch": flops,
                "coef_flops_per_pair": {"fp64": c64, "fp32": c32}, "steps_per_launch": K, "avg_launch_ms": avg_ms,
                "share_of_timed_region": pair_ms / ms if ms > 0 else None,
                "step_kernels_ms_per_step": step_ms / max(launches * K, 1),
                "step_form": {0: "general (12 launches per step)", 1: "fused (1 launch per step)",
                              2: "block (1 cooperative launch per 16 steps)"}[info["fused_step"]]}
    line = {
        "metric": "pair-updates/s", "value": value, "unit": "pair-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair sum + f64 state (mixed)" if mixed else "f64",
        "data": "synthetic (seeded dots and pulse of the stated distributions)",
        "config": config_dict(args),
        "roofline": roof if otf else table_roofline(mixed, kname, variant, achieved, hbm, src, traffic, alg_bytes,
                                                    fp64_tf, fp64_peak, flops, K, avg_ms, pair_ms, ms, step_ms,
                                                    launches, info),
        "e2e": {"value": e2e_value, "unit": "pair-updates/s", "seconds": e2e_s,
                "h2d_bytes_per_step": (n * 72 + 80) / total, "d2h_bytes_per_step": n * 32,
                "includes": "qg_create (dots upload + %s) + qg_run with every step's rho read back" %
                            ("max-delay and pair-list kernels" if otf else "table build")},
        "gpu_launches": launches + step_launches,
        "near_pairs": info["near_pairs"], "mid_pairs": info["mid_pairs"], "max_delay": info["max_delay"],
        "nonfinite_from_step": nonfinite,
        "table_build_ms": info["table_build_ms"],
    }
    cs = clocks.summary()
    if cs is not None:
        line["clocks"] = cs
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not otf:
        line["cpu_baseline"] = cpu_baseline(args)
    if mixed and rank == 0:
        line["max_rel_err_vs_fp64"] = accuracy_vs_fp64(args, weights)
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batched(args, world, rank, local):
    """The batched workload: independent ensembles, N log-uniform in
    [64, 4096], side U[0.05, 0.3], E_0 U[1, 30], steps U[2000, 20000],
    all in one batch (one persistent far-pair launch + 16 step launches per
    16-step block, replayed as a CUDA graph); finished ensembles are retired
    as they finish."""
    import torch

    from quest_b200 import capi, serving
    torch.cuda.set_device(local)
    reqs = serving.batched_ensembles(args.ensembles, seed=40 + rank)
    weights = capi.pc_weights()
    prec = capi.PREC_MIXED if args.precision == "mixed" else capi.PREC_FP64
    sims = [capi.Simulation(r.dots, r.pulse, r.constants, weights=weights, precision=prec) for r in reqs]
    batch = capi.Batch(len(sims))
    for s in sims:
        batch.add(s)
    total = sum(r.pair_updates for r in reqs)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    live = list(zip(reqs, sims))
    blocks = 0
    while live:
        batch.run(args.blocks_per_round)
        blocks += args.blocks_per_round
        done = [(r, s) for r, s in live if s.next_step >= r.constants.num_timesteps]
        for r, s in done:
            batch.remove(s)
        live = [(r, s) for r, s in live if s.next_step < r.constants.num_timesteps]
    torch.cuda.synchronize()
    wall = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    ns = np.array([r.n for r in reqs])
    line = {"metric": "pair-updates/s", "value": world * total / wall, "unit": "pair-updates/s",
            "n_gpus": world, "steps": int(blocks * 16), "warmup": 0, "ms_per_step": wall * 1e3 / (blocks * 16),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pair sum + f64 state (mixed)" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded ensembles)",
            "config": {"workload": f"batched_{args.ensembles}_ensembles", "ensembles": args.ensembles,
                       "N_min": int(ns.min()), "N_max": int(ns.max()), "sum_N2T": total,
                       "precision": args.precision, "coef_mode": "table"},
            "wall_s": wall}
    for s in sims:
        s.close()
    batch.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_serving(args, world, rank, local):
    """The serving workload: Poisson arrivals at --rate requests/s, N
    log-uniform in [32, --serve-nmax], side U[0.05, 0.5], steps U[1000,
    20000], admitted under a --budget-gb memory budget; p50/p99
    time-to-completion and aggregate pair-updates/s."""
    import torch

    from quest_b200 import capi, serving
    torch.cuda.set_device(local)
    rates = [float(r) for r in args.rate_sweep.split(",")] if args.rate_sweep else [args.rate]
    for rate in rates:
        reqs = serving.serving_requests(args.requests, rate, seed=70 + rank, n_range=(32, args.serve_nmax))
        srv = serving.Server(budget_bytes=args.budget_gb * 1e9, weights=capi.pc_weights(),
                             precision=capi.PREC_MIXED if args.precision == "mixed" else capi.PREC_FP64)
        barrier(world)
        stats = srv.serve(reqs)
        srv.close()
        stats["pair_updates_per_s"] = max_over_ranks(stats["pair_updates_per_s"], world)
        line = {"metric": "pair-updates/s", "value": world * stats["pair_updates_per_s"], "unit": "pair-updates/s",
                "n_gpus": world, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 pair sum + f64 state (mixed)" if args.precision == "mixed" else "f64",
                "data": "synthetic (seeded Poisson request stream)",
                "config": {"workload": "serving", "requests": args.requests, "rate_per_s": rate,
                           "N_max": args.serve_nmax, "budget_gb": args.budget_gb, "precision": args.precision},
                "serving": stats}
        if rank == 0:
            print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--pulse-delay", type=float, default=5.0)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--cpu-t0", type=int, default=400)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dipole-scale", type=float, default=1.0)
    ap.add_argument("--far-variant", type=int, default=None)
    ap.add_argument("--workload", choices=["table", "otf", "batched", "serving"], default="table")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--ensembles", type=int, default=256)
    ap.add_argument("--blocks-per-round", type=int, default=8)
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--rate-sweep", default="", help="comma-separated arrival rates (one line each)")
    ap.add_argument("--serve-nmax", type=int, default=16384)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    args = ap.parse_args()
    otf = args.workload == "otf"
    if args.n is None:
        args.n = 65536 if otf else 4096
    if args.steps is None:
        args.steps = 160 if otf else 19950
    if args.warmup is None:
        args.warmup = 16 if otf else 50
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "batched":
            run_batched(args, world, rank, local)
        elif args.workload == "serving":
            run_serving(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
