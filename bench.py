"""Benchmark of the retarded-interaction time step on B200.

Workload (default line): N = 4096 dots uniform in a centred 0.2 cube
(seeded), omega_0 ~ N(200, 0.5^2), T1 = T2 = 10, unit-random dipoles x 2e-3,
Gaussian pulse (15, 5, 1, 200, (200,0,0), (0,0,1)), c = 1, hbar = 1, mu0 = 1,
omega_L = 200, dt = 1e-3, 20000 steps, interpolation order 5, FP64 per-pair
coefficient table.  A "step" is one time step of the integrator: the pair sum
over all N(N-1)/2 pairs and 6 taps, then predictor + 11 evaluations + 10
corrections for every dot.

Metric: pair-updates/s = N^2 * steps / time (each ordered pair advanced one
step counts once; the reference evaluates the pair sum 11 times per step,
this implementation once plus the delay-0 terms per iteration, both credited
the same N^2 per step).

Timed window.  The far-pair kernel runs once per 16-step block and computes
the far field of all 16 steps of its block, so the warm-up and the timed
steps are whole blocks: the warm-up is rounded up to a multiple of 16 and to
at least the largest delay + q + 1 steps (from there on every tap of every
pair reads live history, the steady state), and the timed count is rounded
up to whole blocks.  The line reports the steps actually timed and checks
that the far launches inside the window are exactly one per 16 timed steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload table|otf|batched|serving] [--precision fp64|mixed]
                  [--sub mixed,otf,batched,serving | --sub none]

The default FP64 table line carries sub-records, each with its own clock
record: `mixed` (the same workload in mixed precision, with its max relative
error against FP64), `otf` (N = 65536 in a 0.5 cube, coefficients on the
fly, FP64 and mixed, with the mixed error at N = 65536), `batched` (256
ensembles, mixed) and `serving` (a Poisson request stream, FP64 and mixed,
p50/p99 time to completion).

For N > 1 (torchrun), every rank advances its own independent ensemble
(seed + rank) on its GPU: weak scaling, no data-path collective.  The
sub-records run on 1 GPU only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from quest_b200 import inputs as I  # noqa: E402

K_BLOCK = 16  # steps per far-pair launch (kTimeBlock in the library)
Q = 5
FALLBACK_HBM_GBS = 6650.0
GOLDEN_WEIGHTS = os.path.join(ROOT, "tests", "golden", "pc_weights_18_22_3.15.txt")
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
STEP_FORMS = {0: "general (12 launches per step)", 1: "fused (1 launch per step)",
              2: "block (1 cooperative launch per 16 steps)"}


def round_up(x: int, m: int) -> int:
    return -(-int(x) // m) * m


def aligned_window(warmup: int, steps: int, max_delay: int, q: int = Q) -> tuple[int, int]:
    """(warm-up steps, timed steps), both whole far blocks: the warm-up reaches
    the steady state (every tap live: step >= largest delay + q + 1)."""
    warm = round_up(max(int(warmup), 3, max_delay + q + 1), K_BLOCK)
    timed = round_up(max(int(steps), 1), K_BLOCK)
    return warm, timed


def load_weights():
    """The frozen predictor-corrector weights (18, 22, 3.15) from the golden
    table, shared by both arms (reading them needs no GPU library)."""
    return I.load_pc_weights(GOLDEN_WEIGHTS)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clocks and clock-event reasons sampled during a timed region.

    NVML is polled from a thread every `period` seconds (the library's calls
    release the GIL while the GPU works), so even a region of a few
    milliseconds gets samples; one sample is also taken when the region
    starts and one when it ends.  Falls back to `nvidia-smi -lms 200` when
    NVML is unavailable.  Reading clocks changes no setting."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, gpu_index: int, period: float = 0.002):
        self.gpu = gpu_index
        self.period = period
        self.samples: list[tuple[float, float, int]] = []
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None
        self._smi = None

    def _sample(self):
        nv, h = self._nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.samples.append((float(sm), float(mx), int(rs)))

    def _loop(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                return
            self._stop.wait(self.period)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            # CUDA and NVML may number devices differently: match by PCI bus id
            h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            try:
                import torch
                props = torch.cuda.get_device_properties(self.gpu)
                bus = "%08X:%02X:%02X.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
                h = nv.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                pass
            self._nvml = (nv, h)
            self._sample()
            self._thread = threading.Thread(target=self._loop, daemon=True)
            self._thread.start()
        except Exception:
            self._nvml = None
            self.path = os.path.join("/tmp", f"quest_clocks_{os.getpid()}.csv")
            try:
                self._f = open(self.path, "w")
                self._smi = subprocess.Popen(
                    ["nvidia-smi", f"--id={self.gpu}", "--query-gpu=clocks.sm,clocks.max.sm,"
                     "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                     "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                     "--format=csv,noheader,nounits", "-lms", "200"], stdout=self._f, stderr=subprocess.DEVNULL)
            except (OSError, FileNotFoundError):
                self._smi = None
        return self

    def __exit__(self, *exc):
        if self._nvml is not None:
            self._stop.set()
            self._thread.join(timeout=2)
            try:
                self._sample()
            except Exception:
                pass
        if self._smi is not None:
            self._smi.terminate()
            try:
                self._smi.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._smi.kill()
            self._f.close()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) < 6:
                    continue
                try:
                    bits = sum(self.REASONS[nm] for nm, v in zip(names, p[2:6]) if v.lower().startswith("active"))
                    self.samples.append((float(p[0]), float(p[1]), bits))
                except ValueError:
                    continue

    def summary(self):
        if not self.samples:
            return None
        sms = [s[0] for s in self.samples]
        reasons = sorted({nm for s in self.samples for nm, bit in self.REASONS.items() if s[2] & bit})
        return {"sm_mhz": float(np.median(sms)), "sm_max_mhz": float(max(s[1] for s in self.samples)),
                "reasons": reasons, "samples": len(sms), "source": "nvml" if self._nvml else "nvidia-smi"}


def fp_peak_tflops(dtype="float64") -> float:
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
# keeps the fastest of the timed candidates): kernel names as ncu lists them
FAR_VARIANTS = {0: "far_kernel<5,false>", 1: "far_kernel_r4<5,false>", 2: "far_kernel_v2<5,false>",
                3: "far_kernel_async<5,false,0>", 4: "far_kernel_async<5,false,1>",
                5: "far_kernel_async<5,false,2>", 6: "far_kernel_async<5,false,3>"}
# 7 and 8: kernels of 0 and 3 with the source-group-major task order
FAR_VARIANTS[7] = FAR_VARIANTS[0]
FAR_VARIANTS[8] = FAR_VARIANTS[3]
FAR_VARIANTS[9] = "far_kernel_bulk<5,false>"
FAR_VARIANTS[10] = FAR_VARIANTS[11] = "far_kernel_wstage<5,false>"
TRAFFIC_NOTE = ("DRAM bytes need a profiler capture; they are not measured inside this run (null). "
                "The committed ncu summaries of the same kernel give them.")


def table_roofline(mixed, kname, variant, achieved, hbm, src, alg_bytes, pipe_tf, pipe_peak, flops, K,
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
    return {"bound": pipe if t_pipe >= t_hbm else "hbm",
            "kernel": kname,
            "achieved": main["achieved"], "peak": main["peak"], "unit": main["unit"], "frac": main["frac"],
            "peak_source": main["peak_source"], "traffic": None, "traffic_note": TRAFFIC_NOTE,
            "algorithmic_bytes_per_launch": alg_bytes,
            "steps_per_launch": K, "avg_launch_ms": avg_ms,
            "share_of_timed_region": pair_ms / ms if ms > 0 else None,
            "step_kernels_ms_per_step": step_ms / max(launches * K, 1),
            "step_form": STEP_FORMS[info["fused_step"]],
            "far_variant": variant,
            "hbm": hbm_obj, pipe: pipe_obj}


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


# ---- CPU baselines -------------------------------------------------------------

def ref_library():
    """oracle/_ref/libquest_ref.so: the reference's own source files compiled
    by oracle/build_ref.sh (None when it was not built)."""
    try:
        from oracle import ref as R
    except ImportError:
        return None
    return R if R.available() else None


def cpu_baseline(args, n: int, steps: int):
    """The reference algorithm on a bounded sample of the table workload:
    `steps` integrator steps from step t0 >= the largest delay on a synthetic
    history.  Prefers the reference's own code (kind "reference": its src/
    files compiled as they are, single thread as the reference runs); else the
    faithful oracle port (kind "port": 11 full pair sweeps per step, single
    thread).  The table build is timed separately and not counted."""
    wl = I.plain_table(seed=2, n=n, steps=args.cpu_t0 + steps)
    c = wl.constants
    ps, cs, fc = load_weights()
    R = None if args.cpu_kind == "port" else ref_library()
    if R is not None:
        r = R.time_steps(wl.dots, wl.pulse, c, args.cpu_t0, steps, seed=0)
        value = n * n * r["steps"] / r["seconds"]
        return {"value": value, "unit": "pair-updates/s", "cores": 1, "kind": "reference",
                "sample": f"N={n}, {r['steps']} steps of the reference's Integrator::solve_step (its src/*.cpp "
                          f"compiled unmodified against this repository's Eigen/Boost subset) from step "
                          f"{args.cpu_t0} on a synthetic history, {r['seconds']:.2f} s; table build "
                          f"{r['table_seconds']:.1f} s not timed"}
    from oracle import oracle as O
    w = O.Weights(ps, cs, fc)
    delays, coefs = O.build_table(wl.dots, c)
    T = c.num_timesteps
    rng = np.random.default_rng(0)
    hist = np.zeros((n, T + O.WINDOW, 2, 2), dtype=np.complex128)
    hist[:, :, 0, 0] = 1.0
    hist[:, : args.cpu_t0 + O.WINDOW, 0, 1] = 1e-4 * (rng.normal(size=(n, args.cpu_t0 + O.WINDOW)) +
                                                     1j * rng.normal(size=(n, args.cpu_t0 + O.WINDOW)))
    t0 = time.perf_counter()
    done = O.faithful_steps(wl.dots, wl.pulse, c, w, T, delays, coefs, hist, args.cpu_t0, steps)
    dt = time.perf_counter() - t0
    return {"value": n * n * done / dt, "unit": "pair-updates/s", "cores": 1, "kind": "port",
            "sample": f"N={n}, {done} faithful oracle steps (11 full pair sweeps each) from step {args.cpu_t0} "
                      f"on a synthetic history, {dt:.2f} s; table build not timed"}


def workload(args, rank: int, total: int) -> I.Workload:
    """This rank's ensemble (seed + rank: every rank its own) for a run of
    `total` steps."""
    if args.workload == "otf":
        wl = I.mixed_large(seed=3 + rank, n=args.n, steps=max(5000, total), pulse_delay=args.pulse_delay)
    else:
        wl = I.plain_table(seed=2 + rank, n=args.n, steps=total, pulse_delay=args.pulse_delay)
    if args.dipole_scale != 1.0:
        wl.dots[:, 6:9] *= args.dipole_scale
    return wl


def main_window(args) -> tuple[int, int]:
    """The main line's aligned (warm-up, timed) steps; with no --steps the
    table workload times the rest of its 20000-step run."""
    otf = args.workload == "otf"
    probe = I.mixed_large(seed=3, n=args.n, steps=1) if otf else I.plain_table(seed=2, n=args.n, steps=1)
    warm, timed = aligned_window(args.warmup, args.steps or 1, I.max_delay_steps(probe.dots, 1.0, 1e-3))
    if not otf and args.steps is None:
        timed = max(K_BLOCK, (20000 - warm) // K_BLOCK * K_BLOCK)
    return warm, timed


def run_reference(args, world, rank):
    """The reference arm: the reference's CPU implementation of the step on
    this host, rank 0 only; the on-the-fly workload (whose table, 215 GB,
    the reference cannot build) is sampled at the table workload's size."""
    if rank != 0:
        return
    steps = max(1, min(args.steps if args.steps is not None else args.cpu_steps, args.cpu_steps))
    n = 4096 if args.workload == "otf" else args.n
    base = cpu_baseline(args, n, steps)
    line = {"impl": "reference", "metric": "pair-updates/s", "value": base["value"], "unit": "pair-updates/s",
            "n_gpus": world, "steps": steps, "warmup": 0, "ms_per_step": n * n / base["value"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict(args, *main_window(args)),
            "steps_note": "a bounded sample (a few seconds per reference step at N = 4096)",
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "pair-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_dict(args, warm, timed):
    if args.workload == "otf":
        return {"workload": f"{args.precision}_otf_N{args.n}_T5000", "N": args.n, "steps_total": 5000,
                "steps_timed_window": [warm, warm + timed], "interpolation_order": 5,
                "side": 0.5, "dt": 1e-3, "c0": 1.0, "hbar": 1.0, "mu0": 1.0, "laser_frequency": 200.0,
                "pulse_delay": args.pulse_delay, "precision": args.precision, "coef_mode": "on_the_fly",
                "l2": "inputs larger than L2 (rho01 ring %.0f MB > 126 MB)" % (args.n * 906 * 16 / 1e6),
                "parallelism": "1 GPU"}
    return {"workload": f"{args.precision}_table_N{args.n}_T{warm + timed}", "N": args.n,
            "steps_total": warm + timed, "steps_timed_window": [warm, warm + timed], "interpolation_order": 5,
            "side": 0.2, "dt": 1e-3, "c0": 1.0, "hbar": 1.0, "mu0": 1.0, "laser_frequency": 200.0,
            "pulse_delay": args.pulse_delay, "precision": args.precision, "coef_mode": "table",
            "l2": "inputs larger than L2 (coefficient table %.0f MB > 126 MB)" %
                  (args.n * (args.n - 1) / 2 * TABLE_BYTES_PER_PAIR(5) / 1e6),
            "parallelism": "independent ensemble per GPU" if int(os.environ.get("WORLD_SIZE", "1")) > 1
            else "1 GPU"}


# ---- device-timed runs ---------------------------------------------------------

def timed_run(sim, warm: int, timed: int, world: int) -> dict:
    """`warm` untimed steps, then `timed` steps between CUDA events on the
    handle's stream (barrier and synchronize on both sides), with the far and
    step kernels' device times and the clocks sampled inside the window."""
    import torch

    from quest_b200 import capi
    nonfinite = None
    # profiling on from the start: its graph instances (with event nodes) are
    # built during the warm-up, not inside the timed window
    sim.set_option("profile", 1)
    try:
        sim.run(warm, record=False)
    except capi.NonFiniteError as e:
        nonfinite = e.step
    sim.kernel_time(reset=True)
    stream = torch.cuda.ExternalStream(capi.lib().qg_stream(sim.h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        e0.record(stream)
        try:
            sim.run(timed, record=False)
        except capi.NonFiniteError as e:
            nonfinite = e.step if nonfinite is None else nonfinite
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    pair_ms, launches, step_ms, step_launches = sim.kernel_times()
    if launches * K_BLOCK != timed:
        raise RuntimeError(f"timed window holds {launches} far launches for {timed} steps: "
                           f"expected one per {K_BLOCK} steps")
    return {"ms": ms, "pair_ms": pair_ms, "launches": launches, "step_ms": step_ms,
            "step_launches": step_launches, "clocks": clocks.summary(), "nonfinite": nonfinite}


def accuracy_vs_fp64(weights, otf: bool, n: int) -> dict:
    """Max relative error in rho of the mixed form against the FP64 form
    (which matches the oracle to 1e-10 in the parity tests) on an excited,
    stable variant of the workload: dipoles x 0.1, pulse delay 0.3, 700 steps
    (table, N = 4096) or 400 steps (on the fly, at the bench's N).
    max |d rho| / max |rho| per component."""
    from quest_b200 import capi
    if otf:
        wl = I.mixed_large(seed=3, n=n, steps=400, pulse_delay=0.3)
        steps, cmode = 400, capi.COEF_ON_THE_FLY
    else:
        wl = I.plain_table(seed=2, n=n, steps=700, pulse_delay=0.3)
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


def otf_roofline(info, t: dict, mixed: bool, pipe_peak: float, fp64_peak: float) -> dict:
    """Compute-bound on-the-fly kernel: every ordered pair's coefficients
    once per launch (FP64; in mixed precision mostly FP32) plus the K-step
    convolution (FP64, or FP32 in mixed)."""
    K = info["time_block"]
    avg_ms = t["pair_ms"] / max(t["launches"], 1)
    conv = 2 * (info["num_pairs"] - info["mid_pairs"]) * K * (Q + 1) * 8
    c64, c32 = OTF_COEF_FLOPS_MIXED if mixed else (OTF_COEF_FLOPS, 0)
    coef_flops = 2 * info["num_pairs"] * (c64 + c32)
    t_s = avg_ms / 1e3
    # time-weighted peak: each kind of flop at its type's measured rate
    ideal_s = (2 * info["num_pairs"] * c64) / (fp64_peak * 1e12) + \
        (2 * info["num_pairs"] * c32 + conv) / (pipe_peak * 1e12)
    return {"bound": "fp64+fp32" if mixed else "fp64",
            "kernel": "far_otf_kernel<5,false,%s>" % ("true" if mixed else "false"),
            "achieved": (coef_flops + conv) / t_s / 1e12, "unit": "TFLOP/s",
            "peak": (coef_flops + conv) / ideal_s / 1e12,
            "peak_source": "measured here: best cuBLAS DGEMM%s 8192^3" % (" and SGEMM (no TF32)" if mixed else ""),
            "frac": ideal_s / t_s, "traffic": None, "traffic_note": TRAFFIC_NOTE,
            "coef_flops_per_launch": coef_flops, "conv_flops_per_launch": conv,
            "coef_flops_per_pair": {"fp64": c64, "fp32": c32}, "steps_per_launch": K, "avg_launch_ms": avg_ms,
            "share_of_timed_region": t["pair_ms"] / t["ms"] if t["ms"] > 0 else None,
            "step_kernels_ms_per_step": t["step_ms"] / max(t["launches"] * K, 1),
            "step_form": STEP_FORMS[info["fused_step"]]}


def run_ours(args, world, rank, local):
    import torch

    from quest_b200 import capi
    torch.cuda.set_device(local)
    otf = args.workload == "otf"
    mixed = args.precision == "mixed"
    n = args.n
    warm, timed = main_window(args)
    total = warm + timed
    wl = workload(args, rank, total)
    weights = load_weights()
    prec = capi.PREC_MIXED if mixed else capi.PREC_FP64
    cmode = capi.COEF_ON_THE_FLY if otf else capi.COEF_TABLE

    # ---- device-resident throughput (value) and the sweep kernel's roofline
    sim = capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=weights, precision=prec, coef_mode=cmode)
    info = sim.info()
    if args.far_variant is not None:
        sim.set_option("far_variant", args.far_variant)
    if args.tune_group and not otf:
        sim.set_option("tune_group", 1)
    t = timed_run(sim, warm, timed, world)
    variant = sim.get_option("far_variant") if not (mixed or otf) else None  # FP64 table only
    tuned = {k: sim.get_option(k) for k in ("far_group", "block_step")}
    sim.close()
    ms_max = max_over_ranks(t["ms"], world)
    value = job_throughput(world, n, timed, ms_max)

    # ---- end to end through the C ABI with host buffers: create (dots
    # upload + table build), every step's rho (N x 2 complex) copied back
    e2e_steps = total if not otf else warm + timed
    rho_host = np.empty((e2e_steps, n, 2), dtype=np.complex128) if not otf else None
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=weights, precision=prec,
                         coef_mode=cmode) as sim2:
        t_created = time.perf_counter()
        if args.far_variant is not None:
            sim2.set_option("far_variant", args.far_variant)
        if args.tune_group and not otf:
            sim2.set_option("tune_group", 1)
        try:
            if otf:
                # 65536 dots x 2 complex per step: read back the last block's states only
                sim2.run(e2e_steps - K_BLOCK, record=False)
                rho_host = np.empty((K_BLOCK, n, 2), dtype=np.complex128)
                sim2.run(K_BLOCK, out=rho_host)
            else:
                sim2.run(e2e_steps, out=rho_host)
        except capi.NonFiniteError:
            pass
        t_ran = time.perf_counter()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    e2e_value = world * n * n * e2e_steps / e2e_s
    d2h = (n * 32) if not otf else n * 32 * K_BLOCK / e2e_steps

    hbm, src = peaks()
    K = info["time_block"]
    pipe_peak = fp_peak_tflops("float32" if mixed else "float64")
    if otf:
        roof = otf_roofline(info, t, mixed, pipe_peak, fp_peak_tflops("float64") if mixed else pipe_peak)
    else:
        # the table holds every ordered pair (each unordered pair twice) and one
        # launch streams it once for K steps; mixed: q+1 complex64 taps + their sum
        per_pair = (4 + 8 * (Q + 2)) if mixed else TABLE_BYTES_PER_PAIR(Q)
        alg_bytes = 2 * info["num_pairs"] * per_pair
        flops = 2 * (info["num_pairs"] - info["mid_pairs"]) * K * (Q + 1) * 8  # complex FMA = 8 flops
        avg_ms = t["pair_ms"] / max(t["launches"], 1)
        kname = "far_kernel_mixed<5,false>" if mixed else FAR_VARIANTS.get(variant)
        roof = table_roofline(mixed, kname, variant, alg_bytes / (avg_ms / 1e3) / 1e9, hbm, src, alg_bytes,
                              flops / (avg_ms / 1e3) / 1e12, pipe_peak, flops, K, avg_ms, t["pair_ms"], t["ms"],
                              t["step_ms"], t["launches"], info)
    line = {
        "metric": "pair-updates/s", "value": value, "unit": "pair-updates/s", "n_gpus": world,
        "steps": timed, "warmup": warm, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "far_launches_timed": t["launches"], "ms_per_step": ms_max / timed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair sum + f64 state (mixed)" if mixed else "f64",
        "data": "synthetic (seeded dots and pulse of the stated distributions)",
        "config": config_dict(args, warm, timed),
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": "pair-updates/s", "seconds": e2e_s, "steps": e2e_steps,
                "create_s": t_created - t0, "run_s": t_ran - t_created,
                "h2d_bytes_per_step": (n * 72 + 80) / e2e_steps, "d2h_bytes_per_step": d2h,
                "includes": "qg_create (dots upload + %s) + qg_run with %s rho read back" %
                            ("max-delay and pair-list kernels" if otf else "table build",
                             "the last block's" if otf else "every step's")},
        "gpu_launches": t["launches"] + t["step_launches"],
        "autotuned": dict(tuned, far_variant=variant),
        "near_pairs": info["near_pairs"], "mid_pairs": info["mid_pairs"], "max_delay": info["max_delay"],
        "nonfinite_from_step": t["nonfinite"],
        "table_build_ms": info["table_build_ms"],
    }
    if t["clocks"] is not None:
        line["clocks"] = t["clocks"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not otf:
        line["cpu_baseline"] = cpu_baseline(args, n, args.cpu_steps)
    if mixed and rank == 0:
        line["max_rel_err_vs_fp64"] = accuracy_vs_fp64(weights, otf, n)
    if world == 1 and not otf and not mixed:
        for name in args.sub:
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            try:
                line[name] = SUB_RECORDS[name](args, weights)
            except Exception as e:  # a failed sub-record is reported, not hidden
                line[name] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---- sub-records of the default line (1 GPU) -------------------------------------

def sub_mixed(args, weights) -> dict:
    """The same N = 4096 table workload in mixed precision, same window."""
    import torch

    from quest_b200 import capi
    wl = I.plain_table(seed=2, n=args.n, steps=1)
    warm, timed = aligned_window(args.warmup, max(args.steps or 0, 1024), I.max_delay_steps(wl.dots, 1.0, 1e-3))
    wl = I.plain_table(seed=2, n=args.n, steps=warm + timed, pulse_delay=args.pulse_delay)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=weights, precision=capi.PREC_MIXED,
                         coef_mode=capi.COEF_TABLE) as sim:
        info = sim.info()
        if args.tune_group:
            sim.set_option("tune_group", 1)
        t = timed_run(sim, warm, timed, 1)
        group = sim.get_option("far_group")
    torch.cuda.synchronize()
    avg_ms = t["pair_ms"] / max(t["launches"], 1)
    flops = 2 * (info["num_pairs"] - info["mid_pairs"]) * K_BLOCK * (Q + 1) * 8
    sgemm = fp_peak_tflops("float32")
    return {"workload": f"mixed_table_N{args.n}", "value": args.n ** 2 * timed / (t["ms"] / 1e3),
            "unit": "pair-updates/s", "steps": timed, "warmup": warm, "ms_per_step": t["ms"] / timed,
            "far_avg_launch_ms": avg_ms, "fp32_tflops": flops / (avg_ms / 1e3) / 1e12, "fp32_peak_tflops": sgemm,
            "fp32_frac": flops / (avg_ms / 1e3) / 1e12 / sgemm,
            "step_kernels_ms_per_step": t["step_ms"] / timed, "far_group": group,
            "gpu_launches": t["launches"] + t["step_launches"],
            "max_rel_err_vs_fp64": accuracy_vs_fp64(weights, False, args.n), "clocks": t["clocks"]}


def sub_otf(args, weights) -> dict:
    """N = 65536 dots in a 0.5 cube, coefficients on the fly: FP64 and mixed,
    each timed over `--otf-blocks` blocks after a steady-state warm-up, and the
    mixed form's error against FP64 at the same N."""
    import torch

    from quest_b200 import capi
    n = args.otf_n
    probe = I.mixed_large(seed=3, n=n, steps=1)
    warm, timed = aligned_window(0, K_BLOCK * args.otf_blocks, I.max_delay_steps(probe.dots, 1.0, 1e-3))
    wl = I.mixed_large(seed=3, n=n, steps=5000, pulse_delay=args.pulse_delay)
    out = {"workload": f"otf_N{n}_T5000", "N": n, "steps": timed, "warmup": warm}
    dgemm = fp_peak_tflops("float64")
    sgemm = fp_peak_tflops("float32")
    for name, prec in (("fp64", capi.PREC_FP64), ("mixed", capi.PREC_MIXED)):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=weights, precision=prec,
                             coef_mode=capi.COEF_ON_THE_FLY) as sim:
            info = sim.info()
            t = timed_run(sim, warm, timed, 1)
        torch.cuda.synchronize()
        mixed = prec == capi.PREC_MIXED
        out[name] = {"value": n * n * timed / (t["ms"] / 1e3), "unit": "pair-updates/s",
                     "ms_per_step": t["ms"] / timed,
                     "roofline": otf_roofline(info, t, mixed, sgemm if mixed else dgemm, dgemm),
                     "gpu_launches": t["launches"] + t["step_launches"], "clocks": t["clocks"],
                     "max_delay": info["max_delay"]}
    out["mixed"]["max_rel_err_vs_fp64"] = accuracy_vs_fp64(weights, True, n)
    return out


def sub_batched(args, weights) -> dict:
    r = batched_record(args, 1, 0, capi_precision="mixed", weights=weights)
    return r


def sub_serving(args, weights) -> dict:
    out = {}
    for prec in ("fp64", "mixed"):
        out[prec] = serving_record(args, 1, 0, prec, args.rate, weights)
    return out


SUB_RECORDS = {"mixed": sub_mixed, "otf": sub_otf, "batched": sub_batched, "serving": sub_serving}


def batched_record(args, world, rank, capi_precision, weights) -> dict:
    """The batched workload: independent ensembles, N log-uniform in
    [64, 4096], side U[0.05, 0.3], E_0 U[1, 30], steps U[2000, 20000],
    all in one batch (one persistent far-pair launch + the step launches per
    16-step block, replayed as a CUDA graph); finished ensembles are retired
    as they finish.  Unless --no-batch-tune-group, the batch's first run
    also times source tiles per far warp for each member size class (the
    choice is in the record).  Wall time of the whole job (all members to
    their last step, the tuning included), pair-updates = sum of N^2 x
    steps."""
    import torch

    from quest_b200 import capi, serving
    reqs = serving.batched_ensembles(args.ensembles, seed=40 + rank)
    prec = capi.PREC_MIXED if capi_precision == "mixed" else capi.PREC_FP64
    sims = [capi.Simulation(r.dots, r.pulse, r.constants, weights=weights, precision=prec) for r in reqs]
    batch = capi.Batch(len(sims))
    if args.batch_tune_group:
        batch.set_option("tune_group", 1)
    for s in sims:
        batch.add(s)
    total = sum(r.pair_updates for r in reqs)
    torch.cuda.synchronize()
    barrier(world)
    with ClockSampler(torch.cuda.current_device(), period=0.05) as clocks:
        t0 = time.perf_counter()
        live = list(zip(reqs, sims))
        blocks = 0
        nonfinite = 0
        while live:
            batch.run(args.blocks_per_round)
            if blocks == 0:
                tuned = {"tuned_far_us": batch.get_option("tuned_far_us"),
                         "far_packed": batch.get_option("far_packed"),
                         "far_gmajor": batch.get_option("far_gmajor"),
                         "tune_group": batch.get_option("tune_group"),
                         "far_group_class": [batch.get_option(f"far_group_class{c}") for c in range(4)]}
            blocks += args.blocks_per_round
            for r, s in [(r, s) for r, s in live if s.next_step >= r.constants.num_timesteps]:
                nonfinite += s.bad_step() >= 0
                batch.remove(s)
            live = [(r, s) for r, s in live if s.next_step < r.constants.num_timesteps]
        torch.cuda.synchronize()
        wall = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    ns = np.array([r.n for r in reqs])
    for s in sims:
        s.close()
    batch.close()
    return {"workload": f"batched_{args.ensembles}_ensembles", "value": world * total / wall,
            "unit": "pair-updates/s", "precision": capi_precision, "wall_s": wall, "blocks": blocks,
            "ensembles": args.ensembles, "N_min": int(ns.min()), "N_max": int(ns.max()), "sum_N2T": total,
            "timing": "wall clock of the whole batch (graph replays, membership changes, retirement)",
            "nonfinite_members": int(nonfinite), "autotuned": tuned,
            "nonfinite_note": "members whose state overflowed (the reference's domain_error) still run every step: "
                              "the work per step does not depend on the values",
            "clocks": clocks.summary()}


def serving_record(args, world, rank, precision: str, rate: float, weights) -> dict:
    """Poisson arrivals at `rate` requests/s, N log-uniform in [32,
    --serve-nmax], side U[0.05, 0.5], steps U[1000, 20000], admitted under a
    --budget-gb memory budget; p50/p99 time-to-completion and aggregate
    pair-updates/s."""
    import torch

    from quest_b200 import capi, serving
    reqs = serving.serving_requests(args.requests, rate, seed=70 + rank, n_range=(32, args.serve_nmax))
    srv = serving.Server(budget_bytes=args.budget_gb * 1e9, weights=weights,
                         precision=capi.PREC_MIXED if precision == "mixed" else capi.PREC_FP64,
                         tune_group=args.serve_tune_group)
    barrier(world)
    with ClockSampler(torch.cuda.current_device(), period=0.05) as clocks:
        stats = srv.serve(reqs)
    srv.close()
    stats["pair_updates_per_s"] = max_over_ranks(stats["pair_updates_per_s"], world)
    return {"workload": "serving", "value": world * stats["pair_updates_per_s"], "unit": "pair-updates/s",
            "precision": precision, "requests": args.requests, "rate_per_s": rate, "N_max": args.serve_nmax,
            "budget_gb": args.budget_gb, "serving": stats, "clocks": clocks.summary()}


def run_batched(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    r = batched_record(args, world, rank, args.precision, load_weights())
    line = {"metric": "pair-updates/s", "value": r["value"], "unit": "pair-updates/s",
            "n_gpus": world, "steps": int(r["blocks"] * K_BLOCK), "warmup": 0,
            "ms_per_step": r["wall_s"] * 1e3 / (r["blocks"] * K_BLOCK),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pair sum + f64 state (mixed)" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded ensembles)",
            "config": {"workload": r["workload"], "ensembles": args.ensembles, "N_min": r["N_min"],
                       "N_max": r["N_max"], "sum_N2T": r["sum_N2T"], "precision": args.precision,
                       "coef_mode": "table"},
            "wall_s": r["wall_s"], "autotuned": r.get("autotuned"), "clocks": r["clocks"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_serving(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    rates = [float(r) for r in args.rate_sweep.split(",")] if args.rate_sweep else [args.rate]
    for rate in rates:
        r = serving_record(args, world, rank, args.precision, rate, load_weights())
        line = {"metric": "pair-updates/s", "value": r["value"], "unit": "pair-updates/s",
                "n_gpus": world, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 pair sum + f64 state (mixed)" if args.precision == "mixed" else "f64",
                "data": "synthetic (seeded Poisson request stream)",
                "config": {"workload": "serving", "requests": args.requests, "rate_per_s": rate,
                           "N_max": args.serve_nmax, "budget_gb": args.budget_gb, "precision": args.precision},
                "serving": r["serving"], "clocks": r["clocks"]}
        if rank == 0:
            print(json.dumps(line), flush=True)


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--pulse-delay", type=float, default=5.0)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--cpu-t0", type=int, default=400)
    ap.add_argument("--cpu-kind", choices=["auto", "port"], default="auto",
                    help="auto: the reference's own code when oracle/_ref is built, else the oracle port")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dipole-scale", type=float, default=1.0)
    ap.add_argument("--far-variant", type=int, default=None)
    ap.add_argument("--workload", choices=["table", "otf", "batched", "serving"], default="table")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--sub", default="mixed,otf,batched,serving",
                    help="sub-records of the default FP64 table line ('none' for none)")
    ap.add_argument("--otf-n", type=int, default=65536)
    ap.add_argument("--otf-blocks", type=int, default=2)
    ap.add_argument("--ensembles", type=int, default=256)
    ap.add_argument("--tune-group", action="store_true",
                    help="table workloads: let the autotuner also pick source tiles per far warp")
    ap.add_argument("--no-batch-tune-group", dest="batch_tune_group", action="store_false",
                    help="batched workload: keep every member's own source tiles per far warp (by default the "
                         "batch tuner picks them per size class; members then equal solo runs with that group)")
    ap.add_argument("--serve-tune-group", action="store_true",
                    help="serving workload: the batch tuner's group search at the service's first run")
    ap.add_argument("--blocks-per-round", type=int, default=8)
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--rate-sweep", default="", help="comma-separated arrival rates (one line each)")
    ap.add_argument("--serve-nmax", type=int, default=16384)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    args = ap.parse_args(argv)
    if args.n is None:
        args.n = 65536 if args.workload == "otf" else 4096
    if args.workload == "otf" and args.steps is None:
        args.steps = 2 * K_BLOCK
    args.sub = [] if args.sub in ("", "none") else [s for s in args.sub.split(",") if s]
    for s in args.sub:
        if s not in SUB_RECORDS:
            ap.error(f"unknown sub-record {s!r}")
    return args


def main():
    args = parse_args()
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
