"""bench.py on CPU: the roofline of the far-pair table kernel (the binding
ceiling, the larger of the table stream's and the multiply-adds' ideal
times, is reported as `bound`, with the other beside it), the timed window
(whole 16-step far blocks from the steady state, whatever --steps and
--warmup say) and the clock sampler's summary."""
import json
import sys

from tests.conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402

INFO = {"fused_step": 2}


def roof(alg_bytes, flops, avg_ms, hbm=6650.0, pipe_peak=35.0, mixed=False, variant=0):
    t = avg_ms / 1e3
    achieved = alg_bytes / t / 1e9
    pipe_tf = flops / t / 1e12
    kname = "far_kernel_mixed<5,false>" if mixed else bench.FAR_VARIANTS[variant]
    return bench.table_roofline(mixed, kname, variant, achieved, hbm, "fallback", alg_bytes, pipe_tf,
                                pipe_peak, flops, 16, avg_ms, 16 * avg_ms, 16 * avg_ms / 0.84, 16 * 0.0075, 16,
                                INFO)


def test_fp64_table_is_bound_by_the_multiply_adds():
    # N = 4096: 1.677 GB of table and 12.86 GFLOP per 16-step launch
    r = roof(1677312000, 12856762368, 0.686)
    assert r["bound"] == "fp64"
    assert r["unit"] == "TFLOP/s"
    assert abs(r["frac"] - r["fp64"]["frac"]) < 1e-12
    assert 0.5 < r["frac"] < 0.56
    assert 0.3 < r["hbm"]["frac"] < 0.4
    assert r["kernel"] == "far_kernel<5,false>"
    assert r["traffic"] is None  # DRAM bytes need a profiler: not measured in the run


def test_table_stream_bound_when_it_is_the_larger_ideal_time():
    # the same bytes with a tenth of the flops: the stream binds
    r = roof(1677312000, 1285676236, 0.3)
    assert r["bound"] == "hbm"
    assert r["unit"] == "GB/s"
    assert abs(r["frac"] - r["hbm"]["frac"]) < 1e-12


def test_mixed_table_reports_the_fp32_pipe():
    r = roof(1006387200, 12856762368, 0.479, pipe_peak=64.0, mixed=True)
    assert r["bound"] == "fp32" and "fp32" in r
    assert r["kernel"] == "far_kernel_mixed<5,false>"


def test_every_far_variant_has_a_kernel_name():
    for v in range(12):
        assert bench.FAR_VARIANTS[v].startswith("far_kernel")


def test_timed_window_is_whole_blocks_from_the_steady_state():
    # the driver's short run: 5 warm-up steps asked, 20 timed
    warm, timed = bench.main_window(bench.parse_args(["--steps", "20", "--warmup", "5"]))
    assert warm % 16 == 0 and timed % 16 == 0
    assert timed == 32
    assert warm >= 346 + 5 + 1  # largest delay bound of the 0.2 cube (0.2 sqrt(3) / 1e-3) + q + 1
    # no flags: the rest of the 20000-step run, whole blocks
    warm, timed = bench.main_window(bench.parse_args([]))
    assert warm + timed == 20000 and timed % 16 == 0
    # on the fly (0.5 cube, delays up to 866 steps)
    warm, timed = bench.main_window(bench.parse_args(["--workload", "otf"]))
    assert warm >= 866 + 6 and warm % 16 == 0 and timed == 32
    for w, s in [(0, 1), (3, 15), (16, 16), (17, 33), (400, 100)]:
        warm, timed = bench.aligned_window(w, s, 100)
        assert warm % 16 == 0 and warm >= max(w, 106) and timed % 16 == 0 and timed >= s


def test_sub_records_are_parsed():
    assert bench.parse_args([]).sub == ["mixed", "otf", "batched", "serving"]
    assert bench.parse_args(["--sub", "none"]).sub == []
    assert bench.parse_args(["--sub", "mixed,otf"]).sub == ["mixed", "otf"]


def test_clock_summary_flags_throttle_reasons():
    cs = bench.ClockSampler(0)
    cs.samples = [(1965.0, 1965.0, 0), (1900.0, 1965.0, 0x4), (1965.0, 1965.0, 0x40)]
    s = cs.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_reference_arm_does_not_load_the_gpu_library():
    """The reference arm times the reference's CPU path only: this
    repository's CUDA library must not be mapped into its process."""
    import subprocess
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--n', '128', '--cpu-steps', '1',"
            " '--cpu-t0', '40']; import bench; bench.main();"
            " maps = open('/proc/self/maps').read();"
            " print(json.dumps({'gpu_lib': 'libquest_gpu' in maps}))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    ref = [ln for ln in lines if ln.get("impl") == "reference"]
    assert ref and ref[0]["value"] > 0 and ref[0]["cpu_baseline"]["cores"] == 1
    assert lines[-1] == {"gpu_lib": False}
