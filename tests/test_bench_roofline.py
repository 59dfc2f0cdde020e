"""bench.py's roofline of the far-pair table kernel, on CPU: the binding
ceiling (the larger of the table stream's and the multiply-adds' ideal
times) is reported as `bound`, with the other beside it, and each far
variant maps to its kernel name and committed ncu summary."""
import os
import sys

from tests.conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402

INFO = {"fused_step": 2}


def roof(alg_bytes, flops, avg_ms, hbm=6650.0, pipe_peak=35.0, mixed=False, variant=0):
    t = avg_ms / 1e3
    achieved = alg_bytes / t / 1e9
    pipe_tf = flops / t / 1e12
    kname, prof = ("far_kernel_mixed<5,false>", "far_kernel_mixed_N4096") if mixed else bench.FAR_VARIANTS[variant]
    return bench.table_roofline(mixed, kname, variant, achieved, hbm, "fallback", None, alg_bytes, pipe_tf,
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


def test_every_far_variant_has_a_kernel_name_and_existing_profiles():
    for v in range(7):
        name, prof = bench.FAR_VARIANTS[v]
        assert name.startswith("far_kernel")
        if prof is not None:
            assert os.path.exists(os.path.join(ROOT, "profiles", prof + ".md")), prof
            assert bench.profile_traffic(prof) is not None
