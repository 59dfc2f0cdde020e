"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Tolerance: max |rho_gpu - rho_oracle| / max |rho_oracle|, per component
(rho00 and rho01 separately), must be <= 1e-10 for the FP64 path.

The GPU sums the pair terms in a different order than the reference (far
pairs K steps at a time, tile by tile), so bitwise equality is not expected.
With interpolation order 5 or 7 the reference's scheme amplifies
rounding-level differences exponentially once the dots are excited (about x10
every 25 steps at dt = 1e-3 in a 0.2 cube): two summation orders of the
oracle itself drift apart the same way, and the run eventually overflows.
Each test therefore stops at a horizon where the oracle's own sensitivity to
summation order (1 vs 7 threads) is at most ~1e-12, so the 1e-10 bound
measures the GPU path and not the instability.  Orders 1 and 3 and the lab
frame are stable and are compared over their whole runs.  The step at which
the overflow happens is compared separately.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from quest_b200 import capi, inputs as I
from tests.conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10


def gpu_run(dots, pulse, c, weights, steps=None, **kw):
    steps = c.num_timesteps if steps is None else steps
    with capi.Simulation(dots, pulse, c, weights=weights, **kw) as sim:
        rho = sim.run(steps)
        info = sim.info()
    return rho, info


def assert_parity(ref_hist, rho, tol=TOL):
    ref = O.rho_trajectory(ref_hist)[: rho.shape[0]]
    e00 = rel_err(ref[..., 0], rho[..., 0])
    e01 = rel_err(ref[..., 1], rho[..., 1])
    assert e00 <= tol and e01 <= tol, (e00, e01)
    return e00, e01


def load_example(n=None, steps=None):
    c, n_cfg, _, _ = I.read_input_cfg(os.path.join(GOLDEN, "example_input.cfg"))
    n = n_cfg if n is None else n
    dots = I.read_dots_cfg(os.path.join(GOLDEN, "example_dots.cfg"), n)
    pulse = I.read_pulse_cfg(os.path.join(GOLDEN, "example_pulse.cfg"))
    if steps is not None:
        c.num_timesteps = steps
    return dots, pulse, c


def test_small_against_faithful_oracle(golden_weights, oracle_weights):
    wl = I.plain_small(n=60, steps=350, pulse_delay=0.2)
    hist, bad = O.run_faithful(wl.dots, wl.pulse, wl.constants, oracle_weights, 350)
    assert bad is None
    rho, info = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    assert info["fused_step"] == 2
    assert_parity(hist, rho)
    assert np.abs(rho[..., 1]).max() > 1e-6


def test_plain_small_delay_half(golden_weights, oracle_weights):
    """N=200, 0.2 cube, order 5, pulse delay 0.5 (the stated delay 5 never
    reaches the dots before t = 2), compared until step 520."""
    wl = I.plain_small(n=200, steps=520, pulse_delay=0.5)
    hist, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 520)
    assert bad is None
    rho, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    assert_parity(hist, rho)


def test_plain_small_overflows_where_the_oracle_does(golden_weights, oracle_weights):
    """The same run continued: the reference's scheme overflows about 400
    steps after the pulse and throws std::domain_error.  By then two valid
    summation orders of the oracle differ by ~10% (802 with one and seven
    threads, 803 with sixteen), so the GPU's first non-finite step is
    compared within 10 steps."""
    wl = I.plain_small(n=200, steps=900, pulse_delay=0.5)
    _, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 900)
    assert bad is not None and 700 < bad < 900
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        with pytest.raises(capi.NonFiniteError) as e:
            sim.run(900)
    assert abs(e.value.step - bad) <= 10, (e.value.step, bad)


def test_cfg2_stated_parameters_until_the_overflow(golden_weights, oracle_weights):
    """cfg 2 as stated (N = 4096 in the 0.2 cube, omega_0 jittered, unit-random
    dipoles x 2e-3, FP64 table), with the pulse moved from delay 5 to 0.1: up
    to the pulse's arrival the state is exactly the ground state, so this is
    the stated run from step ~4900 on.  Its dots are excited at once and the
    reference's scheme overflows 24 steps later (the whole stated run at
    delay 5 overflows at step 4958); two summation orders of the oracle agree
    to 1e-15 until then.  The GPU must match the oracle to 1e-10 on every step
    before the overflow and report the same first non-finite step."""
    T = 30
    wl = I.plain_table(seed=2, n=4096, steps=T, pulse_delay=0.1)
    hist, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, T)
    assert bad == 24
    ref = O.rho_trajectory(hist)[:bad]
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights,
                         coef_mode=capi.COEF_TABLE) as sim:
        got = sim.run(bad)
        assert np.abs(got[..., 1]).max() > 0.1  # strongly excited
        for k in range(2):
            assert rel_err(ref[..., k], got[..., k]) <= 1e-10
        with pytest.raises(capi.NonFiniteError) as e:
            sim.run(T - bad)
    assert e.value.step == bad


def test_plain_small_as_stated_stays_in_ground_state(golden_weights, oracle_weights):
    wl = I.plain_small(n=200, steps=2000, pulse_delay=5.0)
    rho, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    hist, _ = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 2000)
    ref = O.rho_trajectory(hist)
    np.testing.assert_allclose(rho[..., 0], ref[..., 0], rtol=0, atol=1e-13)
    assert np.abs(rho[..., 1]).max() < 1e-13
    assert np.abs(rho[..., 0] - 1).max() < 1e-12


def test_reference_example_two_dots(golden_weights, oracle_weights):
    """examples/ verbatim: N=2, order 3, 4000 steps, the pair at delay 0."""
    dots, pulse, c = load_example()
    hist, bad = O.run_faithful(dots, pulse, c, oracle_weights, c.num_timesteps)
    assert bad is None
    rho, info = gpu_run(dots, pulse, c, golden_weights)
    assert info["near_pairs"] == 1 and info["fused_step"] == 2
    assert_parity(hist, rho)


def test_reference_example_all_pairs_near(golden_weights, oracle_weights):
    """examples/ with 256 dots: every pair at delay 0, coupled in every
    corrector iteration; the group exceeds one block, so the general
    (one launch per evaluation) form runs."""
    dots, pulse, c = load_example(n=256, steps=1150)
    hist, bad = O.run_fast(dots, pulse, c, oracle_weights, 1150)
    assert bad is None
    rho, info = gpu_run(dots, pulse, c, golden_weights)
    assert info["fused_step"] == 0 and info["near_pairs"] == 256 * 255 // 2
    assert_parity(hist, rho)


def near_group_workload(steps=400):
    """N=300 with 12 planted pairs and one triple closer than c dt (delay 0),
    dipoles 2e-4 (weak enough that order 5 stays stable with them)."""
    wl = I.plain_small(n=300, steps=steps, pulse_delay=0.15)
    d = wl.dots
    d[:, 8] = 2e-4
    rng = np.random.default_rng(1)
    for k in range(12):
        v = rng.normal(size=3)
        d[2 * k + 1, :3] = d[2 * k, :3] + 8e-4 * v / np.linalg.norm(v)
    d[30, :3] = d[28, :3] + 8e-4 * np.array([0, 1.0, 0])
    d[29, :3] = d[28, :3] + 8e-4 * np.array([1.0, 0, 0])
    return wl


def test_small_near_groups_fused(golden_weights, oracle_weights):
    """Delay-0 pairs in an otherwise retarded system: the fused kernel with
    the coupled groups packed into blocks, iterated with the correctors."""
    wl = near_group_workload()
    hist, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 400)
    assert bad is None
    rho, info = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    assert info["near_pairs"] >= 14 and info["fused_step"] == 2
    assert_parity(hist, rho)


@pytest.mark.parametrize("q,steps", [(1, 300), (3, 300), (7, 200)])
def test_interpolation_orders(golden_weights, oracle_weights, q, steps):
    wl = I.plain_small(n=90, steps=steps, pulse_delay=0.15)
    wl.constants.interpolation_order = q
    hist, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, steps)
    assert bad is None
    rho, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    assert_parity(hist, rho)


def test_lab_frame(golden_weights, oracle_weights):
    """GreenFunction::Dyadic (green_function.cpp:3-20) with prefactor 2 Re rho01."""
    wl = I.plain_small(n=64, steps=300, pulse_delay=0.15)
    wl.constants.frame = 1
    hist, bad = O.run_faithful(wl.dots, wl.pulse, wl.constants, oracle_weights, 300)
    assert bad is None
    rho, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    assert_parity(hist, rho)


def test_default_weights_are_the_golden_ones(oracle_weights):
    wl = I.plain_small(n=40, steps=200, pulse_delay=0.1)
    hist, _ = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 200)
    rho, _ = gpu_run(wl.dots, wl.pulse, wl.constants, None)
    assert_parity(hist, rho)


def test_history_evaluate_matches_reference_sum(golden_weights):
    """HistoryInteraction::evaluate on an arbitrary history, all steps."""
    wl = I.plain_small(n=150, steps=400)
    c = wl.constants
    n = wl.n
    rng = np.random.default_rng(5)
    T = 400
    hist = np.zeros((n, T + O.WINDOW, 2, 2), dtype=np.complex128)
    hist[:, :, 0, 1] = rng.normal(size=(n, T + O.WINDOW)) + 1j * rng.normal(size=(n, T + O.WINDOW))
    delays, coefs = O.build_table(wl.dots, c)
    with capi.Simulation(wl.dots, wl.pulse, c, weights=golden_weights) as sim:
        W = sim.info()["ring_depth"]
        for step in [0, 5, 60, 250, 399]:
            lo = max(-O.WINDOW, step - W + 1)
            sim.set_history(lo, hist[:, lo + O.WINDOW: step + O.WINDOW, 0, 1].T)
            got = sim.history_evaluate(step, hist[:, step + O.WINDOW, 0, 1])
            ref = O.history_evaluate(wl.dots, c, delays, coefs, hist, step)
            assert rel_err(ref, got) < 1e-12, step
            # a second call at the same step re-uses the past sum
            got2 = sim.history_evaluate(step, hist[:, step + O.WINDOW, 0, 1] * 0.5)
            hist2 = hist.copy()
            hist2[:, step + O.WINDOW, 0, 1] *= 0.5
            ref2 = O.history_evaluate(wl.dots, c, delays, coefs, hist2, step)
            assert rel_err(ref2, got2) < 1e-12, step


def test_pulse_evaluate(golden_weights):
    wl = I.plain_small(n=50, steps=10, pulse_delay=0.0)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        for step in [0, 3, 9]:
            # same operations; CUDA's exp and glibc's differ by at most 1 ulp
            np.testing.assert_allclose(sim.pulse_evaluate(step),
                                       O.pulse_evaluate(wl.dots, wl.pulse, wl.constants, step),
                                       rtol=4.5e-16, atol=0)


def stable_small(n, steps, pulse_delay):
    """Dipoles 2e-4: weak enough coupling that the reference's order-5 scheme
    stays stable over the whole run (at 2e-3 it overflows a few hundred steps
    after the pulse, at any order once close pairs are present), for tests
    that compare whole runs with each other."""
    wl = I.plain_small(n=n, steps=steps, pulse_delay=pulse_delay)
    wl.dots[:, 8] = 2e-4
    return wl


def test_run_in_pieces_equals_one_run(golden_weights):
    wl = stable_small(100, 600, 0.1)
    a, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        parts = [sim.run(k) for k in (1, 99, 300, 200)]
        assert sim.next_step == 600
    np.testing.assert_array_equal(a, np.concatenate(parts))


def test_deterministic(golden_weights):
    wl = stable_small(333, 300, 0.1)
    a, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    b, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    np.testing.assert_array_equal(a, b)


def test_graph_and_direct_launches_agree(golden_weights):
    wl = stable_small(100, 200, 0.1)
    a, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        sim.set_option("graph", 0)
        b = sim.run(100)
        sim.set_option("profile", 1)
        c = sim.run(100)
        ms, launches = sim.kernel_time()
    np.testing.assert_array_equal(a, np.concatenate([b, c]))
    assert launches >= 6 and ms > 0  # one far-kernel launch per 16-step block


def test_profiling_in_graph_mode_changes_nothing(golden_weights):
    wl = stable_small(200, 200, 0.1)
    a, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        sim.set_option("profile", 1)
        b = sim.run(200)
        far_ms, far_n, step_ms, step_n = sim.kernel_times()
        block = sim.info()["fused_step"] == 2
    np.testing.assert_array_equal(a, b)
    # 12 graphed 16-step blocks + 8 direct steps; the block form runs each
    # block's steps (and the last 8) as one launch
    assert far_n == 13 and step_n == (13 if block else 200)
    assert far_ms > 0 and step_ms > 0


@pytest.mark.parametrize("graph", [1, 0])
def test_block_step_matches_per_step_launches(golden_weights, graph):
    """One cooperative launch per 16-step block against one launch per step:
    same kernels' arithmetic, so bitwise-equal trajectories, including runs
    that start and stop off a block boundary."""
    wl = stable_small(300, 200, 0.1)
    outs = []
    for block in (0, 1):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
            assert sim.info()["fused_step"] == 2
            sim.set_option("block_step", block)
            sim.set_option("graph", graph)
            outs.append(np.concatenate([sim.run(37), sim.run(100), sim.run(63)]))
    np.testing.assert_array_equal(outs[0], outs[1])


def test_far_kernel_variants_agree_bitwise(golden_weights):
    """The far-kernel variants differ only in register budget, load width and
    task order; their arithmetic, and so their results, are identical."""
    wl = stable_small(300, 160, 0.06)
    outs = []
    variants = (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11)
    for v in variants:
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
            sim.set_option("far_variant", v)
            outs.append(sim.run(160))
    for i in range(1, len(variants)):
        np.testing.assert_array_equal(outs[0], outs[i])


@pytest.mark.parametrize("geometry", ["line", "cluster_and_line"])
def test_staged_window_variants_on_long_and_short_runs(golden_weights, geometry):
    """Variants 10 and 11 copy a source's window run (all 32 targets'
    windows) into shared memory when it fits 128 samples and read global
    memory when it does not: a line of dots 5 c dt apart gives every source
    runs of ~180 samples, a tight cluster beside it gives short ones.  Both
    paths, and the ring's wrap, give variant 0's bits."""
    if geometry == "line":
        wl = line_of_dots(256, 5e-3)
    else:
        wl = line_of_dots(256, 4e-3)
        rng = np.random.default_rng(8)
        wl.dots[:128, 0:3] = rng.uniform(-0.01, 0.01, size=(128, 3))
        wl.dots[:128, 8] = 2e-5
    outs = []
    for v in (0, 10, 11):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
            sim.set_option("far_variant", v)
            outs.append(sim.run(300))
    assert np.abs(outs[0][..., 1]).max() > 1e-8
    for o in outs[1:]:
        np.testing.assert_array_equal(outs[0], o)


@pytest.mark.parametrize("variant", [0, 7])
def test_first_blocks_form_changes_nothing(golden_weights, variant):
    """The far kernel's first-blocks form (warps whose lanes' windows are
    partly live run one loop with dead samples zeroed) gives the bits of the
    two-loop form through all the blocks where windows still start before
    step -22 (max delay ~300 steps here)."""
    wl = I.plain_table(seed=4, n=1024, steps=400, pulse_delay=0.05)
    wl.dots[:, 6:9] *= 0.1
    outs = []
    for early in (1, 0):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
            sim.set_option("far_variant", variant)
            sim.set_option("far_early", early)
            assert sim.get_option("far_early") == early
            outs.append(sim.run(400))
    assert np.abs(outs[0][..., 1]).max() > 1e-8
    np.testing.assert_array_equal(outs[0], outs[1])


def test_far_autotuner_runs_at_the_first_run_and_keeps_an_explicit_choice(golden_weights):
    """FP64 table handles of 512 dots or more time the far variants at their
    first qg_run and keep the fastest; a variant set before that run is kept.
    Either way the results are the same bits."""
    wl = I.plain_table(seed=4, n=600, steps=64, pulse_delay=0.05)
    outs = []
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        outs.append(sim.run(48))
        assert sim.get_option("far_variant") in (0, 3, 5, 6, 7, 8, 9, 10, 11)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        sim.set_option("far_variant", 4)
        outs.append(sim.run(48))
        assert sim.get_option("far_variant") == 4
    np.testing.assert_array_equal(outs[0], outs[1])


def line_of_dots(n, spacing, seed=5):
    """n dots on a line along x, `spacing` apart (c dt = 1e-3): neighbours at
    floor delay 1, none at delay 0, so the groups coupled at delay <= 1 are
    the whole line and the step-block kernel waits on other blocks."""
    wl = I.plain_small(n=n, steps=300, pulse_delay=0.02)
    # jittered spacing: an exactly regular line puts some delays on integers,
    # where the reference's Lagrange weights are NaN (tested separately)
    jitter = 1.0 + 0.2 * (np.random.default_rng(seed).random(n) - 0.5)
    wl.dots[:, 0] = np.cumsum(spacing * jitter) - 0.5 * n * spacing
    wl.dots[:, 1] = 0.0
    wl.dots[:, 2] = 0.0
    wl.dots[:, 8] = 2e-4
    return wl


@pytest.mark.parametrize("case", ["delay1_chain", "dense_mid_list"])
def test_step_block_paths_against_oracle(golden_weights, oracle_weights, case):
    """Paths of the step-block kernel the random workloads rarely reach:
    delay-1 partners in other blocks (warp 0 waits for their previous step),
    and blocks whose mid list does not fit the shared-memory cache (entries
    read from the lists in HBM, several staging chunks)."""
    if case == "delay1_chain":
        wl = line_of_dots(256, 1.5e-3)
        steps = 300
    else:
        wl = I.plain_small(n=1024, steps=200, pulse_delay=0.02)
        wl.dots[:, 0:3] *= 0.03 / 0.2
        wl.dots[:, 8] = 2e-5
        steps = 200
    hist, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, steps)
    assert bad is None
    outs = []
    for block in (1, 0):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
            info = sim.info()
            if block:
                assert info["fused_step"] == 2, info
            sim.set_option("block_step", block)
            outs.append(sim.run(steps))
    np.testing.assert_array_equal(outs[0], outs[1])
    assert_parity(hist, outs[0])
    assert np.abs(outs[0][..., 1]).max() > 1e-8


def test_autotuned_variant_changes_nothing(golden_weights):
    """The autotuner (at creation, and on request) chooses among far-kernel
    variants with identical arithmetic, so the trajectory does not depend on
    its choice."""
    wl = stable_small(600, 160, 0.06)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        a = sim.run(64)
        sim.set_option("autotune", 1)
        a = np.concatenate([a, sim.run(96)])
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        sim.set_option("far_variant", 0)
        b = sim.run(160)
    np.testing.assert_array_equal(a, b)


def test_coincident_dots_raise_at_step_zero(golden_weights):
    dots = I.make_dots(5, 0.1, 3)
    dots[3, :3] = dots[1, :3]
    c = I.Constants(num_timesteps=10)
    with capi.Simulation(dots, I.make_pulse(delay=0.0), c, weights=golden_weights) as sim:
        with pytest.raises(capi.NonFiniteError) as e:
            sim.run(10)
    assert e.value.step == 0
    assert "unbounded history values at or before step 0" in str(e.value)


def test_integer_delay_raises_where_the_reference_does(golden_weights, oracle_weights):
    c = I.Constants(c0=1.0, dt=0.125, num_timesteps=40)
    dots = np.array([[0.0, 0, 0, 200, 10, 10, 0, 0, 2e-3],
                     [5.0, 0, 0, 200, 10, 10, 0, 0, 2e-3]])
    _, bad = O.run_faithful(dots, I.make_pulse(delay=0.0), c, oracle_weights, 40)
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        with capi.Simulation(dots, I.make_pulse(delay=0.0), c, weights=golden_weights, precision=prec) as sim:
            with pytest.raises(capi.NonFiniteError) as e:
                sim.run(40)
        assert e.value.step == bad == 19, prec


def test_steps_past_the_end_are_rejected(golden_weights):
    wl = I.plain_small(n=10, steps=20)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        sim.run(15, record=False)
        with pytest.raises(capi.QuestError) as e:
            sim.run(6)
        assert e.value.code == capi.QG_ERR_INVALID_ARG


def test_single_dot_and_ragged_sizes(golden_weights, oracle_weights):
    for n in [1, 2, 63, 64, 65, 129]:
        wl = I.plain_small(n=n, steps=120, pulse_delay=0.06)
        hist, _ = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 120)
        rho, _ = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
        assert_parity(hist, rho)


@pytest.mark.slow
def test_fp64_table_n4096_truncated(golden_weights, oracle_weights):
    """The N=4096 FP64-table geometry over 700 steps (past the largest delay,
    ~330, so every tap of every pair is live), pulse moved to t = 0.3.  The
    dipoles are scaled to 2e-4: at 2e-3 the closest pairs (~8e-4 apart) make
    the reference's scheme overflow within ~250 steps of the first non-zero
    field, in the oracle as well."""
    wl = I.plain_table(n=4096, steps=700, pulse_delay=0.3)
    wl.dots[:, 6:9] *= 0.1
    hist, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 700)
    assert bad is None
    rho, info = gpu_run(wl.dots, wl.pulse, wl.constants, golden_weights)
    assert info["max_delay"] >= 300
    e = assert_parity(hist, rho)
    print("N=4096 rel err rho00 %.3e rho01 %.3e" % e)
