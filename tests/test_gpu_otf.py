"""On-the-fly coefficients (no table): the far-pair kernel computes every
pair's floor delay and q+1 coefficients in registers each K-step block, in
an algebraically equal form of the reference's table build.

Checks: the interaction-level sum (HistoryInteraction::evaluate) against the
oracle's reference-order table on random histories, whole runs against the
oracle at the FP64 tolerance (1e-10), against the table path, in the lab
frame and at other interpolation orders, mixed precision (FP32
coefficients) against FP64, the reference's non-finite run at an integer
delay, and the N = 65536 workload (whose table would need 215 GB) for a
few blocks."""
import numpy as np
import pytest

from oracle import oracle as O
from quest_b200 import capi, inputs as I
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10


def run(wl, weights, steps, **kw):
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=weights, **kw) as sim:
        rho = sim.run(steps)
        info = sim.info()
    return rho, info


def parity(hist, rho):
    ref = O.rho_trajectory(hist)[: rho.shape[0]]
    return rel_err(ref[..., 0], rho[..., 0]), rel_err(ref[..., 1], rho[..., 1])


def stable(n, steps, pulse_delay, side=0.2, seed=2):
    wl = I.plain_small(n=n, steps=steps, pulse_delay=pulse_delay)
    wl.dots[:, 8] = 2e-4
    return wl


def test_otf_info_matches_table(golden_weights):
    wl = stable(700, 32, 0.1)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights,
                         coef_mode=capi.COEF_TABLE) as a, \
            capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights,
                            coef_mode=capi.COEF_ON_THE_FLY) as b:
        ia, ib = a.info(), b.info()
    assert ib["coef_mode"] == capi.COEF_ON_THE_FLY and ia["coef_mode"] == capi.COEF_TABLE
    for key in ("max_delay", "ring_depth", "near_pairs", "mid_pairs", "num_pairs"):
        assert ia[key] == ib[key], key
    assert ib["device_bytes"] < ia["device_bytes"]


def test_otf_history_evaluate_matches_reference_table(golden_weights):
    wl = I.plain_small(n=150, steps=400)
    c = wl.constants
    n = wl.n
    rng = np.random.default_rng(11)
    T = 400
    hist = np.zeros((n, T + O.WINDOW, 2, 2), dtype=np.complex128)
    hist[:, :, 0, 1] = rng.normal(size=(n, T + O.WINDOW)) + 1j * rng.normal(size=(n, T + O.WINDOW))
    delays, coefs = O.build_table(wl.dots, c)
    with capi.Simulation(wl.dots, wl.pulse, c, weights=golden_weights, coef_mode=capi.COEF_ON_THE_FLY) as sim:
        W = sim.info()["ring_depth"]
        for step in [0, 60, 250, 399]:
            lo = max(-O.WINDOW, step - W + 1)
            sim.set_history(lo, hist[:, lo + O.WINDOW: step + O.WINDOW, 0, 1].T)
            got = sim.history_evaluate(step, hist[:, step + O.WINDOW, 0, 1])
            ref = O.history_evaluate(wl.dots, c, delays, coefs, hist, step)
            assert rel_err(ref, got) < 1e-12, step


def test_otf_against_oracle(golden_weights, oracle_weights):
    wl = I.plain_small(n=60, steps=350, pulse_delay=0.2)
    hist, bad = O.run_faithful(wl.dots, wl.pulse, wl.constants, oracle_weights, 350)
    assert bad is None
    rho, info = run(wl, golden_weights, 350, coef_mode=capi.COEF_ON_THE_FLY)
    assert info["coef_mode"] == capi.COEF_ON_THE_FLY
    e00, e01 = parity(hist, rho)
    assert e00 <= TOL and e01 <= TOL, (e00, e01)
    assert np.abs(rho[..., 1]).max() > 1e-6


def test_otf_stable_run_against_oracle_and_table(golden_weights, oracle_weights):
    wl = stable(1000, 600, 0.1)
    hist, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 600)
    assert bad is None
    got, _ = run(wl, golden_weights, 600, coef_mode=capi.COEF_ON_THE_FLY)
    e00, e01 = parity(hist, got)
    assert e00 <= TOL and e01 <= TOL, (e00, e01)
    tab, _ = run(wl, golden_weights, 600, coef_mode=capi.COEF_TABLE)
    assert rel_err(tab[..., 1], got[..., 1]) <= 1e-11
    assert rel_err(tab[..., 0], got[..., 0]) <= 1e-11


@pytest.mark.parametrize("q,frame,steps", [(3, 0, 300), (7, 0, 200), (5, 1, 300)])
def test_otf_orders_and_lab_frame(golden_weights, oracle_weights, q, frame, steps):
    """Horizons as in the table path's tests: order 7 amplifies rounding
    differences (here: coefficient rounding) faster than order 5."""
    wl = I.plain_small(n=90, steps=steps, pulse_delay=0.15)
    wl.constants.interpolation_order = q
    wl.constants.frame = frame
    hist, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, steps)
    assert bad is None
    rho, _ = run(wl, golden_weights, steps, coef_mode=capi.COEF_ON_THE_FLY)
    e00, e01 = parity(hist, rho)
    assert e00 <= TOL and e01 <= TOL, (e00, e01)


def test_otf_mixed_matches_fp64(golden_weights):
    wl = stable(1000, 600, 0.1)
    ref, _ = run(wl, golden_weights, 600, coef_mode=capi.COEF_ON_THE_FLY)
    got, info = run(wl, golden_weights, 600, coef_mode=capi.COEF_ON_THE_FLY, precision=capi.PREC_MIXED)
    assert info["precision"] == capi.PREC_MIXED and info["coef_mode"] == capi.COEF_ON_THE_FLY
    assert rel_err(ref[..., 0], got[..., 0]) <= 1e-6
    assert rel_err(ref[..., 1], got[..., 1]) <= 1e-6


def test_otf_integer_delay_raises_where_the_reference_does(golden_weights, oracle_weights):
    """A pair at an exactly integer delay (distance 5, c dt = 0.125: 40
    steps, a far pair) has NaN Lagrange weights in the reference; the
    on-the-fly coefficients, FP64 and FP32, make the run non-finite at the
    step the reference and the table path do."""
    c = I.Constants(c0=1.0, dt=0.125, num_timesteps=40)
    dots = np.array([[0.0, 0, 0, 200, 10, 10, 0, 0, 2e-3],
                     [5.0, 0, 0, 200, 10, 10, 0, 0, 2e-3]])
    _, bad = O.run_faithful(dots, I.make_pulse(delay=0.0), c, oracle_weights, 40)
    assert bad is not None
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        with capi.Simulation(dots, I.make_pulse(delay=0.0), c, weights=golden_weights, precision=prec,
                             coef_mode=capi.COEF_ON_THE_FLY) as sim:
            with pytest.raises(capi.NonFiniteError) as e:
                sim.run(40)
        assert e.value.step == bad, (prec, e.value.step, bad)


def test_otf_rejected_where_a_table_is_needed(golden_weights):
    import ctypes
    import torch

    wl = stable(100, 32, 0.1)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights,
                         coef_mode=capi.COEF_ON_THE_FLY) as sim:
        out = torch.empty((wl.n,), dtype=torch.complex128, device="cuda")
        rc = capi.lib().qg_history_evaluate_noalloc(sim.h, 0, None, ctypes.c_void_p(out.data_ptr()), None)
        assert rc == capi.QG_ERR_UNSUPPORTED
        assert "on the fly" in capi.lib().qg_last_error().decode()
        b = capi.Batch(2)
        try:
            with pytest.raises(capi.QuestError):
                b.add(sim)
        finally:
            b.close()


def test_otf_n65536_blocks(golden_weights):
    """The N = 65536, 0.5-cube workload (table: 215 GB): creation, two
    16-step blocks in mixed precision and FP64, finite states, the far
    field nonzero once the history is."""
    wl = I.mixed_large(n=65536, steps=5000)
    for prec in (capi.PREC_MIXED, capi.PREC_FP64):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=prec) as sim:
            info = sim.info()
            assert info["coef_mode"] == capi.COEF_ON_THE_FLY
            assert 850 <= info["max_delay"] <= 870
            sim.run(32, record=False)
            st = sim.state()
            assert np.all(np.isfinite(st))


def test_otf_n65536_evaluate_sampled_targets_against_oracle(golden_weights):
    """cfg 3 at full size (N = 65536 in the 0.5 cube, delays up to ~866
    steps): HistoryInteraction::evaluate (history_interaction.cpp:47-70)
    through qg_history_evaluate with on-the-fly FP64 coefficients, on a
    random rho01 history covering every tap read, against the oracle's
    per-target sum (coefficients on the fly in the reference's pair
    orientation, O(N) per target) for 64 sampled targets."""
    wl = I.mixed_large(n=65536, steps=5000)
    n = wl.n
    rng = np.random.default_rng(65536)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=capi.PREC_FP64,
                         coef_mode=capi.COEF_ON_THE_FLY) as sim:
        info = sim.info()
        W = info["ring_depth"]
        step = 1000
        t_lo = step - W + 1
        assert t_lo <= step - info["max_delay"] - 5
        # (steps, N) for qg_set_history, complex64 draws widened to keep the host copy small
        hist = (rng.standard_normal((W, n), dtype=np.float32) +
                1j * rng.standard_normal((W, n), dtype=np.float32)).astype(np.complex128)
        sim.set_history(t_lo, hist)
        got = sim.history_evaluate(step)
    targets = np.sort(rng.choice(n, size=64, replace=False))
    ref = O.history_evaluate_targets(wl.dots, wl.constants, np.ascontiguousarray(hist.T), t_lo, step, targets)
    assert np.all(np.abs(ref) > 0)
    assert rel_err(ref, got[targets]) <= 1e-12


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_otf_task_orders_agree_bitwise(golden_weights, precision):
    """far_variant 7 runs the on-the-fly kernel's tasks source-group major,
    1 holds it to 3 blocks per SM, 8 does both; each target's sums are
    unchanged."""
    wl = stable(1000, 96, 0.1)
    outs = []
    for v in (None, 7, 1, 8):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=precision,
                             coef_mode=capi.COEF_ON_THE_FLY) as sim:
            if v is not None:
                sim.set_option("far_variant", v)
            outs.append(sim.run(96))
    for o in outs[1:]:
        np.testing.assert_array_equal(outs[0], o)
