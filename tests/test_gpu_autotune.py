"""The autotuner: the far kernel's resource shape (bit-identical variants,
timed at the first qg_run) and, with QG_COEF_TUNED, the per-pair table
against on-the-fly coefficients (timed; the loser's memory returned).  The
reference has no counterpart (history_interaction.cpp:21-45 always builds the
table).  Whatever the tuner picks, the results agree with the fixed choices:
bitwise among the table variants, within 1e-11 relative between the table
and the on-the-fly form (algebraically equal coefficients)."""
import numpy as np
import pytest

from quest_b200 import capi, inputs as I
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_tuned_choice_is_reported_and_agrees_with_both_forms(golden_weights, precision):
    wl = I.plain_table(seed=2, n=1024, steps=400, pulse_delay=0.3)
    wl.dots[:, 6:9] *= 0.1
    out = {}
    for mode in (capi.COEF_TABLE, capi.COEF_ON_THE_FLY, capi.COEF_TUNED):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=precision,
                             coef_mode=mode) as sim:
            before = sim.info()["device_bytes"]
            out[mode] = sim.run(400)
            if mode == capi.COEF_TUNED:
                chosen = sim.get_option("coef_mode")
                assert chosen in (capi.COEF_TABLE, capi.COEF_ON_THE_FLY)
                assert sim.get_option("tuned_far_us") > 0
                if chosen == capi.COEF_ON_THE_FLY:
                    assert sim.info()["device_bytes"] < before  # the table was freed
    tol = 1e-11 if precision == capi.PREC_FP64 else 1e-6
    for k in range(2):
        assert rel_err(out[capi.COEF_TABLE][..., k], out[capi.COEF_ON_THE_FLY][..., k]) < tol
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=precision,
                         coef_mode=capi.COEF_TUNED) as sim:
        sim.run(16, record=False)
        same = out[sim.get_option("coef_mode")]
    np.testing.assert_array_equal(out[capi.COEF_TUNED], same)


def test_far_variants_are_timed_and_identical(golden_weights):
    wl = I.plain_table(seed=2, n=1024, steps=64, pulse_delay=0.3)
    res = []
    for v in (None, 0, 3, 5, 6, 7, 8, 9, 10, 11):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights,
                             coef_mode=capi.COEF_TABLE) as sim:
            if v is not None:
                sim.set_option("far_variant", v)
            res.append(sim.run(64))
            if v is None:
                assert sim.get_option("far_variant") in (0, 3, 5, 6, 7, 8, 9, 10, 11)
                assert sim.get_option("tuned_far_us") > 0
    for r in res[1:]:
        np.testing.assert_array_equal(r, res[0])


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_group_search_is_reported_and_within_rounding(golden_weights, precision):
    """"tune_group" adds source tiles per warp (1, 2, 4, 8) to the search: a
    different association of the far sums, so the tuned handle agrees with
    the default grouping to rounding and bitwise with the same group set by
    hand."""
    wl = I.plain_table(seed=5, n=2048, steps=96, pulse_delay=0.02)
    wl.dots[:, 6:9] *= 0.1

    def run(**opts):
        with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=precision,
                             coef_mode=capi.COEF_TABLE) as sim:
            for k, v in opts.items():
                sim.set_option(k, v)
            r = sim.run(96)
            return r, sim.get_option("far_group"), sim.get_option("far_variant"), sim.get_option("tune_group")

    default, g0, _, _ = run()
    tuned, g, v, flag = run(tune_group=1)
    assert flag == 1 and g in (1, 2, 4, 8, g0)
    by_hand, g2, _, _ = run(far_group=g, far_variant=v)
    assert g2 == g
    np.testing.assert_array_equal(tuned, by_hand)
    tol = 1e-12 if precision == capi.PREC_FP64 else 1e-6
    for k in range(2):
        assert rel_err(tuned[..., k], default[..., k]) < tol
