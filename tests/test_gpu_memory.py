"""Handle memory comes from a per-device pool that keeps freed blocks for the
next handles, so a new handle's buffers may hold a destroyed handle's
values.  Nothing may depend on what a buffer held before: the same inputs
give the same bits whatever ran before them, in both precisions and with a
recorded trajectory."""
import numpy as np
import pytest

from quest_b200 import capi, inputs as I

pytestmark = pytest.mark.gpu


def run(wl, weights, precision, steps):
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=weights, precision=precision) as sim:
        rho = sim.run(steps)
        return rho, sim.state(), sim.bad_step()


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_reused_memory_changes_nothing(golden_weights, precision):
    a = I.plain_table(seed=11, n=700, steps=96, pulse_delay=0.02)
    b = I.plain_table(seed=12, n=700, steps=96, pulse_delay=0.05)
    a.dots[:, 6:9] *= 0.1
    b.dots[:, 6:9] *= 0.3
    first = run(a, golden_weights, precision, 96)
    for _ in range(3):
        other = run(b, golden_weights, precision, 96)  # same sizes: its blocks come back to `a`
        again = run(a, golden_weights, precision, 96)
        np.testing.assert_array_equal(again[0], first[0])
        np.testing.assert_array_equal(again[1], first[1])
        assert again[2] == first[2] == -1
    assert np.abs(other[0] - first[0]).max() > 0  # the other ensemble really differs


def test_many_handles_come_and_go(golden_weights):
    """Create and destroy handles of several sizes in turn (as a service
    does); each result equals that input's first run."""
    wls = [I.plain_table(seed=20 + i, n=n, steps=48, pulse_delay=0.02) for i, n in enumerate((150, 900, 2100))]
    for wl in wls:
        wl.dots[:, 6:9] *= 0.1
    ref = [run(wl, golden_weights, capi.PREC_FP64, 48)[0] for wl in wls]
    for k in range(6):
        i = (2 * k + 1) % 3
        np.testing.assert_array_equal(run(wls[i], golden_weights, capi.PREC_FP64, 48)[0], ref[i])
