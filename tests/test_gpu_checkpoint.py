"""Checkpoint / resume: the device state saved after some steps and loaded
into a fresh handle with the same inputs continues bit-identically, in FP64
and mixed precision, from a block boundary and from the middle of a block;
loading into a handle of another configuration is refused."""
import numpy as np
import pytest

from quest_b200 import capi, inputs as I

pytestmark = pytest.mark.gpu


def workload():
    wl = I.plain_small(n=300, steps=400, pulse_delay=0.1)
    wl.dots[:, 8] = 2e-4
    return wl


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
@pytest.mark.parametrize("stop", [160, 173])
def test_resume_is_bit_identical(golden_weights, precision, stop):
    wl = workload()
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=precision) as a:
        whole = a.run(300)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=precision) as b:
        first = b.run(stop)
        ck = b.checkpoint()
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=precision) as c:
        c.restore(ck)
        assert c.next_step == stop
        rest = c.run(300 - stop)
    np.testing.assert_array_equal(whole[:stop], first)
    np.testing.assert_array_equal(whole[stop:], rest)


def test_checkpoint_of_another_configuration_is_refused(golden_weights):
    wl = workload()
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as a:
        a.run(32)
        ck = a.checkpoint()
    other = I.plain_small(n=200, steps=400, pulse_delay=0.1)
    with capi.Simulation(other.dots, other.pulse, other.constants, weights=golden_weights) as b:
        with pytest.raises(capi.QuestError, match="another configuration"):
            b.restore(ck)
        with pytest.raises(capi.QuestError, match="not a checkpoint"):
            b.restore(b"\0" * 256)
