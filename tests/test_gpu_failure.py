"""Failure detection on the GPU, without a GPU fault.

The step-block kernel (16 steps in one cooperative launch) lets each 32-dot
block wait for the blocks that hold its partners; every wait is bounded and a
wait that runs out ends the launch with an error status the host reads, so
the context stays usable.  A test hook makes one block never post its steps,
with a short wait limit: the run must return QG_ERR_CUDA "timed out" and the
same handle (after "reset") and a fresh one must then run clean.

Non-finite states are the reference's domain_error (integrator.cpp:200-207):
a batch member that goes non-finite is reported at its first bad step while
the other members stay bitwise equal to their solo runs.
"""
import numpy as np
import pytest

from oracle import oracle as O
from quest_b200 import capi, inputs as I
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def test_wait_that_runs_out_returns_an_error_and_the_handle_recovers(golden_weights, oracle_weights):
    wl = I.plain_small(n=200, steps=400, pulse_delay=0.12)
    wl.dots[:, 6:9] *= 0.1  # a stable case: parity with the oracle over the whole run
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        info = sim.info()
        assert info["fused_step"] == 2  # the step-block form with several blocks
        assert sim.get_option("test_skip_post") == -1 and sim.get_option("wait_limit") == 0
        sim.set_option("wait_limit", 2000)
        sim.set_option("test_skip_post", 1)
        with pytest.raises(capi.QuestError) as e:
            sim.run(32, record=False)
        assert e.value.code == capi.QG_ERR_CUDA and "timed out" in str(e.value)
        # the context is intact: the same handle restarts and runs clean
        sim.set_option("test_skip_post", -1)
        sim.set_option("wait_limit", 0)
        sim.set_option("reset", 1)
        rho = sim.run(200)
    hist, bad = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 200)
    assert bad is None
    ref = O.rho_trajectory(hist)
    for k in range(2):
        assert rel_err(ref[..., k], rho[..., k]) <= 1e-10
    # and so does a fresh one
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim2:
        rho2 = sim2.run(200)
    np.testing.assert_array_equal(rho, rho2)


def test_wait_limit_option_is_checked(golden_weights):
    wl = I.plain_small(n=64, steps=32)
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        with pytest.raises(capi.QuestError):
            sim.set_option("wait_limit", -1)
        with pytest.raises(capi.QuestError):
            sim.set_option("test_skip_post", 99)
