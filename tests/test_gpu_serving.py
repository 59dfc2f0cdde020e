"""Continuous batching: requests admitted while others run, under a memory
budget that forces queueing; each result must be exactly what the request
gives when simulated alone."""
import numpy as np
import pytest

from quest_b200 import capi, inputs as I, serving

pytestmark = pytest.mark.gpu


def test_served_results_equal_solo_runs(golden_weights):
    reqs = serving.serving_requests(6, rate_per_s=200.0, seed=5, n_range=(40, 600), side_range=(0.05, 0.2),
                                    step_range=(48, 200), dipole_magnitude=2e-4)
    for r in reqs:
        r.pulse[1] = 0.02  # pulse inside the short runs
    srv = serving.Server(budget_bytes=0, weights=golden_weights)  # budget 0: one at a time unless idle
    # budget just above the largest request: at least two run together
    big = max(srv.footprint(r) for r in reqs)
    srv.budget = 2.2 * big
    stats = srv.serve(reqs)
    srv.close()
    assert stats["requests"] == len(reqs)
    assert stats["p99_s"] >= stats["p50_s"] > 0
    by_id = {r.rid: r for r in srv.results}
    for req in reqs:
        with capi.Simulation(req.dots, req.pulse, req.constants, weights=golden_weights) as sim:
            sim.run(req.constants.num_timesteps, record=False)
            ref = sim.state()
        np.testing.assert_array_equal(by_id[req.rid].state, ref)
        assert by_id[req.rid].bad_step == -1
