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


def test_failed_request_is_retired_at_its_first_bad_step(golden_weights):
    """A request with a dot of T1 = 0 goes non-finite at step 0 (the
    reference's domain_error there); the service retires it after the first
    block with that step, and the requests around it are unaffected."""
    reqs = serving.serving_requests(4, rate_per_s=500.0, seed=8, n_range=(40, 300), side_range=(0.05, 0.15),
                                    step_range=(64, 160), dipole_magnitude=2e-4)
    for r in reqs:
        r.pulse[1] = 0.02
    reqs[2].dots[5, 4] = 0.0  # T1 = 0
    srv = serving.Server(budget_bytes=1e12, weights=golden_weights)
    stats = srv.serve(reqs)
    srv.close()
    by_id = {r.rid: r for r in srv.results}
    assert stats["requests"] == 4 and stats["failed"] == 1
    assert by_id[2].bad_step == 0 and by_id[2].steps_done == 16
    for req in reqs:
        if req.rid == 2:
            continue
        with capi.Simulation(req.dots, req.pulse, req.constants, weights=golden_weights) as sim:
            sim.run(req.constants.num_timesteps, record=False)
            ref = sim.state()
        np.testing.assert_array_equal(by_id[req.rid].state, ref)
        assert by_id[req.rid].bad_step == -1 and by_id[req.rid].steps_done == req.constants.num_timesteps
