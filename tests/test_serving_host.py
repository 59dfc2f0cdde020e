"""The serving loop's host logic on CPU, with fake handles in place of the
library: first-come first-served admission under the memory budget (builds
in flight count against it), builds on the worker thread joining the batch
in admission order, every request retired once its last step is done, and
the latency statistics.  The GPU run of the same loop (same result alone
and in the mix) is tests/test_gpu_serving.py."""
import threading
import time

import numpy as np

from quest_b200 import capi, inputs as I, serving


class FakeSim:
    """A handle that advances 16 steps per batch block."""

    def __init__(self, dots, pulse, constants, weights=None, precision=0):
        self.n = dots.shape[0]
        self.steps = constants.num_timesteps
        self.next_step = 0
        self.closed = False
        self.thread = threading.current_thread().name
        # a dot with T1 = 0 makes the state non-finite at step 0, as on the GPU
        self.fails_at = 0 if np.any(dots[:, 4] == 0) else None
        time.sleep(0.01)  # a build takes a while

    def state(self):
        return np.zeros((self.n, 2), dtype=np.complex128)

    def bad_step(self):
        return self.fails_at if (self.fails_at is not None and self.next_step > self.fails_at) else -1

    def close(self):
        self.closed = True


class FakeBatch:
    def __init__(self, capacity):
        self.members = []
        self.max_members = 0
        self.log = []

    def add(self, sim):
        self.members.append(sim)
        self.max_members = max(self.max_members, len(self.members))
        self.log.append(("add", sim))

    def remove(self, sim):
        self.members.remove(sim)
        self.log.append(("remove", sim))

    def run(self, n_blocks):
        time.sleep(0.002)
        for s in self.members:
            s.next_step = min(s.steps, s.next_step + 16 * n_blocks)

    def close(self):
        pass


def make_requests(sizes, steps, gap):
    reqs = []
    for i, (n, t) in enumerate(zip(sizes, steps)):
        dots = I.make_dots(n, 0.1, 100 + i, omega_sigma=0.5, dipole=None)
        reqs.append(serving.Request(i, dots, I.make_pulse(), I.Constants(num_timesteps=t), arrival=i * gap))
    return reqs


def run_server(monkeypatch, reqs, budget, footprint):
    monkeypatch.setattr(capi, "Simulation", FakeSim)
    monkeypatch.setattr(capi, "Batch", FakeBatch)
    monkeypatch.setattr(capi, "footprint", lambda n, c, side, precision=0: footprint(n))
    srv = serving.Server(budget_bytes=budget, weights=(None, None, None))
    stats = srv.serve(reqs)
    batch = srv.batch
    results = srv.results
    srv.close()
    return stats, batch, results


def test_every_request_finishes_with_its_latency(monkeypatch):
    reqs = make_requests([40, 70, 30, 90, 50], [64, 160, 32, 96, 48], gap=0.005)
    stats, batch, results = run_server(monkeypatch, reqs, budget=1e12, footprint=lambda n: n)
    assert stats["requests"] == 5
    assert sorted(r.rid for r in results) == [0, 1, 2, 3, 4]
    for r in results:
        assert r.steps == reqs[r.rid].constants.num_timesteps
        assert r.finished >= r.admitted >= r.arrival - 1e-9
        assert r.latency > 0
    assert stats["pair_updates"] == sum(q.pair_updates for q in reqs)
    assert stats["p99_s"] >= stats["p50_s"] > 0
    assert batch.members == []


def test_builds_run_on_the_worker_thread_and_join_in_admission_order(monkeypatch):
    reqs = make_requests([40, 50, 60, 70], [320, 320, 320, 320], gap=0.0)
    _, batch, _ = run_server(monkeypatch, reqs, budget=1e12, footprint=lambda n: n)
    added = [s for op, s in batch.log if op == "add"]
    assert [s.n for s in added] == [40, 50, 60, 70]
    assert all(s.thread != threading.main_thread().name for s in added)
    assert all(s.closed for s in added)


def test_budget_limits_the_running_and_building_set(monkeypatch):
    # each request needs 10 units, the budget holds 25: at most two at once
    reqs = make_requests([32] * 6, [64] * 6, gap=0.0)
    stats, batch, _ = run_server(monkeypatch, reqs, budget=25, footprint=lambda n: 10)
    assert stats["requests"] == 6
    assert batch.max_members <= 2


def test_a_request_larger_than_the_budget_runs_alone(monkeypatch):
    reqs = make_requests([32, 32, 32], [64, 64, 64], gap=0.0)
    stats, batch, _ = run_server(monkeypatch, reqs, budget=5, footprint=lambda n: 10)
    assert stats["requests"] == 3
    assert batch.max_members == 1


def test_a_member_that_goes_nonfinite_is_retired_at_once(monkeypatch):
    reqs = make_requests([40, 50, 60], [320, 320, 320], gap=0.0)
    reqs[1].dots[3, 4] = 0.0  # T1 = 0
    stats, batch, results = run_server(monkeypatch, reqs, budget=1e12, footprint=lambda n: n)
    by = {r.rid: r for r in results}
    assert stats["requests"] == 3 and stats["failed"] == 1
    assert by[1].failed and by[1].bad_step == 0 and by[1].steps_done == 16  # retired after its first block
    assert not by[0].failed and by[0].steps_done == 320 and by[2].steps_done == 320
    assert stats["pair_updates"] == 40 ** 2 * 320 + 50 ** 2 * 16 + 60 ** 2 * 320
