"""Continuous-batching service for ensemble simulations.

Requests (one ensemble each: dots, pulse, constants) arrive over time.  The
service admits them first-come first-served while their device footprint
(coefficient table + history rings + integrator state, qg_footprint) fits
the memory budget, builds each admitted ensemble (qg_create: upload and table
build) on a worker thread while the batch keeps running, and adds it to the
running batch at the first 16-step block after its build is done.  Every
block advances all running ensembles in one persistent far-pair launch and
16 step launches (qg_batch_run); ensembles that reach their last step are
retired, their final state read back and their memory returned, which lets
waiting requests in.  An ensemble whose state goes non-finite is retired at
the first batch run that sees it, with that first bad step as its error (the
reference stops a run there with std::domain_error, integrator.cpp:200-207);
the other ensembles go on unchanged.  Results do not depend on what else is running: a
batch member is advanced by the same kernels, in the same order, as it
would be alone.

There is no reference counterpart; the reference runs one ensemble per
process (src/main.cpp).
"""
from __future__ import annotations

import collections
import concurrent.futures
import dataclasses
import math
import time
from typing import Optional

import numpy as np

from . import capi, inputs as I


@dataclasses.dataclass
class Request:
    rid: int
    dots: np.ndarray
    pulse: np.ndarray
    constants: I.Constants
    arrival: float = 0.0          # seconds after the service starts

    @property
    def n(self) -> int:
        return int(self.dots.shape[0])

    @property
    def pair_updates(self) -> float:
        return float(self.n) ** 2 * self.constants.num_timesteps

    def side(self) -> float:
        ext = self.dots[:, 0:3].max(axis=0) - self.dots[:, 0:3].min(axis=0)
        return float(ext.max())


@dataclasses.dataclass
class Result:
    rid: int
    n: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    state: np.ndarray             # (N, 2) complex: rho00, rho01 after the last step
    bad_step: int                 # first non-finite step, -1 if none
    steps_done: int = 0           # steps computed (num_timesteps unless it failed earlier)

    @property
    def failed(self) -> bool:
        return self.bad_step >= 0

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Server:
    def __init__(self, budget_bytes: float = 150e9, capacity: int = 1024, weights=None,
                 blocks_per_round: int = 1, precision: int = capi.PREC_FP64, tune_group: bool = False):
        self.precision = precision
        self.budget = float(budget_bytes)
        self.capacity = capacity
        self.weights = weights if weights is not None else capi.pc_weights()
        self.blocks_per_round = blocks_per_round
        self.batch = capi.Batch(capacity)
        if tune_group:
            # the batch's first run also times source tiles per far warp for
            # each size class present; later requests of a tuned class take
            # its group (their results then match solo runs with that group)
            self.batch.set_option("tune_group", 1)
        self.running: dict[int, tuple[Request, capi.Simulation, float, int]] = {}
        # builds in flight, in admission order: (request, future, admitted, footprint)
        self.building: collections.deque = collections.deque()
        self._pool = concurrent.futures.ThreadPoolExecutor(max_workers=1)
        import torch
        # the worker builds on the caller's GPU
        self._device = torch.cuda.current_device() if torch.cuda.is_available() else None
        self.used = 0.0
        self.results: list[Result] = []
        self.pair_updates_done = 0.0

    def footprint(self, req: Request) -> int:
        return capi.footprint(req.n, req.constants, req.side(), precision=self.precision)

    def _build(self, req: Request) -> capi.Simulation:
        # runs on the worker thread: the library's calls release the GIL, its
        # error state is per thread, and the new handle has a stream of its own
        if self._device is not None:
            import torch
            torch.cuda.set_device(self._device)
        return capi.Simulation(req.dots, req.pulse, req.constants, weights=self.weights, precision=self.precision)

    def _admit(self, req: Request, now: float) -> None:
        fp = self.footprint(req)
        self.building.append((req, self._pool.submit(self._build, req), now, fp))
        self.used += fp

    def _join_built(self, wait: bool) -> None:
        """Moves finished builds (in admission order) into the batch; with
        `wait`, blocks for the oldest one first."""
        while self.building and (wait or self.building[0][1].done()):
            req, fut, admitted, fp = self.building.popleft()
            sim = fut.result()
            self.batch.add(sim)
            self.running[req.rid] = (req, sim, admitted, fp)
            wait = False

    def _retire(self, rid: int, now: float) -> None:
        req, sim, admitted, fp = self.running.pop(rid)
        state = sim.state()
        bad = sim.bad_step()
        done = sim.next_step
        self.batch.remove(sim)
        sim.close()
        self.used -= fp
        self.pair_updates_done += float(req.n) ** 2 * done
        self.results.append(Result(req.rid, req.n, req.constants.num_timesteps, req.arrival, admitted, now,
                                   state, bad, done))

    def serve(self, requests: list[Request], clock=time.perf_counter) -> dict:
        """Runs until every request is finished.  Arrival times are seconds
        from the start; a request is visible to the scheduler once the clock
        passes its arrival time."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queue: collections.deque[Request] = collections.deque()
        t0 = clock()
        busy = 0.0
        while pending or queue or self.running or self.building:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            # admit first-come first-served while memory and slots allow
            while queue and len(self.running) + len(self.building) < self.capacity:
                fp = self.footprint(queue[0])
                if (self.running or self.building) and self.used + fp > self.budget:
                    break
                self._admit(queue.popleft(), clock() - t0)
            self._join_built(wait=not self.running and bool(self.building))
            if not self.running:
                if pending:  # idle until the next arrival
                    time.sleep(max(0.0, min(pending[0].arrival - (clock() - t0), 0.01)))
                continue
            b0 = clock()
            self.batch.run(self.blocks_per_round)
            busy += clock() - b0
            now = clock() - t0
            # finished, or non-finite (the batch run gathered every member's
            # first bad step, so bad_step() costs no device round trip)
            for rid in [r for r, (req, sim, _, _) in self.running.items()
                        if sim.next_step >= req.constants.num_timesteps or sim.bad_step() >= 0]:
                self._retire(rid, now)
        wall = clock() - t0
        lat = np.array([r.latency for r in self.results])
        ok = np.array([r.latency for r in self.results if not r.failed])
        return {
            "requests": len(self.results),
            "failed": sum(1 for r in self.results if r.failed),
            "wall_s": wall,
            "busy_s": busy,
            "pair_updates": self.pair_updates_done,
            "pair_updates_per_s": self.pair_updates_done / wall if wall > 0 else 0.0,
            "p50_s_completed": float(np.percentile(ok, 50)) if ok.size else None,
            "p99_s_completed": float(np.percentile(ok, 99)) if ok.size else None,
            "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_s": float(np.percentile(lat, 99)) if lat.size else None,
        }

    def close(self) -> None:
        while self.building:
            _, fut, _, _ = self.building.popleft()
            fut.result().close()
        self._pool.shutdown(wait=True)
        for rid in list(self.running):
            _, sim, _, _ = self.running.pop(rid)
            sim.close()
        self.batch.close()


def serving_requests(count: int, rate_per_s: float, seed: int, n_range=(32, 16384), side_range=(0.05, 0.5),
                     step_range=(1000, 20000), dipole_magnitude: float = 2e-3) -> list[Request]:
    """The serving workload: Poisson arrivals at `rate_per_s`, N log-uniform
    in n_range, cube side uniform in side_range, steps uniform in step_range
    (rounded down to a multiple of 16), pulse E_0 uniform in [1, 30],
    omega_0 ~ N(200, 0.5^2), T1 = T2 = 10, unit-random dipoles."""
    u = I.uniform(seed, 6 * count, stream=7).reshape(count, 6)
    reqs = []
    t = 0.0
    for i in range(count):
        t += -math.log(1.0 - u[i, 0]) / rate_per_s
        lo, hi = math.log(n_range[0]), math.log(n_range[1])
        n = int(round(math.exp(lo + u[i, 1] * (hi - lo))))
        side = side_range[0] + u[i, 2] * (side_range[1] - side_range[0])
        steps = int(step_range[0] + u[i, 3] * (step_range[1] - step_range[0]))
        steps = max(16, steps - steps % 16)
        amp = 1.0 + 29.0 * u[i, 4]
        dots = I.make_dots(n, side, seed * 100003 + i, omega_sigma=0.5, dipole=None,
                           dipole_magnitude=dipole_magnitude)
        reqs.append(Request(i, dots, I.make_pulse(amplitude=amp), I.Constants(num_timesteps=steps), t))
    return reqs


def batched_ensembles(count: int, seed: int, n_range=(64, 4096), side_range=(0.05, 0.3),
                      step_range=(2000, 20000), dipole_magnitude: float = 2e-3) -> list[Request]:
    """The batched workload: `count` ensembles present from the start, N
    log-uniform in n_range, side uniform in side_range, steps uniform in
    step_range, pulse and dot parameters as in serving_requests."""
    reqs = serving_requests(count, 1.0, seed, n_range=n_range, side_range=side_range, step_range=step_range,
                            dipole_magnitude=dipole_magnitude)
    for r in reqs:
        r.arrival = 0.0
    return reqs
