"""The allocation-free evaluation, qg_history_evaluate_noalloc, against the
regular qg_history_evaluate.

Callers that cannot allocate device memory when they need the field (code
inside a global-mode CUDA stream capture, where cudaMalloc is prohibited, or a
host whose memory pool owns all device memory) use the no-alloc entry point:
they pass device buffers they own, and the library's scratch is a fixed array
in its own device memory.  This file is collected last so that a run stopping
at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from quest_b200 import capi, inputs as I
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def test_noalloc_matches_history_evaluate(golden_weights):
    import torch

    wl = I.plain_small(n=150, steps=400)
    c = wl.constants
    n = wl.n
    rng = np.random.default_rng(9)
    T = 400
    hist = rng.normal(size=(n, T + O.WINDOW)) + 1j * rng.normal(size=(n, T + O.WINDOW))
    with capi.Simulation(wl.dots, wl.pulse, c, weights=golden_weights) as sim:
        W = sim.info()["ring_depth"]
        lo = 300 - W + 1
        sim.set_history(lo, np.ascontiguousarray(hist[:, lo + O.WINDOW: 300 + O.WINDOW].T))
        # two calls in a row (two different current iterates at step 300),
        # each checked against the regular entry point
        step = 300
        for scale in (1.0, 0.5):
            cur = np.ascontiguousarray(hist[:, step + O.WINDOW]) * scale
            ref = sim.history_evaluate(step, cur)
            d_in = torch.from_numpy(cur.copy()).to("cuda")
            d_out = torch.full((n,), complex("nan+nanj"), dtype=torch.complex128, device="cuda")
            rc = capi.lib().qg_history_evaluate_noalloc(sim.h, step, ctypes.c_void_p(d_in.data_ptr()),
                                                         ctypes.c_void_p(d_out.data_ptr()), None)
            assert rc == capi.QG_OK, capi.lib().qg_last_error().decode()
            torch.cuda.synchronize()
            got = d_out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert rel_err(ref, got) < 1e-12
        # a second step right after, without the optional history write
        step = 301
        sim.set_history(step, np.ascontiguousarray(hist[:, step + O.WINDOW][None, :]))
        ref = sim.history_evaluate(step)
        d_out = torch.empty((n,), dtype=torch.complex128, device="cuda")
        rc = capi.lib().qg_history_evaluate_noalloc(sim.h, step, None, ctypes.c_void_p(d_out.data_ptr()), None)
        assert rc == capi.QG_OK, capi.lib().qg_last_error().decode()
        torch.cuda.synchronize()
        assert rel_err(ref, d_out.cpu().numpy()) < 1e-12


def test_noalloc_rejects_handles_beyond_its_scratch(golden_weights):
    import torch

    wl = I.plain_small(n=4100, steps=10)
    d_out = torch.empty((wl.n,), dtype=torch.complex128, device="cuda")
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights) as sim:
        rc = capi.lib().qg_history_evaluate_noalloc(sim.h, 0, None, ctypes.c_void_p(d_out.data_ptr()), None)
        assert rc == capi.QG_ERR_INVALID_ARG
        assert "4096" in capi.lib().qg_last_error().decode()


def _noalloc(sim, step, d_in, d_out, stream=None):
    rc = capi.lib().qg_history_evaluate_noalloc(sim.h, step, ctypes.c_void_p(d_in.data_ptr()) if d_in is not None
                                                else None, ctypes.c_void_p(d_out.data_ptr()), stream)
    assert rc == capi.QG_OK, capi.lib().qg_last_error().decode()


def _history_case(n, T, seed, frame=0, precision=capi.PREC_FP64, golden_weights=None):
    wl = I.plain_small(n=n, steps=T)
    wl.constants.frame = frame
    rng = np.random.default_rng(seed)
    hist = 1e-3 * (rng.normal(size=(n, T + O.WINDOW)) + 1j * rng.normal(size=(n, T + O.WINDOW)))
    sim = capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=precision,
                          coef_mode=capi.COEF_TABLE)
    W = sim.info()["ring_depth"]
    lo = T - 100 - W + 1
    sim.set_history(lo, np.ascontiguousarray(hist[:, lo + O.WINDOW: T - 100 + O.WINDOW].T))
    return sim, hist


@pytest.mark.parametrize("frame", [0, 1])
def test_noalloc_mixed_precision_handle(golden_weights, frame):
    """Mixed-precision handles take the FP32 one-step body with the fixed
    group size; they agree with qg_history_evaluate (16-step FP32 kernel,
    its own grouping) within the mixed form's tolerance, on two calls."""
    import torch

    sim, hist = _history_case(170, 500, 11, frame=frame, precision=capi.PREC_MIXED, golden_weights=golden_weights)
    with sim:
        step = 400
        for scale in (1.0, -0.25):
            cur = np.ascontiguousarray(hist[:, step + O.WINDOW]) * scale
            ref = sim.history_evaluate(step, cur)
            d_in = torch.from_numpy(cur.copy()).to("cuda")
            d_out = torch.full((sim.n,), complex("nan+nanj"), dtype=torch.complex128, device="cuda")
            _noalloc(sim, step, d_in, d_out)
            torch.cuda.synchronize()
            got = d_out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert rel_err(ref, got) < 1e-6


def test_noalloc_lab_frame_fp64(golden_weights):
    import torch

    sim, hist = _history_case(130, 500, 12, frame=1, golden_weights=golden_weights)
    with sim:
        for step in (400, 401):
            cur = np.ascontiguousarray(hist[:, step + O.WINDOW])
            ref = sim.history_evaluate(step, cur)
            d_in = torch.from_numpy(cur.copy()).to("cuda")
            d_out = torch.empty((sim.n,), dtype=torch.complex128, device="cuda")
            _noalloc(sim, step, d_in, d_out)
            torch.cuda.synchronize()
            assert rel_err(ref, d_out.cpu().numpy()) < 1e-12


def test_noalloc_on_a_caller_stream(golden_weights):
    """Work enqueued on the caller's stream (ordered after the handle's, which
    qg_set_history leaves idle): the result is there once that stream is."""
    import torch

    sim, hist = _history_case(150, 500, 13, golden_weights=golden_weights)
    with sim:
        s = torch.cuda.Stream()
        step = 400
        cur = np.ascontiguousarray(hist[:, step + O.WINDOW])
        ref = sim.history_evaluate(step, cur)
        with torch.cuda.stream(s):
            d_in = torch.from_numpy(cur.copy()).to("cuda", non_blocking=False)
            d_out = torch.full((sim.n,), complex("nan+nanj"), dtype=torch.complex128, device="cuda")
        for _ in range(2):
            _noalloc(sim, step, d_in, d_out, ctypes.c_void_p(s.cuda_stream))
            s.synchronize()
            assert rel_err(ref, d_out.cpu().numpy()) < 1e-12
