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
