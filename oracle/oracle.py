"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py's CPU-baseline leg.  The product library never
imports it.  See quest_oracle.h for what each function restates and for what
parity is pinned against.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
WINDOW = 22


class OrParams(ctypes.Structure):
    _fields_ = [("c0", ctypes.c_double), ("hbar", ctypes.c_double), ("mu0", ctypes.c_double),
                ("laser_frequency", ctypes.c_double), ("dt", ctypes.c_double),
                ("interpolation_order", ctypes.c_int), ("frame", ctypes.c_int)]


class OrWeights(ctypes.Structure):
    _fields_ = [("n_time", ctypes.c_int), ("ps", ctypes.POINTER(ctypes.c_double)),
                ("cs", ctypes.POINTER(ctypes.c_double)), ("future_coef", ctypes.c_double)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.or_lagrange_weights.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, dp]
        L.or_pair_coefficients.argtypes = [dp, dp, ctypes.POINTER(OrParams), ip, dp]
        L.or_build_table.argtypes = [dp, ctypes.c_int, ctypes.POINTER(OrParams), ip, dp]
        L.or_history_evaluate.argtypes = [ctypes.c_int, ctypes.POINTER(OrParams), ip, dp, dp,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        L.or_pulse_evaluate.argtypes = [dp, ctypes.c_int, dp, ctypes.POINTER(OrParams), ctypes.c_int, dp]
        L.or_liouville_rhs.argtypes = [dp, dp, dp, ctypes.c_double, dp]
        L.or_isfinite.argtypes = [dp]
        L.or_run_faithful.argtypes = [dp, ctypes.c_int, dp, ctypes.POINTER(OrParams),
                                      ctypes.POINTER(OrWeights), ctypes.c_int, dp, ip]
        L.or_run_fast.argtypes = [dp, ctypes.c_int, dp, ctypes.POINTER(OrParams),
                                  ctypes.POINTER(OrWeights), ctypes.c_int, dp, ip, ctypes.c_int]
        L.or_faithful_steps.argtypes = [dp, ctypes.c_int, dp, ctypes.POINTER(OrParams),
                                        ctypes.POINTER(OrWeights), ctypes.c_int, ip, dp, dp,
                                        ctypes.c_int, ctypes.c_int]
        L.or_faithful_steps.restype = ctypes.c_int
        L.or_history_evaluate_targets.argtypes = [dp, ctypes.c_int, ctypes.POINTER(OrParams), dp, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_int, ip, ctypes.c_int, dp]
        L.or_history_evaluate_targets.restype = ctypes.c_int
        L.or_faithful_step_range.argtypes = [dp, ctypes.c_int, dp, ctypes.POINTER(OrParams),
                                             ctypes.POINTER(OrWeights), ctypes.c_int, ip, dp, dp, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int]
        L.or_faithful_step_range.restype = ctypes.c_int
        L.or_coord2idx.argtypes = [ctypes.c_int, ctypes.c_int]
        L.or_coord2idx.restype = ctypes.c_longlong
        L.or_idx2coord.argtypes = [ctypes.c_longlong, ip, ip]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def params(c) -> OrParams:
    return OrParams(c.c0, c.hbar, c.mu0, c.laser_frequency, c.dt, c.interpolation_order, c.frame)


class Weights:
    def __init__(self, ps: np.ndarray, cs: np.ndarray, fc: float):
        self.ps = np.ascontiguousarray(ps, dtype=np.float64)
        self.cs = np.ascontiguousarray(cs, dtype=np.float64)
        self.fc = float(fc)
        self.s = OrWeights(self.ps.shape[1], _dp(self.ps), _dp(self.cs), self.fc)


def lagrange_weights(x: float, dt: float, q: int) -> np.ndarray:
    w = np.zeros(3 * (q + 1))
    lib().or_lagrange_weights(x, dt, q, _dp(w))
    return w.reshape(3, q + 1)


def pair_coefficients(src: np.ndarray, obs: np.ndarray, c) -> tuple[int, np.ndarray]:
    q = c.interpolation_order
    coef = np.zeros(2 * (q + 1))
    d = np.zeros(1, dtype=np.int32)
    p = params(c)
    lib().or_pair_coefficients(_dp(np.ascontiguousarray(src, dtype=np.float64)),
                               _dp(np.ascontiguousarray(obs, dtype=np.float64)),
                               ctypes.byref(p), _ip(d), _dp(coef))
    return int(d[0]), coef.view(np.complex128)


def build_table(dots: np.ndarray, c) -> tuple[np.ndarray, np.ndarray]:
    n = dots.shape[0]
    q = c.interpolation_order
    P = n * (n - 1) // 2
    delays = np.zeros(max(P, 1), dtype=np.int32)
    coefs = np.zeros(max(P, 1) * 2 * (q + 1))
    p = params(c)
    lib().or_build_table(_dp(np.ascontiguousarray(dots)), n, ctypes.byref(p), _ip(delays), _dp(coefs))
    return delays[:P], coefs[: P * 2 * (q + 1)].view(np.complex128).reshape(P, q + 1)


def history_evaluate(dots, c, delays, coefs, hist, step) -> np.ndarray:
    """hist: complex128 (N, window+T, 2, 2) reference layout."""
    n = dots.shape[0]
    T = hist.shape[1] - WINDOW
    out = np.zeros(2 * n)
    p = params(c)
    cf = np.ascontiguousarray(coefs).view(np.float64).reshape(-1)
    h = np.ascontiguousarray(hist).view(np.float64).reshape(-1)
    lib().or_history_evaluate(n, ctypes.byref(p), _ip(np.ascontiguousarray(delays, dtype=np.int32)),
                              _dp(cf), _dp(h), WINDOW, T, step, _dp(out))
    return out.view(np.complex128)


def history_evaluate_targets(dots, c, rho01: np.ndarray, t_lo: int, step: int, targets) -> np.ndarray:
    """HistoryInteraction::evaluate(step) for the given target dots only,
    coefficients on the fly (O(N) per target).  rho01: complex (N, nt) for
    steps t_lo .. t_lo + nt - 1."""
    n = dots.shape[0]
    tg = np.ascontiguousarray(targets, dtype=np.int32)
    r = np.ascontiguousarray(rho01, dtype=np.complex128)
    out = np.zeros(2 * tg.size)
    p = params(c)
    rc = lib().or_history_evaluate_targets(_dp(np.ascontiguousarray(dots)), n, ctypes.byref(p),
                                           _dp(r.view(np.float64).reshape(-1)), t_lo, r.shape[1], step, _ip(tg),
                                           tg.size, _dp(out))
    if rc != 0:
        raise ValueError("the rho01 window does not cover every tap the targets read")
    return out.view(np.complex128)


def pulse_evaluate(dots, pulse, c, step) -> np.ndarray:
    n = dots.shape[0]
    out = np.zeros(2 * n)
    p = params(c)
    lib().or_pulse_evaluate(_dp(np.ascontiguousarray(dots)), n, _dp(np.ascontiguousarray(pulse)),
                            ctypes.byref(p), step, _dp(out))
    return out.view(np.complex128)


def liouville_rhs(dot, rho, rabi, laser_freq) -> np.ndarray:
    r = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128)).view(np.float64)
    o = np.ascontiguousarray(np.asarray([rabi], dtype=np.complex128)).view(np.float64)
    out = np.zeros(4)
    lib().or_liouville_rhs(_dp(np.ascontiguousarray(dot, dtype=np.float64)), _dp(r), _dp(o),
                           laser_freq, _dp(out))
    return out.view(np.complex128)


def isfinite(sol) -> bool:
    s = np.ascontiguousarray(np.asarray(sol, dtype=np.complex128)).view(np.float64)
    return bool(lib().or_isfinite(_dp(s)))


def _run(fn, dots, pulse, c, w: Weights, T, *extra):
    n = dots.shape[0]
    hist = np.zeros((n, T + WINDOW, 2, 2), dtype=np.complex128)
    bad = np.full(1, -1, dtype=np.int32)
    p = params(c)
    rc = fn(_dp(np.ascontiguousarray(dots)), n, _dp(np.ascontiguousarray(pulse)), ctypes.byref(p),
            ctypes.byref(w.s), T, _dp(hist.view(np.float64).reshape(-1)), _ip(bad), *extra)
    return hist, (int(bad[0]) if rc else None)


def run_faithful(dots, pulse, c, w: Weights, T: int):
    """Full reference integrator (11 pair sweeps per step).  Returns
    (history complex128 (N, 22+T, 2, 2), bad_step or None)."""
    return _run(lib().or_run_faithful, dots, pulse, c, w, T)


def run_fast(dots, pulse, c, w: Weights, T: int, nthreads: int = 0):
    """Same integrator with one past sweep per step plus the near list."""
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    return _run(lib().or_run_fast, dots, pulse, c, w, T, nthreads)


def faithful_steps(dots, pulse, c, w: Weights, T, delays, coefs, hist, t0, nsteps) -> int:
    """Run faithful steps on an existing history (CPU-baseline timing)."""
    n = dots.shape[0]
    p = params(c)
    cf = np.ascontiguousarray(coefs).view(np.float64).reshape(-1)
    return lib().or_faithful_steps(_dp(np.ascontiguousarray(dots)), n, _dp(np.ascontiguousarray(pulse)),
                                   ctypes.byref(p), ctypes.byref(w.s), T,
                                   _ip(np.ascontiguousarray(delays, dtype=np.int32)), _dp(cf),
                                   _dp(hist.view(np.float64).reshape(-1)), t0, nsteps)


def init_history(n: int, T: int) -> np.ndarray:
    """The reference's initial History (main.cpp:30-36): rho = (1, 0) for
    t <= 0, zeros elsewhere; complex128 (N, 22 + T, 2, 2)."""
    hist = np.zeros((n, T + WINDOW, 2, 2), dtype=np.complex128)
    hist[:, : WINDOW + 1, 0, 0] = 1.0
    return hist


def faithful_step_range(dots, pulse, c, w: Weights, T, delays, coefs, hist, step, lo, hi) -> None:
    """One faithful step for dots [lo, hi) of `hist` in place (the others'
    history read as it stands)."""
    n = dots.shape[0]
    p = params(c)
    cf = np.ascontiguousarray(coefs).view(np.float64).reshape(-1)
    assert hist.flags.c_contiguous and hist.dtype == np.complex128
    rc = lib().or_faithful_step_range(_dp(np.ascontiguousarray(dots)), n, _dp(np.ascontiguousarray(pulse)),
                                      ctypes.byref(p), ctypes.byref(w.s), T,
                                      _ip(np.ascontiguousarray(delays, dtype=np.int32)), _dp(cf),
                                      _dp(hist.view(np.float64).reshape(-1)), step, lo, hi)
    if rc != 0:
        raise ValueError("a delay-0 pair crosses the range [lo, hi)")


def rho_trajectory(hist: np.ndarray) -> np.ndarray:
    """(T, N, 2) complex: rho00, rho01 at steps 0..T-1 (what write_history
    emits, src/history.cpp:27-33)."""
    return np.ascontiguousarray(hist[:, WINDOW:, 0, :].transpose(1, 0, 2))
