"""ctypes wrapper of oracle/_ref/libquest_ref.so: the reference's own src/*.cpp
files compiled unmodified (against the Eigen/Boost subset in oracle/ref_shim)
with the C entry points of oracle/ref_harness.cpp.  `make -C oracle ref`
builds it where the reference checkout exists; the built library travels
with the repository, the reference's sources do not.

TEST INFRASTRUCTURE ONLY: imported by tests/ (to pin the oracle and the GPU
path to the reference's code) and by bench.py's CPU-baseline leg.  The
product never imports it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libquest_ref.so")
WINDOW = 22


class RefParams(ctypes.Structure):
    _fields_ = [("c0", ctypes.c_double), ("hbar", ctypes.c_double), ("mu0", ctypes.c_double),
                ("laser_frequency", ctypes.c_double), ("dt", ctypes.c_double),
                ("interpolation_order", ctypes.c_int), ("frame", ctypes.c_int)]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise OSError(f"{LIB_PATH} is missing: `make -C oracle ref` builds it from the reference checkout")
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        pp = ctypes.POINTER(RefParams)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_weights.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp, dp]
        L.ref_lagrange_weights.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, dp]
        L.ref_build_table.argtypes = [dp, ctypes.c_int, pp, ip, dp]
        L.ref_history_evaluate.argtypes = [dp, ctypes.c_int, pp, dp, ctypes.c_int, ctypes.c_int, dp]
        L.ref_pulse_evaluate.argtypes = [dp, ctypes.c_int, dp, pp, ctypes.c_int, dp]
        L.ref_liouville_rhs.argtypes = [dp, dp, dp, ctypes.c_double, dp]
        L.ref_run.argtypes = [dp, ctypes.c_int, dp, pp, dp, dp, ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, ip]
        L.ref_time_steps.argtypes = [dp, ctypes.c_int, dp, pp, dp, dp, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, dp, dp]
        L.ref_time_steps.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def params(c) -> RefParams:
    return RefParams(c.c0, c.hbar, c.mu0, c.laser_frequency, c.dt, c.interpolation_order, c.frame)


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().ref_last_error().decode())


def weights(n_lambda=18, n_time=22, radius=3.15):
    """PredictorCorrector::Weights built by the reference's code (its
    least-squares step solved exactly by the shim)."""
    ps = np.zeros((2, n_time))
    cs = np.zeros((2, n_time))
    fc = np.zeros(1)
    _check(lib().ref_weights(n_lambda, n_time, radius, _dp(ps), _dp(cs), _dp(fc)))
    return ps, cs, float(fc[0])


def lagrange_weights(x: float, dt: float, q: int) -> np.ndarray:
    w = np.zeros((3, q + 1))
    _check(lib().ref_lagrange_weights(x, dt, q, _dp(w)))
    return w


def build_table(dots, c):
    """(delays[P], coefs[P, q+1] complex) in the reference's triangular order."""
    n = dots.shape[0]
    q = c.interpolation_order
    P = n * (n - 1) // 2
    delays = np.zeros(max(P, 1), dtype=np.int32)
    coefs = np.zeros(max(P, 1) * 2 * (q + 1))
    p = params(c)
    _check(lib().ref_build_table(_dp(_f64(dots)), n, ctypes.byref(p),
                                 delays.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(coefs)))
    return delays[:P], coefs[: P * 2 * (q + 1)].view(np.complex128).reshape(P, q + 1)


def history_evaluate(dots, c, hist: np.ndarray, step: int) -> np.ndarray:
    """hist: complex128 (N, 22 + T, 2, 2) in the reference's layout."""
    n = dots.shape[0]
    T = hist.shape[1] - WINDOW
    out = np.zeros(2 * n)
    p = params(c)
    h = np.ascontiguousarray(hist, dtype=np.complex128).view(np.float64).reshape(-1)
    _check(lib().ref_history_evaluate(_dp(_f64(dots)), n, ctypes.byref(p), _dp(h), T, step, _dp(out)))
    return out.view(np.complex128)


def pulse_evaluate(dots, pulse, c, step: int) -> np.ndarray:
    n = dots.shape[0]
    out = np.zeros(2 * n)
    p = params(c)
    _check(lib().ref_pulse_evaluate(_dp(_f64(dots)), n, _dp(_f64(pulse)), ctypes.byref(p), step, _dp(out)))
    return out.view(np.complex128)


def liouville_rhs(dot, rho, rabi, laser_freq) -> np.ndarray:
    r = np.ascontiguousarray(np.asarray(rho, dtype=np.complex128)).view(np.float64)
    o = np.ascontiguousarray(np.asarray([rabi], dtype=np.complex128)).view(np.float64)
    out = np.zeros(4)
    _check(lib().ref_liouville_rhs(_dp(_f64(dot)), _dp(r), _dp(o), laser_freq, _dp(out)))
    return out.view(np.complex128)


def run(dots, pulse, c, weights_, T: int):
    """The reference's whole solve (main.cpp:25-55) over T steps with the
    given weights.  Returns (history complex128 (N, 22 + T, 2, 2), bad_step
    or None)."""
    ps, cs, fc = weights_
    ps = _f64(ps)
    cs = _f64(cs)
    n = dots.shape[0]
    hist = np.zeros((n, T + WINDOW, 2, 2), dtype=np.complex128)
    bad = np.full(1, -1, dtype=np.int32)
    p = params(c)
    _check(lib().ref_run(_dp(_f64(dots)), n, _dp(_f64(pulse)), ctypes.byref(p), _dp(ps), _dp(cs), float(fc),
                         ps.shape[1], T, _dp(hist.view(np.float64).reshape(-1)),
                         bad.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
    return hist, (int(bad[0]) if bad[0] >= 0 else None)


def time_steps(dots, pulse, c, t0: int, nsteps: int, seed: int = 0, weights_=None) -> dict:
    """Wall time of `nsteps` calls of the reference's Integrator::solve_step
    from step t0 on a synthetic history (the CPU baseline), single thread."""
    if weights_ is None:
        from quest_b200.inputs import load_pc_weights
        weights_ = load_pc_weights(os.path.join(os.path.dirname(HERE), "tests", "golden",
                                                "pc_weights_18_22_3.15.txt"))
    ps, cs, fc = weights_
    ps = _f64(ps)
    cs = _f64(cs)
    n = dots.shape[0]
    p = params(c)
    sec = ctypes.c_double()
    tab = ctypes.c_double()
    done = lib().ref_time_steps(_dp(_f64(dots)), n, _dp(_f64(pulse)), ctypes.byref(p), _dp(ps), _dp(cs),
                                float(fc), ps.shape[1], t0, nsteps, seed, ctypes.byref(sec), ctypes.byref(tab))
    if done < 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return {"steps": done, "seconds": sec.value, "table_seconds": tab.value}
