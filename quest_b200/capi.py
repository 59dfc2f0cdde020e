"""ctypes binding of the C ABI in include/quest_gpu.h (quest_b200/libquest_gpu.so).

The library is the only compute path: there is no CPU fallback.  Loading it
fails with an exception when the shared object is missing; device calls fail
with QuestError when no CUDA device is present.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libquest_gpu.so")

QG_OK, QG_ERR_INVALID_ARG, QG_ERR_CUDA, QG_ERR_OOM, QG_ERR_NONFINITE, QG_ERR_UNSUPPORTED = range(6)
FRAME_ROTATING, FRAME_LAB = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
COEF_AUTO, COEF_TABLE, COEF_ON_THE_FLY, COEF_TUNED = 0, 1, 2, 3


class QuestError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class NonFiniteError(QuestError):
    """The reference's std::domain_error("unbounded history values at or
    before step N") (src/integrator.cpp:200-207)."""

    def __init__(self, code: int, msg: str, step: int):
        super().__init__(code, msg)
        self.step = step


class QgDot(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_double * 3), ("freq", ctypes.c_double), ("t1", ctypes.c_double),
                ("t2", ctypes.c_double), ("dip", ctypes.c_double * 3)]


class QgPulse(ctypes.Structure):
    _fields_ = [("amplitude", ctypes.c_double), ("delay", ctypes.c_double), ("width", ctypes.c_double),
                ("freq", ctypes.c_double), ("wavevector", ctypes.c_double * 3),
                ("polarization", ctypes.c_double * 3)]


class QgParams(ctypes.Structure):
    _fields_ = [("c0", ctypes.c_double), ("hbar", ctypes.c_double), ("mu0", ctypes.c_double),
                ("laser_frequency", ctypes.c_double), ("dt", ctypes.c_double),
                ("interpolation_order", ctypes.c_int), ("num_timesteps", ctypes.c_int),
                ("frame", ctypes.c_int), ("precision", ctypes.c_int), ("coef_mode", ctypes.c_int),
                ("reserved", ctypes.c_int * 3)]


class QgWeights(ctypes.Structure):
    _fields_ = [("n_time", ctypes.c_int), ("ps", ctypes.c_double * 64), ("cs", ctypes.c_double * 64),
                ("future_coef", ctypes.c_double)]


class QgInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("max_delay", ctypes.c_int), ("ring_depth", ctypes.c_int),
                ("num_pairs", ctypes.c_longlong), ("near_pairs", ctypes.c_longlong),
                ("mid_pairs", ctypes.c_longlong), ("time_block", ctypes.c_int),
                ("coef_mode", ctypes.c_int), ("precision", ctypes.c_int), ("fused_step", ctypes.c_int),
                ("device_bytes", ctypes.c_size_t), ("table_build_ms", ctypes.c_double)]


# Every symbol include/quest_gpu.h declares (checked by the CPU test suite).
EXPORTS = ["qg_last_error", "qg_version", "qg_pc_weights", "qg_create", "qg_destroy", "qg_run",
           "qg_next_step", "qg_history_evaluate", "qg_pulse_evaluate", "qg_set_history",
           "qg_get_history", "qg_get_info", "qg_footprint", "qg_stream", "qg_kernel_time",
           "qg_set_option", "qg_get_option", "qg_history_evaluate_noalloc", "qg_get_state", "qg_bad_step",
           "qg_batch_create", "qg_batch_destroy", "qg_batch_add", "qg_batch_remove", "qg_batch_run",
           "qg_batch_size", "qg_batch_set_option", "qg_batch_kernel_time", "qg_checkpoint_size",
           "qg_checkpoint_save", "qg_checkpoint_load", "qg_shard_create", "qg_shard_layout", "qg_shard_step",
           "qg_shard_import", "qg_batch_get_option"]

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `make -C quest_b200/csrc` "
                          "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.qg_last_error.restype = ctypes.c_char_p
        L.qg_version.restype = ctypes.c_char_p
        L.qg_pc_weights.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(QgWeights)]
        L.qg_create.argtypes = [ctypes.POINTER(QgDot), ctypes.c_int, ctypes.POINTER(QgPulse),
                                ctypes.POINTER(QgParams), ctypes.POINTER(QgWeights), ctypes.POINTER(vp)]
        L.qg_destroy.argtypes = [vp]
        L.qg_run.argtypes = [vp, ctypes.c_int, dp, ip]
        L.qg_next_step.argtypes = [vp, ip]
        L.qg_history_evaluate.argtypes = [vp, ctypes.c_int, dp, dp]
        L.qg_pulse_evaluate.argtypes = [vp, ctypes.c_int, dp]
        L.qg_set_history.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.qg_get_history.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.qg_get_info.argtypes = [vp, ctypes.POINTER(QgInfo)]
        L.qg_footprint.argtypes = [ctypes.c_int, ctypes.POINTER(QgParams), ctypes.c_double,
                                   ctypes.POINTER(ctypes.c_size_t)]
        L.qg_stream.argtypes = [vp]
        L.qg_stream.restype = vp
        L.qg_kernel_time.argtypes = [vp, ctypes.c_int, dp, ip, dp, ip]
        L.qg_set_option.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L.qg_get_option.argtypes = [vp, ctypes.c_char_p, ip]
        L.qg_history_evaluate_noalloc.argtypes = [vp, ctypes.c_int, vp, vp, vp]
        L.qg_get_state.argtypes = [vp, dp]
        L.qg_checkpoint_size.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
        L.qg_checkpoint_save.argtypes = [vp, vp, ctypes.c_size_t]
        L.qg_checkpoint_load.argtypes = [vp, vp, ctypes.c_size_t]
        L.qg_bad_step.argtypes = [vp, ip]
        L.qg_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
        L.qg_batch_destroy.argtypes = [vp]
        L.qg_batch_add.argtypes = [vp, vp]
        L.qg_batch_remove.argtypes = [vp, vp]
        L.qg_batch_run.argtypes = [vp, ctypes.c_int]
        L.qg_batch_size.argtypes = [vp, ip, ip, ip]
        L.qg_batch_set_option.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L.qg_batch_get_option.argtypes = [vp, ctypes.c_char_p, ip]
        L.qg_shard_create.argtypes = [ctypes.POINTER(QgDot), ctypes.c_int, ctypes.POINTER(QgPulse),
                                      ctypes.POINTER(QgParams), ctypes.POINTER(QgWeights), ctypes.c_int,
                                      ctypes.c_int, ctypes.POINTER(vp)]
        L.qg_shard_layout.argtypes = [vp, ip, ip, ip, ip]
        L.qg_shard_step.argtypes = [vp, dp]
        L.qg_shard_import.argtypes = [vp, dp]
        L.qg_batch_kernel_time.argtypes = [vp, ctypes.c_int, dp, ip, dp, ip]
        _lib = L
    return _lib


def _check(rc: int, bad: Optional[int] = None):
    if rc != QG_OK:
        msg = lib().qg_last_error().decode()
        if rc == QG_ERR_NONFINITE:
            raise NonFiniteError(rc, msg, bad if bad is not None else -1)
        raise QuestError(rc, msg)


def _dp(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def pc_weights(n_lambda: int = 18, n_time: int = 22, radius: float = 3.15):
    """PredictorCorrector::Weights: returns (ps (2, n_time), cs (2, n_time), future_coef)."""
    w = QgWeights()
    _check(lib().qg_pc_weights(n_lambda, n_time, radius, ctypes.byref(w)))
    ps = np.array(w.ps[: 2 * n_time]).reshape(2, n_time)
    cs = np.array(w.cs[: 2 * n_time]).reshape(2, n_time)
    return ps, cs, w.future_coef


def make_weights(ps: np.ndarray, cs: np.ndarray, fc: float) -> QgWeights:
    w = QgWeights()
    n_time = ps.shape[1]
    w.n_time = n_time
    for i, v in enumerate(np.asarray(ps, dtype=np.float64).reshape(-1)):
        w.ps[i] = v
    for i, v in enumerate(np.asarray(cs, dtype=np.float64).reshape(-1)):
        w.cs[i] = v
    w.future_coef = fc
    return w


def make_params(c, precision=PREC_FP64, coef_mode=COEF_AUTO) -> QgParams:
    p = QgParams()
    p.c0, p.hbar, p.mu0, p.laser_frequency, p.dt = c.c0, c.hbar, c.mu0, c.laser_frequency, c.dt
    p.interpolation_order = c.interpolation_order
    p.num_timesteps = c.num_timesteps
    p.frame = c.frame
    p.precision = precision
    p.coef_mode = coef_mode
    return p


def dots_array(dots: np.ndarray):
    dots = np.ascontiguousarray(dots, dtype=np.float64)
    assert dots.ndim == 2 and dots.shape[1] == 9
    arr = (QgDot * dots.shape[0])()
    ctypes.memmove(arr, dots.ctypes.data, dots.nbytes)
    return arr


def pulse_struct(pulse: np.ndarray) -> QgPulse:
    p = QgPulse()
    ctypes.memmove(ctypes.byref(p), np.ascontiguousarray(pulse, dtype=np.float64).ctypes.data, 80)
    return p


class Simulation:
    """One handle: the reference's dots + History + PulseInteraction +
    HistoryInteraction + PredictorCorrector::Integrator (src/main.cpp:25-52)."""

    def __init__(self, dots: np.ndarray, pulse: np.ndarray, constants, weights=None,
                 precision=PREC_FP64, coef_mode=COEF_AUTO):
        self.n = int(dots.shape[0])
        self.constants = constants
        self._dots = dots_array(dots)
        self._pulse = pulse_struct(pulse)
        self._params = make_params(constants, precision, coef_mode)
        self._w = make_weights(*weights) if weights is not None else None
        h = ctypes.c_void_p()
        _check(lib().qg_create(self._dots, self.n, ctypes.byref(self._pulse), ctypes.byref(self._params),
                               ctypes.byref(self._w) if self._w is not None else None, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().qg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def next_step(self) -> int:
        s = ctypes.c_int()
        _check(lib().qg_next_step(self.h, ctypes.byref(s)))
        return s.value

    def run(self, n_steps: int, record: bool = True, out: Optional[np.ndarray] = None):
        """Advance n_steps; returns rho (n_steps, N, 2) complex128 when record."""
        bad = ctypes.c_int(-1)
        if record:
            if out is None:
                out = np.empty((n_steps, self.n, 2), dtype=np.complex128)
            rc = lib().qg_run(self.h, n_steps, _dp(out.view(np.float64)), ctypes.byref(bad))
        else:
            rc = lib().qg_run(self.h, n_steps, None, ctypes.byref(bad))
        _check(rc, bad.value)
        return out

    def history_evaluate(self, step: int, rho01_step: Optional[np.ndarray] = None) -> np.ndarray:
        out = np.empty(self.n, dtype=np.complex128)
        src = None
        if rho01_step is not None:
            src = np.ascontiguousarray(rho01_step, dtype=np.complex128)
        _check(lib().qg_history_evaluate(self.h, step, _dp(src.view(np.float64)) if src is not None else None,
                                         _dp(out.view(np.float64))))
        return out

    def pulse_evaluate(self, step: int) -> np.ndarray:
        out = np.empty(self.n, dtype=np.complex128)
        _check(lib().qg_pulse_evaluate(self.h, step, _dp(out.view(np.float64))))
        return out

    def set_history(self, t0: int, rho01: np.ndarray) -> None:
        """rho01: (n_steps, N) complex for steps t0, t0+1, ..."""
        src = np.ascontiguousarray(rho01, dtype=np.complex128)
        _check(lib().qg_set_history(self.h, t0, src.shape[0], _dp(src.view(np.float64))))

    def get_history(self, t0: int, n: int) -> np.ndarray:
        out = np.empty((n, self.n), dtype=np.complex128)
        _check(lib().qg_get_history(self.h, t0, n, _dp(out.view(np.float64))))
        return out

    def state(self) -> np.ndarray:
        """rho (N, 2) complex after the last computed step."""
        out = np.empty((self.n, 2), dtype=np.complex128)
        _check(lib().qg_get_state(self.h, _dp(out.view(np.float64))))
        return out

    def checkpoint(self) -> bytes:
        """The device state after the last computed step (qg_checkpoint_save)."""
        size = ctypes.c_size_t()
        _check(lib().qg_checkpoint_size(self.h, ctypes.byref(size)))
        buf = ctypes.create_string_buffer(size.value)
        _check(lib().qg_checkpoint_save(self.h, buf, size.value))
        return buf.raw

    def restore(self, data: bytes) -> None:
        """Continue from a checkpoint of a simulation with the same inputs."""
        buf = ctypes.create_string_buffer(data, len(data))
        _check(lib().qg_checkpoint_load(self.h, buf, len(data)))

    def bad_step(self) -> int:
        b = ctypes.c_int()
        _check(lib().qg_bad_step(self.h, ctypes.byref(b)))
        return b.value

    def info(self) -> dict:
        i = QgInfo()
        _check(lib().qg_get_info(self.h, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in QgInfo._fields_}

    def set_option(self, key: str, value: int) -> None:
        _check(lib().qg_set_option(self.h, key.encode(), int(value)))

    def get_option(self, key: str) -> int:
        v = ctypes.c_int()
        _check(lib().qg_get_option(self.h, key.encode(), ctypes.byref(v)))
        return v.value

    def kernel_time(self, reset: bool = False) -> tuple[float, int]:
        """(far-pair kernel ms, launches) accumulated in profile mode."""
        return self.kernel_times(reset)[:2]

    def kernel_times(self, reset: bool = False) -> tuple[float, int, float, int]:
        """(far ms, far launches, per-step kernels ms, step launches)."""
        ms, n, sms, sn = ctypes.c_double(), ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        _check(lib().qg_kernel_time(self.h, int(reset), ctypes.byref(ms), ctypes.byref(n), ctypes.byref(sms),
                                    ctypes.byref(sn)))
        return ms.value, n.value, sms.value, sn.value


class Batch:
    """Many ensembles advanced together (qg_batch_*)."""

    def __init__(self, capacity: int):
        b = ctypes.c_void_p()
        _check(lib().qg_batch_create(capacity, ctypes.byref(b)))
        self.b = b
        self.members: list[Simulation] = []

    def add(self, sim: Simulation) -> None:
        _check(lib().qg_batch_add(self.b, sim.h))
        self.members.append(sim)

    def remove(self, sim: Simulation) -> None:
        _check(lib().qg_batch_remove(self.b, sim.h))
        self.members.remove(sim)

    def run(self, n_blocks: int) -> None:
        _check(lib().qg_batch_run(self.b, n_blocks))

    def set_option(self, key: str, value: int) -> None:
        _check(lib().qg_batch_set_option(self.b, key.encode(), int(value)))

    def get_option(self, key: str) -> int:
        v = ctypes.c_int()
        _check(lib().qg_batch_get_option(self.b, key.encode(), ctypes.byref(v)))
        return v.value

    def kernel_times(self, reset: bool = False) -> tuple[float, int, float, int]:
        """(far ms, far launches, step ms, step launches) while "profile" is on."""
        ms, n, sms, sn = ctypes.c_double(), ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        _check(lib().qg_batch_kernel_time(self.b, int(reset), ctypes.byref(ms), ctypes.byref(n),
                                          ctypes.byref(sms), ctypes.byref(sn)))
        return ms.value, n.value, sms.value, sn.value

    def size(self) -> tuple[int, int, int]:
        m, t, bl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().qg_batch_size(self.b, ctypes.byref(m), ctypes.byref(t), ctypes.byref(bl)))
        return m.value, t.value, bl.value

    def close(self) -> None:
        if getattr(self, "b", None) is not None and self.b.value:
            lib().qg_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(n: int, constants, side: float, precision=PREC_FP64, coef_mode=COEF_AUTO) -> int:
    b = ctypes.c_size_t()
    p = make_params(constants, precision, coef_mode)
    _check(lib().qg_footprint(n, ctypes.byref(p), side, ctypes.byref(b)))
    return int(b.value)
