"""Seeded synthetic inputs and reference-format configuration files.

Dots are float64 arrays of shape (N, 9) in the column order of a dots.cfg line
(x y z omega_0 T1 T2 dx dy dz; reference src/quantum_dot.cpp:33-38).  A pulse
is a float64 array of 10 values in pulse.cfg order (E_0 delay sigma omega_L kx
ky kz px py pz; src/pulse.cpp:29-35).  Physical constants follow the
reference's input.cfg keys (src/configuration.cpp:17-42).

The generator is counter based (splitmix64), so the same seed gives the same
doubles on every machine.  Cubes are centred at the origin, as the reference's
point generator does (tools/point_gen.cpp:57-60).

Constants the workload descriptions leave open are fixed here and recorded
with every result: hbar = 1, mu0 = 1, laser_frequency = omega_L = 200.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """`count` 64-bit outputs of splitmix64 for (seed, stream)."""
    with np.errstate(over="ignore"):
        base = np.uint64((seed * 0x9E3779B97F4A7C15 + stream * 0xD1B54A32D192ED03) & 0xFFFFFFFFFFFFFFFF)
        z = base + (np.arange(1, count + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """Uniform doubles in [0, 1) from the top 53 bits."""
    return (splitmix64(seed, count, stream) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """Standard normal doubles by Box-Muller."""
    m = (count + 1) // 2
    u = uniform(seed, 2 * m, stream)
    # scalar libm calls: numpy's SIMD log/cos may differ in the last bit
    # between CPUs, glibc's do not
    r = [math.sqrt(-2.0 * math.log(1.0 - float(x))) for x in u[:m]]
    a = [2.0 * math.pi * float(x) for x in u[m:]]
    z = np.array([ri * math.cos(ai) for ri, ai in zip(r, a)] +
                 [ri * math.sin(ai) for ri, ai in zip(r, a)], dtype=np.float64)
    return z[:count]


@dataclasses.dataclass
class Constants:
    """input.cfg [constants] and [parameters] values (configuration.cpp:17-42)."""
    c0: float = 1.0
    hbar: float = 1.0
    mu0: float = 1.0
    laser_frequency: float = 200.0
    dt: float = 1e-3
    interpolation_order: int = 5
    num_timesteps: int = 2000
    frame: int = 0  # 0 rotating frame (what the reference's main uses), 1 lab frame


def make_dots(n: int, side: float, seed: int, *, omega0: float = 200.0, omega_sigma: float = 0.0,
              t1: float = 10.0, t2: float = 10.0, dipole: Optional[tuple] = (0.0, 0.0, 2e-3),
              dipole_magnitude: float = 2e-3) -> np.ndarray:
    """N dots uniform in a centred cube of the given side.

    dipole=None draws unit-random directions (normalised Gaussian 3-vectors)
    scaled by dipole_magnitude; omega_sigma > 0 jitters omega_0 with N(omega0,
    omega_sigma^2).
    """
    d = np.empty((n, 9), dtype=np.float64)
    pos = uniform(seed, 3 * n, stream=1).reshape(n, 3)
    d[:, 0:3] = (pos - 0.5) * side
    if omega_sigma > 0:
        d[:, 3] = omega0 + omega_sigma * normal(seed, n, stream=2)
    else:
        d[:, 3] = omega0
    d[:, 4] = t1
    d[:, 5] = t2
    if dipole is None:
        g = normal(seed, 3 * n, stream=3).reshape(n, 3)
        g /= np.linalg.norm(g, axis=1, keepdims=True)
        d[:, 6:9] = g * dipole_magnitude
    else:
        d[:, 6:9] = np.asarray(dipole, dtype=np.float64)
    return d


def make_pulse(amplitude=15.0, delay=5.0, width=1.0, freq=200.0, wavevector=(200.0, 0.0, 0.0),
               polarization=(0.0, 0.0, 1.0)) -> np.ndarray:
    return np.array([amplitude, delay, width, freq, *wavevector, *polarization], dtype=np.float64)


@dataclasses.dataclass
class Workload:
    name: str
    dots: np.ndarray
    pulse: np.ndarray
    constants: Constants
    seed: int

    @property
    def n(self) -> int:
        return int(self.dots.shape[0])


def plain_small(seed: int = 1, n: int = 200, steps: int = 2000, pulse_delay: float = 5.0) -> Workload:
    """N=200 identical dots in a 0.2 cube, omega_0 = 200, T1 = T2 = 10, dipole
    (0, 0, 2e-3); pulse (15, delay, 1, 200, (200,0,0), (0,0,1)); c = 1,
    dt = 1e-3, 2000 steps, order 5.  With pulse delay 5 the pulse never reaches
    the dots before t = 2 and every trajectory stays (1, 0); delay 0.5 gives a
    non-trivial case of the same size."""
    dots = make_dots(n, 0.2, seed)
    return Workload(f"plain_N{n}_T{steps}_delay{pulse_delay:g}", dots, make_pulse(delay=pulse_delay),
                    Constants(num_timesteps=steps), seed)


def plain_table(seed: int = 2, n: int = 4096, steps: int = 20000, pulse_delay: float = 5.0) -> Workload:
    """N=4096 dots in a 0.2 cube, omega_0 ~ N(200, 0.5^2), T1 = T2 = 10,
    unit-random dipoles x 2e-3, same pulse, c = 1, dt = 1e-3, 20000 steps,
    order 5 (the FP64 per-pair-table workload)."""
    dots = make_dots(n, 0.2, seed, omega_sigma=0.5, dipole=None)
    return Workload(f"fp64_table_N{n}_T{steps}", dots, make_pulse(delay=pulse_delay),
                    Constants(num_timesteps=steps), seed)


def mixed_large(seed: int = 3, n: int = 65536, steps: int = 5000, side: float = 0.5,
                pulse_delay: float = 5.0) -> Workload:
    """N=65536 dots in a 0.5 cube (retarded delays up to ~866 steps), same dot
    and pulse distributions, dt = 1e-3, 5000 steps, order 5 (the on-the-fly
    workload)."""
    dots = make_dots(n, side, seed, omega_sigma=0.5, dipole=None)
    return Workload(f"otf_N{n}_T{steps}", dots, make_pulse(delay=pulse_delay),
                    Constants(num_timesteps=steps), seed)


def max_delay_steps(dots: np.ndarray, c0: float, dt: float) -> int:
    """Upper bound of floor(|r_ij| / (c0 dt)) from the bounding box."""
    lo = dots[:, 0:3].min(axis=0)
    hi = dots[:, 0:3].max(axis=0)
    return int(math.floor(float(np.linalg.norm(hi - lo)) / (c0 * dt)))


# ---- reference file formats -------------------------------------------------

def write_dots_cfg(path: str, dots: np.ndarray) -> None:
    with open(path, "w") as f:
        for row in dots:
            f.write(" ".join("%.17g" % v for v in row) + "\n")


def read_dots_cfg(path: str, num_particles: Optional[int] = None) -> np.ndarray:
    """istream_iterator<QuantumDot> over whitespace-separated values
    (src/quantum_dot.cpp:40-47); then resize to num_particles (main.cpp:26),
    which pads with zero-initialised dots when the file is short."""
    vals = np.array(open(path).read().split(), dtype=np.float64)
    n_full = vals.size // 9
    dots = vals[: n_full * 9].reshape(n_full, 9)
    if num_particles is not None:
        if num_particles <= n_full:
            dots = dots[:num_particles]
        else:
            dots = np.vstack([dots, np.zeros((num_particles - n_full, 9))])
    return np.ascontiguousarray(dots)


def write_pulse_cfg(path: str, pulse: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write(" ".join("%.17g" % v for v in pulse) + "\n")


def read_pulse_cfg(path: str) -> np.ndarray:
    vals = np.array(open(path).read().split(), dtype=np.float64)
    if vals.size < 10:
        raise RuntimeError("Could not read pulse from " + path)
    return vals[:10].copy()


def read_input_cfg(path: str) -> tuple[Constants, int, str, str]:
    """The INI keys of parse_configs (src/configuration.cpp:17-42).  Returns
    (constants, num_particles, qd_path, pulse_path); num_timesteps is
    ceil(total_time / timestep) as in configuration.cpp:37-39."""
    section = ""
    kv = {}
    for raw in open(path):
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        if line.startswith("[") and line.endswith("]"):
            section = line[1:-1].strip()
            continue
        k, v = line.split("=", 1)
        kv[f"{section}.{k.strip()}"] = v.strip()
    required = ["constants.c0", "constants.hbar", "constants.mu0", "constants.laser_frequency",
                "parameters.num_particles", "parameters.total_time", "parameters.timestep",
                "parameters.interpolation_order"]
    for k in required:
        if k not in kv:
            raise RuntimeError(f"the option '{k}' is required but missing")
    dt = float(kv["parameters.timestep"])
    c = Constants(c0=float(kv["constants.c0"]), hbar=float(kv["constants.hbar"]),
                  mu0=float(kv["constants.mu0"]), laser_frequency=float(kv["constants.laser_frequency"]),
                  dt=dt, interpolation_order=int(kv["parameters.interpolation_order"]),
                  num_timesteps=int(math.ceil(float(kv["parameters.total_time"]) / dt)))
    return (c, int(kv["parameters.num_particles"]), kv.get("files.qd_path", "dots.cfg"),
            kv.get("files.pulse_path", "pulse.cfg"))


def write_input_cfg(path: str, c: Constants, num_particles: int, qd_path="dots.cfg",
                    pulse_path="pulse.cfg") -> None:
    with open(path, "w") as f:
        f.write("[files]\n")
        f.write(f"  qd_path = {qd_path}\n  pulse_path = {pulse_path}\n")
        f.write("[parameters]\n")
        f.write(f"  num_particles = {num_particles}\n")
        f.write(f"  total_time = {c.num_timesteps * c.dt:.17g}\n")
        f.write(f"  timestep = {c.dt:.17g}\n")
        f.write(f"  interpolation_order = {c.interpolation_order}\n")
        f.write("[constants]\n")
        f.write(f"  c0 = {c.c0:.17g}\n  hbar = {c.hbar:.17g}\n  mu0 = {c.mu0:.17g}\n")
        f.write(f"  laser_frequency = {c.laser_frequency:.17g}\n")


def read_output_dat(path: str) -> np.ndarray:
    """output.dat as History::write_history writes it (src/history.cpp:17-34):
    one line per step, each dot's rho00 and rho01 as "(re,im)".  Returns
    (T, N, 2) complex."""
    rows = []
    for line in open(path):
        toks = line.replace("(", " ").replace(")", " ").split()
        vals = [complex(float(a), float(b)) for a, b in (t.split(",") for t in toks)]
        rows.append(vals)
    arr = np.array(rows, dtype=np.complex128)
    return arr.reshape(arr.shape[0], -1, 2)


def load_pc_weights(path: str) -> tuple[np.ndarray, np.ndarray, float]:
    """Read a weight table: n_time, ps rows 0-1, cs rows 0-1, future_coef."""
    rows = [ln for ln in open(path) if ln.strip() and not ln.startswith("#")]
    n_time = int(rows[0])
    vals = [np.array(r.split(), dtype=np.float64) for r in rows[1:5]]
    ps = np.vstack(vals[0:2])
    cs = np.vstack(vals[2:4])
    assert ps.shape == (2, n_time) and cs.shape == (2, n_time)
    return ps, cs, float(rows[5])
