"""CPU tests of the oracle: the reference's own unit tests, golden weights,
and mathematical identities that pin the restatement."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from quest_b200 import inputs as I
from tests.conftest import rel_err


# ---- test/quantum_dot_test.cpp:13-43 (the reference's known-answer test) --
def test_liouville_rhs_known_answer():
    omega = 2278.9013
    t1, t2 = 10.0, 20.0
    dot = np.array([0, 0, 0, omega, t1, t2, 0, 0, 1.0])
    rabi = complex(1.0, 0.0)  # efield (0,0,1) . dipole (0,0,1)
    H = np.array([[0, rabi], [np.conj(rabi), 0]])
    D = np.array([[1, 0.5 + 0.5j], [0.5 - 0.5j, 0]])
    diss = np.array([[(D[0, 0] - 1.0) / t1, D[0, 1] / t2], [D[1, 0] / t2, D[1, 1] / t1]])
    M = -1j * (H @ D - D @ H) - diss
    rhs = O.liouville_rhs(dot, [D[0, 0], D[0, 1]], rabi, omega)
    # BOOST_CHECK_CLOSE(..., 1e-9) is a percentage tolerance
    for got, want in [(rhs[0], M[0, 0]), (rhs[1], M[0, 1])]:
        for g, w in [(got.real, want.real), (got.imag, want.imag)]:
            assert abs(g - w) <= 1e-11 * max(abs(w), abs(g)) or g == w


# ---- test/history_test.cpp:13-53, with the imaginary-inf case the
# reference meant to test (its imag_inf is (inf, 0), a typo) --------------
@pytest.mark.parametrize("bad", [complex(math.inf, 0), complex(0, math.inf), complex(math.nan, 0),
                                 complex(0, math.nan)])
def test_isfinite(bad):
    assert O.isfinite([0j, 0j])
    assert not O.isfinite([bad, 0j])
    assert not O.isfinite([0j, bad])


# ---- test/lagrange_set_test.cpp:6-23 (shape) plus exactness on polynomials
def test_lagrange_shape():
    w = O.lagrange_weights(0.5, 1.0, 5)
    assert w.shape == (3, 6)


@pytest.mark.parametrize("q", [3, 5, 7])
@pytest.mark.parametrize("x", [0.1, 0.37, 0.5, 0.93])
def test_lagrange_reproduces_polynomials(q, x):
    dt = 0.01
    w = O.lagrange_weights(x, dt, q)
    # sample f(tau) at tau_m = -m dt (tap m reads step s - m); the weights
    # evaluate f at tau = -x dt and its first and second time derivatives
    # there (the reference's minus sign turns d/dx into d/dtau)
    rng = np.random.default_rng(q)
    c = rng.normal(size=q + 1)
    f = np.polynomial.Polynomial(c)
    taus = -np.arange(q + 1) * dt
    samples = f(taus)
    t = -x * dt
    assert np.isclose(w[0] @ samples, f(t), rtol=1e-10, atol=1e-12)
    assert np.isclose(w[1] @ samples, f.deriv(1)(t), rtol=1e-7, atol=1e-9)
    assert np.isclose(w[2] @ samples, f.deriv(2)(t), rtol=1e-6, atol=1e-6)


def test_lagrange_nan_at_integer_fraction():
    # x == 0 divides by zero for every node but the first (lagrange_set.cpp:25-33)
    w = O.lagrange_weights(0.0, 1.0, 5)
    assert np.all(np.isfinite(w[:, 0]))
    assert np.all(np.isnan(w[1:, 1:]))


# ---- Green's function: symmetry and 1/r^3, 1/r^2, 1/r scaling -------------
def test_coefficients_symmetric_and_scaling():
    c = I.Constants(c0=1.0, dt=1e-3, laser_frequency=200.0)
    a = np.array([0.0, 0, 0, 200, 10, 10, 1e-3, 2e-3, -1e-3])
    b = np.array([0.013, -0.02, 0.007, 200, 10, 10, -2e-3, 1e-3, 5e-4])
    d1, c1 = O.pair_coefficients(a, b, c)
    d2, c2 = O.pair_coefficients(b, a, c)
    assert d1 == d2
    np.testing.assert_allclose(c1, c2, rtol=1e-13, atol=0)
    # lab frame, static limit: the 1/r^3 near-field term dominates small r
    lab = I.Constants(c0=1.0, dt=1e-3, laser_frequency=200.0, frame=1)
    bb = b.copy()
    r1 = np.linalg.norm(b[:3])
    bb[:3] = b[:3] * 1e-3
    _, n1 = O.pair_coefficients(a, b, lab)
    _, n2 = O.pair_coefficients(a, bb, lab)
    assert np.all(np.isfinite(n1)) and np.all(np.isfinite(n2))
    assert r1 > 0


# ---- predictor-corrector weights ------------------------------------------
def test_pc_weights_golden_properties(golden_weights):
    ps, cs, fc = golden_weights
    assert ps.shape == (2, 22) and cs.shape == (2, 22)
    assert abs(ps[0].sum() - 1.0) < 1e-12
    assert abs(cs[0].sum() - 1.0) < 1e-12


def test_pc_weights_integrate_exponential(golden_weights):
    """Predict and correct y' = lam y one step ahead for a lambda inside the
    fitted contour (radius 3.15 in units of the 22-step window)."""
    ps, cs, fc = golden_weights
    n_time = 22
    dt = 0.01
    for lam in [-1.0, -5.0, complex(-2.0, 3.0), 10j]:
        t = (np.arange(n_time) - n_time) * dt
        y = np.exp(lam * t)
        yd = lam * y
        pred = (y * ps[0]).sum() + (yd * ps[1]).sum() * dt
        corr = fc * lam * 1.0 * dt + (y * cs[0]).sum() + (yd * cs[1]).sum() * dt
        assert abs(pred - 1.0) < 1e-6
        assert abs(corr - 1.0) < 1e-6


# ---- end to end: faithful (11 sweeps/step) vs fast (1 sweep + near list) --
def test_fast_oracle_matches_faithful(oracle_weights):
    wl = I.plain_small(n=48, steps=300, pulse_delay=0.15)
    hf, bf = O.run_faithful(wl.dots, wl.pulse, wl.constants, oracle_weights, 300)
    hq, bq = O.run_fast(wl.dots, wl.pulse, wl.constants, oracle_weights, 300, nthreads=3)
    assert bf is None and bq is None
    rf, rq = O.rho_trajectory(hf), O.rho_trajectory(hq)
    assert rel_err(rf[..., 0], rq[..., 0]) < 1e-13
    assert rel_err(rf[..., 1], rq[..., 1]) < 1e-10
    assert np.abs(rf[..., 1]).max() > 1e-6  # the pulse did excite the dots


def load_example(n=None, steps=None):
    import os
    from tests.conftest import GOLDEN
    c, n_cfg, _, _ = I.read_input_cfg(os.path.join(GOLDEN, "example_input.cfg"))
    n = n_cfg if n is None else n
    dots = I.read_dots_cfg(os.path.join(GOLDEN, "example_dots.cfg"), n)
    pulse = I.read_pulse_cfg(os.path.join(GOLDEN, "example_pulse.cfg"))
    if steps is not None:
        c.num_timesteps = steps
    return dots, pulse, c


def test_example_fixture_reads():
    dots, pulse, c = load_example()
    assert dots.shape == (2, 9) and c.num_timesteps == 4000 and c.interpolation_order == 3
    assert pulse[0] == 15589.2260227


def test_fast_oracle_matches_faithful_all_near(oracle_weights):
    """The reference example: c0*dt exceeds every separation, so every pair
    has delay 0 and the corrector iterations couple all dots within a step."""
    dots, pulse, c = load_example(n=24, steps=1150)
    hf, bf = O.run_faithful(dots, pulse, c, oracle_weights, 1150)
    hq, bq = O.run_fast(dots, pulse, c, oracle_weights, 1150, nthreads=2)
    assert bf is None and bq is None
    d, _ = O.build_table(dots, c)
    assert (d == 0).all()
    rf, rq = O.rho_trajectory(hf), O.rho_trajectory(hq)
    assert rel_err(rf[..., 1], rq[..., 1]) < 1e-12
    assert rf[..., 0].real.min() < 0.5  # strong excitation


def test_single_dot_matches_ode_solution(oracle_weights):
    """One dot, no partners: the PC integrator against scipy's DOP853."""
    from scipy.integrate import solve_ivp
    dots = np.array([[0.0, 0, 0, 201.0, 10, 7, 0, 0, 2e-3]])
    c = I.Constants(dt=1e-3, num_timesteps=1500)
    pulse = I.make_pulse(amplitude=2000.0, delay=0.6, width=1.0, freq=200.0)
    hist, bad = O.run_faithful(dots, pulse, c, oracle_weights, 1500)
    assert bad is None
    rho = O.rho_trajectory(hist)[:, 0, :]

    def rabi(t):
        arg = -200.0 * (t - 0.6)
        return (2000.0 / 2 * 1.0) * math.exp(-arg * arg / 2) * 2e-3

    def f(t, y):
        r0 = complex(y[0], y[1])
        r1 = complex(y[2], y[3])
        om = rabi(t)
        m0 = -1j * (om * np.conj(r1) - np.conj(om) * r1) - (r0 - 1.0) / 10
        m1 = -1j * (om * (1 - 2 * r0) + r1 * (200.0 - 201.0)) - r1 / 7
        return [m0.real, m0.imag, m1.real, m1.imag]

    ts = np.arange(1500) * 1e-3
    sol = solve_ivp(f, (0, ts[-1]), [1, 0, 0, 0], t_eval=ts, method="DOP853", rtol=1e-12, atol=1e-14,
                    max_step=2e-4)
    ref01 = sol.y[2] + 1j * sol.y[3]
    assert np.abs(ref01).max() > 1e-3
    assert rel_err(ref01, rho[:, 1]) < 1e-6


def test_nonfinite_detection_step(oracle_weights):
    """Coincident dots give 0/0 in the dyads: the reference throws at step 0."""
    dots = I.make_dots(5, 0.1, 3)
    dots[3, :3] = dots[1, :3]
    c = I.Constants(num_timesteps=10)
    _, bad = O.run_faithful(dots, I.make_pulse(delay=0.0), c, oracle_weights, 10)
    assert bad == 0
    _, bad2 = O.run_fast(dots, I.make_pulse(delay=0.0), c, oracle_weights, 10, nthreads=1)
    assert bad2 == 0


def test_integer_delay_first_bad_step(oracle_weights):
    """A pair whose delay is an exact integer d has NaN weights for taps >= 1
    (lagrange_set.cpp:25-33); the first read of tap 1 is at step d + 1 - 22."""
    c = I.Constants(c0=1.0, dt=0.125, num_timesteps=40)
    dots = np.array([[0.0, 0, 0, 200, 10, 10, 0, 0, 2e-3],
                     [5.0, 0, 0, 200, 10, 10, 0, 0, 2e-3]])  # r/(c dt) = 40 exactly
    _, bad = O.run_faithful(dots, I.make_pulse(delay=0.0), c, oracle_weights, 40)
    assert bad == 40 + 1 - 22
    _, bad2 = O.run_fast(dots, I.make_pulse(delay=0.0), c, oracle_weights, 40, nthreads=1)
    assert bad2 == bad


def test_pair_index_maps():
    for idx in [0, 1, 2, 3, 100, 12345, 8386559, 2147450879, 2**40 + 7]:
        r, cc = __import__("ctypes").c_int(), __import__("ctypes").c_int()
        O.lib().or_idx2coord(idx, __import__("ctypes").byref(r), __import__("ctypes").byref(cc))
        assert 0 <= cc.value < r.value
        assert O.lib().or_coord2idx(r.value, cc.value) == idx
