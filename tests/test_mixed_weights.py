"""The algebra behind the mixed on-the-fly kernel's FP32 Lagrange weights
(pair_coef_otf_mixed): with e_k the elementary symmetric polynomials of
{x - m : m != b} and den = prod_{m != b} (b - m), the reference's weights
(lagrange_set.cpp:17-41) are w0 = e_Q / den, w1 = -e_{Q-1} / (den dt) and
w2 = 2 e_{Q-2} / (den dt^2).  Checked here against the reference's formula
evaluated in 50-digit arithmetic: the symmetric form in FP64 and in FP32 (the
kernel's operation order), the identities sum w0 = 1, sum w1 = sum w2 = 0
that give the tap sum, and the reference's NaN pattern at x = 0."""
import mpmath
import numpy as np
import pytest


def exact_weights(x, q, dt):
    """The reference's formula in 50-digit arithmetic (x given as a double)."""
    with mpmath.workdps(50):
        x = mpmath.mpf(x)
        w = np.zeros((3, q + 1))
        for b in range(q + 1):
            d0, d1, d2 = mpmath.mpf(1), mpmath.mpf(0), mpmath.mpf(0)
            for m in range(q + 1):
                if m == b:
                    continue
                d0 *= (x - m) / (b - m)
                d1 -= 1 / (x - m)
                d2 -= (x - m) ** -2
            w1 = d0 * d1
            w[0, b] = float(d0)
            w[1, b] = float(w1 / dt)
            w[2, b] = float((d0 * d2 + w1 ** 2 / d0) / dt ** 2)
        return w


def reference_weights(x, q, dt):
    w = np.zeros((3, q + 1))
    for b in range(q + 1):
        d0, d1, d2 = 1.0, 0.0, 0.0
        for m in range(q + 1):
            if m == b:
                continue
            d0 *= (x - m) / (b - m)
            d1 -= 1 / (x - m) if x != m else np.inf
            d2 -= (x - m) ** -2.0 if x != m else np.inf
        w[0, b] = d0
        with np.errstate(invalid="ignore", divide="ignore"):
            w[1, b] = d0 * d1
            w[2, b] = d0 * d2 + w[1, b] ** 2 / d0
    w[1] /= dt
    w[2] /= dt ** 2
    return w


def symmetric_weights(x, q, dt, dtype):
    f = dtype
    x = f(x)
    inv_dt = f(1.0 / dt)
    w = np.zeros((3, q + 1), dtype=dtype)
    for b in range(q + 1):
        e = [f(1)] + [f(0)] * q
        n = 0
        for m in range(q + 1):
            if m == b:
                continue
            fm = f(x - f(m))
            n += 1
            for k in range(q, 0, -1):
                if k <= n:
                    e[k] = f(f(fm * e[k - 1]) + e[k])  # one fused multiply-add in the kernel
        den = f(1)
        for m in range(q + 1):
            if m != b:
                den = f(den * f(b - m))
        idn = f(f(1) / den)
        w[0, b] = f(e[q] * idn)
        w[1, b] = f(-f(e[q - 1] * idn) * inv_dt)
        w[2, b] = f(f(f(2) * f(e[q - 2] * idn)) * f(inv_dt * inv_dt)) if q >= 2 else f(0)
    return w


@pytest.mark.parametrize("q", [2, 3, 5, 7])
def test_symmetric_form_equals_the_reference_formula(q):
    """Against the reference's formula evaluated exactly: the symmetric form
    in FP64 is within 1e-14 of the largest weight everywhere, the formula
    itself in FP64 only away from the nodes (near x = 1 its w0 d2 + w1^2/w0
    cancels)."""
    rng = np.random.default_rng(11)
    for x in list(rng.random(100)) + [0.5, 0.999999, 1e-3, 1e-7]:
        ex = exact_weights(x, q, 1e-3)
        got = symmetric_weights(x, q, 1e-3, np.float64)
        for j in range(3):
            scale = np.abs(ex[j]).max()
            assert np.abs(got[j] - ex[j]).max() <= 1e-14 * scale, (q, x, j)
    ex = exact_weights(0.999999, q, 1e-3)
    ref = reference_weights(0.999999, q, 1e-3)
    assert np.abs(ref[2] - ex[2]).max() > 1e-12 * np.abs(ex[2]).max()


@pytest.mark.parametrize("q", [3, 5, 7])
def test_fp32_weights_within_a_few_ulps_of_the_largest(q):
    rng = np.random.default_rng(12)
    worst = 0.0
    for x in list(rng.random(200)) + [1e-6, 1e-4, 0.999]:
        ref = exact_weights(x, q, 1e-3)
        got = symmetric_weights(x, q, 1e-3, np.float32).astype(np.float64)
        for j in range(3):
            worst = max(worst, np.abs(got[j] - ref[j]).max() / np.abs(ref[j]).max())
    assert worst < 2e-6, worst  # about 10 FP32 ulps of the largest weight


@pytest.mark.parametrize("q", [3, 5])
def test_tap_sum_identities(q):
    for x in (0.1, 0.37, 0.9):
        w = symmetric_weights(x, q, 1e-3, np.float64)
        assert abs(w[0].sum() - 1.0) < 1e-13
        assert abs(w[1].sum()) < 1e-12 * np.abs(w[1]).max()
        assert abs(w[2].sum()) < 1e-12 * np.abs(w[2]).max()


def test_reference_nan_pattern_at_an_integer_delay():
    """At x = 0 the reference's node-0 weights are finite and every other
    node's w1 and w2 are NaN (0 * inf); the kernel sets those taps (and the
    tap sum) to NaN and keeps tap 0."""
    ref = reference_weights(0.0, 5, 1e-3)
    assert np.all(np.isfinite(ref[:, 0]))
    assert np.all(np.isnan(ref[1:, 1:]))
    got = symmetric_weights(0.0, 5, 1e-3, np.float64)
    np.testing.assert_allclose(got[:, 0], ref[:, 0], rtol=1e-13)
