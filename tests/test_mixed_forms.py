"""Two ways to sum one pair's taps in FP32, measured against FP64 on CPU.

A far pair's contribution to output k is sum_i c_i w_{k+q-i}
(history_interaction.cpp:55-65): q+1 = 6 taps whose coefficients carry the
Lagrange weights w0 ~ 1, w1 ~ 1/dt and w2 ~ 1/dt^2 (lagrange_set.cpp:17-41),
applied to a slowly varying rho01 history.  With dt = 1e-3 the taps are
orders of magnitude larger than their sum, so the exact result is a
near-total cancellation.

* Compensated accumulation: taps and samples stored in FP32, every product
  made error-free (TwoProduct, Veltkamp split) and summed with TwoSum
  (Ogita, Rump and Oishi's Dot2), i.e. the sum is as good as a
  double-length computation on the FP32 inputs.  The error that remains is
  the rounding of the inputs to FP32: each tap's ~6e-8 relative error meets
  a product far larger than the result.
* The difference form the library uses (qg_conv.cuh, MixedAcc): the tap
  sum (sum_i c_i, formed in FP64) times the window's first sample, plus the
  taps times the running sum of the step-to-step differences (formed in
  FP64, stored in FP32), all with plain FP32 multiply-adds.  The large
  weights meet only the small differences.

Every operation below is an IEEE float32 operation in numpy, so this is the
arithmetic the kernels do, and the numbers are reproducible anywhere.  The
difference form is both cheaper (one multiply-add per term against about
ten for Dot2's error-free transformations) and about two orders of
magnitude more accurate on these inputs (measured: 2.5e-5 against 2.7e-7
worst relative error of one pair's 16 outputs).
"""
import numpy as np

from oracle import oracle as O
from quest_b200 import inputs as I

f32 = np.float32


def two_sum(a, b):
    s = f32(a + b)
    bb = f32(s - a)
    return s, f32(f32(a - f32(s - bb)) + f32(b - bb))


def split(a):
    c = f32(f32(4097.0) * a)
    hi = f32(c - f32(c - a))
    return hi, f32(a - hi)


def two_prod(a, b):
    p = f32(a * b)
    ah, al = split(a)
    bh, bl = split(b)
    e = f32(f32(f32(f32(ah * bh) - p) + f32(ah * bl)) + f32(al * bh)) + f32(al * bl)
    return p, f32(e)


def dot2(xs, ys):
    """Compensated FP32 dot product (Dot2) of real sequences."""
    s, c = f32(0), f32(0)
    for x, y in zip(xs, ys):
        p, q = two_prod(f32(x), f32(y))
        s, r = two_sum(s, p)
        c = f32(c + f32(q + r))
    return f32(s + c)


def complex_dot2(c, w):
    """sum_i c_i w_i for complex FP32 inputs, each real product through Dot2."""
    re = dot2([*c.real, *(-c.imag)], [*w.real, *w.imag])
    im = dot2([*c.real, *c.imag], [*w.imag, *w.real])
    return complex(re, im)


def difference_form(c64, w64, K, q):
    """The kernel's arithmetic for K outputs: FP32 taps and tap sum (the sum
    formed in FP64), FP32 first sample and FP32 differences (formed in
    FP64), plain FP32 multiply-adds (numpy rounds each product and each sum,
    which is what separate fmaf rounding differs from by at most one ulp per
    operation)."""
    c = c64.astype(np.complex64)
    csum = np.complex64(c64.sum())
    w0 = np.complex64(w64[0])
    d = (w64[1:] - w64[:-1]).astype(np.complex64)
    base = np.complex64(csum * w0)
    out = np.zeros(K, dtype=np.complex64)
    u = np.complex64(0)
    for m in range(1, K + q):
        u = np.complex64(u + d[m - 1])
        for k in range(max(m - q, 0), min(m, K - 1) + 1):
            out[k] = np.complex64(out[k] + np.complex64(c[k + q - m] * u))
    return out.astype(np.complex128) + complex(base)


def test_difference_form_beats_compensated_fp32_accumulation(oracle_weights):
    q, K = 5, 16
    wl = I.plain_table(seed=2, n=64, steps=10)
    c = wl.constants
    rng = np.random.default_rng(3)
    worst_dot2, worst_diff = 0.0, 0.0
    for trial in range(24):
        a, b = rng.choice(wl.n, size=2, replace=False)
        d, coef = O.pair_coefficients(wl.dots[max(a, b)], wl.dots[min(a, b)], c)
        if d < 16:
            continue
        # a rho01 history of the kind the bench sees: a slow rotating-frame
        # oscillation (detuning ~ 0.5 rad per unit time) plus small noise
        t = np.arange(K + q) * c.dt
        amp = 1e-2 * (rng.normal() + 1j * rng.normal())
        w = amp * np.exp(1j * (0.5 * t + rng.uniform(0, 6.3))) * (1 + 1e-3 * rng.normal(size=K + q))
        exact = np.array([sum(coef[i] * w[k + q - i] for i in range(q + 1)) for k in range(K)])
        scale = np.abs(exact).max()
        comp = np.array([complex_dot2(coef[::-1].astype(np.complex64),
                                      w[k: k + q + 1].astype(np.complex64)) for k in range(K)])
        diff = difference_form(coef, w, K, q)
        worst_dot2 = max(worst_dot2, float(np.abs(comp - exact).max() / scale))
        worst_diff = max(worst_diff, float(np.abs(diff - exact).max() / scale))
    print(f"worst relative error: compensated FP32 {worst_dot2:.2e}, difference form {worst_diff:.2e}")
    # input rounding to FP32, amplified by the cancellation, bounds the
    # compensated sum; the difference form stays near FP32 resolution
    assert worst_dot2 > 1e-5
    assert worst_diff < 1e-6
    assert worst_dot2 > 30 * worst_diff
