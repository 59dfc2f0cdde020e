"""Generate the frozen predictor-corrector weight table with mpmath.

The reference fits its multistep weights by a complex least-squares problem
(src/integrator.cpp:5-102, PredictorCorrector::Weights / WeightsBuilder):

* 18 contour points lambda_j = radius * semidisk(x_j), x_j = j*(pi+2)/n_lambda
  (integrator.cpp:5-14, 41-42);
* n_time = 22 nodes t_k = -1 + 2k/(n_time-1) (integrator.cpp:37);
* predictor matrix [exp(lambda t), lambda exp(lambda t)] (integrator.cpp:45-56);
* corrector matrix adds the column lambda*exp(lambda*(1+h)) (integrator.cpp:58-67);
* right-hand side exp(lambda*(1+h)) (integrator.cpp:69-73);
* minimum-norm solution, real part (integrator.cpp:75-83);
* reshape to 2 x n_time and scale the derivative row by (n_time-1)/2
  (integrator.cpp:85-102).

The system is ill-conditioned (condition number about 3e13), so double
precision solvers disagree in the third significant digit.  This script solves
the exact mathematical problem at 80 significant digits and writes the result
rounded to double with 17 significant digits.  Both the oracle and the CUDA
library's own quad-precision solver are checked against this file.

Usage: python tests/golden/make_pc_weights.py [n_lambda n_time radius]
"""
import sys

import mpmath as mp

mp.mp.dps = 80


def semidisk(t):
    pi = mp.pi
    if 0 <= t < 1:
        return mp.mpc(0, t)
    if 1 <= t < pi + 1:
        return mp.exp(mp.mpc(0, 1) * (t + pi / 2 - 1))
    if pi + 1 <= t < pi + 2:
        return mp.mpc(0, 1) * (t - (pi + 2))
    return mp.mpc(0)


def min_norm_solve(A, b):
    # x = A^H (A A^H)^{-1} b; exact enough at 80 digits (cond^2 ~ 1e27).
    AH = A.transpose_conj()
    return AH * mp.lu_solve(A * AH, b)


def weights(n_lambda=18, n_time=22, radius=3.15):
    radius = mp.mpf(float(radius))  # the double the C API receives
    xs = [mp.mpf(j) * (mp.pi + 2) / n_lambda for j in range(n_lambda + 1)]
    lambdas = [radius * semidisk(xs[j]) for j in range(n_lambda)]
    times = [mp.mpf(-1) + mp.mpf(2) * k / (n_time - 1) for k in range(n_time)]
    h = mp.mpf(2) / (n_time - 1)
    future = 1 + h
    P = mp.matrix(n_lambda, 2 * n_time)
    C = mp.matrix(n_lambda, 2 * n_time + 1)
    rhs = mp.matrix(n_lambda, 1)
    for j, lam in enumerate(lambdas):
        for k, t in enumerate(times):
            e = mp.exp(lam * t)
            P[j, k] = e
            P[j, n_time + k] = lam * e
            C[j, k] = e
            C[j, n_time + k] = lam * e
        rhs[j] = mp.exp(lam * future)
        C[j, 2 * n_time] = lam * rhs[j]
    p = min_norm_solve(P, rhs)
    c = min_norm_solve(C, rhs)
    step_factor = mp.mpf(n_time - 1) / 2
    ps = [[mp.re(p[k]) for k in range(n_time)],
          [mp.re(p[n_time + k]) * step_factor for k in range(n_time)]]
    cs = [[mp.re(c[k]) for k in range(n_time)],
          [mp.re(c[n_time + k]) * step_factor for k in range(n_time)]]
    fc = mp.re(c[2 * n_time]) * step_factor
    return ps, cs, fc


def main():
    args = sys.argv[1:]
    n_lambda, n_time, radius = (18, 22, "3.15") if not args else (int(args[0]), int(args[1]), args[2])
    # the radius enters as the IEEE double nearest to the given decimal
    ps, cs, fc = weights(n_lambda, n_time, radius)
    out = f"tests/golden/pc_weights_{n_lambda}_{n_time}_{radius}.txt"
    with open(out, "w") as f:
        f.write(f"# predictor-corrector weights n_lambda={n_lambda} n_time={n_time} radius={radius}\n")
        f.write("# generated by tests/golden/make_pc_weights.py (mpmath, 80 digits, min-norm solve)\n")
        f.write("# layout: n_time, then ps row 0, ps row 1, cs row 0, cs row 1 (n_time values each), then future_coef\n")
        f.write(f"{n_time}\n")
        for row in ps + cs:
            f.write(" ".join("%.17g" % float(v) for v in row) + "\n")
        f.write("%.17g\n" % float(fc))
    print("wrote", out)


if __name__ == "__main__":
    main()
