// Predictor-corrector weight fit, PredictorCorrector::Weights
// (reference src/integrator.cpp:5-102).
//
// The reference builds an n_lambda x (2 n_time [+1]) complex system from
// contour points lambda_j on a semidisk and solves it in the least-squares
// sense with Eigen's JacobiSVD, keeping the real part.  The system has full
// row rank but a condition number near 3e13, so the answer of any
// double-precision solver is only good to about three digits.  This file
// computes the exact minimum-norm solution x = A^H (A A^H)^{-1} b through a
// Householder QR factorisation of A^H in IEEE binary128 (libquadmath), whose
// error (about 1e-34 * 3e13) is far below double rounding, then rounds to
// double.  The inputs are the mathematical ones: x_j = j (pi + 2) / n_lambda,
// t_k = -1 + 2k / (n_time - 1), with radius taken as the given double.
#include <quadmath.h>

#include <cstring>
#include <vector>

#include "../../include/quest_gpu.h"
#include "qg_internal.h"

namespace {

typedef __float128 qf;

struct qc {
  qf re, im;
};
inline qc operator+(qc a, qc b) { return {a.re + b.re, a.im + b.im}; }
inline qc operator-(qc a, qc b) { return {a.re - b.re, a.im - b.im}; }
inline qc operator*(qc a, qc b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline qc operator*(qf s, qc a) { return {s * a.re, s * a.im}; }
inline qc conj(qc a) { return {a.re, -a.im}; }
inline qf abs2(qc a) { return a.re * a.re + a.im * a.im; }
inline qc div(qc a, qc b)
{
  const qf d = abs2(b);
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
inline qc cexp_q(qc z)
{
  const qf e = expq(z.re);
  return {e * cosq(z.im), e * sinq(z.im)};
}

// semidisk contour, integrator.cpp:5-14
qc semidisk(qf t)
{
  const qf pi = M_PIq;
  if(0 <= t && t < 1) return {0, t};
  if(1 <= t && t < pi + 1) return cexp_q({0, t + pi / 2 - 1});
  if(pi + 1 <= t && t < pi + 2) return {0, t - (pi + 2)};
  return {0, 0};
}

// Minimum-norm solution of A x = b for a full-row-rank m x n (m < n) matrix
// stored row-major.  QR of B = A^H (n x m) by Householder reflections; then
// R^H y = b by forward substitution and x = Q [y; 0].
std::vector<qc> min_norm(const std::vector<qc> &A, int m, int n, const std::vector<qc> &b)
{
  std::vector<qc> B((size_t)n * m);  // B[i*m + j] = conj(A[j*n + i])
  for(int i = 0; i < n; ++i)
    for(int j = 0; j < m; ++j) B[(size_t)i * m + j] = conj(A[(size_t)j * n + i]);
  std::vector<std::vector<qc>> U(m);
  std::vector<qc> Rdiag(m);
  for(int k = 0; k < m; ++k) {
    qf nrm2 = 0;
    for(int i = k; i < n; ++i) nrm2 += abs2(B[(size_t)i * m + k]);
    const qf nrm = sqrtq(nrm2);
    const qc x0 = B[(size_t)k * m + k];
    const qf a0 = sqrtq(abs2(x0));
    qc phase = (a0 > 0) ? qc{x0.re / a0, x0.im / a0} : qc{1, 0};
    const qc alpha = (-nrm) * phase;
    std::vector<qc> u(n - k);
    for(int i = k; i < n; ++i) u[i - k] = B[(size_t)i * m + k];
    u[0] = u[0] - alpha;
    qf uu = 0;
    for(auto &e : u) uu += abs2(e);
    // apply H = I - 2 u u^H / (u^H u) to columns k..m-1
    for(int j = k; j < m; ++j) {
      qc s = {0, 0};
      for(int i = k; i < n; ++i) s = s + conj(u[i - k]) * B[(size_t)i * m + j];
      const qc f = (qf(2) / uu) * s;
      for(int i = k; i < n; ++i) B[(size_t)i * m + j] = B[(size_t)i * m + j] - u[i - k] * f;
    }
    Rdiag[k] = B[(size_t)k * m + k];
    U[k] = u;
  }
  // R^H y = b: y_i = (b_i - sum_{j<i} conj(R_ji) y_j) / conj(R_ii)
  std::vector<qc> y(m);
  for(int i = 0; i < m; ++i) {
    qc s = b[i];
    for(int j = 0; j < i; ++j) s = s - conj(B[(size_t)j * m + i]) * y[j];
    y[i] = div(s, conj(Rdiag[i]));
  }
  std::vector<qc> x(n, qc{0, 0});
  for(int i = 0; i < m; ++i) x[i] = y[i];
  for(int k = m - 1; k >= 0; --k) {
    const auto &u = U[k];
    qf uu = 0;
    for(auto &e : u) uu += abs2(e);
    qc s = {0, 0};
    for(int i = k; i < n; ++i) s = s + conj(u[i - k]) * x[i];
    const qc f = (qf(2) / uu) * s;
    for(int i = k; i < n; ++i) x[i] = x[i] - u[i - k] * f;
  }
  return x;
}

}  // namespace

extern "C" qg_status qg_pc_weights(int n_lambda, int n_time, double radius, qg_weights *out)
{
  if(!out) return qg_fail(QG_ERR_INVALID_ARG, "qg_pc_weights: out is NULL");
  if(n_time < 2 || n_time > 32)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_pc_weights: n_time must be in [2, 32]");
  if(n_lambda < 1 || n_lambda >= 2 * n_time)
    return qg_fail(QG_ERR_INVALID_ARG,
                   "qg_pc_weights: need 1 <= n_lambda < 2*n_time (underdetermined fit)");
  if(!(radius > 0))
    return qg_fail(QG_ERR_INVALID_ARG, "qg_pc_weights: radius must be positive");

  const qf pi = M_PIq;
  std::vector<qc> lambdas(n_lambda);
  for(int j = 0; j < n_lambda; ++j) {
    const qf xj = qf(j) * (pi + 2) / qf(n_lambda);
    lambdas[j] = qf(radius) * semidisk(xj);
  }
  std::vector<qf> times(n_time);
  for(int k = 0; k < n_time; ++k) times[k] = qf(-1) + qf(2) * qf(k) / qf(n_time - 1);
  const qf future = 1 + qf(2) / qf(n_time - 1);

  const int np = 2 * n_time, nc = 2 * n_time + 1;
  std::vector<qc> P((size_t)n_lambda * np), C((size_t)n_lambda * nc), rhs(n_lambda);
  for(int j = 0; j < n_lambda; ++j) {
    const qc lam = lambdas[j];
    for(int k = 0; k < n_time; ++k) {
      const qc e = cexp_q(times[k] * lam);
      P[(size_t)j * np + k] = e;
      P[(size_t)j * np + n_time + k] = lam * e;
      C[(size_t)j * nc + k] = e;
      C[(size_t)j * nc + n_time + k] = lam * e;
    }
    rhs[j] = cexp_q(future * lam);
    C[(size_t)j * nc + 2 * n_time] = lam * rhs[j];
  }
  const std::vector<qc> p = min_norm(P, n_lambda, np, rhs);
  const std::vector<qc> c = min_norm(C, n_lambda, nc, rhs);
  const qf step_factor = qf(n_time - 1) / 2;

  std::memset(out, 0, sizeof *out);
  out->n_time = n_time;
  for(int k = 0; k < n_time; ++k) {
    out->ps[k] = (double)p[k].re;
    out->ps[n_time + k] = (double)(p[n_time + k].re * step_factor);
    out->cs[k] = (double)c[k].re;
    out->cs[n_time + k] = (double)(c[n_time + k].re * step_factor);
  }
  out->future_coef = (double)(c[2 * n_time].re * step_factor);
  return QG_OK;
}
