/*
 * CPU oracle for the QuEST retarded-interaction time step.
 * TEST INFRASTRUCTURE ONLY -- see quest_oracle.h for its role and for what
 * its parity is pinned against.  Compile with -ffp-contract=off.
 *
 * Complex numbers are pairs of doubles.  Each complex expression of the
 * reference is expanded into the real operations std::complex<double> and
 * Eigen perform for finite operands: (a+bi)(c+di) = (ac-bd) + (ad+bc)i,
 * complex*real scales both parts, complex/real divides both parts, and Eigen
 * reductions over 3-vectors sum left to right.
 */
#include "quest_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define WINDOW 22 /* main.cpp:30 make_shared_history(N, 22, T) */
#define NUM_CORRECTOR_STEPS 10 /* integrator.cpp:3 */

int or_window(void) { return WINDOW; }

typedef struct {
  double re, im;
} cx;

static inline cx cmul(cx a, cx b)
{
  cx r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.re * b.im + a.im * b.re;
  return r;
}
static inline cx cadd(cx a, cx b)
{
  cx r = {a.re + b.re, a.im + b.im};
  return r;
}
static inline cx cscale(cx a, double s)
{
  cx r = {a.re * s, a.im * s};
  return r;
}

/* ---- lagrange_set.cpp:17-41 ------------------------------------------- */
void or_lagrange_weights(double x, double dt, int q, double *w)
{
  const int n = q + 1;
  for(int b = 0; b <= q; ++b) {
    double d0 = 1, d1 = 0, d2 = 0;
    for(int m = 0; m <= q; ++m) {
      if(m == b) continue;
      d0 *= (x - m) / (double)(b - m);
      d1 -= 1 / (x - m);
      d2 -= pow(x - m, -2);
    }
    w[0 * n + b] = d0;
    w[1 * n + b] = w[0 * n + b] * d1;
    w[2 * n + b] = w[0 * n + b] * d2 + pow(w[1 * n + b], 2) / w[0 * n + b];
  }
  for(int i = 0; i <= q; ++i) {
    w[1 * n + i] *= pow(dt, -1);
    w[2 * n + i] *= pow(dt, -2);
  }
}

/* ---- green_function.h:32-55: the three spatial dyads ------------------ */
static void spatial_dyads(const double dr[3], double c, double dy[3][9])
{
  const double sq = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
  const double nrm = sqrt(sq);
  const double c2 = pow(c, 2);
  const double n3 = pow(nrm, 3);
  for(int r = 0; r < 3; ++r) {
    for(int k = 0; k < 3; ++k) {
      const double rhat = (dr[r] * dr[k]) / sq;  /* rhat_dyadic */
      const double id = (r == k) ? 1.0 : 0.0;
      const double i3 = id - 3 * rhat;           /* identity_minus_3rsq */
      const double i1 = id - rhat;               /* identity_minus_rsq */
      dy[0][3 * r + k] = (i3 * c2) / n3;
      dy[1][3 * r + k] = (i3 * c) / sq;
      dy[2][3 * r + k] = i1 / nrm;
    }
  }
}

/* d_obs . (M * d_src) for a complex 3x3 M (history_interaction.cpp:41-42). */
static cx contract(const double dobs[3], const cx M[9], const double dsrc[3])
{
  cx v[3];
  for(int r = 0; r < 3; ++r) {
    cx acc = cscale(M[3 * r + 0], dsrc[0]);
    acc = cadd(acc, cscale(M[3 * r + 1], dsrc[1]));
    acc = cadd(acc, cscale(M[3 * r + 2], dsrc[2]));
    v[r] = acc;
  }
  cx out = cscale(v[0], dobs[0]);
  out = cadd(out, cscale(v[1], dobs[1]));
  out = cadd(out, cscale(v[2], dobs[2]));
  return out;
}

/* ---- history_interaction.cpp:29-43 with rotating_green_function.cpp:3-24
 *      (frame 0) or green_function.cpp:3-20 (frame 1) ------------------- */
void or_pair_coefficients(const or_dot *src, const or_dot *obs,
                          const or_params *p, int *floor_delay, double *coef)
{
  const int q = p->interpolation_order;
  const int n = q + 1;
  double dr[3];
  for(int k = 0; k < 3; ++k) dr[k] = obs->pos[k] - src->pos[k]; /* separation */
  const double nrm = sqrt((dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2]);

  /* split_double(dr.norm() / (c0 * dt)), history_interaction.cpp:88-97 */
  double idelay;
  const double frac = modf(nrm / (p->c0 * p->dt), &idelay);
  *floor_delay = (int)idelay;

  double w[3 * 16];
  or_lagrange_weights(frac, p->dt, q, w);

  double dy[3][9];
  spatial_dyads(dr, p->c0, dy);
  const double A = p->mu0 / (4 * M_PI * p->hbar); /* green_function.h:19 */

  if(p->frame == 0) {
    /* s = -A * exp(-i*omega*r/c) */
    const double om = p->laser_frequency;
    const double y = (-om * nrm) / p->c0;
    cx e = {cos(y), sin(y)};
    cx s = {-A * e.re, -A * e.im};
    const double om2 = pow(om, 2);
    for(int i = 0; i <= q; ++i) {
      const double w0 = w[0 * n + i], w1 = w[1 * n + i], w2 = w[2 * n + i];
      const cx t1 = {w1, om * w0};                 /* w1 + i*omega*w0 */
      const cx t2 = {w2 - om2 * w0, (2.0 * om) * w1}; /* w2 + 2i*omega*w1 - omega^2 w0 */
      cx M[9];
      for(int e9 = 0; e9 < 9; ++e9) {
        cx a = {dy[0][e9] * w0, 0.0};
        cx b = cmul((cx){dy[1][e9], 0.0}, t1);
        cx c = cmul((cx){dy[2][e9], 0.0}, t2);
        M[e9] = cmul(s, cadd(cadd(a, b), c));
      }
      cx v = contract(obs->dip, M, src->dip);
      coef[2 * i] = v.re;
      coef[2 * i + 1] = v.im;
    }
  } else {
    for(int i = 0; i <= q; ++i) {
      cx M[9];
      for(int e9 = 0; e9 < 9; ++e9) {
        cx acc = {0.0, 0.0};
        for(int term = 0; term < 3; ++term) {
          cx t = {(A * dy[term][e9]) * w[term * n + i], (A * 0.0) * w[term * n + i]};
          acc = cadd(acc, t);
        }
        M[e9] = acc;
      }
      cx v = contract(obs->dip, M, src->dip);
      coef[2 * i] = v.re;
      coef[2 * i + 1] = v.im;
    }
  }
}

/* ---- history_interaction.cpp:72-86 (64-bit, so no int overflow) ------- */
long long or_coord2idx(int row, int col)
{
  if(col > row) {
    int t = row;
    row = col;
    col = t;
  }
  return (long long)row * (row - 1) / 2 + col;
}

void or_idx2coord(long long idx, int *row, int *col)
{
  long long r = (long long)floor((sqrt(1.0 + 8.0 * (double)idx) + 1) / 2.0);
  /* guard the floating-point estimate for large idx */
  while(r * (r - 1) / 2 > idx) --r;
  while((r + 1) * r / 2 <= idx) ++r;
  *row = (int)r;
  *col = (int)(idx - r * (r - 1) / 2);
}

/* ---- history_interaction.cpp:21-45 ------------------------------------ */
void or_build_table(const or_dot *dots, int n, const or_params *p, int *delays,
                    double *coefs)
{
  const int nc = 2 * (p->interpolation_order + 1);
  const long long P = (long long)n * (n - 1) / 2;
#pragma omp parallel for schedule(static)
  for(long long idx = 0; idx < P; ++idx) {
    int src, obs;
    or_idx2coord(idx, &src, &obs);
    or_pair_coefficients(&dots[src], &dots[obs], p, &delays[idx],
                         &coefs[idx * nc]);
  }
}

static inline const double *hist_at(const double *hist, int window, int T,
                                    int dot, int t, int which)
{
  return hist + (((size_t)dot * (T + window) + (size_t)(t + window)) * 2 + which) * 4;
}
static inline double *hist_atw(double *hist, int window, int T, int dot, int t,
                               int which)
{
  return hist + (((size_t)dot * (T + window) + (size_t)(t + window)) * 2 + which) * 4;
}

/* polarization_prefactor: rotating -> rho01 (rotating_green_function.h:17-21),
 * lab -> 2*Re(rho01) (green_function.h:23-27). */
static inline cx prefactor(const double *sol, int frame)
{
  cx r;
  if(frame == 0) {
    r.re = sol[2];
    r.im = sol[3];
  } else {
    r.re = 2 * sol[2];
    r.im = 0.0;
  }
  return r;
}

/* ---- history_interaction.cpp:47-70 ------------------------------------ */
void or_history_evaluate(int n, const or_params *p, const int *delays,
                         const double *coefs, const double *hist, int window,
                         int T, int step, double *out)
{
  const int q = p->interpolation_order;
  const int nc = 2 * (q + 1);
  const long long P = (long long)n * (n - 1) / 2;
  memset(out, 0, sizeof(double) * 2 * n);
  for(long long idx = 0; idx < P; ++idx) {
    int src, obs;
    or_idx2coord(idx, &src, &obs);
    const int s = step - delays[idx];
    for(int i = 0; i <= q; ++i) {
      if(s - i < -window) continue;
      const cx c = {coefs[idx * nc + 2 * i], coefs[idx * nc + 2 * i + 1]};
      const cx ro = prefactor(hist_at(hist, window, T, obs, s - i, 0), p->frame);
      const cx rs = prefactor(hist_at(hist, window, T, src, s - i, 0), p->frame);
      const cx a = cmul(ro, c);
      out[2 * src] += a.re;
      out[2 * src + 1] += a.im;
      const cx b = cmul(rs, c);
      out[2 * obs] += b.re;
      out[2 * obs + 1] += b.im;
    }
  }
}

/* history_interaction.cpp:47-70 for selected target dots only, each pair's
 * coefficients computed on the fly in the table's orientation (src = the
 * larger index, obs = the smaller, history_interaction.cpp:29-43), so the
 * cost is O(N) per target.  rho01: [dot][t - t_lo] complex for steps
 * t_lo .. t_lo + nt - 1, which must cover every tap read (returns -1 with
 * out untouched for the offending target otherwise).  out: one complex per
 * target. */
int or_history_evaluate_targets(const or_dot *dots, int n, const or_params *p, const double *rho01, int t_lo,
                                int nt, int step, const int *targets, int ntargets, double *out)
{
  const int q = p->interpolation_order;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
  for(int k = 0; k < ntargets; ++k) {
    const int a = targets[k];
    cx acc = {0.0, 0.0};
    double coef[2 * 16];
    for(int b = 0; b < n && !bad; ++b) {
      if(b == a) continue;
      const int src = a > b ? a : b, obs = a > b ? b : a;
      int d;
      or_pair_coefficients(&dots[src], &dots[obs], p, &d, coef);
      const int s = step - d;
      for(int i = 0; i <= q; ++i) {
        const int t = s - i;
        if(t < -WINDOW) continue;
        if(t < t_lo || t >= t_lo + nt) {
          bad = 1;
          break;
        }
        const double *z = rho01 + 2 * ((size_t)b * nt + (size_t)(t - t_lo));
        const cx pr = p->frame == 0 ? (cx){z[0], z[1]} : (cx){2 * z[0], 0.0};
        const cx c = {coef[2 * i], coef[2 * i + 1]};
        acc = cadd(acc, cmul(pr, c));
      }
    }
    out[2 * k] = acc.re;
    out[2 * k + 1] = acc.im;
  }
  return bad ? -1 : 0;
}

/* ---- pulse_interaction.cpp:9-20, pulse.cpp:15-20, math_utils.cpp:27-30 */
static inline double gaussian(double t) { return exp(-pow(t, 2) / 2); }

void or_pulse_evaluate(const or_dot *dots, int n, const or_pulse *pulse,
                       const or_params *p, int step, double *out)
{
  const double time = step * p->dt;
  for(int i = 0; i < n; ++i) {
    const double *r = dots[i].pos;
    const double arg = ((pulse->wavevector[0] * r[0] + pulse->wavevector[1] * r[1]) +
                        pulse->wavevector[2] * r[2]) -
                       pulse->freq * (time - pulse->delay);
    const double g = gaussian(arg / pulse->width);
    double e[3];
    for(int k = 0; k < 3; ++k) e[k] = (pulse->amplitude / 2 * pulse->polarization[k]) * g;
    const double d = (e[0] * dots[i].dip[0] + e[1] * dots[i].dip[1]) + e[2] * dots[i].dip[2];
    out[2 * i] = d / p->hbar;
    out[2 * i + 1] = 0.0;
  }
}

/* ---- quantum_dot.cpp:10-19 -------------------------------------------- */
void or_liouville_rhs(const or_dot *dot, const double *rho, const double *rabi,
                      double laser_freq, double *out)
{
  const cx r0 = {rho[0], rho[1]}, r1 = {rho[2], rho[3]};
  const cx om = {rabi[0], rabi[1]};
  const cx r1c = {r1.re, -r1.im}, omc = {om.re, -om.im};
  const cx mi = {-0.0, -1.0}; /* -iu */
  /* m0 = -iu*(rabi*conj(rho1) - conj(rabi)*rho1) - (rho0 - 1.0)/T1 */
  cx u = cmul(om, r1c), v = cmul(omc, r1);
  cx d = {u.re - v.re, u.im - v.im};
  cx m0 = cmul(mi, d);
  cx g = {(r0.re - 1.0) / dot->t1, r0.im / dot->t1};
  m0.re = m0.re - g.re;
  m0.im = m0.im - g.im;
  /* m1 = -iu*(rabi*(1.0 - 2.0*rho0) + rho1*(laser_freq - freq)) - rho1/T2 */
  cx two_r0 = {2.0 * r0.re, 2.0 * r0.im};
  cx one_m = {1.0 - two_r0.re, -two_r0.im};
  cx a = cmul(om, one_m);
  const double det = laser_freq - dot->freq;
  cx b = {r1.re * det, r1.im * det};
  cx ab = {a.re + b.re, a.im + b.im};
  cx m1 = cmul(mi, ab);
  m1.re = m1.re - r1.re / dot->t2;
  m1.im = m1.im - r1.im / dot->t2;
  out[0] = m0.re;
  out[1] = m0.im;
  out[2] = m1.re;
  out[3] = m1.im;
}

int or_isfinite(const double *sol)
{
  return isfinite(sol[0]) && isfinite(sol[1]) && isfinite(sol[2]) && isfinite(sol[3]);
}

/* ---- integrator.cpp:142-169 ------------------------------------------- */
static void predictor_one(double *hist, int window, int T, int dot, int step,
                          const or_weights *w, double dt)
{
  const int width = w->n_time;
  const int start = step - width;
  double *out = hist_atw(hist, window, T, dot, step, 0);
  double acc[4] = {0, 0, 0, 0};
  for(int h = 0; h < width; ++h) {
    const double *x = hist_at(hist, window, T, dot, start + h, 0);
    const double *y = hist_at(hist, window, T, dot, start + h, 1);
    for(int c = 0; c < 4; ++c)
      acc[c] += x[c] * w->ps[h] + (y[c] * w->ps[width + h]) * dt;
  }
  memcpy(out, acc, sizeof acc);
}

static void corrector_one(double *hist, int window, int T, int dot, int step,
                          const or_weights *w, double dt)
{
  const int width = w->n_time;
  const int start = step - width;
  double *out = hist_atw(hist, window, T, dot, step, 0);
  const double *cur = hist_at(hist, window, T, dot, step, 1);
  double acc[4];
  for(int c = 0; c < 4; ++c) acc[c] = (w->future_coef * cur[c]) * dt;
  for(int h = 0; h < width; ++h) {
    const double *x = hist_at(hist, window, T, dot, start + h, 0);
    const double *y = hist_at(hist, window, T, dot, start + h, 1);
    for(int c = 0; c < 4; ++c)
      acc[c] += x[c] * w->cs[h] + (y[c] * w->cs[width + h]) * dt;
  }
  memcpy(out, acc, sizeof acc);
}

/* main.cpp:30-36: rho = (1, 0) for t in [-22, 0]; rho-dot at t < 0 is never
 * written by the reference (left as fresh zero pages), set to 0 here. */
static void init_history(double *hist, int n, int window, int T)
{
  memset(hist, 0, sizeof(double) * (size_t)n * (T + window) * 8);
  for(int t = -window; t <= 0 && t < T; ++t)
    for(int i = 0; i < n; ++i) {
      double *s = hist_atw(hist, window, T, i, t, 0);
      s[0] = 1.0;
      s[1] = 0.0;
      s[2] = 0.0;
      s[3] = 0.0;
    }
}

/* evaluator (integrator.cpp:171-185): efield = (0 + pulse) + history. */
static void evaluator_all(const or_dot *dots, int n, const or_params *p,
                          const double *pulse_f, const double *hist_f,
                          double *hist, int window, int T, int step)
{
  for(int i = 0; i < n; ++i) {
    double rabi[2] = {(0.0 + pulse_f[2 * i]) + hist_f[2 * i],
                      (0.0 + pulse_f[2 * i + 1]) + hist_f[2 * i + 1]};
    const double *rho = hist_at(hist, window, T, i, step, 0);
    double *drho = hist_atw(hist, window, T, i, step, 1);
    double out[4];
    or_liouville_rhs(&dots[i], rho, rabi, p->laser_frequency, out);
    memcpy(drho, out, sizeof out);
  }
}

static int all_finite(const double *hist, int n, int window, int T, int step)
{
  for(int i = 0; i < n; ++i)
    if(!or_isfinite(hist_at(hist, window, T, i, step, 0)) ||
       !or_isfinite(hist_at(hist, window, T, i, step, 1)))
      return 0;
  return 1;
}

static void faithful_step(const or_dot *dots, int n, const or_pulse *pulse,
                          const or_params *p, const or_weights *w, int T,
                          const int *delays, const double *coefs, double *hist,
                          int step, double *pf, double *hf)
{
  for(int i = 0; i < n; ++i) predictor_one(hist, WINDOW, T, i, step, w, p->dt);
  or_pulse_evaluate(dots, n, pulse, p, step, pf);
  or_history_evaluate(n, p, delays, coefs, hist, WINDOW, T, step, hf);
  evaluator_all(dots, n, p, pf, hf, hist, WINDOW, T, step);
  for(int m = 0; m < NUM_CORRECTOR_STEPS; ++m) {
    for(int i = 0; i < n; ++i) corrector_one(hist, WINDOW, T, i, step, w, p->dt);
    or_pulse_evaluate(dots, n, pulse, p, step, pf);
    or_history_evaluate(n, p, delays, coefs, hist, WINDOW, T, step, hf);
    evaluator_all(dots, n, p, pf, hf, hist, WINDOW, T, step);
  }
}

/* One faithful step (integrator.cpp:128-140) for dots [lo, hi) only, the
 * others' history read as it stands: each owned target's pair sum runs over
 * its partners in the pair order of history_interaction.cpp:47-70, so the
 * result is that of faithful_step bit for bit.  The current step's delay-0
 * terms read partners' iterates of this step, which exist here only for
 * owned partners: returns -1 (nothing done) when a delay-0 pair crosses the
 * range.  Test infrastructure for the target-sharded driver. */
int or_faithful_step_range(const or_dot *dots, int n, const or_pulse *pulse, const or_params *p,
                           const or_weights *w, int T, const int *delays, const double *coefs, double *hist,
                           int step, int lo, int hi)
{
  const int q = p->interpolation_order;
  const int nc = 2 * (q + 1);
  for(int a = lo; a < hi; ++a)
    for(int b = 0; b < n; ++b)
      if(b != a && (b < lo || b >= hi) && delays[or_coord2idx(a, b)] == 0) return -1;
  double *pf = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  double *hf = (double *)calloc(2 * (size_t)(n > 0 ? n : 1), sizeof(double));
  for(int a = lo; a < hi; ++a) predictor_one(hist, WINDOW, T, a, step, w, p->dt);
  for(int it = 0; it <= NUM_CORRECTOR_STEPS; ++it) {
    if(it > 0)
      for(int a = lo; a < hi; ++a) corrector_one(hist, WINDOW, T, a, step, w, p->dt);
    or_pulse_evaluate(dots, n, pulse, p, step, pf);
    for(int a = lo; a < hi; ++a) {
      double re = 0, im = 0;
      for(int b = 0; b < n; ++b) {
        if(b == a) continue;
        const long long idx = or_coord2idx(a, b);
        const int s = step - delays[idx];
        for(int i = 0; i <= q; ++i) {
          if(s - i < -WINDOW) continue;
          const cx c = {coefs[idx * nc + 2 * i], coefs[idx * nc + 2 * i + 1]};
          const cx v = cmul(prefactor(hist_at(hist, WINDOW, T, b, s - i, 0), p->frame), c);
          re += v.re;
          im += v.im;
        }
      }
      hf[2 * a] = re;
      hf[2 * a + 1] = im;
    }
    for(int a = lo; a < hi; ++a) {
      double rabi[2] = {(0.0 + pf[2 * a]) + hf[2 * a], (0.0 + pf[2 * a + 1]) + hf[2 * a + 1]};
      double out[4];
      or_liouville_rhs(&dots[a], hist_at(hist, WINDOW, T, a, step, 0), rabi, p->laser_frequency, out);
      memcpy(hist_atw(hist, WINDOW, T, a, step, 1), out, sizeof out);
    }
  }
  free(pf);
  free(hf);
  return 0;
}

/* ---- integrator.cpp:120-140, 187-207 ---------------------------------- */
int or_run_faithful(const or_dot *dots, int n, const or_pulse *pulse,
                    const or_params *p, const or_weights *w, int T,
                    double *hist, int *bad_step)
{
  const long long P = (long long)n * (n - 1) / 2;
  const int nc = 2 * (p->interpolation_order + 1);
  int *delays = (int *)malloc(sizeof(int) * (P > 0 ? P : 1));
  double *coefs = (double *)malloc(sizeof(double) * (P > 0 ? P : 1) * nc);
  double *pf = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  double *hf = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  or_build_table(dots, n, p, delays, coefs);
  init_history(hist, n, WINDOW, T);
  int rc = 0;
  for(int step = 0; step < T; ++step) {
    faithful_step(dots, n, pulse, p, w, T, delays, coefs, hist, step, pf, hf);
    if(!all_finite(hist, n, WINDOW, T, step)) {
      *bad_step = step;
      rc = 1;
      break;
    }
  }
  free(delays);
  free(coefs);
  free(pf);
  free(hf);
  return rc;
}

int or_faithful_steps(const or_dot *dots, int n, const or_pulse *pulse,
                      const or_params *p, const or_weights *w, int T,
                      const int *delays, const double *coefs, double *hist,
                      int t0, int nsteps)
{
  double *pf = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  double *hf = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  int done = 0;
  for(int step = t0; step < t0 + nsteps && step < T; ++step, ++done)
    faithful_step(dots, n, pulse, p, w, T, delays, coefs, hist, step, pf, hf);
  free(pf);
  free(hf);
  return done;
}

/* ---- fast oracle: one sweep per step + near list ---------------------- */
typedef struct {
  int a, b;       /* src (row), obs (col) */
  double c0[2];   /* tap-0 coefficient */
} near_pair;

int or_run_fast(const or_dot *dots, int n, const or_pulse *pulse,
                const or_params *p, const or_weights *w, int T, double *hist,
                int *bad_step, int nthreads)
{
  const int q = p->interpolation_order;
  const int nc = 2 * (q + 1);
  const long long P = (long long)n * (n - 1) / 2;
  int *delays = (int *)malloc(sizeof(int) * (P > 0 ? P : 1));
  double *coefs = (double *)malloc(sizeof(double) * (P > 0 ? P : 1) * nc);
  double *pf = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  double *past = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  double *hf = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  if(nthreads < 1) nthreads = 1;
#ifdef _OPENMP
  omp_set_num_threads(nthreads);
#else
  nthreads = 1;
#endif
  double *priv = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1) * nthreads);
  or_build_table(dots, n, p, delays, coefs);
  init_history(hist, n, WINDOW, T);

  long long nn = 0;
  for(long long idx = 0; idx < P; ++idx) nn += delays[idx] == 0;
  near_pair *near = (near_pair *)malloc(sizeof(near_pair) * (nn > 0 ? nn : 1));
  nn = 0;
  for(long long idx = 0; idx < P; ++idx)
    if(delays[idx] == 0) {
      int src, obs;
      or_idx2coord(idx, &src, &obs);
      near[nn].a = src;
      near[nn].b = obs;
      near[nn].c0[0] = coefs[idx * nc];
      near[nn].c0[1] = coefs[idx * nc + 1];
      ++nn;
    }

  int rc = 0;
  for(int step = 0; step < T; ++step) {
    for(int i = 0; i < n; ++i) predictor_one(hist, WINDOW, T, i, step, w, p->dt);
    /* strictly-past sweep: every (pair, tap) except delay 0 / tap 0 */
#pragma omp parallel num_threads(nthreads)
    {
#ifdef _OPENMP
      const int tid = omp_get_thread_num();
      const int nth = omp_get_num_threads();
#else
      const int tid = 0, nth = 1;
#endif
      double *acc = priv + (size_t)tid * 2 * n;
      memset(acc, 0, sizeof(double) * 2 * n);
      const long long lo = P * tid / nth, hi = P * (tid + 1) / nth;
      int src = 0, obs = 0;
      if(lo < hi) or_idx2coord(lo, &src, &obs);
      for(long long idx = lo; idx < hi; ++idx) {
        const int s = step - delays[idx];
        for(int i = 0; i <= q; ++i) {
          if(s - i < -WINDOW) continue;
          if(s - i == step) continue; /* current step: near list */
          const cx c = {coefs[idx * nc + 2 * i], coefs[idx * nc + 2 * i + 1]};
          const cx ro = prefactor(hist_at(hist, WINDOW, T, obs, s - i, 0), p->frame);
          const cx rs = prefactor(hist_at(hist, WINDOW, T, src, s - i, 0), p->frame);
          const cx a = cmul(ro, c), b = cmul(rs, c);
          acc[2 * src] += a.re;
          acc[2 * src + 1] += a.im;
          acc[2 * obs] += b.re;
          acc[2 * obs + 1] += b.im;
        }
        if(++obs == src) {
          ++src;
          obs = 0;
        }
      }
    }
    for(int i = 0; i < 2 * n; ++i) {
      double s = 0;
      for(int t = 0; t < nthreads; ++t) s += priv[(size_t)t * 2 * n + i];
      past[i] = s;
    }
    or_pulse_evaluate(dots, n, pulse, p, step, pf);
    for(int it = 0; it <= NUM_CORRECTOR_STEPS; ++it) {
      if(it > 0)
        for(int i = 0; i < n; ++i) corrector_one(hist, WINDOW, T, i, step, w, p->dt);
      memcpy(hf, past, sizeof(double) * 2 * n);
      for(long long k = 0; k < nn; ++k) {
        const cx c = {near[k].c0[0], near[k].c0[1]};
        const cx ro = prefactor(hist_at(hist, WINDOW, T, near[k].b, step, 0), p->frame);
        const cx rs = prefactor(hist_at(hist, WINDOW, T, near[k].a, step, 0), p->frame);
        const cx a = cmul(ro, c), b = cmul(rs, c);
        hf[2 * near[k].a] += a.re;
        hf[2 * near[k].a + 1] += a.im;
        hf[2 * near[k].b] += b.re;
        hf[2 * near[k].b + 1] += b.im;
      }
      evaluator_all(dots, n, p, pf, hf, hist, WINDOW, T, step);
    }
    if(!all_finite(hist, n, WINDOW, T, step)) {
      *bad_step = step;
      rc = 1;
      break;
    }
  }
  free(near);
  free(priv);
  free(delays);
  free(coefs);
  free(pf);
  free(past);
  free(hf);
  return rc;
}
