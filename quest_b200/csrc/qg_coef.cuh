// Per-pair retarded-interaction coefficients on the device, following the
// reference's table build operation by operation:
//   separation / norm / split_double   history_interaction.cpp:29-35, 88-97
//   UniformLagrangeSet::calculate_weights   lagrange_set.cpp:17-41
//   spatial dyads                      green_function.h:32-55
//   RotatingDyadic::coefficients       rotating_green_function.cpp:3-24
//   Dyadic::coefficients (lab frame)   green_function.cpp:3-20
//   d_obs . (M d_src)                  history_interaction.cpp:40-43
// Included by translation units compiled with -fmad=false, so each multiply
// and add rounds separately as in the reference's x86-64 build.
#pragma once

#include "qg_internal.h"

namespace qg {

// lagrange_set.cpp:17-41; w[k][i] for derivative k = 0..2, node i = 0..q.
template <int Q>
__device__ __forceinline__ void lagrange_weights_ref(double x, double dt, double (&w)[3][Q + 1])
{
#pragma unroll
  for(int b = 0; b <= Q; ++b) {
    double d0 = 1, d1 = 0, d2 = 0;
#pragma unroll
    for(int m = 0; m <= Q; ++m) {
      if(m == b) continue;
      d0 *= (x - m) / (double)(b - m);
      d1 -= 1 / (x - m);
      d2 -= pow(x - m, -2.0);
    }
    w[0][b] = d0;
    w[1][b] = w[0][b] * d1;
    w[2][b] = w[0][b] * d2 + (w[1][b] * w[1][b]) / w[0][b];
  }
  const double inv_dt = 1.0 / dt;  // gcc folds pow(dt, -1) to 1/dt
  const double inv_dt2 = pow(dt, -2.0);
#pragma unroll
  for(int i = 0; i <= Q; ++i) {
    w[1][i] *= inv_dt;
    w[2][i] *= inv_dt2;
  }
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b)
{
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 cscale(double2 a, double s)
{
  return make_double2(a.x * s, a.y * s);
}

// d_obs . (M d_src) with Eigen's left-to-right sums over 3-vectors.
__device__ __forceinline__ double2 contract3(const double (&dobs)[3], const double2 (&M)[9],
                                             const double (&dsrc)[3])
{
  double2 v[3];
#pragma unroll
  for(int r = 0; r < 3; ++r) {
    double2 acc = cscale(M[3 * r + 0], dsrc[0]);
    acc = cadd(acc, cscale(M[3 * r + 1], dsrc[1]));
    acc = cadd(acc, cscale(M[3 * r + 2], dsrc[2]));
    v[r] = acc;
  }
  double2 out = cscale(v[0], dobs[0]);
  out = cadd(out, cscale(v[1], dobs[1]));
  out = cadd(out, cscale(v[2], dobs[2]));
  return out;
}

// Floor delay and q+1 coefficients of the pair (src = larger user index,
// obs = smaller), exactly the quantities build_coefficient_table stores.
template <int Q>
__device__ __forceinline__ int pair_coef_ref(const double (&psrc)[3], const double (&pobs)[3],
                                             const double (&dsrc)[3], const double (&dobs)[3],
                                             const CoefParams &p, double2 (&coef)[Q + 1])
{
  double dr[3];
#pragma unroll
  for(int k = 0; k < 3; ++k) dr[k] = pobs[k] - psrc[k];
  const double sq = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
  const double nrm = sqrt(sq);
  double idelay;
  const double frac = modf(nrm / (p.c0 * p.dt), &idelay);
  const int fd = (int)idelay;

  double w[3][Q + 1];
  lagrange_weights_ref<Q>(frac, p.dt, w);

  // spatial dyads (green_function.h:32-40)
  double dy[3][9];
  const double c2 = p.c0 * p.c0;       // pow(c, 2)
  const double n3 = pow(nrm, 3.0);     // pow(|r|, 3)
#pragma unroll
  for(int r = 0; r < 3; ++r) {
#pragma unroll
    for(int k = 0; k < 3; ++k) {
      const double rhat = (dr[r] * dr[k]) / sq;
      const double id = (r == k) ? 1.0 : 0.0;
      const double i3 = id - 3 * rhat;
      const double i1 = id - rhat;
      dy[0][3 * r + k] = (i3 * c2) / n3;
      dy[1][3 * r + k] = (i3 * p.c0) / sq;
      dy[2][3 * r + k] = i1 / nrm;
    }
  }
  const double A = p.mu0 / (4 * M_PI * p.hbar);

  if(p.frame == 0) {
    const double om = p.omega;
    const double y = (-om * nrm) / p.c0;
    double sn, cs;
    sincos(y, &sn, &cs);
    const double2 s = make_double2(-A * cs, -A * sn);
    const double om2 = om * om;
#pragma unroll
    for(int i = 0; i <= Q; ++i) {
      const double w0 = w[0][i], w1 = w[1][i], w2 = w[2][i];
      const double2 t1 = make_double2(w1, om * w0);
      const double2 t2 = make_double2(w2 - om2 * w0, (2.0 * om) * w1);
      double2 M[9];
#pragma unroll
      for(int e = 0; e < 9; ++e) {
        const double2 a = make_double2(dy[0][e] * w0, 0.0);
        const double2 b = cmul(make_double2(dy[1][e], 0.0), t1);
        const double2 c = cmul(make_double2(dy[2][e], 0.0), t2);
        M[e] = cmul(s, cadd(cadd(a, b), c));
      }
      coef[i] = contract3(dobs, M, dsrc);
    }
  } else {
#pragma unroll
    for(int i = 0; i <= Q; ++i) {
      double2 M[9];
#pragma unroll
      for(int e = 0; e < 9; ++e) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for(int term = 0; term < 3; ++term) {
          const double2 t = make_double2((A * dy[term][e]) * w[term][i], (A * 0.0) * w[term][i]);
          acc = cadd(acc, t);
        }
        M[e] = acc;
      }
      coef[i] = contract3(dobs, M, dsrc);
    }
  }
  return fd;
}

// The same pair's floor delay and coefficients for the on-the-fly path,
// in an algebraically equal but cheaper form (about 400 instead of about
// 5000 instructions per pair):
//   Lagrange weights   one reciprocal r_m = 1/(x-m) per node, then for node b
//                      w0 = prod_{m!=b} (x-m) / prod_{m!=b} (b-m),
//                      w1 = w0 d1 / dt, w2 = w0 (d2 + d1^2) / dt^2 with
//                      d1 = -sum_{m!=b} r_m, d2 = -sum_{m!=b} r_m^2
//                      (the reference's w0 d2 + w1^2 / w0 with w1 = w0 d1);
//   dyads              contracted with the dipoles first: d_obs.(I - 3 rr).d_src
//                      = dd - 3 (d_obs.r)(d_src.r)/r^2 and d_obs.(I - rr).d_src
//                      = dd - (d_obs.r)(d_src.r)/r^2, so each tap needs three
//                      real scalars G0 = (dd - 3ab/r^2) c^2/r^3,
//                      G1 = (dd - 3ab/r^2) c/r^2, G2 = (dd - ab/r^2)/r;
//   rotating frame     coef_i = s (G0 w0 + G1 (w1 + i om w0) + G2 (w2 + 2 i om w1
//                      - om^2 w0)), s = -mu0/(4 pi hbar) e^{-i om r/c};
//   lab frame          coef_i = mu0/(4 pi hbar) (G0 w0 + G1 w1 + G2 w2).
// The floor delay uses exactly the operations of pair_coef_ref (and of the
// near-pair search), so the far / mid split is the same as the table's; the
// coefficients agree with the reference's to rounding.
template <int Q>
__device__ __forceinline__ int pair_coef_otf(const double (&psrc)[3], const double (&pobs)[3],
                                             const double (&dsrc)[3], const double (&dobs)[3],
                                             const CoefParams &p, double2 (&coef)[Q + 1])
{
  double dr[3];
#pragma unroll
  for(int k = 0; k < 3; ++k) dr[k] = pobs[k] - psrc[k];
  const double sq = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
  const double nrm = sqrt(sq);
  double idelay;
  const double x = modf(nrm / (p.c0 * p.dt), &idelay);
  const int fd = (int)idelay;

  double xm[Q + 1], rm[Q + 1];
#pragma unroll
  for(int m = 0; m <= Q; ++m) {
    xm[m] = x - m;
    rm[m] = 1.0 / xm[m];
  }
  const double inv_dt = 1.0 / p.dt, inv_dt2 = inv_dt * inv_dt;
  double w0[Q + 1], w1[Q + 1], w2[Q + 1];
#pragma unroll
  for(int b = 0; b <= Q; ++b) {
    double num = 1.0, den = 1.0, d1 = 0.0, d2 = 0.0;
#pragma unroll
    for(int m = 0; m <= Q; ++m) {
      if(m == b) continue;
      num *= xm[m];
      den *= (double)(b - m);
      d1 -= rm[m];
      d2 -= rm[m] * rm[m];
    }
    w0[b] = num / den;
    w1[b] = (w0[b] * d1) * inv_dt;
    w2[b] = (w0[b] * (d2 + d1 * d1)) * inv_dt2;
  }

  const double dd = (dobs[0] * dsrc[0] + dobs[1] * dsrc[1]) + dobs[2] * dsrc[2];
  const double ar = (dobs[0] * dr[0] + dobs[1] * dr[1]) + dobs[2] * dr[2];
  const double br = (dsrc[0] * dr[0] + dsrc[1] * dr[1]) + dsrc[2] * dr[2];
  const double inv_r = 1.0 / nrm, inv_sq = 1.0 / sq;
  const double ab = (ar * br) * inv_sq;
  const double g3 = dd - 3.0 * ab, g1 = dd - ab;
  const double G0 = (g3 * (p.c0 * p.c0)) * (inv_sq * inv_r);
  const double G1 = (g3 * p.c0) * inv_sq;
  const double G2 = g1 * inv_r;
  const double A = p.mu0 / (4 * M_PI * p.hbar);
  if(p.frame == 0) {
    const double om = p.omega;
    double sn, cs;
    sincos((-om * nrm) / p.c0, &sn, &cs);
    const double2 s = make_double2(-A * cs, -A * sn);
    const double om2 = om * om;
#pragma unroll
    for(int i = 0; i <= Q; ++i) {
      const double re = (G0 * w0[i] + G1 * w1[i]) + G2 * (w2[i] - om2 * w0[i]);
      const double im = om * (G1 * w0[i] + 2.0 * (G2 * w1[i]));
      coef[i] = cmul(s, make_double2(re, im));
    }
  } else {
#pragma unroll
    for(int i = 0; i <= Q; ++i) coef[i] = make_double2(A * ((G0 * w0[i] + G1 * w1[i]) + G2 * w2[i]), 0.0);
  }
  return fd;
}

// Mixed-precision coefficients of one pair for the on-the-fly kernel.  FP64
// is kept for the distance and the split of r / (c dt) into the floor delay
// and the fraction x (the operations of pair_coef_otf, so the far / mid split
// is the same), and for reducing the phase argument -omega r / c to
// [-pi, pi]; the Lagrange weights, the dyad factors and the taps are FP32.
//
// Weights: with f_m = x - m and e_k the elementary symmetric polynomials of
// {f_m : m != b}, the reference's w0 = prod f_m / den, w1 = w0 sum(-1/f_m) / dt
// and w2 = w0 (sum(-1/f_m^2) + (sum 1/f_m)^2) / dt^2 (lagrange_set.cpp:17-41)
// are w0 = e_Q / den, w1 = -e_{Q-1} / (den dt), w2 = 2 e_{Q-2} / (den dt^2):
// no reciprocals, so no cancellation between 1/x-sized terms as x -> 0.
//
// cf[0..Q] are the taps and cf[Q+1] their sum, taken from the identities
// sum w0 = 1, sum w1 = sum w2 = 0 as the w0-only coefficient: the
// difference-form convolution multiplies the sum by the window's first
// sample and each tap by a step difference, so the sum must be accurate to
// FP32 rounding while the taps (each ~1e-7 relative) only meet differences.
// An integer delay (x = 0) gives NaN taps 1..Q (and sum) and a finite tap 0,
// as the reference's weights do, so a run turns non-finite at the same step.
template <int Q>
__device__ __forceinline__ int pair_coef_otf_mixed(const double (&psrc)[3], const double (&pobs)[3],
                                                   const double (&dsrc)[3], const double (&dobs)[3],
                                                   const CoefParams &p, float2 (&cf)[Q + 2])
{
  double dr[3];
#pragma unroll
  for(int k = 0; k < 3; ++k) dr[k] = pobs[k] - psrc[k];
  const double sq = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
  const double nrm = sqrt(sq);
  double idelay;
  const double xd = modf(nrm / (p.c0 * p.dt), &idelay);
  const int fd = (int)idelay;

  const float x = (float)xd;
  const float inv_dt = (float)(1.0 / p.dt);
  float w0[Q + 1], w1[Q + 1], w2[Q + 1];
#pragma unroll
  for(int b = 0; b <= Q; ++b) {
    float e[Q + 1];
    e[0] = 1.f;
#pragma unroll
    for(int k = 1; k <= Q; ++k) e[k] = 0.f;
    int n = 0;
#pragma unroll
    for(int m = 0; m <= Q; ++m) {
      if(m == b) continue;
      const float f = x - (float)m;
      ++n;
#pragma unroll
      for(int k = Q; k >= 1; --k)
        if(k <= n) e[k] = fmaf(f, e[k - 1], e[k]);
    }
    float den = 1.f;
#pragma unroll
    for(int m = 0; m <= Q; ++m)
      if(m != b) den *= (float)(b - m);  // an exact integer (|den| <= 7!)
    const float id = 1.f / den;
    w0[b] = e[Q] * id;
    w1[b] = -(e[Q - 1] * id) * inv_dt;
    w2[b] = Q >= 2 ? (2.f * (e[Q >= 2 ? Q - 2 : 0] * id)) * (inv_dt * inv_dt) : 0.f;
  }

  const float drf[3] = {(float)dr[0], (float)dr[1], (float)dr[2]};
  const float df_s[3] = {(float)dsrc[0], (float)dsrc[1], (float)dsrc[2]};
  const float df_o[3] = {(float)dobs[0], (float)dobs[1], (float)dobs[2]};
  const float dd = fmaf(df_o[2], df_s[2], fmaf(df_o[1], df_s[1], df_o[0] * df_s[0]));
  const float ar = fmaf(df_o[2], drf[2], fmaf(df_o[1], drf[1], df_o[0] * drf[0]));
  const float br = fmaf(df_s[2], drf[2], fmaf(df_s[1], drf[1], df_s[0] * drf[0]));
  const float inv_r = (float)(1.0 / nrm), inv_sq = inv_r * inv_r;
  const float ab = (ar * br) * inv_sq;
  const float g3 = fmaf(-3.f, ab, dd), g1 = dd - ab;
  const float c0 = (float)p.c0;
  const float G0 = (g3 * (c0 * c0)) * (inv_sq * inv_r);
  const float G1 = (g3 * c0) * inv_sq;
  const float G2 = g1 * inv_r;
  const float A = (float)(p.mu0 / (4 * M_PI * p.hbar));
  if(p.frame == 0) {
    const double om = p.omega;
    const double ph = (-om * nrm) / p.c0;
    const double red = ph - 6.283185307179586 * rint(ph * 0.15915494309189535);
    float sn, cs;
    sincosf((float)red, &sn, &cs);
    const float2 sc = make_float2(-A * cs, -A * sn);
    const float omf = (float)om, om2 = omf * omf;
#pragma unroll
    for(int i = 0; i <= Q; ++i) {
      const float re = fmaf(G2, fmaf(-om2, w0[i], w2[i]), fmaf(G0, w0[i], G1 * w1[i]));
      const float im = omf * fmaf(G1, w0[i], 2.f * (G2 * w1[i]));
      cf[i] = make_float2(fmaf(sc.x, re, -sc.y * im), fmaf(sc.x, im, sc.y * re));
    }
    const float rs = fmaf(-om2, G2, G0), is = omf * G1;
    cf[Q + 1] = make_float2(fmaf(sc.x, rs, -sc.y * is), fmaf(sc.x, is, sc.y * rs));
  } else {
#pragma unroll
    for(int i = 0; i <= Q; ++i) cf[i] = make_float2(A * fmaf(G2, w2[i], fmaf(G0, w0[i], G1 * w1[i])), 0.f);
    cf[Q + 1] = make_float2(A * G0, 0.f);
  }
  if(xd == 0.0) {
    // the reference's weights at x = 0: node 0's are finite, every other
    // node's w1 and w2 are 0 * inf = NaN (lagrange_set.cpp:25-33); the sum
    // carries them
#pragma unroll
    for(int i = 1; i <= Q + 1; ++i) cf[i] = make_float2(__int_as_float(0x7fc00000), 0.f);
  }
  return fd;
}

}  // namespace qg
