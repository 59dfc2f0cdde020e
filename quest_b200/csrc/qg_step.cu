// Per-dot work of one time step: the integrator, the pulse and the Bloch
// right-hand side.
//
//   predictor            reference src/integrator.cpp:142-154
//   corrector            integrator.cpp:156-169
//   evaluator            integrator.cpp:171-185 (field = (0 + pulse) + history)
//   PulseInteraction     src/interactions/pulse_interaction.cpp:9-20,
//                        src/pulse.cpp:15-20, src/math_utils.cpp:27-30
//   liouville_rhs        src/quantum_dot.cpp:10-19
//   all_finite           integrator.cpp:187-198
//
// The strictly-past part of the history field has two sources: the far-pair
// kernel's partial sums (pairs with floor delay >= K, computed once per K
// steps) and the mid list (pairs with delay < K), summed here every step.
// The (delay 0, tap 0) terms, which read the current step's iterate, are
// re-evaluated in each of the 11 evaluations from a near list.  Work does not
// stop after a non-finite value: the first such step is recorded and every
// step is computed, so the cost per step does not depend on the data.
//
// Two forms.  The fused kernel runs predictor, 11 evaluations and 10
// corrections in one launch: every connected group of dots coupled at delay
// 0 is placed inside one thread block, so a __syncthreads between
// iterations is the only synchronisation needed.  The general form (used when
// such a group is larger than a block, e.g. when c0*dt exceeds the dot
// spacing and every pair has delay 0) runs one launch per evaluation.
//
// Per-dot state in HBM:
//   pcr[slot][k][dot]   k = rho00, rho01, drho00, drho01 for the last 23
//                       steps (slot = t mod 23): the integrator's window
//   ring[dot][slot]     rho01 by step (slot = t mod W, first kRingMirror
//                       slots mirrored after W-1), read by the sweep
//
// Compiled with -fmad=false: the predictor, corrector and right-hand side
// round each operation as the reference does.
#include <cuda_runtime.h>

#include "qg_coef.cuh"

namespace qg {

__device__ __forceinline__ int pc_slot(int t) { return ((t % kPcDepth) + kPcDepth) % kPcDepth; }

__device__ __forceinline__ double2 prefactor(double2 r, int frame)
{
  // rotating frame: rho01 (rotating_green_function.h:17-21);
  // lab frame: 2 Re rho01 (green_function.h:23-27)
  return frame == 0 ? r : make_double2(2 * r.x, 0.0);
}

// x / t given y = 1/t correctly rounded: q0 = x*y, the remainder x - q0*t
// exact in one fused multiply-add, then q0 + r*y rounded once.  This is
// Markstein's correction step (P. W. Markstein, IBM J. Res. Develop. 34(1),
// 1990): with y within half an ulp of 1/t and q0 within one ulp of x/t it
// returns the correctly rounded quotient, i.e. exactly x / t, barring
// underflow and overflow.  r == 0 means q0 is exact (and keeps the sign of a
// zero quotient).  Four independent divisions per evaluation become twelve
// independent flops instead of four serial division sequences.
__device__ __forceinline__ double div_by(double x, double t, double y)
{
  const double q0 = x * y;
  const double r = fma(-q0, t, x);
  return r == 0.0 ? q0 : fma(r, y, q0);
}

// Per-dot constants of the right-hand side.
struct DotConst {
  double det, t1, t2, inv1, inv2;
};

__device__ __forceinline__ DotConst dot_const(const StepArgs &a, int idx, bool live)
{
  DotConst c{0.0, 1.0, 1.0, 1.0, 1.0};
  if(live) {
    c.det = a.laser_freq - a.freq[idx];
    c.t1 = a.t1[idx];
    c.t2 = a.t2[idx];
    c.inv1 = 1.0 / c.t1;
    c.inv2 = 1.0 / c.t2;
  }
  return c;
}

__device__ __forceinline__ void liouville(double2 r0, double2 r1, double2 om, const DotConst &dc, double2 &m0,
                                          double2 &m1)
{
  const double2 r1c = make_double2(r1.x, -r1.y), omc = make_double2(om.x, -om.y);
  const double2 mi = make_double2(-0.0, -1.0);  // -iu
  const double2 u = cmul(om, r1c), v = cmul(omc, r1);
  m0 = cmul(mi, make_double2(u.x - v.x, u.y - v.y));
  m0.x = m0.x - div_by(r0.x - 1.0, dc.t1, dc.inv1);
  m0.y = m0.y - div_by(r0.y, dc.t1, dc.inv1);
  const double2 one_m = make_double2(1.0 - 2.0 * r0.x, -(2.0 * r0.y));
  const double2 aa = cmul(om, one_m);
  const double2 ab = make_double2(aa.x + r1.x * dc.det, aa.y + r1.y * dc.det);
  m1 = cmul(mi, ab);
  m1.x = m1.x - div_by(r1.x, dc.t2, dc.inv2);
  m1.y = m1.y - div_by(r1.y, dc.t2, dc.inv2);
}

// The pulse term from a dot's k.r and dipole (pulse_kr, then pulse_at).
__device__ __forceinline__ double pulse_kr(const StepArgs &a, int idx)
{
  const double *p = a.pos + 3 * idx;
  const PulseParams &P = a.pulse;
  return (P.k[0] * p[0] + P.k[1] * p[1]) + P.k[2] * p[2];
}

__device__ __forceinline__ double pulse_at(const StepArgs &a, double kr, double d0, double d1, double d2, int t)
{
  const PulseParams &P = a.pulse;
  const double time = t * a.dt;
  const double arg = kr - P.freq * (time - P.delay);
  const double x = arg / P.width;
  const double g = exp(-(x * x) / 2);
  const double e0 = P.amp_pol[0] * g, e1 = P.amp_pol[1] * g, e2 = P.amp_pol[2] * g;
  return ((e0 * d0 + e1 * d1) + e2 * d2) / a.hbar;
}

__device__ __forceinline__ double pulse_rabi(const StepArgs &a, int idx, int t)
{
  const double *d = a.dip + 3 * idx;
  return pulse_at(a, pulse_kr(a, idx), d[0], d[1], d[2], t);
}

// Predictor value P and corrector base H (the history part of the
// corrector sum) from the n_time-step window (NT > 0: compile-time width,
// loop unrolled so the window's loads are all in flight together).
template <int NT>
__device__ __forceinline__ void pc_window(const StepArgs &a, int idx, int t, double2 (&P)[2],
                                          double2 (&H)[2])
{
  P[0] = P[1] = H[0] = H[1] = make_double2(0.0, 0.0);
  const int nt = NT > 0 ? NT : a.w.n_time;
  const double dt = a.dt;
#pragma unroll
  for(int h = 0; h < (NT > 0 ? NT : a.w.n_time); ++h) {
    const int s = pc_slot(t - nt + h);
    const double2 *base = a.pcr + (long long)s * 4 * a.n_pad + idx;
    const double2 x0 = base[0], x1 = base[a.n_pad], y0 = base[2 * a.n_pad], y1 = base[3 * a.n_pad];
    const double p0 = a.w.ps[h], p1 = a.w.ps[nt + h];
    const double c0 = a.w.cs[h], c1 = a.w.cs[nt + h];
    P[0].x += x0.x * p0 + (y0.x * p1) * dt;
    P[0].y += x0.y * p0 + (y0.y * p1) * dt;
    P[1].x += x1.x * p0 + (y1.x * p1) * dt;
    P[1].y += x1.y * p0 + (y1.y * p1) * dt;
    H[0].x += x0.x * c0 + (y0.x * c1) * dt;
    H[0].y += x0.y * c0 + (y0.y * c1) * dt;
    H[1].x += x1.x * c0 + (y1.x * c1) * dt;
    H[1].y += x1.y * c0 + (y1.y * c1) * dt;
  }
}

__device__ __forceinline__ int ring_slot(int t, int W) { return ((t % W) + W) % W; }

// Field at step t from every tap that reads a step before t: the far-pair
// field of this step's slice, then the mid-list pairs (delay < K), taps
// before step -22 skipped and the (delay 0, tap 0) term left to the near list.
__device__ __forceinline__ double2 past_field(const StepArgs &a, int idx, int t, int slice)
{
  double2 f = a.far_field[(long long)slice * a.n_pad + idx];
  const int q = a.q;
  for(int e = a.mid_ptr[idx]; e < a.mid_ptr[idx + 1]; ++e) {
    const int b = a.mid_idx[e];
    const int d = a.mid_delay[e];
    const double2 *c = a.mid_coef + (long long)e * (q + 1);
    const double2 *ring = a.ring + (long long)b * a.stride;
    const int s = t - d;
    for(int i = (d == 0) ? 1 : 0; i <= q && s - i >= -kWindow; ++i) {
      const double2 v = cmul(prefactor(ring[ring_slot(s - i, a.W)], a.frame), c[i]);
      f.x += v.x;
      f.y += v.y;
    }
  }
  return f;
}

__device__ __forceinline__ void corrector(const StepArgs &a, const double2 (&dr)[2],
                                          const double2 (&H)[2], double2 (&r)[2])
{
  const double fc = a.w.fc, dt = a.dt;
#pragma unroll
  for(int c = 0; c < 2; ++c) {
    r[c].x = (fc * dr[c].x) * dt + H[c].x;
    r[c].y = (fc * dr[c].y) * dt + H[c].y;
  }
}

__device__ __forceinline__ bool finite4(double2 a, double2 b)
{
  return isfinite(a.x) && isfinite(a.y) && isfinite(b.x) && isfinite(b.y);
}

// Stores the step's rho01 in the ring (and, in mixed precision, the FP32
// rings), which other dots read.
__device__ __forceinline__ void finish_ring(const StepArgs &a, int idx, int t, const double2 (&r)[2])
{
  const int slot = t % a.W;
  double2 *ring = a.ring + (long long)idx * a.stride;
  if(a.ring32w) {
    // mixed precision: FP32 value and FP32 step-to-step difference, the
    // difference formed in FP64 from the previous step's rho01
    const double2 prev = ring[ring_slot(t - 1, a.W)];
    const float2 w = make_float2((float)r[1].x, (float)r[1].y);
    const float2 d = make_float2((float)(r[1].x - prev.x), (float)(r[1].y - prev.y));
    float2 *rw = a.ring32w + (long long)idx * a.stride, *rd = a.ring32d + (long long)idx * a.stride;
    rw[slot] = w;
    rd[slot] = d;
    if(slot < kRingMirror) {
      rw[a.W + slot] = w;
      rd[a.W + slot] = d;
    }
  }
  ring[slot] = r[1];
  if(slot < kRingMirror) ring[a.W + slot] = r[1];
}

// Stores the rest of the step's final state: PC window, trajectory row and
// the non-finite flag.
__device__ __forceinline__ void finish_state(const StepArgs &a, int idx, int t, const double2 (&r)[2],
                                             const double2 (&dr)[2])
{
  double2 *base = a.pcr + (long long)pc_slot(t) * 4 * a.n_pad + idx;
  base[0] = r[0];
  base[a.n_pad] = r[1];
  base[2 * a.n_pad] = dr[0];
  base[3 * a.n_pad] = dr[1];
  if(a.traj) {
    const int row = t - *a.traj_t0;
    if(row >= 0 && row < a.traj_rows) {
      double2 *tr = a.traj + ((long long)row * a.n + a.user[idx]) * 2;
      tr[0] = r[0];
      tr[1] = r[1];
    } else {
      atomicMin(a.d_bad, -1);
    }
  }
  if(!finite4(r[0], r[1]) || !finite4(dr[0], dr[1])) atomicMin(a.d_bad, t);
}

__device__ __forceinline__ void finish_dot(const StepArgs &a, int idx, int t, const double2 (&r)[2],
                                           const double2 (&dr)[2])
{
  finish_ring(a, idx, t, r);
  finish_state(a, idx, t, r, dr);
}

// The step index is the far block's first step plus the launch's offset k;
// the last step of a block tells the next far-kernel launch where it starts.
__device__ __forceinline__ void publish_next_block(const StepArgs &a, int blk, int k, int t)
{
  if(k == kTimeBlock - 1 && blk == 0 && threadIdx.x == 0) *a.d_next = t + 1;
}

// ---- the fused step --------------------------------------------------------------
// One step for 32 dots per thread block: predictor, 11 evaluations and 10
// corrections run in warp 0 (lane = dot); dots coupled at delay 0 share the
// block and exchange their iterates through shared memory after each
// correction.  The other warps form the step's sums.
//
// Summation order, shared by the per-step kernel and the step-block kernel
// so that both give the same bits:
//   window sums  P = S123 + T with S123 = (S1 + S2) + S3: S_p adds the
//                window terms h = p-1, p+2, ... (h <= nt-2) in increasing h
//                and T is the newest term (h = nt-1, step t-1); H likewise;
//   past field   (F + M_old) + M_new: F is the far-pair field; M_old adds,
//                over the dot's mid-list entries in list order, each entry's
//                taps that read step t-2 or earlier (in tap order); M_new
//                adds the taps that read step t-1 (delay 1 tap 0, delay 0
//                tap 1) in new-list order.
// S_p, F + M_old and the pulse need nothing from step t-1, so the
// step-block kernel forms them for step t+1 while step t iterates.
constexpr int kParts = 4;       // warps per block of the per-step kernel
constexpr int kMidChunk = 384;  // mid-list entries staged per pass

// Window term h (step t - nt + h) of one dot added to acc = {P0, P1, H0, H1};
// ps, cs: the predictor and corrector weights (kernel parameters or a copy
// in shared memory).
__device__ __forceinline__ void pc_term(const StepArgs &a, const double *ps, const double *cs, int nt, int h,
                                        double2 x0, double2 x1, double2 y0, double2 y1, double2 (&acc)[4])
{
  const double dt = a.dt;
  const double p0 = ps[h], p1 = ps[nt + h];
  const double c0 = cs[h], c1 = cs[nt + h];
  acc[0].x += x0.x * p0 + (y0.x * p1) * dt;
  acc[0].y += x0.y * p0 + (y0.y * p1) * dt;
  acc[1].x += x1.x * p0 + (y1.x * p1) * dt;
  acc[1].y += x1.y * p0 + (y1.y * p1) * dt;
  acc[2].x += x0.x * c0 + (y0.x * c1) * dt;
  acc[2].y += x0.y * c0 + (y0.y * c1) * dt;
  acc[3].x += x1.x * c0 + (y1.x * c1) * dt;
  acc[3].y += x1.y * c0 + (y1.y * c1) * dt;
}

// Window sources: the predictor-corrector ring in HBM, or a block's copy of
// it in shared memory ([slot][rho00, rho01, drho00, drho01][lane]).
struct PcrWindow {
  const double2 *pcr;
  int n_pad, idx;
  __device__ __forceinline__ double2 operator()(int slot, int c) const
  {
    return pcr[((long long)slot * 4 + c) * n_pad + idx];
  }
};
struct SmemWindow {
  const double2 (*win)[4][32];
  int lane;
  __device__ __forceinline__ double2 operator()(int slot, int c) const { return win[slot][c][lane]; }
};

// S_p (p = 1, 2, 3) of the window sums of step t.
template <int NT, class Win>
__device__ __forceinline__ void pc_partial(const StepArgs &a, const double *ps, const double *cs, int t, int p,
                                           const Win &win, double2 (&acc)[4])
{
  const int nt = NT > 0 ? NT : a.w.n_time;
#pragma unroll
  for(int v = 0; v < 4; ++v) acc[v] = make_double2(0.0, 0.0);
#pragma unroll
  for(int h0 = 0; h0 < (NT > 0 ? NT : 32); h0 += 3) {
    const int h = h0 + p - 1;
    if(h <= nt - 2) {
      const int s = pc_slot(t - nt + h);
      pc_term(a, ps, cs, nt, h, win(s, 0), win(s, 1), win(s, 2), win(s, 3), acc);
    }
  }
}

// T: the newest window term of step t (step t-1).
template <class Win>
__device__ __forceinline__ void pc_newest(const StepArgs &a, const double *ps, const double *cs, int t, int nt,
                                          const Win &win, double2 (&acc)[4])
{
#pragma unroll
  for(int v = 0; v < 4; ++v) acc[v] = make_double2(0.0, 0.0);
  const int s = pc_slot(t - 1);
  pc_term(a, ps, cs, nt, nt - 1, win(s, 0), win(s, 1), win(s, 2), win(s, 3), acc);
}

// The taps of a mid-list entry at step t that read step t-2 or earlier
// (taps before step -22 skipped): partner b, delay d < W - q, coefficients
// c[0..q], tslot = ring_slot(t).  All the taps are fetched before any is
// used, so their loads are in flight together.  CG: loads through L2 only,
// for data another block may have written since this SM last read the line
// (an L1 copy of that line would be stale); otherwise ordinary loads, for
// data written before the kernel started.
template <bool CG>
__device__ __forceinline__ void mid_old_fetch(const StepArgs &a, int b, int d, int t, int tslot,
                                              double2 (&v)[kMaxOrder + 1])
{
  const int q = a.q;
  const double2 *ring = a.ring + (long long)b * a.stride;
  const int s = t - d;
  int base = tslot - d - q;  // slot of step s - q; tap i at base + q - i (mirrored)
  if(base < 0) base += a.W;
#pragma unroll
  for(int i = 0; i <= kMaxOrder; ++i) {
    const bool use = i <= q && s - i >= -kWindow && d + i >= 2;
    v[i] = make_double2(0.0, 0.0);
    if(use) v[i] = CG ? __ldcg(ring + base + q - i) : ring[base + q - i];
  }
}

// The taps' products are independent and summed as a fixed pairwise tree
// over the eight tap slots (absent taps contribute exact zeros), so the
// dependent chain is three adds deep instead of q+1.
__device__ __forceinline__ double2 mid_old_sum(const StepArgs &a, int d, int t, const double2 *c, int cstride,
                                               const double2 (&v)[kMaxOrder + 1])
{
  const int q = a.q;
  const int s = t - d;
  double2 p[kMaxOrder + 1];
#pragma unroll
  for(int i = 0; i <= kMaxOrder; ++i)
    p[i] = (i <= q && s - i >= -kWindow && d + i >= 2) ? cmul(prefactor(v[i], a.frame), c[i * cstride])
                                                        : make_double2(0.0, 0.0);
  static_assert(kMaxOrder + 1 == 8, "tree over 8 tap slots");
  const double2 s01 = make_double2(p[0].x + p[1].x, p[0].y + p[1].y);
  const double2 s23 = make_double2(p[2].x + p[3].x, p[2].y + p[3].y);
  const double2 s45 = make_double2(p[4].x + p[5].x, p[4].y + p[5].y);
  const double2 s67 = make_double2(p[6].x + p[7].x, p[6].y + p[7].y);
  return make_double2((s01.x + s23.x) + (s45.x + s67.x), (s01.y + s23.y) + (s45.y + s67.y));
}

// A dot's staged mid-list entries [lo, hi) of one chunk: even and odd
// positions in two running sums, then their sum (half the dependent chain).
__device__ __forceinline__ double2 entry_sum(const double2 *v, int lo, int hi)
{
  double2 e = make_double2(0.0, 0.0), o = e;
  for(int j = lo; j < hi; j += 2) {
    e.x += v[j].x;
    e.y += v[j].y;
    if(j + 1 < hi) {
      o.x += v[j + 1].x;
      o.y += v[j + 1].y;
    }
  }
  return make_double2(e.x + o.x, e.y + o.y);
}

__device__ __forceinline__ double2 mid_old(const StepArgs &a, int e, int t, int tslot)
{
  const int d = a.mid_delay[e];
  double2 v[kMaxOrder + 1];
  mid_old_fetch<true>(a, a.mid_idx[e], d, t, tslot, v);
  return mid_old_sum(a, d, t, a.mid_coef + (long long)e * (a.q + 1), 1, v);
}

// mid_old of entries [c0, c1) (at most kMidChunk) into out[e - c0], each
// thread taking entries threadIdx.x + j * blockDim.x.  A thread's partners
// and delays are fetched first, then its entries' history samples two
// entries ahead of the sums, so their memory latencies overlap; every
// entry's sum is mid_old's, the same operations in the same order.
__device__ __forceinline__ void mid_old_stage(const StepArgs &a, int c0, int c1, int t, int tslot, double2 *out)
{
  constexpr int U = kMidChunk / (32 * kParts);
  static_assert(U * 32 * kParts == kMidChunk, "chunk = U entries per thread");
  int b[U], d[U];
#pragma unroll
  for(int j = 0; j < U; ++j) {
    const int e = c0 + threadIdx.x + j * 32 * kParts;
    b[j] = e < c1 ? a.mid_idx[e] : 0;
    d[j] = e < c1 ? a.mid_delay[e] : kTimeBlock;
  }
  double2 v0[kMaxOrder + 1], v1[kMaxOrder + 1];
  mid_old_fetch<true>(a, b[0], d[0], t, tslot, v0);
#pragma unroll
  for(int j = 0; j < U; ++j) {
    double2(&cur)[kMaxOrder + 1] = (j & 1) ? v1 : v0;
    double2(&nxt)[kMaxOrder + 1] = (j & 1) ? v0 : v1;
    if(j + 1 < U) mid_old_fetch<true>(a, b[j + 1], d[j + 1], t, tslot, nxt);
    const int e = c0 + threadIdx.x + j * 32 * kParts;
    if(e < c1) out[e - c0] = mid_old_sum(a, d[j], t, a.mid_coef + (long long)e * (a.q + 1), 1, cur);
  }
}

// M_new of dot idx; prev(b) = rho01 of partner b at step t-1.
template <class Prev>
__device__ __forceinline__ double2 mid_new(const StepArgs &a, int j0, int j1, const Prev &prev)
{
  double2 M = make_double2(0.0, 0.0);
  for(int j = j0; j < j1; ++j) {
    const double2 v = cmul(prefactor(prev(a.new_idx[j]), a.frame), a.new_coef[j]);
    M.x += v.x;
    M.y += v.y;
  }
  return M;
}

// A dot's delay-0 partners (slot in the block, tap-0 coefficient): the first
// kNearRegs in registers, any further ones read from the list.
constexpr int kNearRegs = 2;
struct NearRegs {
  int e0, e1;
  int idx[kNearRegs];
  double2 coef[kNearRegs];
};

__device__ __forceinline__ NearRegs near_regs(const StepArgs &a, int idx)
{
  NearRegs n;
  n.e0 = a.near_ptr[idx];
  n.e1 = a.near_ptr[idx + 1];
#pragma unroll
  for(int j = 0; j < kNearRegs; ++j) {
    const bool has = n.e0 + j < n.e1;
    n.idx[j] = has ? a.near_idx[n.e0 + j] : 0;
    n.coef[j] = has ? a.near_coef[n.e0 + j] : make_double2(0.0, 0.0);
  }
  return n;
}

// Predictor, 11 evaluations and 10 corrections of one dot (warp 0, lane =
// dot); the delay-0 partners' iterates are exchanged through cur[].
__device__ __forceinline__ void dot_iterate(const StepArgs &a, bool live, bool block_near, const NearRegs &nr,
                                            double2 *cur, int lane, const double2 (&P)[2], const double2 (&H)[2],
                                            double2 past, double pul, const DotConst &dc, double2 (&r)[2],
                                            double2 (&dr)[2])
{
  r[0] = P[0];
  r[1] = P[1];
  for(int it = 0; it <= kCorrectorSteps; ++it) {
    if(it > 0 && live) corrector(a, dr, H, r);
    double2 nf = make_double2(0.0, 0.0);
    if(block_near) {
      __syncwarp();
      cur[lane] = live ? prefactor(r[1], a.frame) : make_double2(0.0, 0.0);
      __syncwarp();
#pragma unroll
      for(int j = 0; j < kNearRegs; ++j)
        if(nr.e0 + j < nr.e1) {
          const double2 v = cmul(cur[nr.idx[j]], nr.coef[j]);
          nf.x += v.x;
          nf.y += v.y;
        }
      for(int e = nr.e0 + kNearRegs; e < nr.e1; ++e) {
        const double2 v = cmul(cur[a.near_idx[e]], a.near_coef[e]);
        nf.x += v.x;
        nf.y += v.y;
      }
    }
    if(live) {
      const double2 om = make_double2((0.0 + pul) + (past.x + nf.x), 0.0 + (past.y + nf.y));
      liouville(r[0], r[1], om, dc, dr[0], dr[1]);
    }
  }
}

// P = S123 + T, H likewise.
__device__ __forceinline__ void pc_combine(const double2 (&S)[4], const double2 (&T)[4], double2 (&P)[2],
                                           double2 (&H)[2])
{
  P[0] = make_double2(S[0].x + T[0].x, S[0].y + T[0].y);
  P[1] = make_double2(S[1].x + T[1].x, S[1].y + T[1].y);
  H[0] = make_double2(S[2].x + T[2].x, S[2].y + T[2].y);
  H[1] = make_double2(S[3].x + T[3].x, S[3].y + T[3].y);
}

// PIPE: the mid list staged by mid_old_stage (several entries' loads in
// flight per thread, 160 registers: 3 blocks per SM) instead of one entry at a
// time (128 registers: 4 blocks per SM); the same sums either way.
template <int NT, bool PIPE = false>
__device__ __forceinline__ void step_fused_body(const StepArgs &a, int blk, int k)
{
  constexpr int BS = 32;
  __shared__ double2 red[3][4][BS];
  __shared__ double2 midv[kMidChunk];
  __shared__ double2 cur[BS];
  const int lane = threadIdx.x & 31, part = threadIdx.x >> 5;
  const int idx = blk * BS + lane;
  const int t = *a.far_t0 + k;
  if(t >= a.T) return;  // past this ensemble's last step (uniform per block)
  const bool live = a.user[idx] >= 0;
  const int nt = NT > 0 ? NT : a.w.n_time;
  const PcrWindow win{a.pcr, a.n_pad, idx};

  // warp 0's inputs, requested before the gathers complete
  double2 F = make_double2(0.0, 0.0), Mn = F, T[4];
  double pul = 0;
  DotConst dc{};
  if(part == 0) {
    dc = dot_const(a, idx, live);
    if(live) {
      F = a.far_field[(long long)k * a.n_pad + idx];
      pul = pulse_rabi(a, idx, t);
      pc_newest(a, a.w.ps, a.w.cs, t, nt, win, T);
      const int slot = ring_slot(t - 1, a.W);
      Mn = mid_new(a, a.new_ptr[idx], a.new_ptr[idx + 1],
                   [&](int b) { return __ldcg(a.ring + (long long)b * a.stride + slot); });
    }
  } else if(live) {
    double2 S[4];
    pc_partial<NT>(a, a.w.ps, a.w.cs, t, part, win, S);
#pragma unroll
    for(int v = 0; v < 4; ++v) red[part - 1][v][lane] = S[v];
  }

  // mid list of the block's 32 dots, CSR range [E0, E1): entries staged by
  // all threads, added per dot in list order by warp 0
  const int E0 = a.mid_ptr[blk * BS], E1 = a.mid_ptr[blk * BS + BS];
  const int my0 = a.mid_ptr[idx], my1 = a.mid_ptr[idx + 1];
  double2 Mo = make_double2(0.0, 0.0);
  const int tslot = ring_slot(t, a.W);
  for(int c0 = E0; c0 < E1; c0 += kMidChunk) {
    const int c1 = min(E1, c0 + kMidChunk);
    if(PIPE)
      mid_old_stage(a, c0, c1, t, tslot, midv);
    else
      for(int e = c0 + threadIdx.x; e < c1; e += 32 * kParts) midv[e - c0] = mid_old(a, e, t, tslot);
    __syncthreads();
    if(part == 0) {
      const double2 cs = entry_sum(midv, max(my0, c0) - c0, min(my1, c1) - c0);
      Mo.x += cs.x;
      Mo.y += cs.y;
    }
    __syncthreads();
  }
  if(E0 == E1) __syncthreads();  // the window partials are complete

  if(part == 0) {
    const bool block_near = a.near_ptr[(blk + 1) * BS] > a.near_ptr[blk * BS];
    double2 P[2], H[2], r[2], dr[2], past = make_double2(0.0, 0.0);
    if(live) {
      double2 S[4];
#pragma unroll
      for(int v = 0; v < 4; ++v)
        S[v] = make_double2((red[0][v][lane].x + red[1][v][lane].x) + red[2][v][lane].x,
                            (red[0][v][lane].y + red[1][v][lane].y) + red[2][v][lane].y);
      pc_combine(S, T, P, H);
      past = make_double2((F.x + Mo.x) + Mn.x, (F.y + Mo.y) + Mn.y);
    }
    dot_iterate(a, live, block_near, near_regs(a, idx), cur, lane, P, H, past, pul, dc, r, dr);
    if(live) finish_dot(a, idx, t, r, dr);
  }
  publish_next_block(a, blk, k, t);
}

template <int NT>
__global__ void __launch_bounds__(32 * kParts) step_fused_kernel(StepArgs a, int k)
{
  step_fused_body<NT>(a, a.blk_lo + blockIdx.x, k);
}

// Many ensembles, one launch: block_off[e] = first 32-dot block of ensemble e.
template <int NT, bool PIPE>
__global__ void __launch_bounds__(32 * kParts) step_batch_kernel(const StepArgs *__restrict__ args,
                                                                 const int *__restrict__ block_off,
                                                                 int n_ens, int k)
{
  const int b = blockIdx.x;
  int lo = 0, hi = n_ens - 1;
  while(lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if(block_off[mid] <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  step_fused_body<NT, PIPE>(args[lo], b - block_off[lo], k);
}

void launch_step_batch(const StepArgs *args, const int *block_off, int n_ens, int total_blocks, int n_time,
                       int k, bool pipe, void *stream)
{
  if(n_ens <= 0 || total_blocks <= 0) return;
  cudaStream_t s = (cudaStream_t)stream;
  if(n_time == 22)
    pipe ? step_batch_kernel<22, true><<<total_blocks, 32 * kParts, 0, s>>>(args, block_off, n_ens, k)
         : step_batch_kernel<22, false><<<total_blocks, 32 * kParts, 0, s>>>(args, block_off, n_ens, k);
  else
    pipe ? step_batch_kernel<0, true><<<total_blocks, 32 * kParts, 0, s>>>(args, block_off, n_ens, k)
         : step_batch_kernel<0, false><<<total_blocks, 32 * kParts, 0, s>>>(args, block_off, n_ens, k);
}

// ---- one launch for a whole 16-step block ------------------------------------
// The steps k0 .. k1-1 of a block in one cooperative launch (every thread
// block resident), 8 warps per 32 dots.  Each block keeps in shared memory
// its dots' predictor-corrector window (23 steps of rho and rho-dot), the
// integrator weights, the launch's far-pair field and pulse, and (when they
// fit) its part of the mid list and the recent rho01 of each distinct
// mid-list partner.  Warp 0 runs step k on a scheduler of its own (warp 4,
// which would share it, stays idle) while warps 1-3 and 5-7 form step k+1's
// window partials S_p and F + M_old (double-buffered).  M_old reads the
// partners' history of step k-1 and earlier, so the helpers first wait until
// every block that holds one of the block's mid-list partners (and the block
// itself) has finished step k-1.  Each block counts its finished steps in
// flags[block * kFlagStride] (zeroed before the launch); warp 0 posts a step
// as soon as its rho01 is stored.  The post is on the critical path between
// blocks (a partner's post, then the helpers' work, bounds the step), so
// warp 0 posts it itself: handing it to another warp through a barrier
// delays it by that warp's wake-up and fence.  Blocks wait only for their
// partners' blocks, so nearby blocks may run a step or two apart and no
// global barrier is needed.
//
// M_new reads step k-1 of the delay-0/1 partners: with a.lag set every such
// partner is in the dot's own block and its value comes from shared memory;
// otherwise warp 0 also waits for its partner blocks' step k-1.
// Every wait is bounded (about a second); a wait that runs out sets
// *a.d_bad to -2 and the kernel returns.
constexpr int kBlockWarps = 8;
constexpr int kHelperWarps = 6;                // warps 1, 2, 3, 5, 6, 7
constexpr int kHelpers = 32 * kHelperWarps;
constexpr int kBarrierSpins = 1 << 24;         // x ~64 ns of sleep: about a second
constexpr int kFastPolls = 64;                 // polls before the first sleep
constexpr int kWeightSlots = 64;               // 2 x n_time, n_time <= 32

// Partner history: the rho01 samples that mid-list taps read, for each of a
// block's distinct partners, slot = step mod kHistDepth, rows padded to
// kHistStride so rows start in different banks.  A step t reads samples
// t-22 .. t-2 (delay <= K-1, tap <= kMaxOrder, delay + tap >= 2).
constexpr int kHistDepth = 24;
constexpr int kHistStride = 25;
constexpr int kHistSpan = (kTimeBlock - 1) + kMaxOrder;  // t - kHistSpan is the oldest sample read

__device__ __forceinline__ int hist_slot(int s) { return ((s % kHistDepth) + kHistDepth) % kHistDepth; }

// Step flags: a block posts a finished step with a release add (its rho01
// stores become visible before the count), and readers poll with acquire
// loads (the posting block's stores are visible once the count is seen).
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void post_step(unsigned *p)
{
  asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(p) : "memory");
}

// Called by a whole warp: waits until flags[list[i] * kFlagStride] >= target
// for every i < n (the lanes poll in parallel, each wait bounded by `limit`
// polls, kBarrierSpins when 0).  False if a wait ran out.
__device__ __forceinline__ bool wait_blocks(const unsigned *flags, const int *list, int n, unsigned target,
                                            int limit)
{
  bool ok = true;
  const int max_spins = limit > 0 ? limit : kBarrierSpins;
  for(int i = threadIdx.x & 31; i < n && ok; i += 32) {
    const unsigned *f = flags + (long long)__ldg(list + i) * kFlagStride;
    int spins = 0;
    while(ld_acquire(f) < target) {
      if(++spins > max_spins) {
        ok = false;
        break;
      }
      if(spins > kFastPolls) __nanosleep(32);
    }
  }
  return __all_sync(0xffffffffu, ok);
}

__device__ __forceinline__ void helpers_sync() { asm volatile("bar.sync 1, %0;" ::"r"(kHelpers)); }

// S_p of either the predictor sums (HQ = false: rho00, rho01) or the
// corrector sums (HQ = true), each accumulator with the same operations as
// pc_partial.
template <int NT, bool HQ, class Win>
__device__ __forceinline__ void pc_partial_half(const StepArgs &a, const double *ps, const double *cs, int t, int p,
                                                const Win &win, double2 (&acc)[2])
{
  const int nt = NT > 0 ? NT : a.w.n_time;
  const double dt = a.dt;
  acc[0] = acc[1] = make_double2(0.0, 0.0);
#pragma unroll
  for(int h0 = 0; h0 < (NT > 0 ? NT : 32); h0 += 3) {
    const int h = h0 + p - 1;
    if(h <= nt - 2) {
      const int s = pc_slot(t - nt + h);
      const double2 x0 = win(s, 0), x1 = win(s, 1), y0 = win(s, 2), y1 = win(s, 3);
      const double w0 = HQ ? cs[h] : ps[h], w1 = HQ ? cs[nt + h] : ps[nt + h];
      acc[0].x += x0.x * w0 + (y0.x * w1) * dt;
      acc[0].y += x0.y * w0 + (y0.y * w1) * dt;
      acc[1].x += x1.x * w0 + (y1.x * w1) * dt;
      acc[1].y += x1.y * w0 + (y1.y * w1) * dt;
    }
  }
}

// Shared-memory layout of the step-block kernel.
struct BlockSmem {
  double2 (*win)[4][32];  // [kPcDepth][4][32]
  double2 *pre_s;         // [2][3][4][32] S_p
  double2 *pre_f;         // [2][32] F + M_old
  double2 *far;           // [K][32] far-pair field of the launch's steps
  double2 *midv;          // [kMidChunk] staged entries
  double2 *cur;           // [32] delay-0 exchange
  double2 *prev01;        // [32] rho01 of step t-1
  double2 *mc_coef;       // [q+1][mid_cache] the block's mid-list coefficients, tap-major
  double2 *hist;          // [hist_cap][kHistStride] rho01 of the block's distinct partners
  double *pul;            // [K][32] pulse of the launch's steps
  double *ps, *cs;        // [kWeightSlots] each
  int *mc_idx, *mc_del;   // [mid_cache] partners (with hist: partner slots) and delays
  int *bp;                // [hist_cap] the distinct partners' internal indices
};

// Per-thread constants of the helpers' step work, read once per launch.
struct BlockConst {
  bool live;
  int E0, E, my0, my1;  // the block's mid-list range; this lane's dot's sub-range (local)
  int NP;               // distinct partners (partner history)
};

__host__ __device__ __forceinline__ size_t block_smem_bytes(int q, int mid_cache, int hist_cap)
{
  return sizeof(double2) * ((size_t)kPcDepth * 4 * 32 + 2 * 3 * 4 * 32 + 2 * 32 + kTimeBlock * 32 + kMidChunk + 32 +
                            32 + (size_t)mid_cache * (q + 1) + (size_t)hist_cap * kHistStride) +
         sizeof(double) * (kTimeBlock * 32 + 2 * kWeightSlots) + sizeof(int) * 2 * (size_t)mid_cache +
         sizeof(int) * (size_t)hist_cap;
}

__device__ __forceinline__ BlockSmem block_smem(double2 *base, int q, int mid_cache, int hist_cap)
{
  BlockSmem m;
  m.win = reinterpret_cast<double2(*)[4][32]>(base);
  m.pre_s = base + kPcDepth * 4 * 32;
  m.pre_f = m.pre_s + 2 * 3 * 4 * 32;
  m.far = m.pre_f + 2 * 32;
  m.midv = m.far + kTimeBlock * 32;
  m.cur = m.midv + kMidChunk;
  m.prev01 = m.cur + 32;
  m.mc_coef = m.prev01 + 32;
  m.hist = m.mc_coef + (size_t)mid_cache * (q + 1);
  m.pul = reinterpret_cast<double *>(m.hist + (size_t)hist_cap * kHistStride);
  m.ps = m.pul + kTimeBlock * 32;
  m.cs = m.ps + kWeightSlots;
  m.mc_idx = reinterpret_cast<int *>(m.cs + kWeightSlots);
  m.mc_del = m.mc_idx + mid_cache;
  m.bp = m.mc_del + mid_cache;
  return m;
}

// Step k's sums by the helper warps (hw = 0..5) into buffer `b`:
// pre_s[b][p-1][v][lane] = S_p of quantity v, pre_f[b] = F + M_old.
template <int NT>
__device__ __forceinline__ void block_precompute(const StepArgs &a, const BlockSmem &m, const BlockConst &bc,
                                                 int k, int t, int b, bool cached, bool hist, int hw)
{
  constexpr int BS = 32;
  const int lane = threadIdx.x & 31;
  const int tid = hw * 32 + lane;
  const bool live = bc.live;
  const int E0 = bc.E0, E = bc.E, my0 = bc.my0, my1 = bc.my1;
  const int q1 = a.q + 1, cap = a.mid_cache;
  if(hist) {
    // the newest sample the old taps read (step t-2, finished by the
    // partners' blocks), one L2 load per distinct partner of the block
    const int sa = t - 2, hs = hist_slot(sa), rs = ring_slot(sa, a.W);
    for(int j = tid; j < bc.NP; j += kHelpers)
      m.hist[j * kHistStride + hs] = __ldcg(a.ring + (long long)m.bp[j] * a.stride + rs);
    helpers_sync();
  }
  // mid-list entries of the block (local index e = entry - E0) staged by
  // the helpers, added per dot in list order by helper warp 0
  const int tslot = ring_slot(t, a.W);
  double2 Mo = make_double2(0.0, 0.0);
  for(int c0 = 0; c0 < E; c0 += kMidChunk) {
    const int c1 = min(E, c0 + kMidChunk);
    for(int e = c0 + tid; e < c1; e += kHelpers) {
      const int pb = cached ? m.mc_idx[e] : a.mid_idx[E0 + e];
      const int d = cached ? m.mc_del[e] : a.mid_delay[E0 + e];
      double2 v[kMaxOrder + 1];
      if(hist) {
        const double2 *h = m.hist + pb * kHistStride;
        const int hb = hist_slot(t - d);
#pragma unroll
        for(int i = 0; i <= kMaxOrder; ++i) {
          const int sl = hb - i < 0 ? hb - i + kHistDepth : hb - i;
          v[i] = (i <= a.q && t - d - i >= -kWindow && d + i >= 2) ? h[sl] : make_double2(0.0, 0.0);
        }
      } else {
        mid_old_fetch<true>(a, pb, d, t, tslot, v);
      }
      m.midv[e - c0] = cached ? mid_old_sum(a, d, t, m.mc_coef + e, cap, v)
                              : mid_old_sum(a, d, t, a.mid_coef + (long long)(E0 + e) * q1, 1, v);
    }
    helpers_sync();
    if(hw == 0) {
      const double2 cs = entry_sum(m.midv, max(my0, c0) - c0, min(my1, c1) - c0);
      Mo.x += cs.x;
      Mo.y += cs.y;
    }
    helpers_sync();
  }
  if(!live) return;
  if(hw == 0) {
    const double2 F = m.far[k * BS + lane];
    m.pre_f[b * BS + lane] = make_double2(F.x + Mo.x, F.y + Mo.y);
  }
  // window partials: helper warp hw takes (p, P or H) = (hw/2 + 1, hw odd)
  const int p = hw / 2 + 1;
  const SmemWindow src{m.win, lane};
  double2 S[2];
  if(hw & 1)
    pc_partial_half<NT, true>(a, m.ps, m.cs, t, p, src, S);
  else
    pc_partial_half<NT, false>(a, m.ps, m.cs, t, p, src, S);
  const int v0 = (hw & 1) ? 2 : 0;
  double2 *ps = m.pre_s + b * 3 * 4 * BS;
  ps[((p - 1) * 4 + v0) * BS + lane] = S[0];
  ps[((p - 1) * 4 + v0 + 1) * BS + lane] = S[1];
}

template <int NT>
__global__ void __launch_bounds__(32 * kBlockWarps, 2) step_block_kernel(StepArgs a, int k0, int k1,
                                                                          unsigned *flags)
{
  constexpr int BS = 32;
  extern __shared__ double2 smem_block[];  // dynamic: above the 48 KB static limit
  const BlockSmem m = block_smem(smem_block, a.q, a.mid_cache, a.hist_cap);
  __shared__ int s_abort;
  const int lane = threadIdx.x & 31, part = threadIdx.x >> 5;
  const int hw = part < 4 ? part - 1 : part - 2;  // helper index; warp 0 -> -1, warp 4 -> 2 (unused)
  const bool helper = part != 0 && part != 4;
  const int blk = blockIdx.x;
  const int idx = blk * BS + lane;
  const int t0 = *a.far_t0;
  const bool live = a.user[idx] >= 0;
  const int nt = NT > 0 ? NT : a.w.n_time;
  const int B0 = a.pb_ptr[blk], NB = a.pb_ptr[blk + 1] - B0;  // blocks holding this block's partners

  // prologue: window, weights, the launch's far field and pulse, prev01, and
  // the block's mid list and partner history when they fit.  The copies are
  // latency-bound (one L2 round trip each), so each thread issues several
  // independent loads before it stores any.
  constexpr int kPro = 4;  // loads in flight per thread in the copy loops
  for(int sl = part; sl < kPcDepth; sl += kBlockWarps) {
    double2 v[4];
#pragma unroll
    for(int c = 0; c < 4; ++c) v[c] = a.pcr[((long long)sl * 4 + c) * a.n_pad + idx];
#pragma unroll
    for(int c = 0; c < 4; ++c) m.win[sl][c][lane] = v[c];
  }
  for(int i = threadIdx.x; i < 2 * nt; i += blockDim.x) {
    m.ps[i] = a.w.ps[i];
    m.cs[i] = a.w.cs[i];
  }
  {
    // the pulse from the dot's k.r and dipole, loaded once (pulse_rabi's
    // operations)
    const double kr = live ? pulse_kr(a, idx) : 0.0;
    const double d0 = live ? a.dip[3 * idx] : 0.0, d1 = live ? a.dip[3 * idx + 1] : 0.0,
                 d2 = live ? a.dip[3 * idx + 2] : 0.0;
    for(int kk = k0 + part; kk < k1; kk += kBlockWarps) {
      m.far[kk * BS + lane] = live ? a.far_field[(long long)kk * a.n_pad + idx] : make_double2(0.0, 0.0);
      m.pul[kk * BS + lane] = live ? pulse_at(a, kr, d0, d1, d2, t0 + kk) : 0.0;
    }
  }
  const int E0 = a.mid_ptr[blk * BS], E = a.mid_ptr[blk * BS + BS] - E0;
  const bool cached = E <= a.mid_cache;
  const int P0 = a.bp_ptr[blk], NP = a.bp_ptr[blk + 1] - P0;
  const bool hist = cached && a.hist_cap > 0 && NP <= a.hist_cap;
  if(cached) {
    const int q1 = a.q + 1, total = E * q1;
    for(int i0 = threadIdx.x; i0 < total; i0 += kPro * blockDim.x) {
      double2 v[kPro];
#pragma unroll
      for(int u = 0; u < kPro; ++u) {
        const int i = i0 + u * blockDim.x;
        if(i < total) v[u] = a.mid_coef[(long long)E0 * q1 + i];
      }
#pragma unroll
      for(int u = 0; u < kPro; ++u) {
        const int i = i0 + u * blockDim.x;
        if(i < total) {
          const int e = i / q1, tap = i - e * q1;
          m.mc_coef[tap * a.mid_cache + e] = v[u];
        }
      }
    }
    for(int i = threadIdx.x; i < E; i += blockDim.x) {
      m.mc_idx[i] = hist ? a.mid_pj[E0 + i] : a.mid_idx[E0 + i];
      m.mc_del[i] = a.mid_delay[E0 + i];
    }
  }
  if(hist) {
    for(int i = threadIdx.x; i < NP; i += blockDim.x) m.bp[i] = a.bp_idx[P0 + i];
    __syncthreads();  // uniform: hist depends on the block only
    // samples t0+k0-22 .. t0+k0-2; later ones are appended step by step
    const int first = t0 + k0 - kHistSpan, count = kHistSpan - 1, total = NP * count;
    for(int i0 = threadIdx.x; i0 < total; i0 += kPro * blockDim.x) {
      double2 v[kPro];
#pragma unroll
      for(int u = 0; u < kPro; ++u) {
        const int i = i0 + u * blockDim.x;
        if(i < total) {
          const int j = i / count, s = first + i % count;
          v[u] = __ldcg(a.ring + (long long)m.bp[j] * a.stride + ring_slot(s, a.W));
        }
      }
#pragma unroll
      for(int u = 0; u < kPro; ++u) {
        const int i = i0 + u * blockDim.x;
        if(i < total) {
          const int j = i / count, s = first + i % count;
          m.hist[j * kHistStride + hist_slot(s)] = v[u];
        }
      }
    }
  }
  if(part == 0) m.prev01[lane] = a.ring[(long long)idx * a.stride + ring_slot(t0 + k0 - 1, a.W)];
  if(threadIdx.x == 0) s_abort = 0;
  BlockConst bc;
  bc.live = live;
  bc.E0 = E0;
  bc.E = E;
  bc.my0 = a.mid_ptr[idx] - E0;
  bc.my1 = a.mid_ptr[idx + 1] - E0;
  bc.NP = NP;
  __syncthreads();
  if(helper && t0 + k0 < a.T) block_precompute<NT>(a, m, bc, k0, t0 + k0, k0 & 1, cached, hist, hw);
  const DotConst dc = dot_const(a, idx, live);
  const bool block_near = a.near_ptr[(blk + 1) * BS] > a.near_ptr[blk * BS];
  const NearRegs nr = near_regs(a, idx);
  const int nw0 = a.new_ptr[idx], nw1 = a.new_ptr[idx + 1];
  __syncthreads();

  for(int k = k0; k < k1; ++k) {
    const int t = t0 + k;
    if(t >= a.T || s_abort) break;  // uniform across the block
    const int buf = k & 1;
    if(part == 0) {
      bool ok = true;
      if(!a.lag && k > k0) ok = wait_blocks(flags, a.pb_idx + B0, NB, k - k0, a.spin_limit);  // partners' step t-1
      if(ok) {
        double2 P[2], H[2], r[2], dr[2], past = make_double2(0.0, 0.0);
        double pul = 0;
        if(live) {
          double2 S[4], T[4];
          const double2 *ps = m.pre_s + buf * 3 * 4 * BS;
#pragma unroll
          for(int v = 0; v < 4; ++v) {
            const double2 s1 = ps[(0 * 4 + v) * BS + lane], s2 = ps[(1 * 4 + v) * BS + lane],
                          s3 = ps[(2 * 4 + v) * BS + lane];
            S[v] = make_double2((s1.x + s2.x) + s3.x, (s1.y + s2.y) + s3.y);
          }
          pc_newest(a, m.ps, m.cs, t, nt, SmemWindow{m.win, lane}, T);
          pc_combine(S, T, P, H);
          double2 Mn;
          if(a.lag) {
            Mn = mid_new(a, nw0, nw1, [&](int b) { return m.prev01[b & 31]; });
          } else {
            const int slot = ring_slot(t - 1, a.W);
            Mn = mid_new(a, nw0, nw1, [&](int b) { return __ldcg(a.ring + (long long)b * a.stride + slot); });
          }
          const double2 F = m.pre_f[buf * BS + lane];
          past = make_double2(F.x + Mn.x, F.y + Mn.y);
          pul = m.pul[k * BS + lane];
        }
        dot_iterate(a, live, block_near, nr, m.cur, lane, P, H, past, pul, dc, r, dr);
        // rho01 first, then post the step, then the rest of the state
        if(live) finish_ring(a, idx, t, r);
        __syncwarp();
        if(lane == 0 && blk != a.skip_post_block) post_step(flags + (long long)blk * kFlagStride);
        if(live) {
          finish_state(a, idx, t, r, dr);
          const int sl = pc_slot(t);
          m.win[sl][0][lane] = r[0];
          m.win[sl][1][lane] = r[1];
          m.win[sl][2][lane] = dr[0];
          m.win[sl][3][lane] = dr[1];
        }
        __syncwarp();
        m.prev01[lane] = live ? r[1] : make_double2(0.0, 0.0);
        if(k == kTimeBlock - 1 && blk == 0 && lane == 0) *a.d_next = t + 1;
      } else if(lane == 0) {
        s_abort = 1;
        atomicMin(a.d_bad, -2);
      }
    } else if(helper && k + 1 < k1 && t + 1 < a.T) {
      // step k+1's sums; M_old needs the partner blocks' step k-1
      if(hw == 0 && k > k0 && !wait_blocks(flags, a.pb_idx + B0, NB, k - k0, a.spin_limit) && lane == 0) {
        s_abort = 1;
        atomicMin(a.d_bad, -2);
      }
      helpers_sync();
      if(!*(volatile int *)&s_abort) block_precompute<NT>(a, m, bc, k + 1, t + 1, buf ^ 1, cached, hist, hw);
    }
    __syncthreads();
  }
}

static void step_block_attrs(size_t smem)
{
  cudaFuncSetAttribute(step_block_kernel<22>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(step_block_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

void launch_step_block(const StepArgs &a, int k0, int k1, int nblocks, unsigned *flags, void *stream)
{
  cudaStream_t s = (cudaStream_t)stream;
  const size_t smem = block_smem_bytes(a.q, a.mid_cache, a.hist_cap);
  step_block_attrs(smem);
  cudaMemsetAsync(flags, 0, sizeof(unsigned) * nblocks * kFlagStride, s);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblocks);
  cfg.blockDim = dim3(32 * kBlockWarps);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeCooperative;
  attr.val.cooperative = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  if(a.w.n_time == 22)
    cudaLaunchKernelEx(&cfg, step_block_kernel<22>, a, k0, k1, flags);
  else
    cudaLaunchKernelEx(&cfg, step_block_kernel<0>, a, k0, k1, flags);
}

// Thread blocks of the step-block kernel that fit on the device at once
// with a mid-list cache of `mid_cache` entries and partner history for
// `hist_cap` partners per block (0 when the shared memory does not fit).
int step_block_max_blocks(int q, int mid_cache, int hist_cap)
{
  const size_t smem = block_smem_bytes(q, mid_cache, hist_cap);
  int dev = 0, sms = 0, per = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if(smem > (size_t)optin) return 0;
  step_block_attrs(smem);
  if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step_block_kernel<22>, 32 * kBlockWarps, smem) !=
     cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return sms * per;
}

// General form, one launch per phase: phase 0 predicts, phases 1..11 are the
// 11 evaluations (each followed by a correction except the last).
// scratch[idx*8 + k]: 0 past field, 1 pulse, 2-3 H, 4-5 rho (even
// iterations), 6-7 rho (odd iterations).
__global__ void __launch_bounds__(kStepBlock) step_general_kernel(StepArgs a, int k, int phase)
{
  const int idx = blockIdx.x * kStepBlock + threadIdx.x;
  const int t = *a.far_t0 + k;
  const bool live = idx < a.n_pad && a.user[idx] >= 0;
  double2 *sc = a.scratch + (long long)idx * 8;
  if(phase == 0) {
    if(live) {
      double2 P[2], H[2];
      if(a.w.n_time == 22)
        pc_window<22>(a, idx, t, P, H);
      else
        pc_window<0>(a, idx, t, P, H);
      sc[0] = past_field(a, idx, t, k);
      sc[1] = make_double2(pulse_rabi(a, idx, t), 0.0);
      sc[2] = H[0];
      sc[3] = H[1];
      sc[4] = P[0];
      sc[5] = P[1];
    }
    return;
  }
  const int it = phase - 1;
  const int rd = (it & 1) ? 6 : 4, wr = (it & 1) ? 4 : 6;
  if(live) {
    double2 r[2] = {sc[rd], sc[rd + 1]};
    double2 nf = make_double2(0.0, 0.0);
    for(int e = a.near_ptr[idx]; e < a.near_ptr[idx + 1]; ++e) {
      const int b = a.near_idx[e];
      const double2 v = cmul(prefactor(a.scratch[(long long)b * 8 + rd + 1], a.frame), a.near_coef[e]);
      nf.x += v.x;
      nf.y += v.y;
    }
    const double2 past = sc[0];
    const double pul = sc[1].x;
    const double2 om = make_double2((0.0 + pul) + (past.x + nf.x), 0.0 + (past.y + nf.y));
    double2 dr[2];
    liouville(r[0], r[1], om, dot_const(a, idx, true), dr[0], dr[1]);
    if(it < kCorrectorSteps) {
      const double2 H[2] = {sc[2], sc[3]};
      corrector(a, dr, H, r);
      sc[wr] = r[0];
      sc[wr + 1] = r[1];
    } else {
      finish_dot(a, idx, t, r, dr);
    }
  }
  if(it == kCorrectorSteps) publish_next_block(a, blockIdx.x, k, t);
}

void launch_step_fused(const StepArgs &a, int k, int nblocks, void *stream)
{
  cudaStream_t s = (cudaStream_t)stream;
  if(a.w.n_time == 22)
    step_fused_kernel<22><<<nblocks, 32 * kParts, 0, s>>>(a, k);
  else
    step_fused_kernel<0><<<nblocks, 32 * kParts, 0, s>>>(a, k);
}

void launch_step_general(const StepArgs &a, int k, int phase, void *stream)
{
  const int nblocks = (a.n_pad + kStepBlock - 1) / kStepBlock;
  step_general_kernel<<<nblocks, kStepBlock, 0, (cudaStream_t)stream>>>(a, k, phase);
}

// HistoryInteraction::evaluate at an explicit step: past partial sums plus
// the delay-0 tap-0 terms read from the ring at `step`, in user order.
__global__ void eval_field_kernel(StepArgs a, const int *d_eval_step, double2 *out)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if(idx >= a.n_pad || a.user[idx] < 0) return;
  const int step = *d_eval_step;
  const int slot = ring_slot(step, a.W);
  double2 f = past_field(a, idx, step, 0);
  for(int e = a.near_ptr[idx]; e < a.near_ptr[idx + 1]; ++e) {
    const int b = a.near_idx[e];
    const double2 v = cmul(prefactor(a.ring[(long long)b * a.stride + slot], a.frame), a.near_coef[e]);
    f.x += v.x;
    f.y += v.y;
  }
  out[a.user[idx]] = f;
}

void launch_eval_field(const StepArgs &a, const int *d_eval_step, double2 *out_user, void *stream)
{
  eval_field_kernel<<<(a.n_pad + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a, d_eval_step, out_user);
}

__global__ void pulse_field_kernel(StepArgs a, int step, double2 *out)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if(idx >= a.n_pad || a.user[idx] < 0) return;
  out[a.user[idx]] = make_double2(pulse_rabi(a, idx, step), 0.0);
}

void launch_pulse_field(const StepArgs &a, int step, double2 *out_user, void *stream)
{
  pulse_field_kernel<<<(a.n_pad + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a, step, out_user);
}

__global__ void set_int_kernel(int *p, int v) { *p = v; }

void launch_set_int(int *p, int v, void *stream)
{
  set_int_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(p, v);
}

// main.cpp:30-36: rho = (1, 0) and rho-dot = 0 in every PC slot (steps
// -22..0); the ring (rho01 = 0 at t <= 0) is zeroed by the caller.
__global__ void init_state_kernel(StepArgs a)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)kPcDepth * a.n_pad;
  if(i >= total) return;
  const long long s = i / a.n_pad, d = i % a.n_pad;
  double2 *base = a.pcr + s * 4 * a.n_pad + d;
  base[0] = make_double2(1.0, 0.0);
  base[a.n_pad] = make_double2(0.0, 0.0);
  base[2 * a.n_pad] = make_double2(0.0, 0.0);
  base[3 * a.n_pad] = make_double2(0.0, 0.0);
}

__global__ void shard_export_kernel(StepArgs a, int t, int lo, int hi, double2 *out)
{
  const int idx = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if(idx >= hi) return;
  out[idx - lo] = a.user[idx] >= 0 ? a.ring[(long long)idx * a.stride + ring_slot(t, a.W)] : make_double2(0.0, 0.0);
}

void launch_shard_export(const StepArgs &a, int t, int lo, int hi, double2 *out, void *stream)
{
  if(hi > lo) shard_export_kernel<<<(hi - lo + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a, t, lo, hi, out);
}

// The other shards' dots: their rho01 at step t written exactly as their own
// step kernel writes it (finish_ring: FP64 ring, and in mixed precision the
// FP32 value and the FP64-formed step difference).
__global__ void shard_import_kernel(StepArgs a, int t, int lo, int hi, const double2 *full)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if(idx >= a.n_pad || (idx >= lo && idx < hi) || a.user[idx] < 0) return;
  double2 r[2];
  r[0] = make_double2(0.0, 0.0);
  r[1] = full[idx];
  finish_ring(a, idx, t, r);
}

void launch_shard_import(const StepArgs &a, int t, int lo, int hi, const double2 *full, void *stream)
{
  shard_import_kernel<<<(a.n_pad + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a, t, lo, hi, full);
}

__global__ void gather_bad_kernel(const StepArgs *args, int n, int *out)
{
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if(e < n) out[e] = *args[e].d_bad;
}

void launch_gather_bad(const StepArgs *args, int n, int *out, void *stream)
{
  if(n > 0) gather_bad_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(args, n, out);
}

void launch_init_state(const StepArgs &a, void *stream)
{
  const long long total = (long long)kPcDepth * a.n_pad;
  init_state_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
}

__global__ void ring_write_kernel(StepArgs a, int t, const double2 *rho01_user)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if(idx >= a.n_pad || a.user[idx] < 0) return;
  const int slot = ((t % a.W) + a.W) % a.W;
  const double2 v = rho01_user[a.user[idx]];
  double2 *ring = a.ring + (long long)idx * a.stride;
  ring[slot] = v;
  if(slot < kRingMirror) ring[a.W + slot] = v;
}

void launch_ring_write(const StepArgs &a, int t, const double2 *rho01_user, void *stream)
{
  ring_write_kernel<<<(a.n_pad + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a, t, rho01_user);
}

__global__ void ring_read_kernel(StepArgs a, int t, double2 *rho01_user)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if(idx >= a.n_pad || a.user[idx] < 0) return;
  const int slot = ((t % a.W) + a.W) % a.W;
  rho01_user[a.user[idx]] = a.ring[(long long)idx * a.stride + slot];
}

void launch_ring_read(const StepArgs &a, int t, double2 *rho01_user, void *stream)
{
  ring_read_kernel<<<(a.n_pad + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a, t, rho01_user);
}

// rho (rho00, rho01) of every dot at step t (t >= -22), user order.
__global__ void state_read_kernel(StepArgs a, int t, double2 *rho_user)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if(idx >= a.n_pad || a.user[idx] < 0) return;
  const double2 *base = a.pcr + (long long)pc_slot(t) * 4 * a.n_pad + idx;
  rho_user[2 * a.user[idx]] = base[0];
  rho_user[2 * a.user[idx] + 1] = base[a.n_pad];
}

void launch_state_read(const StepArgs &a, int t, double2 *rho_user, void *stream)
{
  state_read_kernel<<<(a.n_pad + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a, t, rho_user);
}

// Mixed precision: the FP32 rings rebuilt from the FP64 ring (after the
// caller wrote history with qg_set_history).
__global__ void ring32_rebuild_kernel(StepArgs a)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= (long long)a.n_pad * a.W) return;
  const int idx = (int)(i / a.W), slot = (int)(i % a.W);
  const double2 *ring = a.ring + (long long)idx * a.stride;
  const double2 v = ring[slot], prev = ring[slot == 0 ? a.W - 1 : slot - 1];
  const float2 w = make_float2((float)v.x, (float)v.y);
  const float2 d = make_float2((float)(v.x - prev.x), (float)(v.y - prev.y));
  float2 *rw = a.ring32w + (long long)idx * a.stride, *rd = a.ring32d + (long long)idx * a.stride;
  rw[slot] = w;
  rd[slot] = d;
  if(slot < kRingMirror) {
    rw[a.W + slot] = w;
    rd[a.W + slot] = d;
  }
}

void launch_ring32_rebuild(const StepArgs &a, void *stream)
{
  if(!a.ring32w) return;
  const long long total = (long long)a.n_pad * a.W;
  ring32_rebuild_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
}

}  // namespace qg
