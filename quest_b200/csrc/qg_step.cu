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

__device__ __forceinline__ void liouville(double2 r0, double2 r1, double2 om, double t1, double t2,
                                          double det, double2 &m0, double2 &m1)
{
  const double2 r1c = make_double2(r1.x, -r1.y), omc = make_double2(om.x, -om.y);
  const double2 mi = make_double2(-0.0, -1.0);  // -iu
  const double2 u = cmul(om, r1c), v = cmul(omc, r1);
  m0 = cmul(mi, make_double2(u.x - v.x, u.y - v.y));
  m0.x = m0.x - (r0.x - 1.0) / t1;
  m0.y = m0.y - r0.y / t1;
  const double2 one_m = make_double2(1.0 - 2.0 * r0.x, -(2.0 * r0.y));
  const double2 aa = cmul(om, one_m);
  const double2 ab = make_double2(aa.x + r1.x * det, aa.y + r1.y * det);
  m1 = cmul(mi, ab);
  m1.x = m1.x - r1.x / t2;
  m1.y = m1.y - r1.y / t2;
}

__device__ __forceinline__ double pulse_rabi(const StepArgs &a, int idx, int t)
{
  const double *p = a.pos + 3 * idx;
  const PulseParams &P = a.pulse;
  const double kr = (P.k[0] * p[0] + P.k[1] * p[1]) + P.k[2] * p[2];
  const double time = t * a.dt;
  const double arg = kr - P.freq * (time - P.delay);
  const double x = arg / P.width;
  const double g = exp(-(x * x) / 2);
  const double *d = a.dip + 3 * idx;
  const double e0 = P.amp_pol[0] * g, e1 = P.amp_pol[1] * g, e2 = P.amp_pol[2] * g;
  return ((e0 * d[0] + e1 * d[1]) + e2 * d[2]) / a.hbar;
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

// Stores the step's final state: PC window, rho01 ring, trajectory row,
// and the non-finite flag.
__device__ __forceinline__ void finish_dot(const StepArgs &a, int idx, int t, const double2 (&r)[2],
                                           const double2 (&dr)[2])
{
  double2 *base = a.pcr + (long long)pc_slot(t) * 4 * a.n_pad + idx;
  base[0] = r[0];
  base[a.n_pad] = r[1];
  base[2 * a.n_pad] = dr[0];
  base[3 * a.n_pad] = dr[1];
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

// The step index is the far block's first step plus the launch's offset k;
// the last step of a block tells the next far-kernel launch where it starts.
__device__ __forceinline__ void publish_next_block(const StepArgs &a, int blk, int k, int t)
{
  if(k == kTimeBlock - 1 && blk == 0 && threadIdx.x == 0) *a.d_next = t + 1;
}

// The gathers of one step, split over the 4 warps of a block (32 dots):
// warp p takes predictor/corrector window slots h = p, p + 4, ... of its
// lane's dot; the block's mid-list entries (delay < K pairs of all 32 dots)
// are spread evenly over all 128 threads, each entry's contribution is
// staged in shared memory and warp 0 adds a dot's entries in list order, so
// a dot with many close partners does not hold up the block and the sums
// are deterministic.
constexpr int kParts = 4;
constexpr int kMidChunk = 512;  // mid-list entries staged per pass

template <int NT>
__device__ __forceinline__ void pc_part(const StepArgs &a, int idx, int t, int part, double2 (&out)[4])
{
  double2 P0 = make_double2(0.0, 0.0), P1 = P0, H0 = P0, H1 = P0;
  const int nt = NT > 0 ? NT : a.w.n_time;
  const double dt = a.dt;
#pragma unroll
  for(int h0 = 0; h0 < (NT > 0 ? NT : 32); h0 += kParts) {
    const int h = h0 + part;
    if(h < nt) {
      const int s = pc_slot(t - nt + h);
      const double2 *base = a.pcr + (long long)s * 4 * a.n_pad + idx;
      const double2 x0 = base[0], x1 = base[a.n_pad], y0 = base[2 * a.n_pad], y1 = base[3 * a.n_pad];
      const double p0 = a.w.ps[h], p1 = a.w.ps[nt + h];
      const double c0 = a.w.cs[h], c1 = a.w.cs[nt + h];
      P0.x += x0.x * p0 + (y0.x * p1) * dt;
      P0.y += x0.y * p0 + (y0.y * p1) * dt;
      P1.x += x1.x * p0 + (y1.x * p1) * dt;
      P1.y += x1.y * p0 + (y1.y * p1) * dt;
      H0.x += x0.x * c0 + (y0.x * c1) * dt;
      H0.y += x0.y * c0 + (y0.y * c1) * dt;
      H1.x += x1.x * c0 + (y1.x * c1) * dt;
      H1.y += x1.y * c0 + (y1.y * c1) * dt;
    }
  }
  out[0] = P0;
  out[1] = P1;
  out[2] = H0;
  out[3] = H1;
}

// One mid-list entry at step t: taps before step -22 skipped, the
// (delay 0, tap 0) term left to the near list.
__device__ __forceinline__ double2 mid_entry(const StepArgs &a, int e, int t)
{
  const int q = a.q;
  const int b = a.mid_idx[e];
  const int d = a.mid_delay[e];
  const double2 *c = a.mid_coef + (long long)e * (q + 1);
  const double2 *ring = a.ring + (long long)b * a.stride;
  const int s = t - d;
  const int base = ring_slot(s - q, a.W);  // tap i at base + q - i (mirrored)
  double2 M = make_double2(0.0, 0.0);
#pragma unroll
  for(int i = 0; i <= kMaxOrder; ++i) {
    if(i <= q && s - i >= -kWindow && !(d == 0 && i == 0)) {
      const double2 v = cmul(prefactor(ring[base + q - i], a.frame), c[i]);
      M.x += v.x;
      M.y += v.y;
    }
  }
  return M;
}

// Fused step for 32 dots per block, 128 threads: the gathers in parallel,
// then warp 0 runs predictor, 11 evaluations and 10 corrections; dots
// coupled at delay 0 share the block and exchange their iterates through
// shared memory after each correction.
template <int NT>
__device__ __forceinline__ void step_fused_body(const StepArgs &a, int blk, int k)
{
  constexpr int BS = 32;
  __shared__ double2 red[kParts][4][BS];
  __shared__ double2 midv[kMidChunk];
  __shared__ double2 cur[BS];
  const int lane = threadIdx.x & 31, part = threadIdx.x >> 5;
  const int idx = blk * BS + lane;
  const int t = *a.far_t0 + k;
  if(t >= a.T) return;  // past this ensemble's last step (uniform per block)
  const bool live = a.user[idx] >= 0;

  // warp 0's per-dot inputs, requested before the gathers complete
  double2 past = make_double2(0.0, 0.0);
  double det = 0, t1 = 1, t2 = 1, pul = 0;
  if(part == 0 && live) {
    past = a.far_field[(long long)k * a.n_pad + idx];
    pul = pulse_rabi(a, idx, t);
    det = a.laser_freq - a.freq[idx];
    t1 = a.t1[idx];
    t2 = a.t2[idx];
  }
  if(live) {
    double2 out[4];
    pc_part<NT>(a, idx, t, part, out);
#pragma unroll
    for(int v = 0; v < 4; ++v) red[part][v][lane] = out[v];
  }

  // mid list of the block's 32 dots: CSR range [E0, E1)
  const int E0 = a.mid_ptr[blk * BS], E1 = a.mid_ptr[blk * BS + BS];
  const int my0 = a.mid_ptr[idx], my1 = a.mid_ptr[idx + 1];
  double2 M = make_double2(0.0, 0.0);
  for(int c0 = E0; c0 < E1; c0 += kMidChunk) {
    const int c1 = min(E1, c0 + kMidChunk);
    for(int e = c0 + threadIdx.x; e < c1; e += 32 * kParts) midv[e - c0] = mid_entry(a, e, t);
    __syncthreads();
    if(part == 0)
      for(int e = max(my0, c0); e < min(my1, c1); ++e) {
        M.x += midv[e - c0].x;
        M.y += midv[e - c0].y;
      }
    __syncthreads();
  }
  if(E0 == E1) __syncthreads();  // the window partials are complete

  if(part == 0) {
    const int nb0 = a.near_ptr[blk * BS];
    const bool block_near = a.near_ptr[(blk + 1) * BS] > nb0;
    double2 P[2], H[2], r[2], dr[2];
    if(live) {
      double2 sum[4];
#pragma unroll
      for(int v = 0; v < 4; ++v) {
        sum[v] = red[0][v][lane];
#pragma unroll
        for(int p = 1; p < kParts; ++p) {
          sum[v].x += red[p][v][lane].x;
          sum[v].y += red[p][v][lane].y;
        }
      }
      P[0] = sum[0];
      P[1] = sum[1];
      H[0] = sum[2];
      H[1] = sum[3];
      past.x += M.x;
      past.y += M.y;
      r[0] = P[0];
      r[1] = P[1];
    }
    const int e0 = a.near_ptr[idx], e1 = a.near_ptr[idx + 1];
    for(int it = 0; it <= kCorrectorSteps; ++it) {
      if(it > 0 && live) corrector(a, dr, H, r);
      double2 nf = make_double2(0.0, 0.0);
      if(block_near) {
        __syncwarp();
        cur[lane] = live ? prefactor(r[1], a.frame) : make_double2(0.0, 0.0);
        __syncwarp();
        for(int e = e0; e < e1; ++e) {
          const double2 v = cmul(cur[a.near_idx[e]], a.near_coef[e]);
          nf.x += v.x;
          nf.y += v.y;
        }
      }
      if(live) {
        const double2 om = make_double2((0.0 + pul) + (past.x + nf.x), 0.0 + (past.y + nf.y));
        liouville(r[0], r[1], om, t1, t2, det, dr[0], dr[1]);
      }
    }
    if(live) finish_dot(a, idx, t, r, dr);
  }
  publish_next_block(a, blk, k, t);
}

template <int NT>
__global__ void __launch_bounds__(32 * kParts) step_fused_kernel(StepArgs a, int k)
{
  step_fused_body<NT>(a, blockIdx.x, k);
}

// Many ensembles, one launch: block_off[e] = first 32-dot block of ensemble e.
template <int NT>
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
  step_fused_body<NT>(args[lo], b - block_off[lo], k);
}

void launch_step_batch(const StepArgs *args, const int *block_off, int n_ens, int total_blocks, int n_time,
                       int k, void *stream)
{
  if(n_ens <= 0 || total_blocks <= 0) return;
  cudaStream_t s = (cudaStream_t)stream;
  if(n_time == 22)
    step_batch_kernel<22><<<total_blocks, 32 * kParts, 0, s>>>(args, block_off, n_ens, k);
  else
    step_batch_kernel<0><<<total_blocks, 32 * kParts, 0, s>>>(args, block_off, n_ens, k);
}

// ---- one launch for a whole 16-step block ------------------------------------
// The same step as step_fused_body, repeated for k = k0 .. k1-1 inside one
// cooperative launch (all blocks resident).  Each block keeps its 32 dots'
// predictor-corrector window (23 steps of rho and rho-dot) in shared memory,
// so a step reads only its mid-list partners' history (written by other
// blocks in the previous step, read through L2).  Steps are separated by a
// grid barrier: an arrival counter and a bounded wait; a wait that runs out
// sets *a.d_bad to -2 and the block returns.
constexpr int kBarrierSpins = 1 << 24;  // x ~64 ns: about a second

__device__ __forceinline__ bool grid_barrier(unsigned *ctr, unsigned target)
{
  __syncthreads();
  int ok = 1;
  if(threadIdx.x == 0) {
    __threadfence();
    atomicAdd(ctr, 1u);
    int spins = 0;
    while(*(volatile unsigned *)ctr < target) {
      if(++spins > kBarrierSpins) {
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
  }
  return __syncthreads_and(threadIdx.x == 0 ? ok : 1) != 0;
}

// mid_entry for the block kernel: partners' history read through L2, since
// other blocks of the same launch wrote it after this SM may have cached it.
__device__ __forceinline__ double2 mid_entry_cg(const StepArgs &a, int e, int t)
{
  const int q = a.q;
  const int b = a.mid_idx[e];
  const int d = a.mid_delay[e];
  const double2 *c = a.mid_coef + (long long)e * (q + 1);
  const double2 *ring = a.ring + (long long)b * a.stride;
  const int s = t - d;
  const int base = ring_slot(s - q, a.W);
  double2 M = make_double2(0.0, 0.0);
#pragma unroll
  for(int i = 0; i <= kMaxOrder; ++i) {
    if(i <= q && s - i >= -kWindow && !(d == 0 && i == 0)) {
      const double2 v = cmul(prefactor(__ldcg(ring + base + q - i), a.frame), c[i]);
      M.x += v.x;
      M.y += v.y;
    }
  }
  return M;
}

template <int NT>
__global__ void __launch_bounds__(32 * kParts) step_block_kernel(StepArgs a, int k0, int k1, unsigned *bar)
{
  constexpr int BS = 32;
  // 62.5 KB of dynamic shared memory (above the 48 KB static limit)
  extern __shared__ double2 smem_block[];
  auto win = reinterpret_cast<double2(*)[4][BS]>(smem_block);  // rho00, rho01, drho00, drho01 by step slot
  auto red = reinterpret_cast<double2(*)[4][BS]>(smem_block + kPcDepth * 4 * BS);
  double2 *midv = smem_block + (kPcDepth + kParts) * 4 * BS;
  double2 *cur = midv + kMidChunk;
  const int lane = threadIdx.x & 31, part = threadIdx.x >> 5;
  const int blk = blockIdx.x;
  const int idx = blk * BS + lane;
  const int t0 = *a.far_t0;
  const bool live = a.user[idx] >= 0;
  const int nt = NT > 0 ? NT : a.w.n_time;

  // the integrator's window: all 23 slots of the predictor-corrector ring
  for(int sl = part; sl < kPcDepth; sl += kParts)
    for(int c = 0; c < 4; ++c) win[sl][c][lane] = a.pcr[((long long)sl * 4 + c) * a.n_pad + idx];
  double det = 0, t1 = 1, t2 = 1;
  if(live) {
    det = a.laser_freq - a.freq[idx];
    t1 = a.t1[idx];
    t2 = a.t2[idx];
  }
  const int E0 = a.mid_ptr[blk * BS], E1 = a.mid_ptr[blk * BS + BS];
  const int my0 = a.mid_ptr[idx], my1 = a.mid_ptr[idx + 1];
  const int nb0 = a.near_ptr[blk * BS];
  const bool block_near = a.near_ptr[(blk + 1) * BS] > nb0;
  const int ne0 = a.near_ptr[idx], ne1 = a.near_ptr[idx + 1];
  __syncthreads();

  for(int k = k0; k < k1; ++k) {
    const int t = t0 + k;
    if(t >= a.T) break;  // uniform: every block stops at the same k
    if(live) {
      double2 P0 = make_double2(0.0, 0.0), P1 = P0, H0 = P0, H1 = P0;
      const double dt = a.dt;
#pragma unroll
      for(int h0 = 0; h0 < (NT > 0 ? NT : 32); h0 += kParts) {
        const int h = h0 + part;
        if(h < nt) {
          const int sl = pc_slot(t - nt + h);
          const double2 x0 = win[sl][0][lane], x1 = win[sl][1][lane], y0 = win[sl][2][lane], y1 = win[sl][3][lane];
          const double p0 = a.w.ps[h], p1 = a.w.ps[nt + h];
          const double c0 = a.w.cs[h], c1 = a.w.cs[nt + h];
          P0.x += x0.x * p0 + (y0.x * p1) * dt;
          P0.y += x0.y * p0 + (y0.y * p1) * dt;
          P1.x += x1.x * p0 + (y1.x * p1) * dt;
          P1.y += x1.y * p0 + (y1.y * p1) * dt;
          H0.x += x0.x * c0 + (y0.x * c1) * dt;
          H0.y += x0.y * c0 + (y0.y * c1) * dt;
          H1.x += x1.x * c0 + (y1.x * c1) * dt;
          H1.y += x1.y * c0 + (y1.y * c1) * dt;
        }
      }
      red[part][0][lane] = P0;
      red[part][1][lane] = P1;
      red[part][2][lane] = H0;
      red[part][3][lane] = H1;
    }
    double2 M = make_double2(0.0, 0.0);
    for(int c0 = E0; c0 < E1; c0 += kMidChunk) {
      const int c1 = min(E1, c0 + kMidChunk);
      for(int e = c0 + threadIdx.x; e < c1; e += 32 * kParts) midv[e - c0] = mid_entry_cg(a, e, t);
      __syncthreads();
      if(part == 0)
        for(int e = max(my0, c0); e < min(my1, c1); ++e) {
          M.x += midv[e - c0].x;
          M.y += midv[e - c0].y;
        }
      __syncthreads();
    }
    if(E0 == E1) __syncthreads();

    if(part == 0) {
      double2 P[2], H[2], r[2], dr[2], past = make_double2(0.0, 0.0);
      double pul = 0;
      if(live) {
        double2 sum[4];
#pragma unroll
        for(int v = 0; v < 4; ++v) {
          sum[v] = red[0][v][lane];
#pragma unroll
          for(int p = 1; p < kParts; ++p) {
            sum[v].x += red[p][v][lane].x;
            sum[v].y += red[p][v][lane].y;
          }
        }
        P[0] = sum[0];
        P[1] = sum[1];
        H[0] = sum[2];
        H[1] = sum[3];
        past = a.far_field[(long long)k * a.n_pad + idx];
        past.x += M.x;
        past.y += M.y;
        pul = pulse_rabi(a, idx, t);
        r[0] = P[0];
        r[1] = P[1];
      }
      for(int it = 0; it <= kCorrectorSteps; ++it) {
        if(it > 0 && live) corrector(a, dr, H, r);
        double2 nf = make_double2(0.0, 0.0);
        if(block_near) {
          __syncwarp();
          cur[lane] = live ? prefactor(r[1], a.frame) : make_double2(0.0, 0.0);
          __syncwarp();
          for(int e = ne0; e < ne1; ++e) {
            const double2 v = cmul(cur[a.near_idx[e]], a.near_coef[e]);
            nf.x += v.x;
            nf.y += v.y;
          }
        }
        if(live) {
          const double2 om = make_double2((0.0 + pul) + (past.x + nf.x), 0.0 + (past.y + nf.y));
          liouville(r[0], r[1], om, t1, t2, det, dr[0], dr[1]);
        }
      }
      if(live) {
        finish_dot(a, idx, t, r, dr);
        const int sl = pc_slot(t);
        win[sl][0][lane] = r[0];
        win[sl][1][lane] = r[1];
        win[sl][2][lane] = dr[0];
        win[sl][3][lane] = dr[1];
      }
    }
    if(k == kTimeBlock - 1 && blk == 0 && threadIdx.x == 0) *a.d_next = t + 1;
    if(k + 1 < k1 && !grid_barrier(bar, (unsigned)(k - k0 + 1) * gridDim.x)) {
      if(threadIdx.x == 0) atomicMin(a.d_bad, -2);
      return;
    }
  }
}

constexpr size_t kStepBlockSmem = sizeof(double2) * ((kPcDepth + kParts) * 4 * 32 + kMidChunk + 32);

static void step_block_attrs()
{
  static int dev_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if(dev < 64 && !dev_done[dev]) {
    cudaFuncSetAttribute(step_block_kernel<22>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStepBlockSmem);
    cudaFuncSetAttribute(step_block_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStepBlockSmem);
    dev_done[dev] = 1;
  }
}

void launch_step_block(const StepArgs &a, int k0, int k1, int nblocks, unsigned *bar, void *stream)
{
  cudaStream_t s = (cudaStream_t)stream;
  step_block_attrs();
  cudaMemsetAsync(bar, 0, sizeof(unsigned), s);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblocks);
  cfg.blockDim = dim3(32 * kParts);
  cfg.dynamicSmemBytes = kStepBlockSmem;
  cfg.stream = s;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeCooperative;
  attr.val.cooperative = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  if(a.w.n_time == 22)
    cudaLaunchKernelEx(&cfg, step_block_kernel<22>, a, k0, k1, bar);
  else
    cudaLaunchKernelEx(&cfg, step_block_kernel<0>, a, k0, k1, bar);
}

int step_block_max_blocks()
{
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  step_block_attrs();
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step_block_kernel<22>, 32 * kParts, kStepBlockSmem);
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
    liouville(r[0], r[1], om, a.t1[idx], a.t2[idx], a.laser_freq - a.freq[idx], dr[0], dr[1]);
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
