// Far-pair kernel: K = kTimeBlock steps of the retarded pair sum from one
// pass over the FP64 coefficient table.
//
// HistoryInteraction::evaluate (reference history_interaction.cpp:47-70)
// sums, for every unordered pair (a, b) and tap i = 0..q,
//     field[a] += prefactor(rho01_b[s-i]) * coef_i,
//     field[b] += prefactor(rho01_a[s-i]) * coef_i,   s = step - delay_ab,
// skipping taps with s - i < -22, and the integrator calls it 11 times per
// step (integrator.cpp:133-139).  For a pair with floor delay d >= K every
// tap of every step in [t0, t0 + K) reads a step before t0, so its K x (q+1)
// terms are fixed once step t0 - 1 is done: one pass over the table at t0
// gives the far-pair part of the field for the next K steps.  Pairs with
// d < K (a few per thousand at the benchmark sizes) are summed per step by
// the dot-step kernel from a compact list.
//
// Per pair and direction the K steps read one window of K + q consecutive
// history samples, held in registers, and form a K-output, (q+1)-tap
// convolution with the pair's coefficients: 2 K (q+1) complex
// multiply-adds per pair per pass, each coefficient read from HBM once per K
// steps.
//
// Schedule.  One warp owns one 32 x 32 tile block (I, J) and walks it in 32
// diagonal steps: at step j lane l takes the pair (a = 32 I + l,
// b = 32 J + (l + j) mod 32).  The row sums (field of a) stay in lane l's
// registers; the column sums (field of b) move one lane down after every
// step, so after 32 steps lane l holds the complete column l.  No reduction
// trees, no atomics: each (dot, partner tile, step) partial is written once,
// and the dot-step kernel adds the partials in a fixed order, so results are
// deterministic.
//
// The rho01 ring holds rho01 by time slot (slot = t mod W) with the first
// kRingMirror slots repeated after slot W-1, so every window is contiguous.
// Polarisation prefactor: rho01 in the rotating frame
// (rotating_green_function.h:17-21), 2 Re rho01 in the lab frame
// (green_function.h:23-27).
#include <cuda_runtime.h>

#include "qg_internal.h"

namespace qg {

__device__ __forceinline__ void decode_block_f(long long blk, int &I, int &J)
{
  long long r = (long long)((sqrt(8.0 * (double)blk + 1.0) - 1.0) * 0.5);
  while(r * (r + 1) / 2 > blk) --r;
  while((r + 1) * (r + 2) / 2 <= blk) ++r;
  I = (int)r;
  J = (int)(blk - r * (r + 1) / 2);
}

__device__ __forceinline__ void cfma(double2 &acc, double2 c, double2 r)
{
  acc.x = fma(c.x, r.x, acc.x);
  acc.x = fma(-c.y, r.y, acc.x);
  acc.y = fma(c.x, r.y, acc.y);
  acc.y = fma(c.y, r.x, acc.y);
}

template <bool LAB>
__device__ __forceinline__ double2 ring_pref(const double2 *p)
{
  const double2 r = __ldg(p);
  return LAB ? make_double2(2 * r.x, 0.0) : r;
}

template <int Q, bool LAB>
__device__ __forceinline__ void window_conv(const double2 *ring, int slot0, int tau0, bool full,
                                            const double2 (&c)[Q + 1], double2 (&acc)[kTimeBlock])
{
  constexpr int K = kTimeBlock;
  double2 w[K + Q];
#pragma unroll
  for(int m = 0; m < K + Q; ++m) w[m] = ring_pref<LAB>(ring + slot0 + m);
  if(full) {
#pragma unroll
    for(int k = 0; k < K; ++k)
#pragma unroll
      for(int i = 0; i <= Q; ++i) cfma(acc[k], c[i], w[k + Q - i]);
  } else {
    // early steps: taps before step -22 are skipped, as the reference does
#pragma unroll
    for(int k = 0; k < K; ++k)
#pragma unroll
      for(int i = 0; i <= Q; ++i)
        if(tau0 + k + Q - i >= -kWindow) cfma(acc[k], c[i], w[k + Q - i]);
  }
}

template <int Q, bool LAB>
__global__ void __launch_bounds__(128) far_kernel(FarArgs a)
{
  constexpr int K = kTimeBlock;
  const int lane = threadIdx.x & 31;
  const long long blk = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
  if(blk >= a.nblk) return;  // uniform per warp
  int I, J;
  decode_block_f(blk, I, J);
  const int t0 = *a.d_t0;
  if(blk == 0 && lane == 0) *a.far_t0_out = t0;
  const int W = a.W;
  const int ia = I * kTile + lane;
  const double2 *ring_a = a.ring + (long long)ia * a.stride;
  const int *bd = a.delay + blk * kTilePairs;
  const double2 *bc = a.coef + blk * (long long)(Q + 1) * kTilePairs;

  double2 racc[K], cacc[K];
#pragma unroll
  for(int k = 0; k < K; ++k) racc[k] = cacc[k] = make_double2(0.0, 0.0);

  int dn = __ldg(bd + lane);
  double2 cn[Q + 1];
#pragma unroll
  for(int i = 0; i <= Q; ++i) cn[i] = __ldg(bc + i * kTilePairs + lane);

  for(int j = 0; j < kTile; ++j) {
    const int d = dn;
    double2 c[Q + 1];
#pragma unroll
    for(int i = 0; i <= Q; ++i) c[i] = cn[i];
    if(j + 1 < kTile) {
      const int e = (j + 1) * kTile + lane;
      dn = __ldg(bd + e);
#pragma unroll
      for(int i = 0; i <= Q; ++i) cn[i] = __ldg(bc + i * kTilePairs + e);
    }
    if(d >= K) {
      const int ib = J * kTile + ((lane + j) & (kTile - 1));
      const int tau0 = t0 - d - Q;
      int slot0 = tau0 % W;
      if(slot0 < 0) slot0 += W;
      const bool full = tau0 >= -kWindow;
      window_conv<Q, LAB>(a.ring + (long long)ib * a.stride, slot0, tau0, full, c, racc);
      window_conv<Q, LAB>(ring_a, slot0, tau0, full, c, cacc);
    }
    const int src = (lane + 1) & (kTile - 1);
#pragma unroll
    for(int k = 0; k < K; ++k) {
      cacc[k].x = __shfl_sync(0xffffffffu, cacc[k].x, src);
      cacc[k].y = __shfl_sync(0xffffffffu, cacc[k].y, src);
    }
  }

  const long long slice = (long long)a.nT * a.n_pad;
#pragma unroll
  for(int k = 0; k < K; ++k) {
    double2 *P = a.partial + k * slice;
    if(I == J) {
      P[(long long)I * a.n_pad + ia] = make_double2(racc[k].x + cacc[k].x, racc[k].y + cacc[k].y);
    } else {
      P[(long long)J * a.n_pad + ia] = racc[k];
      P[(long long)I * a.n_pad + J * kTile + lane] = cacc[k];
    }
  }
}

template <bool LAB>
static void launch_far_frame(const FarArgs &a, cudaStream_t s)
{
  const unsigned blocks = (unsigned)((a.nblk + 3) / 4);
  switch(a.q) {
    case 1: far_kernel<1, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 2: far_kernel<2, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 3: far_kernel<3, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 4: far_kernel<4, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 5: far_kernel<5, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 6: far_kernel<6, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 7: far_kernel<7, LAB><<<blocks, 128, 0, s>>>(a); break;
    default: break;
  }
}

void launch_far(const FarArgs &a, void *stream)
{
  if(a.nblk <= 0) return;
  if(a.frame == 0)
    launch_far_frame<false>(a, (cudaStream_t)stream);
  else
    launch_far_frame<true>(a, (cudaStream_t)stream);
}

}  // namespace qg
