// Strictly-past pair sum over the FP64 coefficient table, once per step.
//
// HistoryInteraction::evaluate (reference history_interaction.cpp:47-70)
// sums, for every unordered pair (a, b) and tap i = 0..q,
//     field[a] += prefactor(rho01_b[s-i]) * coef_i,
//     field[b] += prefactor(rho01_a[s-i]) * coef_i,   s = step - delay_ab,
// skipping taps with s - i < -22.  The integrator calls it 11 times per step
// (integrator.cpp:133-139), but every tap except (delay 0, tap 0) reads a
// strictly earlier step, so those terms are identical in all 11 calls.  This
// kernel computes them once per step; the (delay 0, tap 0) terms are added
// per iteration by the dot-step kernel from its near list.
//
// One CTA (256 threads, 8 warps) processes one 64 x 64 tile block (I, J) of
// the table, reading each unordered pair's coefficients once and applying
// them in both directions.  Warp w owns rows la = w, w+8, ..., lane l owns
// columns lb = l and l+32.  Row sums are reduced across the warp with
// shuffles, column sums across the 8 warps through shared memory.  Partial
// sums go to partial[other tile][dot], one slot per (dot, partner tile),
// each written exactly once, so the final reduction in the dot-step kernel
// has a fixed order and results are deterministic.
//
// The rho01 ring holds rho01 by time slot; slots 0..kRingMirror-1 are
// mirrored after slot W-1, so the q+1 taps of a window are contiguous.  The
// polarisation prefactor is rho01 itself in the rotating frame
// (rotating_green_function.h:17-21) and 2 Re rho01 in the lab frame
// (green_function.h:23-27).
#include <cuda_runtime.h>

#include "qg_internal.h"

namespace qg {

__device__ __forceinline__ void decode_block_s(long long blk, int &I, int &J)
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

__device__ __forceinline__ double2 warp_sum(double2 v)
{
#pragma unroll
  for(int off = 16; off > 0; off >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
  }
  return v;
}

template <int Q, bool LAB>
__global__ void __launch_bounds__(256, 2) sweep_table_kernel(SweepArgs a)
{
  __shared__ double2 srow[kTile];
  __shared__ double2 scol[8][kTile];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t = *a.d_step;
  int I, J;
  decode_block_s(blockIdx.x, I, J);
  const bool diag = (I == J);
  const int *bd = a.delay + (long long)blockIdx.x * kTilePairs;
  const double2 *bc = a.coef + (long long)blockIdx.x * (Q + 1) * kTilePairs;
  const int W = a.W;

  double2 col0 = make_double2(0.0, 0.0), col1 = make_double2(0.0, 0.0);
  for(int k = 0; k < kTile / 8; ++k) {
    const int la = warp + 8 * k;
    const int ia = I * kTile + la;
    const double2 *ra = a.ring + (long long)ia * a.stride;
    double2 row = make_double2(0.0, 0.0);
#pragma unroll
    for(int h = 0; h < 2; ++h) {
      const int lb = h * 32 + lane;
      const int e = la * kTile + lb;
      const int d = __ldg(bd + e);
      if(d >= 0) {
        const int ib = J * kTile + lb;
        const double2 *rb = a.ring + (long long)ib * a.stride;
        const int s = t - d;
        // taps i in [ilo, ihi] are read: s - i >= -22, and (d, i) != (0, 0)
        const int ilo = (d == 0) ? 1 : 0;
        const int ihi = min(Q, s + kWindow);
        int base = (s - Q) % W;
        if(base < 0) base += W;
        double2 acc_r = make_double2(0.0, 0.0), acc_c = make_double2(0.0, 0.0);
#pragma unroll
        for(int i = 0; i <= Q; ++i) {
          if(i >= ilo && i <= ihi) {
            const double2 c = __ldg(bc + (long long)i * kTilePairs + e);
            const int slot = base + (Q - i);
            cfma(acc_r, c, ring_pref<LAB>(rb + slot));
            cfma(acc_c, c, ring_pref<LAB>(ra + slot));
          }
        }
        row.x += acc_r.x;
        row.y += acc_r.y;
        if(h == 0) {
          col0.x += acc_c.x;
          col0.y += acc_c.y;
        } else {
          col1.x += acc_c.x;
          col1.y += acc_c.y;
        }
      }
    }
    row = warp_sum(row);
    if(lane == 0) srow[la] = row;
  }
  scol[warp][lane] = col0;
  scol[warp][lane + 32] = col1;
  __syncthreads();
  if(tid < kTile) {
    double2 cs = make_double2(0.0, 0.0);
#pragma unroll
    for(int w = 0; w < 8; ++w) {
      cs.x += scol[w][tid].x;
      cs.y += scol[w][tid].y;
    }
    if(diag) {
      double2 v = srow[tid];
      v.x += cs.x;
      v.y += cs.y;
      a.partial[(long long)I * a.n_pad + I * kTile + tid] = v;
    } else {
      a.partial[(long long)J * a.n_pad + I * kTile + tid] = srow[tid];
      a.partial[(long long)I * a.n_pad + J * kTile + tid] = cs;
    }
  }
}

template <bool LAB>
static void launch_sweep_frame(const SweepArgs &a, cudaStream_t s)
{
  const unsigned blocks = (unsigned)a.nblk;
  switch(a.q) {
    case 1: sweep_table_kernel<1, LAB><<<blocks, 256, 0, s>>>(a); break;
    case 2: sweep_table_kernel<2, LAB><<<blocks, 256, 0, s>>>(a); break;
    case 3: sweep_table_kernel<3, LAB><<<blocks, 256, 0, s>>>(a); break;
    case 4: sweep_table_kernel<4, LAB><<<blocks, 256, 0, s>>>(a); break;
    case 5: sweep_table_kernel<5, LAB><<<blocks, 256, 0, s>>>(a); break;
    case 6: sweep_table_kernel<6, LAB><<<blocks, 256, 0, s>>>(a); break;
    case 7: sweep_table_kernel<7, LAB><<<blocks, 256, 0, s>>>(a); break;
    default: break;
  }
}

void launch_sweep_table(const SweepArgs &a, void *stream)
{
  if(a.frame == 0)
    launch_sweep_frame<false>(a, (cudaStream_t)stream);
  else
    launch_sweep_frame<true>(a, (cudaStream_t)stream);
}

}  // namespace qg
