// Convolution and reduction pieces shared by the far-pair kernels (table
// and on-the-fly coefficients).  Every product is an explicit fused
// multiply-add and every other operation a plain add, so the results do not
// depend on the translation unit's contraction setting.
#pragma once

#include <cuda_runtime.h>

#include "qg_internal.h"

namespace qg {

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

// acc[k] += sum_i c[i] * w[k + Q - i] over the window w[m] = ring[slot0 + m],
// m = 0 .. K+Q-1, whose first sample is step tau0.  Samples before step -22
// are skipped (their taps are skipped by the reference).
template <int Q, bool LAB, int K>
__device__ __forceinline__ void window_conv(const double2 *ring, int slot0, int tau0,
                                            const double2 (&c)[Q + 1], double2 (&acc)[K])
{
  if(tau0 >= -kWindow) {
#pragma unroll
    for(int m = 0; m < K + Q; ++m) {
      const double2 w = ring_pref<LAB>(ring + slot0 + m);
#pragma unroll
      for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) cfma(acc[k], c[k + Q - m], w);
    }
  } else {
#pragma unroll
    for(int m = 0; m < K + Q; ++m) {
      if(tau0 + m < -kWindow) continue;
      const double2 w = ring_pref<LAB>(ring + slot0 + m);
#pragma unroll
      for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) cfma(acc[k], c[k + Q - m], w);
    }
  }
}

// window_conv's result for the first blocks of a run, where some lanes'
// windows start before step -22 and others do not: rather than split such a
// warp between window_conv's two loops, every lane runs one loop in which a
// sample before step -22 is replaced by zero.  Its products are +-0 (the
// coefficients are finite: a table with a non-finite far coefficient, from
// an integer delay, never takes this form, so such a NaN still appears at
// the step where the reference's does), and adding +-0 leaves an
// accumulator that started at +0 bit for bit as it was (a sum is -0 only
// when both addends are), so each lane gets the skipping loop's result.
template <int Q, bool LAB, int K>
__device__ __forceinline__ void window_conv_uniform(const double2 *ring, int slot0, int tau0,
                                                    const double2 (&c)[Q + 1], double2 (&acc)[K])
{
  // A warp whose windows are all live, or all partly dead, takes
  // window_conv, which then runs one loop for all its lanes (the second
  // skips the dead samples' work); only a warp with both kinds runs the
  // zeroing loop.  The votes only pick a loop: every loop gives the same
  // bits for its lane.
  const unsigned act = __activemask();
  const bool live = tau0 >= -kWindow;
  if(__all_sync(act, live) || __all_sync(act, !live)) {
    window_conv<Q, LAB, K>(ring, slot0, tau0, c, acc);
    return;
  }
#pragma unroll
  for(int m = 0; m < K + Q; ++m) {
    double2 w = ring_pref<LAB>(ring + slot0 + m);
    if(tau0 + m < -kWindow) w = make_double2(0.0, 0.0);
#pragma unroll
    for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) cfma(acc[k], c[k + Q - m], w);
  }
}

// Two samples per 32-byte load (ld.global.nc.v4.f64).  Ring rows start on
// 32-byte boundaries (even row stride, 16-byte samples), so a load must start
// at an even slot.
template <bool LAB>
__device__ __forceinline__ void ld_pair(const double2 *p, double2 &x, double2 &y)
{
  double a0, a1, a2, a3;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a0), "=d"(a1), "=d"(a2), "=d"(a3) : "l"(p));
  x = LAB ? make_double2(2 * a0, 0.0) : make_double2(a0, a1);
  y = LAB ? make_double2(2 * a2, 0.0) : make_double2(a2, a3);
}

__device__ __forceinline__ double2 sel2(bool odd, double2 a, double2 b) { return odd ? a : b; }

// window_conv's result from 32-byte loads, for windows whose samples are all
// live (tau0 >= -22).  The 32 lanes of a warp read windows at different
// delays, so their first slots have different parities; a branch on the
// parity would run the convolution twice.  Every lane instead loads
// (K+Q+1)/2 rounded up pairs from the even slot at or below its first one,
// L[0 ..], and takes sample m as L[m + par] by a select: the same products
// in the same order as window_conv, hence the same result bit for bit, with
// half the load instructions (each warp load touches about as many cache
// lines as a 16-byte one, so the L1 wavefronts halve too).  The last sample
// read is at slot0 + K + Q, inside the row's kRingMirror mirrored slots.
template <int Q, bool LAB, int K>
__device__ __forceinline__ void window_conv_pairs(const double2 *ring, int slot0, const double2 (&c)[Q + 1],
                                                  double2 (&acc)[K])
{
  constexpr int M = K + Q;             // window samples
  constexpr int NV = (M + 1 + 1) / 2;  // pairs loaded: L[0 .. M] (and one more when M is odd)
  const bool odd = slot0 & 1;
  const double2 *p = ring + (slot0 - (odd ? 1 : 0));
  double2 prev = make_double2(0.0, 0.0);
#pragma unroll
  for(int v = 0; v < NV; ++v) {
    double2 x, y;  // L[2v], L[2v+1]
    ld_pair<LAB>(p + 2 * v, x, y);
    // sample m = 2v-1 is L[2v] (odd) or L[2v-1] (even); sample 2v is L[2v+1] or L[2v]
#pragma unroll
    for(int e = 0; e < 2; ++e) {
      const int m = 2 * v - 1 + e;
      if(m < 0 || m >= M) continue;
      const double2 w = e == 0 ? sel2(odd, x, prev) : sel2(odd, y, x);
#pragma unroll
      for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) cfma(acc[k], c[k + Q - m], w);
    }
    prev = y;
  }
}

__device__ __forceinline__ void cfmaf(float2 &acc, float2 c, float2 r)
{
  acc.x = fmaf(c.x, r.x, acc.x);
  acc.x = fmaf(-c.y, r.y, acc.x);
  acc.y = fmaf(c.x, r.y, acc.y);
  acc.y = fmaf(c.y, r.x, acc.y);
}

template <bool LAB>
__device__ __forceinline__ float2 pref32(float2 r)
{
  return LAB ? make_float2(2.f * r.x, 0.f) : r;
}

// Packed FP32 pairs (Blackwell fma.rn.f32x2 / add.rn.f32x2): one instruction
// does two independent FP32 operations, each rounded as the scalar one is.
__device__ __forceinline__ unsigned long long pk2(float2 v)
{
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
  return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long r)
{
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b, unsigned long long c)
{
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ unsigned long long fadd2(unsigned long long a, unsigned long long b)
{
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
// Accumulators of the mixed-precision convolution (difference form, see
// qg_far.cu).  A complex multiply-add acc += c u is kept as two real pairs,
// a += (c.x, c.x) (u.x, u.y) and b += (c.y, c.y) (u.x, u.y), so a packed
// FP32 pair instruction (fma.rn.f32x2) does each without first swapping u's
// halves; the product's real part is a.x - b.y and its imaginary part
// a.y + b.x, formed in FP64 when the partial is written.  `base` collects the
// tap-sum term (sum_i c_i) w_0, which is the same for all K outputs of a
// pair, once per pair.  The packed form (PACKED) and the scalar form do the
// same operations on the same values in the same order: the same bits.
template <int K, bool PACKED>
struct MixedAcc;

template <int K>
struct MixedAcc<K, false> {
  float2 a[K], b[K];
  float2 base;
  __device__ __forceinline__ void zero()
  {
#pragma unroll
    for(int k = 0; k < K; ++k) a[k] = b[k] = make_float2(0.f, 0.f);
    base = make_float2(0.f, 0.f);
  }
  // a[k] += (cx, cx) u, b[k] += (cy, cy) u
  __device__ __forceinline__ void mac(int k, float2 c, float2 u)
  {
    a[k].x = fmaf(c.x, u.x, a[k].x);
    a[k].y = fmaf(c.x, u.y, a[k].y);
    b[k].x = fmaf(c.y, u.x, b[k].x);
    b[k].y = fmaf(c.y, u.y, b[k].y);
  }
  __device__ __forceinline__ float2 av(int k) const { return a[k]; }
  __device__ __forceinline__ float2 bv(int k) const { return b[k]; }
};

template <int K>
struct MixedAcc<K, true> {
  unsigned long long a[K], b[K];
  float2 base;
  __device__ __forceinline__ void zero()
  {
#pragma unroll
    for(int k = 0; k < K; ++k) a[k] = b[k] = pk2(make_float2(0.f, 0.f));
    base = make_float2(0.f, 0.f);
  }
  __device__ __forceinline__ float2 av(int k) const { return upk2(a[k]); }
  __device__ __forceinline__ float2 bv(int k) const { return upk2(b[k]); }
};

// The convolution's output k of one warp's sum, in FP64.
template <int K, bool PACKED>
__device__ __forceinline__ double2 mixed_out(const MixedAcc<K, PACKED> &m, int k)
{
  const float2 a = m.av(k), b = m.bv(k);
  return make_double2(((double)a.x - (double)b.y) + (double)m.base.x,
                      ((double)a.y + (double)b.x) + (double)m.base.y);
}

// acc[k] += sum_i c_i w_{k+Q-i} over the window w_m, m = 0 .. K+Q-1, whose
// first sample w_0 (step tau0) is rw[slot0] and whose later samples are
// w_0 + u_m, u_m the running sum of the FP32 step-to-step differences
// rd[slot0 + 1 .. slot0 + m].  c[Q+1] is the pair's tap sum.  When every
// sample is live (tau0 >= -22) this is (sum_i c_i) w_0 + sum_i c_i u_{k+Q-i}:
// the first term goes to `base` once and the differences meet only the taps.
// Samples before step -22 are skipped (their taps are skipped by the
// reference); there the absolute samples w_0 + u_m meet the live taps.
template <int Q, bool LAB, int K, bool PACKED>
__device__ __forceinline__ void window_conv_mixed(const float2 *rw, const float2 *rd, int slot0, int tau0,
                                                  const float2 (&c)[Q + 2], MixedAcc<K, PACKED> &acc)
{
  const float2 w0 = pref32<LAB>(__ldg(rw + slot0));
  if(tau0 >= -kWindow) {
    cfmaf(acc.base, c[Q + 1], w0);
    if constexpr(PACKED) {
      unsigned long long cx[Q + 1], cy[Q + 1];
#pragma unroll
      for(int i = 0; i <= Q; ++i) {
        cx[i] = pk2(make_float2(c[i].x, c[i].x));
        cy[i] = pk2(make_float2(c[i].y, c[i].y));
      }
      unsigned long long u = pk2(make_float2(0.f, 0.f));
#pragma unroll
      for(int m = 1; m < K + Q; ++m) {
        u = fadd2(u, pk2(pref32<LAB>(__ldg(rd + slot0 + m))));
#pragma unroll
        for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) {
          acc.a[k] = ffma2(cx[k + Q - m], u, acc.a[k]);
          acc.b[k] = ffma2(cy[k + Q - m], u, acc.b[k]);
        }
      }
    } else {
      float2 u = make_float2(0.f, 0.f);
#pragma unroll
      for(int m = 1; m < K + Q; ++m) {
        const float2 d = pref32<LAB>(__ldg(rd + slot0 + m));
        u.x += d.x;
        u.y += d.y;
#pragma unroll
        for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) acc.mac(k, c[k + Q - m], u);
      }
    }
  } else {
    // early steps: absolute samples, taps before step -22 skipped
    float2 u = make_float2(0.f, 0.f);
#pragma unroll
    for(int m = 0; m < K + Q; ++m) {
      if(m > 0) {
        const float2 d = pref32<LAB>(__ldg(rd + slot0 + m));
        u.x += d.x;
        u.y += d.y;
      }
      if(tau0 + m < -kWindow) continue;
      const float2 w = make_float2(w0.x + u.x, w0.y + u.y);
#pragma unroll
      for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) {
        if constexpr(PACKED) {
          acc.a[k] = ffma2(pk2(make_float2(c[k + Q - m].x, c[k + Q - m].x)), pk2(w), acc.a[k]);
          acc.b[k] = ffma2(pk2(make_float2(c[k + Q - m].y, c[k + Q - m].y)), pk2(w), acc.b[k]);
        } else {
          acc.mac(k, c[k + Q - m], w);
        }
      }
    }
  }
}

// Writes a warp's K accumulators as the partial of source group g for target
// tile I; the last warp of the tile (completion counter) adds the nG partials
// in group order, so the result does not depend on scheduling.
template <int K>
__device__ __forceinline__ void group_partials_reduce(const FarArgs &a, int I, int g, const double2 (&acc)[K])
{
  const int lane = threadIdx.x & 31;
  const int ia = I * kTile + lane;
  const long long gslice = (long long)a.nG * a.n_pad;
#pragma unroll
  for(int k = 0; k < K; ++k) a.partial[k * gslice + (long long)g * a.n_pad + ia] = acc[k];
  __threadfence();
  unsigned prev = 0;
  if(lane == 0) prev = atomicAdd(a.tile_done + I, 1u);
  prev = __shfl_sync(0xffffffffu, prev, 0);
  if(prev == (unsigned)(a.nG - 1)) {
    __threadfence();
#pragma unroll 1
    for(int k = 0; k < K; ++k) {
      double2 f = make_double2(0.0, 0.0);
      const double2 *P = a.partial + k * gslice + ia;
      for(int gg = 0; gg < a.nG; ++gg) {
        const double2 v = __ldcg(P + (long long)gg * a.n_pad);
        f.x += v.x;
        f.y += v.y;
      }
      a.field[(long long)k * a.n_pad + ia] = f;
    }
    if(lane == 0) a.tile_done[I] = 0;
  }
}

}  // namespace qg
