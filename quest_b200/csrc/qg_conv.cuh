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
// does the two lanes of a complex component pair.  A complex multiply-add
// acc += c r is two packed FMAs, (acc.x, acc.y) += (c.x, c.x) (r.x, r.y), then
// += (-c.y, c.y) (r.y, r.x): per component exactly cfmaf's two fmaf in the
// same order, so the results are bit-identical to the scalar form.
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
// acc += c r with c given as its packed pair (cxx = (c.x, c.x), cyy = (-c.y, c.y))
__device__ __forceinline__ void cfma2(unsigned long long &acc, unsigned long long cxx, unsigned long long cyy,
                                      unsigned long long r, unsigned long long rsw)
{
  acc = ffma2(cxx, r, acc);
  acc = ffma2(cyy, rsw, acc);
}

// The mixed-precision window convolution (difference form, see qg_far.cu):
// acc[k] += sum_i c_i w_{k+Q-i}, w_m = w_0 + sum_{j<=m} d_j.  PACKED selects
// the packed-pair form (bit-identical; faster where registers allow).
template <int Q, bool LAB, int K>
__device__ __forceinline__ void window_conv_mixed_packed(const float2 *rw, const float2 *rd, int slot0, int tau0,
                                                         const float2 (&c)[Q + 2], float2 (&accf)[K]);

template <int Q, bool LAB, int K, bool PACKED = false>
__device__ __forceinline__ void window_conv_mixed(const float2 *rw, const float2 *rd, int slot0, int tau0,
                                                  const float2 (&c)[Q + 2], float2 (&acc)[K])
{
  if(PACKED) {
    window_conv_mixed_packed<Q, LAB, K>(rw, rd, slot0, tau0, c, acc);
    return;
  }
  const float2 w0 = pref32<LAB>(__ldg(rw + slot0));
  float2 u = make_float2(0.f, 0.f);
  if(tau0 >= -kWindow) {
#pragma unroll
    for(int k = 0; k < K; ++k) cfmaf(acc[k], c[Q + 1], w0);
#pragma unroll
    for(int m = 1; m < K + Q; ++m) {
      const float2 d = pref32<LAB>(__ldg(rd + slot0 + m));
      u.x += d.x;
      u.y += d.y;
#pragma unroll
      for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) cfmaf(acc[k], c[k + Q - m], u);
    }
  } else {
    // early steps: absolute samples, taps before step -22 skipped
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
      for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) cfmaf(acc[k], c[k + Q - m], w);
    }
  }
}

// The same convolution with the accumulators and coefficients as packed
// FP32 pairs: half the FMA instructions, more registers.
template <int Q, bool LAB, int K>
__device__ __forceinline__ void window_conv_mixed_packed(const float2 *rw, const float2 *rd, int slot0, int tau0,
                                                  const float2 (&c)[Q + 2], float2 (&accf)[K])
{
  unsigned long long cxx[Q + 2], cyy[Q + 2], acc[K];
#pragma unroll
  for(int i = 0; i <= Q + 1; ++i) {
    cxx[i] = pk2(make_float2(c[i].x, c[i].x));
    cyy[i] = pk2(make_float2(-c[i].y, c[i].y));
  }
#pragma unroll
  for(int k = 0; k < K; ++k) acc[k] = pk2(accf[k]);
  const float2 w0f = pref32<LAB>(__ldg(rw + slot0));
  const unsigned long long w0 = pk2(w0f), w0s = pk2(make_float2(w0f.y, w0f.x));
  unsigned long long u = pk2(make_float2(0.f, 0.f));
  if(tau0 >= -kWindow) {
#pragma unroll
    for(int k = 0; k < K; ++k) cfma2(acc[k], cxx[Q + 1], cyy[Q + 1], w0, w0s);
#pragma unroll
    for(int m = 1; m < K + Q; ++m) {
      u = fadd2(u, pk2(pref32<LAB>(__ldg(rd + slot0 + m))));
      const float2 uf = upk2(u);
      const unsigned long long us = pk2(make_float2(uf.y, uf.x));
#pragma unroll
      for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k)
        cfma2(acc[k], cxx[k + Q - m], cyy[k + Q - m], u, us);
    }
  } else {
    // early steps: absolute samples, taps before step -22 skipped
#pragma unroll
    for(int m = 0; m < K + Q; ++m) {
      if(m > 0) u = fadd2(u, pk2(pref32<LAB>(__ldg(rd + slot0 + m))));
      if(tau0 + m < -kWindow) continue;
      const float2 wf = make_float2(w0f.x + upk2(u).x, w0f.y + upk2(u).y);
      const unsigned long long w = pk2(wf), ws = pk2(make_float2(wf.y, wf.x));
#pragma unroll
      for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k)
        cfma2(acc[k], cxx[k + Q - m], cyy[k + Q - m], w, ws);
    }
  }
#pragma unroll
  for(int k = 0; k < K; ++k) accf[k] = upk2(acc[k]);
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
