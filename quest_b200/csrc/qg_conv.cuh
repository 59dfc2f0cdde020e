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
