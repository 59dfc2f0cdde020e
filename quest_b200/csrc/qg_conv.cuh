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

template <int Q, bool LAB, int K>
__device__ __forceinline__ void window_conv_mixed(const float2 *rw, const float2 *rd, int slot0, int tau0,
                                                  const float2 (&c)[Q + 2], float2 (&acc)[K])
{
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
