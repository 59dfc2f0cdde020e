// Far-pair kernel with on-the-fly coefficients: the same K-step sum as the
// table path (qg_far.cu) for ensembles whose coefficient table does not fit
// in device memory (N = 65536 needs 215 GB in FP64).  Each warp owns a
// target tile (lane = target dot) and a group of `group` source tiles; for
// every source the 32 lanes compute their pair's floor delay and q+1
// coefficients (pair_coef_otf, in the reference's orientation: src = larger
// user index) and, for pairs with delay >= K, apply them to the source's
// K + q window exactly as the table path does.  The coefficients are
// computed once per pair per K steps, so about 400 instructions of
// coefficient work are shared by K = 16 steps of (q+1)-tap convolution.
//
// FP64: FP64 coefficients and convolution.  Mixed: FP32 coefficients
// (pair_coef_otf_mixed: FP64 only for the distance, the delay split and the
// phase reduction) with their sum from the Lagrange identities, and the FP32
// difference-form convolution of the mixed table path.
//
// Compiled with -fmad=false (the delay arithmetic must match the near-pair
// search bit for bit); the convolution's products are explicit fused
// multiply-adds, so they round as in the table path.
#include <cuda_runtime.h>

#include "qg_coef.cuh"
#include "qg_conv.cuh"

namespace qg {

// PACKED: the mixed convolution with packed FP32 pairs (same bits).
template <int Q, bool LAB, bool MIXED, int K = kTimeBlock, bool PACKED = false>
__device__ __forceinline__ void far_body_otf(const FarArgs &a, int task)
{
  const int lane = threadIdx.x & 31;
  const int n_tiles = a.tile_n > 0 ? a.tile_n : a.nT;  // target tiles of this launch
  if(task >= n_tiles * a.nG) return;                   // uniform per warp
  const int I = a.tile_lo + (a.gmajor ? task % n_tiles : task / a.nG);
  const int g = a.gmajor ? task / n_tiles : task % a.nG;
  const int J0 = g * a.group;
  const int nJ = min(a.group, a.nT - J0);
  const int t0 = *a.d_t0;
  if(task == 0 && lane == 0) *a.far_t0_out = t0;
  const int W = a.W;
  const int ia = I * kTile + lane;
  const int ua = a.user[ia];
  double pa[3], da[3];
#pragma unroll
  for(int k = 0; k < 3; ++k) {
    pa[k] = a.pos[3 * ia + k];
    da[k] = a.dip[3 * ia + k];
  }

  double2 acc[K];
  MixedAcc<K, PACKED> accf;
#pragma unroll
  for(int k = 0; k < K; ++k) acc[k] = make_double2(0.0, 0.0);
  if(MIXED) accf.zero();

  const int iters = nJ * kTile;
  for(int it = 0; it < iters; ++it) {
    const int ib = J0 * kTile + it;
    const int ub = __ldg(a.user + ib);  // the same source for all lanes
    const bool valid = ia != ib && ua >= 0 && ub >= 0;
    if(!__any_sync(0xffffffffu, valid)) continue;
    double pb[3], db[3];
#pragma unroll
    for(int k = 0; k < 3; ++k) {
      pb[k] = __ldg(a.pos + 3 * ib + k);
      db[k] = __ldg(a.dip + 3 * ib + k);
    }
    // reference orientation: src = larger user index
    const bool a_src = ua > ub;
    double ps[3], po[3], ds[3], dob[3];
#pragma unroll
    for(int k = 0; k < 3; ++k) {
      ps[k] = a_src ? pa[k] : pb[k];
      po[k] = a_src ? pb[k] : pa[k];
      ds[k] = a_src ? da[k] : db[k];
      dob[k] = a_src ? db[k] : da[k];
    }
    if(MIXED) {
      float2 cf[Q + 2];
      const int d = pair_coef_otf_mixed<Q>(ps, po, ds, dob, a.cp, cf);
      if(valid && d >= kTimeBlock) {
        const int tau0 = t0 - d - Q;
        int slot0 = tau0 % W;
        if(slot0 < 0) slot0 += W;
        window_conv_mixed<Q, LAB, K, PACKED>(a.ring32w + (long long)ib * a.stride,
                                             a.ring32d + (long long)ib * a.stride, slot0, tau0, cf, accf);
      }
    } else {
      double2 c[Q + 1];
      const int d = pair_coef_otf<Q>(ps, po, ds, dob, a.cp, c);
      if(valid && d >= kTimeBlock) {
        const int tau0 = t0 - d - Q;
        int slot0 = tau0 % W;
        if(slot0 < 0) slot0 += W;
        window_conv<Q, LAB, K>(a.ring + (long long)ib * a.stride, slot0, tau0, c, acc);
      }
    }
  }
  if(MIXED) {
#pragma unroll
    for(int k = 0; k < K; ++k) acc[k] = mixed_out(accf, k);
  }
  group_partials_reduce<K>(a, I, g, acc);
}

template <int Q, bool LAB, bool MIXED>
__global__ void __launch_bounds__(128) far_otf_kernel(FarArgs a)
{
  far_body_otf<Q, LAB, MIXED>(a, blockIdx.x * 4 + (threadIdx.x >> 5));
}

// The same held to 3 blocks per SM (the FP64 form takes 186 registers and
// fits 2 uncapped); same results.
template <int Q, bool LAB, bool MIXED>
__global__ void __launch_bounds__(128, 3) far_otf_kernel_r3(FarArgs a)
{
  far_body_otf<Q, LAB, MIXED>(a, blockIdx.x * 4 + (threadIdx.x >> 5));
}

template <bool LAB, bool MIXED>
static void launch_otf_q(const FarArgs &a, bool r3, cudaStream_t s)
{
  const unsigned blocks = (unsigned)(((long long)(a.tile_n > 0 ? a.tile_n : a.nT) * a.nG + 3) / 4);
#define QG_OTF_CASE(QQ)                                                  \
  case QQ:                                                               \
    if(r3)                                                               \
      far_otf_kernel_r3<QQ, LAB, MIXED><<<blocks, 128, 0, s>>>(a);       \
    else                                                                 \
      far_otf_kernel<QQ, LAB, MIXED><<<blocks, 128, 0, s>>>(a);          \
    break;
  switch(a.q) {
    QG_OTF_CASE(1)
    QG_OTF_CASE(2)
    QG_OTF_CASE(3)
    QG_OTF_CASE(4)
    QG_OTF_CASE(5)
    QG_OTF_CASE(6)
    QG_OTF_CASE(7)
    default: break;
  }
#undef QG_OTF_CASE
}

void launch_far_otf(const FarArgs &a0, void *stream)
{
  if(a0.nT <= 0) return;
  FarArgs a = a0;
  // 7 and 8: source-group-major task order; 1 and 8: held to 3 blocks per
  // SM (same sums either way)
  a.gmajor = a0.variant == 7 || a0.variant == 8;
  const bool r3 = a0.variant == 1 || a0.variant == 8;
  cudaStream_t s = (cudaStream_t)stream;
  if(a.frame == 0) {
    if(a.mixed)
      launch_otf_q<false, true>(a, r3, s);
    else
      launch_otf_q<false, false>(a, r3, s);
  } else {
    if(a.mixed)
      launch_otf_q<true, true>(a, r3, s);
    else
      launch_otf_q<true, false>(a, r3, s);
  }
}

}  // namespace qg
