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
// Per ordered pair the K steps read one window of K + q consecutive history
// samples of the source and form a K-output, (q+1)-tap convolution with the
// pair's coefficients: K (q+1) complex multiply-adds per ordered pair per
// pass, each coefficient read from HBM once per K steps.  The window is
// consumed one sample at a time (each sample feeds up to q+1 outputs), so
// only the K accumulators and the q+1 coefficients stay in registers.
//
// Schedule.  One warp owns a target tile I (lane l = dot 32 I + l) and a
// group of a.group source tiles.  At each step all 32 lanes take the same
// source b, so their windows, at the 32 different delays d(a_l, b), fall in
// one short stretch of b's history row: a handful of cache lines per load
// instead of 32.  The sums over the group are written as partials; the last
// warp of a target tile (completion counter) adds the nG partials in a fixed
// order, so the result does not depend on scheduling.
//
// The rho01 ring holds rho01 by time slot (slot = t mod W) with the first
// kRingMirror slots repeated after slot W-1, so every window is contiguous.
// Polarisation prefactor: rho01 in the rotating frame
// (rotating_green_function.h:17-21), 2 Re rho01 in the lab frame
// (green_function.h:23-27).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "qg_conv.cuh"

namespace qg {

// Same convolution reading two samples per 32-byte load (ld.global.nc.v4.f64).
// The window starts at slot0; the loads start at the even slot below it
// (rows are 32-byte aligned: even stride, even W), PAR = slot0 & 1.
template <bool LAB>
__device__ __forceinline__ void ld2(const double2 *p, double2 &x, double2 &y)
{
  double a0, a1, a2, a3;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a0), "=d"(a1), "=d"(a2), "=d"(a3) : "l"(p));
  x = LAB ? make_double2(2 * a0, 0.0) : make_double2(a0, a1);
  y = LAB ? make_double2(2 * a2, 0.0) : make_double2(a2, a3);
}

template <int Q, bool LAB, int PAR, int K>
__device__ __forceinline__ void window_conv2(const double2 *ring, int slot_even, int tau0,
                                             const double2 (&c)[Q + 1], double2 (&acc)[K])
{
  constexpr int NV = (K + Q + PAR + 1) / 2;
  const bool full = tau0 >= -kWindow;
#pragma unroll
  for(int v = 0; v < NV; ++v) {
    double2 w2[2];
    ld2<LAB>(ring + slot_even + 2 * v, w2[0], w2[1]);
#pragma unroll
    for(int e = 0; e < 2; ++e) {
      const int m = 2 * v + e - PAR;
      if(m < 0 || m >= K + Q) continue;
      if(!full && tau0 + m < -kWindow) continue;
#pragma unroll
      for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) cfma(acc[k], c[k + Q - m], w2[e]);
    }
  }
}

// K outputs: the first K steps of the block (K = kTimeBlock in the run; 1 for
// a single-step evaluation).  Pairs with delay < kTimeBlock are left to the
// mid list in either case.
template <int Q, bool LAB, int VEC, int K = kTimeBlock, bool EARLY = false>
__device__ __forceinline__ void far_body(const FarArgs &a, int task)
{
  const int lane = threadIdx.x & 31;
  static_assert(VEC == 0 || VEC == 1, "VEC");
  if(task >= a.nT * a.nG) return;  // uniform per warp
  const int I = a.gmajor ? task % a.nT : task / a.nG, g = a.gmajor ? task / a.nT : task % a.nG;
  const int J0 = g * a.group;
  const int nJ = min(a.group, a.nT - J0);
  const int t0 = *a.d_t0;
  if(task == 0 && lane == 0) *a.far_t0_out = t0;
  const int W = a.W;

  double2 acc[K];
#pragma unroll
  for(int k = 0; k < K; ++k) acc[k] = make_double2(0.0, 0.0);

  const long long tile0 = (long long)I * a.nT + J0;
  const int iters = nJ * kTile;
  // software prefetch of the next source's delay and coefficients
  // the table is streamed once per pass: evict-first loads keep the history
  // ring and the per-step kernels' data resident in L2
  int dn = __ldcs(a.delay + tile0 * kTilePairs + lane);
  double2 cn[Q + 1];
#pragma unroll
  for(int i = 0; i <= Q; ++i) cn[i] = __ldcs(a.coef + (tile0 * (Q + 1) + i) * kTilePairs + lane);
  for(int it = 0; it < iters; ++it) {
    const int d = dn;
    double2 c[Q + 1];
#pragma unroll
    for(int i = 0; i <= Q; ++i) c[i] = cn[i];
    if(it + 1 < iters) {
      const long long tile = tile0 + (it + 1) / kTile;
      const int e = ((it + 1) % kTile) * kTile + lane;
      dn = __ldcs(a.delay + tile * kTilePairs + e);
#pragma unroll
      for(int i = 0; i <= Q; ++i) cn[i] = __ldcs(a.coef + (tile * (Q + 1) + i) * kTilePairs + e);
    }
    if(d >= kTimeBlock) {
      const int ib = (J0 + it / kTile) * kTile + (it % kTile);
      const int tau0 = t0 - d - Q;
      int slot0 = tau0 % W;
      if(slot0 < 0) slot0 += W;
      const double2 *row = a.ring + (long long)ib * a.stride;
      if(VEC == 1) {
        if(slot0 & 1)
          window_conv2<Q, LAB, 1, K>(row, slot0 - 1, tau0, c, acc);
        else
          window_conv2<Q, LAB, 0, K>(row, slot0, tau0, c, acc);
      } else if(EARLY) {
        window_conv_uniform<Q, LAB, K>(row, slot0, tau0, c, acc);
      } else {
        window_conv<Q, LAB, K>(row, slot0, tau0, c, acc);
      }
    }
  }

  group_partials_reduce<K>(a, I, g, acc);
}

__device__ __forceinline__ int warp_task() { return blockIdx.x * 4 + (threadIdx.x >> 5); }

// Table entries staged in shared memory by asynchronous copies (cp.async),
// P sources ahead of the convolution: each lane copies its own delay and
// q+1 coefficients of source it + P - 1 while it convolves source it, so the
// HBM latency of the table stream is covered without holding prefetched
// values in registers.  The copies carry an L2 evict-first policy (the table
// is streamed once per launch; the history ring should stay in L2).
template <int Q, int P>
struct FarStage {
  double2 coef[P][Q + 1][32];
  int delay[P][32];
};

__device__ __forceinline__ void cp_async16(void *dst, const void *src, unsigned long long pol)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "l"(pol));
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src, unsigned long long pol)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "l"(pol));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N)); }

template <int Q, bool LAB, int P, int VEC, int K = kTimeBlock>
__device__ __forceinline__ void far_body_async(const FarArgs &a, int task, FarStage<Q, P> &st)
{
  const int lane = threadIdx.x & 31;
  if(task >= a.nT * a.nG) return;  // uniform per warp
  const int I = a.gmajor ? task % a.nT : task / a.nG, g = a.gmajor ? task / a.nT : task % a.nG;
  const int J0 = g * a.group;
  const int nJ = min(a.group, a.nT - J0);
  const int t0 = *a.d_t0;
  if(task == 0 && lane == 0) *a.far_t0_out = t0;
  const int W = a.W;
  unsigned long long pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));

  double2 acc[K];
#pragma unroll
  for(int k = 0; k < K; ++k) acc[k] = make_double2(0.0, 0.0);

  const long long tile0 = (long long)I * a.nT + J0;
  const int iters = nJ * kTile;
  auto issue = [&](int it) {
    const int slot = it % P;
    const long long tile = tile0 + it / kTile;
    const int e = (it % kTile) * kTile + lane;
#pragma unroll
    for(int i = 0; i <= Q; ++i) cp_async16(&st.coef[slot][i][lane], a.coef + (tile * (Q + 1) + i) * kTilePairs + e, pol);
    cp_async4(&st.delay[slot][lane], a.delay + tile * kTilePairs + e, pol);
  };
#pragma unroll
  for(int p = 0; p < P - 1; ++p) {
    if(p < iters) issue(p);
    cp_async_commit();
  }
  for(int it = 0; it < iters; ++it) {
    if(it + P - 1 < iters) issue(it + P - 1);
    cp_async_commit();
    if(VEC == 2) {
      // sources it and it+1 have landed; pull it+1's history window into L1
      // while `it` is convolved (its lanes' windows span a few lines)
      cp_async_wait<P - 2>();
      if(it + 1 < iters) {
        const int d1 = st.delay[(it + 1) % P][lane];
        if(d1 >= kTimeBlock) {
          int s1 = (t0 - d1 - Q) % W;
          if(s1 < 0) s1 += W;
          const char *p1 = reinterpret_cast<const char *>(
              a.ring + (long long)((J0 + (it + 1) / kTile) * kTile + ((it + 1) % kTile)) * a.stride + s1);
#pragma unroll
          for(int b = 0; b < 3; ++b) asm volatile("prefetch.global.L1 [%0];" ::"l"(p1 + 128 * b));
          asm volatile("prefetch.global.L1 [%0];" ::"l"(p1 + 16 * (K + Q) - 1));
        }
      }
    } else {
      cp_async_wait<P - 1>();  // the group holding source `it` has landed
    }
    const int slot = it % P;
    const int d = st.delay[slot][lane];
    if(d >= kTimeBlock) {
      double2 c[Q + 1];
#pragma unroll
      for(int i = 0; i <= Q; ++i) c[i] = st.coef[slot][i][lane];
      const int ib = (J0 + it / kTile) * kTile + (it % kTile);
      const int tau0 = t0 - d - Q;
      int slot0 = tau0 % W;
      if(slot0 < 0) slot0 += W;
      const double2 *row = a.ring + (long long)ib * a.stride;
      if(VEC == 1) {
        if(slot0 & 1)
          window_conv2<Q, LAB, 1, K>(row, slot0 - 1, tau0, c, acc);
        else
          window_conv2<Q, LAB, 0, K>(row, slot0, tau0, c, acc);
      } else if(VEC == 3 && tau0 >= -kWindow) {
        window_conv_pairs<Q, LAB, K>(row, slot0, c, acc);
      } else {
        window_conv<Q, LAB, K>(row, slot0, tau0, c, acc);
      }
    }
  }
  cp_async_wait<0>();
  group_partials_reduce<K>(a, I, g, acc);
}

constexpr int kFarStages = 3;
static_assert(4 * sizeof(FarStage<kMaxOrder, kFarStages>) <= 227 * 1024, "far stage buffers");

// ---- table staged by the bulk-copy (TMA) engine ---------------------------------
// Variant 9: for each source, lane 0 asks the copy engine for the source's
// q+1 coefficient rows (32 lanes x 16 B = 512 B each) and its delay row
// (128 B) with cp.async.bulk, completing on a per-stage mbarrier, P - 1
// sources ahead; the lanes wait on the barrier's phase and read their entries
// from shared memory.  The copies are plain global -> own shared memory (no
// cluster multicast); sizes and addresses are multiples of 16 B (rows start
// on 512-B and 128-B boundaries of 256-B aligned allocations).  Every wait is
// bounded: one that runs out sets *a.d_bad = -3, waits (bounded again) for the
// copies still in flight into this warp's buffers, and ends the warp.
constexpr int kBulkSpins = 1 << 20;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// true once the barrier's phase with the given parity has completed, false
// when kBulkSpins polls ran out
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity)
{
  for(int spin = 0; spin < kBulkSpins; ++spin) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if(done) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar,
                                         unsigned long long pol)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}

template <int Q, bool LAB, int P, int K = kTimeBlock>
__device__ __forceinline__ void far_body_bulk(const FarArgs &a, int task, FarStage<Q, P> &st,
                                              unsigned long long *bar)
{
  const int lane = threadIdx.x & 31;
  if(task >= a.nT * a.nG) return;  // uniform per warp; the barriers are this warp's alone
  const int I = a.gmajor ? task % a.nT : task / a.nG, g = a.gmajor ? task / a.nT : task % a.nG;
  const int J0 = g * a.group;
  const int nJ = min(a.group, a.nT - J0);
  const int t0 = *a.d_t0;
  if(task == 0 && lane == 0) *a.far_t0_out = t0;
  const int W = a.W;
  unsigned long long pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  constexpr unsigned kStageBytes = (Q + 1) * kTile * sizeof(double2) + kTile * sizeof(int);

  if(lane == 0) {
#pragma unroll
    for(int p = 0; p < P; ++p) mbar_init(&bar[p], 1);
    mbar_init_fence();
  }
  __syncwarp();

  double2 acc[K];
#pragma unroll
  for(int k = 0; k < K; ++k) acc[k] = make_double2(0.0, 0.0);

  const long long tile0 = (long long)I * a.nT + J0;
  const int iters = nJ * kTile;
  // source `it` goes to stage it % P; its barrier completes phase it / P
  auto issue = [&](int it) {  // lane 0
    const int slot = it % P;
    const long long tile = tile0 + it / kTile;
    const int j = it % kTile;
    mbar_arrive_expect_tx(&bar[slot], kStageBytes);
#pragma unroll
    for(int i = 0; i <= Q; ++i)
      bulk_g2s(&st.coef[slot][i][0], a.coef + (tile * (Q + 1) + i) * kTilePairs + j * kTile,
               kTile * sizeof(double2), &bar[slot], pol);
    bulk_g2s(&st.delay[slot][0], a.delay + tile * kTilePairs + j * kTile, kTile * sizeof(int), &bar[slot], pol);
  };
  if(lane == 0) {
#pragma unroll
    for(int p = 0; p < P - 1; ++p)
      if(p < iters) issue(p);
  }
  int it = 0;
  bool ok = true;
  for(; it < iters; ++it) {
    // the stage of source it - 1 was read by every lane (syncwarp below)
    if(lane == 0 && it + P - 1 < iters) issue(it + P - 1);
    const int slot = it % P;
    ok = __all_sync(0xffffffffu, mbar_wait(&bar[slot], (unsigned)((it / P) & 1)));
    if(!ok) break;
    const int d = st.delay[slot][lane];
    double2 c[Q + 1];
#pragma unroll
    for(int i = 0; i <= Q; ++i) c[i] = st.coef[slot][i][lane];
    __syncwarp();
    if(d >= kTimeBlock) {
      const int ib = (J0 + it / kTile) * kTile + (it % kTile);
      const int tau0 = t0 - d - Q;
      int slot0 = tau0 % W;
      if(slot0 < 0) slot0 += W;
      window_conv<Q, LAB, K>(a.ring + (long long)ib * a.stride, slot0, tau0, c, acc);
    }
  }
  if(!ok) {
    // record the failure, let the copies already issued into this warp's
    // stages (sources it .. it + P - 1) land, then stop
    if(lane == 0) atomicMin(a.d_bad, -3);
    for(int r = it; r < min(iters, it + P); ++r) mbar_wait(&bar[r % P], (unsigned)((r / P) & 1));
    return;
  }
  group_partials_reduce<K>(a, I, g, acc);
}

template <int Q, bool LAB>
__global__ void __launch_bounds__(128) far_kernel_bulk(FarArgs a)
{
  extern __shared__ double2 far_smem[];
  __shared__ unsigned long long bars[4][kFarStages];
  FarStage<Q, kFarStages> *st = reinterpret_cast<FarStage<Q, kFarStages> *>(far_smem);
  far_body_bulk<Q, LAB, kFarStages>(a, warp_task(), st[threadIdx.x >> 5], bars[threadIdx.x >> 5]);
}

// ---- history windows staged in shared memory --------------------------------
// Variants 10 and 11 (11: source-group-major order): each source's history
// window union staged in shared memory.  For source b the 32 lanes' windows
// (one per target's delay d_l) cover steps t0 - max_l d_l - q ..
// t0 - min_l d_l + K - 1 of b's ring row: one contiguous run of at most
// kWinCap samples for compact target tiles.  The warp copies that run with
// coalesced 16-byte cp.async (each lane up to kWinCap / 32 chunks, bypassing
// L1) one source ahead of the convolution, and the lanes read their windows
// from shared memory at offset max d - d_l; the table is staged as in
// variant 3.  A source whose run is longer than kWinCap is read from global
// memory as in variant 0.  The products and their order are variant 0's, so
// the sums are identical.
//
// Pipeline (cp.async groups, committed in this order at iteration it): the
// table stage of source it + 2, then, once source it + 1's delays have
// landed, its window run.  Waiting for all but the newest group therefore
// completes source it + 1's table stage and source it's window.
constexpr int kWinCap = 128;  // samples per staged window run (2 KB)
constexpr int kWinStages = 3;

template <int Q>
struct FarWinStage {
  FarStage<Q, kWinStages> tab;
  double2 win[2][kWinCap];
};

template <int Q, bool LAB, int K>
__device__ __forceinline__ void window_conv_shared(const double2 *w, int tau0, const double2 (&c)[Q + 1],
                                                   double2 (&acc)[K])
{
#pragma unroll
  for(int m = 0; m < K + Q; ++m) {
    if(tau0 < -kWindow && tau0 + m < -kWindow) continue;
    const double2 r = w[m];
    const double2 v = LAB ? make_double2(2 * r.x, 0.0) : r;
#pragma unroll
    for(int k = (m - Q > 0 ? m - Q : 0); k <= (m < K - 1 ? m : K - 1); ++k) cfma(acc[k], c[k + Q - m], v);
  }
}

__device__ __forceinline__ void cp_async16_l2(void *dst, const void *src)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src));
}

template <int Q, bool LAB, int K = kTimeBlock>
__device__ __forceinline__ void far_body_wstage(const FarArgs &a, int task, FarWinStage<Q> &ws)
{
  constexpr int P = kWinStages;
  const int lane = threadIdx.x & 31;
  if(task >= a.nT * a.nG) return;  // uniform per warp
  const int I = a.gmajor ? task % a.nT : task / a.nG, g = a.gmajor ? task / a.nT : task % a.nG;
  const int J0 = g * a.group;
  const int nJ = min(a.group, a.nT - J0);
  const int t0 = *a.d_t0;
  if(task == 0 && lane == 0) *a.far_t0_out = t0;
  const int W = a.W;
  unsigned long long pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  FarStage<Q, P> &st = ws.tab;

  double2 acc[K];
#pragma unroll
  for(int k = 0; k < K; ++k) acc[k] = make_double2(0.0, 0.0);

  const long long tile0 = (long long)I * a.nT + J0;
  const int iters = nJ * kTile;
  auto issue_table = [&](int it) {
    if(it < iters) {
      const int slot = it % P;
      const long long tile = tile0 + it / kTile;
      const int e = (it % kTile) * kTile + lane;
#pragma unroll
      for(int i = 0; i <= Q; ++i)
        cp_async16(&st.coef[slot][i][lane], a.coef + (tile * (Q + 1) + i) * kTilePairs + e, pol);
      cp_async4(&st.delay[slot][lane], a.delay + tile * kTilePairs + e, pol);
    }
    cp_async_commit();
  };
  auto row_of = [&](int it) { return a.ring + (long long)((J0 + it / kTile) * kTile + (it % kTile)) * a.stride; };
  // source it's window run, its delays having landed: returns the largest
  // delay among the lanes that need the source (-1: none does), and whether
  // the run was staged (it fits kWinCap)
  auto issue_window = [&](int it, bool &staged) {
    int dmax = -1;
    staged = false;
    if(it < iters) {
      const int d = st.delay[it % P][lane];
      const bool need = d >= kTimeBlock;
      dmax = __reduce_max_sync(0xffffffffu, need ? d : -1);
      const int dmin = __reduce_min_sync(0xffffffffu, need ? d : 0x7fffffff);
      const int span = dmax - dmin + K + Q;
      if(dmax >= 0 && span <= kWinCap) {
        staged = true;
        int lo = (t0 - dmax - Q) % W;
        if(lo < 0) lo += W;
        const double2 *row = row_of(it);
        double2 *dst = ws.win[it & 1];
#pragma unroll
        for(int r = 0; r < kWinCap / 32; ++r) {
          const int m = lane + 32 * r;
          if(m < span) {
            int sl = lo + m;
            if(sl >= W) sl -= W;
            cp_async16_l2(dst + m, row + sl);
          }
        }
      }
    }
    cp_async_commit();
    return dmax;
  };

  // prologue: table stages 0 and 1, then source 0's window
  issue_table(0);
  issue_table(1);
  cp_async_wait<1>();
  __syncwarp();
  bool staged_cur;
  int dmax_cur = issue_window(0, staged_cur);
  for(int it = 0; it < iters; ++it) {
    // every lane has finished with source it - 1's table stage and window
    __syncwarp();
    issue_table(it + 2);
    cp_async_wait<1>();  // source it + 1's table stage and source it's window
    __syncwarp();
    bool staged_next;
    const int dmax_next = issue_window(it + 1, staged_next);
    const int slot = it % P;
    const int d = st.delay[slot][lane];
    if(d >= kTimeBlock) {
      double2 c[Q + 1];
#pragma unroll
      for(int i = 0; i <= Q; ++i) c[i] = st.coef[slot][i][lane];
      const int tau0 = t0 - d - Q;
      if(staged_cur) {
        window_conv_shared<Q, LAB, K>(&ws.win[it & 1][dmax_cur - d], tau0, c, acc);
      } else {
        int slot0 = tau0 % W;
        if(slot0 < 0) slot0 += W;
        window_conv<Q, LAB, K>(row_of(it), slot0, tau0, c, acc);
      }
    }
    staged_cur = staged_next;
    dmax_cur = dmax_next;
  }
  cp_async_wait<0>();
  group_partials_reduce<K>(a, I, g, acc);
}

template <int Q, bool LAB>
__global__ void __launch_bounds__(128) far_kernel_wstage(FarArgs a)
{
  extern __shared__ double2 far_smem[];
  FarWinStage<Q> *ws = reinterpret_cast<FarWinStage<Q> *>(far_smem);
  far_body_wstage<Q, LAB>(a, warp_task(), ws[threadIdx.x >> 5]);
}

// Variant 6 is held to 128 registers (4 blocks, 16 warps per SM); uncapped
// it takes 132 and fits 3 blocks.
template <int Q, bool LAB, int VEC>
__global__ void __launch_bounds__(128, VEC == 3 ? 4 : 3) far_kernel_async(FarArgs a)
{
  extern __shared__ double2 far_smem[];
  constexpr int P = VEC == 2 ? kFarStages + 1 : kFarStages;
  FarStage<Q, P> *st = reinterpret_cast<FarStage<Q, P> *>(far_smem);
  far_body_async<Q, LAB, P, VEC>(a, warp_task(), st[threadIdx.x >> 5]);
}

// Variants of the same kernel (identical arithmetic and results):
//   far_kernel        3 blocks of 4 warps per SM, one sample per load
//   far_kernel_r4     registers capped for 4 blocks per SM
//   far_kernel_v2     capped, two samples per 32-byte load
//   far_kernel_async  table staged in shared memory by cp.async, 3 sources
//                     ahead; one sample (variant 3) or two (variant 4, a
//                     branch on each lane's window parity) per load; variant
//                     5: 4 stages and the next source's history window
//                     prefetched into L1; variant 6: two samples per load
//                     with the parity taken by selects (window_conv_pairs)
// ---- mixed precision ---------------------------------------------------------
// The tap sum of one pair, sum_i c_i w_i, is formed as
//     (sum_i c_i) w_0 + sum_i c_i (w_i - w_0),
// w_0 the window's first sample and w_i - w_0 the running sum of the FP32
// step-to-step differences (themselves computed in FP64).  The large
// interpolation weights (w1 ~ 1/dt, w2 ~ 1/dt^2) multiply only differences,
// and sum_i c_i carries no such factor, so FP32 storage loses no more than a
// few units in the last place of the pair's contribution.  The first term is
// the same for all K outputs and is accumulated once per pair (MixedAcc).
template <int Q, bool LAB, int K = kTimeBlock, bool PACKED = false>
__device__ __forceinline__ void far_body_mixed(const FarArgs &a, int task)
{
  const int lane = threadIdx.x & 31;
  if(task >= a.nT * a.nG) return;  // uniform per warp
  const int I = a.gmajor ? task % a.nT : task / a.nG, g = a.gmajor ? task / a.nT : task % a.nG;
  const int J0 = g * a.group;
  const int nJ = min(a.group, a.nT - J0);
  const int t0 = *a.d_t0;
  if(task == 0 && lane == 0) *a.far_t0_out = t0;
  const int W = a.W;

  MixedAcc<K, PACKED> acc;
  acc.zero();

  const long long tile0 = (long long)I * a.nT + J0;
  const int iters = nJ * kTile;
  int dn = __ldcs(a.delay + tile0 * kTilePairs + lane);
  float2 cn[Q + 2];
#pragma unroll
  for(int i = 0; i <= Q + 1; ++i) cn[i] = __ldcs(a.coef32 + (tile0 * (Q + 2) + i) * kTilePairs + lane);
  for(int it = 0; it < iters; ++it) {
    const int d = dn;
    float2 c[Q + 2];
#pragma unroll
    for(int i = 0; i <= Q + 1; ++i) c[i] = cn[i];
    if(it + 1 < iters) {
      const long long tile = tile0 + (it + 1) / kTile;
      const int e = ((it + 1) % kTile) * kTile + lane;
      dn = __ldcs(a.delay + tile * kTilePairs + e);
#pragma unroll
      for(int i = 0; i <= Q + 1; ++i) cn[i] = __ldcs(a.coef32 + (tile * (Q + 2) + i) * kTilePairs + e);
    }
    if(d >= kTimeBlock) {
      const int ib = (J0 + it / kTile) * kTile + (it % kTile);
      const int tau0 = t0 - d - Q;
      int slot0 = tau0 % W;
      if(slot0 < 0) slot0 += W;
      window_conv_mixed<Q, LAB, K, PACKED>(a.ring32w + (long long)ib * a.stride,
                                           a.ring32d + (long long)ib * a.stride, slot0, tau0, c, acc);
    }
  }

  // the per-dot sums across groups are carried in FP64
  double2 acc64[K];
#pragma unroll
  for(int k = 0; k < K; ++k) acc64[k] = mixed_out(acc, k);
  group_partials_reduce<K>(a, I, g, acc64);
}


template <int Q, bool LAB>
__global__ void __launch_bounds__(128) far_kernel(FarArgs a) { far_body<Q, LAB, 0>(a, warp_task()); }
// The same for the first blocks of a run (some windows start before step
// -22): one loop for all lanes of a warp (window_conv_uniform), same
// results; held to 3 blocks per SM like far_kernel (uncapped, its extra loop
// takes 182 registers and 2 blocks).
template <int Q, bool LAB>
__global__ void __launch_bounds__(128, 3) far_kernel_early(FarArgs a)
{
  far_body<Q, LAB, 0, kTimeBlock, true>(a, warp_task());
}
template <int Q, bool LAB>
__global__ void __launch_bounds__(128, 4) far_kernel_r4(FarArgs a) { far_body<Q, LAB, 0>(a, warp_task()); }
template <int Q, bool LAB>
__global__ void __launch_bounds__(128, 4) far_kernel_v2(FarArgs a) { far_body<Q, LAB, 1>(a, warp_task()); }

// Many ensembles in one persistent launch: a work list of (ensemble,
// target tile, source-tile group) tasks, task_off[e] = first task of
// ensemble e (prefix sums, task_off[n_ens] = total).  Warps stride over the
// list; every task writes its own partial slot, so the assignment of tasks to
// warps does not change any result.
template <int Q, bool LAB, bool MIXED, bool PACKED = false>
__global__ void __launch_bounds__(128) far_batch_kernel(const FarArgs *__restrict__ args,
                                                        const int *__restrict__ task_off, int n_ens)
{
  const int total = task_off[n_ens];
  for(int task = warp_task(); task < total; task += gridDim.x * 4) {
    int lo = 0, hi = n_ens - 1;
    while(lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if(task_off[mid] <= task)
        lo = mid;
      else
        hi = mid - 1;
    }
    const FarArgs a = args[lo];  // a copy: the bodies read its fields in their inner loops
    if(MIXED)
      far_body_mixed<Q, LAB, kTimeBlock, PACKED>(a, task - task_off[lo]);
    else
      far_body<Q, LAB, 0>(a, task - task_off[lo]);
  }
}

// FP64 members take far_kernel's body (table prefetched in registers, the
// fastest FP64 variant, 168 registers: 3 blocks per SM, the persistent
// grid's shape); mixed members the FP32 convolution, scalar (mixed == 1) or
// with packed pairs (mixed == 2).  Every form gives the same bits, so a
// member's result is the same alone and in a batch.
template <int Q, bool LAB, bool MIXED>
static void launch_far_batch_q(const FarArgs *args, const int *task_off, int n_ens, int grid, bool packed,
                               cudaStream_t s)
{
  if(MIXED && packed)
    far_batch_kernel<Q, LAB, MIXED, true><<<grid, 128, 0, s>>>(args, task_off, n_ens);
  else
    far_batch_kernel<Q, LAB, MIXED, false><<<grid, 128, 0, s>>>(args, task_off, n_ens);
}

template <bool LAB, bool MIXED>
static void launch_far_batch_frame(const FarArgs *args, const int *task_off, int n_ens, int q, int grid,
                                   bool packed, cudaStream_t s)
{
  switch(q) {
    case 1: launch_far_batch_q<1, LAB, MIXED>(args, task_off, n_ens, grid, packed, s); break;
    case 2: launch_far_batch_q<2, LAB, MIXED>(args, task_off, n_ens, grid, packed, s); break;
    case 3: launch_far_batch_q<3, LAB, MIXED>(args, task_off, n_ens, grid, packed, s); break;
    case 4: launch_far_batch_q<4, LAB, MIXED>(args, task_off, n_ens, grid, packed, s); break;
    case 5: launch_far_batch_q<5, LAB, MIXED>(args, task_off, n_ens, grid, packed, s); break;
    case 6: launch_far_batch_q<6, LAB, MIXED>(args, task_off, n_ens, grid, packed, s); break;
    case 7: launch_far_batch_q<7, LAB, MIXED>(args, task_off, n_ens, grid, packed, s); break;
    default: break;
  }
}

void launch_far_batch(const FarArgs *args, const int *task_off, int n_ens, int q, int frame, int mixed,
                      int grid, void *stream)
{
  if(n_ens <= 0) return;
  cudaStream_t s = (cudaStream_t)stream;
  const bool packed = mixed == 2;
  if(frame == 0)
    mixed ? launch_far_batch_frame<false, true>(args, task_off, n_ens, q, grid, packed, s)
          : launch_far_batch_frame<false, false>(args, task_off, n_ens, q, grid, packed, s);
  else
    mixed ? launch_far_batch_frame<true, true>(args, task_off, n_ens, q, grid, packed, s)
          : launch_far_batch_frame<true, false>(args, task_off, n_ens, q, grid, packed, s);
}

template <int Q, bool LAB>
__global__ void __launch_bounds__(128) far_kernel_mixed(FarArgs a)
{
  far_body_mixed<Q, LAB, kTimeBlock, true>(a, warp_task());
}

// The same held to 128 registers (4 blocks, 16 warps per SM, against 3):
// more warps to cover the window gathers' latency; same results.
template <int Q, bool LAB>
__global__ void __launch_bounds__(128, 4) far_kernel_mixed_r4(FarArgs a)
{
  far_body_mixed<Q, LAB, kTimeBlock, true>(a, warp_task());
}

template <int Q, bool LAB>
static void launch_far_q(const FarArgs &a0, cudaStream_t s)
{
  FarArgs a = a0;
  const unsigned blocks = (unsigned)((a.nT * a.nG + 3) / 4);
  if(a.mixed) {
    // mixed precision: 0 and 7 at 150 registers, 1 and 8 held to 128; 7 and
    // 8 in the source-group-major task order
    a.gmajor = a0.variant == 7 || a0.variant == 8;
    if(a0.variant == 1 || a0.variant == 8)
      far_kernel_mixed_r4<Q, LAB><<<blocks, 128, 0, s>>>(a);
    else
      far_kernel_mixed<Q, LAB><<<blocks, 128, 0, s>>>(a);
    return;
  }
  // the first blocks of a run take the first-blocks form whatever the
  // variant (every variant gives the same bits), source-group major
  if(a.early) {
    a.gmajor = 1;
    far_kernel_early<Q, LAB><<<blocks, 128, 0, s>>>(a);
    return;
  }
  // variants 7 and 8 are 0 and 3 with the source-group-major task order
  if(a.variant == 7 || a.variant == 8) {
    a.gmajor = 1;
    a.variant = a.variant == 7 ? 0 : 3;
  }
  if(a.variant == 1)
    far_kernel_r4<Q, LAB><<<blocks, 128, 0, s>>>(a);
  else if(a.variant == 2)
    far_kernel_v2<Q, LAB><<<blocks, 128, 0, s>>>(a);
  else if(a.variant == 10 || a.variant == 11) {
    // 10: windows staged in shared memory (3 table stages + 2 window runs per
    // warp: 54 KB a block at q = 5); 11: the same in the source-group-major
    // order
    a.gmajor = a0.variant == 11;
    const size_t smem = 4 * sizeof(FarWinStage<Q>);
    static bool attr_w[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if(dev >= 64 || !attr_w[dev]) {
      cudaFuncSetAttribute(far_kernel_wstage<Q, LAB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if(dev < 64) attr_w[dev] = true;
    }
    far_kernel_wstage<Q, LAB><<<blocks, 128, smem, s>>>(a);
  }
  else if((a.variant >= 3 && a.variant <= 6) || a.variant == 9) {
    // 38 KB at q = 5, 51 KB at q = 7 (above the 48 KB default: opt in);
    // variant 5 keeps one more stage
    const size_t smem = 4 * sizeof(FarStage<Q, kFarStages>), smem5 = 4 * sizeof(FarStage<Q, kFarStages + 1>);
    static bool attr_set[64] = {};  // the attribute is per function and device
    int dev = 0;
    cudaGetDevice(&dev);
    if(dev >= 64 || !attr_set[dev]) {
      cudaFuncSetAttribute(far_kernel_async<Q, LAB, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaFuncSetAttribute(far_kernel_async<Q, LAB, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaFuncSetAttribute(far_kernel_async<Q, LAB, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem5);
      cudaFuncSetAttribute(far_kernel_async<Q, LAB, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaFuncSetAttribute(far_kernel_bulk<Q, LAB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if(dev < 64) attr_set[dev] = true;
    }
    if(a.variant == 3)
      far_kernel_async<Q, LAB, 0><<<blocks, 128, smem, s>>>(a);
    else if(a.variant == 4)
      far_kernel_async<Q, LAB, 1><<<blocks, 128, smem, s>>>(a);
    else if(a.variant == 6)
      far_kernel_async<Q, LAB, 3><<<blocks, 128, smem, s>>>(a);
    else if(a.variant == 9)
      far_kernel_bulk<Q, LAB><<<blocks, 128, smem, s>>>(a);
    else
      far_kernel_async<Q, LAB, 2><<<blocks, 128, smem5, s>>>(a);
  }
  else
    far_kernel<Q, LAB><<<blocks, 128, 0, s>>>(a);
}

template <bool LAB>
static void launch_far_frame(const FarArgs &a, cudaStream_t s)
{
  switch(a.q) {
    case 1: launch_far_q<1, LAB>(a, s); break;
    case 2: launch_far_q<2, LAB>(a, s); break;
    case 3: launch_far_q<3, LAB>(a, s); break;
    case 4: launch_far_q<4, LAB>(a, s); break;
    case 5: launch_far_q<5, LAB>(a, s); break;
    case 6: launch_far_q<6, LAB>(a, s); break;
    case 7: launch_far_q<7, LAB>(a, s); break;
    default: break;
  }
}

void launch_far(const FarArgs &a, void *stream)
{
  if(a.nT <= 0) return;
  if(a.otf) {
    launch_far_otf(a, stream);
    return;
  }
  if(a.frame == 0)
    launch_far_frame<false>(a, (cudaStream_t)stream);
  else
    launch_far_frame<true>(a, (cudaStream_t)stream);
}

// ---- single-step evaluation without device allocation ----------------------
// Scratch of qg_history_evaluate_noalloc: one file-scope array, carved into
// the group partials, the reduced far field, the tile completion counters and
// two step indices.  Sized for at most kNoAllocMaxDots (padded) dots.
constexpr size_t kNoAllocPartialBytes = sizeof(double2) * kNoAllocMaxGroups * kNoAllocMaxDots;
constexpr size_t kNoAllocFieldBytes = sizeof(double2) * kNoAllocMaxDots;
constexpr size_t kNoAllocTileBytes = 256 * ((sizeof(unsigned) * kNoAllocMaxTiles + 255) / 256);
constexpr size_t kNoAllocScratchBytes = kNoAllocPartialBytes + kNoAllocFieldBytes + kNoAllocTileBytes + 256;
static_assert(kNoAllocScratchBytes == kNoAllocScratchTotal, "scratch size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch on the current device.  In host code the
// symbol is only a stand-in; the address comes from cudaGetSymbolAddress,
// looked up once per device (the first call on a device does it, so that
// call must precede any stream capture).
qg_status noalloc_scratch(NoAllocScratch *out)
{
  static std::mutex mu;
  static void *addr[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e != cudaSuccess) return qg_fail(QG_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  if(dev < 0 || dev >= 64) return qg_fail(QG_ERR_UNSUPPORTED, "device index %d beyond 63", dev);
  void *p = nullptr;
  {
    std::lock_guard<std::mutex> lock(mu);
    if(!addr[dev]) {
      e = cudaGetSymbolAddress(&addr[dev], g_noalloc_scratch);
      if(e != cudaSuccess) {
        addr[dev] = nullptr;
        return qg_fail(QG_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s",
                       cudaGetErrorString(e));
      }
    }
    p = addr[dev];
  }
  unsigned char *b = (unsigned char *)p;
  out->partial = (double2 *)b;
  out->field = (double2 *)(b + kNoAllocPartialBytes);
  out->tile_done = (unsigned *)(b + kNoAllocPartialBytes + kNoAllocFieldBytes);
  out->ints = (int *)(b + kNoAllocPartialBytes + kNoAllocFieldBytes + kNoAllocTileBytes);
  out->tile_bytes = kNoAllocTileBytes;
  return QG_OK;
}

template <int Q, bool LAB>
__global__ void __launch_bounds__(128) far_kernel_step1(FarArgs a)
{
  if(a.mixed)
    far_body_mixed<Q, LAB, 1>(a, warp_task());
  else
    far_body<Q, LAB, 0, 1>(a, warp_task());
}

template <bool LAB>
static void launch_far1_frame(const FarArgs &a, cudaStream_t s)
{
  const unsigned blocks = (unsigned)((a.nT * a.nG + 3) / 4);
  switch(a.q) {
    case 1: far_kernel_step1<1, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 2: far_kernel_step1<2, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 3: far_kernel_step1<3, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 4: far_kernel_step1<4, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 5: far_kernel_step1<5, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 6: far_kernel_step1<6, LAB><<<blocks, 128, 0, s>>>(a); break;
    case 7: far_kernel_step1<7, LAB><<<blocks, 128, 0, s>>>(a); break;
    default: break;
  }
}

// The far-pair field of one step (slice 0) into the scratch's field.
void launch_far_step1(const FarArgs &a, void *stream)
{
  if(a.nT <= 0) return;
  if(a.frame == 0)
    launch_far1_frame<false>(a, (cudaStream_t)stream);
  else
    launch_far1_frame<true>(a, (cudaStream_t)stream);
}

}  // namespace qg
