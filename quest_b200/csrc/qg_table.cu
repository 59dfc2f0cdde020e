// Coefficient-table build: HistoryInteraction::build_coefficient_table
// (reference src/interactions/history_interaction.cpp:21-45) as one kernel.
//
// Layout in HBM.  Dots are in internal (Morton) order, padded to a multiple
// of kTile = 32.  The unordered pairs are grouped into tile blocks (I, J),
// I >= J, numbered blk = I(I+1)/2 + J.  Block blk holds kTilePairs = 1024
// entries in diagonal-major order: entry e = 32 j + l is the pair of dot
// a = 32 I + l and dot b = 32 J + ((l + j) mod 32), so at step j of the
// far-pair kernel lane l of a warp reads entry 32 j + l:
//   delay[blk][e]          int32 floor delay, -1 when the entry is no pair
//                          (padding, or b >= a on a diagonal block)
//   coef [blk][i][e]       double2 coefficient of tap i = 0..q
// A warp reading one tap of one diagonal is one 512-byte transaction.  Each
// pair is computed in the reference's own orientation (src = larger user
// index, obs = smaller) so its rounding is the reference's.
//
// Compiled with -fmad=false.
#include <cuda_runtime.h>

#include "qg_coef.cuh"

namespace qg {

__device__ __forceinline__ void decode_block(long long blk, int &I, int &J)
{
  long long r = (long long)((sqrt(8.0 * (double)blk + 1.0) - 1.0) * 0.5);
  while(r * (r + 1) / 2 > blk) --r;
  while((r + 1) * (r + 2) / 2 <= blk) ++r;
  I = (int)r;
  J = (int)(blk - r * (r + 1) / 2);
}

template <int Q>
__global__ void __launch_bounds__(128) table_build_kernel(TableArgs a)
{
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = a.nblk * kTilePairs;
  if(gid >= total) return;
  const long long blk = gid / kTilePairs;
  const int e = (int)(gid % kTilePairs);
  int I, J;
  decode_block(blk, I, J);
  const int la = e % kTile, lb = (la + e / kTile) % kTile;
  const int ia = I * kTile + la, ib = J * kTile + lb;
  int *dptr = a.delay + blk * kTilePairs + e;
  double2 *cptr = a.coef + blk * (long long)(Q + 1) * kTilePairs + e;
  const bool valid = ia < a.n && ib < a.n && !(I == J && lb >= la);
  if(!valid) {
    *dptr = -1;
#pragma unroll
    for(int i = 0; i <= Q; ++i) cptr[(long long)i * kTilePairs] = make_double2(0.0, 0.0);
    return;
  }
  // reference orientation: src = row = larger user index, obs = col
  const int ua = a.user[ia], ub = a.user[ib];
  const int is = ua > ub ? ia : ib;
  const int io = ua > ub ? ib : ia;
  double ps[3], po[3], ds[3], dob[3];
#pragma unroll
  for(int k = 0; k < 3; ++k) {
    ps[k] = a.pos[3 * is + k];
    po[k] = a.pos[3 * io + k];
    ds[k] = a.dip[3 * is + k];
    dob[k] = a.dip[3 * io + k];
  }
  double2 coef[Q + 1];
  const int fd = pair_coef_ref<Q>(ps, po, ds, dob, a.cp, coef);
  *dptr = fd;
#pragma unroll
  for(int i = 0; i <= Q; ++i) cptr[(long long)i * kTilePairs] = coef[i];
  atomicMax(a.max_delay, fd);
  if(fd == 0) atomicAdd(a.near_count, 1ULL);
  if(fd < kTimeBlock) atomicAdd(a.near_count + 1, 1ULL);
}

void launch_table_build(const TableArgs &a, int q, void *stream)
{
  const long long total = a.nblk * kTilePairs;
  const int threads = 128;
  const unsigned blocks = (unsigned)((total + threads - 1) / threads);
  cudaStream_t s = (cudaStream_t)stream;
  switch(q) {
    case 1: table_build_kernel<1><<<blocks, threads, 0, s>>>(a); break;
    case 2: table_build_kernel<2><<<blocks, threads, 0, s>>>(a); break;
    case 3: table_build_kernel<3><<<blocks, threads, 0, s>>>(a); break;
    case 4: table_build_kernel<4><<<blocks, threads, 0, s>>>(a); break;
    case 5: table_build_kernel<5><<<blocks, threads, 0, s>>>(a); break;
    case 6: table_build_kernel<6><<<blocks, threads, 0, s>>>(a); break;
    case 7: table_build_kernel<7><<<blocks, threads, 0, s>>>(a); break;
    default: break;
  }
}

// Compacts the pairs with floor delay < K (the ones the far-pair kernel
// leaves to the per-step kernels) into (a, b, delay) + q+1 coefficients; the
// host sorts them.
__global__ void mid_extract_kernel(const int *delay, const double2 *coef, long long nblk, int q,
                                   int *out_pairs, double2 *out_coef, unsigned long long *counter,
                                   unsigned long long cap)
{
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if(gid >= nblk * kTilePairs) return;
  const int d = delay[gid];
  if(d < 0 || d >= kTimeBlock) return;
  const long long blk = gid / kTilePairs;
  const int e = (int)(gid % kTilePairs);
  int I, J;
  decode_block(blk, I, J);
  const unsigned long long slot = atomicAdd(counter, 1ULL);
  if(slot >= cap) return;
  const int la = e % kTile, lb = (la + e / kTile) % kTile;
  out_pairs[3 * slot] = I * kTile + la;
  out_pairs[3 * slot + 1] = J * kTile + lb;
  out_pairs[3 * slot + 2] = d;
  for(int i = 0; i <= q; ++i)
    out_coef[slot * (q + 1) + i] = coef[blk * (long long)(q + 1) * kTilePairs + (long long)i * kTilePairs + e];
}

void launch_mid_extract(const int *delay, const double2 *coef, long long nblk, int q, int *out_pairs,
                        double2 *out_coef, unsigned long long *counter, unsigned long long cap,
                        void *stream)
{
  const long long total = nblk * kTilePairs;
  const int threads = 256;
  const unsigned blocks = (unsigned)((total + threads - 1) / threads);
  mid_extract_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(delay, coef, nblk, q, out_pairs,
                                                                   out_coef, counter, cap);
}

}  // namespace qg
