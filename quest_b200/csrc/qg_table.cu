// Coefficient-table build: HistoryInteraction::build_coefficient_table
// (reference src/interactions/history_interaction.cpp:21-45) as one kernel.
//
// Layout in HBM.  Dots are in internal (Morton) order, padded to a multiple
// of kTile = 32.  The table is stored for ordered tile pairs: tile (I, J)
// holds the 32 x 32 pairs with target a = 32 I + l and source b = 32 J + j
// at entry e = 32 j + l, so the 32 lanes of a warp (one per target) read one
// source's entries as one coalesced transaction:
//   delay[I][J][e]          int32 floor delay, -1 when the entry is no pair
//                           (padding, or a == b)
//   coef [I][J][i][e]       double2 coefficient of tap i = 0..q
// Every unordered pair is computed once, in the reference's own orientation
// (src = larger user index, obs = smaller, so its rounding is the
// reference's), and written to both (I, J) and (J, I).  The two copies
// double the table's size; in exchange the far-pair kernel reads windows of
// one source row per warp step instead of 32.
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

template <int Q, bool MIXED>
__global__ void __launch_bounds__(128) table_build_kernel(TableArgs a)
{
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = a.nblk * kTilePairs;
  if(gid >= total) return;
  const long long blk = gid / kTilePairs;
  const int e = (int)(gid % kTilePairs);
  int I, J;
  decode_block(blk, I, J);  // I >= J
  const int la = e / kTile, lb = e % kTile;
  if(I == J && la < lb) return;  // written by the (lb, la) thread
  const int ia = I * kTile + la, ib = J * kTile + lb;
  const long long T1 = (long long)I * a.nT + J, T2 = (long long)J * a.nT + I;
  const int e1 = lb * kTile + la;  // in (I, J): target a, source b
  const int e2 = la * kTile + lb;  // in (J, I): target b, source a
  int *d1 = a.delay + T1 * kTilePairs + e1, *d2 = a.delay + T2 * kTilePairs + e2;
  // FP64: q+1 taps; mixed: q+1 taps and their sum, in FP32
  double2 *c1 = a.coef + T1 * (Q + 1) * kTilePairs + e1;
  double2 *c2 = a.coef + T2 * (Q + 1) * kTilePairs + e2;
  float2 *f1 = a.coef32 + T1 * (Q + 2) * kTilePairs + e1;
  float2 *f2 = a.coef32 + T2 * (Q + 2) * kTilePairs + e2;
  const bool valid = ia != ib && a.user[ia] >= 0 && a.user[ib] >= 0;
  if(!valid) {
    *d1 = -1;
    *d2 = -1;
    if(MIXED) {
#pragma unroll
      for(int i = 0; i <= Q + 1; ++i) f1[(long long)i * kTilePairs] = f2[(long long)i * kTilePairs] = make_float2(0.f, 0.f);
    } else {
#pragma unroll
      for(int i = 0; i <= Q; ++i) c1[(long long)i * kTilePairs] = c2[(long long)i * kTilePairs] = make_double2(0.0, 0.0);
    }
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
  *d1 = fd;
  *d2 = fd;
  if(MIXED) {
    double2 sum = make_double2(0.0, 0.0);
#pragma unroll
    for(int i = 0; i <= Q; ++i) {
      const float2 v = make_float2((float)coef[i].x, (float)coef[i].y);
      f1[(long long)i * kTilePairs] = f2[(long long)i * kTilePairs] = v;
      sum.x += coef[i].x;
      sum.y += coef[i].y;
    }
    f1[(long long)(Q + 1) * kTilePairs] = f2[(long long)(Q + 1) * kTilePairs] = make_float2((float)sum.x, (float)sum.y);
  } else {
#pragma unroll
    for(int i = 0; i <= Q; ++i) c1[(long long)i * kTilePairs] = c2[(long long)i * kTilePairs] = coef[i];
  }
  atomicMax(a.max_delay, fd);
  if(fd == 0) atomicAdd(a.near_count, 1ULL);
  if(fd < kTimeBlock) atomicAdd(a.near_count + 1, 1ULL);
  if(fd >= kTimeBlock) {
    // far pairs with a non-finite coefficient (an integer delay): the far
    // kernels' first-blocks form is not used for such a table
    bool fin = true;
#pragma unroll
    for(int i = 0; i <= Q; ++i) fin = fin && isfinite(coef[i].x) && isfinite(coef[i].y);
    if(!fin) atomicAdd(a.near_count + 3, 1ULL);
  }
}

template <bool MIXED>
static void launch_table_build_p(const TableArgs &a, int q, cudaStream_t s)
{
  const long long total = a.nblk * kTilePairs;
  const int threads = 128;
  const unsigned blocks = (unsigned)((total + threads - 1) / threads);
  switch(q) {
    case 1: table_build_kernel<1, MIXED><<<blocks, threads, 0, s>>>(a); break;
    case 2: table_build_kernel<2, MIXED><<<blocks, threads, 0, s>>>(a); break;
    case 3: table_build_kernel<3, MIXED><<<blocks, threads, 0, s>>>(a); break;
    case 4: table_build_kernel<4, MIXED><<<blocks, threads, 0, s>>>(a); break;
    case 5: table_build_kernel<5, MIXED><<<blocks, threads, 0, s>>>(a); break;
    case 6: table_build_kernel<6, MIXED><<<blocks, threads, 0, s>>>(a); break;
    case 7: table_build_kernel<7, MIXED><<<blocks, threads, 0, s>>>(a); break;
    default: break;
  }
}

void launch_table_build(const TableArgs &a, int q, void *stream)
{
  if(a.mixed)
    launch_table_build_p<true>(a, q, (cudaStream_t)stream);
  else
    launch_table_build_p<false>(a, q, (cudaStream_t)stream);
}

// Pairs with floor delay below `below`: 1 finds the delay-0 pairs before
// the table exists, so the dot order can put every group coupled at delay 0
// inside one 32-dot step block; kTimeBlock finds the mid-list pairs.  The
// delay is computed with exactly the operations of pair_coef_ref (reference
// orientation, norm, division, modf), so it agrees with the table.
__global__ void near_find_kernel(const double *pos, const int *user, int n_pad, double c0dt, int below,
                                 int *out_pairs, unsigned long long *counter, unsigned long long cap)
{
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nt = (n_pad + kTile - 1) / kTile;
  const long long nblk = nt * (nt + 1) / 2;
  if(gid >= nblk * kTilePairs) return;
  int I, J;
  decode_block(gid / kTilePairs, I, J);
  const int e = (int)(gid % kTilePairs);
  const int la = e / kTile, lb = e % kTile;
  if(I == J && la <= lb) return;
  const int ia = I * kTile + la, ib = J * kTile + lb;
  if(ia >= n_pad || ib >= n_pad) return;
  const int ua = user[ia], ub = user[ib];
  if(ua < 0 || ub < 0) return;
  const int is = ua > ub ? ia : ib, io = ua > ub ? ib : ia;
  double dr[3];
#pragma unroll
  for(int k = 0; k < 3; ++k) dr[k] = pos[3 * io + k] - pos[3 * is + k];
  const double nrm = sqrt((dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2]);
  double idelay;
  modf(nrm / c0dt, &idelay);
  if((int)idelay >= below) return;
  const unsigned long long slot = atomicAdd(counter, 1ULL);
  if(slot >= cap) return;
  out_pairs[3 * slot] = ia;
  out_pairs[3 * slot + 1] = ib;
  out_pairs[3 * slot + 2] = (int)idelay;
}

// The largest floor delay over all pairs (for the ring depth when no table
// is built), with the delay arithmetic of pair_coef_ref.
__global__ void __launch_bounds__(256) max_delay_kernel(const double *pos, const int *user, int n_pad, double c0dt,
                                                        int *out)
{
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nt = (n_pad + kTile - 1) / kTile;
  const long long nblk = nt * (nt + 1) / 2;
  int v = -1;
  if(gid < nblk * kTilePairs) {
    int I, J;
    decode_block(gid / kTilePairs, I, J);
    const int e = (int)(gid % kTilePairs);
    const int la = e / kTile, lb = e % kTile;
    const int ia = I * kTile + la, ib = J * kTile + lb;
    if(!(I == J && la <= lb) && ia < n_pad && ib < n_pad && user[ia] >= 0 && user[ib] >= 0) {
      const int ua = user[ia], ub = user[ib];
      const int is = ua > ub ? ia : ib, io = ua > ub ? ib : ia;
      double dr[3];
#pragma unroll
      for(int k = 0; k < 3; ++k) dr[k] = pos[3 * io + k] - pos[3 * is + k];
      const double nrm = sqrt((dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2]);
      double idelay;
      modf(nrm / c0dt, &idelay);
      v = (int)idelay;
    }
  }
  v = __reduce_max_sync(0xffffffffu, v);
  if((threadIdx.x & 31) == 0 && v >= 0) atomicMax(out, v);
}

void launch_max_delay(const double *pos, const int *user, int n_pad, double c0dt, int *max_delay, void *stream)
{
  const long long nt = (n_pad + kTile - 1) / kTile;
  const long long total = nt * (nt + 1) / 2 * kTilePairs;
  const unsigned blocks = (unsigned)((total + 255) / 256);
  max_delay_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(pos, user, n_pad, c0dt, max_delay);
}

// FP64 coefficients of listed pairs (the per-step mid list), computed as the
// table build computes them.
template <int Q>
__global__ void pair_list_coef_kernel(TableArgs a, const int *pairs, long long m, double2 *out)
{
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if(k >= m) return;
  const int ia = pairs[3 * k], ib = pairs[3 * k + 1];
  const int ua = a.user[ia], ub = a.user[ib];
  const int is = ua > ub ? ia : ib, io = ua > ub ? ib : ia;
  double ps[3], po[3], ds[3], dob[3];
#pragma unroll
  for(int c = 0; c < 3; ++c) {
    ps[c] = a.pos[3 * is + c];
    po[c] = a.pos[3 * io + c];
    ds[c] = a.dip[3 * is + c];
    dob[c] = a.dip[3 * io + c];
  }
  double2 coef[Q + 1];
  pair_coef_ref<Q>(ps, po, ds, dob, a.cp, coef);
#pragma unroll
  for(int i = 0; i <= Q; ++i) out[k * (Q + 1) + i] = coef[i];
}

// dst row j (width values) = src row rows[j]: the mid list's coefficients
// placed in list order on the device, from the pair-order array
__global__ void gather_rows_kernel(const double2 *__restrict__ src, const long long *__restrict__ rows, int width,
                                   long long n, double2 *__restrict__ dst)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n * width) return;
  const long long j = i / width;
  dst[i] = src[rows[j] * width + (i - j * width)];
}

void launch_gather_rows(const double2 *src, const long long *rows, int width, long long n, double2 *dst,
                        void *stream)
{
  const long long total = n * width;
  if(total <= 0) return;
  gather_rows_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(src, rows, width, n, dst);
}

void launch_pair_list_coef(const TableArgs &a, int q, const int *pairs, long long m, double2 *out, void *stream)
{
  if(m <= 0) return;
  const unsigned blocks = (unsigned)((m + 127) / 128);
  cudaStream_t s = (cudaStream_t)stream;
  switch(q) {
    case 1: pair_list_coef_kernel<1><<<blocks, 128, 0, s>>>(a, pairs, m, out); break;
    case 2: pair_list_coef_kernel<2><<<blocks, 128, 0, s>>>(a, pairs, m, out); break;
    case 3: pair_list_coef_kernel<3><<<blocks, 128, 0, s>>>(a, pairs, m, out); break;
    case 4: pair_list_coef_kernel<4><<<blocks, 128, 0, s>>>(a, pairs, m, out); break;
    case 5: pair_list_coef_kernel<5><<<blocks, 128, 0, s>>>(a, pairs, m, out); break;
    case 6: pair_list_coef_kernel<6><<<blocks, 128, 0, s>>>(a, pairs, m, out); break;
    case 7: pair_list_coef_kernel<7><<<blocks, 128, 0, s>>>(a, pairs, m, out); break;
    default: break;
  }
}

void launch_near_find(const double *pos, const int *user, int n_pad, double c0dt, int below, int *out_pairs,
                      unsigned long long *counter, unsigned long long cap, void *stream)
{
  const long long nt = (n_pad + kTile - 1) / kTile;
  const long long total = nt * (nt + 1) / 2 * kTilePairs;
  const int threads = 256;
  near_find_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, (cudaStream_t)stream>>>(
      pos, user, n_pad, c0dt, below, out_pairs, counter, cap);
}

}  // namespace qg
