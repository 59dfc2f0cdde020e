// Internal declarations shared by the library's translation units.
#pragma once

#include <cstddef>
#include <cstdint>

#include <vector_types.h>  // double2

#include "../../include/quest_gpu.h"

// Records the message for qg_last_error() on this thread and returns code.
qg_status qg_fail(qg_status code, const char *fmt, ...);

namespace qg {

constexpr int kWindow = 22;      // History's negative-time extent (main.cpp:30)
constexpr int kCorrectorSteps = 10;  // NUM_CORRECTOR_STEPS (integrator.cpp:3)
constexpr int kMaxOrder = 7;     // largest interpolation order built
constexpr int kTimeBlock = 16;   // K: steps per pass of the far-pair kernel
constexpr int kRingMirror = 24;  // slots mirrored past the ring end (>= K+q)
constexpr int kTile = 32;        // dots per table tile (a warp's 32 targets)
constexpr int kTilePairs = kTile * kTile;
constexpr int kTileGroup = 4;    // source tiles one warp sums before writing
constexpr int kPcDepth = 23;     // PC ring: 22 past steps + the current one
constexpr int kStepBlock = 128;  // threads per block of the dot-step kernel
constexpr int kBadNone = 0x7fffffff;

// Weights as passed to kernels (copy of qg_weights).
struct PCW {
  int n_time;
  double ps[64];
  double cs[64];
  double fc;
};

// Per-pair physics constants for coefficient kernels.
struct CoefParams {
  double c0, dt, mu0, hbar, omega;
  int q;
  int frame;
};

struct PulseParams {
  double amp_pol[3];  // (amplitude / 2) * polarisation_k
  double k[3];        // wavevector
  double freq, delay, width;
};

// Arguments of the table-build kernel.
struct TableArgs {
  const double *pos;   // [n_pad][3] internal order
  const double *dip;   // [n_pad][3]
  const int *user;     // internal -> user index, -1 for padding
  int n, n_pad, nT;
  long long nblk;
  int *delay;          // [nT][nT][kTilePairs]
  double2 *coef;       // FP64: [nT][nT][q+1][kTilePairs]
  float2 *coef32;      // mixed: [nT][nT][q+2][kTilePairs] (taps, then their sum)
  int mixed;
  int *max_delay;      // atomicMax
  // [0] pairs with delay 0, [1] pairs with delay < K, [3] pairs with delay
  // >= K and a non-finite coefficient ([2] is the list builder's counter)
  unsigned long long *near_count;
  CoefParams cp;
};

// Arguments of the far-pair kernel: K steps of the pair sum for every pair
// with floor delay >= K, from one pass over the table.
struct FarArgs {
  const int *delay;     // [nT][nT][kTilePairs] ordered tile pairs
  const double2 *coef;  // [nT][nT][q+1][kTilePairs]
  const double2 *ring;  // [n_pad][stride]: rho01 by time slot
  // mixed precision: FP32 table with the tap sum after the taps, and FP32
  // rings of rho01 and of its step-to-step differences (computed in FP64)
  const float2 *coef32;
  const float2 *ring32w;
  const float2 *ring32d;
  int mixed;
  double2 *partial;     // [K][nG][n_pad] per source-tile group
  double2 *field;       // [K][n_pad] far-pair field
  unsigned *tile_done;  // [nT] completion counters (zero between launches)
  int n_pad, nT, nG, W, stride, q, frame;
  const int *d_t0;      // first step of the block
  int *far_t0_out;      // receives *d_t0 (read by the dot-step kernels)
  int variant;          // kernel variant (same results), see qg_far.cu
  // task order: 0 target-tile major (a block's warps take consecutive source
  // groups of one target tile), 1 source-group major (they take one source
  // group of consecutive target tiles, so they read the same history rows);
  // the same sums either way
  int gmajor;
  int *d_bad;           // a far-kernel wait that ran out sets it to -3
  // 1: some windows may start before step -22 (the first blocks of a run)
  // and every far pair's coefficients are finite; the FP64 table launch then
  // takes the first-blocks form whatever the variant (same results)
  int early;
  // on-the-fly coefficients (no table): dot data, constants, and the source
  // tiles per warp (nG = ceil(nT / group) groups)
  int otf;
  int group;
  const double *pos;    // [n_pad][3]
  const double *dip;    // [n_pad][3]
  const int *user;      // internal -> user index, -1 for padding
  CoefParams cp;
  // target tiles [tile_lo, tile_lo + tile_n) only (a shard of a sharded
  // handle; on-the-fly kernel); tile_n == 0: all nT
  int tile_lo, tile_n;
};

// Arguments of the per-dot step kernels.
struct StepArgs {
  int n, n_pad, nT, W, stride, q, frame;
  int T;                 // num_timesteps: steps at or past T are not computed
  double dt, laser_freq, hbar;
  PulseParams pulse;
  const double *pos;     // [n_pad][3] internal order
  const double *dip;     // [n_pad][3]
  const double *freq, *t1, *t2;
  const int *user;       // internal -> user index, -1 for padding
  const double2 *far_field;  // [K][n_pad] far-pair field of the current block
  const int *far_t0;     // first step of the far block far_field holds
  // pairs with floor delay < K (taps not covered by the far kernel): CSR by
  // internal index, partner, delay and q+1 coefficients
  const int *mid_ptr;
  const int *mid_idx;
  const int *mid_delay;
  const double2 *mid_coef;  // [entry][q+1]
  // the mid-list taps that read step t-1 (delay 1 tap 0, delay 0 tap 1): CSR
  // by internal index, partner (internal index) and coefficient; lag = 1 when
  // every such partner is in the dot's own 32-dot block
  const int *new_ptr;
  const int *new_idx;
  const double2 *new_coef;
  int lag;
  int mid_cache;  // step-block kernel: mid-list entries a block keeps in shared memory
  // step-block kernel partner history: per 32-dot block its distinct mid-list
  // partners (CSR by block, internal indices), each entry's partner as an
  // index into its block's list, and the partners a block can hold (0: off)
  const int *bp_ptr;
  const int *bp_idx;
  const int *mid_pj;
  int hist_cap;
  // step-block kernel: per 32-dot block, the blocks holding its mid-list
  // partners, itself included (CSR by block)
  const int *pb_ptr;
  const int *pb_idx;
  double2 *pcr;          // [kPcDepth][4][n_pad]
  double2 *ring;         // [n_pad][stride] rho01 by step slot
  float2 *ring32w;       // mixed: FP32 rho01 by slot (null in FP64)
  float2 *ring32d;       // mixed: FP32 rho01(t) - rho01(t-1), differences in FP64
  // current-step coupling: CSR by slot (fused: partner = local slot in the
  // block; general: partner = internal index)
  const int *near_ptr;
  const int *near_idx;
  const double2 *near_coef;
  // general path scratch
  double2 *scratch;      // [n_pad][8]: past field, pulse, H (2 complex), cur rho x2
  double2 *traj;         // [k][n][2] user order or null
  int traj_rows;         // rows allocated in traj
  const int *traj_t0;
  int *d_next;           // first step of the next far block (set by the last
                         // step kernel of a block, read by the far kernel)
  int *d_bad;
  // step-block kernel: polls per wait on a partner block before it gives up
  // (0: the default, about a second), and a block that never posts its steps
  // (-1: none; set only by failure-detection tests, so that waits run out)
  int spin_limit;
  int skip_post_block;
  int blk_lo;  // first 32-dot block of the per-step launch (a shard's range)
  PCW w;
};

// Scratch of the allocation-free evaluation (qg_history_evaluate_noalloc):
// a static device array in qg_far.cu, at most kNoAllocMaxDots padded dots.
constexpr int kNoAllocMaxDots = 4096;
constexpr int kNoAllocMaxTiles = kNoAllocMaxDots / kTile;
constexpr int kNoAllocMaxGroups = (kNoAllocMaxTiles + kTileGroup - 1) / kTileGroup;
constexpr size_t kNoAllocScratchTotal = 16ull * kNoAllocMaxGroups * kNoAllocMaxDots + 16ull * kNoAllocMaxDots +
                                        256 * ((4ull * kNoAllocMaxTiles + 255) / 256) + 256;
struct NoAllocScratch {
  double2 *partial;    // [kNoAllocMaxGroups][n_pad]
  double2 *field;      // [n_pad]
  unsigned *tile_done; // [nT]
  int *ints;           // [0] step, [1] far_t0 written by the kernel
  size_t tile_bytes;
};
qg_status noalloc_scratch(NoAllocScratch *out);
void launch_far_step1(const FarArgs &a, void *stream);
// mixed: 0 FP64 members, 1 mixed (scalar FP32 convolution), 2 mixed (packed
// FP32 pairs; the same bits as 1)
void launch_far_batch(const FarArgs *args, const int *task_off, int n_ens, int q, int frame, int mixed,
                      int grid, void *stream);
void launch_ring32_rebuild(const StepArgs &a, void *stream);
// Sharded handles: a shard's rho01 at step t for internal dots [lo, hi)
// into out[0 .. hi-lo), and the other dots' rho01 at step t from the full
// internal-order vector into the rings (as the step kernel writes its own)
void launch_shard_export(const StepArgs &a, int t, int lo, int hi, double2 *out, void *stream);
void launch_shard_import(const StepArgs &a, int t, int lo, int hi, const double2 *full, void *stream);
// out[e] = *args[e].d_bad for the n members of a batch
void launch_gather_bad(const StepArgs *args, int n, int *out, void *stream);
// The step-block kernel's per-block step counts, one per 128-byte line (so
// the polls on one block's count do not queue behind those on another's).
constexpr int kFlagStride = 32;
void launch_step_block(const StepArgs &a, int k0, int k1, int nblocks, unsigned *flags, void *stream);
int step_block_max_blocks(int q, int mid_cache, int hist_cap);
// pipe: the mid list staged with several entries' loads in flight (same sums)
void launch_step_batch(const StepArgs *args, const int *block_off, int n_ens, int total_blocks, int n_time,
                       int k, bool pipe, void *stream);

// Launchers (defined in the .cu files).
void launch_table_build(const TableArgs &a, int q, void *stream);
void launch_far(const FarArgs &a, void *stream);
void launch_far_otf(const FarArgs &a, void *stream);
void launch_max_delay(const double *pos, const int *user, int n_pad, double c0dt, int *max_delay, void *stream);
void launch_near_find(const double *pos, const int *user, int n_pad, double c0dt, int below, int *out_pairs,
                      unsigned long long *counter, unsigned long long cap, void *stream);
void launch_pair_list_coef(const TableArgs &a, int q, const int *pairs, long long m, double2 *out, void *stream);
// dst[j][0 .. width) = src[rows[j]][0 .. width), j < n
void launch_gather_rows(const double2 *src, const long long *rows, int width, long long n, double2 *dst,
                        void *stream);
void launch_step_fused(const StepArgs &a, int k, int nblocks, void *stream);
void launch_step_general(const StepArgs &a, int k, int phase, void *stream);
void launch_eval_field(const StepArgs &a, const int *d_eval_step, double2 *out_user, void *stream);
void launch_pulse_field(const StepArgs &a, int step, double2 *out_user, void *stream);
void launch_set_int(int *p, int v, void *stream);
void launch_init_state(const StepArgs &a, void *stream);
void launch_ring_write(const StepArgs &a, int t, const double2 *rho01_user, void *stream);
void launch_ring_read(const StepArgs &a, int t, double2 *rho01_user, void *stream);
void launch_state_read(const StepArgs &a, int t, double2 *rho_user, void *stream);

}  // namespace qg
