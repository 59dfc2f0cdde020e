// C ABI of the library: handle lifetime, device memory, the step loop.
//
// A handle corresponds to the objects the reference's main() builds
// (src/main.cpp:25-52): the dots, the History array, the PulseInteraction,
// the HistoryInteraction with its coefficient table, and the
// PredictorCorrector::Integrator.  Device memory is allocated once in
// qg_create and released in qg_destroy.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "qg_internal.h"

using namespace qg;

static thread_local std::string g_last_error;

qg_status qg_fail(qg_status code, const char *fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

extern "C" const char *qg_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *qg_version(void) { return "quest_b200 0.1 (sm_100a)"; }

#define QG_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t err_ = (call);                                                               \
    if(err_ != cudaSuccess) {                                                                \
      qg_status code_ = (err_ == cudaErrorMemoryAllocation) ? QG_ERR_OOM : QG_ERR_CUDA;      \
      return qg_fail(code_, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_),        \
                     __FILE__, __LINE__);                                                    \
    }                                                                                        \
  } while(0)

// The on-the-fly far kernel's form: source-group-major tasks, held to 3
// blocks per SM (qg_otf.cu variant 8).
constexpr int kOtfVariant = 8;

struct qg_handle_s {
  int n = 0, n_pad = 0, nT = 0, q = 0, T = 0;
  long long nblk = 0, P = 0;
  qg_params params{};
  qg_pulse pulse{};
  PCW w{};
  int device = 0;
  cudaStream_t stream = nullptr, copy_stream = nullptr;

  std::vector<void *> allocs;
  size_t bytes = 0;

  double *d_pos = nullptr, *d_dip = nullptr, *d_freq = nullptr, *d_t1 = nullptr, *d_t2 = nullptr;
  int *d_user = nullptr;
  int *d_delay = nullptr;
  double2 *d_coef = nullptr;
  float2 *d_coef32 = nullptr;              // mixed precision table
  float2 *d_ring32w = nullptr, *d_ring32d = nullptr;
  bool mixed = false;
  bool otf = false;  // coefficients computed in the far kernel (no table)
  int group = kTileGroup;  // source tiles per far-kernel warp
  int max_groups = 0;      // source groups the partial buffer holds
  double2 *d_ring = nullptr;
  int W = 0, stride = 0;
  double2 *d_pcr = nullptr, *d_partial = nullptr, *d_field = nullptr, *d_scratch = nullptr;
  unsigned *d_tile_done = nullptr;
  int nG = 0;
  int *d_fnear_ptr = nullptr, *d_fnear_idx = nullptr;  // fused: by slot, local partner
  double2 *d_fnear_coef = nullptr;
  int *d_gnear_ptr = nullptr, *d_gnear_idx = nullptr;  // general: by internal index
  double2 *d_gnear_coef = nullptr;
  int *d_mid_ptr = nullptr, *d_mid_idx = nullptr, *d_mid_delay = nullptr;  // delay < K pairs
  double2 *d_mid_coef = nullptr;
  int *d_new_ptr = nullptr, *d_new_idx = nullptr;  // taps reading step t-1
  double2 *d_new_coef = nullptr;
  bool lag = false;  // every delay-0/1 partner shares the dot's 32-dot block
  // d_ints: 0 step, 1 done, 2 bad, 3 traj_t0, 4 eval_step, 5 max_delay,
  //         6 far_t0 (run), 7 far block start request, 8 far_t0 (evaluate)
  int *d_ints = nullptr;
  unsigned long long *d_u64 = nullptr;
  double2 *d_traj = nullptr;  // 2 * traj_k steps x N x 2
  int traj_k = 0;
  double2 *d_io = nullptr;    // N complex device staging for evaluate / set_history
  double2 *h_io = nullptr;    // pinned N complex, made at the first evaluate / history copy

  bool fused = true;
  int step_blocks = 0;
  // all 16 steps of a block in one cooperative launch (fused form, every
  // 32-dot block resident at once); otherwise one launch per step
  bool block_step = false, block_step_ok = false;
  int mid_cache = 0;  // mid-list entries per block kept in shared memory by that kernel
  int hist_cap = 0;   // distinct partners per block whose history that kernel keeps
  int *d_bp_ptr = nullptr, *d_bp_idx = nullptr, *d_mid_pj = nullptr;
  int *d_pb_ptr = nullptr, *d_pb_idx = nullptr;
  unsigned *d_flags = nullptr;  // the step-block kernel's per-block step counts
  int max_delay = 0;
  long long near_pairs = 0, mid_pairs = 0;
  int far_block = -0x7fffffff;  // first step of the far block the partials hold
  double table_ms = 0;
  int next_step = 0;
  int eval_cached = -0x7fffffff;

  // K-step block graphs, [traj off, traj on] + 2 for blocks whose far launch
  // takes its first-blocks form (some windows start before step -22)
  cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
  // profiling in graph mode: kProfRing instances of the block graph, each
  // with its own events around the far kernel and around the K step kernels;
  // an instance's times are collected when it is reused, so the stream stays full
  static constexpr int kProfRing = 8;
  cudaGraphExec_t gprof[4][kProfRing] = {};
  cudaEvent_t pev[kProfRing][3];
  bool pev_ready = false, pending[kProfRing] = {};
  int prof_next = 0;
  bool use_graph = true;
  int far_variant = 3;  // cp.async-staged table (see qg_far.cu); the autotuner may change it
  float tuned_far_ms = 0;  // far-kernel time of the autotuner's choice
  bool tune_coef = false;  // QG_COEF_TUNED: also time the on-the-fly kernel against the table
  bool tune_group = false;  // "tune_group": also time source tiles per warp 1, 2, 4, 8
  bool far_early = true;    // "far_early": the far kernels' first-blocks form where it applies
  bool far_nonfinite = false;  // a far pair's table coefficient is not finite (integer delay)
  bool tune_pending = false;  // the far-kernel autotuner runs at the first qg_run
  bool profile = false;
  // first bad step as the last batch run read it (qg_bad_step answers from it
  // without a device copy while valid; any other run invalidates it)
  int batch_bad = kBadNone;
  bool batch_bad_valid = false;
  // target sharding: this handle computes the 32-dot blocks [blk_lo, blk_hi)
  // of the internal order (all of them unless it is a shard)
  int shard_rank = 0, shard_world = 1;
  int blk_lo = 0, blk_hi = 0;
  double2 *d_shard_io = nullptr;  // n_pad complex: a shard's exchange staging
  int spin_limit = 0;       // step-block kernel polls per wait (0: its default, about a second)
  int skip_post = -1;       // failure-detection tests: a block that never posts its steps
  cudaEvent_t ev_a[256], ev_b[256], ev_c[256], ev_d[256];
  bool events_ready = false;
  double pair_ms = 0, step_ms = 0;
  int pair_launches = 0, step_launches = 0;
  cudaEvent_t ev_chunk[2] = {nullptr, nullptr}, ev_copy[2] = {nullptr, nullptr};

  FarArgs far_args(const int *d_t0, int *far_t0_out) const
  {
    FarArgs s{};
    s.delay = d_delay;
    s.coef = d_coef;
    s.coef32 = d_coef32;
    s.ring32w = d_ring32w;
    s.ring32d = d_ring32d;
    s.mixed = mixed ? 1 : 0;
    s.ring = d_ring;
    s.partial = d_partial;
    s.field = d_field;
    s.tile_done = d_tile_done;
    s.n_pad = n_pad;
    s.nT = nT;
    s.nG = nG;
    s.W = W;
    s.stride = stride;
    s.q = q;
    s.frame = params.frame;
    s.d_t0 = d_t0;
    s.far_t0_out = far_t0_out;
    s.variant = far_variant;
    s.gmajor = 0;
    s.d_bad = d_ints + 2;
    s.otf = otf ? 1 : 0;
    s.group = group;
    s.pos = d_pos;
    s.dip = d_dip;
    s.user = d_user;
    s.cp.c0 = params.c0;
    s.cp.dt = params.dt;
    s.cp.mu0 = params.mu0;
    s.cp.hbar = params.hbar;
    s.cp.omega = params.laser_frequency;
    s.cp.q = q;
    s.cp.frame = params.frame;
    s.tile_lo = shard_world > 1 ? blk_lo : 0;  // 32-dot blocks are the 32-dot target tiles
    s.tile_n = shard_world > 1 ? blk_hi - blk_lo : 0;
    return s;
  }

  StepArgs step_args(bool general) const
  {
    StepArgs a{};
    a.n = n;
    a.n_pad = n_pad;
    a.nT = nT;
    a.T = T;
    a.W = W;
    a.stride = stride;
    a.q = q;
    a.frame = params.frame;
    a.dt = params.dt;
    a.laser_freq = params.laser_frequency;
    a.hbar = params.hbar;
    for(int k = 0; k < 3; ++k) {
      a.pulse.amp_pol[k] = pulse.amplitude / 2 * pulse.polarization[k];
      a.pulse.k[k] = pulse.wavevector[k];
    }
    a.pulse.freq = pulse.freq;
    a.pulse.delay = pulse.delay;
    a.pulse.width = pulse.width;
    a.pos = d_pos;
    a.dip = d_dip;
    a.freq = d_freq;
    a.t1 = d_t1;
    a.t2 = d_t2;
    a.user = d_user;
    a.far_field = d_field;
    a.far_t0 = d_ints + 6;
    a.mid_ptr = d_mid_ptr;
    a.mid_idx = d_mid_idx;
    a.mid_delay = d_mid_delay;
    a.mid_coef = d_mid_coef;
    a.new_ptr = d_new_ptr;
    a.new_idx = d_new_idx;
    a.new_coef = d_new_coef;
    a.lag = lag ? 1 : 0;
    a.mid_cache = mid_cache;
    a.bp_ptr = d_bp_ptr;
    a.bp_idx = d_bp_idx;
    a.mid_pj = d_mid_pj;
    a.hist_cap = hist_cap;
    a.pb_ptr = d_pb_ptr;
    a.pb_idx = d_pb_idx;
    a.pcr = d_pcr;
    a.ring = d_ring;
    a.ring32w = d_ring32w;
    a.ring32d = d_ring32d;
    a.near_ptr = general ? d_gnear_ptr : d_fnear_ptr;
    a.near_idx = general ? d_gnear_idx : d_fnear_idx;
    a.near_coef = general ? d_gnear_coef : d_fnear_coef;
    a.scratch = d_scratch;
    a.traj = nullptr;
    a.traj_rows = 2 * traj_k;
    a.traj_t0 = d_ints + 3;
    a.d_next = d_ints + 0;
    a.d_bad = d_ints + 2;
    a.spin_limit = spin_limit;
    a.skip_post_block = skip_post;
    a.blk_lo = shard_world > 1 ? blk_lo : 0;
    a.w = w;
    return a;
  }
};

// ---- device memory -------------------------------------------------------------
// Handle buffers come from one stream-ordered pool per device that keeps the
// blocks freed by destroyed handles (up to half the device's memory) for the
// next ones: a service that creates and destroys handles then neither maps
// memory again for each nor synchronises the device on every free, as
// cudaFree does, so freeing a 27 GB table does not stall a batch running on
// another stream.  An allocation the device cannot hold first returns the
// pool's unused blocks and tries again.
static cudaMemPool_t handle_pool(int device)
{
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(device);
  if(it != pools.end()) return it->second;
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  if(cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  unsigned long long keep = total_b / 2;  // cudaMemPoolAttrReleaseThreshold: a 64-bit count
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[device] = pool;
  return pool;
}

// `bytes` from the device's pool on the handle's stream; the stream is
// synchronised so the memory can be used from any stream at once.
static cudaError_t pool_alloc(qg_handle *h, void **ptr, size_t bytes)
{
  cudaMemPool_t pool = handle_pool(h->device);
  if(!pool) return cudaMalloc(ptr, bytes);
  cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, pool, h->stream);
  if(e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    // blocks freed on other streams return to the device once those frees
    // have run
    cudaDeviceSynchronize();
    cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocFromPoolAsync(ptr, bytes, pool, h->stream);
  }
  if(e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return e;
}

// Returns a block to the pool once the handle's stream reaches this point
// (the callers have synchronised every stream that used it).
static void pool_free(qg_handle *h, void *p)
{
  if(!p) return;
  if(handle_pool(h->device))
    cudaFreeAsync(p, h->stream);
  else
    cudaFree(p);
}

template <typename T>
static qg_status dalloc(qg_handle *h, T **p, size_t count)
{
  void *ptr = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = pool_alloc(h, &ptr, bytes);
  if(e != cudaSuccess) {
    cudaGetLastError();
    return qg_fail(e == cudaErrorMemoryAllocation ? QG_ERR_OOM : QG_ERR_CUDA,
                   "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
  }
  h->allocs.push_back(ptr);
  h->bytes += bytes;
  *p = (T *)ptr;
  return QG_OK;
}

#define QG_TRY(expr)                 \
  do {                               \
    qg_status st_ = (expr);          \
    if(st_ != QG_OK) return st_;     \
  } while(0)

static void destroy_handle(qg_handle *h)
{
  if(!h) return;
  if(h->stream) cudaStreamSynchronize(h->stream);
  if(h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  for(auto &g : h->graph)
    if(g) cudaGraphExecDestroy(g);
  for(auto &row : h->gprof)
    for(auto &g : row)
      if(g) cudaGraphExecDestroy(g);
  if(h->pev_ready)
    for(auto &row : h->pev)
      for(auto &e : row) cudaEventDestroy(e);
  if(h->events_ready) {
    for(int i = 0; i < 256; ++i) {
      cudaEventDestroy(h->ev_a[i]);
      cudaEventDestroy(h->ev_b[i]);
      cudaEventDestroy(h->ev_c[i]);
      cudaEventDestroy(h->ev_d[i]);
    }
  }
  for(int i = 0; i < 2; ++i) {
    if(h->ev_chunk[i]) cudaEventDestroy(h->ev_chunk[i]);
    if(h->ev_copy[i]) cudaEventDestroy(h->ev_copy[i]);
  }
  for(void *p : h->allocs) pool_free(h, p);
  if(h->h_io) cudaFreeHost(h->h_io);
  if(h->stream) cudaStreamDestroy(h->stream);
  if(h->copy_stream) cudaStreamDestroy(h->copy_stream);
  delete h;
}

// Morton (Z-order) key of a position quantised to 21 bits per axis.
static inline uint64_t spread3(uint64_t x)
{
  x &= 0x1fffff;
  x = (x | x << 32) & 0x1f00000000ffffULL;
  x = (x | x << 16) & 0x1f0000ff0000ffULL;
  x = (x | x << 8) & 0x100f00f00f00f00fULL;
  x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
  x = (x | x << 2) & 0x1249249249249249ULL;
  return x;
}

static std::vector<int> morton_order(const qg_dot *dots, int n)
{
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for(int i = 0; i < n; ++i)
    for(int k = 0; k < 3; ++k) {
      const double v = dots[i].pos[k];
      if(std::isfinite(v)) {
        lo[k] = std::min(lo[k], v);
        hi[k] = std::max(hi[k], v);
      }
    }
  double ext = 0;
  for(int k = 0; k < 3; ++k)
    if(hi[k] > lo[k]) ext = std::max(ext, hi[k] - lo[k]);
  std::vector<std::pair<uint64_t, int>> keys(n);
  for(int i = 0; i < n; ++i) {
    uint64_t code = 0;
    for(int k = 0; k < 3; ++k) {
      double v = dots[i].pos[k];
      double f = (ext > 0 && std::isfinite(v)) ? (v - lo[k]) / ext : 0.0;
      f = std::min(std::max(f, 0.0), 1.0);
      code |= spread3((uint64_t)(f * 2097151.0)) << k;
    }
    keys[i] = {code, i};
  }
  std::sort(keys.begin(), keys.end());
  std::vector<int> perm(n);
  for(int i = 0; i < n; ++i) perm[i] = keys[i].second;
  return perm;
}

// Union-find over the current-step (delay 0) coupling graph.
struct DSU {
  std::vector<int> p;
  explicit DSU(int n) : p(n) { std::iota(p.begin(), p.end(), 0); }
  int find(int x)
  {
    while(p[x] != x) x = p[x] = p[p[x]];
    return x;
  }
  void unite(int a, int b) { p[find(a)] = find(b); }
};

static qg_status validate(const qg_dot *dots, int n, const qg_pulse *pulse, const qg_params *p)
{
  if(!dots || !pulse || !p) return qg_fail(QG_ERR_INVALID_ARG, "qg_create: NULL argument");
  if(n < 1) return qg_fail(QG_ERR_INVALID_ARG, "qg_create: need at least one dot (n = %d)", n);
  if(n > (1 << 24)) return qg_fail(QG_ERR_INVALID_ARG, "qg_create: n = %d exceeds 2^24", n);
  if(p->interpolation_order < 1 || p->interpolation_order > kMaxOrder)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_create: interpolation_order %d outside [1, %d]",
                   p->interpolation_order, kMaxOrder);
  if(!(p->dt > 0) || !(p->c0 > 0) || !(p->hbar != 0) || !std::isfinite(p->dt))
    return qg_fail(QG_ERR_INVALID_ARG, "qg_create: dt and c0 must be positive, hbar non-zero");
  if(p->num_timesteps < 0) return qg_fail(QG_ERR_INVALID_ARG, "qg_create: num_timesteps < 0");
  if(p->frame != QG_FRAME_ROTATING && p->frame != QG_FRAME_LAB)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_create: unknown frame %d", p->frame);
  if(p->precision != QG_PREC_FP64 && p->precision != QG_PREC_MIXED)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_create: unknown precision %d", p->precision);
  if(p->coef_mode != QG_COEF_AUTO && p->coef_mode != QG_COEF_TABLE && p->coef_mode != QG_COEF_ON_THE_FLY &&
     p->coef_mode != QG_COEF_TUNED)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_create: unknown coef_mode %d", p->coef_mode);
  return QG_OK;
}

// Ordered tile pairs: every unordered pair is stored twice.  FP64: q+1
// complex128 taps; mixed: q+1 complex64 taps and their sum.
static size_t table_bytes(int nT, int q, bool mixed)
{
  const size_t per = mixed ? sizeof(int) + sizeof(float2) * (q + 2) : sizeof(int) + sizeof(double2) * (q + 1);
  return (size_t)nT * nT * kTilePairs * per;
}

// Source tiles per far-kernel warp (see create_impl).
static int far_group(bool mixed, int nT) { return mixed && nT < 256 ? 2 : kTileGroup; }

// Even, so every ring row starts 32-byte aligned for paired-sample loads.
static int ring_depth(int max_delay, int q)
{
  const int w = max_delay + q + kTimeBlock + 2;
  return w + (w & 1);
}

// Steps per trajectory chunk: a multiple of K, about 4 MiB (small chunks
// let each chunk's copy to the host overlap the next chunk's steps).
static int traj_steps(int n)
{
  long long k = std::min<long long>(256, (4ll << 20) / (32ll * n));
  k = std::max<long long>(kTimeBlock, k - k % kTimeBlock);
  return (int)k;
}

// Builds the per-step lists from the pairs with floor delay < K: the mid
// list (all their taps, read by the dot-step kernels every step) and the near
// list (tap 0 of the delay-0 pairs, re-read in every corrector iteration),
// and packs the groups of dots coupled at delay 0 into step blocks.
static qg_status build_lists(qg_handle *h, const TableArgs &ta)
{
  const int q1 = h->q + 1;
  // pairs with floor delay < K (same delay arithmetic as the table), then
  // their FP64 coefficients: the mid list is FP64 in both precisions
  int *d_pairs = nullptr;
  double2 *d_mc = nullptr;
  // the temporaries go back to the pool on every return path
  struct Temp {
    qg_handle *h;
    void **p;
    ~Temp()
    {
      if(*p) pool_free(h, *p);
    }
  } keep_pairs{h, (void **)&d_pairs}, keep_mc{h, (void **)&d_mc};
  unsigned long long cnt = 0;
  const double c0dt = h->params.c0 * h->params.dt;
  for(int pass = 0; pass < 2; ++pass) {
    const unsigned long long cap = pass == 0 ? 0 : std::max<unsigned long long>(cnt, 1);
    if(pass == 1) {
      QG_CUDA(pool_alloc(h, (void **)&d_pairs, sizeof(int) * 3 * cap));
      QG_CUDA(pool_alloc(h, (void **)&d_mc, sizeof(double2) * q1 * cap));
    }
    QG_CUDA(cudaMemsetAsync(h->d_u64 + 2, 0, sizeof(unsigned long long), h->stream));
    launch_near_find(h->d_pos, h->d_user, h->n_pad, c0dt, kTimeBlock, d_pairs, h->d_u64 + 2, cap, h->stream);
    QG_CUDA(cudaGetLastError());
    QG_CUDA(cudaMemcpyAsync(&cnt, h->d_u64 + 2, sizeof cnt, cudaMemcpyDeviceToHost, h->stream));
    QG_CUDA(cudaStreamSynchronize(h->stream));
  }
  h->mid_pairs = (long long)cnt;
  launch_pair_list_coef(ta, h->q, d_pairs, (long long)cnt, d_mc, h->stream);
  QG_CUDA(cudaGetLastError());
  const unsigned long long cap = std::max<unsigned long long>(cnt, 1);
  std::vector<int> pairs(3 * cap);
  std::vector<double2> mc(q1 * cap);
  QG_CUDA(cudaMemcpyAsync(pairs.data(), d_pairs, sizeof(int) * 3 * cap, cudaMemcpyDeviceToHost, h->stream));
  QG_CUDA(cudaMemcpyAsync(mc.data(), d_mc, sizeof(double2) * q1 * cap, cudaMemcpyDeviceToHost, h->stream));
  QG_CUDA(cudaStreamSynchronize(h->stream));
  pool_free(h, d_pairs);
  d_pairs = nullptr;
  const long long m = h->mid_pairs;
  const int n = h->n_pad;  // internal indices (padding holes have no pairs)

  // mid list: both directions, partners in increasing order (a counting
  // pass places each dot's entries, then its short segment is sorted: the
  // pairs arrive in the device's append order, which varies run to run)
  struct MidEntry {
    int b, d;
    long long k;  // index into pairs / mc
  };
  std::vector<int> mptr(n + 1, 0);  // n = n_pad here
  for(long long k = 0; k < m; ++k) {
    ++mptr[pairs[3 * k] + 1];
    ++mptr[pairs[3 * k + 1] + 1];
  }
  for(int i = 0; i < n; ++i) mptr[i + 1] += mptr[i];
  std::vector<MidEntry> ment((size_t)mptr[n]);
  {
    std::vector<int> fill(mptr.begin(), mptr.end() - 1);
    for(long long k = 0; k < m; ++k) {
      const int a = pairs[3 * k], b = pairs[3 * k + 1], d = pairs[3 * k + 2];
      ment[fill[a]++] = {b, d, k};
      ment[fill[b]++] = {a, d, k};
    }
  }
  std::vector<std::vector<std::pair<int, double2>>> adj(n);  // delay-0 tap-0 coupling
  DSU dsu(n);
  for(long long k = 0; k < m; ++k) {
    const int a = pairs[3 * k], b = pairs[3 * k + 1], d = pairs[3 * k + 2];
    if(d == 0) {
      if(h->otf) ++h->near_pairs;
      adj[a].push_back({b, mc[k * q1]});
      adj[b].push_back({a, mc[k * q1]});
      dsu.unite(a, b);
    }
  }
  // the entries' coefficients are gathered into list order on the device
  // (msrc[e] = the entry's pair), from the pair-order array still there
  std::vector<int> midx((size_t)mptr[n]), mdel((size_t)mptr[n]);
  std::vector<long long> msrc((size_t)mptr[n]);
  for(int i = 0; i < n; ++i) {
    std::sort(ment.begin() + mptr[i], ment.begin() + mptr[i + 1],
              [](const MidEntry &x, const MidEntry &y) { return x.b < y.b; });
    for(int e = mptr[i]; e < mptr[i + 1]; ++e) {
      midx[e] = ment[e].b;
      mdel[e] = ment[e].d;
      msrc[e] = ment[e].k;
    }
  }
  for(auto &v : adj)
    std::sort(v.begin(), v.end(), [](const std::pair<int, double2> &x,
                                     const std::pair<int, double2> &y) { return x.first < y.first; });
  // taps that read step t-1 (delay 1 tap 0, delay 0 tap 1), by dot in mid-list order
  std::vector<int> nptr(n + 1, 0), nidx;
  std::vector<double2> ncoef;
  bool lag = true;
  for(int i = 0; i < n; ++i) {
    for(int j = mptr[i]; j < mptr[i + 1]; ++j)
      if(const MidEntry &e = ment[j]; e.d <= 1) {
        nidx.push_back(e.b);
        ncoef.push_back(mc[e.k * q1 + (1 - e.d)]);
        if(e.b / 32 != i / 32) lag = false;
      }
    nptr[i + 1] = (int)nidx.size();
  }
  std::vector<int> gptr(n + 1, 0), gidx;
  std::vector<double2> gcoef;
  for(int i = 0; i < n; ++i) {
    for(auto &e : adj[i]) {
      gidx.push_back(e.first);
      gcoef.push_back(e.second);
    }
    gptr[i + 1] = (int)gidx.size();
  }

  // fused form: the dot order already places every delay-0 group inside one
  // 32-dot block (see order_for_near_groups); partners are addressed by
  // their position in the block
  std::vector<int> fptr(1, 0), fidx;
  std::vector<double2> fcoef;
  const int np = h->n_pad;
  if(h->fused) {
    // every delay-0 partner must share the dot's 32-dot block
    for(int i = 0; i < np && h->fused; ++i)
      for(auto &e : adj[i])
        if(e.first / 32 != i / 32) {
          h->fused = false;
          break;
        }
  }
  if(h->fused) {
    for(int i = 0; i < np; ++i) {
      if(i < n)
        for(auto &e : adj[i]) {
          fidx.push_back(e.first - (i / 32) * 32);
          fcoef.push_back(e.second);
        }
      fptr.push_back((int)fidx.size());
    }
  } else {
    fptr.assign(np + 1, 0);
  }
  h->step_blocks = np / 32;
  // the step-block kernel: all blocks resident, each with its part of the
  // mid list in shared memory when that still fits
  // and, again when it fits, the history of each block's distinct partners
  // per block: its distinct partners in order of first use (mpj[e] = the
  // entry's partner's position among them) and the blocks that hold them
  // (the block itself first); stamps instead of sorts, one pass per block
  int max_e = 0, max_p = 0;
  std::vector<int> bptr(1, 0), bidx, mpj(midx.size()), pbptr(1, 0), pbidx;
  std::vector<int> seen(np, -1), where(np, 0), bseen(std::max(h->step_blocks, 1), -1);
  for(int b = 0; b < h->step_blocks; ++b) {
    const int e0 = mptr[32 * b], e1 = mptr[32 * (b + 1)];
    max_e = std::max(max_e, e1 - e0);
    const int p0 = (int)bidx.size();
    for(int e = e0; e < e1; ++e) {
      const int pp = midx[e];
      if(seen[pp] != b) {
        seen[pp] = b;
        where[pp] = (int)bidx.size() - p0;
        bidx.push_back(pp);
      }
      mpj[e] = where[pp];
    }
    bseen[b] = b;
    pbidx.push_back(b);
    for(int j = p0; j < (int)bidx.size(); ++j)
      if(bseen[bidx[j] / 32] != b) {
        bseen[bidx[j] / 32] = b;
        pbidx.push_back(bidx[j] / 32);
      }
    pbptr.push_back((int)pbidx.size());
    bptr.push_back((int)bidx.size());
    max_p = std::max(max_p, (int)bidx.size() - p0);
  }
  h->mid_cache = 0;
  h->hist_cap = 0;
  h->block_step_ok = false;
  if(h->fused) {
    if(h->step_blocks <= step_block_max_blocks(h->q, max_e, max_p)) {
      h->mid_cache = max_e;
      h->hist_cap = max_p;
      h->block_step_ok = true;
    } else if(h->step_blocks <= step_block_max_blocks(h->q, max_e, 0)) {
      h->mid_cache = max_e;
      h->block_step_ok = true;
    } else if(h->step_blocks <= step_block_max_blocks(h->q, 0, 0)) {
      h->block_step_ok = true;
    }
  }
  h->block_step = h->block_step_ok;

  auto upload_i = [&](int **dst, const std::vector<int> &v) -> qg_status {
    QG_TRY(dalloc(h, dst, v.size()));
    if(!v.empty())
      QG_CUDA(cudaMemcpyAsync(*dst, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice, h->stream));
    return QG_OK;
  };
  auto upload_c = [&](double2 **dst, const std::vector<double2> &v) -> qg_status {
    QG_TRY(dalloc(h, dst, v.size()));
    if(!v.empty())
      QG_CUDA(cudaMemcpyAsync(*dst, v.data(), sizeof(double2) * v.size(), cudaMemcpyHostToDevice, h->stream));
    return QG_OK;
  };
  QG_TRY(upload_i(&h->d_mid_ptr, mptr));
  QG_TRY(upload_i(&h->d_mid_idx, midx));
  QG_TRY(upload_i(&h->d_mid_delay, mdel));
  {
    const long long ne = (long long)midx.size();
    QG_TRY(dalloc(h, &h->d_mid_coef, (size_t)ne * q1));
    long long *d_msrc = nullptr;
    cudaError_t ce = pool_alloc(h, (void **)&d_msrc, sizeof(long long) * (size_t)std::max<long long>(ne, 1));
    if(ce == cudaSuccess && ne > 0)
      ce = cudaMemcpyAsync(d_msrc, msrc.data(), sizeof(long long) * (size_t)ne, cudaMemcpyHostToDevice, h->stream);
    if(ce == cudaSuccess) {
      launch_gather_rows(d_mc, d_msrc, q1, ne, h->d_mid_coef, h->stream);
      ce = cudaGetLastError();
    }
    if(ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
    pool_free(h, d_msrc);
    pool_free(h, d_mc);
    d_mc = nullptr;
    QG_CUDA(ce);
  }
  QG_TRY(upload_i(&h->d_gnear_ptr, gptr));
  QG_TRY(upload_i(&h->d_gnear_idx, gidx));
  QG_TRY(upload_c(&h->d_gnear_coef, gcoef));
  QG_TRY(upload_i(&h->d_fnear_ptr, fptr));
  QG_TRY(upload_i(&h->d_fnear_idx, fidx));
  QG_TRY(upload_c(&h->d_fnear_coef, fcoef));
  QG_TRY(upload_i(&h->d_new_ptr, nptr));
  QG_TRY(upload_i(&h->d_new_idx, nidx));
  QG_TRY(upload_c(&h->d_new_coef, ncoef));
  QG_TRY(upload_i(&h->d_bp_ptr, bptr));
  QG_TRY(upload_i(&h->d_bp_idx, bidx));
  QG_TRY(upload_i(&h->d_mid_pj, mpj));
  QG_TRY(upload_i(&h->d_pb_ptr, pbptr));
  QG_TRY(upload_i(&h->d_pb_idx, pbidx));
  QG_TRY(dalloc(h, &h->d_flags, (size_t)std::max(h->step_blocks, 1) * kFlagStride));
  h->lag = h->fused && lag;
  return QG_OK;
}

static qg_status reset_state(qg_handle *h)
{
  h->batch_bad_valid = false;
  QG_CUDA(cudaMemsetAsync(h->d_ring, 0, sizeof(double2) * (size_t)h->n_pad * h->stride, h->stream));
  if(h->mixed) {
    QG_CUDA(cudaMemsetAsync(h->d_ring32w, 0, sizeof(float2) * (size_t)h->n_pad * h->stride, h->stream));
    QG_CUDA(cudaMemsetAsync(h->d_ring32d, 0, sizeof(float2) * (size_t)h->n_pad * h->stride, h->stream));
  }
  QG_CUDA(cudaMemsetAsync(h->d_partial, 0,
                          sizeof(double2) * (size_t)kTimeBlock * h->nG * h->n_pad, h->stream));
  QG_CUDA(cudaMemsetAsync(h->d_field, 0, sizeof(double2) * (size_t)kTimeBlock * h->n_pad, h->stream));
  QG_CUDA(cudaMemsetAsync(h->d_tile_done, 0, sizeof(unsigned) * (size_t)h->nT, h->stream));
  launch_init_state(h->step_args(false), h->stream);
  int init[9] = {0, 0, kBadNone, 0, 0, h->max_delay, 0, 0, 0};
  QG_CUDA(cudaMemcpyAsync(h->d_ints, init, sizeof init, cudaMemcpyHostToDevice, h->stream));
  QG_CUDA(cudaStreamSynchronize(h->stream));
  h->next_step = 0;
  h->eval_cached = -0x7fffffff;
  h->far_block = -0x7fffffff;
  return QG_OK;
}

// Finds the pairs at floor delay 0 (one cheap kernel over all pairs) and
// chooses the internal dot order: Morton order, with every connected group
// of delay-0 pairs moved into one 32-dot block so the fused step kernel can
// iterate the group with warp-level synchronisation only.  Groups larger
// than 32 dots select the general step form and keep Morton order.
static qg_status order_for_near_groups(qg_handle *h, const qg_dot *dots, const std::vector<int> &morton,
                                       std::vector<int> &order)
{
  const int n = h->n;
  const int np0 = ((n + kTile - 1) / kTile) * kTile;
  std::vector<double> pos((size_t)np0 * 3, 0.0);
  std::vector<int> user(np0, -1);
  for(int i = 0; i < n; ++i) {
    for(int k = 0; k < 3; ++k) pos[3 * i + k] = dots[morton[i]].pos[k];
    user[i] = morton[i];
  }
  double *d_pos = nullptr;
  int *d_user = nullptr, *d_pairs = nullptr;
  unsigned long long *d_cnt = nullptr;
  QG_CUDA(pool_alloc(h, (void **)&d_pos, sizeof(double) * pos.size()));
  QG_CUDA(pool_alloc(h, (void **)&d_user, sizeof(int) * user.size()));
  QG_CUDA(pool_alloc(h, (void **)&d_cnt, sizeof(unsigned long long)));
  QG_CUDA(cudaMemcpyAsync(d_pos, pos.data(), sizeof(double) * pos.size(), cudaMemcpyHostToDevice, h->stream));
  QG_CUDA(cudaMemcpyAsync(d_user, user.data(), sizeof(int) * user.size(), cudaMemcpyHostToDevice, h->stream));
  const double c0dt = h->params.c0 * h->params.dt;
  unsigned long long cnt = 0;
  for(int pass = 0; pass < 2; ++pass) {
    const unsigned long long cap = pass == 0 ? 0 : std::max<unsigned long long>(cnt, 1);
    if(pass == 1) QG_CUDA(pool_alloc(h, (void **)&d_pairs, sizeof(int) * 3 * cap));
    QG_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), h->stream));
    launch_near_find(d_pos, d_user, np0, c0dt, 2, d_pairs, d_cnt, cap, h->stream);
    QG_CUDA(cudaGetLastError());
    QG_CUDA(cudaMemcpyAsync(&cnt, d_cnt, sizeof cnt, cudaMemcpyDeviceToHost, h->stream));
    QG_CUDA(cudaStreamSynchronize(h->stream));
  }
  std::vector<int> pairs(3 * std::max<unsigned long long>(cnt, 1));
  if(cnt) {
    QG_CUDA(cudaMemcpyAsync(pairs.data(), d_pairs, sizeof(int) * 3 * cnt, cudaMemcpyDeviceToHost, h->stream));
    QG_CUDA(cudaStreamSynchronize(h->stream));
  }
  pool_free(h, d_pos);
  pool_free(h, d_user);
  pool_free(h, d_cnt);
  pool_free(h, d_pairs);

  // groups over Morton positions: the connected components of the pairs at
  // floor delay <= 1 when each fits in a block (then the delay-1 partners
  // share the block too, and the step-block kernel never waits for a step
  // just finished in another block), else of the delay-0 pairs alone
  std::vector<char> coupled;
  std::vector<std::vector<int>> comps;
  size_t largest = 0;
  for(int level = 1; level >= 0; --level) {
    DSU dsu(n);
    coupled.assign(n, 0);
    for(unsigned long long k = 0; k < cnt; ++k) {
      if(pairs[3 * k + 2] > level) continue;
      dsu.unite(pairs[3 * k], pairs[3 * k + 1]);
      coupled[pairs[3 * k]] = coupled[pairs[3 * k + 1]] = 1;
    }
    comps.clear();
    std::vector<int> root_to_comp(n, -1);
    for(int i = 0; i < n; ++i) {
      if(!coupled[i]) continue;
      const int r = dsu.find(i);
      if(root_to_comp[r] < 0) {
        root_to_comp[r] = (int)comps.size();
        comps.emplace_back();
      }
      comps[root_to_comp[r]].push_back(i);
    }
    largest = 0;
    for(auto &c : comps) largest = std::max(largest, c.size());
    if(largest <= 32) break;
  }
  h->fused = largest <= 32;
  order.clear();
  if(!h->fused || comps.empty()) {
    for(int i = 0; i < n; ++i) order.push_back(morton[i]);
    while(order.size() % kTile) order.push_back(-1);
    return QG_OK;
  }
  std::sort(comps.begin(), comps.end(),
            [](const std::vector<int> &x, const std::vector<int> &y) { return x.size() > y.size(); });
  std::vector<std::vector<int>> bins;
  for(auto &c : comps) {
    size_t b = 0;
    for(; b < bins.size(); ++b)
      if(bins[b].size() + c.size() <= 32) break;
    if(b == bins.size()) bins.emplace_back();
    bins[b].insert(bins[b].end(), c.begin(), c.end());
  }
  size_t fill = 0;
  for(int i = 0; i < n; ++i) {
    if(coupled[i]) continue;
    while(fill < bins.size() && bins[fill].size() >= 32) ++fill;
    if(fill == bins.size()) bins.emplace_back();
    bins[fill].push_back(i);
  }
  for(auto &b : bins) {
    for(int i : b) order.push_back(morton[i]);
    for(size_t j = b.size(); j < 32; ++j) order.push_back(-1);
  }
  return QG_OK;
}

static qg_status autotune_far(qg_handle *h);

static qg_status create_impl(const qg_dot *dots, int n, const qg_pulse *pulse, const qg_params *p,
                             const qg_weights *weights, qg_handle *h)
{
  QG_CUDA(cudaGetDevice(&h->device));
  QG_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  QG_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
  h->n = n;
  h->q = p->interpolation_order;
  h->T = p->num_timesteps;
  h->params = *p;
  h->pulse = *pulse;
  h->P = (long long)n * (n - 1) / 2;

  qg_weights wt;
  if(weights) {
    wt = *weights;
    if(wt.n_time < 2 || wt.n_time > 32)
      return qg_fail(QG_ERR_INVALID_ARG, "qg_create: weights.n_time %d outside [2, 32]", wt.n_time);
    if(wt.n_time > kWindow)
      return qg_fail(QG_ERR_UNSUPPORTED, "qg_create: weights.n_time %d exceeds the 22-step window",
                     wt.n_time);
  } else {
    QG_TRY(qg_pc_weights(18, 22, 3.15, &wt));
  }
  h->w.n_time = wt.n_time;
  for(int i = 0; i < 2 * wt.n_time; ++i) {
    h->w.ps[i] = wt.ps[i];
    h->w.cs[i] = wt.cs[i];
  }
  h->w.fc = wt.future_coef;

  // internal order: Morton, delay-0 groups packed into 32-dot blocks
  std::vector<int> order;
  QG_TRY(order_for_near_groups(h, dots, morton_order(dots, n), order));
  h->n_pad = (int)order.size();
  h->nT = h->n_pad / kTile;
  // source tiles per far-kernel warp: 4 in FP64; 2 for the mixed path up to
  // 255 tiles (twice as many warps balance its shorter per-source work
  // better), 4 from 256 tiles, where the partial sums (16 steps x groups x
  // N, FP64) would otherwise add ~13 % to the FP32 table stream
  h->group = far_group(p->precision == QG_PREC_MIXED, h->nT);
  h->nG = (h->nT + h->group - 1) / h->group;
  h->nblk = (long long)h->nT * (h->nT + 1) / 2;
  std::vector<double> pos((size_t)h->n_pad * 3, 0.0), dip((size_t)h->n_pad * 3, 0.0);
  std::vector<double> fr(h->n_pad, 0.0), t1(h->n_pad, 1.0), t2(h->n_pad, 1.0);
  std::vector<int> user(h->n_pad, -1);
  for(int i = 0; i < h->n_pad; ++i) {
    if(order[i] < 0) continue;
    const qg_dot &d = dots[order[i]];
    for(int k = 0; k < 3; ++k) {
      pos[3 * i + k] = d.pos[k];
      dip[3 * i + k] = d.dip[k];
    }
    fr[i] = d.freq;
    t1[i] = d.t1;
    t2[i] = d.t2;
    user[i] = order[i];
  }
  QG_TRY(dalloc(h, &h->d_pos, pos.size()));
  QG_TRY(dalloc(h, &h->d_dip, dip.size()));
  QG_TRY(dalloc(h, &h->d_freq, fr.size()));
  QG_TRY(dalloc(h, &h->d_t1, t1.size()));
  QG_TRY(dalloc(h, &h->d_t2, t2.size()));
  QG_TRY(dalloc(h, &h->d_user, user.size()));
  QG_CUDA(cudaMemcpyAsync(h->d_pos, pos.data(), sizeof(double) * pos.size(), cudaMemcpyHostToDevice, h->stream));
  QG_CUDA(cudaMemcpyAsync(h->d_dip, dip.data(), sizeof(double) * dip.size(), cudaMemcpyHostToDevice, h->stream));
  QG_CUDA(cudaMemcpyAsync(h->d_freq, fr.data(), sizeof(double) * fr.size(), cudaMemcpyHostToDevice, h->stream));
  QG_CUDA(cudaMemcpyAsync(h->d_t1, t1.data(), sizeof(double) * t1.size(), cudaMemcpyHostToDevice, h->stream));
  QG_CUDA(cudaMemcpyAsync(h->d_t2, t2.data(), sizeof(double) * t2.size(), cudaMemcpyHostToDevice, h->stream));
  QG_CUDA(cudaMemcpyAsync(h->d_user, user.data(), sizeof(int) * user.size(), cudaMemcpyHostToDevice, h->stream));
  QG_TRY(dalloc(h, &h->d_ints, 16));
  QG_TRY(dalloc(h, &h->d_u64, 4));
  QG_CUDA(cudaMemsetAsync(h->d_ints, 0, sizeof(int) * 16, h->stream));
  QG_CUDA(cudaMemsetAsync(h->d_u64, 0, sizeof(unsigned long long) * 4, h->stream));

  // coefficients: a table when asked for, or (auto) when it takes at most
  // half of the free device memory; otherwise computed in the far kernel
  h->mixed = p->precision == QG_PREC_MIXED;
  const size_t tb = table_bytes(h->nT, h->q, h->mixed);
  size_t free_b = 0, total_b = 0;
  QG_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const bool rule = p->coef_mode == QG_COEF_AUTO || p->coef_mode == QG_COEF_TUNED;
  h->otf = p->coef_mode == QG_COEF_ON_THE_FLY || (rule && tb > free_b / 2);
  // on the fly: source-group-major tasks, 3 blocks per SM (measured at
  // N = 65536: 274 against 322 ms per FP64 launch for 7, 168 against 177
  // mixed; same sums)
  if(h->otf) h->far_variant = kOtfVariant;
  h->tune_coef = p->coef_mode == QG_COEF_TUNED && !h->otf;
  if(!h->otf && tb > free_b * 0.9)
    return qg_fail(QG_ERR_OOM, "qg_create: coefficient table needs %zu bytes, %zu free", tb, free_b);
  if(h->otf) {
    // about 16 source groups per target tile: enough warps for the device,
    // partial sums of K x 16 x n_pad
    h->group = (h->nT + 15) / 16;
    h->nG = (h->nT + h->group - 1) / h->group;
  } else {
    QG_TRY(dalloc(h, &h->d_delay, (size_t)h->nT * h->nT * kTilePairs));
    if(h->mixed)
      QG_TRY(dalloc(h, &h->d_coef32, (size_t)h->nT * h->nT * kTilePairs * (h->q + 2)));
    else
      QG_TRY(dalloc(h, &h->d_coef, (size_t)h->nT * h->nT * kTilePairs * (h->q + 1)));
  }
  TableArgs ta{};
  ta.pos = h->d_pos;
  ta.dip = h->d_dip;
  ta.user = h->d_user;
  ta.n = n;
  ta.n_pad = h->n_pad;
  ta.nT = h->nT;
  ta.nblk = h->nblk;
  ta.delay = h->d_delay;
  ta.coef = h->d_coef;
  ta.coef32 = h->d_coef32;
  ta.mixed = h->mixed ? 1 : 0;
  ta.max_delay = h->d_ints + 5;
  ta.near_count = h->d_u64;
  ta.cp.c0 = p->c0;
  ta.cp.dt = p->dt;
  ta.cp.mu0 = p->mu0;
  ta.cp.hbar = p->hbar;
  ta.cp.omega = p->laser_frequency;
  ta.cp.q = h->q;
  ta.cp.frame = p->frame;
  cudaEvent_t e0, e1;
  QG_CUDA(cudaEventCreate(&e0));
  QG_CUDA(cudaEventCreate(&e1));
  QG_CUDA(cudaEventRecord(e0, h->stream));
  if(h->otf)
    launch_max_delay(h->d_pos, h->d_user, h->n_pad, p->c0 * p->dt, h->d_ints + 5, h->stream);
  else
    launch_table_build(ta, h->q, h->stream);
  QG_CUDA(cudaGetLastError());
  QG_CUDA(cudaEventRecord(e1, h->stream));
  int md = 0;
  unsigned long long nn[4] = {0, 0, 0, 0};
  QG_CUDA(cudaMemcpyAsync(&md, h->d_ints + 5, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  QG_CUDA(cudaMemcpyAsync(nn, h->d_u64, sizeof nn, cudaMemcpyDeviceToHost, h->stream));
  QG_CUDA(cudaStreamSynchronize(h->stream));
  float tms = 0;
  cudaEventElapsedTime(&tms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->table_ms = tms;
  if(md < 0 || md > (1 << 26))
    return qg_fail(QG_ERR_INVALID_ARG, "qg_create: floor delay %d out of range (non-finite positions?)",
                   md);
  h->max_delay = md;
  h->near_pairs = (long long)nn[0];  // on the fly: counted from the mid list below
  h->mid_pairs = (long long)nn[1];
  h->far_nonfinite = nn[3] > 0;

  // rings and scratch.  W covers the oldest sample a far block reads
  // (t0 - max_delay - q) even when the block is recomputed up to K - 1
  // steps after t0.
  h->W = ring_depth(md, h->q);
  h->stride = h->W + kRingMirror;
  QG_TRY(dalloc(h, &h->d_ring, (size_t)h->n_pad * h->stride));
  if(h->mixed) {
    QG_TRY(dalloc(h, &h->d_ring32w, (size_t)h->n_pad * h->stride));
    QG_TRY(dalloc(h, &h->d_ring32d, (size_t)h->n_pad * h->stride));
  }
  QG_TRY(dalloc(h, &h->d_pcr, (size_t)kPcDepth * 4 * h->n_pad));
  // partials for the smallest group size the "far_group" option allows
  h->max_groups = h->otf ? h->nG : (h->nT <= 512 ? h->nT : h->nG);
  QG_TRY(dalloc(h, &h->d_partial, (size_t)kTimeBlock * h->max_groups * h->n_pad));
  QG_TRY(dalloc(h, &h->d_field, (size_t)kTimeBlock * h->n_pad));
  QG_TRY(dalloc(h, &h->d_tile_done, (size_t)h->nT));
  QG_TRY(dalloc(h, &h->d_scratch, (size_t)h->n_pad * 8));
  h->traj_k = traj_steps(n);
  QG_TRY(dalloc(h, &h->d_traj, (size_t)2 * h->traj_k * n * 2));
  QG_TRY(dalloc(h, &h->d_io, (size_t)n));
  for(int i = 0; i < 2; ++i) {
    QG_CUDA(cudaEventCreateWithFlags(&h->ev_chunk[i], cudaEventDisableTiming));
    QG_CUDA(cudaEventCreateWithFlags(&h->ev_copy[i], cudaEventDisableTiming));
  }

  QG_TRY(build_lists(h, ta));
  QG_TRY(reset_state(h));
  // the far-kernel autotuner runs at the first qg_run: a batch member never
  // runs alone (the batch kernel has its own form), so it is never timed
  h->tune_pending = true;
  return QG_OK;
}

// The far-kernel autotuner.  The FP64 table path has several kernels with
// identical arithmetic (and so identical results) but different resource
// shapes; which one is fastest depends on N and on the device.  Each is
// launched twice untimed (first use, clocks settling), then timed in three
// rounds (candidates interleaved, best of the three kept), at a block start
// past the largest delay (every tap live, as in the steady state); the
// fastest is kept.  The history
// is whatever the handle holds (its values do not change the work), and the
// far field and partials are recomputed by the next run.
static qg_status switch_to_otf(qg_handle *h);

static qg_status time_far(qg_handle *h, int rounds_untimed, int rounds_timed, float *best_ms)
{
  cudaEvent_t e0, e1;
  QG_CUDA(cudaEventCreate(&e0));
  QG_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for(int round = 0; round < rounds_untimed + rounds_timed; ++round) {
    const FarArgs fa = h->far_args(h->d_ints + 7, h->d_ints + 6);
    if(round < rounds_untimed) {
      launch_far(fa, h->stream);
      continue;
    }
    QG_CUDA(cudaEventRecord(e0, h->stream));
    launch_far(fa, h->stream);
    QG_CUDA(cudaEventRecord(e1, h->stream));
    QG_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    QG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *best_ms = best;
  return QG_OK;
}

// QG_COEF_TUNED: the on-the-fly kernel (its own source grouping) against the
// table kernel's time; when it wins, the handle switches to it and frees the
// table.
static qg_status autotune_coef(qg_handle *h)
{
  const int group_t = h->group, nG_t = h->nG, variant_t = h->far_variant;
  h->otf = true;
  h->group = (h->nT + 15) / 16;
  h->nG = (h->nT + h->group - 1) / h->group;
  h->far_variant = kOtfVariant;
  float otf_ms = 0;
  const qg_status st = time_far(h, 2, 3, &otf_ms);
  if(st != QG_OK || otf_ms >= h->tuned_far_ms) {
    h->otf = false;
    h->group = group_t;
    h->nG = nG_t;
    h->far_variant = variant_t;
    return st;
  }
  // the on-the-fly kernel is faster: keep it, return the table's memory
  QG_TRY(switch_to_otf(h));
  h->tuned_far_ms = otf_ms;
  return QG_OK;
}

// A table handle moves to on-the-fly coefficients (the QG_COEF_TUNED choice)
// and frees its table.
static qg_status switch_to_otf(qg_handle *h)
{
  h->otf = true;
  h->far_variant = kOtfVariant;
  h->group = (h->nT + 15) / 16;
  h->nG = (h->nT + h->group - 1) / h->group;
  QG_CUDA(cudaStreamSynchronize(h->stream));
  for(void *p : {(void *)h->d_delay, (void *)h->d_coef, (void *)h->d_coef32}) {
    if(!p) continue;
    auto it = std::find(h->allocs.begin(), h->allocs.end(), p);
    if(it != h->allocs.end()) h->allocs.erase(it);
    pool_free(h, p);
  }
  h->bytes -= table_bytes(h->nT, h->q, h->mixed);
  h->d_delay = nullptr;
  h->d_coef = nullptr;
  h->d_coef32 = nullptr;
  return QG_OK;
}

// Source tiles per far-kernel warp (the "far_group" option): each group
// writes one partial per target and step, and the partials are then summed
// over groups, so the group size changes the association of the far sums
// (results move within rounding, not bit for bit).  The search therefore
// runs only when asked for ("tune_group"), after the variant is chosen, and
// keeps the faster of the default and each of 1, 2, 4 and 8 that the
// handle's partial buffer holds.
static qg_status autotune_group(qg_handle *h)
{
  const int g0 = h->group;
  int best_g = g0;
  float best = h->tuned_far_ms;
  for(int g : {1, 2, 4, 8}) {
    if(g == g0 || (h->nT + g - 1) / g > h->max_groups) continue;
    h->group = g;
    h->nG = (h->nT + g - 1) / g;
    float t = 0;
    QG_TRY(time_far(h, 2, 3, &t));
    if(t < best) {
      best = t;
      best_g = g;
    }
  }
  h->group = best_g;
  h->nG = (h->nT + best_g - 1) / best_g;
  h->tuned_far_ms = best;
  return QG_OK;
}

static qg_status autotune_far(qg_handle *h)
{
  if(h->otf || h->nT < 16) return QG_OK;  // one kernel, or too small to matter
  if(h->mixed) {
    // one table kernel at two register budgets (0 and 7: 150 registers, 1
    // and 8: 128) in two task orders (7 and 8 source-group major), the same
    // sums; the fastest one's time is the one the coefficient choice compares
    launch_set_int(h->d_ints + 7, h->max_delay + h->q + 2 * kTimeBlock, h->stream);
    float best = 1e30f;
    int best_v = 0;
    for(int v : {0, 7, 1, 8}) {
      h->far_variant = v;
      float t = 0;
      QG_TRY(time_far(h, 2, 3, &t));
      if(t < best) {
        best = t;
        best_v = v;
      }
    }
    h->far_variant = best_v;
    h->tuned_far_ms = best;
    if(h->tune_group) QG_TRY(autotune_group(h));
    if(h->tune_coef) QG_TRY(autotune_coef(h));
    h->far_block = -0x7fffffff;
    h->eval_cached = -0x7fffffff;
    return QG_OK;
  }
  static const int candidates[] = {0, 3, 5, 6, 7, 8, 9, 10, 11};
  const int t_test = h->max_delay + h->q + 2 * kTimeBlock;
  cudaEvent_t e0, e1;
  QG_CUDA(cudaEventCreate(&e0));
  QG_CUDA(cudaEventCreate(&e1));
  constexpr int nc = sizeof(candidates) / sizeof(candidates[0]);
  float t_best[nc];
  launch_set_int(h->d_ints + 7, t_test, h->stream);
  for(int round = 0; round < 5; ++round)
    for(int c = 0; c < nc; ++c) {
      h->far_variant = candidates[c];
      const FarArgs fa = h->far_args(h->d_ints + 7, h->d_ints + 6);
      if(round < 2) {
        launch_far(fa, h->stream);  // untimed: first use of the kernel, clocks settling
        continue;
      }
      QG_CUDA(cudaEventRecord(e0, h->stream));
      launch_far(fa, h->stream);
      QG_CUDA(cudaEventRecord(e1, h->stream));
      QG_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      QG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      t_best[c] = round == 2 ? ms : std::min(t_best[c], ms);
    }
  float best = 1e30f;
  int best_v = candidates[0];
  for(int c = 0; c < nc; ++c)
    if(t_best[c] < best) {
      best = t_best[c];
      best_v = candidates[c];
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  QG_CUDA(cudaGetLastError());
  h->far_variant = best_v;
  h->tuned_far_ms = best;
  if(h->tune_group) QG_TRY(autotune_group(h));
  if(h->tune_coef) QG_TRY(autotune_coef(h));
  h->far_block = -0x7fffffff;
  h->eval_cached = -0x7fffffff;
  return QG_OK;
}

// The autotuner's choices, remembered for the process: handles of the same
// kind (device, tiles, order, frame, precision, coefficient mode) take the
// first one's choice without timing again.
struct TuneKey {
  int device, nT, q, frame, mixed, tune_coef, group;
  bool operator<(const TuneKey &o) const
  {
    return std::tie(device, nT, q, frame, mixed, tune_coef, group) <
           std::tie(o.device, o.nT, o.q, o.frame, o.mixed, o.tune_coef, o.group);
  }
};
struct TuneChoice {
  int variant, group;
  float far_ms;
  bool otf;
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneChoice> g_tune;

static qg_status switch_to_otf(qg_handle *h);

static qg_status autotune_cached(qg_handle *h, bool force)
{
  if(h->otf || h->nT < 16) return QG_OK;
  // the group part of the key: 0 when the group is searched, else the one set
  const TuneKey key{h->device, h->nT,  h->q, h->params.frame, h->mixed ? 1 : 0, h->tune_coef ? 1 : 0,
                    h->tune_group ? 0 : h->group};
  if(!force) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(key);
    if(it != g_tune.end()) {
      h->far_variant = it->second.variant;
      h->tuned_far_ms = it->second.far_ms;
      h->group = it->second.group;
      h->nG = (h->nT + h->group - 1) / h->group;
      if(it->second.otf) QG_TRY(switch_to_otf(h));
      h->far_block = -0x7fffffff;
      h->eval_cached = -0x7fffffff;
      return QG_OK;
    }
  }
  QG_TRY(autotune_far(h));
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune[key] = TuneChoice{h->far_variant, h->group, h->tuned_far_ms, h->otf};
  return QG_OK;
}

extern "C" qg_status qg_create(const qg_dot *dots, int n, const qg_pulse *pulse,
                               const qg_params *params, const qg_weights *weights, qg_handle **out)
{
  if(!out) return qg_fail(QG_ERR_INVALID_ARG, "qg_create: out is NULL");
  *out = nullptr;
  QG_TRY(validate(dots, n, pulse, params));
  qg_handle *h = new qg_handle();
  const qg_status st = create_impl(dots, n, pulse, params, weights, h);
  if(st != QG_OK) {
    destroy_handle(h);
    return st;
  }
  *out = h;
  return QG_OK;
}

extern "C" qg_status qg_destroy(qg_handle *h)
{
  destroy_handle(h);
  return QG_OK;
}

// The far-pair kernel for the block that starts at t0.  At a block
// boundary it reads t0 from the device step counter (so it can live in a
// CUDA graph); a block resumed part-way (after qg_history_evaluate reused the
// partial buffer, or when a run starts off a boundary) gets t0 explicitly.
// Inside a stream capture an event must be recorded as an external node to
// be readable after the graph runs; outside a capture that flag is invalid.
static void record_event(qg_handle *h, cudaEvent_t e)
{
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(h->stream, &st);
  if(st == cudaStreamCaptureStatusActive)
    cudaEventRecordWithFlags(e, h->stream, cudaEventRecordExternal);
  else
    cudaEventRecord(e, h->stream);
}

// Far blocks before this step start some windows before step -22 (the far
// kernels' first-blocks form is faster there; both forms give the same bits).
static bool early_block(const qg_handle *h, int t0)
{
  return h->far_early && !h->far_nonfinite && t0 < h->max_delay + h->q - kWindow;
}

static void enqueue_far(qg_handle *h, int t0, bool at_boundary, cudaEvent_t ea, cudaEvent_t eb, bool early)
{
  // at a boundary the previous block's last step kernel (or launch_steps)
  // has stored t0 in d_ints[0]; that read keeps the launch graph-capturable
  const int *src = h->d_ints + 0;
  if(!at_boundary) {
    launch_set_int(h->d_ints + 7, t0, h->stream);
    src = h->d_ints + 7;
  }
  if(ea) record_event(h, ea);
  FarArgs fa = h->far_args(src, h->d_ints + 6);
  fa.early = early ? 1 : 0;
  launch_far(fa, h->stream);
  if(eb) record_event(h, eb);
}

// Steps k0 .. k1-1 of the current block in one cooperative launch.
static void enqueue_step_block(qg_handle *h, int k0, int k1, bool traj)
{
  StepArgs a = h->step_args(false);
  if(traj) a.traj = h->d_traj;
  launch_step_block(a, k0, k1, h->step_blocks, h->d_flags, h->stream);
}

static void enqueue_dot_step(qg_handle *h, int k, bool traj)
{
  StepArgs a = h->step_args(!h->fused);
  if(traj) a.traj = h->d_traj;
  if(h->fused) {
    launch_step_fused(a, k, h->shard_world > 1 ? h->blk_hi - h->blk_lo : h->step_blocks, h->stream);
  } else {
    for(int ph = 0; ph <= kCorrectorSteps + 1; ++ph) launch_step_general(a, k, ph, h->stream);
  }
}

// One K-step block starting on a boundary: far kernel + K dot steps
// (prof >= 0: instance `prof` of the profiling ring, with event nodes).
static qg_status capture_block(qg_handle *h, int gi, int prof, cudaGraphExec_t *out)
{
  const int traj = gi & 1;
  cudaGraph_t g;
  QG_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  enqueue_far(h, 0, true, prof >= 0 ? h->pev[prof][0] : nullptr, prof >= 0 ? h->pev[prof][1] : nullptr,
              gi >= 2);
  if(h->block_step)
    enqueue_step_block(h, 0, kTimeBlock, traj != 0);
  else
    for(int k = 0; k < kTimeBlock; ++k) enqueue_dot_step(h, k, traj != 0);
  if(prof >= 0) record_event(h, h->pev[prof][2]);
  QG_CUDA(cudaStreamEndCapture(h->stream, &g));
  QG_CUDA(cudaGraphInstantiate(out, g, 0));
  cudaGraphDestroy(g);
  return QG_OK;
}

static qg_status ensure_graph(qg_handle *h, int gi)
{
  if(h->graph[gi]) return QG_OK;
  return capture_block(h, gi, -1, &h->graph[gi]);
}

static qg_status collect_prof(qg_handle *h, int i)
{
  if(!h->pending[i]) return QG_OK;
  QG_CUDA(cudaEventSynchronize(h->pev[i][2]));
  float far = 0, steps = 0;
  cudaEventElapsedTime(&far, h->pev[i][0], h->pev[i][1]);
  cudaEventElapsedTime(&steps, h->pev[i][1], h->pev[i][2]);
  h->pair_ms += far;
  h->pair_launches += 1;
  h->step_ms += steps;
  h->step_launches += h->block_step ? 1 : kTimeBlock * (h->fused ? 1 : kCorrectorSteps + 2);
  h->pending[i] = false;
  return QG_OK;
}

static qg_status launch_prof_block(qg_handle *h, int gi)
{
  if(!h->pev_ready) {
    for(auto &row : h->pev)
      for(auto &e : row) QG_CUDA(cudaEventCreate(&e));
    h->pev_ready = true;
  }
  const int i = h->prof_next;
  h->prof_next = (h->prof_next + 1) % qg_handle_s::kProfRing;
  QG_TRY(collect_prof(h, i));
  // a form's whole ring at its first use, so that the instances are made
  // while a caller warms up, not in a later timed block
  if(!h->gprof[gi][i])
    for(int j = 0; j < qg_handle_s::kProfRing; ++j)
      if(!h->gprof[gi][j]) QG_TRY(capture_block(h, gi, j, &h->gprof[gi][j]));
  QG_CUDA(cudaGraphLaunch(h->gprof[gi][i], h->stream));
  h->pending[i] = true;
  return QG_OK;
}

// The profiling events, made on first use.
static qg_status ensure_events(qg_handle *h)
{
  if(h->events_ready) return QG_OK;
  for(int i = 0; i < 256; ++i) {
    QG_CUDA(cudaEventCreate(&h->ev_a[i]));
    QG_CUDA(cudaEventCreate(&h->ev_b[i]));
    QG_CUDA(cudaEventCreate(&h->ev_c[i]));
    QG_CUDA(cudaEventCreate(&h->ev_d[i]));
  }
  h->events_ready = true;
  return QG_OK;
}

static qg_status collect_events(qg_handle *h, int nev, int nstep)
{
  if(nev > 0) {
    QG_CUDA(cudaEventSynchronize(h->ev_b[nev - 1]));
    for(int j = 0; j < nev; ++j) {
      float ms = 0;
      cudaEventElapsedTime(&ms, h->ev_a[j], h->ev_b[j]);
      h->pair_ms += ms;
    }
    h->pair_launches += nev;
  }
  if(nstep > 0) {
    QG_CUDA(cudaEventSynchronize(h->ev_d[nstep - 1]));
    for(int j = 0; j < nstep; ++j) {
      float ms = 0;
      cudaEventElapsedTime(&ms, h->ev_c[j], h->ev_d[j]);
      h->step_ms += ms;
    }
    h->step_launches += h->fused ? nstep : nstep * (kCorrectorSteps + 2);
  }
  return QG_OK;
}

// Enqueues steps [t, t + count); whole aligned blocks replay the graph.
static qg_status launch_steps(qg_handle *h, int t, int count, bool traj)
{
  int nev = 0, nstep = 0;
  if(count > 0 && t % kTimeBlock == 0) launch_set_int(h->d_ints + 0, t, h->stream);
  while(count > 0) {
    const int t0 = t - t % kTimeBlock;
    if(t == t0 && count >= kTimeBlock && h->use_graph) {
      if(h->profile) {
        QG_TRY(launch_prof_block(h, (traj ? 1 : 0) + (early_block(h, t0) ? 2 : 0)));
      } else {
        const int gi = (traj ? 1 : 0) + (early_block(h, t0) ? 2 : 0);
        QG_TRY(ensure_graph(h, gi));
        QG_CUDA(cudaGraphLaunch(h->graph[gi], h->stream));
      }
      h->far_block = t0;
      t += kTimeBlock;
      count -= kTimeBlock;
      continue;
    }
    if(h->far_block != t0) {
      enqueue_far(h, t0, t == t0, h->profile ? h->ev_a[nev] : nullptr,
                  h->profile ? h->ev_b[nev] : nullptr, early_block(h, t0));
      if(h->profile) ++nev;
      h->far_block = t0;
    }
    // the rest of this block (or of the run) in one launch when allowed
    const int span = h->block_step ? std::min(count, t0 + kTimeBlock - t) : 1;
    if(h->profile) cudaEventRecord(h->ev_c[nstep], h->stream);
    if(span > 1)
      enqueue_step_block(h, t - t0, t - t0 + span, traj);
    else
      enqueue_dot_step(h, t - t0, traj);
    if(h->profile) cudaEventRecord(h->ev_d[nstep++], h->stream);
    if(h->profile && (nev == 256 || nstep == 256)) {
      QG_TRY(collect_events(h, nev, nstep));
      nev = nstep = 0;
    }
    t += span;
    count -= span;
  }
  QG_CUDA(cudaGetLastError());
  if(h->profile) {
    QG_TRY(collect_events(h, nev, nstep));
    for(int i = 0; i < qg_handle_s::kProfRing; ++i) QG_TRY(collect_prof(h, i));
  }
  return QG_OK;
}

// ---- target sharding of one ensemble ------------------------------------------
// A shard computes the targets in its range of 32-dot blocks of the internal
// order (Morton order with every delay-0 group inside one block, so the
// current-step coupling never crosses shards) and keeps every dot's rho01
// history, which the far and mid terms read.  Coefficients are computed on the
// fly (sharding is for ensembles whose table would not fit one GPU).  A step:
// qg_shard_step computes the shard's dots and exports their new rho01; the
// caller gathers all shards' slices (NCCL all-gather, peer copies, ...) into
// the internal-order vector and hands it to qg_shard_import, which writes the
// other shards' dots into the rings exactly as their own step kernels wrote
// theirs.  Each target's sums are those of the unsharded handle, term for
// term, so a sharded run gives the unsharded run's bits.
extern "C" qg_status qg_shard_create(const qg_dot *dots, int n, const qg_pulse *pulse, const qg_params *params,
                                     const qg_weights *weights, int rank, int world, qg_handle **out)
{
  if(!out) return qg_fail(QG_ERR_INVALID_ARG, "qg_shard_create: out is NULL");
  *out = nullptr;
  if(world < 1 || rank < 0 || rank >= world)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_shard_create: rank %d outside [0, %d)", rank, world);
  QG_TRY(validate(dots, n, pulse, params));
  if(params->coef_mode == QG_COEF_TABLE)
    return qg_fail(QG_ERR_UNSUPPORTED, "qg_shard_create: shards compute their coefficients on the fly");
  qg_params p = *params;
  p.coef_mode = QG_COEF_ON_THE_FLY;
  qg_handle *h = new qg_handle();
  qg_status st = create_impl(dots, n, pulse, &p, weights, h);
  if(st == QG_OK && !h->fused)
    st = qg_fail(QG_ERR_UNSUPPORTED,
                 "qg_shard_create: a group of dots coupled at delay 0 exceeds 32; it cannot be sharded");
  if(st == QG_OK && h->step_blocks < world)
    st = qg_fail(QG_ERR_INVALID_ARG, "qg_shard_create: %d blocks of 32 dots for %d shards", h->step_blocks,
                 world);
  if(st == QG_OK) {
    h->shard_rank = rank;
    h->shard_world = world;
    h->blk_lo = (int)((long long)h->step_blocks * rank / world);
    h->blk_hi = (int)((long long)h->step_blocks * (rank + 1) / world);
    h->block_step = false;  // partners' steps come from other devices between steps
    h->use_graph = false;
    h->tune_pending = false;
    st = dalloc(h, &h->d_shard_io, (size_t)h->n_pad);
  }
  if(st != QG_OK) {
    destroy_handle(h);
    return st;
  }
  *out = h;
  return QG_OK;
}

// This shard's internal dots [*first, *first + *count) and the internal ->
// user map of all n_pad internal slots (nullable; -1 marks padding).
extern "C" qg_status qg_shard_layout(const qg_handle *h, int *first, int *count, int *n_pad, int *user)
{
  if(!h) return qg_fail(QG_ERR_INVALID_ARG, "qg_shard_layout: NULL handle");
  const int lo = h->shard_world > 1 ? h->blk_lo * kTile : 0;
  const int hi = h->shard_world > 1 ? h->blk_hi * kTile : h->n_pad;
  if(first) *first = lo;
  if(count) *count = hi - lo;
  if(n_pad) *n_pad = h->n_pad;
  if(user) {
    QG_CUDA(cudaSetDevice(h->device));
    QG_CUDA(cudaMemcpy(user, h->d_user, sizeof(int) * (size_t)h->n_pad, cudaMemcpyDeviceToHost));
  }
  return QG_OK;
}

// One step of this shard's dots (the far field at block starts, then the
// step kernel), and their new rho01 (count complex, internal order) into the
// device buffer d_slice.  Returns when d_slice is written.
extern "C" qg_status qg_shard_step(qg_handle *h, double *d_slice)
{
  if(!h || !d_slice) return qg_fail(QG_ERR_INVALID_ARG, "qg_shard_step: NULL argument");
  if(h->shard_world < 2) return qg_fail(QG_ERR_INVALID_ARG, "qg_shard_step: not a shard (qg_shard_create)");
  if(h->next_step >= h->T)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_shard_step: step %d is past num_timesteps %d", h->next_step, h->T);
  QG_CUDA(cudaSetDevice(h->device));
  h->batch_bad_valid = false;
  const int t = h->next_step, t0 = t - t % kTimeBlock;
  if(h->far_block != t0) {
    enqueue_far(h, t0, false, nullptr, nullptr, early_block(h, t0));
    h->far_block = t0;
  }
  enqueue_dot_step(h, t - t0, false);
  launch_shard_export(h->step_args(false), t, h->blk_lo * kTile, h->blk_hi * kTile, (double2 *)d_slice,
                      h->stream);
  QG_CUDA(cudaGetLastError());
  QG_CUDA(cudaStreamSynchronize(h->stream));
  return QG_OK;
}

// The step just computed by every shard: d_full holds all n_pad dots' rho01
// at that step (internal order, device memory); the other shards' dots go
// into this shard's rings, and the shard moves to the next step.
extern "C" qg_status qg_shard_import(qg_handle *h, const double *d_full)
{
  if(!h || !d_full) return qg_fail(QG_ERR_INVALID_ARG, "qg_shard_import: NULL argument");
  if(h->shard_world < 2) return qg_fail(QG_ERR_INVALID_ARG, "qg_shard_import: not a shard (qg_shard_create)");
  QG_CUDA(cudaSetDevice(h->device));
  launch_shard_import(h->step_args(false), h->next_step, h->blk_lo * kTile, h->blk_hi * kTile,
                      (const double2 *)d_full, h->stream);
  QG_CUDA(cudaGetLastError());
  QG_CUDA(cudaStreamSynchronize(h->stream));
  h->next_step += 1;
  return QG_OK;
}

extern "C" qg_status qg_run(qg_handle *h, int n_steps, double *rho_out, int *bad_step)
{
  if(!h) return qg_fail(QG_ERR_INVALID_ARG, "qg_run: NULL handle");
  if(n_steps < 0) return qg_fail(QG_ERR_INVALID_ARG, "qg_run: n_steps < 0");
  if(h->next_step + (long long)n_steps > h->T)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_run: steps [%d, %d) exceed num_timesteps %d", h->next_step,
                   h->next_step + n_steps, h->T);
  if(bad_step) *bad_step = -1;
  h->batch_bad_valid = false;
  QG_CUDA(cudaSetDevice(h->device));
  if(h->tune_pending) {
    // at any step: it only clobbers the far field and partials, which the
    // run recomputes (far_block is invalidated)
    h->tune_pending = false;
    QG_TRY(autotune_cached(h, false));
  }
  const int t_start = h->next_step;
  h->eval_cached = -0x7fffffff;
  const size_t row = (size_t)h->n * 2;  // double2 per step
  if(!rho_out) {
    QG_TRY(launch_steps(h, t_start, n_steps, false));
  } else {
    // Every step's state straight into the caller's buffer.  Chunks of
    // traj_k steps alternate between the two halves of d_traj.  Chunk c's
    // copy is issued after chunk c + 1's launches are queued: a copy into
    // pageable memory returns only when it is done, and meanwhile the device
    // computes the next chunk; chunk c + 2 waits for chunk c's copy before
    // it reuses that half.
    const int K = h->traj_k;
    const int nchunks = (n_steps + K - 1) / K;
    auto copy_out = [&](int c) -> cudaError_t {
      const int b = c & 1;
      const int k = std::min(K, n_steps - c * K);
      cudaError_t e = cudaStreamWaitEvent(h->copy_stream, h->ev_chunk[b], 0);
      if(e == cudaSuccess)
        e = cudaMemcpyAsync(rho_out + (size_t)c * K * row * 2, h->d_traj + (size_t)b * K * row,
                            sizeof(double2) * row * k, cudaMemcpyDeviceToHost, h->copy_stream);
      if(e == cudaSuccess) e = cudaEventRecord(h->ev_copy[b], h->copy_stream);
      return e;
    };
    qg_status st = QG_OK;
    cudaError_t ce = cudaSuccess;
    for(int c = 0; c < nchunks && st == QG_OK && ce == cudaSuccess; ++c) {
      const int b = c & 1;
      const int k = std::min(K, n_steps - c * K);
      if(c >= 2) ce = cudaStreamWaitEvent(h->stream, h->ev_copy[b], 0);
      if(ce != cudaSuccess) break;
      launch_set_int(h->d_ints + 3, t_start + c * K - b * K, h->stream);
      st = launch_steps(h, t_start + c * K, k, true);
      if(st != QG_OK) break;
      ce = cudaEventRecord(h->ev_chunk[b], h->stream);
      if(ce == cudaSuccess && c >= 1) ce = copy_out(c - 1);
      if(ce == cudaSuccess && c == nchunks - 1) ce = copy_out(c);
    }
    // no copy into the caller's buffer may outlive the call
    const cudaError_t ce2 = cudaStreamSynchronize(h->copy_stream);
    if(st != QG_OK) return st;
    QG_CUDA(ce);
    QG_CUDA(ce2);
  }
  int bad = kBadNone;
  QG_CUDA(cudaMemcpyAsync(&bad, h->d_ints + 2, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  QG_CUDA(cudaStreamSynchronize(h->stream));
  QG_CUDA(cudaGetLastError());
  h->next_step = t_start + n_steps;
  if(bad == -2)
    return qg_fail(QG_ERR_CUDA, "qg_run: a wait in the step-block kernel timed out");
  if(bad == -3)
    return qg_fail(QG_ERR_CUDA, "qg_run: a wait for the far kernel's bulk table copies timed out");
  if(bad < 0)
    return qg_fail(QG_ERR_CUDA, "qg_run: internal scheduling error (far block or trajectory row)");
  if(bad != kBadNone) {
    if(bad_step) *bad_step = bad;
    return qg_fail(QG_ERR_NONFINITE, "unbounded history values at or before step %d", bad);
  }
  return QG_OK;
}

// ---- batches: many ensembles advanced together -----------------------------
struct qg_batch_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  int capacity = 0;
  std::vector<qg_handle *> members;
  FarArgs *d_far = nullptr;
  StepArgs *d_step = nullptr;
  int *d_task_off = nullptr, *d_block_off = nullptr;
  int q = -1, frame = -1, n_time = -1, mixed = 0;
  int total_tasks = 0, total_blocks = 0;
  int far_grid = 0;
  bool dirty = true;
  cudaGraphExec_t graph = nullptr;
  int *d_bad_all = nullptr;  // members' first bad steps, gathered after each run
  int *h_bad_all = nullptr;  // pinned copy
  // "profile": blocks launched without the graph, CUDA events around the far
  // launch and around the block's step launches
  bool profile = false;
  // defaults measured on B200 with the 256-ensemble workload: packed FP32
  // pairs 17.1 against 19.7 ms per far launch, and the source-group-major
  // order 16.3 (mixed) and 22.5 against 23.9 ms (FP64)
  bool far_packed = true;   // mixed members: the packed FP32 convolution (same bits)
  bool far_gmajor = true;   // members' tasks in source-group-major order (same bits)
  bool mid_pipe = false;    // step launches stage mid entries several at a time (same bits)
  // the far launch's forms (far_packed x far_gmajor) are timed at the first
  // run, unless set explicitly; tuned_far_us reads the winner's time back
  bool tune_pending = true;
  float tuned_far_ms = 0;
  // "tune_group": the tuner also times source tiles per warp (1, 2, 4, 8)
  // for each size class of members (tiles < 4, < 16, < 64, more); a member
  // of a tuned class takes its class's group when the batch is rebuilt
  // (0: the member's own)
  bool tune_group = false;
  int class_group[4] = {0, 0, 0, 0};
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  double far_ms = 0, step_ms = 0;
  int far_launches = 0, step_launches = 0;
};

extern "C" qg_status qg_batch_create(int capacity, qg_batch **out)
{
  if(!out || capacity < 1) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_create: bad argument");
  *out = nullptr;
  qg_batch *b = new qg_batch();
  b->capacity = capacity;
  auto fail = [&](qg_status st) {
    if(b->d_bad_all) cudaFree(b->d_bad_all);
    if(b->h_bad_all) cudaFreeHost(b->h_bad_all);
    if(b->d_far) cudaFree(b->d_far);
    if(b->d_step) cudaFree(b->d_step);
    if(b->d_task_off) cudaFree(b->d_task_off);
    if(b->d_block_off) cudaFree(b->d_block_off);
    if(b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return st;
  };
  cudaError_t e;
  if((e = cudaGetDevice(&b->device)) != cudaSuccess ||
     (e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
     (e = cudaMalloc(&b->d_far, sizeof(FarArgs) * capacity)) != cudaSuccess ||
     (e = cudaMalloc(&b->d_step, sizeof(StepArgs) * capacity)) != cudaSuccess ||
     (e = cudaMalloc(&b->d_task_off, sizeof(int) * (capacity + 1))) != cudaSuccess ||
     (e = cudaMalloc(&b->d_block_off, sizeof(int) * (capacity + 1))) != cudaSuccess ||
     (e = cudaMalloc(&b->d_bad_all, sizeof(int) * capacity)) != cudaSuccess ||
     (e = cudaMallocHost(&b->h_bad_all, sizeof(int) * capacity)) != cudaSuccess)
    return fail(qg_fail(e == cudaErrorMemoryAllocation ? QG_ERR_OOM : QG_ERR_CUDA, "qg_batch_create: %s",
                        cudaGetErrorString(e)));
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  per_sm = 3;  // persistent far grid: 3 blocks of 4 warps per SM (measured best)
  b->far_grid = std::max(1, sms * per_sm);
  *out = b;
  return QG_OK;
}

extern "C" qg_status qg_batch_destroy(qg_batch *b)
{
  if(!b) return QG_OK;
  cudaStreamSynchronize(b->stream);
  if(b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->d_far);
  cudaFree(b->d_step);
  cudaFree(b->d_task_off);
  cudaFree(b->d_block_off);
  cudaFree(b->d_bad_all);
  cudaFreeHost(b->h_bad_all);
  for(auto e : b->ev)
    if(e) cudaEventDestroy(e);
  cudaStreamDestroy(b->stream);
  delete b;
  return QG_OK;
}

extern "C" qg_status qg_batch_add(qg_batch *b, qg_handle *h)
{
  if(!b || !h) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_add: NULL argument");
  if((int)b->members.size() >= b->capacity)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_add: batch is full (%d members)", b->capacity);
  if(std::find(b->members.begin(), b->members.end(), h) != b->members.end())
    return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_add: handle already in the batch");
  if(h->device != b->device) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_add: handle on another device");
  if(!h->fused)
    return qg_fail(QG_ERR_UNSUPPORTED,
                   "qg_batch_add: a group of dots coupled at delay 0 exceeds 32; run this handle alone");
  if(h->otf)
    return qg_fail(QG_ERR_UNSUPPORTED,
                   "qg_batch_add: the handle computes its coefficients on the fly; run it alone");
  if(h->next_step % kTimeBlock != 0)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_add: next step %d is not a multiple of %d", h->next_step,
                   kTimeBlock);
  if(!b->members.empty() && (h->q != b->q || h->params.frame != b->frame || h->w.n_time != b->n_time ||
                             (int)h->mixed != b->mixed))
    return qg_fail(QG_ERR_INVALID_ARG,
                   "qg_batch_add: members must share interpolation order, frame, history width and precision");
  b->q = h->q;
  b->mixed = (int)h->mixed;
  b->frame = h->params.frame;
  b->n_time = h->w.n_time;
  // the member's device state must name the next block's first step
  QG_CUDA(cudaStreamSynchronize(h->stream));
  launch_set_int(h->d_ints + 0, h->next_step, b->stream);
  b->members.push_back(h);
  b->dirty = true;
  return QG_OK;
}

extern "C" qg_status qg_batch_remove(qg_batch *b, qg_handle *h)
{
  if(!b || !h) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_remove: NULL argument");
  auto it = std::find(b->members.begin(), b->members.end(), h);
  if(it == b->members.end()) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_remove: handle not in the batch");
  QG_CUDA(cudaStreamSynchronize(b->stream));
  b->members.erase(it);
  b->dirty = true;
  return QG_OK;
}

static int size_class(int nT) { return nT < 4 ? 0 : nT < 16 ? 1 : nT < 64 ? 2 : 3; }

static void drop_graphs(qg_handle *h)
{
  for(auto &g : h->graph)
    if(g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  for(auto &row : h->gprof)
    for(auto &g : row)
      if(g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
}

static qg_status batch_rebuild(qg_batch *b)
{
  const int n = (int)b->members.size();
  if(b->tune_group)
    for(qg_handle *h : b->members) {
      const int g = b->class_group[size_class(h->nT)];
      if(g > 0 && g != h->group && !h->otf && (h->nT + g - 1) / g <= h->max_groups) {
        h->group = g;
        h->nG = (h->nT + g - 1) / g;
        h->far_block = -0x7fffffff;
        drop_graphs(h);
      }
    }
  // members with the longest mid lists per 32-dot block first: the step
  // launches' blocks are dispatched about in index order and those blocks
  // take longest, so starting them first shortens the launch's tail (the
  // order changes no member's arithmetic)
  std::stable_sort(b->members.begin(), b->members.end(), [](const qg_handle *x, const qg_handle *y) {
    return x->mid_pairs * y->step_blocks > y->mid_pairs * x->step_blocks;
  });
  std::vector<FarArgs> fa(n);
  std::vector<StepArgs> sa(n);
  std::vector<int> toff(n + 1, 0), boff(n + 1, 0);
  for(int e = 0; e < n; ++e) {
    qg_handle *h = b->members[e];
    fa[e] = h->far_args(h->d_ints + 0, h->d_ints + 6);
    fa[e].gmajor = b->far_gmajor ? 1 : 0;
    sa[e] = h->step_args(false);
    toff[e + 1] = toff[e] + h->nT * h->nG;
    boff[e + 1] = boff[e] + h->step_blocks;
  }
  b->total_tasks = toff[n];
  b->total_blocks = boff[n];
  if(n > 0) {
    QG_CUDA(cudaMemcpyAsync(b->d_far, fa.data(), sizeof(FarArgs) * n, cudaMemcpyHostToDevice, b->stream));
    QG_CUDA(cudaMemcpyAsync(b->d_step, sa.data(), sizeof(StepArgs) * n, cudaMemcpyHostToDevice, b->stream));
  }
  QG_CUDA(cudaMemcpyAsync(b->d_task_off, toff.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, b->stream));
  QG_CUDA(cudaMemcpyAsync(b->d_block_off, boff.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, b->stream));
  QG_CUDA(cudaStreamSynchronize(b->stream));
  if(b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  if(n > 0) {
    cudaGraph_t g;
    QG_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    launch_far_batch(b->d_far, b->d_task_off, n, b->q, b->frame, b->mixed ? (b->far_packed ? 2 : 1) : 0,
                     b->far_grid, b->stream);
    for(int k = 0; k < kTimeBlock; ++k)
      launch_step_batch(b->d_step, b->d_block_off, n, b->total_blocks, b->n_time, k, b->mid_pipe, b->stream);
    QG_CUDA(cudaStreamEndCapture(b->stream, &g));
    QG_CUDA(cudaGraphInstantiate(&b->graph, g, 0));
    cudaGraphDestroy(g);
  }
  b->dirty = false;
  return QG_OK;
}

// The batch's autotuner: its far launch in each of the forms that sum the
// same terms (mixed: scalar or packed FP32 pairs; both: target-tile or
// source-group-major task order), one untimed and two timed launches each,
// the fastest kept.  The launch recomputes the far field of every member's
// next block from history the run has not touched yet, so timing it changes
// nothing the run then computes.
static qg_status batch_autotune(qg_batch *b)
{
  b->tune_pending = false;
  const int n = (int)b->members.size();
  cudaEvent_t e0, e1;
  QG_CUDA(cudaEventCreate(&e0));
  QG_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  bool best_p = b->far_packed, best_g = b->far_gmajor;
  for(int packed = 0; packed < (b->mixed ? 2 : 1); ++packed)
    for(int gmajor = 0; gmajor < 2; ++gmajor) {
      b->far_packed = packed != 0;
      b->far_gmajor = gmajor != 0;
      QG_TRY(batch_rebuild(b));  // the members' FarArgs carry the task order
      float t = 1e30f;
      for(int r = 0; r < 3; ++r) {
        QG_CUDA(cudaEventRecord(e0, b->stream));
        launch_far_batch(b->d_far, b->d_task_off, n, b->q, b->frame, b->mixed ? (b->far_packed ? 2 : 1) : 0,
                         b->far_grid, b->stream);
        QG_CUDA(cudaEventRecord(e1, b->stream));
        QG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        QG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if(r > 0) t = std::min(t, ms);
      }
      if(t < best) {
        best = t;
        best_p = b->far_packed;
        best_g = b->far_gmajor;
      }
    }
  b->far_packed = best_p;
  b->far_gmajor = best_g;
  if(b->tune_group) {
    // one pass over the size classes present, each keeping the group that
    // made the whole launch fastest with the others fixed
    bool present[4] = {false, false, false, false};
    for(const qg_handle *h : b->members) present[size_class(h->nT)] = true;
    for(int c = 0; c < 4; ++c) {
      if(!present[c]) continue;
      int best_c = b->class_group[c];
      for(int g : {1, 2, 4, 8}) {
        b->class_group[c] = g;
        QG_TRY(batch_rebuild(b));
        float t = 1e30f;
        for(int r = 0; r < 3; ++r) {
          QG_CUDA(cudaEventRecord(e0, b->stream));
          launch_far_batch(b->d_far, b->d_task_off, n, b->q, b->frame, b->mixed ? (b->far_packed ? 2 : 1) : 0,
                           b->far_grid, b->stream);
          QG_CUDA(cudaEventRecord(e1, b->stream));
          QG_CUDA(cudaEventSynchronize(e1));
          float ms = 0;
          QG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          if(r > 0) t = std::min(t, ms);
        }
        if(t < best) {
          best = t;
          best_c = g;
        }
      }
      b->class_group[c] = best_c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->tuned_far_ms = best;
  return batch_rebuild(b);
}

extern "C" qg_status qg_batch_run(qg_batch *b, int n_blocks)
{
  if(!b || n_blocks < 0) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_run: bad argument");
  QG_CUDA(cudaSetDevice(b->device));
  if(b->dirty) QG_TRY(batch_rebuild(b));
  if(b->members.empty()) return QG_OK;
  if(b->tune_pending && n_blocks > 0) QG_TRY(batch_autotune(b));
  const int nm0 = (int)b->members.size();
  for(int i = 0; i < n_blocks; ++i) {
    if(!b->profile) {
      QG_CUDA(cudaGraphLaunch(b->graph, b->stream));
      continue;
    }
    // the graph's kernels one by one, timed
    QG_CUDA(cudaEventRecord(b->ev[0], b->stream));
    launch_far_batch(b->d_far, b->d_task_off, nm0, b->q, b->frame, b->mixed ? (b->far_packed ? 2 : 1) : 0,
                     b->far_grid, b->stream);
    QG_CUDA(cudaEventRecord(b->ev[1], b->stream));
    for(int k = 0; k < kTimeBlock; ++k)
      launch_step_batch(b->d_step, b->d_block_off, nm0, b->total_blocks, b->n_time, k, b->mid_pipe, b->stream);
    QG_CUDA(cudaEventRecord(b->ev[2], b->stream));
    QG_CUDA(cudaEventSynchronize(b->ev[2]));
    float f = 0, g = 0;
    QG_CUDA(cudaEventElapsedTime(&f, b->ev[0], b->ev[1]));
    QG_CUDA(cudaEventElapsedTime(&g, b->ev[1], b->ev[2]));
    b->far_ms += f;
    b->step_ms += g;
    b->far_launches += 1;
    b->step_launches += kTimeBlock;
  }
  // every member's first bad step in one copy, so a caller can retire a
  // member that went non-finite without a device round trip per member
  const int nm = (int)b->members.size();
  launch_gather_bad(b->d_step, nm, b->d_bad_all, b->stream);
  QG_CUDA(cudaMemcpyAsync(b->h_bad_all, b->d_bad_all, sizeof(int) * nm, cudaMemcpyDeviceToHost, b->stream));
  QG_CUDA(cudaStreamSynchronize(b->stream));
  QG_CUDA(cudaGetLastError());
  for(int e = 0; e < nm; ++e) {
    qg_handle *h = b->members[e];
    const int start = h->next_step;
    h->next_step = std::min(h->T, start + n_blocks * kTimeBlock);
    h->far_block = start + (n_blocks - 1) * kTimeBlock;
    h->eval_cached = -0x7fffffff;
    h->batch_bad = b->h_bad_all[e];
    h->batch_bad_valid = true;
  }
  return QG_OK;
}

extern "C" qg_status qg_batch_set_option(qg_batch *b, const char *key, int value)
{
  if(!b || !key) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_set_option: NULL argument");
  if(!std::strcmp(key, "profile")) {
    QG_CUDA(cudaSetDevice(b->device));
    for(auto &e : b->ev)
      if(!e) QG_CUDA(cudaEventCreate(&e));
    b->profile = value != 0;
    return QG_OK;
  }
  if(!std::strcmp(key, "far_packed")) {
    b->far_packed = value != 0;
    b->dirty = true;  // the block graph holds the kernel
    b->tune_pending = false;  // an explicit choice is kept
    return QG_OK;
  }
  if(!std::strcmp(key, "far_gmajor")) {
    b->far_gmajor = value != 0;
    b->dirty = true;
    b->tune_pending = false;
    return QG_OK;
  }
  if(!std::strcmp(key, "autotune")) {
    b->tune_pending = value != 0;
    return QG_OK;
  }
  if(!std::strcmp(key, "mid_pipe")) {
    b->mid_pipe = value != 0;
    b->dirty = true;
    return QG_OK;
  }
  if(!std::strcmp(key, "tune_group")) {
    b->tune_group = value != 0;
    if(b->tune_group) b->tune_pending = true;
    b->dirty = true;
    return QG_OK;
  }
  return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_set_option: unknown key '%s'", key);
}

extern "C" qg_status qg_batch_get_option(const qg_batch *b, const char *key, int *value)
{
  if(!b || !key || !value) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_get_option: NULL argument");
  if(!std::strcmp(key, "far_packed"))
    *value = b->far_packed ? 1 : 0;
  else if(!std::strcmp(key, "far_gmajor"))
    *value = b->far_gmajor ? 1 : 0;
  else if(!std::strcmp(key, "mid_pipe"))
    *value = b->mid_pipe ? 1 : 0;
  else if(!std::strcmp(key, "profile"))
    *value = b->profile ? 1 : 0;
  else if(!std::strcmp(key, "tuned_far_us"))
    *value = (int)(b->tuned_far_ms * 1000.0f + 0.5f);
  else if(!std::strcmp(key, "tune_group"))
    *value = b->tune_group ? 1 : 0;
  else if(!std::strncmp(key, "far_group_class", 15) && key[15] >= '0' && key[15] <= '3' && !key[16])
    *value = b->class_group[key[15] - '0'];
  else
    return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_get_option: unknown key '%s'", key);
  return QG_OK;
}

extern "C" qg_status qg_batch_kernel_time(qg_batch *b, int reset, double *far_ms, int *far_launches,
                                          double *step_ms, int *step_launches)
{
  if(!b) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_kernel_time: NULL batch");
  if(far_ms) *far_ms = b->far_ms;
  if(far_launches) *far_launches = b->far_launches;
  if(step_ms) *step_ms = b->step_ms;
  if(step_launches) *step_launches = b->step_launches;
  if(reset) {
    b->far_ms = b->step_ms = 0;
    b->far_launches = b->step_launches = 0;
  }
  return QG_OK;
}

extern "C" qg_status qg_batch_size(const qg_batch *b, int *members, int *tasks, int *blocks)
{
  if(!b) return qg_fail(QG_ERR_INVALID_ARG, "qg_batch_size: NULL batch");
  if(members) *members = (int)b->members.size();
  if(tasks) *tasks = b->total_tasks;
  if(blocks) *blocks = b->total_blocks;
  return QG_OK;
}

extern "C" qg_status qg_bad_step(qg_handle *h, int *bad_step)
{
  if(!h || !bad_step) return qg_fail(QG_ERR_INVALID_ARG, "qg_bad_step: NULL argument");
  int bad = kBadNone;
  if(h->batch_bad_valid) {
    bad = h->batch_bad;
  } else {
    QG_CUDA(cudaSetDevice(h->device));
    QG_CUDA(cudaMemcpy(&bad, h->d_ints + 2, sizeof(int), cudaMemcpyDeviceToHost));
  }
  *bad_step = bad == kBadNone ? -1 : bad;
  return QG_OK;
}

extern "C" qg_status qg_get_state(qg_handle *h, double *rho_out)
{
  if(!h || !rho_out) return qg_fail(QG_ERR_INVALID_ARG, "qg_get_state: NULL argument");
  QG_CUDA(cudaSetDevice(h->device));
  QG_CUDA(cudaStreamSynchronize(h->stream));
  launch_state_read(h->step_args(true), h->next_step - 1, h->d_traj, h->stream);
  QG_CUDA(cudaGetLastError());
  QG_CUDA(cudaMemcpyAsync(rho_out, h->d_traj, sizeof(double2) * 2 * (size_t)h->n, cudaMemcpyDeviceToHost,
                          h->stream));
  QG_CUDA(cudaStreamSynchronize(h->stream));
  return QG_OK;
}

// ---- checkpoint / resume ------------------------------------------------------
// A checkpoint is the integrator's device state after step next_step - 1:
// the rho01 ring (and, in mixed precision, the FP32 rings), the 23-step
// predictor-corrector window, the next step and the first non-finite step.
// The coefficient table and lists are not part of it: they follow from the
// inputs, so a checkpoint is loaded into a handle created from the same
// dots, pulse and parameters.  Resuming gives the same bits as not stopping
// (a far block is recomputed from history that the steps after its start do
// not touch).
struct CheckpointHeader {
  char magic[8];
  int version, n, n_pad, q, W, stride, mixed, next_step, T, bad;
  double dt, c0;
  unsigned long long ring_bytes, ring32_bytes, pcr_bytes;
};

static void checkpoint_header(const qg_handle *h, CheckpointHeader &hd)
{
  std::memset(&hd, 0, sizeof hd);
  std::memcpy(hd.magic, "QGCKPT\0", 8);
  hd.version = 1;
  hd.n = h->n;
  hd.n_pad = h->n_pad;
  hd.q = h->q;
  hd.W = h->W;
  hd.stride = h->stride;
  hd.mixed = h->mixed ? 1 : 0;
  hd.next_step = h->next_step;
  hd.T = h->T;
  hd.dt = h->params.dt;
  hd.c0 = h->params.c0;
  hd.ring_bytes = sizeof(double2) * (unsigned long long)h->n_pad * h->stride;
  hd.ring32_bytes = h->mixed ? sizeof(float2) * (unsigned long long)h->n_pad * h->stride : 0;
  hd.pcr_bytes = sizeof(double2) * (unsigned long long)kPcDepth * 4 * h->n_pad;
}

extern "C" qg_status qg_checkpoint_size(const qg_handle *h, size_t *bytes)
{
  if(!h || !bytes) return qg_fail(QG_ERR_INVALID_ARG, "qg_checkpoint_size: NULL argument");
  CheckpointHeader hd;
  checkpoint_header(h, hd);
  *bytes = sizeof hd + hd.ring_bytes + 2 * hd.ring32_bytes + hd.pcr_bytes;
  return QG_OK;
}

extern "C" qg_status qg_checkpoint_save(qg_handle *h, void *buf, size_t bytes)
{
  if(!h || !buf) return qg_fail(QG_ERR_INVALID_ARG, "qg_checkpoint_save: NULL argument");
  size_t need = 0;
  QG_TRY(qg_checkpoint_size(h, &need));
  if(bytes < need) return qg_fail(QG_ERR_INVALID_ARG, "qg_checkpoint_save: buffer of %zu bytes, need %zu", bytes, need);
  QG_CUDA(cudaSetDevice(h->device));
  CheckpointHeader hd;
  checkpoint_header(h, hd);
  QG_CUDA(cudaMemcpyAsync(&hd.bad, h->d_ints + 2, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  char *p = static_cast<char *>(buf) + sizeof hd;
  QG_CUDA(cudaMemcpyAsync(p, h->d_ring, hd.ring_bytes, cudaMemcpyDeviceToHost, h->stream));
  p += hd.ring_bytes;
  if(h->mixed) {
    QG_CUDA(cudaMemcpyAsync(p, h->d_ring32w, hd.ring32_bytes, cudaMemcpyDeviceToHost, h->stream));
    p += hd.ring32_bytes;
    QG_CUDA(cudaMemcpyAsync(p, h->d_ring32d, hd.ring32_bytes, cudaMemcpyDeviceToHost, h->stream));
    p += hd.ring32_bytes;
  }
  QG_CUDA(cudaMemcpyAsync(p, h->d_pcr, hd.pcr_bytes, cudaMemcpyDeviceToHost, h->stream));
  QG_CUDA(cudaStreamSynchronize(h->stream));
  std::memcpy(buf, &hd, sizeof hd);
  return QG_OK;
}

extern "C" qg_status qg_checkpoint_load(qg_handle *h, const void *buf, size_t bytes)
{
  if(!h || !buf) return qg_fail(QG_ERR_INVALID_ARG, "qg_checkpoint_load: NULL argument");
  CheckpointHeader hd, mine;
  if(bytes < sizeof hd) return qg_fail(QG_ERR_INVALID_ARG, "qg_checkpoint_load: buffer too small");
  std::memcpy(&hd, buf, sizeof hd);
  checkpoint_header(h, mine);
  if(std::memcmp(hd.magic, mine.magic, 8) != 0 || hd.version != 1)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_checkpoint_load: not a checkpoint of this library");
  if(hd.n != mine.n || hd.n_pad != mine.n_pad || hd.q != mine.q || hd.W != mine.W || hd.stride != mine.stride ||
     hd.mixed != mine.mixed || hd.T != mine.T || hd.dt != mine.dt || hd.c0 != mine.c0)
    return qg_fail(QG_ERR_INVALID_ARG,
                   "qg_checkpoint_load: checkpoint of another configuration (N %d, q %d, W %d, precision %d, T %d; "
                   "this handle: N %d, q %d, W %d, precision %d, T %d)",
                   hd.n, hd.q, hd.W, hd.mixed, hd.T, mine.n, mine.q, mine.W, mine.mixed, mine.T);
  if(hd.next_step < 0 || hd.next_step > hd.T)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_checkpoint_load: step %d outside [0, %d]", hd.next_step, hd.T);
  const size_t need = sizeof hd + hd.ring_bytes + 2 * hd.ring32_bytes + hd.pcr_bytes;
  if(bytes < need) return qg_fail(QG_ERR_INVALID_ARG, "qg_checkpoint_load: buffer of %zu bytes, need %zu", bytes, need);
  h->batch_bad_valid = false;
  QG_CUDA(cudaSetDevice(h->device));
  for(int i = 0; i < qg_handle_s::kProfRing; ++i) QG_TRY(collect_prof(h, i));
  const char *p = static_cast<const char *>(buf) + sizeof hd;
  QG_CUDA(cudaMemcpyAsync(h->d_ring, p, hd.ring_bytes, cudaMemcpyHostToDevice, h->stream));
  p += hd.ring_bytes;
  if(h->mixed) {
    QG_CUDA(cudaMemcpyAsync(h->d_ring32w, p, hd.ring32_bytes, cudaMemcpyHostToDevice, h->stream));
    p += hd.ring32_bytes;
    QG_CUDA(cudaMemcpyAsync(h->d_ring32d, p, hd.ring32_bytes, cudaMemcpyHostToDevice, h->stream));
    p += hd.ring32_bytes;
  }
  QG_CUDA(cudaMemcpyAsync(h->d_pcr, p, hd.pcr_bytes, cudaMemcpyHostToDevice, h->stream));
  QG_CUDA(cudaMemcpyAsync(h->d_ints + 2, &hd.bad, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  QG_CUDA(cudaStreamSynchronize(h->stream));
  h->next_step = hd.next_step;
  h->far_block = -0x7fffffff;
  h->eval_cached = -0x7fffffff;
  return QG_OK;
}

extern "C" qg_status qg_next_step(const qg_handle *h, int *step)
{
  if(!h || !step) return qg_fail(QG_ERR_INVALID_ARG, "qg_next_step: NULL argument");
  *step = h->next_step;
  return QG_OK;
}

// The pinned staging of evaluate and the history copies, made on first use
// (a pinned allocation costs about a millisecond; most handles never need it).
static qg_status ensure_h_io(qg_handle *h)
{
  if(!h->h_io) QG_CUDA(cudaMallocHost((void **)&h->h_io, sizeof(double2) * (size_t)h->n));
  return QG_OK;
}

static qg_status upload_io(qg_handle *h, const double *src)
{
  QG_TRY(ensure_h_io(h));
  std::memcpy(h->h_io, src, sizeof(double2) * h->n);
  QG_CUDA(cudaMemcpyAsync(h->d_io, h->h_io, sizeof(double2) * h->n, cudaMemcpyHostToDevice, h->stream));
  return QG_OK;
}

static qg_status download_io(qg_handle *h, double *dst)
{
  QG_TRY(ensure_h_io(h));
  QG_CUDA(cudaMemcpyAsync(h->h_io, h->d_io, sizeof(double2) * h->n, cudaMemcpyDeviceToHost, h->stream));
  QG_CUDA(cudaStreamSynchronize(h->stream));
  std::memcpy(dst, h->h_io, sizeof(double2) * h->n);
  return QG_OK;
}

extern "C" qg_status qg_history_evaluate(qg_handle *h, int step, const double *rho01_step,
                                         double *field_out)
{
  if(!h || !field_out) return qg_fail(QG_ERR_INVALID_ARG, "qg_history_evaluate: NULL argument");
  if(step < 0 || step >= std::max(h->T, 1))
    return qg_fail(QG_ERR_INVALID_ARG, "qg_history_evaluate: step %d outside [0, %d)", step, h->T);
  QG_CUDA(cudaSetDevice(h->device));
  StepArgs a = h->step_args(true);
  if(rho01_step) {
    QG_TRY(upload_io(h, rho01_step));
    launch_ring_write(a, step, h->d_io, h->stream);
    launch_ring32_rebuild(a, h->stream);
  }
  if(h->eval_cached != step) {
    // the far partials of [step, step + K) in the run's buffer
    launch_set_int(h->d_ints + 4, step, h->stream);
    launch_far(h->far_args(h->d_ints + 4, h->d_ints + 8), h->stream);
    h->eval_cached = step;
    h->far_block = -0x7fffffff;
  }
  a.far_t0 = h->d_ints + 4;
  launch_eval_field(a, h->d_ints + 4, h->d_io, h->stream);
  QG_CUDA(cudaGetLastError());
  return download_io(h, field_out);
}

extern "C" qg_status qg_history_evaluate_noalloc(qg_handle *h, int step, const double *d_rho01_step,
                                                 double *d_field_out, void *stream)
{
  if(!h || !d_field_out)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_history_evaluate_noalloc: NULL handle or output");
  if(step < 0 || step >= std::max(h->T, 1))
    return qg_fail(QG_ERR_INVALID_ARG, "qg_history_evaluate_noalloc: step %d outside [0, %d)", step, h->T);
  if(h->otf)
    return qg_fail(QG_ERR_UNSUPPORTED,
                   "qg_history_evaluate_noalloc: the handle computes its coefficients on the fly; "
                   "use qg_history_evaluate");
  if(h->n_pad > kNoAllocMaxDots)
    return qg_fail(QG_ERR_INVALID_ARG,
                   "qg_history_evaluate_noalloc: %d dots (%d padded) exceed the fixed scratch, "
                   "which holds at most %d padded dots; use qg_history_evaluate",
                   h->n, h->n_pad, kNoAllocMaxDots);
  QG_CUDA(cudaSetDevice(h->device));
  NoAllocScratch sc;
  QG_TRY(noalloc_scratch(&sc));
  cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
  StepArgs a = h->step_args(true);
  if(d_rho01_step) {
    launch_ring_write(a, step, (const double2 *)d_rho01_step, s);
    launch_ring32_rebuild(a, s);
    h->eval_cached = -0x7fffffff;
    h->far_block = -0x7fffffff;
  }
  // the completion counters must start at zero; the rest is overwritten
  QG_CUDA(cudaMemsetAsync(sc.tile_done, 0, sc.tile_bytes, s));
  launch_set_int(sc.ints + 0, step, s);
  FarArgs fa = h->far_args(sc.ints + 0, sc.ints + 1);
  fa.group = kTileGroup;  // the fixed scratch holds the partials of this group size
  fa.nG = (h->nT + kTileGroup - 1) / kTileGroup;
  fa.partial = sc.partial;
  fa.field = sc.field;
  fa.tile_done = sc.tile_done;
  launch_far_step1(fa, s);
  a.far_field = sc.field;
  a.far_t0 = sc.ints + 0;
  launch_eval_field(a, sc.ints + 0, (double2 *)d_field_out, s);
  QG_CUDA(cudaGetLastError());
  return QG_OK;
}

extern "C" qg_status qg_pulse_evaluate(qg_handle *h, int step, double *field_out)
{
  if(!h || !field_out) return qg_fail(QG_ERR_INVALID_ARG, "qg_pulse_evaluate: NULL argument");
  QG_CUDA(cudaSetDevice(h->device));
  launch_pulse_field(h->step_args(true), step, h->d_io, h->stream);
  QG_CUDA(cudaGetLastError());
  return download_io(h, field_out);
}

extern "C" qg_status qg_set_history(qg_handle *h, int t0, int n, const double *rho01)
{
  if(!h || (n > 0 && !rho01)) return qg_fail(QG_ERR_INVALID_ARG, "qg_set_history: NULL argument");
  if(t0 < -kWindow || n < 0)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_set_history: t0 = %d < -%d or n < 0", t0, kWindow);
  QG_CUDA(cudaSetDevice(h->device));
  StepArgs a = h->step_args(true);
  for(int k = 0; k < n; ++k) {
    QG_TRY(upload_io(h, rho01 + (size_t)k * h->n * 2));
    launch_ring_write(a, t0 + k, h->d_io, h->stream);
    QG_CUDA(cudaStreamSynchronize(h->stream));
  }
  launch_ring32_rebuild(a, h->stream);
  QG_CUDA(cudaGetLastError());
  // the history is complete when the call returns, so work the caller
  // enqueues on another stream (qg_history_evaluate_noalloc) sees all of it
  QG_CUDA(cudaStreamSynchronize(h->stream));
  h->eval_cached = -0x7fffffff;
  h->far_block = -0x7fffffff;
  return QG_OK;
}

extern "C" qg_status qg_get_history(qg_handle *h, int t0, int n, double *rho01_out)
{
  if(!h || (n > 0 && !rho01_out)) return qg_fail(QG_ERR_INVALID_ARG, "qg_get_history: NULL argument");
  if(n < 0 || n > h->W || t0 < -kWindow)
    return qg_fail(QG_ERR_INVALID_ARG, "qg_get_history: need -22 <= t0 and 0 <= n <= %d", h->W);
  QG_CUDA(cudaSetDevice(h->device));
  StepArgs a = h->step_args(true);
  for(int k = 0; k < n; ++k) {
    launch_ring_read(a, t0 + k, h->d_io, h->stream);
    QG_TRY(download_io(h, rho01_out + (size_t)k * h->n * 2));
  }
  return QG_OK;
}

extern "C" qg_status qg_get_info(const qg_handle *h, qg_info *info)
{
  if(!h || !info) return qg_fail(QG_ERR_INVALID_ARG, "qg_get_info: NULL argument");
  std::memset(info, 0, sizeof *info);
  info->n = h->n;
  info->max_delay = h->max_delay;
  info->ring_depth = h->W;
  info->num_pairs = h->P;
  info->near_pairs = h->near_pairs;
  info->mid_pairs = h->mid_pairs;
  info->time_block = kTimeBlock;
  info->coef_mode = h->otf ? QG_COEF_ON_THE_FLY : QG_COEF_TABLE;
  info->precision = h->mixed ? QG_PREC_MIXED : QG_PREC_FP64;
  info->fused_step = h->fused ? (h->block_step ? 2 : 1) : 0;
  info->device_bytes = h->bytes;
  info->table_build_ms = h->table_ms;
  return QG_OK;
}

extern "C" qg_status qg_footprint(int n, const qg_params *p, double side, size_t *bytes)
{
  if(!p || !bytes || n < 1) return qg_fail(QG_ERR_INVALID_ARG, "qg_footprint: bad argument");
  const int nT = (n + kTile - 1) / kTile, n_pad = nT * kTile;
  const bool otf = p->coef_mode == QG_COEF_ON_THE_FLY;
  const int group = otf ? (nT + 15) / 16 : far_group(p->precision == QG_PREC_MIXED, nT);
  const int nG = otf ? (nT + group - 1) / group : (nT <= 512 ? nT : (nT + group - 1) / group);
  const int q = p->interpolation_order;
  const int md = (int)std::floor(side * std::sqrt(3.0) / (p->c0 * p->dt));
  const int W = ring_depth(md, q);
  const bool mixed = p->precision == QG_PREC_MIXED;
  size_t b = otf ? 0 : table_bytes(nT, q, mixed);
  b += sizeof(double2) * (size_t)n_pad * (W + kRingMirror) * (mixed ? 2 : 1);
  b += sizeof(double2) * (size_t)kPcDepth * 4 * n_pad;
  b += sizeof(double2) * (size_t)kTimeBlock * (nG + 1) * n_pad + sizeof(unsigned) * nT;
  b += sizeof(double2) * (size_t)n_pad * 8;
  b += sizeof(double) * (size_t)n_pad * 9 + sizeof(int) * (size_t)n_pad * 2;
  const long long K = traj_steps(n);
  b += sizeof(double2) * (size_t)(2 * K * n * 2) + sizeof(double2) * (size_t)n;  // trajectory + io staging
  *bytes = b;
  return QG_OK;
}

extern "C" void *qg_stream(qg_handle *h) { return h ? (void *)h->stream : nullptr; }

extern "C" qg_status qg_kernel_time(qg_handle *h, int reset, double *pair_ms, int *pair_launches,
                                    double *step_ms, int *step_launches)
{
  if(!h) return qg_fail(QG_ERR_INVALID_ARG, "qg_kernel_time: NULL handle");
  if(pair_ms) *pair_ms = h->pair_ms;
  if(pair_launches) *pair_launches = h->pair_launches;
  if(step_ms) *step_ms = h->step_ms;
  if(step_launches) *step_launches = h->step_launches;
  if(reset) {
    h->pair_ms = h->step_ms = 0;
    h->pair_launches = h->step_launches = 0;
  }
  return QG_OK;
}

extern "C" qg_status qg_set_option(qg_handle *h, const char *key, int value)
{
  if(!h || !key) return qg_fail(QG_ERR_INVALID_ARG, "qg_set_option: NULL argument");
  if(!std::strcmp(key, "graph")) {
    h->use_graph = value != 0;
  } else if(!std::strcmp(key, "profile")) {
    if(value) QG_TRY(ensure_events(h));
    h->profile = value != 0;
  } else if(!std::strcmp(key, "far_variant") || !std::strcmp(key, "block_step") ||
            !std::strcmp(key, "far_group") || !std::strcmp(key, "wait_limit") ||
            !std::strcmp(key, "test_skip_post") || !std::strcmp(key, "tune_group") ||
            !std::strcmp(key, "far_early")) {
    if(!std::strcmp(key, "far_early")) {
      h->far_early = value != 0;
    } else if(!std::strcmp(key, "tune_group")) {
      if(h->otf) return qg_fail(QG_ERR_UNSUPPORTED, "qg_set_option: tune_group is for table handles");
      h->tune_group = value != 0;
      if(h->tune_group) h->tune_pending = true;  // the next run times the groups
    } else if(!std::strcmp(key, "wait_limit")) {
      if(value < 0) return qg_fail(QG_ERR_INVALID_ARG, "qg_set_option: wait_limit >= 0 (0: the default)");
      h->spin_limit = value;
    } else if(!std::strcmp(key, "test_skip_post")) {
      if(value < -1 || value >= std::max(h->step_blocks, 1))
        return qg_fail(QG_ERR_INVALID_ARG, "qg_set_option: test_skip_post in -1 .. %d", h->step_blocks - 1);
      h->skip_post = value;
    } else if(!std::strcmp(key, "far_group")) {
      if(h->otf || value < 1 || (h->nT + value - 1) / value > h->max_groups)
        return qg_fail(QG_ERR_INVALID_ARG, "qg_set_option: far_group %d not available (table handles, "
                       "at least %d)", value, (h->nT + h->max_groups - 1) / std::max(h->max_groups, 1));
      h->group = value;
      h->nG = (h->nT + value - 1) / value;
    } else if(!std::strcmp(key, "far_variant")) {
      if(value < 0 || value > 11) return qg_fail(QG_ERR_INVALID_ARG, "qg_set_option: far_variant in 0..11");
      h->far_variant = value;
      h->tune_pending = false;  // an explicit choice is kept
    } else {
      if(value && !h->block_step_ok)
        return qg_fail(QG_ERR_UNSUPPORTED, "qg_set_option: block_step needs the fused form with all %d "
                       "blocks resident", h->step_blocks);
      h->block_step = value != 0;
    }
    for(auto &g : h->graph)
      if(g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
    for(int i = 0; i < qg_handle_s::kProfRing; ++i) QG_TRY(collect_prof(h, i));
    for(auto &row : h->gprof)
      for(auto &g : row)
        if(g) {
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
  } else if(!std::strcmp(key, "reset")) {
    return reset_state(h);
  } else if(!std::strcmp(key, "autotune")) {
    // clobbers the far field and partials: only between runs on a block
    // boundary (the next run recomputes them)
    if(h->next_step % kTimeBlock != 0)
      return qg_fail(QG_ERR_INVALID_ARG, "qg_set_option: autotune only at a block boundary (next step %d)",
                     h->next_step);
    if(value) {
      for(int i = 0; i < qg_handle_s::kProfRing; ++i) QG_TRY(collect_prof(h, i));
      h->tune_pending = false;
      QG_TRY(autotune_cached(h, true));
      for(auto &g : h->graph)
        if(g) {
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
      for(auto &row : h->gprof)
        for(auto &g : row)
          if(g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
          }
    }
  } else {
    return qg_fail(QG_ERR_INVALID_ARG, "qg_set_option: unknown key '%s'", key);
  }
  return QG_OK;
}

extern "C" qg_status qg_get_option(const qg_handle *h, const char *key, int *value)
{
  if(!h || !key || !value) return qg_fail(QG_ERR_INVALID_ARG, "qg_get_option: NULL argument");
  if(!std::strcmp(key, "graph"))
    *value = h->use_graph ? 1 : 0;
  else if(!std::strcmp(key, "profile"))
    *value = h->profile ? 1 : 0;
  else if(!std::strcmp(key, "far_variant"))
    *value = h->far_variant;
  else if(!std::strcmp(key, "block_step"))
    *value = h->block_step ? 1 : 0;
  else if(!std::strcmp(key, "far_group"))
    *value = h->group;
  else if(!std::strcmp(key, "wait_limit"))
    *value = h->spin_limit;
  else if(!std::strcmp(key, "coef_mode"))
    *value = h->otf ? QG_COEF_ON_THE_FLY : QG_COEF_TABLE;
  else if(!std::strcmp(key, "tuned_far_us"))
    *value = (int)(h->tuned_far_ms * 1000.0f + 0.5f);
  else if(!std::strcmp(key, "test_skip_post"))
    *value = h->skip_post;
  else if(!std::strcmp(key, "tune_group"))
    *value = h->tune_group ? 1 : 0;
  else if(!std::strcmp(key, "far_early"))
    *value = h->far_early ? 1 : 0;
  else
    return qg_fail(QG_ERR_INVALID_ARG, "qg_get_option: unknown key '%s'", key);
  return QG_OK;
}
