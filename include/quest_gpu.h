/*
 * quest_gpu.h -- C ABI of the B200 (sm_100a) implementation of QuEST's
 * retarded-interaction time step.
 *
 * The reference (cglosser/QuEST) exposes the path through three C++
 * interfaces.  Each entry point below names the one it replaces:
 *
 *   Interaction::evaluate(int)          src/interactions/interaction.h:16
 *   HistoryInteraction (ctor, table)    src/interactions/history_interaction.h:16-21,
 *                                       history_interaction.cpp:5-45
 *   HistoryInteraction::evaluate        history_interaction.cpp:47-70
 *   PulseInteraction::evaluate          src/interactions/pulse_interaction.cpp:9-20
 *   History::HistoryArray               src/history.h:13-14, history.cpp:3-9
 *   PredictorCorrector::Weights         src/integrator.h:23-33, integrator.cpp:5-102
 *   PredictorCorrector::Integrator      src/integrator.h:35-41, integrator.cpp:104-207
 *
 * Conventions.
 *  - Complex numbers are interleaved double[2] (layout-compatible with
 *    std::complex<double> and Eigen::Vector2cd components).
 *  - Dots and pulses use the field order of the reference's dots.cfg and
 *    pulse.cfg lines (src/quantum_dot.cpp:33-38, src/pulse.cpp:29-35).
 *  - All host pointers are plain host memory; the library copies.
 *  - Every call returns a qg_status; qg_last_error() gives the message of the
 *    last failure on the calling thread.
 *  - One handle owns one CUDA stream and its device state.  Calls on the same
 *    handle must not overlap (the reference's objects are not reentrant
 *    either); different handles are independent.
 *  - The library allocates its device memory in qg_create and frees it in
 *    qg_destroy; no call in between allocates device memory (the first
 *    evaluate or history copy of a handle allocates its small pinned host
 *    staging buffer).  The memory
 *    comes from a stream-ordered pool per device that keeps freed blocks (up
 *    to half the device's memory) for later handles, so qg_destroy does not
 *    synchronise the device; an allocation that does not fit first returns
 *    the pool's idle blocks to the device.
 */
#ifndef QUEST_GPU_H
#define QUEST_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  QG_OK = 0,
  QG_ERR_INVALID_ARG = 1,  /* a size, pointer or option is out of range */
  QG_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  QG_ERR_OOM = 3,          /* device memory exhausted */
  QG_ERR_NONFINITE = 4,    /* non-finite history: the reference's
                              std::domain_error("unbounded history values at
                              or before step N"), integrator.cpp:200-207 */
  QG_ERR_UNSUPPORTED = 5   /* valid request this build does not implement */
} qg_status;

/* One quantum dot: x y z omega_0 T1 T2 dx dy dz (QuantumDot,
 * src/quantum_dot.h:21-48). */
typedef struct {
  double pos[3];
  double freq;
  double t1, t2;
  double dip[3];
} qg_dot;

/* Incident Gaussian pulse: E_0 delay sigma omega_L k p (Pulse,
 * src/pulse.h:10-24).  The polarisation is used as given, matching the
 * reference's read_pulse_config (pulse.cpp:29-45), which does not normalise. */
typedef struct {
  double amplitude, delay, width, freq;
  double wavevector[3];
  double polarization[3];
} qg_pulse;

typedef enum { QG_FRAME_ROTATING = 0, QG_FRAME_LAB = 1 } qg_frame;
typedef enum { QG_PREC_FP64 = 0, QG_PREC_MIXED = 1 } qg_precision;
/* QG_COEF_AUTO: the per-pair table when it takes at most half of the free
 * device memory, else on the fly.  QG_COEF_TUNED: where the table fits, the
 * first qg_run times the table kernel (its fastest variant) against the
 * on-the-fly kernel and keeps the faster, freeing the table if it loses; the
 * two coefficient forms are algebraically equal, so results differ only in
 * the last bits (qg_get_option "coef_mode" reports the choice). */
typedef enum { QG_COEF_AUTO = 0, QG_COEF_TABLE = 1, QG_COEF_ON_THE_FLY = 2, QG_COEF_TUNED = 3 } qg_coef_mode;

/* Everything the reference reads from its global `config`
 * (src/configuration.h:12-19) plus this library's options. */
typedef struct {
  double c0, hbar, mu0;
  double laser_frequency;   /* config.omega: rotating frame and detuning */
  double dt;
  int interpolation_order;  /* q, 1..7 */
  int num_timesteps;        /* T: steps 0..T-1, as config.num_timesteps */
  int frame;                /* qg_frame */
  int precision;            /* qg_precision */
  int coef_mode;            /* qg_coef_mode */
  int reserved[3];          /* must be zero */
} qg_params;

/* Predictor-corrector weights in the layout of PredictorCorrector::Weights:
 * ps and cs are 2 x n_time row-major (row 0 for rho, row 1 for rho-dot
 * already scaled by (n_time-1)/2), future_coef the corrector's weight on the
 * new derivative. */
typedef struct {
  int n_time;               /* history width; the reference uses 22 */
  double ps[2 * 32];
  double cs[2 * 32];
  double future_coef;
} qg_weights;

typedef struct qg_handle_s qg_handle;

/* Message of the last failed call on this thread ("" if none). */
const char *qg_last_error(void);

/* Library version string. */
const char *qg_version(void);

/* PredictorCorrector::Weights(n_lambda, n_time, radius)
 * (integrator.cpp:85-102): the contour-fitted weights, computed as the exact
 * minimum-norm solution in 113-bit floating point and rounded to double (the
 * fit's condition number is about 3e13, so double-precision solvers disagree
 * in the third digit).  n_time <= 32. */
qg_status qg_pc_weights(int n_lambda, int n_time, double radius, qg_weights *out);

/* Builds the device state for N dots: HistoryInteraction's constructor and
 * coefficient table (history_interaction.cpp:5-45), PulseInteraction, the
 * History array initialised as main.cpp:30-36 does (rho = (1,0) for
 * t <= 0), and the Integrator's weights.  weights == NULL uses
 * qg_pc_weights(18, 22, 3.15), the values main.cpp:48-49 hard-codes. */
qg_status qg_create(const qg_dot *dots, int n, const qg_pulse *pulse,
                    const qg_params *params, const qg_weights *weights,
                    qg_handle **out);

qg_status qg_destroy(qg_handle *h);

/* Integrator::solve over steps [next, next + n_steps) (integrator.cpp:120-140):
 * predictor, evaluation, 10 x (corrector, evaluation) per step, with the
 * pair sum over all N(N-1)/2 pairs and q+1 interpolation taps.
 * rho_out (nullable): n_steps * N * 2 complex = (rho00, rho01) per dot per
 * step, the rows History::write_history prints (history.cpp:27-33).
 * On a non-finite value returns QG_ERR_NONFINITE with *bad_step (nullable)
 * set to the first such step, as throw_if_unbounded_solution does.  Steps
 * past num_timesteps are an error. */
qg_status qg_run(qg_handle *h, int n_steps, double *rho_out, int *bad_step);

/* Index of the next step qg_run will compute. */
qg_status qg_next_step(const qg_handle *h, int *step);

/* HistoryInteraction::evaluate(step) (history_interaction.cpp:47-70):
 * field[i] = sum over pairs and taps of coefficient * prefactor(rho01 of the
 * partner at the retarded step).  rho01_step (nullable, N complex) first
 * overwrites the history's rho01 at `step` (the integrator's current
 * iterate); field_out receives N complex. */
qg_status qg_history_evaluate(qg_handle *h, int step, const double *rho01_step,
                              double *field_out);

/* HistoryInteraction::evaluate(step) as qg_history_evaluate computes it, for
 * callers that cannot allocate device memory at the point of the call: code
 * running inside a global-mode CUDA stream capture (where cudaMalloc is
 * prohibited), or hosts whose memory pool owns all device memory and must not
 * see allocations from a library.  It has no counterpart in the reference.
 *
 * Inputs and output are device pointers the caller owns: d_rho01_step
 * (nullable, N complex, user order) first overwrites the history's rho01 at
 * `step` (the handle's device history, like qg_history_evaluate);
 * d_field_out receives N complex, user order.  Work is enqueued on `stream`
 * (a cudaStream_t; NULL = the handle's stream) and the call returns without
 * waiting; the result is ready when that stream reaches this point.  The
 * call reads and writes the handle's device history: a non-NULL stream must
 * already be ordered after any work still pending on the handle's stream
 * (qg_stream; qg_run, qg_history_evaluate and qg_set_history finish theirs
 * before they return), and the handle's own calls must not overlap it.
 *
 * The call allocates nothing and copies nothing to or from the host: its
 * scratch is a fixed 2.2 MB array in the library's device memory, held on
 * every device that loads the library until the process exits.  It holds at
 * most 4096 dots (after padding to multiples of 32); larger handles get
 * QG_ERR_INVALID_ARG.  All calls share that array, so calls whose work
 * overlaps on the GPU (other streams, other handles on the same device) race
 * and must be ordered by the caller.  The first call on each device looks
 * up the array's device address; make that first call before any stream
 * capture begins. */
qg_status qg_history_evaluate_noalloc(qg_handle *h, int step, const double *d_rho01_step,
                                      double *d_field_out, void *stream);

/* PulseInteraction::evaluate(step) (pulse_interaction.cpp:9-20): N complex. */
qg_status qg_pulse_evaluate(qg_handle *h, int step, double *field_out);

/* Writes rho01 (N complex per step, user order) for steps [t0, t0 + n) into
 * the device history that the pair sum reads, as a caller filling
 * History::HistoryArray[.][t][0][1] would.  t0 >= -22.  The device keeps the
 * last W steps per dot (W = max delay + q + 2, qg_info.ring_depth); a step
 * older than that is overwritten by later ones.  The integrator's own window
 * (rho, rho-dot of the last 22 steps) is not changed. */
qg_status qg_set_history(qg_handle *h, int t0, int n, const double *rho01);

/* Reads back rho01 for steps [t0, t0 + n) still held on the device: N
 * complex per step. */
qg_status qg_get_history(qg_handle *h, int t0, int n, double *rho01_out);

/* Current state: rho (rho00, rho01) of every dot after the last computed
 * step (main.cpp:34's initial value before any step), 2 complex per dot,
 * user order. */
qg_status qg_get_state(qg_handle *h, double *rho_out);

/* First step at which a non-finite value appeared, or -1.  For a batch
 * member it is the value the batch's last qg_batch_run read (one gathered
 * copy for all members), so a caller can retire a failed member after every
 * batch run without a device round trip per member. */
qg_status qg_bad_step(qg_handle *h, int *bad_step);

/* Checkpoint / resume (no reference counterpart; the reference keeps the
 * whole history in host memory).  A checkpoint holds the device state after
 * step next_step - 1: the rho01 history ring (plus the FP32 rings in mixed
 * precision), the 23-step predictor-corrector window, the next step and the
 * first non-finite step.  Load it into a handle created from the same dots,
 * pulse and parameters; the resumed run is bit-identical to an uninterrupted
 * one.  qg_checkpoint_size gives the buffer size (host memory). */
qg_status qg_checkpoint_size(const qg_handle *h, size_t *bytes);
qg_status qg_checkpoint_save(qg_handle *h, void *buf, size_t bytes);
qg_status qg_checkpoint_load(qg_handle *h, const void *buf, size_t bytes);

/* Batches: many independent ensembles (handles) advanced together, one
 * persistent far-pair launch and one step launch per step for all of them,
 * driven by an (ensemble, target tile, source-tile group) work list, the
 * 16-step block replayed as one CUDA graph.  No reference counterpart: the
 * reference runs one ensemble per process.  Members keep their own device
 * state and are advanced exactly as qg_run would advance them (bitwise the
 * same results); they must share interpolation order, frame and history
 * width, must join at a step that is a multiple of 16, and must not be run on
 * their own while in a batch.  A member that reaches num_timesteps stops
 * there while the others go on. */
typedef struct qg_batch_s qg_batch;
qg_status qg_batch_create(int capacity, qg_batch **out);
qg_status qg_batch_destroy(qg_batch *b);
qg_status qg_batch_add(qg_batch *b, qg_handle *h);
qg_status qg_batch_remove(qg_batch *b, qg_handle *h);
/* Advances every member by n_blocks x 16 steps (capped at its num_timesteps). */
qg_status qg_batch_run(qg_batch *b, int n_blocks);
qg_status qg_batch_size(const qg_batch *b, int *members, int *tasks, int *blocks);
/* Batch options: "profile" (1 = each block's kernels launched one by one
 * instead of as the graph, with CUDA events around the far-pair launch and
 * around the step launches; same results), "far_packed" (mixed-precision
 * members: 1 = the FP32 convolution with packed pairs, the default, 0 =
 * scalar; same results), "far_gmajor" (1 = each member's far tasks in
 * source-group-major order, so a thread block's warps read the same history
 * rows, the default; same results), "mid_pipe" (1 = the step launches fetch
 * several mid-range pair entries per thread before summing them, which helps
 * members with long mid lists; same results), "tune_group" (1 = the next
 * run's autotuner also times source tiles per far-kernel warp, 1, 2, 4 and
 * 8, for each size class of members present (fewer than 4 tiles, fewer than
 * 16, fewer than 64, more) and gives every member of a class, present or
 * joining later, that class's group; a member's results then equal a solo
 * run with the same "far_group", not one with its default; off by default),
 * "autotune" (1 = time again at the next run). */
qg_status qg_batch_set_option(qg_batch *b, const char *key, int value);
/* Reads a batch option back: "far_packed", "far_gmajor", "mid_pipe",
 * "profile", "tune_group", "far_group_class0" .. "far_group_class3" (the
 * group tuned for each size class, 0 = members keep their own),
 * "tuned_far_us" (the far launch's time the batch's autotuner measured for
 * its choice, microseconds; 0 if it did not run).  The autotuner times the
 * far launch's forms that sum the same terms (far_packed for mixed members x
 * far_gmajor) at the batch's first qg_batch_run and keeps the fastest, unless
 * one was set; "autotune" (1) asks for it again at the next run. */
qg_status qg_batch_get_option(const qg_batch *b, const char *key, int *value);
/* Device time in milliseconds of the batch's far-pair launches and step
 * launches (each nullable), accumulated while "profile" is on. */
qg_status qg_batch_kernel_time(qg_batch *b, int reset, double *far_ms, int *far_launches, double *step_ms,
                               int *step_launches);

/* Target sharding of one ensemble over several GPUs (one process per GPU):
 * the reference sums every pair in one loop (history_interaction.cpp:47-70);
 * here shard `rank` of `world` computes the targets in its range of 32-dot
 * blocks of the internal order (every group of dots coupled at delay 0 lies
 * inside one block, so the current-step coupling never crosses shards) and
 * holds every dot's rho01 history, which its far and mid terms read.  Shards
 * compute their coefficients on the fly (coef_mode TABLE is refused).  Each
 * step: qg_shard_step computes this shard's dots and writes their new rho01
 * (count complex, internal order) to the device buffer d_slice; the caller
 * gathers all shards' slices in rank order into one internal-order vector of
 * n_pad complex (NCCL all-gather, peer copies) and passes it to
 * qg_shard_import, which writes the other shards' dots into this shard's
 * history as their own steps wrote theirs, and moves on one step.  Each
 * target's sums are the unsharded handle's, term for term: a sharded run
 * gives the unsharded run's results bit for bit.  qg_get_state, qg_bad_step
 * and qg_checkpoint_* report this shard's dots only; qg_run is not used. */
qg_status qg_shard_create(const qg_dot *dots, int n, const qg_pulse *pulse, const qg_params *params,
                          const qg_weights *weights, int rank, int world, qg_handle **out);
/* This shard's internal dots [*first, *first + *count), the internal slot
 * count, and (user nullable, n_pad ints) the internal -> user index map, -1
 * for padding. */
qg_status qg_shard_layout(const qg_handle *h, int *first, int *count, int *n_pad, int *user);
qg_status qg_shard_step(qg_handle *h, double *d_slice);
qg_status qg_shard_import(qg_handle *h, const double *d_full);

/* Diagnostics of the built state. */
typedef struct {
  int n;                 /* dots */
  int max_delay;         /* largest floor delay over all pairs */
  int ring_depth;        /* W: rho01 steps kept per dot */
  long long num_pairs;   /* N(N-1)/2 */
  long long near_pairs;  /* pairs with floor delay 0 (current-step coupling) */
  long long mid_pairs;   /* pairs with floor delay < time_block (summed per step) */
  int time_block;        /* K: steps per pass of the far-pair kernel */
  int coef_mode;         /* resolved qg_coef_mode */
  int precision;         /* qg_precision */
  int fused_step;        /* 1 when all current-step coupling fits one block;
                            2 when, in addition, a whole K-step block runs as
                            one cooperative launch (all 32-dot blocks resident) */
  size_t device_bytes;   /* device memory held by the handle */
  double table_build_ms; /* time of the coefficient-table kernel */
} qg_info;

qg_status qg_get_info(const qg_handle *h, qg_info *info);

/* Device memory a handle with these inputs would hold (admission control). */
qg_status qg_footprint(int n, const qg_params *params, double side, size_t *bytes);

/* Timing hooks: the handle's cudaStream_t (as void*), and the device time in
 * milliseconds of the far-pair kernel and of the per-step kernels (each
 * nullable), accumulated over qg_run calls made while the "profile" option
 * is on. */
void *qg_stream(qg_handle *h);
qg_status qg_kernel_time(qg_handle *h, int reset, double *pair_ms, int *pair_launches,
                         double *step_ms, int *step_launches);

/* Options: "graph" (1 = replay each K-step block as a CUDA graph, default),
 * "profile" (1 = CUDA events around the far-pair kernel and the step
 * kernels: event nodes inside the block graphs, or around each launch when
 * "graph" is 0),
 * "far_variant" (0..11: resource shape and task order of the far-pair
 *   kernel, same results; 7 and 8 are 0 and 3 with each block's warps on one
 *   source group of consecutive target tiles; the first qg_run of an FP64
 *   table handle of 512 dots or more picks the fastest of 0, 3, 5, 6, 7, 8,
 *   9, 10 and 11 (9: the table staged by bulk-copy-engine copies on an
 *   mbarrier; 10 and 11: each source's history window run staged in shared
 *   memory, in the two task orders) by timing launches of each, unless a
 *   variant was set; mixed-precision
 *   table handles choose the same way among 0, 7 (its kernel at 150
 *   registers, target-tile and source-group major) and 1, 8 (at 128);
 *   on-the-fly handles take 8 (source-group-major order, held to 3 blocks
 *   per SM; 0 and 3: target-tile major, 1: held, 7: source-group major,
 *   all with the same results); the
 *   choice is remembered for the process, and later handles of the same kind
 *   (device, size, order, frame, precision, coefficient mode) take it
 *   without timing; batch members are not timed, the batch kernel having its
 *   own),
 * "autotune" (1 = time the far-kernel variants again now; at a block
 *   boundary between runs),
 * "far_early" (1 = the default: FP64 table handles use the far kernel's
 *   first-blocks form, whatever the variant, in the blocks where some
 *   windows start before step -22: one loop for all lanes of a warp instead
 *   of two; 0 = never; same results),
 * "far_group" (source tiles each far-kernel warp sums before writing its
 *   partial, table handles; default 4, mixed precision 2 below 256 tiles;
 *   changes the summation grouping, so results change in the last bits),
 * "tune_group" (1 = the next qg_run times the far variants and then
 *   far_group 1, 2, 4 and 8 against the default and keeps the fastest;
 *   table handles; off by default because the group changes the last bits,
 *   so a tuned handle's results depend on which group won; the choice is
 *   remembered for the process like the variant's),
 * "block_step" (1 = the K steps of a block in one cooperative launch, the
 *   default where every 32-dot block fits on the device at once; 0 = one
 *   launch per step; same results),
 * "wait_limit" (polls the step-block kernel makes on a partner block's step
 *   count before it gives up; 0 = the default, about a second.  A wait that
 *   runs out ends the launch: qg_run returns QG_ERR_CUDA "timed out" and the
 *   handle needs "reset" or a checkpoint load before it runs again),
 * "test_skip_post" (failure-detection tests only: the index of a 32-dot block
 *   that never posts its finished steps, so that its partners' waits run
 *   out; -1 = none, the default),
 * "reset" (restart the history at step 0, main.cpp:30-36). */
qg_status qg_set_option(qg_handle *h, const char *key, int value);

/* Reads an option back: "graph", "profile", "far_variant" (the variant in
 * use, which after the first qg_run is the autotuner's choice), "block_step",
 * "far_group", "tune_group", "far_early", "wait_limit", "test_skip_post", "coef_mode" (QG_COEF_TABLE or
 * QG_COEF_ON_THE_FLY: the form in use), "tuned_far_us" (the far kernel's
 * launch time the autotuner measured for its choice, microseconds; 0 if it
 * did not run).  No reference counterpart (the reference has no options). */
qg_status qg_get_option(const qg_handle *h, const char *key, int *value);

#ifdef __cplusplus
}
#endif
#endif
