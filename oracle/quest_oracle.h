/*
 * CPU oracle for the QuEST retarded-interaction time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm used to check the CUDA library.  Only the test suite, the smoke
 * check in __graft_entry__.py and the CPU-baseline leg of bench.py may load
 * it.  The product library (quest_b200/libquest_gpu.so) never links, calls or
 * falls back to it.
 *
 * Parity status.  The reference (cglosser/QuEST) cannot be compiled here: it
 * needs Eigen3 and Boost, which are absent.  The oracle is therefore pinned
 * (a) against the reference's own known-answer test of liouville_rhs
 * (test/quantum_dot_test.cpp:13-43) and its non-finite tests
 * (test/history_test.cpp:13-53), (b) against a frozen 80-digit solution of
 * the predictor-corrector weight fit (tests/golden/pc_weights_*.txt), and
 * (c) against mathematical identities (Lagrange exactness on polynomials,
 * dyad symmetry and scaling, single-dot ODE solution).  Bit-level parity with
 * the original binary's Eigen arithmetic is unpinned.
 *
 * Every function cites the reference file:line it restates.  Arithmetic is
 * written as explicit real operations in the order the reference's complex
 * and Eigen expressions evaluate, and the file is compiled with
 * -ffp-contract=off so no fused multiply-adds change the rounding.
 */
#ifndef QUEST_ORACLE_H
#define QUEST_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One dots.cfg line: x y z omega_0 T1 T2 dx dy dz (src/quantum_dot.cpp:33-38). */
typedef struct {
  double pos[3];
  double freq;
  double t1, t2;
  double dip[3];
} or_dot;

/* One pulse.cfg line: E_0 delay sigma omega_L kx ky kz px py pz
 * (src/pulse.cpp:29-35).  The polarisation is used as given, exactly as the
 * reference's stream reader leaves it un-normalised. */
typedef struct {
  double amplitude, delay, width, freq;
  double wavevector[3];
  double polarization[3];
} or_pulse;

/* Configuration values the reference reads from its global `config`
 * (src/configuration.h:12-19). frame: 0 = rotating (RotatingDyadic, the one
 * main() uses), 1 = lab frame (GreenFunction::Dyadic). */
typedef struct {
  double c0, hbar, mu0, laser_frequency, dt;
  int interpolation_order;
  int frame;
} or_params;

/* Predictor-corrector weights, layout of PredictorCorrector::Weights
 * (src/integrator.h:23-33): ps/cs are 2 x n_time row-major. */
typedef struct {
  int n_time;
  const double *ps;
  const double *cs;
  double future_coef;
} or_weights;

/* History array in the reference layout History::HistoryArray
 * [N][t = -window .. T-1][0: rho, 1: rho-dot] of Eigen::Vector2cd
 * (src/history.h:13-14, src/history.cpp:3-9): doubles index
 * ((dot*(T+window) + (t+window))*2 + which)*4 + {re00, im00, re01, im01}. */

/* UniformLagrangeSet::calculate_weights (src/lagrange_set.cpp:17-41).
 * w has 3*(q+1) doubles: w[k*(q+1)+i] for derivative k and node i. */
void or_lagrange_weights(double x, double dt, int q, double *w);

/* One pair's floor delay and q+1 complex coefficients, built exactly as
 * HistoryInteraction::build_coefficient_table does for (src, obs)
 * (src/interactions/history_interaction.cpp:29-43).  coef: 2*(q+1) doubles. */
void or_pair_coefficients(const or_dot *src, const or_dot *obs,
                          const or_params *p, int *floor_delay, double *coef);

/* Triangular pair index maps (history_interaction.cpp:72-86), 64-bit. */
long long or_coord2idx(int row, int col);
void or_idx2coord(long long idx, int *row, int *col);

/* build_coefficient_table over all N(N-1)/2 pairs in the reference order
 * (history_interaction.cpp:21-45). delays: P ints, coefs: P*2*(q+1). */
void or_build_table(const or_dot *dots, int n, const or_params *p,
                    int *delays, double *coefs);

/* HistoryInteraction::evaluate (history_interaction.cpp:47-70) on a full
 * reference-layout history with `window` negative slots and T steps.
 * out: 2*N doubles. */
void or_history_evaluate(int n, const or_params *p, const int *delays,
                         const double *coefs, const double *hist, int window,
                         int T, int step, double *out);

/* PulseInteraction::evaluate (src/interactions/pulse_interaction.cpp:9-20,
 * src/pulse.cpp:15-20, src/math_utils.cpp:27-30). out: 2*N doubles. */
/* history_interaction.cpp:47-70 for a few target dots, coefficients on the
 * fly (O(N) per target); rho01 [dot][t - t_lo] complex, nt steps. */
int or_history_evaluate_targets(const or_dot *dots, int n, const or_params *p, const double *rho01, int t_lo,
                                int nt, int step, const int *targets, int ntargets, double *out);

void or_pulse_evaluate(const or_dot *dots, int n, const or_pulse *pulse,
                       const or_params *p, int step, double *out);

/* QuantumDot::liouville_rhs (src/quantum_dot.cpp:10-19).
 * rho, rabi, out: interleaved complex (rho00, rho01) / rabi / (drho00, drho01). */
void or_liouville_rhs(const or_dot *dot, const double *rho, const double *rabi,
                      double laser_freq, double *out);

/* History::isfinite (src/history.cpp:11-15) on one Vector2cd (4 doubles). */
int or_isfinite(const double *sol);

/* Faithful integrator: main.cpp:30-36 initialisation followed by
 * Integrator::solve (src/integrator.cpp:120-207) with 11 full pair sweeps
 * per step.  hist must hold N*(T+window)*8 doubles; it is fully initialised
 * here.  Returns 0, or 1 with *bad_step set when a step produced a
 * non-finite value (the reference throws std::domain_error there). */
int or_run_faithful(const or_dot *dots, int n, const or_pulse *pulse,
                    const or_params *p, const or_weights *w, int T,
                    double *hist, int *bad_step);

/* Same result, reorganised: the strictly-past part of the pair sum is
 * computed once per step and only the delay-0, tap-0 "near" pairs are
 * re-evaluated in each corrector iteration.  Pair sums run on nthreads
 * OpenMP threads with a fixed static partition and a fixed-order reduction,
 * so results are deterministic for a given thread count. */
int or_run_fast(const or_dot *dots, int n, const or_pulse *pulse,
                const or_params *p, const or_weights *w, int T,
                double *hist, int *bad_step, int nthreads);

/* CPU baseline timing helper: run `nsteps` faithful steps (11 sweeps each)
 * starting at step t0 on an already-populated history and table.  Returns the
 * number of steps completed. */
int or_faithful_steps(const or_dot *dots, int n, const or_pulse *pulse,
                      const or_params *p, const or_weights *w, int T,
                      const int *delays, const double *coefs, double *hist,
                      int t0, int nsteps);

/* One faithful step for dots [lo, hi) only (the target-sharded driver's
 * test backend); -1 when a delay-0 pair crosses the range. */
int or_faithful_step_range(const or_dot *dots, int n, const or_pulse *pulse, const or_params *p,
                           const or_weights *w, int T, const int *delays, const double *coefs, double *hist,
                           int step, int lo, int hi);

int or_window(void); /* 22: the history's negative-time extent (main.cpp:30) */

#ifdef __cplusplus
}
#endif
#endif
