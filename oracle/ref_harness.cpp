// C entry points over the reference's own classes, compiled together with
// the reference's unmodified src/*.cpp files (oracle/build_ref.sh) into
// oracle/_ref/libquest_ref.so.  TEST INFRASTRUCTURE ONLY: the checker that
// pins the oracle and the GPU path to the reference's code, and the timed CPU
// baseline.  Nothing in the product links or loads it.
//
// Each entry point builds what src/main.cpp:25-52 builds: the dots, the
// History array initialised to the ground state for t <= 0 (main.cpp:30-36),
// PulseInteraction and HistoryInteraction (RotatingDyadic as main.cpp uses,
// or the lab-frame Dyadic), and PredictorCorrector::Integrator.  The global
// `config` that configuration.cpp would fill from input.cfg is set directly.
//
// Private members are reached by compiling the reference's headers with
// `private` defined as `public` in this file only (the reference's .cpp files
// are compiled as they are): the integrator's weights are replaced by the
// frozen table (the reference's fit is ill-conditioned and depends on the
// least-squares solver), and the table, the history and single steps are
// read or driven for the comparisons.
#include <algorithm>
#include <array>
#include <cassert>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <memory>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <Eigen/Dense>
#include <boost/multi_array.hpp>
#include <boost/program_options.hpp>

#define private public
#define protected public
#include "configuration.h"
#include "history.h"
#include "integrator.h"
#include "interactions/green_function.h"
#include "interactions/history_interaction.h"
#include "interactions/pulse_interaction.h"
#include "interactions/rotating_green_function.h"
#include "lagrange_set.h"
#include "pulse.h"
#include "quantum_dot.h"
#undef private
#undef protected

// the reference's global configuration (configuration.h:29), normally filled
// by parse_configs
Configuration config;

extern "C" {

// physical constants and options: input.cfg's [constants] and
// interpolation order, and the Green's function frame (0 rotating, 1 lab)
typedef struct {
  double c0, hbar, mu0, laser_frequency, dt;
  int interpolation_order;
  int frame;
} ref_params;

}  // extern "C"

namespace {

std::string g_error;

void set_config(const ref_params *p, int n, int T)
{
  config.num_particles = n;
  config.num_timesteps = T;
  config.c0 = p->c0;
  config.hbar = p->hbar;
  config.mu0 = p->mu0;
  config.omega = p->laser_frequency;
  config.dt = p->dt;
  config.total_time = T * p->dt;
  config.interpolation_order = p->interpolation_order;
}

// dots: n rows of x y z omega_0 T1 T2 dx dy dz (a dots.cfg line)
std::shared_ptr<DotVector> make_dots(const double *d, int n)
{
  auto dots = std::make_shared<DotVector>();
  dots->reserve(n);
  for(int i = 0; i < n; ++i) {
    const double *r = d + 9 * (size_t)i;
    dots->emplace_back(Eigen::Vector3d(r[0], r[1], r[2]), r[3], std::make_pair(r[4], r[5]),
                       Eigen::Vector3d(r[6], r[7], r[8]));
  }
  return dots;
}

// the pulse as read_pulse_config reads it (pulse.cpp:29-45: no normalisation)
std::shared_ptr<Pulse> make_pulse(const double *v)
{
  std::ostringstream os;
  os << std::setprecision(17);
  for(int k = 0; k < 10; ++k) os << v[k] << " ";
  std::istringstream is(os.str());
  auto p = std::make_shared<Pulse>();
  is >> *p;
  return p;
}

std::shared_ptr<GreenFunction::Dyadic> make_dyadic(const ref_params *p)
{
  if(p->frame == 0)
    return std::make_shared<GreenFunction::RotatingDyadic>(p->mu0, p->c0, p->hbar, p->laser_frequency);
  return std::make_shared<GreenFunction::Dyadic>(p->mu0, p->c0, p->hbar);
}

// History for steps -22 .. T-1, ground state for t <= 0 (main.cpp:30-36)
std::shared_ptr<History::HistoryArray> make_history(int n, int T)
{
  auto h = History::make_shared_history(n, 22, T);
  for(int t = -22; t <= 0; ++t)
    for(int i = 0; i < n; ++i) (*h)[i][t][0] = Eigen::Vector2cd(1, 0);
  return h;
}

// layout of the flat history buffers: (N, 22 + T, 2, 2) complex =
// [dot][t + 22][rho or rho-dot][component]
void copy_history_in(History::HistoryArray &h, const double *src, int n, int T)
{
  for(int i = 0; i < n; ++i)
    for(int t = -22; t < T; ++t)
      for(int k = 0; k < 2; ++k)
        for(int c = 0; c < 2; ++c) {
          const double *z = src + 2 * ((((size_t)i * (T + 22) + (t + 22)) * 2 + k) * 2 + c);
          h[i][t][k][c] = std::complex<double>(z[0], z[1]);
        }
}

void copy_history_out(const History::HistoryArray &h, double *dst, int n, int T)
{
  for(int i = 0; i < n; ++i)
    for(int t = -22; t < T; ++t)
      for(int k = 0; k < 2; ++k)
        for(int c = 0; c < 2; ++c) {
          double *z = dst + 2 * ((((size_t)i * (T + 22) + (t + 22)) * 2 + k) * 2 + c);
          const std::complex<double> v = h[i][t][k][c];
          z[0] = v.real();
          z[1] = v.imag();
        }
}

void set_weights(PredictorCorrector::Integrator &in, const double *ps, const double *cs, double fc, int n_time)
{
  for(int r = 0; r < 2; ++r)
    for(int h = 0; h < n_time; ++h) {
      in.weights.ps(r, h) = ps[r * n_time + h];
      in.weights.cs(r, h) = cs[r * n_time + h];
    }
  in.weights.future_coef = fc;
}

// discards the integrator's progress lines (integrator.cpp:209-216) while alive
struct QuietCout {
  std::streambuf *old;
  std::ostringstream sink;
  QuietCout() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~QuietCout() { std::cout.rdbuf(old); }
};

int parse_bad_step(const std::string &msg)
{
  const std::string key = "at or before step ";
  const size_t at = msg.find(key);
  return at == std::string::npos ? -2 : std::atoi(msg.c_str() + at + key.size());
}

}  // namespace

extern "C" {

const char *ref_last_error(void) { return g_error.c_str(); }

// PredictorCorrector::Weights(n_lambda, n_time, radius) exactly as the
// reference builds it (integrator.cpp:85-102), its least-squares step solved
// by this repository's JacobiSVD stand-in (exact minimum norm).  ps and cs
// are 2 x n_time row-major.
int ref_weights(int n_lambda, int n_time, double radius, double *ps, double *cs, double *fc)
{
  PredictorCorrector::Weights w(n_lambda, n_time, radius);
  for(int r = 0; r < 2; ++r)
    for(int h = 0; h < n_time; ++h) {
      ps[r * n_time + h] = w.ps(r, h);
      cs[r * n_time + h] = w.cs(r, h);
    }
  *fc = w.future_coef;
  return 0;
}

// UniformLagrangeSet::calculate_weights (lagrange_set.cpp:17-41): 3 x (q+1)
int ref_lagrange_weights(double x, double dt, int q, double *out)
{
  Interpolation::UniformLagrangeSet s(q);
  s.calculate_weights(x, dt);
  for(int d = 0; d < 3; ++d)
    for(int i = 0; i <= q; ++i) out[d * (q + 1) + i] = s.weights[d][i];
  return 0;
}

// HistoryInteraction's table (history_interaction.cpp:21-45), in its own
// triangular pair order: delays[P], coefs[P][q+1] complex.
int ref_build_table(const double *dots, int n, const ref_params *p, int *delays, double *coefs)
{
  try {
    set_config(p, n, 1);
    auto d = make_dots(dots, n);
    auto h = make_history(n, 1);
    HistoryInteraction hi(d, h, make_dyadic(p), p->interpolation_order);
    const long long P = (long long)n * (n - 1) / 2;
    const int q = p->interpolation_order;
    for(long long k = 0; k < P; ++k) {
      delays[k] = hi.floor_delays[k];
      for(int i = 0; i <= q; ++i) {
        coefs[2 * (k * (q + 1) + i)] = hi.coefficients[k][i].real();
        coefs[2 * (k * (q + 1) + i) + 1] = hi.coefficients[k][i].imag();
      }
    }
    return 0;
  } catch(const std::exception &e) {
    g_error = e.what();
    return 1;
  }
}

// HistoryInteraction::evaluate(step) (history_interaction.cpp:47-70) on a
// given history (N, 22 + T, 2, 2) complex: out = N complex.
int ref_history_evaluate(const double *dots, int n, const ref_params *p, const double *hist, int T, int step,
                         double *out)
{
  try {
    set_config(p, n, T);
    auto d = make_dots(dots, n);
    auto h = History::make_shared_history(n, 22, T);
    copy_history_in(*h, hist, n, T);
    HistoryInteraction hi(d, h, make_dyadic(p), p->interpolation_order);
    const auto &r = hi.evaluate(step);
    for(int i = 0; i < n; ++i) {
      out[2 * i] = r[i].real();
      out[2 * i + 1] = r[i].imag();
    }
    return 0;
  } catch(const std::exception &e) {
    g_error = e.what();
    return 1;
  }
}

// PulseInteraction::evaluate(step) (pulse_interaction.cpp:9-20): N complex.
int ref_pulse_evaluate(const double *dots, int n, const double *pulse, const ref_params *p, int step,
                       double *out)
{
  set_config(p, n, step + 1);
  auto d = make_dots(dots, n);
  PulseInteraction pi(d, make_pulse(pulse));
  const auto &r = pi.evaluate(step);
  for(int i = 0; i < n; ++i) {
    out[2 * i] = r[i].real();
    out[2 * i + 1] = r[i].imag();
  }
  return 0;
}

// QuantumDot::liouville_rhs (quantum_dot.cpp:10-19) for one dot (a dots.cfg
// row), rho = 2 complex, rabi = 1 complex: out = 2 complex.
int ref_liouville_rhs(const double *dot, const double *rho, const double *rabi, double laser_freq, double *out)
{
  auto d = make_dots(dot, 1);
  const matrix_elements r(std::complex<double>(rho[0], rho[1]), std::complex<double>(rho[2], rho[3]));
  const matrix_elements m = (*d)[0].liouville_rhs(r, std::complex<double>(rabi[0], rabi[1]), laser_freq);
  for(int k = 0; k < 2; ++k) {
    out[2 * k] = m[k].real();
    out[2 * k + 1] = m[k].imag();
  }
  return 0;
}

// main.cpp:25-55 without the files: the whole solve over T steps with the
// given weights (ps, cs 2 x n_time row-major).  hist_out: (N, 22 + T, 2, 2)
// complex; *bad_step = the step of the reference's domain_error, or -1.
// T >= 10 (log_percentage_complete divides by T / 10).
int ref_run(const double *dots, int n, const double *pulse, const ref_params *p, const double *ps,
            const double *cs, double fc, int n_time, int T, double *hist_out, int *bad_step)
{
  if(T < 10) {
    g_error = "T must be at least 10 (integrator.cpp:212 divides by T / 10)";
    return 1;
  }
  try {
    set_config(p, n, T);
    auto d = make_dots(dots, n);
    auto rhs = rhs_functions(*d, config.omega);
    auto h = make_history(n, T);
    std::vector<std::shared_ptr<Interaction>> interactions{
        std::make_shared<PulseInteraction>(d, make_pulse(pulse)),
        std::make_shared<HistoryInteraction>(d, h, make_dyadic(p), p->interpolation_order)};
    PredictorCorrector::Integrator in(config.dt, 18, n_time, 3.15, h, rhs, std::move(interactions));
    set_weights(in, ps, cs, fc, n_time);
    *bad_step = -1;
    {
      QuietCout quiet;
      try {
        in.solve();
      } catch(const std::domain_error &e) {
        *bad_step = parse_bad_step(e.what());
      }
    }
    copy_history_out(*h, hist_out, n, T);
    return 0;
  } catch(const std::exception &e) {
    g_error = e.what();
    return 1;
  }
}

// The timed CPU baseline: the reference's Integrator::solve_step for steps
// t0 .. t0 + nsteps - 1 (each: predictor, evaluate, 10 x (corrector,
// evaluate), integrator.cpp:128-140, then the finiteness check) on a history
// whose steps before t0 are synthetic (rho = (1, 1e-4 (g1 + i g2)), g Gaussian
// from a fixed generator, rho-dot 0).  Returns the steps done; seconds and
// table_seconds (HistoryInteraction's constructor) are wall times.
int ref_time_steps(const double *dots, int n, const double *pulse, const ref_params *p, const double *ps,
                   const double *cs, double fc, int n_time, int t0, int nsteps, unsigned long long seed,
                   double *seconds, double *table_seconds)
{
  try {
    const int T = t0 + nsteps;
    set_config(p, n, T);
    auto d = make_dots(dots, n);
    auto rhs = rhs_functions(*d, config.omega);
    auto h = make_history(n, T);
    // splitmix64 -> Box-Muller
    uint64_t s = seed;
    auto next = [&s]() {
      uint64_t z = (s += 0x9E3779B97F4A7C15ull);
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      return ((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    for(int i = 0; i < n; ++i)
      for(int t = -22; t < t0; ++t) {
        const double r = std::sqrt(-2.0 * std::log(1.0 - next())), a = 2 * M_PI * next();
        (*h)[i][t][0] = Eigen::Vector2cd(1.0, std::complex<double>(1e-4 * r * std::cos(a), 1e-4 * r * std::sin(a)));
      }
    const auto c0 = std::chrono::steady_clock::now();
    auto hist_int = std::make_shared<HistoryInteraction>(d, h, make_dyadic(p), p->interpolation_order);
    const auto c1 = std::chrono::steady_clock::now();
    std::vector<std::shared_ptr<Interaction>> interactions{
        std::make_shared<PulseInteraction>(d, make_pulse(pulse)), hist_int};
    PredictorCorrector::Integrator in(config.dt, 18, n_time, 3.15, h, rhs, std::move(interactions));
    set_weights(in, ps, cs, fc, n_time);
    int done = 0;
    const auto c2 = std::chrono::steady_clock::now();
    try {
      for(int t = t0; t < T; ++t) {
        in.solve_step(t);
        ++done;
        in.throw_if_unbounded_solution(t);
      }
    } catch(const std::domain_error &) {
    }
    const auto c3 = std::chrono::steady_clock::now();
    *table_seconds = std::chrono::duration<double>(c1 - c0).count();
    *seconds = std::chrono::duration<double>(c3 - c2).count();
    return done;
  } catch(const std::exception &e) {
    g_error = e.what();
    return -1;
  }
}

}  // extern "C"
