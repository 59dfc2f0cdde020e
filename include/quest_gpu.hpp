/* C++ adapters over the C ABI of quest_gpu.h, shaped like the reference's
 * operator interfaces so a C++ caller can swap them in:
 *
 *   quest_gpu::HistoryInteraction   Interaction / HistoryInteraction
 *                                   (src/interactions/interaction.h:9-21,
 *                                   history_interaction.h:14-35): evaluate(t)
 *                                   returns a reference to an internal array,
 *                                   valid until the next call; operator[].
 *   quest_gpu::Integrator           PredictorCorrector::Integrator
 *                                   (src/integrator.h:35-41): solve() advances
 *                                   every step and keeps the trajectory.
 *   quest_gpu::write_history        History::write_history (src/history.cpp:17-34)
 *
 * Errors become exceptions as in the reference: a non-finite state throws
 * std::domain_error with the reference's message (integrator.cpp:203-206),
 * anything else quest_gpu::Error (a std::runtime_error).  Header-only; link
 * with libquest_gpu.so.  Device code cannot call the reference's
 * std::function right-hand sides, so the adapters take the dots' parameters
 * (qg_dot) instead. */
#pragma once

#include <complex>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "quest_gpu.h"

namespace quest_gpu {

using cmplx = std::complex<double>;

class Error : public std::runtime_error {
 public:
  Error(qg_status code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
  qg_status code() const { return code_; }

 private:
  qg_status code_;
};

inline void check(qg_status st)
{
  if(st == QG_OK) return;
  const std::string msg = qg_last_error();
  if(st == QG_ERR_NONFINITE) throw std::domain_error(msg);
  throw Error(st, msg);
}

/* One simulation handle (qg_create / qg_destroy), move-only. */
class Simulation {
 public:
  Simulation(const std::vector<qg_dot> &dots, const qg_pulse &pulse, const qg_params &params,
             const qg_weights *weights = nullptr)
      : n_((int)dots.size()), T_(params.num_timesteps)
  {
    check(qg_create(dots.data(), n_, &pulse, &params, weights, &h_));
  }
  Simulation(const Simulation &) = delete;
  Simulation &operator=(const Simulation &) = delete;
  Simulation(Simulation &&o) noexcept : h_(o.h_), n_(o.n_), T_(o.T_) { o.h_ = nullptr; }
  ~Simulation()
  {
    if(h_) qg_destroy(h_);
  }

  qg_handle *handle() const { return h_; }
  int size() const { return n_; }
  int num_timesteps() const { return T_; }
  int next_step() const
  {
    int t = 0;
    check(qg_next_step(h_, &t));
    return t;
  }

  /* Advances n_steps; rho_out (nullable) receives n_steps x N x (rho00, rho01). */
  void run(int n_steps, cmplx *rho_out = nullptr)
  {
    int bad = -1;
    check(qg_run(h_, n_steps, reinterpret_cast<double *>(rho_out), &bad));
  }

  qg_info info() const
  {
    qg_info i;
    check(qg_get_info(h_, &i));
    return i;
  }

 private:
  qg_handle *h_ = nullptr;
  int n_ = 0;
  int T_ = 0;
};

/* HistoryInteraction: the retarded field of every dot at step t from the
 * rho01 history the caller supplies (steps before t through set_history, or
 * the current iterate as evaluate's argument). */
class HistoryInteraction {
 public:
  using ResultArray = std::vector<cmplx>;

  explicit HistoryInteraction(Simulation &sim) : sim_(&sim), results_(sim.size()) {}

  /* Stores rho01 of steps [t0, t0 + n) (n x N values). */
  void set_history(int t0, int n, const cmplx *rho01)
  {
    check(qg_set_history(sim_->handle(), t0, n, reinterpret_cast<const double *>(rho01)));
  }

  /* interaction.h:20: the field at step t; rho01_t (nullable) is the current
   * iterate of step t, the only step the tap-0 terms of delay-0 pairs read. */
  const ResultArray &evaluate(int t, const cmplx *rho01_t = nullptr)
  {
    check(qg_history_evaluate(sim_->handle(), t, reinterpret_cast<const double *>(rho01_t),
                              reinterpret_cast<double *>(results_.data())));
    return results_;
  }

  const cmplx &operator[](int i) const { return results_[i]; }

 private:
  Simulation *sim_;
  ResultArray results_;
};

/* PredictorCorrector::Integrator with the whole step (pulse, history field,
 * Bloch right-hand side, predictor and 10 corrections) on the device. */
class Integrator {
 public:
  explicit Integrator(Simulation &sim) : sim_(&sim) {}

  /* integrator.cpp:104-121: every remaining step; the trajectory (T x N x 2)
   * is kept for history(). */
  void solve()
  {
    const int t0 = sim_->next_step();
    const int n = sim_->num_timesteps() - t0;
    traj_.resize((size_t)sim_->num_timesteps() * sim_->size() * 2);
    if(n > 0) sim_->run(n, traj_.data() + (size_t)t0 * sim_->size() * 2);
  }

  /* rho00 (k = 0) or rho01 (k = 1) of dot i at step t. */
  const cmplx &rho(int t, int i, int k) const { return traj_[((size_t)t * sim_->size() + i) * 2 + k]; }
  const std::vector<cmplx> &trajectory() const { return traj_; }

 private:
  Simulation *sim_;
  std::vector<cmplx> traj_;
};

/* One output.dat line per step, as History::write_history prints it: each
 * dot's (rho00, rho01) as Eigen prints a 1 x 2 complex row (both fields
 * right-aligned to the wider of the two, one space between), followed by a
 * space; 12 significant digits, scientific. */
inline std::string format_complex(const cmplx &z)
{
  char buf[96];
  std::snprintf(buf, sizeof buf, "(%.12e,%.12e)", z.real(), z.imag());
  return buf;
}

inline void write_step(std::FILE *f, const cmplx *rho_step, int n)
{
  std::string line;
  for(int i = 0; i < n; ++i) {
    const std::string a = format_complex(rho_step[2 * i]), b = format_complex(rho_step[2 * i + 1]);
    const size_t w = a.size() > b.size() ? a.size() : b.size();
    line.append(w - a.size(), ' ');
    line += a;
    line += ' ';
    line.append(w - b.size(), ' ');
    line += b;
    line += ' ';
  }
  line += '\n';
  std::fwrite(line.data(), 1, line.size(), f);
}

}  // namespace quest_gpu
