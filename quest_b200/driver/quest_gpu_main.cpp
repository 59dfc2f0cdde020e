// quest-gpu: the reference's `quest` executable (src/main.cpp:17-63) over
// the B200 library.  Same command line (--help, --version/-v, --config/-c,
// default input.cfg), same configuration keys (src/configuration.cpp:17-42:
// [files] qd_path pulse_path, [constants] c0 hbar mu0 laser_frequency,
// [parameters] num_particles total_time timestep interpolation_order;
// num_timesteps = ceil(total_time / timestep)), same dot and pulse files
// (quantum_dot.cpp:33-47, pulse.cpp:29-45), same progress lines and the same
// output.dat (history.cpp:17-34).  Options of this build only:
//   --output PATH        output file (default output.dat)
//   --precision fp64|mixed
//   --coefficients auto|table|on-the-fly|tuned
// A non-finite state ends the run with the reference's std::domain_error
// message on stderr and exit status 1, before any output is written (the
// reference's uncaught exception also leaves no output.dat).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "quest_gpu.hpp"

namespace {

struct Options {
  std::string config = "input.cfg";
  std::string output = "output.dat";
  int precision = QG_PREC_FP64;
  int coef_mode = QG_COEF_AUTO;
  bool help = false, version = false;
};

void usage(std::ostream &os)
{
  os << "QuEST options:\n"
        "Command line options:\n"
        "  --help                 print this help message\n"
        "  -v [ --version ]       print version string\n"
        "  -c [ --config ] arg (=input.cfg) path to configuration file\n"
        "  --output arg (=output.dat)       path of the trajectory output\n"
        "  --precision arg (=fp64)          fp64 or mixed\n"
        "  --coefficients arg (=auto)       auto, table, on-the-fly or tuned (timed)\n"
        "\n"
        "Configuration files:\n"
        "  --files.qd_path arg (=dots.cfg)     path to dot configuration file\n"
        "  --files.pulse_path arg (=pulse.cfg) path to pulse configuration file\n"
        "\n"
        "Physical constants:\n"
        "  --constants.c0 arg                  speed of light in vacuum\n"
        "  --constants.hbar arg                reduced Planck constant\n"
        "  --constants.mu0 arg                 vacuum permeability\n"
        "  --constants.laser_frequency arg     (angular) frequency of incident pulse\n"
        "\n"
        "System parameters:\n"
        "  --parameters.num_particles arg      number of particles in the system\n"
        "  --parameters.total_time arg         total simulation duration\n"
        "  --parameters.timestep arg           timestep size\n"
        "  --parameters.interpolation_order arg order of the Lagrange interpolants\n";
}

bool parse_args(int argc, char **argv, Options &o)
{
  for(int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto value = [&](const std::string &name) -> std::string {
      const std::string eq = name + "=";
      if(a.compare(0, eq.size(), eq) == 0) return a.substr(eq.size());
      if(i + 1 >= argc) throw std::runtime_error("the required argument for option '" + name + "' is missing");
      return argv[++i];
    };
    if(a == "--help") {
      o.help = true;
    } else if(a == "--version" || a == "-v") {
      o.version = true;
    } else if(a == "--config" || a == "-c" || a.rfind("--config=", 0) == 0) {
      o.config = value(a[1] == 'c' ? "-c" : "--config");
    } else if(a == "--output" || a.rfind("--output=", 0) == 0) {
      o.output = value("--output");
    } else if(a == "--precision" || a.rfind("--precision=", 0) == 0) {
      const std::string v = value("--precision");
      if(v == "fp64")
        o.precision = QG_PREC_FP64;
      else if(v == "mixed")
        o.precision = QG_PREC_MIXED;
      else
        throw std::runtime_error("the argument ('" + v + "') for option '--precision' is invalid");
    } else if(a == "--coefficients" || a.rfind("--coefficients=", 0) == 0) {
      const std::string v = value("--coefficients");
      if(v == "auto")
        o.coef_mode = QG_COEF_AUTO;
      else if(v == "table")
        o.coef_mode = QG_COEF_TABLE;
      else if(v == "on-the-fly")
        o.coef_mode = QG_COEF_ON_THE_FLY;
      else if(v == "tuned")
        o.coef_mode = QG_COEF_TUNED;
      else
        throw std::runtime_error("the argument ('" + v + "') for option '--coefficients' is invalid");
    } else {
      throw std::runtime_error("unrecognised option '" + a + "'");
    }
  }
  return true;
}

// INI as boost::program_options::parse_config_file reads it: [section],
// key = value, '#' comments.
std::map<std::string, std::string> read_config(std::istream &is)
{
  std::map<std::string, std::string> kv;
  std::string line, section;
  auto trim = [](std::string s) {
    const char *ws = " \t\r\n";
    s.erase(0, s.find_first_not_of(ws));
    s.erase(s.find_last_not_of(ws) + 1);
    return s;
  };
  while(std::getline(is, line)) {
    line = trim(line.substr(0, line.find('#')));
    if(line.empty()) continue;
    if(line.front() == '[' && line.back() == ']') {
      section = trim(line.substr(1, line.size() - 2));
      continue;
    }
    const size_t eq = line.find('=');
    if(eq == std::string::npos) throw std::runtime_error("invalid line in configuration file: " + line);
    kv[section + "." + trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
  }
  return kv;
}

double number(const std::map<std::string, std::string> &kv, const std::string &key)
{
  auto it = kv.find(key);
  if(it == kv.end()) throw std::runtime_error("the option '" + key + "' is required but missing");
  std::istringstream is(it->second);
  double v;
  if(!(is >> v)) throw std::runtime_error("the argument ('" + it->second + "') for option '" + key + "' is invalid");
  return v;
}

// istream_iterator<QuantumDot> over the file, then resize to num_particles
// (main.cpp:25-26): a short file is padded with zero-initialised dots.
std::vector<qg_dot> read_dots(const std::string &path, int num_particles)
{
  std::ifstream is(path);
  if(!is) throw std::runtime_error("Could not open " + path);
  std::vector<qg_dot> dots;
  qg_dot d;
  while(is >> d.pos[0] >> d.pos[1] >> d.pos[2] >> d.freq >> d.t1 >> d.t2 >> d.dip[0] >> d.dip[1] >> d.dip[2])
    dots.push_back(d);
  qg_dot zero;
  std::memset(&zero, 0, sizeof zero);
  dots.resize(num_particles, zero);
  return dots;
}

qg_pulse read_pulse(const std::string &path)
{
  std::ifstream is(path);
  if(!is) throw std::runtime_error("Could not open " + path);
  qg_pulse p;
  if(!(is >> p.amplitude >> p.delay >> p.width >> p.freq >> p.wavevector[0] >> p.wavevector[1] >> p.wavevector[2] >>
       p.polarization[0] >> p.polarization[1] >> p.polarization[2]))
    throw std::runtime_error("Could not read pulse from " + path);
  return p;
}

}  // namespace

int main(int argc, char **argv)
{
  Options o;
  try {
    parse_args(argc, argv, o);
  } catch(const std::exception &e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
  if(o.help) {
    usage(std::cout);
    return 0;
  }
  if(o.version) {
    std::cout << "Quantum Electromagnetics Simulation Toolbox (QuEST), B200 build, library " << qg_version()
              << std::endl;
    return 0;
  }
  std::ifstream cfg(o.config);
  if(!cfg) {
    std::cerr << "ERROR: " << o.config << " not found" << std::endl;
    return 0;  // the reference reports this and exits normally
  }
  try {
    const auto kv = read_config(cfg);
    qg_params p;
    std::memset(&p, 0, sizeof p);
    p.c0 = number(kv, "constants.c0");
    p.hbar = number(kv, "constants.hbar");
    p.mu0 = number(kv, "constants.mu0");
    p.laser_frequency = number(kv, "constants.laser_frequency");
    const int num_particles = (int)number(kv, "parameters.num_particles");
    const double total_time = number(kv, "parameters.total_time");
    p.dt = number(kv, "parameters.timestep");
    p.interpolation_order = (int)number(kv, "parameters.interpolation_order");
    p.num_timesteps = (int)std::ceil(total_time / p.dt);
    p.frame = QG_FRAME_ROTATING;  // main.cpp:40-41 uses the rotating dyadic
    p.precision = o.precision;
    p.coef_mode = o.coef_mode;
    const std::string qd_path = kv.count("files.qd_path") ? kv.at("files.qd_path") : "dots.cfg";
    const std::string pulse_path = kv.count("files.pulse_path") ? kv.at("files.pulse_path") : "pulse.cfg";

    std::cout << "Initializing..." << std::endl;
    const std::vector<qg_dot> dots = read_dots(qd_path, num_particles);
    const qg_pulse pulse = read_pulse(pulse_path);
    quest_gpu::Simulation sim(dots, pulse, p);

    // the trajectory is computed in chunks into host memory, then written;
    // the whole run is kept so that a non-finite state leaves no output
    std::cout << "Solving..." << std::endl;
    const int n = num_particles, T = p.num_timesteps;
    std::vector<quest_gpu::cmplx> traj((size_t)T * n * 2);
    const int chunk = 1024;
    for(int t = 0; t < T; t += chunk) sim.run(std::min(chunk, T - t), traj.data() + (size_t)t * n * 2);

    std::cout << "Writing output..." << std::endl;
    std::FILE *f = std::fopen(o.output.c_str(), "w");
    if(!f) throw std::runtime_error("Could not open " + o.output);
    for(int t = 0; t < T; ++t) quest_gpu::write_step(f, traj.data() + (size_t)t * n * 2, n);
    std::fclose(f);
  } catch(const std::domain_error &e) {
    std::cerr << "terminate called after throwing an instance of 'std::domain_error'\n  what():  " << e.what()
              << std::endl;
    return 1;
  } catch(const std::exception &e) {
    std::cerr << "ERROR: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
