// sa_cli.cpp -- the annealing / parallel-tempering command-line front end
// (the reference's annealing_gpu, src/main_gpu.cu) on this engine: the same
// flags (src/main_gpu.cu:56-131), the same modes and the same output.
//
//   timing   -t: sweeps of one system timed one by one with CUDA events;
//            seconds per replica spin-flip attempt: mean, std, min, max
//            (src/main_gpu.cu:159-210).
//   anneal   -T: annealing over one system, T *= a after every step of -S
//            sweeps; the -H vector after every sweep (PRINT_E), or with -r
//            the running maximum after each of r restarts from new random
//            spins (PRINT_MIN) (src/main_gpu.cu:280-303).
//   PT       -P/--Pb/--P_file/--reload: parallel tempering, -s steps of -S
//            sweeps + one exchange attempt; with -r, r independent runs
//            continued in chunks of -s steps, each checkpointed to
//            <tmp><id>_<i>.tempsys, until for every replica more than half
//            of the runs agree on the lowest energy (repeat until ground
//            state, src/main_gpu.cu:304-415, src/tools.hpp:6-33); SIGUSR1
//            copies the checkpoints to --home and prints the --reload
//            command line.
//
// Systems are built as the reference builds them (src/main_gpu.cu:251-277):
// set_seed(seed); init_J (or load_J); set_seed(seed); init_rand. -d takes
// the reference's 2p (gpu_2d: open in x) and 3, and also 2 (cpu_2d's fully
// periodic lattice); --rng mt19937_64 draws from the CPU reference's stream.
//
// --two-lattice runs the reference GPU systems' own shape, 128 replicas per
// system (b200_sys128: the two configurations of gpu_2d's / gpu_3d's two
// lattices); without it a system holds 64 replicas (one lattice, as the CPU
// classes). A PT run's E_min is split into vectors of 64 per run and the
// repeat loop stops when, for every replica, more than half of those vectors
// hold the lowest energy -- with 128 replicas exactly the reference's test
// (two vectors per run, more than r of 2r, src/main_gpu.cu:387-396).
//
// Differences, each a reference defect: the timing mode's min and max are
// computed (the reference starts them at NAN and std::min/max keep NAN);
// --reload reads the number of temperatures from the checkpoint (the
// reference builds one system and overruns it).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <csignal>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "sa_b200.h"
#include "sa_b200_drivers.hpp"
#include "sa_b200_sys.hpp"

using sa_b200::annealing;
using sa_b200::parallel_tempering;
using sa_b200::PRINT_E;
using sa_b200::PRINT_MIN;

namespace {

volatile std::sig_atomic_t g_usr1 = 0;
void on_signal(int s) {
  if (s == SIGUSR1) g_usr1 = 1;
}

int g_verbosity = 4;
const char* kLogFile = "gpulogfile.log";

// LOG(LOG_INFO)-style messages: stderr and the log file
void log_msg(int level, const std::string& msg) {
  if (level > g_verbosity) return;
  static const char* label[] = {"", "", "Error:   ", "Warning: ", "Info:    ", "Timing:  ", "Debug:   "};
  const std::string line = std::string(label[std::min(level, 6)]) + msg;
  std::cerr << line << std::endl;
  std::ofstream f(kLogFile, std::ios::app);
  if (f) f << line << "\n";
}
enum { LOG_ERROR = 2, LOG_WARNING = 3, LOG_INFO = 4 };

// A temperature block "start step stop" (src/block.cpp): size() values
// start + i*step, the last one clamped to stop.
struct Block {
  double start = 0, step = 0, stop = 0;
  int size() const {
    if ((start + (int)((stop - start) / step) * step) < stop * 0.9999) return (int)((stop - start) / step + 2);
    return (int)((stop - start) / step + 1);
  }
  double at(int i) const { return std::min(start + i * step, stop); }
};

bool parse_block(const std::string& s, Block* b) {
  std::string t = s;
  std::replace(t.begin(), t.end(), ',', ' ');
  std::istringstream in(t);
  if (!(in >> b->start >> b->step >> b->stop)) return false;
  if (b->start > b->stop || !(b->step > 0)) return false;
  return true;
}

struct Options {
  int steps = 100, sweeps = 100, L = 64, repeat = 1, maxiter = 10;
  double a = 0.9, T = 2.26, h = 0.0;
  long seed = 1234;
  long verbosity = 4;
  std::vector<double> P;
  std::vector<Block> Pb;
  std::string P_file, reload, output = "cout", outputT = "out_%.dat", load_J, save_J, dim = "2p";
  std::string tmp = "/tmp/", home = ".", rng = "philox";
  bool timing = false, image = false, swap = false, two_lattice = false;
  bool T_set = false, P_set = false, Pb_set = false, P_file_set = false, reload_set = false;
  bool repeat_set = false, maxiter_set = false, output_set = false;
};

[[noreturn]] void usage(const char* prog, const std::string& err) {
  if (!err.empty()) std::cerr << "PARSE ERROR: " << err << "\n\n";
  std::cerr << "USAGE: " << prog
            << " {-T <double>|-P <double> ...|--Pb \"start step stop\" ...|--P_file <file>|--reload <prefix>}\n"
               "  [-s|--steps <int>=100] [-a|--a <double>=0.9] [-S|--sweeps <int>=100] [-L|--size <int>=64]\n"
               "  [-m|--h <double>=0] [-o|--output <file>] [--outputT <name with %>=out_%.dat] [--seed <long>=1234]\n"
               "  [-j|--load_J <file>] [-J|--save_J <file>] [-d|--dim 2p|3|2] [-t|--timing] [-i|--image] [--swap]\n"
               "  [-v|--verbosity <int>=4] [-r|--repeat <int>=1] [--tmp <dir>=/tmp/] [--home <dir>=.]\n"
               "  [--maxiter <int>=10] [--rng philox|mt19937_64] [--two-lattice]\n";
  std::exit(1);
}

Options parse(int argc, char** argv) {
  Options o;
  // "--name=value" is "--name value"
  std::vector<std::string> args;
  for (int i = 1; i < argc; ++i) {
    const std::string t = argv[i];
    const size_t eq = t.find('=');
    if (t.rfind("--", 0) == 0 && eq != std::string::npos) {
      args.push_back(t.substr(0, eq));
      args.push_back(t.substr(eq + 1));
    } else {
      args.push_back(t);
    }
  }
  auto num = [&](const std::string& v, const std::string& name) -> double {
    char* end = nullptr;
    const double d = std::strtod(v.c_str(), &end);
    if (end == v.c_str() || *end) usage(argv[0], "bad value \"" + v + "\" for " + name);
    return d;
  };
  auto integer = [&](const std::string& v, const std::string& name) -> long {
    char* end = nullptr;
    const long d = std::strtol(v.c_str(), &end, 10);
    if (end == v.c_str() || *end) usage(argv[0], "bad value \"" + v + "\" for " + name);
    return d;
  };
  for (size_t i = 0; i < args.size(); ++i) {
    const std::string a = args[i];
    auto v = [&](const std::string& name) -> std::string {
      if (i + 1 >= args.size()) usage(argv[0], "missing value for " + name);
      return args[++i];
    };
    if (a == "-s" || a == "--steps") o.steps = (int)integer(v(a), a);
    else if (a == "-a" || a == "--a") o.a = num(v(a), a);
    else if (a == "-S" || a == "--sweeps") o.sweeps = (int)integer(v(a), a);
    else if (a == "-L" || a == "--size") o.L = (int)integer(v(a), a);
    else if (a == "-T" || a == "--T") { o.T = num(v(a), a); o.T_set = true; }
    else if (a == "-P" || a == "--parallel_tempering") { o.P.push_back(num(v(a), a)); o.P_set = true; }
    else if (a == "--Pb") {
      Block b;
      const std::string s = v(a);
      if (!parse_block(s, &b)) usage(argv[0], "bad temperature block \"" + s + "\" (start step stop)");
      o.Pb.push_back(b);
      o.Pb_set = true;
    } else if (a == "--P_file") { o.P_file = v(a); o.P_file_set = true; }
    else if (a == "--reload") { o.reload = v(a); o.reload_set = true; }
    else if (a == "-m" || a == "--h") o.h = num(v(a), a);
    else if (a == "-o" || a == "--output") { o.output = v(a); o.output_set = true; }
    else if (a == "--outputT") o.outputT = v(a);
    else if (a == "--seed") o.seed = integer(v(a), a);
    else if (a == "-j" || a == "--load_J") o.load_J = v(a);
    else if (a == "-J" || a == "--save_J") o.save_J = v(a);
    else if (a == "-d" || a == "--dim") {
      o.dim = v(a);
      if (o.dim != "2p" && o.dim != "3" && o.dim != "2") usage(argv[0], "-d must be 2p, 3 or 2");
    } else if (a == "-t" || a == "--timing") o.timing = true;
    else if (a == "-i" || a == "--image") o.image = true;
    else if (a == "--swap") o.swap = true;
    else if (a == "--two-lattice") o.two_lattice = true;
    else if (a == "-v" || a == "--verbosity") o.verbosity = integer(v(a), a);
    else if (a == "-r" || a == "--repeat") { o.repeat = (int)integer(v(a), a); o.repeat_set = true; }
    else if (a == "--tmp") o.tmp = v(a);
    else if (a == "--home") o.home = v(a);
    else if (a == "--maxiter") { o.maxiter = (int)integer(v(a), a); o.maxiter_set = true; }
    else if (a == "--rng") {
      o.rng = v(a);
      if (o.rng != "philox" && o.rng != "mt19937_64") usage(argv[0], "--rng must be philox or mt19937_64");
    } else if (a == "-h" || a == "--help") usage(argv[0], "");
    else usage(argv[0], "unknown argument " + a);
  }
  const int xo = o.T_set + o.P_set + o.Pb_set + o.P_file_set + o.reload_set;
  if (xo != 1) usage(argv[0], "exactly one of -T, -P, --Pb, --P_file, --reload is required");
  if (o.repeat < 1) usage(argv[0], "-r must be >= 1");
  if (o.two_lattice && o.rng != "philox") usage(argv[0], "--two-lattice runs in Philox mode only");
  return o;
}

int lattice_of(const std::string& d) {
  return d == "3" ? SA_LATTICE_3D : d == "2" ? SA_LATTICE_2D : SA_LATTICE_2D_OPEN_X;
}

template <class Sys>
Sys* make_system(const Options& o, double T) {
  Sys* s = new Sys(lattice_of(o.dim), o.L, T, o.h);
  if (o.rng == "mt19937_64") s->set_rng_mode(SA_RNG_MT19937_64);
  return s;
}

// annealing<>'s running maximum over a whole schedule on the device
// (sa_sys_anneal), for each of the system's 64-replica lattices
std::vector<float> anneal_min(b200_sys* s, const std::vector<double>& sched, int sweeps) {
  std::vector<float> mn(64, 0.f);
  if (sa_sys_anneal(s->handle(), sched.data(), (int)sched.size(), sweeps, 1, mn.data(), nullptr) != SA_OK)
    log_msg(LOG_ERROR, std::string("anneal: ") + sa_last_error());
  return mn;
}
std::vector<float> anneal_min(b200_sys128* s, const std::vector<double>& sched, int sweeps) {
  std::vector<float> a = anneal_min(&s->first(), sched, sweeps), b = anneal_min(&s->second(), sched, sweeps);
  a.insert(a.end(), b.begin(), b.end());
  return a;
}

// 5 random lowercase letters (the reference's random_string, src/random_str.cpp)
std::string random_id() {
  std::mt19937 gen{std::random_device{}()};
  std::uniform_int_distribution<int> dist{'a', 'z'};
  std::string s(5, 'a');
  for (auto& c : s) c = (char)dist(gen);
  return s;
}

// For every replica: how many of the n vectors hold the largest value
// (src/tools.hpp:6-24).
std::vector<int> max_count(const std::vector<std::vector<float>>& x) {
  std::vector<int> count(x[0].size(), 1);
  std::vector<float> mx = x[0];
  for (size_t i = 1; i < x.size(); ++i)
    for (size_t j = 0; j < count.size() && j < x[i].size(); ++j) {
      if (mx[j] < x[i][j]) {
        mx[j] = x[i][j];
        count[j] = 1;
      } else if (mx[j] == x[i][j]) {
        count[j]++;
      }
    }
  return count;
}

template <class Sys>
int run_timing(const Options& o) {
  Sys* s = make_system<Sys>(o, o.T);
  cudaStream_t st;
  cudaStreamCreate(&st);
  s->set_stream(st);
  s->init_J();
  s->init_rand();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double t = 0, t2 = 0, tmin = INFINITY, tmax = 0;
  for (int i = 0; i < o.steps; ++i) {
    cudaEventRecord(e0, st);
    s->sweep();
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    t += ms;
    t2 += (double)ms * ms;
    tmin = std::min(tmin, (double)ms);
    tmax = std::max(tmax, (double)ms);
  }
  int dev = 0;
  cudaDeviceProp prop;
  cudaGetDevice(&dev);
  cudaGetDeviceProperties(&prop, dev);
  log_msg(LOG_INFO, sa_version());
  log_msg(LOG_INFO, prop.name);
  std::ostringstream a, b;
  a << o.dim << "\t" << o.L << "\t" << o.steps;
  log_msg(LOG_INFO, a.str());
  const double flips = (double)s->get_N() * Sys::replicas();  // src/main_gpu.cu:199: N*64*2 for 128
  const double m = t / (o.steps * 1000 * flips);
  b << m << "\t" << std::sqrt(std::max(0.0, t2 / (o.steps * 1000 * flips) / (1000 * flips) - m * m)) << "\t"
    << tmin / (1000 * flips) << "\t" << tmax / (1000 * flips);
  log_msg(LOG_INFO, b.str());
  // the same figures on stdout for scripts: seconds per attempt, then attempts/ns
  std::cout << m << "\t" << 1e-9 / m << std::endl;
  s->gpu_free();
  delete s;
  cudaStreamDestroy(st);
  return 0;
}

std::vector<double> temperatures(const Options& o) {
  std::vector<double> T;
  if (o.P_set) return o.P;
  std::vector<Block> blocks = o.Pb;
  if (o.P_file_set) {
    std::ifstream f(o.P_file);
    if (!f.is_open()) {
      log_msg(LOG_ERROR, "cannot open temperature block file " + o.P_file);
      std::exit(-1);
    }
    Block b;
    while (f >> b.start >> b.step >> b.stop) blocks.push_back(b);
  }
  for (const Block& b : blocks)
    for (int j = 0; j < b.size(); ++j) T.push_back(b.at(j));
  return T;
}

// the number of temperatures a .tempsys checkpoint holds (its T vector)
long checkpoint_slots(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return -1;
  size_t glen = 0;
  sa_pt_gen_t g = nullptr;
  sa_pt_gen_create(2, &g);
  sa_pt_gen_save(g, nullptr, 0, &glen);
  sa_pt_gen_destroy(g);
  f.seekg((std::streamoff)(sizeof(long) + 2 + glen));
  size_t n = 0;
  f.read(reinterpret_cast<char*>(&n), sizeof n);
  f.seekg((std::streamoff)n, std::ios::cur);
  f.read(reinterpret_cast<char*>(&n), sizeof n);
  return f ? (long)n : -1;
}

}  // namespace

template <class Sys>
int run(const Options& o, int argc, char** argv) {
  std::string info = "#";
  for (int i = 0; i < argc; ++i) info += std::string(" ") + argv[i];
  info += "\n# Version : ";
  info += sa_version();
  info += "\n";
  const std::string rand_id = random_id();

  if (o.timing) return run_timing<Sys>(o);

  std::ostream* fp = &std::cout;
  std::ofstream fout;
  if (o.output_set) {
    fout.open(o.output);
    if (!fout.is_open()) {
      log_msg(LOG_ERROR, "cannot open the output file " + o.output);
      return -1;
    }
    fp = &fout;
  }

  std::vector<double> T;
  int num = 1;
  if (o.P_set || o.Pb_set || o.P_file_set) {
    T = temperatures(o);
    num = (int)T.size();
  } else if (o.reload_set) {
    const long n = checkpoint_slots(o.reload + "_0.tempsys");
    if (n < 2) {
      log_msg(LOG_ERROR, "cannot read the checkpoint " + o.reload + "_0.tempsys");
      return -1;
    }
    num = (int)n;
    T.assign(num, o.T);
  }
  std::vector<Sys*> sys;
  for (int i = 0; i < num; ++i) {
    Sys* s = make_system<Sys>(o, o.T);
    if (!o.load_J.empty()) {
      s->load_J(o.load_J);
    } else {
      s->set_seed(o.seed);
      s->init_J();
      if (!o.save_J.empty()) s->save_J(o.save_J);
    }
    s->set_seed(o.seed);
    s->init_rand();
    sys.push_back(s);
  }

  if (o.T_set) {
    annealing<Sys> annealer(o.T, o.sweeps, o.a, sys[0], *fp);
    (*fp) << info;
    if (!o.repeat_set) {
      for (int i = 0; i < o.steps; ++i) annealer.step(1, PRINT_E);
    } else {
      // PRINT_MIN: each restart's schedule on the device (sa_sys_anneal keeps
      // the template's running maximum of the measured -H). Step k runs at
      // T*a^k; the template's set_T resets only the driver's temperature, so
      // every restart after the first begins at the previous run's last
      // cooled temperature T*a^steps (src/annealing.hpp:96-98, :129-139).
      std::vector<double> sched(std::max(o.steps, 1));
      for (int k = 0; k < o.steps; ++k) sched[k] = (k == 0) ? o.T : sched[k - 1] * o.a;
      double last = o.T;
      for (int k = 0; k < o.steps; ++k) last *= o.a;
      for (int j = 0; j < o.repeat; ++j) {
        if (j == 1 && o.steps > 0) sched[0] = last;
        std::vector<float> mn(Sys::replicas(), 0.f);
        if (o.steps > 0) mn = anneal_min(sys[0], std::vector<double>(sched.begin(), sched.begin() + o.steps), o.sweeps);
        sys[0]->set_T(last);
        for (float v : mn) (*fp) << v << "\t";
        (*fp) << std::endl;
        sys[0]->init_rand();
      }
    }
  } else {
    if (o.P_set && T.size() < 2) {
      log_msg(LOG_ERROR, "not enough temperatures: " + std::to_string(T.size()));
      return -1;
    }
    if (o.swap) (*fp) << info;
    parallel_tempering<Sys> tempering(sys, T, o.sweeps, o.outputT);
    tempering.set_info(info, o.repeat_set ? PRINT_MIN : PRINT_E);
    const int nrep = o.repeat;
    std::vector<std::vector<float>> E_min;
    bool found = false, first = true;
    int count = -1;
    auto tmpname = [&](int i) { return o.tmp + rand_id + "_" + std::to_string(i) + ".tempsys"; };
    while (!found) {
      count++;
      if (g_usr1) {
        const std::string cmd = "cp " + o.tmp + rand_id + "_* " + o.home;
        if (std::system(cmd.c_str()) != 0) log_msg(LOG_ERROR, "copying the checkpoints failed");
        for (int i = 0; i < argc; ++i) std::cout << " " << argv[i];
        std::cout << " --reload " << o.home + "/" + rand_id << std::endl;
        return 0;
      }
      E_min.clear();
      for (int i = 0; i < nrep; ++i) {
        if (!first) {
          std::ifstream in(tmpname(i), std::ios::binary);
          if (!in.good()) log_msg(LOG_ERROR, "error opening " + tmpname(i));
          tempering.load(in);
        } else if (o.reload_set) {
          std::ifstream in(o.reload + "_" + std::to_string(i) + ".tempsys", std::ios::binary);
          tempering.load(in);
        }
        for (int j = 0; j < o.steps; ++j) tempering.step(o.repeat_set ? 0 : 1);
        if (o.swap) tempering.print_swap(*fp);
        if (o.repeat_set) {
          std::ofstream out(tmpname(i), std::ios::binary | std::ios::out | std::ios::trunc);
          if (!out.good()) log_msg(LOG_ERROR, "error opening " + tmpname(i));
          const std::vector<float> e = tempering.get_E_min();
          for (size_t w = 0; w + 64 <= e.size(); w += 64) E_min.emplace_back(e.begin() + w, e.begin() + w + 64);
          tempering.save(out);
          out.close();
          tempering.reset();
        }
      }
      if (o.repeat_set && nrep != 1) {
        first = false;
        const std::vector<int> c = max_count(E_min);
        found = true;
        for (int v : c) found = found && (2 * v > (int)E_min.size());
      } else {
        found = true;
      }
      if (o.maxiter_set && count > o.maxiter) found = true;
      if (found && o.repeat_set) {
        for (int i = 0; i < nrep; ++i) {
          std::ifstream in(tmpname(i), std::ios::binary);
          tempering.load(in);
          tempering.print(PRINT_MIN);
        }
      }
    }
    if (o.image)
      for (Sys* s : tempering.systems()) s->save_sys("gpu_sys_");
  }
  if (o.T_set && o.image) sys[0]->save_sys("gpu_sys_");
  for (Sys* s : sys) {
    s->gpu_free();
    delete s;
  }
  return 0;
}

int main(int argc, char** argv) {
  std::signal(SIGUSR1, on_signal);
  Options o = parse(argc, argv);
  g_verbosity = (int)o.verbosity;
  return o.two_lattice ? run<b200_sys128>(o, argc, argv) : run<b200_sys>(o, argc, argv);
}
