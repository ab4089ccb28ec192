// Drop-in proof: the reference's own annealing<gpu_sys> and
// parallel_tempering<gpu_sys> templates (src/annealing.hpp,
// src/parallel_tempering.hpp, unmodified, included from the reference tree at
// build time) driving this engine's b200 systems through gpu_sys.
//
//   dropin pt <lattice> <L> <nslots> <seed_J> <seed> <steps> <T...>
//   dropin anneal <lattice> <L> <seed_J> <seed> <T0> <alfa> <nsteps> <sweeps>
// Output lines: "X <pair> <mask>" per exchange, "E <slot> <64 floats>",
// "S <slot> <N words>", "A <acceptance per pair>", "M <64 floats>".
#include "gpu_sys.cuh"
#define SA_HAVE_REFERENCE_GPU_SYS
#include "sa_b200_sys.hpp"

#include "annealing.hpp"
#include "parallel_tempering.hpp"

#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

struct Log {
  std::vector<std::pair<int, unsigned long long>> swaps;
};

// forwards every call; records the exchanges the template decides
class spy : public gpu_sys {
 public:
  b200_sys* in;
  int id;
  Log* log;
  spy(b200_sys* s, int i, Log* l) : in(s), id(i), log(l) {}
  void sweep() override { in->sweep(); }
  void set_T(double T) override { in->set_T(T); }
  void set_h(double h) override { in->set_h(h); }
  void set_seed(long long s) override { in->set_seed(s); }
  vector<float> measure() override { return in->measure(); }
  void gpu_free() override { in->gpu_free(); }
  void load_J(string f) override { in->load_J(f); }
  void save_J(string f) override { in->save_J(f); }
  void init_J() override { in->init_J(); }
  void init_rand() override { in->init_rand(); }
  void save_sys(string p) override { in->save_sys(p); }
  long get_N() override { return in->get_N(); }
  void swap(gpu_sys* o, std::unique_ptr<spin_t[]> m) override {
    log->swaps.push_back({id, m[0]});
    in->swap(static_cast<spy*>(o)->in, std::move(m));
  }
  ostream& save(ostream& s) override { return in->save(s); }
  istream& load(istream& s) override { return in->load(s); }
};

static void print_spins(b200_sys* s, int slot) {
  std::vector<uint64_t> w(s->get_N());
  s->get_spins(w.data());
  std::cout << "S " << slot;
  for (uint64_t v : w) std::cout << " " << v;
  std::cout << "\n";
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  std::string mode = argv[1];
  std::cout.precision(9);
  if (mode == "pt") {
    int lat = atoi(argv[2]), L = atoi(argv[3]), n = atoi(argv[4]);
    long long sJ = atoll(argv[5]), s = atoll(argv[6]);
    int steps = atoi(argv[7]);
    std::vector<double> T;
    for (int i = 0; i < n; ++i) T.push_back(atof(argv[8 + i]));
    Log log;
    std::vector<b200_sys*> sys;
    std::vector<gpu_sys*> spies;
    for (int i = 0; i < n; ++i) {
      sys.push_back(new b200_sys(lat, L, 1.0, 0.0));
      // the reference driver's set-up order (src/main_gpu.cu:262-276)
      sys[i]->set_seed(sJ);
      sys[i]->init_J();
      sys[i]->set_seed(s);
      sys[i]->init_rand();
      spies.push_back(new spy(sys[i], i, &log));
    }
    std::string fname = "unused_%";
    parallel_tempering<gpu_sys> pt(spies, T, 1, fname);
    for (int k = 0; k < steps; ++k) pt.step(0);
    for (auto& e : log.swaps) std::cout << "X " << e.first << " " << e.second << "\n";
    for (int i = 0; i < n; ++i) {
      std::vector<float> E = sys[i]->measure();
      std::cout << "E " << i;
      for (float v : E) std::cout << " " << v;
      std::cout << "\n";
      print_spins(sys[i], i);
    }
    std::ostringstream acc;
    pt.print_swap(acc);
    std::istringstream in(acc.str());
    std::string line;
    std::cout << "A";
    while (std::getline(in, line)) std::cout << " " << line.substr(line.find(':') + 1);
    std::cout << "\n";
    for (auto* p : spies) delete p;
    for (auto* p : sys) delete p;
  } else if (mode == "anneal") {
    int lat = atoi(argv[2]), L = atoi(argv[3]);
    long long sJ = atoll(argv[4]), s = atoll(argv[5]);
    double T0 = atof(argv[6]), alfa = atof(argv[7]);
    int nsteps = atoi(argv[8]), sweeps = atoi(argv[9]);
    b200_sys sys(lat, L, T0, 0.0);
    sys.set_seed(sJ);
    sys.init_J();
    sys.set_seed(s);
    sys.init_rand();
    std::ostringstream out;
    annealing<gpu_sys> a(T0, sweeps, alfa, &sys, out);
    for (int k = 0; k < nsteps; ++k) a.step(1, PRINT_MIN);
    std::ostringstream mn;
    annealing<gpu_sys>* ap = &a;
    (void)mn;
    ap->print(PRINT_MIN);
    std::cout << "M " << out.str();
    print_spins(&sys, 0);
  } else {
    return 2;
  }
  return 0;
}
