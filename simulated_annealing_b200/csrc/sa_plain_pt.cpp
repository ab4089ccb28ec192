// sa_plain_pt -- the plain one-instance-per-launch form of parallel tempering,
// timed for comparison with the batched engine.
//
// Each instance is run the way parallel_tempering<gpu_sys>
// (src/parallel_tempering.hpp:81-115) runs gpu_2d/gpu_3d systems: one system
// per temperature slot, and every step sweeps each slot once (one launch per
// half-sweep), measures each slot (a device->host copy), draws the exchange
// pair and uniform from the std::mt19937(123) sequence and swaps the accepted
// replica bits. Instances run one after another on one stream each.
//
//   sa_plain_pt <budget_seconds> <sweeps>   < lines "lattice L seed n T1 .. Tn"
//
// Prints "instances <k> attempts <a> seconds <t>" for the timed sweep loops
// (system set-up excluded), stopping after the instance during which the
// budget ran out.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "sa_b200.h"

static void die(int st, const char* what) {
  std::fprintf(stderr, "sa_plain_pt: %s: %s (%s)\n", what, sa_status_string(st), sa_last_error());
  std::exit(1);
}

#define TRY(x)                   \
  do {                           \
    int st_ = (x);               \
    if (st_ != SA_OK) die(st_, #x); \
  } while (0)

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: sa_plain_pt <budget_seconds> <sweeps>  < instance lines\n");
    return 2;
  }
  const double budget = std::atof(argv[1]);
  const int sweeps = std::atoi(argv[2]);
  double seconds = 0;
  long double attempts = 0;
  long done = 0;
  std::string line;
  while (seconds < budget && std::getline(std::cin, line)) {
    std::istringstream in(line);
    int lat, L, n;
    unsigned long long seed;
    if (!(in >> lat >> L >> seed >> n) || n < 2) continue;
    std::vector<double> T(n);
    for (double& t : T) in >> t;
    std::vector<sa_system_t> sys(n, nullptr);
    for (int j = 0; j < n; ++j) {
      TRY(sa_sys_create(lat, L, T[j], 0.0, &sys[j]));
      TRY(sa_sys_set_seed(sys[j], seed));
      TRY(sa_sys_init_J(sys[j]));
      TRY(sa_sys_set_seed(sys[j], seed));
      TRY(sa_sys_init_rand(sys[j]));
    }
    long N = 0;
    TRY(sa_sys_get_N(sys[0], &N));
    std::vector<int32_t> pair(sweeps);
    std::vector<double> r(sweeps);
    TRY(sa_pt_sequence(n, 0, sweeps, pair.data(), r.data()));
    std::vector<std::vector<float>> E(n, std::vector<float>(64));
    for (int j = 0; j < n; ++j) TRY(sa_sys_sync(sys[j]));
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < sweeps; ++k) {
      for (int j = 0; j < n; ++j) {
        TRY(sa_sys_sweep(sys[j], 1));
        TRY(sa_sys_measure_float(sys[j], E[j].data()));
      }
      const int i = pair[k];
      const uint64_t mask = sa_pt_mask(E[i].data(), E[i + 1].data(), T[i], T[i + 1], r[k]);
      TRY(sa_sys_swap(sys[i], sys[i + 1], mask));
    }
    for (int j = 0; j < n; ++j) TRY(sa_sys_sync(sys[j]));
    seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    attempts += (long double)sweeps * n * N * 64;
    done += 1;
    for (auto s : sys) sa_sys_destroy(s);
  }
  std::printf("instances %ld attempts %.0Lf seconds %.6f\n", done, attempts, seconds);
  return 0;
}
