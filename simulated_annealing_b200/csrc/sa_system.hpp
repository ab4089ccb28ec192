// sa_system.hpp -- the single-system handle behind sa_system_t.
#pragma once
#include <cuda_runtime.h>

#include "sa_device.cuh"

struct sa_system {
  int lattice = 0, dim = 2, L = 0;
  long N = 0, half = 0, nbonds = 0;
  double T = 1.0, h = 0.0;
  unsigned long long seed = 1234, draw = 0, epoch = 0;
  int device = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  sa::word_t* d_s = nullptr;       // spins [colour][row][k]
  sa::word_t* d_J = nullptr;       // own couplings [axis][colour][row][k]
  sa::word_t* d_stage = nullptr;   // row-major staging for host transfers
  unsigned long long* d_counts = nullptr;  // measure scratch (128 counters)
  int64_t* d_EM = nullptr;         // measure output E[64], M[64]
  sa::Thresholds thr{};
  // Random-number mode: SA_RNG_PHILOX (the GPU reference's schedule; seed and
  // draw counter above) or SA_RNG_MT19937_64 (the CPU reference's stream; its
  // state lives on the device in d_mt, the pass's outputs in d_draws).
  int rng_mode = 0;
  // Colour of the first half-sweep of every sweep (draw t+2n; the other
  // colour takes t+2n+1). 1 is the second configuration of the reference GPU
  // systems' two-lattice pair (src/gpu_2d.cu:109-120): its odd sites are
  // updated first. Philox mode only.
  int first_colour = 0;
  // The reference's SPLIT_H update (bond and field parts accepted with two
  // draws per site per half-sweep: t+2m and t+2m+1); Philox mode only.
  int split = 0;
  sa::SplitThresholds sthr{};
  uint64_t* d_mt = nullptr;        // [kMtN + 1]: state words, next index
  uint64_t* d_draws = nullptr;     // dim * N outputs (init_J is the largest pass)
  sa::ThresholdsMT thr_mt{};
};

namespace sa {
int launch_halfsweep(sa_system* sy, int c, unsigned long long draw);
// MT mode: one sweep drawing its N outputs from the device generator.
int mt_sweep(sa_system* sy);
// MT mode: the device generator's next n outputs into d_draws.
int mt_generate(sa_system* sy, long n);
int launch_measure(sa_system* sy, int64_t* d_E, int64_t* d_M);
// The shared-memory-resident batch kernel applied to one system (zero field,
// L >= 4): nsteps steps of `sweeps` sweeps at T[k], -H measured every `stride`
// sweeps of a step (0 = never). Host outputs, each may be null: Emax[64]
// (running max of -H), step_E[nsteps*64] (last measurement of every step),
// *measured (measurements taken). Advances the system's draw counter.
bool resident_ok(const sa_system* sy);
int resident_run(sa_system* sy, const double* T, int nsteps, int sweeps, int stride, int64_t* Emax,
                 int64_t* step_E, int* measured);
}  // namespace sa
