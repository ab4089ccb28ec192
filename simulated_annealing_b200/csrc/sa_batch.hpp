// sa_batch.hpp -- device-visible tables of the batched persistent engine.
#pragma once
#include <cstdint>

#include "sa_device.cuh"

namespace sa {

// Acceptance thresholds of one temperature at h = 0 (spin up and down share
// them): dn[k] for k satisfied bonds, bdn[k] for open-x border sites.
struct BThr {
  uint32_t dn[8];
  uint32_t bdn[8];
};

// One exchange attempt of a ladder: pair (i, i+1) and the accepted interval
// lo <= dE <= hi of dE = E_{i+1} - E_i (the reference's -(E_i - E_{i+1})).
struct Decision {
  int32_t pair, lo, hi, pad;
};

// Launch shape of the resident kernel for one bucket of instances
// (lattice, L, slots): cluster size C, slots per lane SL (lanes per site
// follow), warps per block, and the high-register form (two-slot 3D only).
// Chosen per bucket by timing on the GPU (simulated_annealing_b200/autotune.py).
struct TuneEntry {
  int32_t lattice, L, nslots, C, SL, warps, hr;
};

struct InstDesc {
  int32_t lattice, L, nslots, P;   // P: lanes per site group (pow2 >= nslots, <= 32)
  int32_t ladder, sched;           // exactly one >= 0
  int32_t sweeps_per_step, thr_count;
  int64_t N, half, nbonds;
  int64_t spin_off;                // words; layout [colour][row][k][slot]
  int64_t J_off;                   // words; layout [axis][colour][row][k]
  int64_t thr_off;                 // index of slot 0 / step 0 in the threshold pool
  int64_t dec_off, dec_count;      // ladder's exchange table
  int64_t pair_off;                // acceptance counters (nslots-1 pairs)
  int64_t hist_off;                // energy histograms: nslots x (nbonds+1) bins, -1 = none
  int64_t state_idx;               // index of this instance's InstState
  uint64_t seed;
  int64_t sweep_limit;             // anneal: steps * sweeps_per_step; PT: -1
};

struct InstState {
  uint64_t draw;     // next Philox draw index of every site
  int64_t sweeps;    // sweeps done
  int64_t xsteps;    // exchange attempts done
  int64_t emax[64];  // anneal: running max of -H per replica
  int64_t elast[64]; // anneal: last measured -H per replica
  int64_t measured;  // anneal: number of measurements folded
};

struct BatchParams {
  const InstDesc* inst;
  InstState* state;
  const int32_t* order;    // work order (most expensive first)
  int32_t ninst;
  int32_t* work;           // work-queue counter (zeroed before the launch)
  word_t* spins;
  const word_t* J;
  const BThr* thr;
  const Decision* dec;
  int64_t* acc;            // accepted replicas per pair
  int64_t* att;            // attempts per pair
  int32_t* rec_pair;       // optional exchange record [inst][cap]
  uint64_t* rec_mask;
  int64_t rec_cap;
  int64_t nsweeps;         // requested sweeps this launch
  int32_t xinterval;       // sweeps between exchanges
  int32_t mstride;         // anneal measure stride (0 = never)
  int32_t* hist;           // energy histograms (bin (E+nbonds)/2), or null
  int32_t hstride;         // histogram every hstride sweeps
  int64_t* step_rec;       // anneal: last measured -H at the end of every step
                           // [state][step][64], or null
};

}  // namespace sa
