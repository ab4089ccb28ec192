// sa_host.hpp -- host-side helpers shared by the engine's translation units:
// error state, Boltzmann tables, integer thresholds, PT decision intervals.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "sa_types.hpp"

namespace sa {

// Per-thread last-error message behind sa_last_error().
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define SA_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t sa_e_ = (expr);                             \
    if (sa_e_ != cudaSuccess) return ::sa::cuda_fail(sa_e_, #expr); \
  } while (0)

// Boltzmann table exactly as the reference builds it (double, glibc exp):
// 2D src/cpu_2dp.cpp:33-40 (20 entries), 3D src/cpu_3d.cpp:218-232 (14 entries).
void boltz_table(int lattice, double T, double h, double* out20);

// u32 -> float in (0,1] used by the reference's per-site uniform draw; the
// midpoint of bucket u (u rounded to binary32, times 2^-32, plus 2^-33).
float uniform_from_u32(uint32_t u);
// Number of u32 values whose uniform is below b (monotone, so u < thr(b)
// is exactly uniform(u) < b).
uint32_t threshold_of(float b);
// Integer thresholds of a lattice at (T, h): float-cast table, then thr().
// Returns false if the table is not monotone where the kernels need it.
bool make_thresholds(int lattice, double T, double h, Thresholds* out);
// #{u : uniform(u) < b} for any float b (2^32 when b > 1)
uint64_t threshold64_of(float b);
// The split tables (src/gpu_2d.cu:133-139, src/gpu_3d.cu:57-63): the bond
// part for n satisfied of z bonds costs 2(2n - z) (border sites 2(2n - 5)),
// accepted always when that is <= 0, else with float(exp(-2 j / T)); the
// field part float(exp(-2 h / T)), not clamped to 1.
bool make_split_thresholds(int lattice, double T, double h, SplitThresholds* out);
// Tables for the mt19937_64 stream (see ThresholdsMT).
bool make_thresholds_mt(int lattice, double T, double h, ThresholdsMT* out);
// The reference CPU classes' uniform: u(g) for a 64-bit generator output.
double uniform_from_u64(uint64_t g);
// mt19937_64 seeding (state words then index kMtN: the next output twists).
void mt64_seed(uint64_t seed, uint64_t* state313);

// Exchange decision of src/parallel_tempering.hpp:141-162 for one replica:
// accept iff (dE*dB > 0) || r < exp(dB*dE), dE = -(E_i - E_{i+1}) as float.
bool pt_accept(float dE, double dB, double r);
// For h = 0 every dE is an integer in [-span, span]; the accepted set is an
// interval [lo, hi] (possibly empty: lo > hi). Computed with the exact host
// expression above at the boundary points.
void pt_accept_interval(double dB, double r, int64_t span, int64_t* lo, int64_t* hi);

inline int lattice_dim(int lattice) { return lattice == 2 ? 3 : 2; }

}  // namespace sa
