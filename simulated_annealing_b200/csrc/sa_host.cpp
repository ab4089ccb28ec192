// sa_host.cpp -- host helpers: error state, Boltzmann tables, thresholds and
// the exchange-decision intervals. Compiled with -ffp-contract=off so every
// expression rounds exactly like the reference's host code.
#include "sa_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>

#include "sa_b200.h"

namespace sa {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char* what) {
  char buf[512];
  snprintf(buf, sizeof buf, "CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
  g_last_error = buf;
  return SA_ERR_CUDA;
}

void boltz_table(int lattice, double T, double h, double* b) {
  for (int i = 0; i < 20; ++i) b[i] = 0.0;
  if (lattice == SA_LATTICE_3D) {
    for (size_t i = 0; i < 7; i++) {
      int j = ((int)i - 3) * 2;
      b[i] = std::min(1., exp(-2 * (1 / T) * (j - h)));
      b[7 + i] = std::min(1., exp(-2 * (1 / T) * (j + h)));
    }
  } else {
    for (size_t i = 0; i < 5; i++) {
      int j = ((int)i - 2) * 2;
      b[i] = std::min(1., exp(-2 * (1 / T) * (j - h)));
      b[5 + i] = std::min(1., exp(-2 * (1 / T) * (j + h)));
      b[10 + i] = std::min(1., (i == 0) ? 0. : exp(-2 * (1 / T) * (j - 1 - h)));
      b[15 + i] = std::min(1., (i == 0) ? 0. : exp(-2 * (1 / T) * (j - 1 + h)));
    }
  }
}

float uniform_from_u32(uint32_t u) {
  volatile float fu = (float)u;
  volatile float scaled = fu * 0x1p-32f;
  return scaled + 0x1p-33f;
}

uint32_t threshold_of(float b) {
  uint64_t lo = 0, hi = 1ULL << 32;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (uniform_from_u32((uint32_t)mid) < b) lo = mid + 1; else hi = mid;
  }
  // b <= 1.0 always (min(1, .)), and uniform(2^32-1) == 1.0, so lo < 2^32.
  return lo >= (1ULL << 32) ? 0xFFFFFFFFu : (uint32_t)lo;
}

uint64_t threshold64_of(float b) {
  uint64_t lo = 0, hi = 1ULL << 32;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (uniform_from_u32((uint32_t)mid) < b) lo = mid + 1; else hi = mid;
  }
  return lo;  // 2^32 when every u passes (b > 1)
}

bool make_split_thresholds(int lattice, double T, double h, SplitThresholds* t) {
  if (!(T > 0)) return false;
  memset(t, 0, sizeof *t);
  const int z = (lattice == SA_LATTICE_3D) ? 6 : 4;
  // the reference's table entries: float(exp(-2.*j*(1./T))) for j = 2n - z
  auto entry = [&](int j) -> uint64_t {
    if (j <= 0) return 1ULL << 32;  // the reference accepts these without a draw
    return threshold64_of((float)std::exp(-2. * j * (1. / T)));
  };
  for (int n = 0; n <= z; ++n) t->bond[n] = entry(2 * n - z);
  if (lattice != SA_LATTICE_3D)
    for (int n = 0; n <= 4; ++n) t->bbond[n] = entry(2 * n - 5);  // the forced bond counts in n
  t->field = threshold64_of((float)std::exp(-2. * h / T));
  return true;
}

bool make_thresholds(int lattice, double T, double h, Thresholds* t) {
  double b[20];
  boltz_table(lattice, T, h, b);
  memset(t, 0, sizeof *t);
  int nb = (lattice == SA_LATTICE_3D) ? 6 : 4;
  int up0 = nb + 1;
  for (int k = 0; k <= nb; ++k) {
    t->dn[k] = threshold_of((float)b[k]);
    t->up[k] = threshold_of((float)b[up0 + k]);
  }
  if (lattice != SA_LATTICE_3D) {
    for (int k = 0; k <= 4; ++k) {
      t->bdn[k] = threshold_of((float)b[10 + k]);
      t->bup[k] = threshold_of((float)b[15 + k]);
    }
    // A border site always has its forced bond satisfied, so k >= 1 and the
    // k = 0 entry (0 in the reference) is never consulted; copying k = 1
    // keeps the prefix property the kernels rely on.
    t->bdn[0] = t->bdn[1];
    t->bup[0] = t->bup[1];
  }
  for (int k = 1; k <= nb; ++k)
    if (t->dn[k] > t->dn[k - 1] || t->up[k] > t->up[k - 1]) return false;
  if (lattice != SA_LATTICE_3D)
    for (int k = 1; k <= 4; ++k)
      if (t->bdn[k] > t->bdn[k - 1] || t->bup[k] > t->bup[k - 1]) return false;
  return true;
}

double uniform_from_u64(uint64_t g) {
  // generate_canonical<double, 53> with a 64-bit engine: one draw scaled by
  // 2^-64; a result that rounds up to 1 is replaced by the largest double < 1
  volatile double d = (double)g;
  volatile double r = d * 0x1p-64;
  return r >= 1.0 ? 0x1.fffffffffffffp-1 : r;
}

// Largest g with u(g) < b (b > 0; u(0) = 0 < b).
static uint64_t threshold_mt(double b) {
  // smallest g in [0, 2^64] with u(g) >= b, by bisection on 128-bit bounds
  unsigned __int128 lo = 0, hi = (unsigned __int128)1 << 64;
  while (lo < hi) {
    const unsigned __int128 mid = (lo + hi) >> 1;
    if (uniform_from_u64((uint64_t)mid) < b) lo = mid + 1;
    else hi = mid;
  }
  return (uint64_t)(lo - 1);  // lo >= 1 since u(0) = 0 < b
}

bool make_thresholds_mt(int lattice, double T, double h, ThresholdsMT* t) {
  double b[20];
  boltz_table(lattice, T, h, b);
  memset(t, 0, sizeof *t);
  const int nb = (lattice == SA_LATTICE_3D) ? 6 : 4;
  const int up0 = nb + 1;
  // entries accepting something (b > 0) must form a prefix of each table
  auto fill = [&](const double* bt, int n, uint64_t* thr, int* nvalid) {
    *nvalid = 0;
    for (int k = 0; k < n; ++k) {
      if (bt[k] > 0) {
        if (*nvalid != k) return false;
        thr[k] = threshold_mt(bt[k]);
        *nvalid = k + 1;
      }
    }
    return true;
  };
  if (!fill(b, nb + 1, t->dn, &t->ndn) || !fill(b + up0, nb + 1, t->up, &t->nup)) return false;
  if (lattice != SA_LATTICE_3D) {
    // entry 0 of the border tables (0 in the reference) is never consulted: a
    // border site's forced bond is satisfied; entry 1 stands in for it
    double bb[5], bu[5];
    for (int k = 0; k <= 4; ++k) {
      bb[k] = b[10 + (k == 0 ? 1 : k)];
      bu[k] = b[15 + (k == 0 ? 1 : k)];
    }
    if (!fill(bb, 5, t->bdn, &t->nbdn) || !fill(bu, 5, t->bup, &t->nbup)) return false;
  }
  for (int k = 1; k < t->ndn; ++k)
    if (t->dn[k] > t->dn[k - 1]) return false;
  for (int k = 1; k < t->nup; ++k)
    if (t->up[k] > t->up[k - 1]) return false;
  for (int k = 1; k < t->nbdn; ++k)
    if (t->bdn[k] > t->bdn[k - 1]) return false;
  for (int k = 1; k < t->nbup; ++k)
    if (t->bup[k] > t->bup[k - 1]) return false;
  return true;
}

void mt64_seed(uint64_t seed, uint64_t* st) {
  st[0] = seed;
  for (int i = 1; i < kMtN; ++i) st[i] = 6364136223846793005ULL * (st[i - 1] ^ (st[i - 1] >> 62)) + (uint64_t)i;
  st[kMtN] = kMtN;
}

bool pt_accept(float dE, double dB, double r) {
  return ((dE * dB) > 0.) || r < exp(dB * dE);
}

void pt_accept_interval(double dB, double r, int64_t span, int64_t* lo, int64_t* hi) {
  auto acc = [&](int64_t x) { return pt_accept((float)x, dB, r); };
  if (!(dB > 0) && !(dB < 0)) {  // dB == 0: exp(0) = 1 > r, every dE accepted
    *lo = -span;
    *hi = span;
    return;
  }
  if (dB > 0) {
    // accepted set is [D, span]; acc(0) holds because r < 1 = exp(0).
    int64_t a = -span, b = 0;  // smallest accepted in [a, b]
    if (acc(a)) { *lo = a; *hi = span; return; }
    while (b - a > 1) {
      int64_t m = a + (b - a) / 2;
      if (acc(m)) b = m; else a = m;
    }
    *lo = b;
    *hi = span;
  } else {
    int64_t a = 0, b = span;  // largest accepted in [a, b]
    if (acc(b)) { *lo = -span; *hi = b; return; }
    while (b - a > 1) {
      int64_t m = a + (b - a) / 2;
      if (acc(m)) a = m; else b = m;
    }
    *lo = -span;
    *hi = a;
  }
}

}  // namespace sa

extern "C" const char* sa_last_error(void) { return sa::g_last_error.c_str(); }

// The exchange sequence of parallel_tempering<> (src/parallel_tempering.hpp:
// 28-30, :59, :112-114): std::mt19937 gen(123); per step i = uni_int(gen) from
// uniform_int_distribution<int>(0, n-2), then r = uni_double(gen) from
// uniform_real_distribution<double>(0, 1) -- libstdc++'s own generators.
extern "C" int sa_pt_sequence(int n, long skip, long count, int32_t* pair, double* r) {
  if (n < 2 || skip < 0 || count < 0 || (count > 0 && (!pair || !r)))
    return sa::fail(SA_ERR_INVALID, "bad arguments to sa_pt_sequence");
  std::mt19937 gen(123);
  std::uniform_int_distribution<int> uni_int(0, n - 2);
  std::uniform_real_distribution<double> uni_double(0., 1.);
  for (long k = 0; k < skip + count; ++k) {
    const int i = uni_int(gen);
    const double u = uni_double(gen);
    if (k >= skip) {
      pair[k - skip] = i;
      r[k - skip] = u;
    }
  }
  return SA_OK;
}

// The exchange generator as an object (the template's gen / uni_int /
// uni_double members). Its checkpoint bytes are the raw objects, as the
// template's save() writes them: libstdc++'s std::mt19937 (624 state words
// of uint_fast32_t and the position), then the two distributions' parameters.
struct sa_pt_gen {
  std::mt19937 gen{123};
  std::uniform_int_distribution<int> uni_int;
  std::uniform_real_distribution<double> uni_double{0., 1.};
  explicit sa_pt_gen(int n) : uni_int(0, n - 2) {}
};

extern "C" int sa_pt_gen_create(int n, sa_pt_gen_t* out) {
  if (n < 2 || !out) return sa::fail(SA_ERR_INVALID, "sa_pt_gen_create: need n >= 2 and an output");
  *out = new sa_pt_gen(n);
  return SA_OK;
}

extern "C" int sa_pt_gen_destroy(sa_pt_gen_t g) {
  delete g;
  return SA_OK;
}

extern "C" int sa_pt_gen_next(sa_pt_gen_t g, long count, int32_t* pair, double* r) {
  if (!g || count < 0 || (count > 0 && (!pair || !r))) return sa::fail(SA_ERR_INVALID, "bad arguments to sa_pt_gen_next");
  for (long k = 0; k < count; ++k) {
    pair[k] = g->uni_int(g->gen);
    r[k] = g->uni_double(g->gen);
  }
  return SA_OK;
}

extern "C" int sa_pt_gen_widen(sa_pt_gen_t g) {
  if (!g) return sa::fail(SA_ERR_INVALID, "null generator");
  g->uni_int = std::uniform_int_distribution<int>(g->uni_int.a(), g->uni_int.b() + 1);
  return SA_OK;
}

static constexpr size_t kPtGenBytes =
    sizeof(std::mt19937) + sizeof(std::uniform_int_distribution<int>) + sizeof(std::uniform_real_distribution<double>);

extern "C" int sa_pt_gen_save(sa_pt_gen_t g, void* buf, size_t cap, size_t* len) {
  if (!g || !len) return sa::fail(SA_ERR_INVALID, "null argument");
  *len = kPtGenBytes;
  if (!buf) return SA_OK;
  if (cap < kPtGenBytes) return sa::fail(SA_ERR_BUFFER, "buffer too small");
  char* p = (char*)buf;
  memcpy(p, &g->gen, sizeof g->gen);
  memcpy(p + sizeof g->gen, &g->uni_int, sizeof g->uni_int);
  memcpy(p + sizeof g->gen + sizeof g->uni_int, &g->uni_double, sizeof g->uni_double);
  return SA_OK;
}

extern "C" int sa_pt_gen_load(sa_pt_gen_t g, const void* buf, size_t len) {
  if (!g || !buf) return sa::fail(SA_ERR_INVALID, "null argument");
  if (len != kPtGenBytes) return sa::fail(SA_ERR_MISMATCH, "generator record has the wrong size");
  const char* p = (const char*)buf;
  memcpy(&g->gen, p, sizeof g->gen);
  memcpy(&g->uni_int, p + sizeof g->gen, sizeof g->uni_int);
  memcpy(&g->uni_double, p + sizeof g->gen + sizeof g->uni_int, sizeof g->uni_double);
  return SA_OK;
}

// The reference's per-replica exchange test (src/parallel_tempering.hpp:
// 141-162) for one pair: mask bit j set iff dE*dB > 0 || r < exp(dB*dE) with
// dE = -(Ei[j] - Ej[j]) as float and dB = 1/Ti - 1/Tj.
extern "C" uint64_t sa_pt_mask(const float* Ei, const float* Ej, double Ti, double Tj, double r) {
  const double dB = (1. / Ti - 1. / Tj);
  uint64_t mask = 0;
  for (int j = 0; j < 64; ++j) {
    const float dE = -(Ei[j] - Ej[j]);
    if (sa::pt_accept(dE, dB, r)) mask |= 1ULL << j;
  }
  return mask;
}
