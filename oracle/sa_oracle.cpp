// sa_oracle.cpp -- CPU ORACLE for the multispin-coded Metropolis path.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product (the CUDA library, the
// C++ shim, the Python package) links, imports or executes this file; only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may use it,
// and only as the checker.
//
// What it restates (reference paths are relative to the reference project):
//   * lattice bit logic      src/cpu_2d.cpp:5-41 (2D periodic),
//                            src/cpu_2dp.cpp:336-383 (2D open in x),
//                            src/cpu_3d.cpp:107-161 (3D periodic)
//   * sweep order            src/cpu_2dp.cpp:106-114, src/cpu_3d.cpp:94-105
//                            (colour (x+y)%2 in BOTH 2D and 3D; in 3D the z
//                            neighbours share a colour, so each half-sweep is
//                            sequential along z inside every (x,y) column)
//   * Boltzmann tables       src/cpu_2dp.cpp:33-40, src/cpu_3d.cpp:218-232
//   * measure (-H)           src/cpu_2d.cpp:67-94, src/cpu_2dp.cpp:196-214,
//                            src/cpu_3d.cpp:333-371
//   * J layout / generation  src/cpu_2dp.cpp:243-260, src/cpu_3d.cpp:281-301,
//                            GPU word assembly src/device_2d.cu:130-138,
//                            src/device_3d.cu:98-125, src/device.cuh:4-8
//   * draw schedule          src/random.cu:15-35, src/device_2d.cu:96-97
//   * swap                   src/tools_inline.hpp:4-9
//   * PT step / creat_mask   src/parallel_tempering.hpp:81-115, 141-162
//   * annealing step         src/annealing.hpp:67-100
//
// Two random-number modes drive the same lattice code:
//   PHILOX  the GPU reference's schedule: site i uses Philox4x32-10 stream
//           (key = seed, subsequence = i); the u32 draw at index n is
//           converted to a float in (0,1] and compared (as float) against the
//           float-cast Boltzmann table, like src/gpu_2d.cu:52-61 +
//           src/device_2d.cu:96-97. Philox4x32-10 is written from Salmon,
//           Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3"
//           (SC'11). Pinned against tests/golden/curand_philox_golden.json.
//   MT      the CPU reference's own generator (std::mt19937_64 +
//           std::uniform_real_distribution<double>, called from libstdc++),
//           double compare against the double table. In this mode the
//           restatement is pinned bit for bit against the reference's own CPU
//           classes compiled from their sources (oracle/_ref).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <random>
#include <vector>

typedef uint64_t word_t;

enum { LAT_2D_PERIODIC = 0, LAT_2D_OPEN_X = 1, LAT_3D_PERIODIC = 2 };
enum { MODE_PHILOX = 0, MODE_MT = 1 };

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al. 2011): 10 rounds of two 32x32->64 multiplies,
// key bumped by the golden-ratio / sqrt(3)-1 Weyl constants between rounds.
// ---------------------------------------------------------------------------
static const uint32_t PHILOX_M0 = 0xD2511F53u, PHILOX_M1 = 0xCD9E8D57u;
static const uint32_t PHILOX_W0 = 0x9E3779B9u, PHILOX_W1 = 0xBB67AE85u;

static inline void philox_block(const uint32_t in[4], const uint32_t key_in[2],
                                uint32_t out[4]) {
  uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
    uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += PHILOX_W0;
    k1 += PHILOX_W1;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Draw number `index` of stream (seed, subsequence): the counter holds the
// block number (index/4) in its low 64 bits and the subsequence in its high
// 64 bits, the key is the 64-bit seed; the draw is lane index%4 of the block.
static inline uint32_t philox_draw(uint64_t seed, uint64_t subseq, uint64_t index) {
  uint64_t blk = index >> 2;
  uint32_t ctr[4] = {(uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)subseq,
                     (uint32_t)(subseq >> 32)};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t out[4];
  philox_block(ctr, key, out);
  return out[index & 3];
}

// u32 -> float in (0,1]: the midpoint of bucket u of width 2^-32, evaluated in
// binary32 (u rounded to float, scaled by 2^-32 exactly, plus 2^-33 rounded).
// Built with -ffp-contract=off so the two roundings stay separate.
static inline float uniform_from_u32(uint32_t u) {
  volatile float fu = (float)u;
  volatile float scaled = fu * 0x1p-32f;
  return scaled + 0x1p-33f;
}

// Number of u32 values whose uniform is strictly below b. Because the map is
// non-decreasing, "uniform(u) < b" is exactly "u < threshold(b)".
static uint64_t threshold_of(float b) {
  uint64_t lo = 0, hi = 1ULL << 32;  // answer in [lo, hi]
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (uniform_from_u32((uint32_t)mid) < b) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// Boltzmann tables, same expressions and evaluation order as the reference.
// 2D: [0,5) spin down, [5,10) spin up, [10,20) the x-border variants.
// 3D: [0,7) spin down, [7,14) spin up.
// ---------------------------------------------------------------------------
static void boltz_table(int lattice, double T, double h, double* b) {
  if (lattice == LAT_3D_PERIODIC) {
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

// ---------------------------------------------------------------------------
// One oracle system (64 replicas), reference-layout J arrays Jx/Jy/Jz[2N]:
// J?[2i] is the bond to the -x/-y/-z neighbour, J?[2i+1] the bond to the
// +x/+y/+z neighbour (a copy of that neighbour's own word).
// ---------------------------------------------------------------------------
struct OSys {
  int lattice, L, dim;
  long N, L2;
  double T, h;
  std::vector<word_t> s, Jx, Jy, Jz;
  int mode;
  // PHILOX state: key, next draw index shared by all sites, spin-init epoch
  uint64_t seed, draw, epoch;
  int first = 0;  // colour of the first half-sweep of a sweep
  int split = 0;  // the reference's SPLIT_H update (PHILOX mode)
  // MT state
  std::mt19937_64 gen;
  std::uniform_real_distribution<double> uni;
  double bd[20];
  float bf[20];
  OSys() : uni(0., 1.) {}
  void tables() {
    boltz_table(lattice, T, h, bd);
    for (int i = 0; i < 20; ++i) bf[i] = (float)bd[i];
  }
};

static inline long nb_w(const OSys& o, long i) { return (i % o.L == 0) ? i + o.L - 1 : i - 1; }
static inline long nb_e(const OSys& o, long i) { return ((i + 1) % o.L == 0) ? i - o.L + 1 : i + 1; }
static inline long nb_n(const OSys& o, long i) {
  return (i % o.L2 < o.L) ? i + o.L2 - o.L : i - o.L;
}
static inline long nb_s(const OSys& o, long i) {
  return ((i + o.L) % o.L2 < o.L) ? i - o.L2 + o.L : i + o.L;
}
static inline long nb_u(const OSys& o, long i) { return (i - o.L2 < 0) ? i + o.N - o.L2 : i - o.L2; }
static inline long nb_d(const OSys& o, long i) { return (i + o.L2 >= o.N) ? i - o.N + o.L2 : i + o.L2; }

// Bit-sliced count of set bits over `n` masks, then per-value equality masks.
static void count_eq(const word_t* m, int n, word_t eq[7]) {
  word_t c0 = 0, c1 = 0, c2 = 0;
  for (int k = 0; k < n; ++k) {
    word_t a = m[k];
    word_t t0 = c0 & a;
    c0 ^= a;
    word_t t1 = c1 & t0;
    c1 ^= t0;
    c2 ^= t1;
  }
  for (int v = 0; v <= 6; ++v) {
    word_t e = ~(word_t)0;
    e &= (v & 1) ? c0 : ~c0;
    e &= (v & 2) ? c1 : ~c1;
    e &= (v & 4) ? c2 : ~c2;
    eq[v] = e;
  }
}

// Acceptance of a single random number against table entries; `use_float`
// selects the GPU (float) or CPU (double) comparison.
struct Draw {
  bool use_float;
  float rf;
  double rd;
  bool lt(const OSys& o, int idx) const {
    return use_float ? (rf < o.bf[idx]) : (rd < o.bd[idx]);
  }
};

static void update_site(OSys& o, long i, const Draw& r) {
  word_t si = o.s[i];
  word_t m[6];
  int nb = 0, down0 = 0, up0 = 0;
  if (o.lattice == LAT_3D_PERIODIC) {
    m[0] = o.Jx[2 * i] ^ si ^ o.s[nb_w(o, i)];
    m[1] = o.Jx[2 * i + 1] ^ si ^ o.s[nb_e(o, i)];
    m[2] = o.Jy[2 * i] ^ si ^ o.s[nb_n(o, i)];
    m[3] = o.Jy[2 * i + 1] ^ si ^ o.s[nb_s(o, i)];
    m[4] = o.Jz[2 * i] ^ si ^ o.s[nb_u(o, i)];
    m[5] = o.Jz[2 * i + 1] ^ si ^ o.s[nb_d(o, i)];
    nb = 6; down0 = 0; up0 = 7;
  } else {
    bool xb_lo = (i % o.L == 0), xb_hi = ((i + 1) % o.L == 0);
    bool open = (o.lattice == LAT_2D_OPEN_X);
    m[0] = (open && xb_lo) ? ~(word_t)0 : (o.Jx[2 * i] ^ o.s[nb_w(o, i)] ^ si);
    m[1] = (open && xb_hi) ? ~(word_t)0 : (o.Jx[2 * i + 1] ^ o.s[nb_e(o, i)] ^ si);
    m[2] = o.Jy[2 * i] ^ o.s[nb_n(o, i)] ^ si;
    m[3] = o.Jy[2 * i + 1] ^ o.s[nb_s(o, i)] ^ si;
    nb = 4;
    if (open && (xb_lo || xb_hi)) { down0 = 10; up0 = 15; } else { down0 = 0; up0 = 5; }
  }
  word_t eq[7];
  count_eq(m, nb, eq);
  word_t flip = 0;
  for (int k = 0; k <= nb; ++k) {
    word_t a_dn = r.lt(o, down0 + k) ? ~(word_t)0 : 0;
    word_t a_up = r.lt(o, up0 + k) ? ~(word_t)0 : 0;
    flip |= eq[k] & ((a_dn & ~si) | (a_up & si));
  }
  o.s[i] = si ^ flip;
}

// The SPLIT_H update restated from the reference's GPU kernels
// (src/device_2d.cu:27-50 with the boundary handling of :114-125,
// src/device_3d.cu:216-245 with :76-89) and tables (src/gpu_2d.cu:133-139,
// src/gpu_3d.cu:57-63): "exactly k satisfied" masks eq[k]; the bond part of
// eq[z] / eq[z-1] (and eq[z-2] in 3D) is accepted iff rand1 < the float entry
// exp(-2 j / T), j = 2k - z (open-x border sites, whose forced bond is in k:
// j = 2k - 5), every smaller k always; an up spin's field part iff
// rand2 < float(exp(-2 h / T)). 3D sites on the boundary use rand2 for both.
static void update_site_split(OSys& o, long i, float r1, float r2) {
  word_t si = o.s[i];
  word_t m[6];
  int nb = 0;
  bool border = false;
  if (o.lattice == LAT_3D_PERIODIC) {
    m[0] = o.Jx[2 * i] ^ si ^ o.s[nb_w(o, i)];
    m[1] = o.Jx[2 * i + 1] ^ si ^ o.s[nb_e(o, i)];
    m[2] = o.Jy[2 * i] ^ si ^ o.s[nb_n(o, i)];
    m[3] = o.Jy[2 * i + 1] ^ si ^ o.s[nb_s(o, i)];
    m[4] = o.Jz[2 * i] ^ si ^ o.s[nb_u(o, i)];
    m[5] = o.Jz[2 * i + 1] ^ si ^ o.s[nb_d(o, i)];
    nb = 6;
    const long x = i % o.L, y = (i / o.L) % o.L, z = i / o.L2;
    if (x == 0 || y == 0 || z == 0 || x == o.L - 1 || y == o.L - 1 || z == o.L - 1) r1 = r2;
  } else {
    bool xb_lo = (i % o.L == 0), xb_hi = ((i + 1) % o.L == 0);
    bool open = (o.lattice == LAT_2D_OPEN_X);
    m[0] = (open && xb_lo) ? ~(word_t)0 : (o.Jx[2 * i] ^ o.s[nb_w(o, i)] ^ si);
    m[1] = (open && xb_hi) ? ~(word_t)0 : (o.Jx[2 * i + 1] ^ o.s[nb_e(o, i)] ^ si);
    m[2] = o.Jy[2 * i] ^ o.s[nb_n(o, i)] ^ si;
    m[3] = o.Jy[2 * i + 1] ^ o.s[nb_s(o, i)] ^ si;
    nb = 4;
    border = open && (xb_lo || xb_hi);
  }
  word_t eq[7];
  count_eq(m, nb, eq);
  word_t bond_ok = 0;
  for (int k = 0; k <= nb; ++k) {
    const int j = border ? 2 * k - 5 : 2 * k - nb;
    const bool acc = (j <= 0) || (r1 < (float)std::exp(-2. * j * (1. / o.T)));
    if (acc) bond_ok |= eq[k];
  }
  const word_t dh = (r2 < (float)std::exp(-2. * o.h / o.T)) ? ~(word_t)0 : 0;
  o.s[i] = si ^ (bond_ok & (~si | dh));
}

static void sweep_once(OSys& o) {
  for (int pass = 0; pass < 2; ++pass) {
    const int offset = pass ^ o.first;  // the colour of this half-sweep
    int zmax = (o.dim == 3) ? o.L : 1;
    for (int z = 0; z < zmax; ++z)
      for (int y = 0; y < o.L; ++y)
        for (int x = (y + offset) % 2; x < o.L; x += 2) {
          long i = (long)z * o.L2 + (long)y * o.L + x;
          if (o.split) {
            const float r1 = uniform_from_u32(philox_draw(o.seed, (uint64_t)i, o.draw + 2 * pass));
            const float r2 = uniform_from_u32(philox_draw(o.seed, (uint64_t)i, o.draw + 2 * pass + 1));
            update_site_split(o, i, r1, r2);
            continue;
          }
          Draw r;
          if (o.mode == MODE_PHILOX) {
            r.use_float = true;
            r.rf = uniform_from_u32(philox_draw(o.seed, (uint64_t)i, o.draw + pass));
            r.rd = 0;
          } else {
            r.use_float = false;
            r.rd = o.uni(o.gen);
            r.rf = 0;
          }
          update_site(o, i, r);
        }
  }
  if (o.mode == MODE_PHILOX) o.draw += o.split ? 4 : 2;
}

// Own bond words (compact, d per site) -> reference layout.
static void own_to_ref(OSys& o, const std::vector<word_t>& ox, const std::vector<word_t>& oy,
                       const std::vector<word_t>& oz) {
  for (long i = 0; i < o.N; ++i) {
    o.Jx[2 * i] = ox[i];
    o.Jx[2 * i + 1] = ox[nb_e(o, i)];
    o.Jy[2 * i] = oy[i];
    o.Jy[2 * i + 1] = oy[nb_s(o, i)];
    if (o.dim == 3) {
      o.Jz[2 * i] = oz[i];
      o.Jz[2 * i + 1] = oz[nb_d(o, i)];
    }
  }
}

extern "C" {

// ----- RNG primitives --------------------------------------------------------
void sao_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  philox_block(ctr, key, out);
}
uint32_t sao_philox_draw(uint64_t seed, uint64_t subseq, uint64_t index) {
  return philox_draw(seed, subseq, index);
}
float sao_uniform_from_u32(uint32_t u) { return uniform_from_u32(u); }

// Draws 0..ndraws-1 of subsequences 0..nsubs-1 of key `seed` and the bit
// patterns of their uniforms, laid out [subsequence][draw] (the layout of
// tests/golden/gen_curand_golden.cu --bulk).
void sao_philox_bulk(uint64_t seed, long nsubs, long ndraws, uint32_t* u32_out, uint32_t* uni_out) {
  for (long s = 0; s < nsubs; ++s)
    for (long k = 0; k < ndraws; ++k) {
      const uint32_t u = philox_draw(seed, (uint64_t)s, (uint64_t)k);
      const float f = uniform_from_u32(u);
      uint32_t bits;
      memcpy(&bits, &f, 4);
      u32_out[s * ndraws + k] = u;
      uni_out[s * ndraws + k] = bits;
    }
}
uint64_t sao_threshold(float b) { return threshold_of(b); }

// Exhaustive: uniform_from_u32 is non-decreasing over all 2^32 inputs, lies in
// (0,1], and reaches 1.0. Returns 0 on success.
int sao_check_uniform_monotone(void) {
  float prev = 0.0f;
  for (uint64_t u = 0; u < (1ULL << 32); ++u) {
    float f = uniform_from_u32((uint32_t)u);
    if (!(f > 0.0f) || f > 1.0f) return 1;
    if (f < prev) return 2;
    prev = f;
  }
  return prev == 1.0f ? 0 : 3;
}

void sao_boltz_table(int lattice, double T, double h, double* out20) {
  for (int i = 0; i < 20; ++i) out20[i] = 0;
  boltz_table(lattice, T, h, out20);
}

// ----- systems -----------------------------------------------------------------
void* sao_sys_new(int lattice, int L, double T, double h, int mode) {
  if (lattice < 0 || lattice > 2 || L < 2 || (L & 1) || mode < 0 || mode > 1) return nullptr;
  OSys* o = new OSys();
  o->lattice = lattice;
  o->L = L;
  o->dim = (lattice == LAT_3D_PERIODIC) ? 3 : 2;
  o->L2 = (long)L * L;
  o->N = (o->dim == 3) ? o->L2 * L : o->L2;
  o->T = T;
  o->h = h;
  o->mode = mode;
  o->s.assign(o->N, 0);
  o->Jx.assign(2 * o->N, 0);
  o->Jy.assign(2 * o->N, 0);
  if (o->dim == 3) o->Jz.assign(2 * o->N, 0);
  o->seed = 1234;  // the reference constructors seed with 1234
  o->draw = 0;
  o->epoch = 0;
  o->gen.seed(1234);
  o->tables();
  return o;
}
void sao_sys_free(void* p) { delete (OSys*)p; }
long sao_sys_N(void* p) { return ((OSys*)p)->N; }

void sao_sys_set_seed(void* p, uint64_t seed) {
  OSys* o = (OSys*)p;
  if (o->mode == MODE_PHILOX) { o->seed = seed; o->draw = 0; o->epoch = 0; }
  else o->gen.seed(seed);
}
void sao_sys_set_T(void* p, double T) { OSys* o = (OSys*)p; o->T = T; o->tables(); }
void sao_sys_set_h(void* p, double h) { OSys* o = (OSys*)p; o->h = h; o->tables(); }
double sao_sys_get_T(void* p) { return ((OSys*)p)->T; }
uint64_t sao_sys_get_draw(void* p) { return ((OSys*)p)->draw; }
void sao_sys_set_draw(void* p, uint64_t d) { ((OSys*)p)->draw = d; }
// colour of each sweep's first half-sweep (PHILOX mode): 1 is the second
// configuration of the reference GPU systems' two-lattice pair
void sao_sys_set_first_colour(void* p, int c) { ((OSys*)p)->first = c ? 1 : 0; }
// the reference's SPLIT_H update (PHILOX mode)
void sao_sys_set_split(void* p, int on) { ((OSys*)p)->split = on ? 1 : 0; }

void sao_sys_init_J(void* p) {
  OSys* o = (OSys*)p;
  std::vector<word_t> ox(o->N), oy(o->N), oz(o->dim == 3 ? o->N : 0);
  if (o->mode == MODE_PHILOX) {
    // src/random.cu:25-35 + src/device_2d.cu:130-138 / src/device_3d.cu:98-125:
    // t = 2*dim u32 draws per site; own word k = draw[2k] | draw[2k+1] << 32.
    for (long i = 0; i < o->N; ++i) {
      uint32_t d[6];
      for (int k = 0; k < 2 * o->dim; ++k) d[k] = philox_draw(o->seed, (uint64_t)i, o->draw + k);
      ox[i] = (word_t)d[0] | ((word_t)d[1] << 32);
      oy[i] = (word_t)d[2] | ((word_t)d[3] << 32);
      if (o->dim == 3) oz[i] = (word_t)d[4] | ((word_t)d[5] << 32);
    }
    o->draw += 2 * o->dim;
  } else {
    // src/cpu_2dp.cpp:243-260, src/cpu_3d.cpp:281-301: one gen() per own word,
    // site-major.
    for (long i = 0; i < o->N; ++i) {
      ox[i] = o->gen();
      oy[i] = o->gen();
      if (o->dim == 3) oz[i] = o->gen();
    }
  }
  own_to_ref(*o, ox, oy, oz);
}

// Initial spins. MT: s[i] = gen() (src/cpu_2dp.cpp:286-290). PHILOX: the
// engine's counter-based init: block (epoch, 0, i, 2^31 | i>>32) of key seed,
// word = lane0 | lane1 << 32; each call advances the epoch.
void sao_sys_init_rand(void* p) {
  OSys* o = (OSys*)p;
  if (o->mode == MODE_PHILOX) {
    uint32_t key[2] = {(uint32_t)o->seed, (uint32_t)(o->seed >> 32)};
    for (long i = 0; i < o->N; ++i) {
      uint32_t ctr[4] = {(uint32_t)o->epoch, (uint32_t)(o->epoch >> 32), (uint32_t)i,
                         (o->first ? 0xC0000000u : 0x80000000u) | (uint32_t)((uint64_t)i >> 32)};
      uint32_t out[4];
      philox_block(ctr, key, out);
      o->s[i] = (word_t)out[0] | ((word_t)out[1] << 32);
    }
    o->epoch += 1;
  } else {
    for (long i = 0; i < o->N; ++i) o->s[i] = o->gen();
  }
}
void sao_sys_init_order(void* p) {
  OSys* o = (OSys*)p;
  for (long i = 0; i < o->N; ++i) o->s[i] = ~(word_t)0;
}

void sao_sys_sweep(void* p, long n) {
  OSys* o = (OSys*)p;
  for (long k = 0; k < n; ++k) sweep_once(*o);
}

// Exact integer parts of -H per replica bit j: E = sum over bonds (sat ? 1 : -1),
// M = sum over sites (up ? 1 : -1). For the open-x lattice only real bonds count.
void sao_sys_measure(void* p, int64_t* E, int64_t* M) {
  OSys* o = (OSys*)p;
  for (int j = 0; j < 64; ++j) { E[j] = 0; M[j] = 0; }
  int64_t nbonds = 0;
  for (long i = 0; i < o->N; ++i) {
    word_t si = o->s[i];
    word_t b[3];
    int nb = 0;
    bool open_skip = (o->lattice == LAT_2D_OPEN_X) && (i % o->L == 0);
    if (!open_skip) b[nb++] = o->Jx[2 * i] ^ si ^ o->s[nb_w(*o, i)];
    b[nb++] = o->Jy[2 * i] ^ si ^ o->s[nb_n(*o, i)];
    if (o->dim == 3) b[nb++] = o->Jz[2 * i] ^ si ^ o->s[nb_u(*o, i)];
    nbonds += nb;
    for (int j = 0; j < 64; ++j) {
      for (int k = 0; k < nb; ++k) E[j] += (int64_t)((b[k] >> j) & 1);
      M[j] += (int64_t)((si >> j) & 1);
    }
  }
  for (int j = 0; j < 64; ++j) {
    E[j] = 2 * E[j] - nbonds;
    M[j] = 2 * M[j] - o->N;
  }
}

// The reference's float vector, index j = replica bit j: the CPU classes add
// bit_to_double(w, j) -- which tests bit 63-j of w (src/tools_inline.hpp:27-31)
// -- into E[63-j] (src/cpu_2d.cpp:82-84, src/cpu_3d.cpp:346-348), so the two
// reversals cancel.
void sao_sys_measure_float(void* p, float* out64) {
  OSys* o = (OSys*)p;
  int64_t E[64], M[64];
  sao_sys_measure(p, E, M);
  for (int j = 0; j < 64; ++j) out64[j] = (float)((double)E[j] + o->h * (double)M[j]);
}

void sao_sys_get_spins(void* p, word_t* out) { OSys* o = (OSys*)p; memcpy(out, o->s.data(), o->N * 8); }
void sao_sys_set_spins(void* p, const word_t* in) { OSys* o = (OSys*)p; memcpy(o->s.data(), in, o->N * 8); }
void sao_sys_get_J(void* p, word_t* jx, word_t* jy, word_t* jz) {
  OSys* o = (OSys*)p;
  memcpy(jx, o->Jx.data(), 2 * o->N * 8);
  memcpy(jy, o->Jy.data(), 2 * o->N * 8);
  if (o->dim == 3 && jz) memcpy(jz, o->Jz.data(), 2 * o->N * 8);
}
void sao_sys_set_J(void* p, const word_t* jx, const word_t* jy, const word_t* jz) {
  OSys* o = (OSys*)p;
  memcpy(o->Jx.data(), jx, 2 * o->N * 8);
  memcpy(o->Jy.data(), jy, 2 * o->N * 8);
  if (o->dim == 3 && jz) memcpy(o->Jz.data(), jz, 2 * o->N * 8);
}

// src/tools_inline.hpp:4-9 over every word.
void sao_sys_swap(void* pa, void* pb, word_t mask) {
  OSys* a = (OSys*)pa;
  OSys* b = (OSys*)pb;
  if (a->N != b->N) return;
  for (long i = 0; i < a->N; ++i) {
    word_t x = a->s[i], y = b->s[i];
    a->s[i] = x ^ ((x ^ y) & mask);
    b->s[i] = y ^ ((y ^ x) & mask);
  }
}

// ----- parallel tempering (src/parallel_tempering.hpp) --------------------------
struct OPT {
  std::vector<OSys*> sys;
  std::vector<double> T;
  std::vector<std::vector<float>> E;
  std::vector<float> E_min;
  long steps;
  std::mt19937 gen;
  std::uniform_int_distribution<int> uni_int;
  std::uniform_real_distribution<double> uni_double;
  std::vector<double> acc_sum;
  std::vector<long long> acc_n;
  OPT(int n) : gen(123), uni_int(0, n - 2), uni_double(0., 1.) {}
};

void* sao_pt_new(void** sys, const double* T, int n, long steps) {
  if (n < 2) return nullptr;
  OPT* pt = new OPT(n);
  for (int i = 0; i < n; ++i) pt->sys.push_back((OSys*)sys[i]);
  pt->T.assign(T, T + n);
  std::sort(pt->T.begin(), pt->T.end());
  pt->steps = steps;
  pt->E.assign(n, std::vector<float>());
  pt->acc_sum.assign(n - 1, 0.0);
  pt->acc_n.assign(n - 1, 0);
  for (int i = 0; i < n; ++i) sao_sys_set_T(pt->sys[i], pt->T[i]);
  return pt;
}
void sao_pt_free(void* p) { delete (OPT*)p; }

static std::vector<float> measure_vec(OSys* o) {
  std::vector<float> v(64);
  sao_sys_measure_float(o, v.data());
  return v;
}

// One PT step: `steps` sweeps of every slot, measure on the last sweep (and on
// every `stride`-th when stride != 0), then one exchange attempt. Writes the
// chosen pair, the exchange mask and the uniform used.
void sao_pt_step(void* p, int stride, int* pair_out, word_t* mask_out, double* r_out) {
  OPT* pt = (OPT*)p;
  int n = (int)pt->T.size();
  for (long i = 0; i < pt->steps; ++i) {
    for (int j = 0; j < n; ++j) {
      sao_sys_sweep(pt->sys[j], 1);
      if (((stride != 0) && ((i % stride) == 0)) || i == (pt->steps - 1))
        pt->E[j] = measure_vec(pt->sys[j]);
    }
    if (stride == 0) {
      if (pt->E_min.empty()) pt->E_min = pt->E[0];
      for (size_t j = 0; j < pt->E_min.size(); ++j)
        pt->E_min[j] = std::max(pt->E[0][j], pt->E_min[j]);
    }
  }
  int i = pt->uni_int(pt->gen);
  double r = pt->uni_double(pt->gen);
  word_t mask = 0;
  int a = 0;
  double dB = (1. / pt->T[i] - 1. / pt->T[i + 1]);
  for (size_t j = 0; j < pt->E[i].size(); ++j) {
    float dE = -(pt->E[i][j] - pt->E[i + 1][j]);
    if (((dE * dB) > 0.) || r < exp(dB * dE)) {
      mask |= (word_t)1 << (j % 64);
      a++;
    }
  }
  pt->acc_sum[i] += a / (double)64.;
  pt->acc_n[i] += 1;
  sao_sys_swap(pt->sys[i], pt->sys[i + 1], mask);
  if (pair_out) *pair_out = i;
  if (mask_out) *mask_out = mask;
  if (r_out) *r_out = r;
}
void sao_pt_energies(void* p, float* out /* n*64 */) {
  OPT* pt = (OPT*)p;
  for (size_t s = 0; s < pt->E.size(); ++s)
    for (size_t j = 0; j < pt->E[s].size(); ++j) out[s * 64 + j] = pt->E[s][j];
}
void sao_pt_acceptance(void* p, double* out) {
  OPT* pt = (OPT*)p;
  for (size_t i = 0; i < pt->acc_sum.size(); ++i)
    out[i] = pt->acc_n[i] ? pt->acc_sum[i] / (double)pt->acc_n[i] : 0.0;
}
void sao_pt_sorted_T(void* p, double* out) {
  OPT* pt = (OPT*)p;
  for (size_t i = 0; i < pt->T.size(); ++i) out[i] = pt->T[i];
}

// ----- annealing (src/annealing.hpp:67-100) -------------------------------------
// nsteps outer steps of `sweeps` sweeps each; measure on sweeps with i%stride==0;
// running max of the float -H per vector index; after each step T is either
// multiplied by alfa (schedule 0, the reference's geometric cooling) or set to
// the next point of the linear schedule T0 + (T1-T0)*k/(nsteps-1) (schedule 1).
// last_E receives the last measured vector of every step (nsteps*64).
void sao_anneal_run(void* p, double T0, int schedule, double alfa_or_T1, int nsteps,
                    int sweeps, int stride, float* min_E, float* last_E) {
  OSys* o = (OSys*)p;
  double T = T0;
  sao_sys_set_T(p, T);
  std::vector<float> mn;
  std::vector<float> res(64, 0.f);
  for (int k = 0; k < nsteps; ++k) {
    for (int i = 0; i < sweeps; ++i) {
      sao_sys_sweep(p, 1);
      if (stride != 0 && i % stride == 0) {
        res = measure_vec(o);
        if (mn.empty()) mn = res;
        for (int j = 0; j < 64; ++j) mn[j] = std::max(res[j], mn[j]);
      }
    }
    if (last_E) for (int j = 0; j < 64; ++j) last_E[k * 64 + j] = res[j];
    if (schedule == 0) T = T * alfa_or_T1;
    else T = (nsteps > 1) ? T0 + (alfa_or_T1 - T0) * (double)(k + 1) / (double)(nsteps - 1) : T0;
    sao_sys_set_T(p, T);
  }
  for (int j = 0; j < 64; ++j) min_E[j] = mn.empty() ? 0.f : mn[j];
}

}  // extern "C"
