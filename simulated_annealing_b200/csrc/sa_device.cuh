// sa_device.cuh -- device building blocks of the multispin-coded Metropolis
// engine: counter-based Philox draws, the bit-sliced site update, and the
// colour-split lattice geometry.
//
// Reference semantics (paths relative to the reference project):
//   bit logic   src/cpu_2d.cpp:5-41, src/cpu_2dp.cpp:336-383, src/cpu_3d.cpp:107-161,
//               src/device_2d.cu:53-87, src/device_3d.cu:246-292
//   draws       src/random.cu:15-35, src/device_2d.cu:96-97
//   colouring   src/cpu_2dp.cpp:106-114, src/cpu_3d.cpp:94-105: a site's colour
//               is (x+y)%2 in 2D AND 3D, so in 3D the z neighbours share a
//               colour and each half-sweep is sequential along z.
#pragma once
#include <cstdint>

#include "sa_types.hpp"

namespace sa {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). Stream (key = seed,
// subsequence = site): draw n is lane n%4 of the block whose 128-bit counter
// is (n/4 in the low 64 bits, subsequence in the high 64 bits).
// ---------------------------------------------------------------------------
constexpr uint32_t kPhiloxM0 = 0xD2511F53u, kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;

struct uint4x { uint32_t x, y, z, w; };

__device__ __forceinline__ uint4x philox10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                           uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    unsigned long long p0 = (unsigned long long)kPhiloxM0 * c0;
    unsigned long long p1 = (unsigned long long)kPhiloxM1 * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
    k0 += kPhiloxW0;
    k1 += kPhiloxW1;
  }
  return {c0, c1, c2, c3};
}

__device__ __forceinline__ uint32_t lane_of(const uint4x& b, unsigned lane) {
  return lane == 0 ? b.x : lane == 1 ? b.y : lane == 2 ? b.z : b.w;
}

// One u32 of stream (seed, subseq) at draw index n.
__device__ __forceinline__ uint32_t philox_draw(unsigned long long seed, unsigned long long subseq,
                                                unsigned long long n) {
  unsigned long long blk = n >> 2;
  uint4x b = philox10((uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)subseq,
                      (uint32_t)(subseq >> 32), (uint32_t)seed, (uint32_t)(seed >> 32));
  return lane_of(b, (unsigned)(n & 3));
}

// ---------------------------------------------------------------------------
// Acceptance thresholds. The reference accepts a flip of a replica whose site
// has k satisfied bonds when uniform(u) < boltz[k] (float compare). uniform()
// is non-decreasing in u, so that is u < thr[k] with thr[k] the number of u32
// values whose uniform lies below boltz[k]; thr is non-increasing in k, so the
// accepted k form a prefix and "accept" is "k < t(u)" with
// t(u) = #{k : u < thr[k]}.
// ---------------------------------------------------------------------------
template <int NB>
__device__ __forceinline__ uint32_t prefix_count(uint32_t u, const uint32_t* thr) {
  uint32_t t = 0;
#pragma unroll
  for (int k = 0; k <= NB; ++k) t += (u < thr[k]) ? 1u : 0u;
  return t;
}

// Bit-sliced count of satisfied bonds (1 = satisfied): planes c0, c1, c2.
__device__ __forceinline__ void count4(word_t a, word_t b, word_t c, word_t d, word_t& c0,
                                       word_t& c1, word_t& c2) {
  word_t s1 = a ^ b ^ c;
  word_t k1 = (a & b) | (c & (a ^ b));
  c0 = s1 ^ d;
  word_t k2 = s1 & d;
  c1 = k1 ^ k2;
  c2 = k1 & k2;
}

__device__ __forceinline__ void count6(word_t a, word_t b, word_t c, word_t d, word_t e, word_t f,
                                       word_t& c0, word_t& c1, word_t& c2) {
  word_t s1 = a ^ b ^ c;
  word_t k1 = (a & b) | (c & (a ^ b));
  word_t s2 = d ^ e ^ f;
  word_t k2 = (d & e) | (f & (d ^ e));
  c0 = s1 ^ s2;
  word_t k3 = s1 & s2;
  c1 = k1 ^ k2 ^ k3;
  c2 = (k1 & k2) | (k3 & (k1 ^ k2));
}

__device__ __forceinline__ word_t bcast(uint32_t bit) { return bit ? ~0ULL : 0ULL; }

// Acceptance prefix t(u) = #{k in 0..7 : u < thr[k]} for a non-increasing
// table with thr[7] == 0 (unused tail entries are 0): three comparisons of a
// binary search, returned as the bits of t broadcast to 32-bit masks.
__device__ __forceinline__ void prefix_bits(uint32_t u, const uint32_t* thr, uint32_t& m0, uint32_t& m1,
                                            uint32_t& m2) {
  const bool b2 = u < thr[3];
  const bool b1 = u < (b2 ? thr[5] : thr[1]);
  const bool b0 = u < (b2 ? (b1 ? thr[6] : thr[4]) : (b1 ? thr[2] : thr[0]));
  m0 = b0 ? 0xFFFFFFFFu : 0u;
  m1 = b1 ? 0xFFFFFFFFu : 0u;
  m2 = b2 ? 0xFFFFFFFFu : 0u;
}

// New spin word: every replica whose satisfied-bond count (c2 c1 c0) is below
// t (bits m2 m1 m0) flips. Evaluated on the 32-bit halves.
__device__ __forceinline__ word_t flip_below(word_t s, word_t c0, word_t c1, word_t c2, uint32_t m0,
                                             uint32_t m1, uint32_t m2) {
  uint32_t r[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t a0 = (uint32_t)(c0 >> (32 * h)), a1 = (uint32_t)(c1 >> (32 * h));
    const uint32_t a2 = (uint32_t)(c2 >> (32 * h)), sh = (uint32_t)(s >> (32 * h));
    const uint32_t g0 = a0 | ~m0;
    const uint32_t g1 = (a1 & ~m1) | (~(a1 ^ m1) & g0);
    const uint32_t ge = (a2 & ~m2) | (~(a2 ^ m2) & g1);
    r[h] = sh ^ ~ge;
  }
  return (word_t)r[0] | ((word_t)r[1] << 32);
}

// Mask of replicas whose bit-sliced count (c2 c1 c0) is >= the scalar t (0..7).
__device__ __forceinline__ word_t ge_scalar(word_t c0, word_t c1, word_t c2, uint32_t t) {
  word_t t0 = bcast(t & 1), t1 = bcast(t & 2), t2 = bcast(t & 4);
  word_t g0 = c0 | ~t0;
  word_t g1 = (c1 & ~t1) | (~(c1 ^ t1) & g0);
  return (c2 & ~t2) | (~(c2 ^ t2) & g1);
}

// New spin word of a site: flip every replica whose satisfied-bond count is
// below its (spin-dependent) acceptance prefix t.
__device__ __forceinline__ word_t flip_word(word_t s, word_t c0, word_t c1, word_t c2,
                                            uint32_t t_dn, uint32_t t_up) {
  word_t keep_dn = ge_scalar(c0, c1, c2, t_dn);
  word_t keep_up = ge_scalar(c0, c1, c2, t_up);
  word_t keep = (keep_dn & ~s) | (keep_up & s);
  return s ^ ~keep;
}

// ---------------------------------------------------------------------------
// Colour-split geometry. Rows r = y + L*z; a row of colour c holds the L/2
// sites x = 2k + ((c+y)&1), k in [0, L/2). Arrays: [colour][row][k] (times a
// slot stride where several replica systems share a lattice).
// ---------------------------------------------------------------------------
struct Geo {
  int L, half_L, dim;
  long rows, half;  // rows per colour, sites per colour
};

__device__ __forceinline__ int wrap_dec(int v, int n) { return v == 0 ? n - 1 : v - 1; }
__device__ __forceinline__ int wrap_inc(int v, int n) { return v == n - 1 ? 0 : v + 1; }

// Neighbour k indices in the other colour for x-1 / x+1.
__device__ __forceinline__ void x_neighbours(int k, int par, int half_L, int& kw, int& ke) {
  if (par == 0) { kw = wrap_dec(k, half_L); ke = k; }
  else { kw = k; ke = wrap_inc(k, half_L); }
}

// Bit-sliced vertical counter: plane b holds bit b of 64 per-replica counts.
template <int B>
struct VCount {
  word_t p[B];
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int b = 0; b < B; ++b) p[b] = 0;
  }
  __device__ __forceinline__ void add(word_t m) {
    word_t carry = m;
#pragma unroll
    for (int b = 0; b < B; ++b) {
      word_t t = p[b] & carry;
      p[b] ^= carry;
      carry = t;
    }
  }
  __device__ __forceinline__ void add_counter(const VCount& o) {
    word_t carry = 0;
#pragma unroll
    for (int b = 0; b < B; ++b) {
      word_t a = p[b], q = o.p[b];
      p[b] = a ^ q ^ carry;
      carry = (a & q) | (carry & (a ^ q));
    }
  }
  // Sum over the lanes of a warp (result valid in every lane).
  __device__ __forceinline__ void warp_sum() { warp_sum_from(1); }
  // Sum over the lanes that share (lane mod first_off); first_off a power of
  // 2. Ripple-carry, fetching the partner's plane just before it is added.
  __device__ __forceinline__ void warp_sum_from(int first_off) {
    for (int off = 16; off >= first_off; off >>= 1) {
      word_t carry = 0;
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const word_t a = p[b];
        const word_t q = __shfl_xor_sync(0xffffffffu, a, off);
        p[b] = a ^ q ^ carry;
        carry = (a & q) | (carry & (a ^ q));
      }
    }
  }
  __device__ __forceinline__ unsigned count_of(int j) const { return count_low<B>(j); }
  // the count of replica j from the low NB planes (the others known zero)
  template <int NB>
  __device__ __forceinline__ unsigned count_low(int j) const {
    unsigned v = 0;
#pragma unroll
    for (int b = 0; b < NB && b < B; ++b) v |= (unsigned)((p[b] >> j) & 1ULL) << b;
    return v;
  }
};

// Adds q0 + 2*q1 (two bit-planes) into a 4-plane counter whose values stay
// below 16 (the caller flushes it often enough).
__device__ __forceinline__ void add2_small(VCount<4>& a, word_t q0, word_t q1) {
  word_t t0 = a.p[0] & q0;
  a.p[0] ^= q0;
  word_t s1 = a.p[1] ^ t0 ^ q1;
  word_t c1 = (a.p[1] & t0) | (q1 & (a.p[1] ^ t0));
  a.p[1] = s1;
  word_t t2 = a.p[2] & c1;
  a.p[2] ^= c1;
  a.p[3] ^= t2;
}

// big += small (small has 4 planes, big B >= 4).
template <int B>
__device__ __forceinline__ void add_small(VCount<B>& big, const VCount<4>& sm) {
  word_t carry = 0;
#pragma unroll
  for (int b = 0; b < B; ++b) {
    word_t q = (b < 4) ? sm.p[b] : 0;
    word_t a = big.p[b];
    big.p[b] = a ^ q ^ carry;
    carry = (a & q) | (carry & (a ^ q));
  }
}

}  // namespace sa
