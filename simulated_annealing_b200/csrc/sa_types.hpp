// sa_types.hpp -- plain types shared by host and device code.
#pragma once
#include <cstdint>

namespace sa {

typedef unsigned long long word_t;

// Acceptance thresholds of one (T, h): the reference accepts a flip of a
// replica whose site has k satisfied bonds when uniform(u) < boltz[k] (float
// compare, src/device_2d.cu:130-150); uniform() is non-decreasing in the u32
// draw u, so that is u < thr[k] with thr[k] = #{u : uniform(u) < boltz[k]}.
// thr is non-increasing in k, so the accepted k form a prefix and "accept" is
// "k < t(u)" with t(u) = #{k : u < thr[k]}.
struct Thresholds {
  uint32_t dn[8];   // spin down (bit 0): boltz[0..z]
  uint32_t up[8];   // spin up   (bit 1): boltz[z+1..2z+1]
  uint32_t bdn[8];  // open-x border sites, spin down: boltz[10..14]
  uint32_t bup[8];  // open-x border sites, spin up:   boltz[15..19]
};

// The same tables for the CPU reference's generator: a 64-bit mt19937_64
// output g becomes the double u(g) = min(fl(g) * 2^-64, 1 - 2^-53) (libstdc++
// generate_canonical<double, 53> + uniform_real_distribution(0, 1)), compared
// as double with the double table. u is non-decreasing in g, so "accept" is
// g <= thr[k] with thr[k] the largest accepted g. Entries whose Boltzmann
// factor underflows to 0 accept nothing; they are the last ones of a table
// (the factor falls with k), so each table keeps the number n* of entries
// that accept anything and the prefix counts only those.
struct ThresholdsMT {
  uint64_t dn[8], up[8], bdn[8], bup[8];
  int ndn, nup, nbdn, nbup;
};

// The split acceptance (the reference's SPLIT_H build, src/device_2d.cu:27-50,
// src/device_3d.cu:216-245): the bond part of a flip is accepted with one
// uniform, the field part of an up spin with a second. bond[n] / bbond[n]
// (open-x border sites, whose forced bond is counted in n): the bond part of
// a replica with n satisfied bonds is accepted iff u1 < bond[n] (2^32:
// always); field: an up spin's field part iff u2 < field. Thresholds are
// counts of u32 values whose uniform lies below the float table entry, as
// in Thresholds, but 64-bit so that "always" (an entry above 1) fits.
struct SplitThresholds {
  uint64_t bond[8];
  uint64_t bbond[8];
  uint64_t field;
};

// mt19937_64 (Matsumoto & Nishimura, the C++ standard's predefined engine):
// 312 state words; the state block on the device holds the words and then
// the index of the next output.
constexpr int kMtN = 312;


}  // namespace sa
