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


}  // namespace sa
