// sa_measure.cuh -- block-level energy / magnetisation counting of one system
// (the reference's measure(), src/cpu_2d.cpp:67-94, src/cpu_2dp.cpp:196-214,
// src/cpu_3d.cpp:333-371, src/device_2d.cu:141-208), shared by the engine's
// measure kernels.
#pragma once
#include "sa_b200.h"
#include "sa_device.cuh"

namespace sa {

constexpr int kMeasureThreads = 256;
constexpr int kMeasureMaxSitesPerThread = 512;  // 3 bonds each: per-warp sum < 2^16

// This block's share of the per-replica counts of one system: satisfied bonds
// into sm[0..63], up spins into sm[64..127] (each bond counted once, from its
// site towards -x/-y/-z; the open-x lattice has no bond across x = 0). The
// grid strides over the sites; the caller combines the blocks' sm[].
__device__ __forceinline__ void measure_block_counts(const word_t* __restrict__ s,
                                                     const word_t* __restrict__ J, int L, int lattice,
                                                     unsigned int* sm) {
  for (int i = threadIdx.x; i < 128; i += blockDim.x) sm[i] = 0;
  __syncthreads();
  const int hL = L >> 1;
  const int dim = (lattice == SA_LATTICE_3D) ? 3 : 2;
  const long rows = (dim == 3) ? (long)L * L : L;
  const long half = rows * hL;
  const long N = 2 * half;
  VCount<16> sat, up;
  sat.clear();
  up.clear();
  const long stride = (long)gridDim.x * blockDim.x;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += stride) {
    const int c = (int)(t / half);
    const long rem = t - (long)c * half;
    const long r = rem / hL;
    const int k = (int)(rem - r * hL);
    const int y = (int)(r % L), z = (int)(r / L);
    const int par = (c + y) & 1, x = 2 * k + par;
    int kw, ke;
    x_neighbours(k, par, hL, kw, ke);
    const word_t* sc = s + (long)c * half;
    const word_t* so = s + (long)(1 - c) * half;
    word_t si = sc[rem];
    up.add(si);
    if (!(lattice == SA_LATTICE_2D_OPEN_X && x == 0))
      sat.add(J[(long)(0 * 2 + c) * half + rem] ^ si ^ so[r * hL + kw]);
    const long rn = (long)wrap_dec(y, L) + (long)L * z;
    sat.add(J[(long)(1 * 2 + c) * half + rem] ^ si ^ so[rn * hL + k]);
    if (dim == 3) {
      const long ru = (long)y + (long)L * wrap_dec(z, L);
      sat.add(J[(long)(2 * 2 + c) * half + rem] ^ si ^ sc[ru * hL + k]);
    }
  }
  sat.warp_sum();
  up.warp_sum();
  const int lane = threadIdx.x & 31;
  atomicAdd(&sm[lane], sat.count_of(lane));
  atomicAdd(&sm[lane + 32], sat.count_of(lane + 32));
  atomicAdd(&sm[64 + lane], up.count_of(lane));
  atomicAdd(&sm[96 + lane], up.count_of(lane + 32));
  __syncthreads();
}


}  // namespace sa
