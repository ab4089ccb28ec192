// sa_system.cu -- single-system engine: the gpu_sys boundary as a C ABI.
//
// One system = one lattice x 64 replicas (src/gpu_sys.cuh:12-29). Device
// layout (colour = (x+y)%2, the reference's sweep colour in 2D and 3D):
//   spins  [colour][row][k]          row = y + L*z, x = 2k + ((colour+y)&1)
//   J      [axis][colour][row][k]    own bond of the site towards -x/-y/-z
// A half-sweep of colour c is one launch. In 2D every site of the colour is
// independent (one thread per site). In 3D the z neighbours share the colour,
// so a thread walks one (x,y) column in increasing z, carrying the updated
// spin of z-1 and the new z=0 spin for the periodic wrap -- exactly the order
// of src/cpu_3d.cpp:94-105.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "sa_b200.h"
#include "sa_device.cuh"
#include "sa_host.hpp"
#include "sa_measure.cuh"
#include "sa_system.hpp"

namespace sa {

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// One 2D half-sweep of colour c; one thread per site of that colour.
// Prefix t(g) = #{k < n : g <= thr[k]} of an mt19937_64 table (ThresholdsMT).
template <int NB>
__device__ __forceinline__ uint32_t prefix_count_mt(uint64_t g, const uint64_t* thr, int n) {
  uint32_t t = 0;
#pragma unroll
  for (int k = 0; k <= NB; ++k) t += (k < n && g <= thr[k]) ? 1u : 0u;
  return t;
}

// The split update (the reference's SPLIT_H build, src/device_2d.cu:27-50,
// src/device_3d.cu:216-245): with n satisfied bonds (bit-sliced c2 c1 c0),
// the bond part is accepted iff u1 < bond[n] -- the accepted n are a prefix
// of 0..NB because bond[] does not increase -- and an up spin's field part
// iff u2 < field; a replica flips when both parts are accepted.
template <int NB>
__device__ __forceinline__ word_t split_flip(word_t si, word_t c0, word_t c1, word_t c2, uint32_t u1, uint32_t u2,
                                             const uint64_t* bond, uint64_t field) {
  uint32_t tb = 0;
#pragma unroll
  for (int n = 0; n <= NB; ++n) tb += ((uint64_t)u1 < bond[n]) ? 1u : 0u;
  const word_t bond_ok = ~ge_scalar(c0, c1, c2, tb);           // n < tb
  const word_t field_ok = ~si | bcast((uint64_t)u2 < field);  // down spins: always
  return si ^ (bond_ok & field_ok);
}

// MT: the site's draw is the pass's mt19937_64 output at its rank in the
// reference's sweep order (draws[idx], idx = row * L/2 + k), not Philox.
// SPLIT: the split update with draws `draw` (bond) and `draw + 1` (field).
template <bool OPEN_X, bool MT = false, bool SPLIT = false>
__global__ void __launch_bounds__(256) k_halfsweep_2d(word_t* __restrict__ s,
                                                      const word_t* __restrict__ J, int L,
                                                      unsigned long long seed,
                                                      unsigned long long draw, int c,
                                                      Thresholds thr, const uint64_t* __restrict__ draws = nullptr,
                                                      ThresholdsMT tm = {}, SplitThresholds st = {}) {
  const int hL = L >> 1;
  const long half = (long)L * hL;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= half) return;
  const int r = (int)(t / hL), k = (int)(t - (long)r * hL);
  const int y = r, par = (c + y) & 1, x = 2 * k + par;
  int kw, ke;
  x_neighbours(k, par, hL, kw, ke);
  const int rn = wrap_dec(r, L), rs = wrap_inc(r, L);
  const word_t* so = s + (long)(1 - c) * half;  // other colour
  word_t* sc = s + (long)c * half;
  const word_t* Jx_c = J + (long)(0 * 2 + c) * half;
  const word_t* Jx_o = J + (long)(0 * 2 + 1 - c) * half;
  const word_t* Jy_c = J + (long)(1 * 2 + c) * half;
  const word_t* Jy_o = J + (long)(1 * 2 + 1 - c) * half;

  const long idx = (long)r * hL + k;
  word_t si = sc[idx];
  word_t mw = Jx_c[idx] ^ so[(long)r * hL + kw] ^ si;
  word_t me = Jx_o[(long)r * hL + ke] ^ so[(long)r * hL + ke] ^ si;
  word_t mn = Jy_c[idx] ^ so[(long)rn * hL + k] ^ si;
  word_t ms = Jy_o[(long)rs * hL + k] ^ so[(long)rs * hL + k] ^ si;
  bool border = false;
  if (OPEN_X) {
    if (x == 0) { mw = ~0ULL; border = true; }
    if (x == L - 1) { me = ~0ULL; border = true; }
  }
  word_t c0, c1, c2;
  count4(mw, me, mn, ms, c0, c1, c2);
  if (SPLIT) {
    const unsigned long long site = (unsigned long long)x + (unsigned long long)L * y;
    const uint32_t u1 = philox_draw(seed, site, draw), u2 = philox_draw(seed, site, draw + 1);
    sc[idx] = split_flip<4>(si, c0, c1, c2, u1, u2, (OPEN_X && border) ? st.bbond : st.bond, st.field);
    return;
  }
  uint32_t tdn, tup;
  if (MT) {
    const uint64_t g = draws[idx];
    if (OPEN_X && border) {
      tdn = prefix_count_mt<4>(g, tm.bdn, tm.nbdn);
      tup = prefix_count_mt<4>(g, tm.bup, tm.nbup);
    } else {
      tdn = prefix_count_mt<4>(g, tm.dn, tm.ndn);
      tup = prefix_count_mt<4>(g, tm.up, tm.nup);
    }
  } else {
    const unsigned long long site = (unsigned long long)x + (unsigned long long)L * y;
    const uint32_t u = philox_draw(seed, site, draw);
    if (OPEN_X && border) {
      tdn = prefix_count<4>(u, thr.bdn);
      tup = prefix_count<4>(u, thr.bup);
    } else {
      tdn = prefix_count<4>(u, thr.dn);
      tup = prefix_count<4>(u, thr.up);
    }
  }
  sc[idx] = flip_word(si, c0, c1, c2, tdn, tup);
}

// One 3D half-sweep of colour c; one thread per (x,y) column, walking z.
// SPLIT: the split update; a site on the lattice's boundary (a coordinate 0
// or L-1) uses its field draw for the bond part too, as the reference's
// boundary branch passes rand2 twice (src/device_3d.cu:76-89).
template <bool MT = false, bool SPLIT = false>
__global__ void __launch_bounds__(128) k_halfsweep_3d(word_t* __restrict__ s,
                                                      const word_t* __restrict__ J, int L,
                                                      unsigned long long seed,
                                                      unsigned long long draw, int c,
                                                      Thresholds thr, const uint64_t* __restrict__ draws = nullptr,
                                                      ThresholdsMT tm = {}, SplitThresholds st = {}) {
  const int hL = L >> 1;
  const long plane = (long)L * hL;  // columns per colour
  const long half = plane * L;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= plane) return;
  const int y = (int)(t / hL), k = (int)(t - (long)y * hL);
  const int par = (c + y) & 1, x = 2 * k + par;
  int kw, ke;
  x_neighbours(k, par, hL, kw, ke);
  const int yn = wrap_dec(y, L), ys = wrap_inc(y, L);
  const word_t* so = s + (long)(1 - c) * half;
  word_t* sc = s + (long)c * half;
  const word_t* Jx_c = J + (long)(0 * 2 + c) * half;
  const word_t* Jx_o = J + (long)(0 * 2 + 1 - c) * half;
  const word_t* Jy_c = J + (long)(1 * 2 + c) * half;
  const word_t* Jy_o = J + (long)(1 * 2 + 1 - c) * half;
  const word_t* Jz_c = J + (long)(2 * 2 + c) * half;

  word_t prev = sc[((long)(y + L * (L - 1))) * hL + k];  // z = L-1, not yet updated
  word_t first = 0;
  for (int z = 0; z < L; ++z) {
    const long r = y + (long)L * z;
    const long idx = r * hL + k;
    const long rd = y + (long)L * (z == L - 1 ? 0 : z + 1);
    word_t si = sc[idx];
    word_t sd = (z == L - 1) ? first : sc[rd * hL + k];
    word_t mw = Jx_c[idx] ^ so[r * hL + kw] ^ si;
    word_t me = Jx_o[r * hL + ke] ^ so[r * hL + ke] ^ si;
    word_t mn = Jy_c[idx] ^ so[(yn + (long)L * z) * hL + k] ^ si;
    word_t ms = Jy_o[(ys + (long)L * z) * hL + k] ^ so[(ys + (long)L * z) * hL + k] ^ si;
    word_t mu = Jz_c[idx] ^ prev ^ si;
    word_t md = Jz_c[rd * hL + k] ^ sd ^ si;
    word_t c0, c1, c2;
    count6(mw, me, mn, ms, mu, md, c0, c1, c2);
    if (SPLIT) {
      const unsigned long long site = (unsigned long long)x + (unsigned long long)L * r;
      const uint32_t u2 = philox_draw(seed, site, draw + 1);
      const bool edge = x == 0 || y == 0 || z == 0 || x == L - 1 || y == L - 1 || z == L - 1;
      const uint32_t u1 = edge ? u2 : philox_draw(seed, site, draw);
      const word_t ns = split_flip<6>(si, c0, c1, c2, u1, u2, st.bond, st.field);
      sc[idx] = ns;
      if (z == 0) first = ns;
      prev = ns;
      continue;
    }
    uint32_t tdn, tup;
    if (MT) {
      const uint64_t g = draws[idx];
      tdn = prefix_count_mt<6>(g, tm.dn, tm.ndn);
      tup = prefix_count_mt<6>(g, tm.up, tm.nup);
    } else {
      const unsigned long long site = (unsigned long long)x + (unsigned long long)L * r;
      const uint32_t u = philox_draw(seed, site, draw);
      tdn = prefix_count<6>(u, thr.dn);
      tup = prefix_count<6>(u, thr.up);
    }
    word_t ns = flip_word(si, c0, c1, c2, tdn, tup);
    sc[idx] = ns;
    if (z == 0) first = ns;
    prev = ns;
  }
}

// Per-replica number of satisfied bonds (counts[0..63]) and of up spins
// (counts[64..127]); one block-level partial per block, added atomically.
__global__ void __launch_bounds__(kMeasureThreads) k_measure(const word_t* __restrict__ s,
                                                             const word_t* __restrict__ J, int L,
                                                             int lattice,
                                                             unsigned long long* counts) {
  __shared__ unsigned int sm[128];
  measure_block_counts(s, J, L, lattice, sm);
  for (int i = threadIdx.x; i < 128; i += blockDim.x)
    if (sm[i]) atomicAdd(&counts[i], (unsigned long long)sm[i]);
}

__global__ void k_measure_finalize(const unsigned long long* counts, long nbonds, long N,
                                   int64_t* E, int64_t* M) {
  int j = threadIdx.x;
  if (j < 64) {
    E[j] = 2 * (int64_t)counts[j] - nbonds;
    M[j] = 2 * (int64_t)counts[64 + j] - N;
  }
}

__global__ void k_swap(word_t* __restrict__ a, word_t* __restrict__ b, word_t mask, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    word_t x = a[i], y = b[i];
    word_t d = (x ^ y) & mask;
    a[i] = x ^ d;
    b[i] = y ^ d;
  }
}

__device__ __forceinline__ long split_index(long i, int L, long half, int hL) {
  // row-major site i = x + L*r -> [colour][row][k]
  long r = i / L;
  int x = (int)(i - r * L);
  int y = (int)(r % L);
  int c = (x + y) & 1;
  return (long)c * half + r * hL + (x >> 1);
}

// init_J: 2*dim draws per site, own word a = draw[2a] | draw[2a+1] << 32
// (src/random.cu:25-35 then src/device_2d.cu:133-136 / src/device_3d.cu:104-123).
__global__ void k_init_J(word_t* __restrict__ J, int L, int dim, long N,
                         unsigned long long seed, unsigned long long draw) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int hL = L >> 1;
  const long half = N / 2;
  long dst = split_index(i, L, half, hL);
  long c = dst / half, rem = dst - c * half;
  uint32_t d[6];
  unsigned long long blk = ~0ULL;
  uint4x b = {0, 0, 0, 0};
  for (int q = 0; q < 2 * dim; ++q) {
    unsigned long long n = draw + q;
    if ((n >> 2) != blk) {
      blk = n >> 2;
      b = philox10((uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)i, (uint32_t)((unsigned long long)i >> 32),
                   (uint32_t)seed, (uint32_t)(seed >> 32));
    }
    d[q] = lane_of(b, (unsigned)(n & 3));
  }
  for (int a = 0; a < dim; ++a)
    J[(long)(a * 2 + c) * half + rem] = (word_t)d[2 * a] | ((word_t)d[2 * a + 1] << 32);
}

// Counter-based initial spins: block (epoch, 0, i, 2^31 | i>>32), lanes 0,1.
// tag: 0x80000000, or 0xC0000000 for a system whose first half-sweep is
// colour 1 (the second configuration of a two-lattice pair draws its initial
// spins from its own counter range)
__global__ void k_init_rand(word_t* __restrict__ s, int L, long N, unsigned long long seed,
                            unsigned long long epoch, uint32_t tag) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  uint4x b = philox10((uint32_t)epoch, (uint32_t)(epoch >> 32), (uint32_t)i,
                      tag | (uint32_t)((unsigned long long)i >> 32), (uint32_t)seed,
                      (uint32_t)(seed >> 32));
  s[split_index(i, L, N / 2, L >> 1)] = (word_t)b.x | ((word_t)b.y << 32);
}

// ---------------------------------------------------------------------------
// mt19937_64 on the device: one block advances the system's generator state
// (st[0..311] words, st[312] the index of the next output) by `count` outputs
// into out[0..count). The twist is the standard recurrence in its three
// dependency phases (words 0..155 read old words 156..311; words 156..310 read
// the new words 0..154; word 311 reads the new words 0 and 155), then every
// output is tempered.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mt64_twist_word(uint64_t a, uint64_t b, uint64_t m) {
  const uint64_t y = (a & 0xFFFFFFFF80000000ULL) | (b & 0x7FFFFFFFULL);
  return m ^ (y >> 1) ^ ((y & 1ULL) ? 0xB5026F5AA96619E9ULL : 0ULL);
}

__device__ __forceinline__ uint64_t mt64_temper(uint64_t z) {
  z ^= (z >> 29) & 0x5555555555555555ULL;
  z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
  z ^= (z << 37) & 0xFFF7EEE000000000ULL;
  z ^= z >> 43;
  return z;
}

__global__ void __launch_bounds__(320) k_mt_gen(uint64_t* __restrict__ st, uint64_t* __restrict__ out, long count) {
  __shared__ uint64_t mt[kMtN];
  const int t = threadIdx.x;
  for (int i = t; i < kMtN; i += blockDim.x) mt[i] = st[i];
  int idx = (int)st[kMtN];
  __syncthreads();
  long pos = 0;
  while (pos < count) {
    if (idx >= kMtN) {
      uint64_t v = 0;
      if (t < 156) v = mt64_twist_word(mt[t], mt[t + 1], mt[t + 156]);
      __syncthreads();
      if (t < 156) mt[t] = v;
      __syncthreads();
      if (t >= 156 && t < kMtN - 1) v = mt64_twist_word(mt[t], mt[t + 1], mt[t - 156]);
      __syncthreads();
      if (t >= 156 && t < kMtN - 1) mt[t] = v;
      __syncthreads();
      if (t == 0) mt[kMtN - 1] = mt64_twist_word(mt[kMtN - 1], mt[0], mt[155]);
      __syncthreads();
      idx = 0;
    }
    const long n = min((long)(kMtN - idx), count - pos);
    for (int i = t; i < n; i += blockDim.x) out[pos + i] = mt64_temper(mt[idx + i]);
    pos += n;
    idx += (int)n;
    __syncthreads();  // the next twist rewrites mt
  }
  for (int i = t; i < kMtN; i += blockDim.x) st[i] = mt[i];
  if (t == 0) st[kMtN] = (uint64_t)idx;
}

// init_J from mt19937_64 outputs: buffer[dim*i + a] is site i's own bond word
// on axis a (src/cpu_2dp.cpp:243-260, src/cpu_3d.cpp:281-301).
__global__ void k_init_J_mt(word_t* __restrict__ J, const uint64_t* __restrict__ buf, int L, int dim, long N) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const long half = N / 2;
  const long dst = split_index(i, L, half, L >> 1);
  const long c = dst / half, rem = dst - c * half;
  for (int a = 0; a < dim; ++a) J[(long)(a * 2 + c) * half + rem] = buf[(long)dim * i + a];
}

__global__ void k_fill(word_t* __restrict__ s, long n, word_t v) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) s[i] = v;
}

__global__ void k_rowmajor_to_split(const word_t* __restrict__ src, word_t* __restrict__ dst, int L,
                                    long N) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) dst[split_index(i, L, N / 2, L >> 1)] = src[i];
}

__global__ void k_split_to_rowmajor(const word_t* __restrict__ src, word_t* __restrict__ dst, int L,
                                    long N) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) dst[i] = src[split_index(i, L, N / 2, L >> 1)];
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

static inline unsigned grid_for(long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

int launch_halfsweep(sa_system* sy, int c, unsigned long long draw) {
  if (sy->split) {
    if (sy->lattice == SA_LATTICE_3D) {
      long plane = (long)sy->L * (sy->L / 2);
      k_halfsweep_3d<false, true><<<grid_for(plane, 128), 128, 0, sy->stream>>>(
          sy->d_s, sy->d_J, sy->L, sy->seed, draw, c, sy->thr, nullptr, ThresholdsMT{}, sy->sthr);
    } else if (sy->lattice == SA_LATTICE_2D_OPEN_X) {
      k_halfsweep_2d<true, false, true><<<grid_for(sy->half, 256), 256, 0, sy->stream>>>(
          sy->d_s, sy->d_J, sy->L, sy->seed, draw, c, sy->thr, nullptr, ThresholdsMT{}, sy->sthr);
    } else {
      k_halfsweep_2d<false, false, true><<<grid_for(sy->half, 256), 256, 0, sy->stream>>>(
          sy->d_s, sy->d_J, sy->L, sy->seed, draw, c, sy->thr, nullptr, ThresholdsMT{}, sy->sthr);
    }
    return SA_OK;
  }
  if (sy->lattice == SA_LATTICE_3D) {
    long plane = (long)sy->L * (sy->L / 2);
    k_halfsweep_3d<false><<<grid_for(plane, 128), 128, 0, sy->stream>>>(sy->d_s, sy->d_J, sy->L, sy->seed,
                                                                  draw, c, sy->thr);
  } else if (sy->lattice == SA_LATTICE_2D_OPEN_X) {
    k_halfsweep_2d<true><<<grid_for(sy->half, 256), 256, 0, sy->stream>>>(sy->d_s, sy->d_J, sy->L,
                                                                          sy->seed, draw, c, sy->thr);
  } else {
    k_halfsweep_2d<false><<<grid_for(sy->half, 256), 256, 0, sy->stream>>>(sy->d_s, sy->d_J, sy->L,
                                                                           sy->seed, draw, c, sy->thr);
  }
  return SA_OK;
}

int mt_generate(sa_system* sy, long n) {
  k_mt_gen<<<1, 320, 0, sy->stream>>>(sy->d_mt, sy->d_draws, n);
  SA_CUDA_TRY(cudaGetLastError());
  return SA_OK;
}

// One sweep in MT mode: the reference visits colour 0 then colour 1, each in
// row-major order, one draw per site (src/cpu_2dp.cpp:106-114,
// src/cpu_3d.cpp:94-105); rank row*L/2 + k of colour c is draw c*N/2 + rank.
int mt_sweep(sa_system* sy) {
  int st = mt_generate(sy, sy->N);
  if (st) return st;
  for (int c = 0; c < 2; ++c) {
    const uint64_t* dr = sy->d_draws + (long)c * sy->half;
    if (sy->lattice == SA_LATTICE_3D) {
      long plane = (long)sy->L * (sy->L / 2);
      k_halfsweep_3d<true><<<grid_for(plane, 128), 128, 0, sy->stream>>>(sy->d_s, sy->d_J, sy->L, sy->seed, 0, c,
                                                                        sy->thr, dr, sy->thr_mt);
    } else if (sy->lattice == SA_LATTICE_2D_OPEN_X) {
      k_halfsweep_2d<true, true><<<grid_for(sy->half, 256), 256, 0, sy->stream>>>(
          sy->d_s, sy->d_J, sy->L, sy->seed, 0, c, sy->thr, dr, sy->thr_mt);
    } else {
      k_halfsweep_2d<false, true><<<grid_for(sy->half, 256), 256, 0, sy->stream>>>(
          sy->d_s, sy->d_J, sy->L, sy->seed, 0, c, sy->thr, dr, sy->thr_mt);
    }
  }
  SA_CUDA_TRY(cudaGetLastError());
  return SA_OK;
}

int launch_measure(sa_system* sy, int64_t* d_E, int64_t* d_M) {
  SA_CUDA_TRY(cudaMemsetAsync(sy->d_counts, 0, 128 * sizeof(unsigned long long), sy->stream));
  // At most kMeasureMaxSitesPerThread sites per thread (counter width), about
  // 8 per thread when the grid stays under 8 blocks per SM of a B200.
  const long per_block = (long)kMeasureThreads * kMeasureMaxSitesPerThread;
  const long min_nb = (sy->N + per_block - 1) / per_block;
  long nb = (sy->N + kMeasureThreads * 8 - 1) / (kMeasureThreads * 8);
  if (nb > 1184) nb = 1184;
  if (nb < min_nb) nb = min_nb;
  if (nb < 1) nb = 1;
  k_measure<<<(unsigned)nb, kMeasureThreads, 0, sy->stream>>>(sy->d_s, sy->d_J, sy->L, sy->lattice,
                                                               sy->d_counts);
  k_measure_finalize<<<1, 64, 0, sy->stream>>>(sy->d_counts, sy->nbonds, sy->N, d_E, d_M);
  return SA_OK;
}

}  // namespace sa

using namespace sa;

// Sweep counts from which sa_sys_sweep hands a zero-field lattice to the
// resident kernel (one launch, lattice held in shared memory) instead of two
// launches per sweep.
static constexpr long kResidentMinSweeps = 16;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* sa_version(void) { return "sa_b200 0.1 (sm_100a)"; }

const char* sa_status_string(int s) {
  switch (s) {
    case SA_OK: return "ok";
    case SA_ERR_INVALID: return "invalid argument";
    case SA_ERR_ODD_L: return "L must be even";
    case SA_ERR_CUDA: return "CUDA error";
    case SA_ERR_NO_DEVICE: return "no CUDA device";
    case SA_ERR_MISMATCH: return "systems differ in shape";
    case SA_ERR_J_INCONSISTENT: return "duplicated coupling words disagree";
    case SA_ERR_BUFFER: return "buffer too small or malformed";
    case SA_ERR_BUDGET: return "memory budget exceeded";
    case SA_ERR_TIMEOUT: return "device-side wait timed out";
    case SA_ERR_UNSUPPORTED: return "unsupported request";
    default: return "unknown status";
  }
}

int sa_sys_create(int lattice, int L, double T, double h, sa_system_t* out) {
  if (!out) return fail(SA_ERR_INVALID, "out is null");
  *out = nullptr;
  if (lattice < 0 || lattice > 2) return fail(SA_ERR_INVALID, "unknown lattice kind");
  if (L < 2) return fail(SA_ERR_INVALID, "L must be >= 2");
  if (L & 1) return fail(SA_ERR_ODD_L, "L must be even for the checkerboard update");
  if (L > 4096 || (lattice == SA_LATTICE_3D && L > 1024))
    return fail(SA_ERR_INVALID, "L too large");
  if (!(T > 0)) return fail(SA_ERR_INVALID, "T must be > 0");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(SA_ERR_NO_DEVICE, "no CUDA device available");
  sa_system* sy = new sa_system();
  sy->lattice = lattice;
  sy->L = L;
  sy->dim = lattice_dim(lattice);
  sy->N = (sy->dim == 3) ? (long)L * L * L : (long)L * L;
  sy->half = sy->N / 2;
  sy->nbonds = (long)sy->dim * sy->N - (lattice == SA_LATTICE_2D_OPEN_X ? L : 0);
  sy->T = T;
  sy->h = h;
  sy->seed = 1234;  // src/gpu_2d.cu:47
  sy->draw = 0;
  sy->epoch = 0;
  cudaGetDevice(&sy->device);
  int st = SA_OK;
  auto chk = [&](cudaError_t e, const char* w) {
    if (e != cudaSuccess && st == SA_OK) st = cuda_fail(e, w);
  };
  chk(cudaStreamCreateWithFlags(&sy->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  sy->stream = sy->own_stream;
  chk(cudaMalloc(&sy->d_s, sy->N * sizeof(word_t)), "cudaMalloc spins");
  chk(cudaMalloc(&sy->d_J, (size_t)sy->dim * sy->N * sizeof(word_t)), "cudaMalloc J");
  chk(cudaMalloc(&sy->d_stage, sy->N * sizeof(word_t)), "cudaMalloc stage");
  chk(cudaMalloc(&sy->d_counts, 128 * sizeof(unsigned long long)), "cudaMalloc counts");
  chk(cudaMalloc(&sy->d_EM, 128 * sizeof(int64_t)), "cudaMalloc E/M");
  chk(cudaMalloc(&sy->d_mt, (kMtN + 1) * sizeof(uint64_t)), "cudaMalloc mt state");
  if (st == SA_OK) {
    chk(cudaMemsetAsync(sy->d_s, 0, sy->N * sizeof(word_t), sy->stream), "memset");
    chk(cudaMemsetAsync(sy->d_J, 0, (size_t)sy->dim * sy->N * sizeof(word_t), sy->stream), "memset");
    chk(cudaStreamSynchronize(sy->stream), "sync");
  }
  if (st == SA_OK && !make_thresholds(lattice, T, h, &sy->thr))
    st = fail(SA_ERR_INVALID, "non-monotone Boltzmann table");
  if (st != SA_OK) {
    sa_sys_destroy(sy);
    return st;
  }
  *out = sy;
  return SA_OK;
}

int sa_sys_destroy(sa_system_t sy) {
  if (!sy) return SA_OK;
  if (sy->own_stream) cudaStreamSynchronize(sy->own_stream);
  if (sy->stream && sy->stream != sy->own_stream) cudaStreamSynchronize(sy->stream);
  cudaFree(sy->d_s);
  cudaFree(sy->d_J);
  cudaFree(sy->d_stage);
  cudaFree(sy->d_counts);
  cudaFree(sy->d_EM);
  cudaFree(sy->d_mt);
  cudaFree(sy->d_draws);
  if (sy->own_stream) cudaStreamDestroy(sy->own_stream);
  delete sy;
  return SA_OK;
}

int sa_sys_set_stream(sa_system_t sy, void* stream) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  sy->stream = stream ? (cudaStream_t)stream : sy->own_stream;
  return SA_OK;
}

int sa_sys_set_T(sa_system_t sy, double T) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  if (!(T > 0)) return fail(SA_ERR_INVALID, "T must be > 0");
  Thresholds t;
  if (!make_thresholds(sy->lattice, T, sy->h, &t)) return fail(SA_ERR_INVALID, "non-monotone table");
  ThresholdsMT tm;
  if (sy->rng_mode == SA_RNG_MT19937_64 && !make_thresholds_mt(sy->lattice, T, sy->h, &tm))
    return fail(SA_ERR_INVALID, "non-monotone table");
  sy->T = T;
  sy->thr = t;  // kernel argument: later launches see it, earlier ones keep theirs
  if (sy->rng_mode == SA_RNG_MT19937_64) sy->thr_mt = tm;
  make_split_thresholds(sy->lattice, sy->T, sy->h, &sy->sthr);
  return SA_OK;
}

int sa_sys_set_h(sa_system_t sy, double h) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  Thresholds t;
  if (!make_thresholds(sy->lattice, sy->T, h, &t)) return fail(SA_ERR_INVALID, "non-monotone table");
  ThresholdsMT tm;
  if (sy->rng_mode == SA_RNG_MT19937_64 && !make_thresholds_mt(sy->lattice, sy->T, h, &tm))
    return fail(SA_ERR_INVALID, "non-monotone table");
  sy->h = h;
  sy->thr = t;
  if (sy->rng_mode == SA_RNG_MT19937_64) sy->thr_mt = tm;
  make_split_thresholds(sy->lattice, sy->T, sy->h, &sy->sthr);
  return SA_OK;
}

int sa_sys_get_T(sa_system_t sy, double* T) {
  if (!sy || !T) return fail(SA_ERR_INVALID, "null argument");
  *T = sy->T;
  return SA_OK;
}

// MT mode: the device generator restarts from `seed` (gen.seed(seed),
// src/cpu_3d.cpp:210). The state is built on the host (312 words).
static int mt_reseed(sa_system* sy) {
  uint64_t st[kMtN + 1];
  mt64_seed(sy->seed, st);
  SA_CUDA_TRY(cudaMemcpyAsync(sy->d_mt, st, sizeof st, cudaMemcpyHostToDevice, sy->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));  // st is on this stack frame
  return SA_OK;
}

int sa_sys_set_seed(sa_system_t sy, uint64_t seed) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  sy->seed = seed;
  sy->draw = 0;
  sy->epoch = 0;
  if (sy->rng_mode == SA_RNG_MT19937_64) return mt_reseed(sy);
  return SA_OK;
}

int sa_sys_set_rng_mode(sa_system_t sy, int mode) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  if (mode != SA_RNG_PHILOX && mode != SA_RNG_MT19937_64) return fail(SA_ERR_INVALID, "unknown random mode");
  if (mode == SA_RNG_MT19937_64 && sy->split)
    return fail(SA_ERR_UNSUPPORTED, "the split update is defined for the GPU reference's Philox draws only");
  if (mode == SA_RNG_MT19937_64 && sy->first_colour != 0)
    return fail(SA_ERR_UNSUPPORTED, "the mt19937_64 stream has one visiting order: first colour must be 0");
  if (mode == SA_RNG_MT19937_64) {
    ThresholdsMT tm;
    if (!make_thresholds_mt(sy->lattice, sy->T, sy->h, &tm)) return fail(SA_ERR_INVALID, "non-monotone table");
    if (!sy->d_draws) SA_CUDA_TRY(cudaMalloc(&sy->d_draws, (size_t)sy->dim * sy->N * sizeof(uint64_t)));
    sy->thr_mt = tm;
    sy->rng_mode = mode;
    return mt_reseed(sy);
  }
  sy->rng_mode = mode;
  return SA_OK;
}

int sa_sys_set_first_colour(sa_system_t sy, int colour) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  if (colour != 0 && colour != 1) return fail(SA_ERR_INVALID, "the first colour is 0 or 1");
  if (colour != 0 && sy->rng_mode != SA_RNG_PHILOX)
    return fail(SA_ERR_UNSUPPORTED, "the first colour can be 1 in Philox mode only");
  sy->first_colour = colour;
  return SA_OK;
}

int sa_sys_set_split_field(sa_system_t sy, int on) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  if (on && sy->rng_mode != SA_RNG_PHILOX)
    return fail(SA_ERR_UNSUPPORTED, "the split update is defined for the GPU reference's Philox draws only");
  sy->split = on ? 1 : 0;
  make_split_thresholds(sy->lattice, sy->T, sy->h, &sy->sthr);
  return SA_OK;
}

int sa_sys_get_split_field(sa_system_t sy, int* on) {
  if (!sy || !on) return fail(SA_ERR_INVALID, "null argument");
  *on = sy->split;
  return SA_OK;
}

int sa_sys_get_first_colour(sa_system_t sy, int* colour) {
  if (!sy || !colour) return fail(SA_ERR_INVALID, "null argument");
  *colour = sy->first_colour;
  return SA_OK;
}

int sa_sys_get_rng_mode(sa_system_t sy, int* mode) {
  if (!sy || !mode) return fail(SA_ERR_INVALID, "null argument");
  *mode = sy->rng_mode;
  return SA_OK;
}

int sa_sys_init_J(sa_system_t sy) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  if (sy->rng_mode == SA_RNG_MT19937_64) {
    int st = mt_generate(sy, (long)sy->dim * sy->N);
    if (st) return st;
    k_init_J_mt<<<grid_for(sy->N, 256), 256, 0, sy->stream>>>(sy->d_J, sy->d_draws, sy->L, sy->dim, sy->N);
    SA_CUDA_TRY(cudaGetLastError());
    return SA_OK;
  }
  k_init_J<<<grid_for(sy->N, 256), 256, 0, sy->stream>>>(sy->d_J, sy->L, sy->dim, sy->N, sy->seed,
                                                          sy->draw);
  SA_CUDA_TRY(cudaGetLastError());
  sy->draw += 2 * sy->dim;
  return SA_OK;
}

int sa_sys_init_rand(sa_system_t sy) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  if (sy->rng_mode == SA_RNG_MT19937_64) {
    // s[i] = gen() in row-major order (src/cpu_2dp.cpp:222-226, src/cpu_3d.cpp:257-263)
    int st = mt_generate(sy, sy->N);
    if (st) return st;
    k_rowmajor_to_split<<<grid_for(sy->N, 256), 256, 0, sy->stream>>>((const word_t*)sy->d_draws, sy->d_s, sy->L,
                                                                    sy->N);
    SA_CUDA_TRY(cudaGetLastError());
    return SA_OK;
  }
  k_init_rand<<<grid_for(sy->N, 256), 256, 0, sy->stream>>>(sy->d_s, sy->L, sy->N, sy->seed, sy->epoch,
                                                              sy->first_colour ? 0xC0000000u : 0x80000000u);
  SA_CUDA_TRY(cudaGetLastError());
  sy->epoch += 1;
  return SA_OK;
}

int sa_sys_init_order(sa_system_t sy) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  k_fill<<<grid_for(sy->N, 256), 256, 0, sy->stream>>>(sy->d_s, sy->N, ~0ULL);
  SA_CUDA_TRY(cudaGetLastError());
  return SA_OK;
}

int sa_sys_set_spins(sa_system_t sy, const uint64_t* s) {
  if (!sy || !s) return fail(SA_ERR_INVALID, "null argument");
  SA_CUDA_TRY(cudaMemcpyAsync(sy->d_stage, s, sy->N * sizeof(word_t), cudaMemcpyHostToDevice, sy->stream));
  k_rowmajor_to_split<<<grid_for(sy->N, 256), 256, 0, sy->stream>>>(sy->d_stage, sy->d_s, sy->L, sy->N);
  SA_CUDA_TRY(cudaGetLastError());
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  return SA_OK;
}

int sa_sys_get_spins(sa_system_t sy, uint64_t* s) {
  if (!sy || !s) return fail(SA_ERR_INVALID, "null argument");
  k_split_to_rowmajor<<<grid_for(sy->N, 256), 256, 0, sy->stream>>>(sy->d_s, sy->d_stage, sy->L, sy->N);
  SA_CUDA_TRY(cudaGetLastError());
  SA_CUDA_TRY(cudaMemcpyAsync(s, sy->d_stage, sy->N * sizeof(word_t), cudaMemcpyDeviceToHost, sy->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  return SA_OK;
}

// Host view of the lattice for the coupling layout conversions.
static void nb_plus(const sa_system* sy, long i, long* e, long* s_, long* d) {
  const long L = sy->L, L2 = L * L;
  *e = ((i + 1) % L == 0) ? i - L + 1 : i + 1;
  *s_ = ((i + L) % L2 < L) ? i - L2 + L : i + L;
  *d = (sy->dim == 3) ? ((i + L2 >= sy->N) ? i - sy->N + L2 : i + L2) : 0;
}

static long host_split(const sa_system* sy, long i) {
  long r = i / sy->L;
  int x = (int)(i - r * sy->L);
  int y = (int)(r % sy->L);
  int c = (x + y) & 1;
  return (long)c * sy->half + r * (sy->L / 2) + (x >> 1);
}

int sa_sys_set_J(sa_system_t sy, const uint64_t* jx, const uint64_t* jy, const uint64_t* jz) {
  if (!sy || !jx || !jy || (sy->dim == 3 && !jz)) return fail(SA_ERR_INVALID, "null argument");
  std::vector<word_t> own((size_t)sy->dim * sy->N);
  for (long i = 0; i < sy->N; ++i) {
    long e, s_, d;
    nb_plus(sy, i, &e, &s_, &d);
    bool x_wrap = ((i + 1) % sy->L == 0);
    if (!(sy->lattice == SA_LATTICE_2D_OPEN_X && x_wrap) && jx[2 * i + 1] != jx[2 * e])
      return fail(SA_ERR_J_INCONSISTENT, "Jx[2i+1] != Jx[2(i+1)] at site " + std::to_string(i));
    if (jy[2 * i + 1] != jy[2 * s_])
      return fail(SA_ERR_J_INCONSISTENT, "Jy[2i+1] != Jy[2(i+L)] at site " + std::to_string(i));
    if (sy->dim == 3 && jz[2 * i + 1] != jz[2 * d])
      return fail(SA_ERR_J_INCONSISTENT, "Jz[2i+1] != Jz[2(i+L2)] at site " + std::to_string(i));
    long o = host_split(sy, i);
    own[o] = jx[2 * i];
    own[sy->N + o] = jy[2 * i];
    if (sy->dim == 3) own[2 * sy->N + o] = jz[2 * i];
  }
  SA_CUDA_TRY(cudaMemcpyAsync(sy->d_J, own.data(), own.size() * sizeof(word_t), cudaMemcpyHostToDevice,
                              sy->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  return SA_OK;
}

int sa_sys_get_J(sa_system_t sy, uint64_t* jx, uint64_t* jy, uint64_t* jz) {
  if (!sy || !jx || !jy || (sy->dim == 3 && !jz)) return fail(SA_ERR_INVALID, "null argument");
  std::vector<word_t> own((size_t)sy->dim * sy->N);
  SA_CUDA_TRY(cudaMemcpyAsync(own.data(), sy->d_J, own.size() * sizeof(word_t), cudaMemcpyDeviceToHost,
                              sy->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  for (long i = 0; i < sy->N; ++i) {
    long e, s_, d;
    nb_plus(sy, i, &e, &s_, &d);
    jx[2 * i] = own[host_split(sy, i)];
    jx[2 * i + 1] = own[host_split(sy, e)];
    jy[2 * i] = own[sy->N + host_split(sy, i)];
    jy[2 * i + 1] = own[sy->N + host_split(sy, s_)];
    if (sy->dim == 3) {
      jz[2 * i] = own[2 * sy->N + host_split(sy, i)];
      jz[2 * i + 1] = own[2 * sy->N + host_split(sy, d)];
    }
  }
  return SA_OK;
}

int sa_sys_sweep(sa_system_t sy, long nsweeps) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  if (nsweeps < 0) return fail(SA_ERR_INVALID, "nsweeps < 0");
  if (sy->rng_mode == SA_RNG_MT19937_64) {
    for (long k = 0; k < nsweeps; ++k) {
      int st = mt_sweep(sy);
      if (st) return st;
    }
    return SA_OK;
  }
  if (nsweeps >= kResidentMinSweeps && nsweeps <= 0x7FFFFFFF && resident_ok(sy)) {
    // long runs at zero field: one launch of the resident kernel
    const double T = sy->T;
    return resident_run(sy, &T, 1, (int)nsweeps, 0, nullptr, nullptr, nullptr);
  }
  const int c0 = sy->first_colour;
  const int per = sy->split ? 2 : 1;  // draws per site per half-sweep
  for (long k = 0; k < nsweeps; ++k) {
    launch_halfsweep(sy, c0, sy->draw);
    launch_halfsweep(sy, 1 - c0, sy->draw + per);
    sy->draw += 2 * per;
  }
  SA_CUDA_TRY(cudaGetLastError());
  return SA_OK;
}

int sa_sys_measure_async(sa_system_t sy, int64_t* d_E, int64_t* d_M) {
  if (!sy || !d_E || !d_M) return fail(SA_ERR_INVALID, "null argument");
  launch_measure(sy, d_E, d_M);
  SA_CUDA_TRY(cudaGetLastError());
  return SA_OK;
}

int sa_sys_measure(sa_system_t sy, int64_t* E, int64_t* M) {
  if (!sy || !E || !M) return fail(SA_ERR_INVALID, "null argument");
  launch_measure(sy, sy->d_EM, sy->d_EM + 64);
  SA_CUDA_TRY(cudaGetLastError());
  int64_t buf[128];
  SA_CUDA_TRY(cudaMemcpyAsync(buf, sy->d_EM, sizeof buf, cudaMemcpyDeviceToHost, sy->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  memcpy(E, buf, 64 * sizeof(int64_t));
  memcpy(M, buf + 64, 64 * sizeof(int64_t));
  return SA_OK;
}

int sa_sys_measure_float(sa_system_t sy, float* out) {
  if (!sy || !out) return fail(SA_ERR_INVALID, "null argument");
  int64_t E[64], M[64];
  int st = sa_sys_measure(sy, E, M);
  if (st) return st;
  for (int j = 0; j < 64; ++j) out[j] = (float)((double)E[j] + sy->h * (double)M[j]);
  return SA_OK;
}

int sa_sys_swap(sa_system_t a, sa_system_t b, uint64_t mask) {
  if (!a || !b) return fail(SA_ERR_INVALID, "null system");
  if (a->lattice != b->lattice || a->L != b->L) return fail(SA_ERR_MISMATCH, "systems differ in shape");
  if (a == b) return SA_OK;
  // b's queued work must finish before a's stream touches b's spins.
  if (a->stream != b->stream) {
    SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  }
  k_swap<<<grid_for(a->N, 256), 256, 0, a->stream>>>(a->d_s, b->d_s, mask, a->N);
  SA_CUDA_TRY(cudaGetLastError());
  if (a->stream != b->stream) SA_CUDA_TRY(cudaStreamSynchronize(a->stream));
  return SA_OK;
}

int sa_sys_get_N(sa_system_t sy, long* N) {
  if (!sy || !N) return fail(SA_ERR_INVALID, "null argument");
  *N = sy->N;
  return SA_OK;
}

int sa_sys_get_rng(sa_system_t sy, uint64_t* seed, uint64_t* draw, uint64_t* epoch) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  if (seed) *seed = sy->seed;
  if (draw) *draw = sy->draw;
  if (epoch) *epoch = sy->epoch;
  return SA_OK;
}

int sa_sys_set_rng(sa_system_t sy, uint64_t seed, uint64_t draw, uint64_t epoch) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  sy->seed = seed;
  sy->draw = draw;
  sy->epoch = epoch;
  return SA_OK;
}

int sa_sys_sync(sa_system_t sy) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  return SA_OK;
}

int sa_sys_device_buffers(sa_system_t sy, uint64_t** d_spins, uint64_t** d_J) {
  if (!sy) return fail(SA_ERR_INVALID, "null system");
  if (d_spins) *d_spins = (uint64_t*)sy->d_s;
  if (d_J) *d_J = (uint64_t*)sy->d_J;
  return SA_OK;
}

// Checkpoint: magic, version, lattice, L, T, h, seed, draw, epoch, then the
// internal spins (N words) and own couplings (dim*N words).
struct CkptHeader {
  char magic[8];
  int32_t version, lattice, L, pad;  // pad: bit 0 the first colour, bit 1 the split update
  double T, h;
  uint64_t seed, draw, epoch;
};

int sa_sys_save(sa_system_t sy, void* buf, size_t cap, size_t* len) {
  if (!sy || !len) return fail(SA_ERR_INVALID, "null argument");
  const size_t mt_bytes = (sy->rng_mode == SA_RNG_MT19937_64) ? (kMtN + 1) * sizeof(uint64_t) : 0;
  size_t need = sizeof(CkptHeader) + (size_t)(1 + sy->dim) * sy->N * sizeof(word_t) + mt_bytes;
  *len = need;
  if (!buf) return SA_OK;
  if (cap < need) return fail(SA_ERR_BUFFER, "checkpoint buffer too small");
  CkptHeader hd;
  memset(&hd, 0, sizeof hd);
  memcpy(hd.magic, "SAB200CK", 8);
  hd.version = mt_bytes ? 2 : 1;  // 2: mt19937_64 mode, generator state appended
  hd.pad = sy->first_colour | (sy->split << 1);  // 0 in records written before these existed
  hd.lattice = sy->lattice;
  hd.L = sy->L;
  hd.T = sy->T;
  hd.h = sy->h;
  hd.seed = sy->seed;
  hd.draw = sy->draw;
  hd.epoch = sy->epoch;
  char* p = (char*)buf;
  memcpy(p, &hd, sizeof hd);
  p += sizeof hd;
  SA_CUDA_TRY(cudaMemcpyAsync(p, sy->d_s, sy->N * sizeof(word_t), cudaMemcpyDeviceToHost, sy->stream));
  p += sy->N * sizeof(word_t);
  SA_CUDA_TRY(cudaMemcpyAsync(p, sy->d_J, (size_t)sy->dim * sy->N * sizeof(word_t),
                              cudaMemcpyDeviceToHost, sy->stream));
  p += (size_t)sy->dim * sy->N * sizeof(word_t);
  if (mt_bytes) SA_CUDA_TRY(cudaMemcpyAsync(p, sy->d_mt, mt_bytes, cudaMemcpyDeviceToHost, sy->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  return SA_OK;
}

int sa_sys_load(sa_system_t sy, const void* buf, size_t len) {
  if (!sy || !buf) return fail(SA_ERR_INVALID, "null argument");
  if (len < sizeof(CkptHeader)) return fail(SA_ERR_BUFFER, "checkpoint truncated");
  CkptHeader hd;
  memcpy(&hd, buf, sizeof hd);
  if (memcmp(hd.magic, "SAB200CK", 8) != 0 || (hd.version != 1 && hd.version != 2))
    return fail(SA_ERR_BUFFER, "not a checkpoint of this engine");
  if (hd.lattice != sy->lattice || hd.L != sy->L)
    return fail(SA_ERR_MISMATCH, "checkpoint is for another lattice shape");
  const bool mt = hd.version == 2;
  const size_t mt_bytes = mt ? (kMtN + 1) * sizeof(uint64_t) : 0;
  size_t need = sizeof(CkptHeader) + (size_t)(1 + sy->dim) * sy->N * sizeof(word_t) + mt_bytes;
  if (len < need) return fail(SA_ERR_BUFFER, "checkpoint truncated");
  Thresholds t;
  if (!(hd.T > 0) || !make_thresholds(sy->lattice, hd.T, hd.h, &t))
    return fail(SA_ERR_BUFFER, "checkpoint has a bad temperature");
  ThresholdsMT tm;
  if (mt && !make_thresholds_mt(sy->lattice, hd.T, hd.h, &tm))
    return fail(SA_ERR_BUFFER, "checkpoint has a bad temperature");
  if (mt && !sy->d_draws) SA_CUDA_TRY(cudaMalloc(&sy->d_draws, (size_t)sy->dim * sy->N * sizeof(uint64_t)));
  const char* p = (const char*)buf + sizeof hd;
  SA_CUDA_TRY(cudaMemcpyAsync(sy->d_s, p, sy->N * sizeof(word_t), cudaMemcpyHostToDevice, sy->stream));
  p += sy->N * sizeof(word_t);
  SA_CUDA_TRY(cudaMemcpyAsync(sy->d_J, p, (size_t)sy->dim * sy->N * sizeof(word_t),
                              cudaMemcpyHostToDevice, sy->stream));
  p += (size_t)sy->dim * sy->N * sizeof(word_t);
  if (mt) SA_CUDA_TRY(cudaMemcpyAsync(sy->d_mt, p, mt_bytes, cudaMemcpyHostToDevice, sy->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  sy->rng_mode = mt ? SA_RNG_MT19937_64 : SA_RNG_PHILOX;
  if (mt) sy->thr_mt = tm;
  sy->T = hd.T;
  sy->h = hd.h;
  sy->thr = t;
  sy->seed = hd.seed;
  sy->draw = hd.draw;
  sy->epoch = hd.epoch;
  sy->first_colour = ((hd.pad & 1) && !mt) ? 1 : 0;
  sy->split = ((hd.pad & 2) && !mt) ? 1 : 0;
  make_split_thresholds(sy->lattice, sy->T, sy->h, &sy->sthr);
  return SA_OK;
}

// ---- the reference CPU classes' checkpoint record (mt19937_64 mode) --------
// cpu_2dp::save / cpu_3d::save (src/cpu_2dp.cpp:444-456, src/cpu_3d.cpp:449-461)
// write, in this order: int L; double T; double h; s[N]; Jx[2N]; Jy[2N];
// (Jz[2N]); the std::mt19937_64 object (312 state words, then the size_t index
// of the next output -- libstdc++'s layout); uniform_real_distribution<double>
// (a, b); uniform_int_distribution<int> (a, b). Only the generator part has
// meaning here; the distributions are written as the reference sets them up.
static size_t ref_record_size(const sa_system* sy) {
  return sizeof(int32_t) + 2 * sizeof(double) + (size_t)sy->N * 8 + (size_t)sy->dim * 2 * sy->N * 8 +
         (kMtN + 1) * sizeof(uint64_t) + 2 * sizeof(double) + 2 * sizeof(int32_t);
}

int sa_sys_save_reference(sa_system_t sy, void* buf, size_t cap, size_t* len) {
  if (!sy || !len) return fail(SA_ERR_INVALID, "null argument");
  if (sy->rng_mode != SA_RNG_MT19937_64)
    return fail(SA_ERR_UNSUPPORTED, "the reference record holds an mt19937_64 generator: set that mode first");
  const size_t need = ref_record_size(sy);
  *len = need;
  if (!buf) return SA_OK;
  if (cap < need) return fail(SA_ERR_BUFFER, "buffer too small");
  std::vector<uint64_t> sp(sy->N), J[3];
  for (int a = 0; a < sy->dim; ++a) J[a].resize(2 * sy->N);
  int st = sa_sys_get_spins(sy, sp.data());
  if (st == SA_OK) st = sa_sys_get_J(sy, J[0].data(), J[1].data(), sy->dim == 3 ? J[2].data() : nullptr);
  if (st != SA_OK) return st;
  uint64_t mt[kMtN + 1];
  SA_CUDA_TRY(cudaMemcpyAsync(mt, sy->d_mt, sizeof mt, cudaMemcpyDeviceToHost, sy->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  char* p = (char*)buf;
  auto put = [&](const void* src, size_t n) {
    memcpy(p, src, n);
    p += n;
  };
  const int32_t L = sy->L;
  put(&L, sizeof L);
  put(&sy->T, sizeof(double));
  put(&sy->h, sizeof(double));
  put(sp.data(), sp.size() * 8);
  for (int a = 0; a < sy->dim; ++a) put(J[a].data(), J[a].size() * 8);
  put(mt, sizeof mt);
  const double ud[2] = {0.0, 1.0};
  const int32_t ui[2] = {0, (int32_t)(sy->N - 1)};
  put(ud, sizeof ud);
  put(ui, sizeof ui);
  return SA_OK;
}

int sa_sys_load_reference(sa_system_t sy, const void* buf, size_t len) {
  if (!sy || !buf) return fail(SA_ERR_INVALID, "null argument");
  if (len < ref_record_size(sy)) return fail(SA_ERR_BUFFER, "record truncated or for another lattice size");
  const char* p = (const char*)buf;
  auto get = [&](void* dst, size_t n) {
    memcpy(dst, p, n);
    p += n;
  };
  int32_t L;
  double T, h;
  get(&L, sizeof L);
  get(&T, sizeof T);
  get(&h, sizeof h);
  if (L != sy->L) return fail(SA_ERR_MISMATCH, "record is for another lattice size");
  std::vector<uint64_t> sp(sy->N), J[3];
  get(sp.data(), sp.size() * 8);
  for (int a = 0; a < sy->dim; ++a) {
    J[a].resize(2 * sy->N);
    get(J[a].data(), J[a].size() * 8);
  }
  uint64_t mt[kMtN + 1];
  get(mt, sizeof mt);
  if (mt[kMtN] > (uint64_t)kMtN) return fail(SA_ERR_BUFFER, "bad generator index in the record");
  int st = sa_sys_set_rng_mode(sy, SA_RNG_MT19937_64);
  if (st == SA_OK) st = sa_sys_set_h(sy, h);
  if (st == SA_OK) st = sa_sys_set_T(sy, T);
  if (st == SA_OK) st = sa_sys_set_J(sy, J[0].data(), J[1].data(), sy->dim == 3 ? J[2].data() : nullptr);
  if (st == SA_OK) st = sa_sys_set_spins(sy, sp.data());
  if (st != SA_OK) return st;
  SA_CUDA_TRY(cudaMemcpyAsync(sy->d_mt, mt, sizeof mt, cudaMemcpyHostToDevice, sy->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(sy->stream));
  return SA_OK;
}

}  // extern "C"
