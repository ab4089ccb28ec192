// sa_wide.cuh -- one single-slot 3D anneal instance spread over the whole GPU.
//
// A lattice alone on the device (the last long request of a serving run, a
// single system's schedule) leaves most SMs idle in the resident kernel: its
// cluster holds at most 16 CTAs. Here every column of one colour is a group of
// G lanes anywhere on the GPU, walking its z-chain in segments exactly as the
// resident segmented walk does (affine maps of the new spin below, composed by
// a shuffle scan), straight from global memory (the lattice and its couplings
// stay in L2). A sweep is three launches: the colour-0 half, the colour-1 half
// (columns of one colour depend only on the other colour and on their own
// column, so a launch needs no grid-wide barrier), and the end-of-sweep
// launch, which counts -H when the sweep is measured, folds it into the
// anneal record and advances the sweep counter. Sweep counter, draw index and
// step thresholds are read from device memory, so the launch sequence is the
// same for every sweep.
#pragma once

#include "sa_batch.hpp"
#include "sa_device.cuh"
#include "sa_resident.cuh"

namespace sa {

// Control block of one wide instance (device memory, one per wide group):
// the counters of the sweep being measured and a mirror of the instance's
// progress that every launch reads in one cache line.
struct WideCtl {
  unsigned cnt[64];   // satisfied bonds of the sweep being measured (zero between sweeps)
  unsigned ticket;    // blocks of the end-of-sweep launch done (zero between sweeps)
  unsigned pad;
  int64_t end;        // sweeps stop at this count (the run's, or the schedule's, end)
  int64_t sweeps;     // sweeps done (mirror of the instance state)
  uint64_t draw;      // next draw index (mirror)
  uint32_t th[8];     // acceptance thresholds of the current step
};

// Everything a wide launch needs, by value: the instance's geometry and
// buffers come from the host, so no launch starts with a chain of dependent
// loads (descriptor, state, thresholds) before its real work.
struct WideParams {
  InstState* st;
  WideCtl* ctl;
  word_t* S;            // the instance's spins, [colour][row][k]
  const word_t* J;      // its couplings, [axis][colour][row][k]
  const BThr* thr;      // its schedule's thresholds, one per step
  int64_t* step_rec;    // last measured -H at the end of every step, [state][step][64], or null
  int64_t half, N, nbonds, state_idx;
  uint64_t seed;
  int32_t L, sweeps_per_step, thr_count;
  int32_t mstride;      // measure every mstride sweeps of a step (0 = never)
};

constexpr int kWideThreads = 256;

// Lanes per column of the wide half-sweep: the largest power of two up to 32
// that leaves every segment at least two planes (at most four for L <= 64).
__host__ __device__ constexpr int wide_lanes(int L) {
  return L >= 64 ? 32 : L >= 32 ? 16 : L >= 16 ? 8 : L >= 8 ? 4 : L >= 4 ? 2 : 1;
}

// Half-sweep of colour c. Thread t serves column t / G (row-major (y, k) over
// the L x L/2 columns of the colour), segment t % G of its planes.
__global__ void __launch_bounds__(kWideThreads) k_wide_half(WideParams p, int c) {
  const WideCtl* ctl = p.ctl;
  const int64_t sweeps = ctl->sweeps;  // written only by the end-of-sweep launch
  if (sweeps >= ctl->end) return;      // the same for the whole grid
  const int L = p.L, hL = L >> 1;
  const int G = wide_lanes(L);
  const int lane = threadIdx.x & 31;
  const long gt = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long ncols = (long)L * hL;
  if ((gt & ~31L) / G >= ncols) return;  // whole warps past the last column
  const int g = lane % G, lead = lane - g;
  const long col = gt / G;
  const bool col_ok = col < ncols;  // lanes past the end read column 0 and store nothing
  const int cc = col_ok ? (int)col : 0;
  const int y = cc / hL, k = cc - y * hL;
  const int par = (c + y) & 1, xx = 2 * k + par;
  int kw, ke;
  x_neighbours(k, par, hL, kw, ke);
  const int yn = (y == 0) ? L - 1 : y - 1, ys = (y == L - 1) ? 0 : y + 1;
  const long zg = (long)L * hL;  // z stride of spins and couplings
  word_t* own = p.S + (long)c * p.half + (long)y * hL + k;
  const word_t* so = p.S + (long)(1 - c) * p.half;
  const word_t* pw = so + (long)y * hL + kw;
  const word_t* pe = so + (long)y * hL + ke;
  const word_t* pn = so + (long)yn * hL + k;
  const word_t* ps = so + (long)ys * hL + k;
  const word_t* Jxc = p.J + (long)(0 + c) * p.half;
  const word_t* Jxo = p.J + (long)(1 - c) * p.half;
  const word_t* Jyc = p.J + (long)(2 + c) * p.half;
  const word_t* Jyo = p.J + (long)(3 - c) * p.half;
  const word_t* Jzc = p.J + (long)(4 + c) * p.half;
  const long jo = (long)y * hL + k, je = (long)y * hL + ke, js = (long)ys * hL + k;
  uint32_t th[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) th[q] = ctl->th[q];
  const uint64_t draw = ctl->draw + c;
  const unsigned long long site0 = (unsigned long long)(xx + L * y), plane = (unsigned long long)L * L;
  // segment g: planes [z0, z0 + ls), sizes as even as L allows (ls >= 2)
  const int sbase = L / G, srem = L % G;
  const int ls = sbase + (g < srem ? 1 : 0);
  const int z0 = g * sbase + min(g, srem);
  // the old top spin: the chain's input below z = 0
  const word_t top = __shfl_sync(0xffffffffu, g == 0 ? own[(L - 1) * zg] : 0ULL, lead);
  word_t A[kSegMax], B[kSegMax];
  auto site_map = [&](int z, word_t sd, word_t& a, word_t& b) {
    const int zn = (z == L - 1) ? 0 : z + 1;
    const long zo = (long)z * zg;
    const word_t si = own[zo];
    const word_t sw = __ldg(pw + zo), se = __ldg(pe + zo), sn = __ldg(pn + zo), ss = __ldg(ps + zo);
    const word_t jw = __ldg(Jxc + jo + zo), jee = __ldg(Jxo + je + zo);
    const word_t jn = __ldg(Jyc + jo + zo), jss = __ldg(Jyo + js + zo);
    const word_t ju = __ldg(Jzc + jo + zo), jd = __ldg(Jzc + jo + (long)zn * zg);
    const uint32_t u = philox_draw(p.seed, site0 + plane * (unsigned)z, draw);
    word_t c0, c1, c2;
    count5(jw ^ sw ^ si, jee ^ se ^ si, jn ^ sn ^ si, jss ^ ss ^ si, jd ^ sd ^ si, c0, c1, c2);
    uint32_t m0, m1, m2;
    prefix_bits(u, th, m0, m1, m2);
    const uint32_t t = (m0 & 1u) | (m1 & 2u) | (m2 & 4u);
    const uint32_t t1 = t ? t - 1 : 0;
    const word_t lo = below(c0, c1, c2, m0, m1, m2);
    const word_t hi = below(c0, c1, c2, (t1 & 1u) ? ~0u : 0u, (t1 & 2u) ? ~0u : 0u, (t1 & 4u) ? ~0u : 0u);
    const word_t gg = ju ^ si;
    const word_t f0 = (gg & hi) | (~gg & lo);
    a = si ^ f0;
    b = lo ^ hi;
  };
  // first plane of every segment (z0 + 1 < L: segments hold >= 2 planes);
  // segment 0's gives the new z = 0 spin
  site_map(z0, own[(long)(z0 + 1) * zg], A[0], B[0]);
  const word_t first = __shfl_sync(0xffffffffu, A[0] ^ (top & B[0]), lead);
#pragma unroll
  for (int i = 1; i < kSegMax; ++i) {
    A[i] = 0;
    B[i] = 0;
    if (i < ls) {
      const int z = z0 + i;
      site_map(z, (z == L - 1) ? first : own[(long)(z + 1) * zg], A[i], B[i]);
    }
  }
  // segment map (first plane applied first), then an inclusive scan over g
  word_t SA = A[0], SB = B[0];
#pragma unroll
  for (int i = 1; i < kSegMax; ++i)
    if (i < ls) {
      SA = A[i] ^ (SA & B[i]);
      SB &= B[i];
    }
#pragma unroll 1
  for (int dd = 1; dd < G; dd <<= 1) {
    const word_t pA = __shfl_up_sync(0xffffffffu, SA, dd, G);
    const word_t pB = __shfl_up_sync(0xffffffffu, SB, dd, G);
    if (g >= dd) {
      SA = SA ^ (pA & SB);
      SB = pB & SB;
    }
  }
  // exclusive prefix (identity for g = 0) applied to the old top spin
  word_t EA = __shfl_up_sync(0xffffffffu, SA, 1, G), EB = __shfl_up_sync(0xffffffffu, SB, 1, G);
  if (g == 0) {
    EA = 0;
    EB = ~0ULL;
  }
  // every lane of the column has read its old words before the scan it fed
  __syncwarp();
  if (col_ok) {
    word_t v = EA ^ (top & EB);
#pragma unroll
    for (int i = 0; i < kSegMax; ++i)
      if (i < ls) {
        v = A[i] ^ (v & B[i]);
        own[(long)(z0 + i) * zg] = v;
      }
  }
}

// End of a sweep. A measured sweep's -H: every block counts the satisfied
// bonds of its sites (each bond once, from its site towards -x/-y/-z) and
// adds them to the control block; the last block to finish (ticket) folds the
// totals into the anneal record. That block then advances the sweep counter,
// the draw index and the step's thresholds for the next sweep's launches.
__global__ void __launch_bounds__(kWideThreads) k_wide_end(WideParams p) {
  __shared__ unsigned s_cnt[64];
  __shared__ int s_last;
  WideCtl* ctl = p.ctl;
  const int64_t sweeps = ctl->sweeps;
  if (sweeps >= ctl->end) return;  // the same for the whole grid: no ticket is taken
  const bool meas = p.mstride > 0 && (sweeps % p.sweeps_per_step) % p.mstride == 0;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 64) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  if (meas) {
    const int L = p.L, hL = L >> 1;
    const long half = p.half, plane = (long)L * hL;
    const word_t* S = p.S;
    const word_t* J = p.J;
    VCount<4> sm;
    VCount<16> big;
    sm.clear();
    big.clear();
    int it = 0;
    // a thread's count stays below 32 (at most 10 sites of 3 bonds: the host
    // sizes the grid for it), so five planes carry it and the warp sum widens
    // by one plane per level
#pragma unroll 2
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < p.N; t += (long)gridDim.x * blockDim.x) {
      const int c = t >= half ? 1 : 0;
      const long rem = t - (long)c * half;
      const long r = rem / hL;
      const int k = (int)(rem - r * hL);
      const int y = (int)(r % L), z = (int)(r / L);
      const int par = (c + y) & 1;
      int kw, ke;
      x_neighbours(k, par, hL, kw, ke);
      const word_t* Sc = S + (long)c * half;
      const word_t* So = S + (long)(1 - c) * half;
      const word_t si = Sc[rem];
      const long zb = (long)z * plane;
      const word_t w = __ldg(J + (long)(0 + c) * half + rem) ^ si ^ So[zb + (long)y * hL + kw];
      const word_t n = __ldg(J + (long)(2 + c) * half + rem) ^ si ^ So[zb + (long)wrap_dec(y, L) * hL + k];
      const word_t u = __ldg(J + (long)(4 + c) * half + rem) ^ si ^ Sc[(long)wrap_dec(z, L) * plane + (long)y * hL + k];
      add2_small(sm, w ^ n ^ u, (w & n) | (u & (w ^ n)));
      if (++it == 5) {  // <= 3 per site: the 4-plane counter stays below 16
        add_small_w<5>(big, sm);
        sm.clear();
        it = 0;
      }
    }
    add_small_w<5>(big, sm);
    warp_sum_grow<1, 5>(big);
    atomicAdd(&s_cnt[lane], big.count_of(lane));
    atomicAdd(&s_cnt[lane + 32], big.count_of(lane + 32));
    __syncthreads();
    if (threadIdx.x < 64 && s_cnt[threadIdx.x]) atomicAdd(ctl->cnt + threadIdx.x, s_cnt[threadIdx.x]);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&ctl->ticket, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  InstState* st = p.st;
  const int64_t s1 = sweeps + 1;
  if (threadIdx.x < 64) {
    const int j = threadIdx.x;
    int64_t elast = st->elast[j];
    if (meas) {
      const int64_t e = 2 * (int64_t)atomicExch(ctl->cnt + j, 0u) - p.nbonds;
      elast = e;
      st->elast[j] = e;
      st->emax[j] = (st->measured == 0) ? e : max(st->emax[j], e);
    }
    if (p.step_rec && s1 % p.sweeps_per_step == 0) {
      const int64_t stp = s1 / p.sweeps_per_step - 1;
      if (stp < p.thr_count) p.step_rec[(p.state_idx * p.thr_count + stp) * 64 + j] = elast;
    }
  }
  if (threadIdx.x >= 64 && threadIdx.x < 72) {
    int64_t sn = s1 / p.sweeps_per_step;
    if (sn > p.thr_count - 1) sn = p.thr_count - 1;
    ctl->th[threadIdx.x - 64] = p.thr[sn].dn[threadIdx.x - 64];
  }
  __syncthreads();  // st->measured has been read
  if (threadIdx.x == 0) {
    if (meas) st->measured += 1;
    st->sweeps = s1;
    st->draw += 2;
    ctl->sweeps = s1;
    ctl->draw += 2;
    ctl->ticket = 0;
  }
}

// Starts a run: the control block takes the instance's progress, the step's
// thresholds and the sweep count at which the run stops.
__global__ void k_wide_begin(WideParams p, int64_t end) {
  WideCtl* ctl = p.ctl;
  const int64_t sweeps = p.st->sweeps;
  int64_t s = sweeps / p.sweeps_per_step;
  if (s > p.thr_count - 1) s = p.thr_count - 1;
  if (threadIdx.x < 8) ctl->th[threadIdx.x] = p.thr[s].dn[threadIdx.x];
  if (threadIdx.x == 0) {
    ctl->end = end;
    ctl->sweeps = sweeps;
    ctl->draw = p.st->draw;
  }
}

}  // namespace sa
