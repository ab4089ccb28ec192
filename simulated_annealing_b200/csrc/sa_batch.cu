// sa_batch.cu -- the batched persistent engine.
//
// Thousands of instances (mixed 2D / 2D open-x / 3D, any even L), each an
// ensemble of up to 32 64-replica slots sharing couplings, advance in ONE
// persistent launch: a CTA takes an instance from a work queue and runs every
// sweep of the launch for all its slots, then the replica exchange
// (src/parallel_tempering.hpp:81-115) or the anneal bookkeeping
// (src/annealing.hpp:67-100), without leaving the kernel.
//
// Layout per instance: spins [colour][row][k][slot] (the slot innermost, so a
// warp's loads for a site group are contiguous), couplings [axis][colour][row][k]
// shared by all slots. A warp maps its lanes to (site, slot) with P lanes per
// site (P = next power of two >= nslots): the P slots of one site share the
// coupling words (one broadcast load) and ONE Philox draw -- every slot of an
// instance draws the same per-site stream, as the reference's slots do when its
// driver seeds them alike (src/main_gpu.cu:262-276) -- which the warp computes
// once per 32 sites and distributes with shuffles.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <random>
#include <string>
#include <vector>

#include "sa_b200.h"
#include "sa_b200_batch.h"
#include "sa_batch.hpp"
#include "sa_device.cuh"
#include "sa_host.hpp"
#include "sa_resident.cuh"
#include "sa_system.hpp"
#include "sa_wide.cuh"

namespace sa {

constexpr int kBatchThreads = 512;
constexpr unsigned kFull = 0xffffffffu;
constexpr int64_t kBatchMaxN = 1 << 18;  // counter width of the pair measure

struct LaneThr {
  uint32_t t[8];
  uint32_t b[8];
};

__device__ __forceinline__ void load_thr(LaneThr& lt, const BThr* src) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    lt.t[k] = src->dn[k];
    lt.b[k] = src->bdn[k];
  }
}

// ---------------------------------------------------------------------------
// Half-sweeps of one instance (all slots), colour c.
// ---------------------------------------------------------------------------
template <int P, bool OPEN_X>
__device__ __forceinline__ void bhalf_2d(const InstDesc& d, word_t* __restrict__ S,
                                         const word_t* __restrict__ J, int c, uint64_t draw,
                                         const LaneThr& th) {
  constexpr int SPS = 32 / P;  // sites per sub-step
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int L = d.L, hL = L >> 1, ns = d.nslots;
  const long half = d.half;
  const int slot = lane % P;
  const bool slot_ok = slot < ns;
  word_t* Sc = S + (long)c * half * ns;
  const word_t* So = S + (long)(1 - c) * half * ns;
  const word_t* Jxc = J + (long)(0 + c) * half;
  const word_t* Jxo = J + (long)(1 - c) * half;
  const word_t* Jyc = J + (long)(2 + c) * half;
  const word_t* Jyo = J + (long)(3 - c) * half;
  for (long base = (long)warp * 32; base < half; base += (long)nwarps * 32) {
    const long my = base + lane;
    uint32_t um = 0;
    if (my < half) {
      const int r = (int)(my / hL), k = (int)(my - (long)r * hL);
      const int x = 2 * k + ((c + r) & 1);
      um = philox_draw(d.seed, (unsigned long long)x + (unsigned long long)L * r, draw);
    }
#pragma unroll 1
    for (int sub = 0; sub < P; ++sub) {
      const int sl = sub * SPS + lane / P;
      const uint32_t u = __shfl_sync(kFull, um, sl);
      const long t = base + sl;
      if (t < half && slot_ok) {
        const int r = (int)(t / hL), k = (int)(t - (long)r * hL);
        const int par = (c + r) & 1, x = 2 * k + par;
        int kw, ke;
        x_neighbours(k, par, hL, kw, ke);
        const long rb = (long)r * hL;
        const long rn = (long)wrap_dec(r, L) * hL, rs = (long)wrap_inc(r, L) * hL;
        const word_t si = Sc[(rb + k) * ns + slot];
        word_t mw = Jxc[rb + k] ^ So[(rb + kw) * ns + slot] ^ si;
        word_t me = Jxo[rb + ke] ^ So[(rb + ke) * ns + slot] ^ si;
        const word_t mn = Jyc[rb + k] ^ So[(rn + k) * ns + slot] ^ si;
        const word_t ms = Jyo[rs + k] ^ So[(rs + k) * ns + slot] ^ si;
        bool border = false;
        if (OPEN_X) {
          if (x == 0) { mw = ~0ULL; border = true; }
          if (x == L - 1) { me = ~0ULL; border = true; }
        }
        word_t c0, c1, c2;
        count4(mw, me, mn, ms, c0, c1, c2);
        const uint32_t tt = (OPEN_X && border) ? prefix_count<4>(u, th.b) : prefix_count<4>(u, th.t);
        Sc[(rb + k) * ns + slot] = si ^ ~ge_scalar(c0, c1, c2, tt);
      }
    }
  }
}

template <int P>
__device__ __forceinline__ void bhalf_3d(const InstDesc& d, word_t* __restrict__ S,
                                         const word_t* __restrict__ J, int c, uint64_t draw,
                                         const LaneThr& th) {
  constexpr int SPS = 32 / P;  // columns per warp pass
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int L = d.L, hL = L >> 1, ns = d.nslots;
  const long half = d.half;
  const long cols = (long)L * hL;
  const int slot = lane % P, cl = lane / P;
  const bool slot_ok = slot < ns;
  word_t* Sc = S + (long)c * half * ns;
  const word_t* So = S + (long)(1 - c) * half * ns;
  const word_t* Jxc = J + (long)(0 + c) * half;
  const word_t* Jxo = J + (long)(1 - c) * half;
  const word_t* Jyc = J + (long)(2 + c) * half;
  const word_t* Jyo = J + (long)(3 - c) * half;
  const word_t* Jzc = J + (long)(4 + c) * half;
  const long plane = cols;  // rows*hL per z step = L*hL
  for (long cb = (long)warp * SPS; cb < cols; cb += (long)nwarps * SPS) {
    const long col = cb + cl;
    const bool col_ok = col < cols;
    const bool valid = col_ok && slot_ok;
    const int y = col_ok ? (int)(col / hL) : 0;
    const int k = col_ok ? (int)(col - (long)y * hL) : 0;
    const int par = (c + y) & 1, x = 2 * k + par;
    int kw, ke;
    x_neighbours(k, par, hL, kw, ke);
    const long yb = (long)y * hL, ynb = (long)wrap_dec(y, L) * hL, ysb = (long)wrap_inc(y, L) * hL;
    word_t prev = valid ? Sc[(yb + (long)(L - 1) * plane + k) * ns + slot] : 0;
    word_t first = 0;
    for (int z0 = 0; z0 < L; z0 += P) {
      const int zd = z0 + (lane % P);
      uint32_t um = 0;
      if (col_ok && zd < L)
        um = philox_draw(d.seed,
                         (unsigned long long)x + (unsigned long long)L * (unsigned long long)(y + (long)L * zd),
                         draw);
#pragma unroll 1
      for (int zi = 0; zi < P; ++zi) {
        const int z = z0 + zi;
        if (z >= L) break;  // warp-uniform
        const uint32_t u = __shfl_sync(kFull, um, cl * P + zi);
        if (valid) {
          const long zb = (long)z * plane;
          const long zdn = (z == L - 1) ? 0 : (long)(z + 1) * plane;
          const long idx = zb + yb + k;
          const word_t si = Sc[idx * ns + slot];
          const word_t sd = (z == L - 1) ? first : Sc[(zdn + yb + k) * ns + slot];
          const word_t mw = Jxc[idx] ^ So[(zb + yb + kw) * ns + slot] ^ si;
          const word_t me = Jxo[zb + yb + ke] ^ So[(zb + yb + ke) * ns + slot] ^ si;
          const word_t mn = Jyc[idx] ^ So[(zb + ynb + k) * ns + slot] ^ si;
          const word_t ms = Jyo[zb + ysb + k] ^ So[(zb + ysb + k) * ns + slot] ^ si;
          const word_t mu = Jzc[idx] ^ prev ^ si;
          const word_t md = Jzc[zdn + yb + k] ^ sd ^ si;
          word_t c0, c1, c2;
          count6(mw, me, mn, ms, mu, md, c0, c1, c2);
          const word_t nsw = si ^ ~ge_scalar(c0, c1, c2, prefix_count<6>(u, th.t));
          Sc[idx * ns + slot] = nsw;
          if (z == 0) first = nsw;
          prev = nsw;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Satisfied-bond counts per replica of slots a .. a+nsl-1 (nsl in {1,2}) into
// cnt[q][j]; every bond counted once from its site towards -x/-y/-z.
// ---------------------------------------------------------------------------
__device__ void measure_slots(const InstDesc& d, const word_t* __restrict__ S,
                              const word_t* __restrict__ J, int a, int nsl, unsigned (*cnt)[64]) {
  for (int i = threadIdx.x; i < 128; i += blockDim.x) (&cnt[0][0])[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int L = d.L, hL = L >> 1, ns = d.nslots;
  const long half = d.half, N = d.N;
  const bool d3 = d.lattice == SA_LATTICE_3D, open = d.lattice == SA_LATTICE_2D_OPEN_X;
  const int per = 32 / nsl;
  const int g = lane / nsl, slot = a + lane % nsl;
  const long plane = (long)L * hL;
  VCount<4> sm;
  VCount<16> big;
  sm.clear();
  big.clear();
  int it = 0;
  for (long base = (long)warp * per; base < N; base += (long)nwarps * per) {
    const long t = base + g;
    if (t < N) {
      const int c = t >= half ? 1 : 0;
      const long rem = t - (long)c * half;
      const long r = rem / hL;
      const int k = (int)(rem - r * hL);
      const int y = (int)(r % L), z = (int)(r / L);
      const int par = (c + y) & 1, x = 2 * k + par;
      int kw, ke;
      x_neighbours(k, par, hL, kw, ke);
      const word_t* Sc = S + (long)c * half * ns;
      const word_t* So = S + (long)(1 - c) * half * ns;
      const word_t si = Sc[rem * ns + slot];
      const long zb = (long)z * plane;
      word_t w = (open && x == 0) ? 0 : (J[(long)(0 + c) * half + rem] ^ si ^ So[(zb + (long)y * hL + kw) * ns + slot]);
      word_t n = J[(long)(2 + c) * half + rem] ^ si ^ So[(zb + (long)wrap_dec(y, L) * hL + k) * ns + slot];
      word_t q0, q1;
      if (d3) {
        word_t u = J[(long)(4 + c) * half + rem] ^ si ^ Sc[((long)wrap_dec(z, L) * plane + (long)y * hL + k) * ns + slot];
        q0 = w ^ n ^ u;
        q1 = (w & n) | (u & (w ^ n));
      } else {
        q0 = w ^ n;
        q1 = w & n;
      }
      add2_small(sm, q0, q1);
    }
    if (++it == 5) {  // <= 3 per site: the 4-plane counter stays below 16
      add_small(big, sm);
      sm.clear();
      it = 0;
    }
  }
  add_small(big, sm);
  big.warp_sum_from(nsl);
  const int q = lane % nsl;
  for (int m = 0; m < 2 * nsl; ++m) {
    const int j = (lane / nsl) + per * m;
    atomicAdd(&cnt[q][j], big.count_of(j));
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// The persistent kernel.
// ---------------------------------------------------------------------------
template <int P>
__device__ void run_instance(const BatchParams& p, const InstDesc& d, int id, unsigned (*cnt)[64],
                             unsigned* smask) {
  InstState* st = p.state + d.state_idx;
  uint64_t draw = st->draw;
  int64_t sweeps = st->sweeps, xsteps = st->xsteps;
  int64_t n = p.nsweeps;
  if (d.sweep_limit >= 0) n = min(n, d.sweep_limit - sweeps);
  if (n <= 0) return;
  word_t* S = p.spins + d.spin_off;
  const word_t* J = p.J + d.J_off;
  const int lane = threadIdx.x & 31;
  const int slot = lane % P;
  LaneThr th;
  int64_t step = -1;
  if (d.sched < 0) load_thr(th, p.thr + d.thr_off + (slot < d.nslots ? slot : 0));
  for (int64_t i = 0; i < n; ++i) {
    if (d.sched >= 0) {
      int64_t s = sweeps / d.sweeps_per_step;
      if (s > d.thr_count - 1) s = d.thr_count - 1;
      if (s != step) {
        step = s;
        load_thr(th, p.thr + d.thr_off + s);
      }
    }
    for (int c = 0; c < 2; ++c) {
      if (d.lattice == SA_LATTICE_3D) bhalf_3d<P>(d, S, J, c, draw + c, th);
      else if (d.lattice == SA_LATTICE_2D_OPEN_X) bhalf_2d<P, true>(d, S, J, c, draw + c, th);
      else bhalf_2d<P, false>(d, S, J, c, draw + c, th);
      __syncthreads();
    }
    draw += 2;
    const int64_t in_step = (d.sched >= 0) ? sweeps % d.sweeps_per_step : 0;
    sweeps += 1;
    if (d.ladder >= 0 && d.nslots > 1 && sweeps % p.xinterval == 0) {
      const Decision dc = p.dec[d.dec_off + xsteps];
      const int a = dc.pair;
      measure_slots(d, S, J, a, 2, cnt);
      if (threadIdx.x < 64) {
        const int j = threadIdx.x;
        const int64_t ea = 2 * (int64_t)cnt[0][j] - d.nbonds;
        const int64_t eb = 2 * (int64_t)cnt[1][j] - d.nbonds;
        const int64_t dE = eb - ea;
        const bool acc = dE >= dc.lo && dE <= dc.hi;
        const unsigned bal = __ballot_sync(kFull, acc);
        if (lane == 0) smask[threadIdx.x >> 5] = bal;
      }
      __syncthreads();
      const word_t mask = (word_t)smask[0] | ((word_t)smask[1] << 32);
      if (mask) {
        const int ns = d.nslots;
        for (long t = threadIdx.x; t < d.N; t += blockDim.x) {
          word_t* w = S + t * ns + a;
          const word_t x0 = w[0], x1 = w[1];
          const word_t dd = (x0 ^ x1) & mask;
          w[0] = x0 ^ dd;
          w[1] = x1 ^ dd;
        }
      }
      if (threadIdx.x == 0) {
        p.acc[d.pair_off + a] += __popcll(mask);
        p.att[d.pair_off + a] += 1;
        if (p.rec_pair && xsteps < p.rec_cap) {
          p.rec_pair[(long)id * p.rec_cap + xsteps] = a;
          p.rec_mask[(long)id * p.rec_cap + xsteps] = mask;
        }
      }
      xsteps += 1;
      __syncthreads();
    }
    if (d.sched >= 0 && p.mstride > 0 && in_step % p.mstride == 0) {
      measure_slots(d, S, J, 0, 1, cnt);
      if (threadIdx.x < 64) {
        const int j = threadIdx.x;
        const int64_t e = 2 * (int64_t)cnt[0][j] - d.nbonds;
        const int64_t m0 = st->measured;
        st->elast[j] = e;
        st->emax[j] = (m0 == 0) ? e : max(st->emax[j], e);
      }
      __syncthreads();
      if (threadIdx.x == 0) st->measured += 1;
      __syncthreads();
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    st->draw = draw;
    st->sweeps = sweeps;
    st->xsteps = xsteps;
  }
}

template <int P>
__global__ void __launch_bounds__(kBatchThreads, 1) k_batch(BatchParams p) {
  __shared__ int s_item;
  __shared__ unsigned s_cnt[2][64];
  __shared__ unsigned s_mask[2];
  __shared__ InstDesc s_d;
  for (;;) {
    if (threadIdx.x == 0) {
      s_item = atomicAdd(p.work, 1);
      if (s_item < p.ninst) s_d = p.inst[p.order[s_item]];
    }
    __syncthreads();
    const int item = s_item;
    if (item >= p.ninst) break;
    run_instance<P>(p, s_d, p.order[item], s_cnt, s_mask);
    __syncthreads();  // s_item / s_d are reused by the next round
  }
}

// ---------------------------------------------------------------------------
// Shared-memory-resident kernel: one cluster of C CTAs per instance.
// ---------------------------------------------------------------------------
// LAT: lattice kind of every instance of the launch; CL: clusters of more
// than one CTA (DSMEM halos and cluster barriers) or single CTAs (block
// barriers only).
// Single-slot 3D variants (segmented walk, fused measurement) hold more state
// per thread: 16 warps at up to 128 registers. Clustered two-slot 2D blocks:
// 8 warps, two blocks per SM.
template <int P, int SL, int LAT, bool CL, bool SEG, bool HR = false>
constexpr int res_max_threads() {
  return HR                                          ? kHiRegThreads
         : (LAT != SA_LATTICE_3D && SL == 2 && CL)   ? kRes2dClThreads
         : (SEG || (P == 1 && SL == 1 && LAT == SA_LATTICE_3D)) ? kSegMaxThreads
                                                                : kResMaxThreads;
}
template <int SL, int LAT, bool CL, bool HR>
constexpr int res_min_blocks() {
  return (!HR && LAT != SA_LATTICE_3D && SL == 2 && CL) ? 2 : 1;
}

// The host's cap on warps per block for a resident group, matching the
// kernel's launch bounds above.
static int res_warp_cap(int lattice, int SL, int RP, int C, bool hr, bool seg) {
  if (hr) return kHiRegThreads / 32;
  if (lattice != SA_LATTICE_3D && SL == 2 && C > 1) return kRes2dClThreads / 32;
  if (seg || (lattice == SA_LATTICE_3D && SL == 1 && RP == 1)) return kSegMaxThreads / 32;
  return kResMaxWarps;
}

// SEG: single-slot 3D instances spread over many SMs walk their columns in
// segments (rhalf_3d1s) instead of whole (rhalf_3d1).
// HR: the high-register form for two slots per lane in 3D: at most
// kHiRegThreads threads, so each can hold ~170 registers (a two-slot 3D walk
// keeps twice the words live; where a CTA has work for few warps anyway this
// trades nothing for no spills).
template <int P, int SL, int LAT, bool CL, bool SEG = false, bool HR = false>
__global__ void __launch_bounds__(res_max_threads<P, SL, LAT, CL, SEG, HR>(), res_min_blocks<SL, LAT, CL, HR>())
    k_resident(BatchParams p) {
  extern __shared__ __align__(16) word_t s_spins[];
  __shared__ unsigned s_cnt[2][64];   // this CTA's partial counts
  __shared__ unsigned s_mask[2];
  cg::cluster_group cluster = cg::this_cluster();
  const int C = CL ? (int)cluster.num_blocks() : 1;
  const int q = CL ? (int)cluster.block_rank() : 0;
  auto sync_all = [&]() {
    if (CL) cluster.sync();
    else __syncthreads();
  };
  const int id = p.order[blockIdx.x / C];
  const InstDesc d = p.inst[id];
  InstState* st = p.state + d.state_idx;
  const uint64_t draw0 = st->draw;
  const int64_t sweeps0 = st->sweeps, xsteps0 = st->xsteps;
  int64_t n = p.nsweeps;
  if (d.sweep_limit >= 0) n = min(n, d.sweep_limit - sweeps0);
  if (n <= 0) return;  // the whole cluster sees the same n

  ResCtx x;
  x.L = d.L;
  x.hL = d.L >> 1;
  x.ns = d.nslots;
  x.zc = (LAT == SA_LATTICE_3D) ? d.L : 1;
  {
    // rows split as evenly as L allows: the first L%C CTAs take one extra
    const int base = d.L / C, rem = d.L % C;
    auto rows_of = [&](int r) { return base + (r < rem ? 1 : 0); };
    x.ny = rows_of(q);
    x.y0 = q * base + min(q, rem);
    x.nyN = rows_of((q + C - 1) % C);
    x.nyS = rows_of((q + 1) % C);
  }
  x.rowW = x.hL * x.ns;
  x.half = (int)d.half;
  x.seed = d.seed;
  x.magic = (uint32_t)(0xFFFFFFFFu / (uint32_t)x.hL) + 1u;
  x.sm = s_spins;
  if (CL) {
    x.smN = cluster.map_shared_rank(s_spins, (unsigned)((q + C - 1) % C));
    x.smS = cluster.map_shared_rank(s_spins, (unsigned)((q + 1) % C));
    x.smNA = cluster_addr(smem_addr(s_spins), (unsigned)((q + C - 1) % C));
    x.smSA = cluster_addr(smem_addr(s_spins), (unsigned)((q + 1) % C));
  } else {
    x.smN = s_spins;
    x.smS = s_spins;
    x.smNA = x.smSA = smem_addr(s_spins);
  }
  x.J = p.J + d.J_off;
  const bool pow2 = (d.nslots & (d.nslots - 1)) == 0;
  x.swsh = SL - 1;
  x.swm = (pow2 && d.nslots > 1) ? ((d.nslots - 1) & ~(SL - 1)) : 0;
  const int lg_ns = __ffs(d.nslots) - 1;  // used only when swizzled (power-of-two slot count)
  // word i of a (colour, plane) block in the global order -> its swizzled place
  auto phys = [&](int i) -> int {
    if (!x.swm) return i;
    const int site = i >> lg_ns;
    return i ^ swz(x, site - div_hl(site, x) * x.hL);
  };
  constexpr bool d3 = LAT == SA_LATTICE_3D, open = LAT == SA_LATTICE_2D_OPEN_X;

  // global [colour][row = y + L*z][k][slot] -> local [colour][z][y_local][k][slot ^ swizzle]
  word_t* gS = p.spins + d.spin_off;
  const int blk = x.ny * x.rowW;
  for (int cz = 0; cz < 2 * x.zc; ++cz) {
    const int c = cz / x.zc, z = cz - c * x.zc;
    const word_t* src = gS + ((long)c * d.half + (long)(z * x.L + x.y0) * x.hL) * x.ns;
    word_t* dst = s_spins + (long)cz * blk;
    for (int i = threadIdx.x; i < blk; i += blockDim.x) dst[phys(i)] = src[i];
  }
  sync_all();

  const int lane = threadIdx.x & 31;
  const int slot = (lane % P) * SL;
  uint32_t th[SL][8], tb[SL][8];
  int64_t step = -1;
  if (d.sched < 0) {
#pragma unroll
    for (int q = 0; q < SL; ++q) {
      const BThr* t = p.thr + d.thr_off + (slot + q < d.nslots ? slot + q : 0);
#pragma unroll
      for (int k = 0; k < 8; ++k) { th[q][k] = t->dn[k]; tb[q][k] = t->bdn[k]; }
    }
  }
  uint64_t draw = draw0;
  int64_t sweeps = sweeps0, xsteps = xsteps0;
  // per-launch accumulators, written back once at the end: exchange counters
  // per pair (smem) and the anneal record (registers of threads 0..63 of rank 0)
  __shared__ int64_t s_acc[32], s_att[32];
  for (int t = threadIdx.x; t < 32; t += blockDim.x) s_acc[t] = s_att[t] = 0;
  int64_t my_emax = 0, my_elast = 0, measured = 0;
  if (d.sched >= 0 && q == 0 && threadIdx.x < 64) {
    my_emax = st->emax[threadIdx.x];
    my_elast = st->elast[threadIdx.x];
  }
  if (d.sched >= 0) measured = st->measured;
  // Fused measurement for single-slot 3D anneal instances walked whole: the
  // energy of a measured sweep is counted inside its colour-1 half and the
  // next sweep's colour-0 half (rhalf_3d1), then folded; only the last
  // measurement of a launch needs the separate pass. Each lane's count must
  // stay below 2048: columns per lane x (6L + 2) bonds, from the largest CTA.
  constexpr bool FUSE_T = (P == 1 && SL == 1 && LAT == SA_LATTICE_3D && !SEG);
  bool fuse = false;
  if constexpr (FUSE_T) {
    const long cols_max = (long)((d.L + C - 1) / C) * (d.L / 2);
    const long rounds = (cols_max + blockDim.x - 1) / blockDim.x;
    fuse = d.sched >= 0 && p.mstride > 0 && d.L > 4 && rounds * (6L * d.L + 2) < 2048;
  }
  BondCount bc;
  bc.clear();
  bool pending = false;     // a measured sweep whose colour-0 bonds are still to count
  int64_t rec_step = -1;    // its step, when it ended a step (the per-step record waits for it)
  // fold the counts in s_cnt (summed over the cluster) into the anneal record
  auto fold_counts = [&]() {
    sync_all();
    if (threadIdx.x < 64) {
      unsigned v = 0;
      if (CL) {
        for (int r = 0; r < C; ++r) v += cluster.map_shared_rank(&s_cnt[0][0], (unsigned)r)[threadIdx.x];
      } else {
        v = s_cnt[0][threadIdx.x];
      }
      if (q == 0) {
        const int64_t e = 2 * (int64_t)v - d.nbonds;
        my_elast = e;
        my_emax = (measured == 0) ? e : max(my_emax, e);
        if (rec_step >= 0 && p.step_rec && rec_step < d.thr_count)
          p.step_rec[((int64_t)d.state_idx * d.thr_count + rec_step) * 64 + threadIdx.x] = e;
      }
    }
    measured += 1;
    rec_step = -1;
    sync_all();  // every CTA has read s_cnt before it is cleared again
  };
  __syncthreads();
  for (int64_t i = 0; i < n; ++i) {
    // The exchange / measurement counters of this sweep start at zero. The
    // previous sweep's readers (every CTA of the cluster) finished before its
    // last cluster barrier, and this sweep's half-sweep barriers separate
    // these stores from the next counts.
    for (int t = threadIdx.x; t < 128; t += blockDim.x) (&s_cnt[0][0])[t] = 0;
    bool hist_now = false;  // a histogram pass used s_cnt in this sweep
    // this sweep's exchange decision, fetched before the half-sweeps hide its latency
    const bool xchg = d.ladder >= 0 && d.nslots > 1 && (sweeps + 1) % p.xinterval == 0;
    Decision dc = {0, 0, 0, 0};
    if (xchg) dc = p.dec[d.dec_off + xsteps];
    // 2D: each warp counts the pair's energies after its colour-1 walk
    // (rmeasure_own_2d), unless a histogram pass needs s_cnt first
    const bool own = !d3 && xchg && !(p.hist && d.hist_off >= 0 && (sweeps + 1) % p.hstride == 0);
    if (d.sched >= 0) {
      int64_t s = sweeps / d.sweeps_per_step;
      if (s > d.thr_count - 1) s = d.thr_count - 1;
      if (s != step) {
        step = s;
        const BThr* t = p.thr + d.thr_off + s;
#pragma unroll
        for (int q = 0; q < SL; ++q)
#pragma unroll
          for (int k = 0; k < 8; ++k) { th[q][k] = t->dn[k]; tb[q][k] = t->bdn[k]; }
      }
    }
    const bool meas_now = d.sched >= 0 && p.mstride > 0 && (sweeps % d.sweeps_per_step) % p.mstride == 0;
    for (int c = 0; c < 2; ++c) {
      if (fuse && c == 0 && pending)
        for (int t = threadIdx.x; t < 128; t += blockDim.x) (&s_cnt[0][0])[t] = 0;
      if (d3) {
        if constexpr (SEG) {
          rhalf_3d1s<CL>(x, c, draw + c, th[0]);
        } else if (P == 1 && SL == 1 && x.L > 4) {
          const int cmode = !fuse ? 0 : (c == 0 ? (pending ? 1 : 0) : (meas_now ? 2 : 0));
          rhalf_3d1<2, CL>(x, c, draw + c, th[0], &bc, cmode);
        } else {
          rhalf_3d<P, SL, CL, HR>(x, c, draw + c, th);
        }
      }
      else {
        rhalf_2d<P, SL, open, CL>(x, c, draw + c, th, tb);
        if (own && c == 1) rmeasure_own_2d<open, CL>(x, dc.pair, s_cnt);
      }
      sync_all();
      if (fuse && c == 0 && pending) {
        // the previous sweep's count is complete: reduce it over the CTA
        bc.flush();
        VCount<16> w;
#pragma unroll
        for (int b = 0; b < 16; ++b) w.p[b] = (b < 11) ? bc.big.p[b] : 0;
        w.warp_sum_from(1);
        atomicAdd(&s_cnt[0][lane], w.count_of(lane));
        atomicAdd(&s_cnt[0][lane + 32], w.count_of(lane + 32));
        bc.clear();
        fold_counts();
        pending = false;
      }
    }
    draw += 2;
    const int64_t in_step = (d.sched >= 0) ? sweeps % d.sweeps_per_step : 0;
    sweeps += 1;
    // energy histograms of every slot, taken before the exchange (the energies
    // the reference's PT step measures, src/parallel_tempering.hpp:85-95)
    if (p.hist && d.hist_off >= 0 && sweeps % p.hstride == 0) {
      hist_now = true;
      for (int a = 0; a < d.nslots; a += 2) {
        const int nh = (a + 1 < d.nslots) ? 2 : 1;
        rmeasure<CL>(x, d3, open, a, nh, s_cnt);
        sync_all();
        // a 64-thread CTA folds two slots in two rounds
        for (int t = threadIdx.x; q == 0 && t < 64 * nh; t += blockDim.x) {
          const int qq = t >> 6, j = t & 63;
          unsigned v = 0;
          if (CL) {
            for (int r = 0; r < C; ++r) v += cluster.map_shared_rank(&s_cnt[0][0], (unsigned)r)[qq * 64 + j];
          } else {
            v = s_cnt[qq][j];
          }
          // E = 2v - nbonds -> bin (E + nbonds) / 2 = v
          atomicAdd(&p.hist[d.hist_off + (long)(a + qq) * (d.nbonds + 1) + v], 1);
        }
        sync_all();
      }
    }
    bool meas = d.sched >= 0 && p.mstride > 0 && in_step % p.mstride == 0;
    if (fuse && meas) {
      pending = true;
      meas = false;
      if (sweeps % d.sweeps_per_step == 0) rec_step = sweeps / d.sweeps_per_step - 1;
    }
    if (xchg || meas) {
      int a = 0, nsl = 1;
      if (xchg) {
        a = dc.pair;
        nsl = 2;
      }
      // s_cnt was zeroed at the start of this sweep unless a histogram pass
      // used it since; four units' loads in flight per lane. The 2D pair
      // counts are already there (own): the barrier after the colour-1 half
      // made them complete.
      if (!own) {
        if (d3 && xchg) {
          // one counter of the pair's difference (rmeasure_pair_3d)
          if (hist_now) {
            for (int t = threadIdx.x; t < 128; t += blockDim.x) (&s_cnt[0][0])[t] = 0;
            __syncthreads();
          }
          rmeasure_pair_3d<CL>(x, a, s_cnt);
        } else {
          rmeasure<CL, 4>(x, d3, open, a, nsl, s_cnt, hist_now);
        }
        sync_all();
      }
      if (xchg) {
        // every CTA of the cluster reaches the same decision from the
        // cluster's totals: 64 threads, one replica each, then one barrier
        if (threadIdx.x < 64) {
          const int j = threadIdx.x;
          unsigned v0 = 0, v1 = 0;
          if (CL) {
            for (int r = 0; r < C; ++r) {
              const unsigned* rc = cluster.map_shared_rank(&s_cnt[0][0], (unsigned)r);
              v0 += rc[j];
              if (!(d3 || own)) v1 += rc[64 + j];
            }
          } else {
            v0 = s_cnt[0][j];
            v1 = s_cnt[1][j];
          }
          // v0 = the difference counter D of the pair (3D, and 2D counted per
          // warp): v(a+1) - v(a) = D - nbonds; else v0, v1 = the two slots'
          // satisfied-bond counts (2D sweeps with a histogram pass)
          const int64_t dv = (d3 || own) ? (int64_t)v0 - (int64_t)d.nbonds : (int64_t)v1 - (int64_t)v0;
          const int64_t dE = 2 * dv;
          const bool acc = dE >= dc.lo && dE <= dc.hi;
          const unsigned bal = __ballot_sync(0xffffffffu, acc);
          if (lane == 0) s_mask[threadIdx.x >> 5] = bal;
        }
        __syncthreads();
        const word_t mask = (word_t)s_mask[0] | ((word_t)s_mask[1] << 32);
        if (mask) {
          const int nloc = 2 * x.zc * x.ny * x.hL;
          for (int t = threadIdx.x; t < nloc; t += blockDim.x) {
            word_t* w = s_spins + (long)t * x.ns;
            const int sw = x.swm ? swz(x, t - div_hl(t, x) * x.hL) : 0;  // t % hL is the site's k
            const word_t x0 = w[a ^ sw], x1 = w[(a + 1) ^ sw];
            const word_t dd = (x0 ^ x1) & mask;
            w[a ^ sw] = x0 ^ dd;
            w[(a + 1) ^ sw] = x1 ^ dd;
          }
        }
        if (q == 0 && threadIdx.x == 0) {
          s_acc[a] += __popcll(mask);
          s_att[a] += 1;
          if (p.rec_pair && xsteps < p.rec_cap) {
            p.rec_pair[(long)id * p.rec_cap + xsteps] = a;
            p.rec_mask[(long)id * p.rec_cap + xsteps] = mask;
          }
        }
        xsteps += 1;
      } else if (q == 0 && threadIdx.x < 64) {
        unsigned v = 0;
        if (CL) {
          for (int r = 0; r < C; ++r) v += cluster.map_shared_rank(&s_cnt[0][0], (unsigned)r)[threadIdx.x];
        } else {
          v = s_cnt[0][threadIdx.x];
        }
        const int64_t e = 2 * (int64_t)v - d.nbonds;
        my_elast = e;
        my_emax = (measured == 0) ? e : max(my_emax, e);
      }
      sync_all();
      if (meas) measured += 1;
    }
    if (p.step_rec && d.sched >= 0 && q == 0 && threadIdx.x < 64 && sweeps % d.sweeps_per_step == 0 &&
        !pending) {
      const int64_t stp = sweeps / d.sweeps_per_step - 1;
      if (stp < d.thr_count) p.step_rec[((int64_t)d.state_idx * d.thr_count + stp) * 64 + threadIdx.x] = my_elast;
    }
  }
  if (pending) {
    // the launch's last measured sweep: count its energy with the separate pass
    rmeasure<CL>(x, d3, open, 0, 1, s_cnt);
    fold_counts();
    pending = false;
  }
  // local -> global
  for (int cz = 0; cz < 2 * x.zc; ++cz) {
    const int c = cz / x.zc, z = cz - c * x.zc;
    word_t* dst = gS + ((long)c * d.half + (long)(z * x.L + x.y0) * x.hL) * x.ns;
    const word_t* src = s_spins + (long)cz * blk;
    for (int i = threadIdx.x; i < blk; i += blockDim.x) dst[i] = src[phys(i)];
  }
  if (q == 0) {
    if (threadIdx.x == 0) {
      st->draw = draw;
      st->sweeps = sweeps;
      st->xsteps = xsteps;
      if (d.sched >= 0) st->measured = measured;
    }
    if (d.sched >= 0 && threadIdx.x < 64) {
      st->emax[threadIdx.x] = my_emax;
      st->elast[threadIdx.x] = my_elast;
    }
    if (d.ladder >= 0)
      for (int t = threadIdx.x; t < d.nslots - 1; t += blockDim.x) {
        p.acc[d.pair_off + t] += s_acc[t];
        p.att[d.pair_off + t] += s_att[t];
      }
  }
  sync_all();  // no CTA leaves while a peer may still read its shared memory
}

// ---------------------------------------------------------------------------
// Set-up kernels: couplings from seed_J (draws 0..2*dim-1, src/random.cu:25-35)
// and spins (engine init, epoch 0) copied into every slot.
// ---------------------------------------------------------------------------
__device__ void init_site(const InstDesc& d, uint64_t sj, long i, word_t* spins, word_t* J) {
  const int L = d.L, hL = L >> 1, dim = d.lattice == SA_LATTICE_3D ? 3 : 2;
  const long r = i / L;
  const int x = (int)(i - r * L), y = (int)(r % L), c = (x + y) & 1;
  const long rem = r * hL + (x >> 1);
  uint4x b0 = philox10(0, 0, (uint32_t)i, (uint32_t)((uint64_t)i >> 32), (uint32_t)sj, (uint32_t)(sj >> 32));
  uint4x b1 = philox10(1, 0, (uint32_t)i, (uint32_t)((uint64_t)i >> 32), (uint32_t)sj, (uint32_t)(sj >> 32));
  const uint32_t dr[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
  word_t* Jd = J + d.J_off;
  for (int a = 0; a < dim; ++a)
    Jd[(long)(2 * a + c) * d.half + rem] = (word_t)dr[2 * a] | ((word_t)dr[2 * a + 1] << 32);
  uint4x s = philox10(0, 0, (uint32_t)i, 0x80000000u | (uint32_t)((uint64_t)i >> 32), (uint32_t)d.seed,
                      (uint32_t)(d.seed >> 32));
  const word_t w = (word_t)s.x | ((word_t)s.y << 32);
  word_t* Sd = spins + d.spin_off + ((long)c * d.half + rem) * d.nslots;
  for (int q = 0; q < d.nslots; ++q) Sd[q] = w;
}

__global__ void k_batch_init(const InstDesc* inst, const uint64_t* seed_J, int ninst, word_t* spins, word_t* J) {
  for (int id = blockIdx.y; id < ninst; id += gridDim.y) {
    const InstDesc d = inst[id];
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.N) init_site(d, seed_J[id], i, spins, J);
  }
}

__global__ void k_batch_gather(const word_t* spins, const InstDesc* inst, int id, int slot, word_t* out) {
  const InstDesc d = inst[id];
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  const int L = d.L, hL = L >> 1;
  const long r = i / L;
  const int x = (int)(i - r * L), y = (int)(r % L), c = (x + y) & 1;
  out[i] = spins[d.spin_off + ((long)c * d.half + r * hL + (x >> 1)) * d.nslots + slot];
}

__global__ void k_batch_measure_one(BatchParams p, int id, int slot, int64_t* E) {
  __shared__ unsigned s_cnt[2][64];
  const InstDesc d = p.inst[id];
  measure_slots(d, p.spins + d.spin_off, p.J + d.J_off, slot, 1, s_cnt);
  if (threadIdx.x < 64) E[threadIdx.x] = 2 * (int64_t)s_cnt[0][threadIdx.x] - d.nbonds;
}

// Energies of every slot of every instance: one block per instance, slots
// measured two at a time; out[e_off + slot*64 + j].
__global__ void __launch_bounds__(kBatchThreads) k_batch_energies(BatchParams p, const int64_t* e_off,
                                                                   int64_t* out) {
  __shared__ unsigned s_cnt[2][64];
  const int id = blockIdx.x;
  const InstDesc d = p.inst[id];
  for (int a = 0; a < d.nslots; a += 2) {
    const int nsl = (a + 1 < d.nslots) ? 2 : 1;
    measure_slots(d, p.spins + d.spin_off, p.J + d.J_off, a, nsl, s_cnt);
    if (threadIdx.x < 64 * nsl) {
      const int q = threadIdx.x >> 6, j = threadIdx.x & 63;
      out[e_off[id] + (long)(a + q) * 64 + j] = 2 * (int64_t)s_cnt[q][j] - d.nbonds;
    }
    __syncthreads();
  }
}

}  // namespace sa

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
using namespace sa;

struct Ladder {
  std::vector<double> T;
  std::mt19937 gen{123};
  std::uniform_int_distribution<int> uni_int;
  std::uniform_real_distribution<double> uni_double{0., 1.};
  std::vector<Decision> dec;
  int64_t span = 0;
  int64_t dec_off = 0;   // device segment start
  int64_t cap = 0;       // device segment capacity
  int64_t uploaded = 0;  // entries already on the device
};

struct Schedule {
  std::vector<double> T;
  int sweeps_per_step = 1;
};

struct sa_batch {
  int device = 0;
  bool finalized = false;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  std::vector<Ladder> ladders;
  std::vector<Schedule> scheds;
  std::vector<InstDesc> inst;
  std::vector<uint64_t> seed_J;
  std::vector<int64_t> h_sweeps, h_xsteps;  // host mirrors of the device counters
  int xinterval = 1, mstride = 1;
  long rec_cap = 0;
  int64_t site_slots = 0;
  // device
  InstDesc* d_inst = nullptr;
  InstState* d_state = nullptr;
  int32_t* d_order = nullptr;
  std::vector<int32_t> h_order;  // the work order of the last finalize (host copy)
  int32_t* d_work = nullptr;
  word_t* d_spins = nullptr;
  word_t* d_J = nullptr;
  BThr* d_thr = nullptr;
  Decision* d_dec = nullptr;
  int64_t dec_cap = 0;
  int64_t* d_acc = nullptr;
  int64_t* d_att = nullptr;
  int32_t* d_rec_pair = nullptr;
  uint64_t* d_rec_mask = nullptr;
  word_t* d_stage = nullptr;
  int64_t* d_E = nullptr;
  int64_t npairs = 0;
  Decision* h_dec = nullptr;  // pinned staging for decision uploads
  int64_t h_dec_cap = 0;
  int64_t h2d_bytes_last = 0;  // host->device bytes of the last sa_batch_run
  int64_t* d_Eall = nullptr;   // all-slot energies
  size_t inst_cap = 0;         // serving: capacity of d_inst / d_order / d_seedJ
  size_t work_cap = 0;         // serving: capacity of d_work
  uint64_t* d_seedJ = nullptr; // serving: seeds of the requests being initialised
  int64_t e_count = 0;         // sum of nslots*64
  bool force_global = false;   // run every instance in the global-memory kernel
  bool no_wide = false;        // never run an instance wide (sa_wide.cuh)
  bool no_spread = false;      // keep full-batch launch shapes even when SMs sit idle
  bool group_timing = false;   // fork / done events with timing (sa_batch_group_times)
  std::vector<TuneEntry> tuning;  // launch shapes per bucket (empty: the built-in table)
  bool tuning_set = false;
  int hstride = 0;             // energy histograms every hstride sweeps (0 = off)
  int32_t* d_hist = nullptr;
  int64_t hist_count = 0;
  // Launch groups: a contiguous range of the work order sharing the kernel
  // (resident or global), the lanes-per-site P and the cluster size C.
  struct Group {
    bool resident;
    int P, C, begin, count, grid;
    size_t smem;
    int threads;        // resident: block size matched to the shape's work
    int lattice, L;     // resident groups hold one shape each
    int SL, RP;         // resident: slots per lane and lanes per site
    bool seg;           // resident: single-slot 3D walked in column segments
    bool hr;            // resident: the high-register launch bound (two slots per lane, 3D)
    const TuneEntry* tune;  // resident: the bucket's tuned shape, or null (heuristic shape)
    bool wide;          // one single-slot 3D anneal spread over the whole GPU (sa_wide.cuh)
    int wide_id;        // wide: the instance
    int wide_slot;      // wide: its scratch block in d_wide
    cudaStream_t stream;
    cudaEvent_t done;
  };
  std::vector<Group> groups;
  cudaEvent_t fork = nullptr;
  std::vector<int> cluster_of;  // per instance: C (0 = global-memory kernel)
  bool spread = false;          // clusters were enlarged to use idle SMs
  std::vector<int64_t> run_start;  // per instance: sweeps done when the current run began
  char* d_wide = nullptr;          // scratch of the wide groups, kWideScratch bytes each
  int wide_cap = 0;                // wide groups the scratch holds
  // CUDA graphs of kWideGraphSweeps wide sweeps, by launch parameters
  struct WideGraph {
    WideParams wp;
    unsigned hgrid, egrid;
    cudaGraphExec_t exec;
  };
  std::vector<WideGraph> wide_graphs;  // destroyed with the batch, after its streams are idle
  sa_batch() = default;
  sa_batch(const sa_batch&) = delete;
  sa_batch& operator=(const sa_batch&) = delete;
  ~sa_batch() {
    for (auto& w : wide_graphs) cudaGraphExecDestroy(w.exec);
  }
};

// Per wide group: its control block (WideCtl).
constexpr size_t kWideScratch = 512;
static_assert(sizeof(WideCtl) <= kWideScratch, "wide control block");
// Sweeps per CUDA graph of the wide form (three kernel nodes each); a run
// replays it and launches the remainder directly.
constexpr int kWideGraphSweeps = 25;
// Wide-form graphs a batch keeps (one per distinct launch parameters).
constexpr size_t kWideGraphCache = 32;
// 3D L from which a single-slot anneal runs wide when the batch leaves SMs
// idle (spread). Alone, per sweep: L=40 34.3 -> 20.6 us, L=48 50.8 -> 23.5,
// L=64 98.7 -> 29.8; L=32 stays on its cluster (15.4 against 22.1 wide). In a
// full batch the resident form stays: the wide launches are latency-bound and
// take SM time from the rest (a backlog-bound stream of 2,000 serving
// requests fell from 1426 to 1233 attempts/ns with them).
constexpr int kWideMinL = 40;

// Shared-memory budget of one CTA of the resident kernel: the 227 KB opt-in
// limit minus room for its static arrays (counters, per-warp planes).
constexpr size_t kResSmemBudget = 232448 - 8192;

// Smallest cluster size C dividing L whose per-CTA share of the instance's
// spins fits the budget; 0 if none does (the instance then runs in the
// global-memory kernel).
// Shared-memory bytes of the largest CTA when an instance's y-rows are split
// over C CTAs (ceil(L/C) rows of every z-plane and both colours).
static size_t resident_bytes(const InstDesc& d, int C) {
  const int zc = (d.lattice == SA_LATTICE_3D) ? d.L : 1;
  const int ny = (d.L + C - 1) / C;
  return (size_t)2 * zc * ny * (d.L / 2) * d.nslots * sizeof(word_t);
}

// Smallest cluster whose CTAs hold their share of the instance in shared
// memory; 0 = too large (the instance streams from global memory instead).
static int choose_cluster(const InstDesc& d) {
  static const int cands[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16};
  for (int C : cands) {
    if (C > d.L) break;
    if (resident_bytes(d, C) <= kResSmemBudget) return C;
  }
  return 0;
}

template <int P>
static int launch_group(sa_batch* b, const sa_batch::Group& g, int gi, long nsweeps);

static std::vector<int32_t> build_groups(sa_batch* b);

static BThr to_bthr(int lattice, double T) {
  Thresholds t;
  make_thresholds(lattice, T, 0.0, &t);
  BThr b;
  memcpy(b.dn, t.dn, sizeof b.dn);
  memcpy(b.bdn, t.bdn, sizeof b.bdn);
  return b;
}

static int batch_params(sa_batch* b, long nsweeps, BatchParams* p) {
  p->inst = b->d_inst;
  p->state = b->d_state;
  p->order = b->d_order;
  p->ninst = (int32_t)b->inst.size();
  p->work = b->d_work;
  p->spins = b->d_spins;
  p->J = b->d_J;
  p->thr = b->d_thr;
  p->dec = b->d_dec;
  p->acc = b->d_acc;
  p->att = b->d_att;
  p->rec_pair = b->d_rec_pair;
  p->rec_mask = b->d_rec_mask;
  p->rec_cap = b->rec_cap;
  p->nsweeps = nsweeps;
  p->xinterval = b->xinterval;
  p->mstride = b->mstride;
  p->hist = b->d_hist;
  p->hstride = b->hstride > 0 ? b->hstride : 1;
  p->step_rec = nullptr;
  return SA_OK;
}

// Work order and launch groups of the current instance table: grouped by
// (kernel, lanes-per-site, cluster size, shape), most expensive first.
// A batch whose smallest clusters leave SMs idle (a few large instances: one
// PT ensemble, the last requests of a serving run) gets larger clusters, so
// each instance's rows are shared by more SMs: every cluster size is scaled by
// the idle factor, up to 16 CTAs and one y-row per CTA.
static void spread_clusters(sa_batch* b) {
  static const int cands[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16};
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  long total = 0;
  for (int C : b->cluster_of) total += C;
  b->spread = false;
  if (total == 0 || total * 2 > sms) return;
  b->spread = true;
  const long factor = sms / total;
  for (size_t i = 0; i < b->inst.size(); ++i) {
    const int C0 = b->cluster_of[i];
    if (C0 == 0) continue;
    const long want = std::min<long>((long)C0 * factor, std::min(16, b->inst[i].L));
    int best = C0;
    for (int C : cands)
      if (C <= want && C > best) best = C;
    b->cluster_of[i] = best;
  }
}

// The tuned launch shapes compiled into the library (sa_tuning.inc, written
// by simulated_annealing_b200/autotune.py from timings on a B200).
static const TuneEntry kBuiltinTuning[] = {
#include "sa_tuning.inc"
    {-1, 0, 0, 0, 0, 0, 0}};

static const std::vector<TuneEntry>& builtin_tuning() {
  static const std::vector<TuneEntry> t = [] {
    std::vector<TuneEntry> v;
    for (const TuneEntry& e : kBuiltinTuning)
      if (e.lattice >= 0) v.push_back(e);
    return v;
  }();
  return t;
}

// A tuned shape usable for instance d at cluster size C (the shape's C fits
// the shared-memory budget, SL = 2 only for an even slot count, two warps at
// least); else null.
static const TuneEntry* tune_for(const sa_batch* b, const InstDesc& d) {
  const std::vector<TuneEntry>& t = b->tuning_set ? b->tuning : builtin_tuning();
  for (const TuneEntry& e : t) {
    if (e.lattice != d.lattice || e.L != d.L || e.nslots != d.nslots) continue;
    if (e.C < 1 || e.C > std::min(16, d.L) || resident_bytes(d, e.C) > kResSmemBudget) return nullptr;
    if (e.SL != 1 && (e.SL != 2 || d.nslots % 2 != 0)) return nullptr;
    // threads 0..63 of a resident CTA hold one replica each (anneal record,
    // exchange decision): two warps at least
    if (e.warps < 2) return nullptr;
    return &e;
  }
  return nullptr;
}

static std::vector<int32_t> build_groups(sa_batch* b) {
  // work order: grouped by (kernel, P, C), most expensive first inside a group
  b->cluster_of.resize(b->inst.size());
  for (size_t i = 0; i < b->inst.size(); ++i) b->cluster_of[i] = b->force_global ? 0 : choose_cluster(b->inst[i]);
  if (b->no_spread) b->spread = false;
  else spread_clusters(b);
  // full batches take the tuned cluster size of their bucket
  if (!b->spread)
    for (size_t i = 0; i < b->inst.size(); ++i)
      if (b->cluster_of[i] != 0)
        if (const TuneEntry* e = tune_for(b, b->inst[i])) b->cluster_of[i] = e->C;
  std::vector<int32_t> order(b->inst.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int32_t)i;
  std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
    const InstDesc &dx = b->inst[x], &dy = b->inst[y];
    const int cx = b->cluster_of[x], cy = b->cluster_of[y];
    if ((cx == 0) != (cy == 0)) return cx != 0;
    if (dx.P != dy.P) return dx.P < dy.P;
    if (cx != cy) return cx > cy;
    if (cx != 0 && (dx.lattice != dy.lattice || dx.L != dy.L))
      return dx.N * dx.nslots != dy.N * dy.nslots ? dx.N * dx.nslots > dy.N * dy.nslots
                                                  : (dx.lattice != dy.lattice ? dx.lattice < dy.lattice : dx.L < dy.L);
    return dx.N * dx.nslots > dy.N * dy.nslots;
  });
  b->groups.clear();
  for (size_t i = 0; i < order.size(); ++i) {
    const InstDesc& d = b->inst[order[i]];
    const int C = b->cluster_of[order[i]];
    const size_t smem = C ? resident_bytes(d, C) : 0;
    // Spread single-slot 3D instances walk columns in segments when a CTA's
    // columns x lanes fit in at most three passes of the block: there the
    // chained walk is latency-bound; beyond that it is throughput-bound and the
    // segments' extra map and scan work costs more than it saves (measured:
    // 3D L=32 on 16 CTAs 49.8 -> 17.2 us per sweep, L=64 97.6 -> 136.7).
    // A single-slot 3D anneal of L >= kWideMinL with the GPU nearly to itself
    // leaves even a 16-CTA cluster latency-bound; it runs wide, over the GPU.
    const bool wide = C != 0 && b->spread && d.lattice == SA_LATTICE_3D && d.nslots == 1 && d.sched >= 0 &&
                      !b->no_wide && d.L >= kWideMinL;
    bool seg = C != 0 && b->spread && d.lattice == SA_LATTICE_3D && d.nslots == 1 && d.L > 4 && !wide;
    if (seg) {
      const long lanes = (long)((d.L + C - 1) / C) * (d.L / 2) * seg_lanes(d.L);
      seg = (lanes + kSegMaxThreads - 1) / kSegMaxThreads <= 3;
    }
    const TuneEntry* te = (!b->spread && C != 0 && !wide && !seg) ? tune_for(b, d) : nullptr;
    if (te && te->C != C) te = nullptr;
    const bool same = !wide && !b->groups.empty() && !b->groups.back().wide &&
                      b->groups.back().resident == (C != 0) && b->groups.back().P == d.P &&
                      b->groups.back().C == C && b->groups.back().seg == seg &&
                      b->groups.back().tune == te &&
                      (C == 0 || (b->groups.back().lattice == d.lattice && b->groups.back().L == d.L));
    if (!same) {
      sa_batch::Group g{};
      g.resident = C != 0 && !wide;
      g.wide = wide;
      g.wide_id = wide ? order[i] : -1;
      g.P = d.P;
      g.C = C;
      g.begin = (int)i;
      g.lattice = d.lattice;
      g.L = d.L;
      g.threads = kBatchThreads;
      g.SL = 1;
      g.RP = d.P;
      g.seg = seg;
      g.hr = false;
      g.tune = te;
      if (te) {
        // the bucket's tuned shape
        g.SL = te->SL;
        g.RP = 1;
        while (g.RP * g.SL < d.nslots) g.RP <<= 1;
        g.hr = te->SL == 2 && te->hr && d.lattice == SA_LATTICE_3D;
        const int wmax = res_warp_cap(d.lattice, g.SL, g.RP, C, g.hr, false);
        g.threads = 32 * std::max(2, std::min(te->warps, wmax));
      } else if (C && !wide) {
        // warp passes of one half-sweep: 3D walks columns, 32/RP per pass; 2D
        // takes tiles of 32 sites (RP sub-steps of 32/RP sites each). Two slots
        // per lane (16-byte accesses, shared addressing and couplings) when the
        // slot count is even and there is still work for >= 12 warps.
        const int ny = (d.L + C - 1) / C, hL = d.L / 2;
        auto passes_for = [&](int rp) {
          if (seg) {
            // seg_lanes(L) lanes per column
            const int cpw = 32 / seg_lanes(d.L);
            return (ny * hL + cpw - 1) / cpw;
          }
          return (d.lattice == SA_LATTICE_3D) ? (ny * hL + (32 / rp) - 1) / (32 / rp) : (ny * hL + 31) / 32;
        };
        if (d.nslots % 2 == 0) {
          int rp2 = 1;
          while (rp2 * 2 < d.nslots) rp2 <<= 1;
          const int p2 = (d.lattice == SA_LATTICE_3D) ? passes_for(rp2) : passes_for(rp2) * rp2 / d.P;
          if (p2 >= 12 || d.lattice != SA_LATTICE_3D) {
            g.SL = 2;
            g.RP = rp2;
          }
        }
        const int passes = passes_for(g.RP);
        const int wmax = res_warp_cap(d.lattice, g.SL, g.RP, C, false, seg);
        int warps = std::min(passes, wmax);
        const int rounds = (passes + warps - 1) / warps;
        warps = std::max(4, (passes + rounds - 1) / rounds);
        if (d.nslots == 1 && smem >= 64 * 1024) {
          // single-slot instances that occupy an SM alone are measured after
          // every sweep: give the measurement pass (one unit = 32 sites of one
          // colour and plane) at least ~4 units per warp of parallelism
          const int units = 2 * ((d.lattice == SA_LATTICE_3D) ? d.L : 1) * ((ny * hL + 31) / 32);
          warps = std::max(warps, std::min(wmax, (units + 3) / 4));
        }
        g.threads = warps * 32;
      }
      b->groups.push_back(g);
    }
    sa_batch::Group& g = b->groups.back();
    g.count += 1;
    if (!wide) g.smem = std::max(g.smem, smem);
  }
  int nw = 0;
  for (auto& g : b->groups)
    if (g.wide) g.wide_slot = nw++;
  return order;
}

// Scratch for the wide groups of the current table (zeroed when allocated;
// the launches leave it zeroed after every sweep).
static int ensure_wide_scratch(sa_batch* b) {
  int nw = 0;
  for (const auto& g : b->groups) nw += g.wide ? 1 : 0;
  if (nw <= b->wide_cap) return SA_OK;
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  cudaFree(b->d_wide);
  b->d_wide = nullptr;
  b->wide_cap = std::max(nw, 2 * b->wide_cap);
  SA_CUDA_TRY(cudaMalloc(&b->d_wide, (size_t)b->wide_cap * kWideScratch));
  SA_CUDA_TRY(cudaMemsetAsync(b->d_wide, 0, (size_t)b->wide_cap * kWideScratch, b->stream));
  return SA_OK;
}

// The sweeps of this run for a wide group: three launches per sweep on the
// group's stream (the two half-sweeps and the end-of-sweep measurement).
static int launch_wide(sa_batch* b, const sa_batch::Group& g, long nsweeps, int64_t* step_rec) {
  const int id = g.wide_id;
  const InstDesc& d = b->inst[id];
  const int64_t start = (id < (int)b->run_start.size()) ? b->run_start[id] : 0;
  int64_t end = start + nsweeps;
  if (d.sweep_limit >= 0) end = std::min<int64_t>(end, d.sweep_limit);
  if (end <= start) return SA_OK;
  WideParams wp;
  memset(&wp, 0, sizeof wp);  // compared bytewise by the graph cache
  wp.st = b->d_state + d.state_idx;
  wp.ctl = reinterpret_cast<WideCtl*>(b->d_wide + (size_t)g.wide_slot * kWideScratch);
  wp.S = b->d_spins + d.spin_off;
  wp.J = b->d_J + d.J_off;
  wp.thr = b->d_thr + d.thr_off;
  wp.step_rec = step_rec;
  wp.half = d.half;
  wp.N = d.N;
  wp.nbonds = d.nbonds;
  wp.state_idx = d.state_idx;
  wp.seed = d.seed;
  wp.L = d.L;
  wp.sweeps_per_step = d.sweeps_per_step;
  wp.thr_count = d.thr_count;
  wp.mstride = b->mstride;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  const long threads = (long)d.L * (d.L / 2) * wide_lanes(d.L);
  const unsigned hgrid = (unsigned)((threads + kWideThreads - 1) / kWideThreads);
  // end-of-sweep grid: one block per SM (few atomics per counter), and enough
  // threads that none counts more than 10 sites (its bond count stays below 32)
  const long egrid = std::max<long>(std::min<long>((d.N + kWideThreads - 1) / kWideThreads, (long)sms),
                                    (d.N + 10L * kWideThreads - 1) / (10L * kWideThreads));
  k_wide_begin<<<1, 32, 0, g.stream>>>(wp, end);
  SA_CUDA_TRY(cudaGetLastError());
  auto sweeps = [&](int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
      k_wide_half<<<hgrid, kWideThreads, 0, g.stream>>>(wp, 0);
      k_wide_half<<<hgrid, kWideThreads, 0, g.stream>>>(wp, 1);
      k_wide_end<<<(unsigned)egrid, kWideThreads, 0, g.stream>>>(wp);
    }
  };
  int64_t n = end - start;
  if (n >= kWideGraphSweeps) {
    // the launch sequence of a sweep never changes (the sweep counter, draw
    // index and thresholds live in device memory): replay a captured graph
    cudaGraphExec_t exec = nullptr;
    for (const auto& w : b->wide_graphs)
      if (w.hgrid == hgrid && w.egrid == (unsigned)egrid && memcmp(&w.wp, &wp, sizeof wp) == 0) exec = w.exec;
    if (!exec && b->wide_graphs.size() >= kWideGraphCache) {
      // a server's requests come and go, each with its own parameters: keep
      // the cache bounded (destroyed once no replay can be in flight)
      SA_CUDA_TRY(cudaDeviceSynchronize());
      for (auto& w : b->wide_graphs) cudaGraphExecDestroy(w.exec);
      b->wide_graphs.clear();
    }
    if (!exec) {
      cudaGraph_t graph = nullptr;
      if (cudaStreamBeginCapture(g.stream, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
        sweeps(kWideGraphSweeps);
        if (cudaStreamEndCapture(g.stream, &graph) == cudaSuccess && graph) {
          if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) exec = nullptr;
          cudaGraphDestroy(graph);
        }
      }
      cudaGetLastError();  // a stream that cannot be captured: launch directly
      if (exec) {
        sa_batch::WideGraph w;
        memcpy(&w.wp, &wp, sizeof wp);
        w.hgrid = hgrid;
        w.egrid = (unsigned)egrid;
        w.exec = exec;
        b->wide_graphs.push_back(w);
      }
    }
    if (exec) {
      for (; n >= kWideGraphSweeps; n -= kWideGraphSweeps) SA_CUDA_TRY(cudaGraphLaunch(exec, g.stream));
    }
  }
  sweeps(n);
  SA_CUDA_TRY(cudaGetLastError());
  return SA_OK;
}

// Extends every ladder's exchange table to cover `need` attempts. Each
// ladder owns a device segment with room for `cap` entries; new entries are
// copied host->device as they are generated (only the new ones), and a
// segment that runs out of room is reallocated with double the capacity.
static int ensure_decisions(sa_batch* b, const std::vector<int64_t>& need) {
  bool relayout = (b->d_dec == nullptr);
  for (size_t l = 0; l < b->ladders.size(); ++l) {
    Ladder& ld = b->ladders[l];
    while ((int64_t)ld.dec.size() < need[l]) {
      Decision dc;
      int i = ld.uni_int(ld.gen);         // src/parallel_tempering.hpp:112
      double r = ld.uni_double(ld.gen);   // src/parallel_tempering.hpp:114
      double dB = (1. / ld.T[i] - 1. / ld.T[i + 1]);
      int64_t lo, hi;
      pt_accept_interval(dB, r, ld.span, &lo, &hi);
      dc.pair = i;
      dc.lo = (int32_t)std::max<int64_t>(lo, -2147483647LL);
      dc.hi = (int32_t)std::min<int64_t>(hi, 2147483647LL);
      dc.pad = 0;
      ld.dec.push_back(dc);
    }
    if ((int64_t)ld.dec.size() > ld.cap) relayout = true;
  }
  if (relayout) {
    int64_t total = 0;
    for (Ladder& ld : b->ladders) {
      ld.cap = std::max<int64_t>(1024, 2 * (int64_t)ld.dec.size());
      ld.dec_off = total;
      ld.uploaded = 0;
      total += ld.cap;
    }
    SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
    cudaFree(b->d_dec);
    b->d_dec = nullptr;
    SA_CUDA_TRY(cudaMalloc(&b->d_dec, std::max<int64_t>(total, 1) * sizeof(Decision)));
    b->dec_cap = total;
    for (InstDesc& d : b->inst)
      if (d.ladder >= 0) d.dec_off = b->ladders[d.ladder].dec_off;
    SA_CUDA_TRY(cudaMemcpyAsync(b->d_inst, b->inst.data(), b->inst.size() * sizeof(InstDesc),
                                cudaMemcpyHostToDevice, b->stream));
  }
  // stage the new entries in pinned memory and copy them after the previous ones
  int64_t fresh = 0;
  for (Ladder& ld : b->ladders) fresh += (int64_t)ld.dec.size() - ld.uploaded;
  if (fresh == 0) return SA_OK;
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));  // the pinned staging buffer is reused
  if (fresh > b->h_dec_cap) {
    if (b->h_dec) cudaFreeHost(b->h_dec);
    b->h_dec = nullptr;
    b->h_dec_cap = std::max<int64_t>(fresh, 4096);
    SA_CUDA_TRY(cudaHostAlloc((void**)&b->h_dec, b->h_dec_cap * sizeof(Decision), cudaHostAllocDefault));
  }
  int64_t pos = 0;
  for (Ladder& ld : b->ladders) {
    const int64_t n = (int64_t)ld.dec.size() - ld.uploaded;
    if (n <= 0) continue;
    memcpy(b->h_dec + pos, ld.dec.data() + ld.uploaded, n * sizeof(Decision));
    SA_CUDA_TRY(cudaMemcpyAsync(b->d_dec + ld.dec_off + ld.uploaded, b->h_dec + pos, n * sizeof(Decision),
                                cudaMemcpyHostToDevice, b->stream));
    b->h2d_bytes_last += n * (int64_t)sizeof(Decision);
    ld.uploaded += n;
    pos += n;
  }
  return SA_OK;
}

// The resident kernel variant of a group: its lattice kind and whether its
// clusters span several CTAs.
template <int P, int SL>
static void (*resident_kernel_sl(const sa_batch::Group& g))(BatchParams) {
  const bool cl = g.C > 1;
  if constexpr (P == 1 && SL == 1)
    if (g.seg) return cl ? k_resident<1, 1, SA_LATTICE_3D, true, true> : k_resident<1, 1, SA_LATTICE_3D, false, true>;
  if (g.lattice == SA_LATTICE_3D) {
    if constexpr (SL == 2)
      if (g.hr) return cl ? k_resident<P, 2, SA_LATTICE_3D, true, false, true> : k_resident<P, 2, SA_LATTICE_3D, false, false, true>;
    return cl ? k_resident<P, SL, SA_LATTICE_3D, true> : k_resident<P, SL, SA_LATTICE_3D, false>;
  }
  if (g.lattice == SA_LATTICE_2D_OPEN_X)
    return cl ? k_resident<P, SL, SA_LATTICE_2D_OPEN_X, true> : k_resident<P, SL, SA_LATTICE_2D_OPEN_X, false>;
  return cl ? k_resident<P, SL, SA_LATTICE_2D, true> : k_resident<P, SL, SA_LATTICE_2D, false>;
}

// Resident groups carry their own lanes-per-site RP and slots-per-lane SL
// (RP * SL >= nslots); P (the instance descriptor's) is for the global kernel.
template <int P>
static void (*resident_kernel(const sa_batch::Group& g))(BatchParams) {
  if (g.SL == 2) {
    switch (g.RP) {
      case 1: return resident_kernel_sl<1, 2>(g);
      case 2: return resident_kernel_sl<2, 2>(g);
      case 4: return resident_kernel_sl<4, 2>(g);
      case 8: return resident_kernel_sl<8, 2>(g);
      default: return resident_kernel_sl<16, 2>(g);
    }
  }
  return resident_kernel_sl<P, 1>(g);
}

template <int P>
static int launch_group(sa_batch* b, const sa_batch::Group& g, int gi, long nsweeps) {
  BatchParams p;
  batch_params(b, nsweeps, &p);
  p.order = b->d_order + g.begin;
  p.ninst = g.count;
  p.work = b->d_work + gi;
  if (g.wide) return launch_wide(b, g, nsweeps, nullptr);
  if (!g.resident) {
    k_batch<P><<<g.grid, kBatchThreads, 0, g.stream>>>(p);
    SA_CUDA_TRY(cudaGetLastError());
    return SA_OK;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(g.count * g.C), 1, 1);
  cfg.blockDim = dim3((unsigned)g.threads, 1, 1);
  cfg.dynamicSmemBytes = g.smem;
  cfg.stream = g.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)g.C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  SA_CUDA_TRY(cudaLaunchKernelEx(&cfg, resident_kernel<P>(g), p));
  return SA_OK;
}

// The per-kernel attributes are shared by every group of the same P, so the
// dynamic shared-memory limit is the largest any such group needs
// (`smem_limit`, set by the caller from all groups).
template <int P>
static int prepare_resident(const sa_batch::Group& g, size_t smem_limit, int* max_clusters) {
  void (*kern)(BatchParams) = resident_kernel<P>(g);
  // the attribute is a ceiling shared by every user of the variant in the
  // process (batches and servers): never lower it below the whole budget
  SA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)std::max(smem_limit, kResSmemBudget)));
  SA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)g.C, 1, 1);
  cfg.blockDim = dim3((unsigned)g.threads, 1, 1);
  cfg.dynamicSmemBytes = g.smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)g.C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  SA_CUDA_TRY(cudaOccupancyMaxActiveClusters(max_clusters, kern, &cfg));
  if (*max_clusters < 1) {
    cudaFuncAttributes fa;
    cudaFuncGetAttributes(&fa, kern);
    char buf[256];
    snprintf(buf, sizeof buf,
             "resident cluster not schedulable: P=%d C=%d threads=%d smem=%zu (kernel: %d regs, "
             "max %d threads, %zu static smem, %d max dynamic smem)",
             P, g.C, g.threads, g.smem, fa.numRegs, fa.maxThreadsPerBlock, fa.sharedSizeBytes,
             fa.maxDynamicSharedSizeBytes);
    return fail(SA_ERR_UNSUPPORTED, buf);
  }
  return SA_OK;
}

// Serving: the kernel variant's attributes are set once, to the whole shared
// memory budget, so rounds with new shapes need no further attribute calls.
template <int P>
static int prepare_resident_once(const sa_batch::Group& g) {
  static std::mutex mu;
  static std::set<std::pair<int, void*>> done;
  void (*kern)(BatchParams) = resident_kernel<P>(g);
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({dev, (void*)kern})) return SA_OK;
  SA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kResSmemBudget));
  SA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  done.insert({dev, (void*)kern});
  return SA_OK;
}

template <int P>
static int group_dispatch(sa_batch* b, const sa_batch::Group& g, int gi, long nsweeps, int prepare,
                          int* max_clusters) {
  if (prepare == 2) return g.resident ? prepare_resident_once<P>(g) : SA_OK;
  if (prepare) {
    if (!g.resident) return SA_OK;
    size_t lim = 0;
    for (const auto& o : b->groups)
      if (o.resident && o.P == g.P && o.SL == g.SL && o.RP == g.RP && o.lattice == g.lattice &&
          (o.C > 1) == (g.C > 1) && o.hr == g.hr)
        lim = std::max(lim, o.smem);
    return prepare_resident<P>(g, lim, max_clusters);
  }
  return launch_group<P>(b, g, gi, nsweeps);
}

static int dispatch(sa_batch* b, const sa_batch::Group& g, int gi, long nsweeps, int prepare, int* mc) {
  switch (g.P) {
    case 1: return group_dispatch<1>(b, g, gi, nsweeps, prepare, mc);
    case 2: return group_dispatch<2>(b, g, gi, nsweeps, prepare, mc);
    case 4: return group_dispatch<4>(b, g, gi, nsweeps, prepare, mc);
    case 8: return group_dispatch<8>(b, g, gi, nsweeps, prepare, mc);
    case 16: return group_dispatch<16>(b, g, gi, nsweeps, prepare, mc);
    default: return group_dispatch<32>(b, g, gi, nsweeps, prepare, mc);
  }
}

extern "C" {

int sa_batch_create(sa_batch_t* out) {
  if (!out) return fail(SA_ERR_INVALID, "out is null");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(SA_ERR_NO_DEVICE, "no CUDA device available");
  sa_batch* b = new sa_batch();
  cudaGetDevice(&b->device);
  cudaError_t e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(e, "cudaStreamCreate");
  }
  b->stream = b->own_stream;
  *out = b;
  return SA_OK;
}

int sa_batch_destroy(sa_batch_t b) {
  if (!b) return SA_OK;
  cudaStreamSynchronize(b->stream);
  cudaFree(b->d_inst);
  cudaFree(b->d_state);
  cudaFree(b->d_order);
  cudaFree(b->d_work);
  cudaFree(b->d_spins);
  cudaFree(b->d_J);
  cudaFree(b->d_thr);
  cudaFree(b->d_dec);
  cudaFree(b->d_acc);
  cudaFree(b->d_att);
  cudaFree(b->d_rec_pair);
  cudaFree(b->d_rec_mask);
  cudaFree(b->d_stage);
  cudaFree(b->d_E);
  cudaFree(b->d_Eall);
  cudaFree(b->d_hist);
  cudaFree(b->d_seedJ);
  cudaFree(b->d_wide);
  for (auto& g : b->groups) {
    if (g.stream) cudaStreamDestroy(g.stream);
    if (g.done) cudaEventDestroy(g.done);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->h_dec) cudaFreeHost(b->h_dec);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
  return SA_OK;
}

int sa_batch_add_ladder(sa_batch_t b, const double* T, int n, int* id) {
  if (!b || !T || !id) return fail(SA_ERR_INVALID, "null argument");
  if (b->finalized) return fail(SA_ERR_INVALID, "batch already finalized");
  if (n < 1 || n > 32) return fail(SA_ERR_UNSUPPORTED, "a ladder holds 1..32 temperatures");
  Ladder ld;
  ld.T.assign(T, T + n);
  for (double t : ld.T)
    if (!(t > 0)) return fail(SA_ERR_INVALID, "temperatures must be > 0");
  std::sort(ld.T.begin(), ld.T.end());
  ld.uni_int = std::uniform_int_distribution<int>(0, std::max(0, n - 2));
  b->ladders.push_back(ld);
  *id = (int)b->ladders.size() - 1;
  return SA_OK;
}

int sa_batch_add_schedule(sa_batch_t b, const double* T, int nsteps, int sweeps_per_step, int* id) {
  if (!b || !T || !id) return fail(SA_ERR_INVALID, "null argument");
  if (b->finalized) return fail(SA_ERR_INVALID, "batch already finalized");
  if (nsteps < 1 || sweeps_per_step < 1) return fail(SA_ERR_INVALID, "empty schedule");
  Schedule s;
  s.T.assign(T, T + nsteps);
  for (double t : s.T)
    if (!(t > 0)) return fail(SA_ERR_INVALID, "temperatures must be > 0");
  s.sweeps_per_step = sweeps_per_step;
  b->scheds.push_back(s);
  *id = (int)b->scheds.size() - 1;
  return SA_OK;
}

int sa_batch_add_instance(sa_batch_t b, int lattice, int L, int ladder, int sched, uint64_t seed_J,
                          uint64_t seed, int* id) {
  if (!b || !id) return fail(SA_ERR_INVALID, "null argument");
  if (b->finalized) return fail(SA_ERR_INVALID, "batch already finalized");
  if (lattice < 0 || lattice > 2) return fail(SA_ERR_INVALID, "unknown lattice kind");
  if (L < 2) return fail(SA_ERR_INVALID, "L must be >= 2");
  if (L & 1) return fail(SA_ERR_ODD_L, "L must be even");
  if ((ladder >= 0) == (sched >= 0)) return fail(SA_ERR_INVALID, "exactly one of ladder / schedule");
  if (ladder >= (int)b->ladders.size() || sched >= (int)b->scheds.size())
    return fail(SA_ERR_INVALID, "unknown ladder / schedule id");
  InstDesc d;
  memset(&d, 0, sizeof d);
  const int dim = lattice_dim(lattice);
  d.lattice = lattice;
  d.L = L;
  d.N = (dim == 3) ? (int64_t)L * L * L : (int64_t)L * L;
  if (d.N > kBatchMaxN) return fail(SA_ERR_UNSUPPORTED, "instance too large for the batched engine");
  d.half = d.N / 2;
  d.nbonds = dim * d.N - (lattice == SA_LATTICE_2D_OPEN_X ? L : 0);
  d.ladder = ladder;
  d.sched = sched;
  d.nslots = (ladder >= 0) ? (int)b->ladders[ladder].T.size() : 1;
  int P = 1;
  while (P < d.nslots) P <<= 1;
  d.P = P;
  d.seed = seed;
  if (sched >= 0) {
    d.sweeps_per_step = b->scheds[sched].sweeps_per_step;
    d.thr_count = (int)b->scheds[sched].T.size();
    d.sweep_limit = (int64_t)d.thr_count * d.sweeps_per_step;
  } else {
    d.sweeps_per_step = 1;
    d.sweep_limit = -1;
    Ladder& ld = b->ladders[ladder];
    ld.span = std::max<int64_t>(ld.span, 2 * d.nbonds);
  }
  d.state_idx = (int64_t)b->inst.size();
  b->inst.push_back(d);
  b->seed_J.push_back(seed_J);
  *id = (int)b->inst.size() - 1;
  return SA_OK;
}

int sa_batch_finalize(sa_batch_t b) {
  if (!b) return fail(SA_ERR_INVALID, "null batch");
  if (b->finalized) return SA_OK;
  if (b->inst.empty()) return fail(SA_ERR_INVALID, "empty batch");
  // offsets and threshold pool: one block per (ladder or schedule, lattice kind)
  std::map<std::pair<int, int>, int64_t> thr_at;  // key (+ladder+1 or -(sched+1), lattice)
  std::vector<BThr> thr;
  int64_t spin_off = 0, J_off = 0, pair_off = 0;
  b->site_slots = 0;
  for (InstDesc& d : b->inst) {
    const int dim = lattice_dim(d.lattice);
    d.spin_off = spin_off;
    spin_off += d.N * d.nslots;
    d.J_off = J_off;
    J_off += dim * d.N;
    d.pair_off = pair_off;
    pair_off += std::max(0, d.nslots - 1);
    b->site_slots += d.N * d.nslots;
    auto key = std::make_pair(d.ladder >= 0 ? d.ladder + 1 : -(d.sched + 1), d.lattice);
    auto it = thr_at.find(key);
    if (it == thr_at.end()) {
      int64_t off = (int64_t)thr.size();
      const std::vector<double>& Ts = d.ladder >= 0 ? b->ladders[d.ladder].T : b->scheds[d.sched].T;
      for (double t : Ts) thr.push_back(to_bthr(d.lattice, t));
      it = thr_at.emplace(key, off).first;
    }
    d.thr_off = it->second;
  }
  b->npairs = pair_off;
  // energy histograms: PT instances only, when requested before finalize
  b->hist_count = 0;
  for (InstDesc& d : b->inst) {
    d.hist_off = -1;
    if (b->hstride > 0 && d.ladder >= 0) {
      d.hist_off = b->hist_count;
      b->hist_count += (int64_t)d.nslots * (d.nbonds + 1);
    }
  }
  if (b->hist_count) {
    for (const auto& gcheck : b->inst)
      if (gcheck.hist_off >= 0 && b->force_global)
        return fail(SA_ERR_UNSUPPORTED, "energy histograms need the resident kernel");
    SA_CUDA_TRY(cudaMalloc(&b->d_hist, b->hist_count * sizeof(int32_t)));
    SA_CUDA_TRY(cudaMemsetAsync(b->d_hist, 0, b->hist_count * sizeof(int32_t), b->stream));
  }
  std::vector<int32_t> order = build_groups(b);
  b->h_order = order;
  if (int st = ensure_wide_scratch(b)) return st;
  const size_t ni = b->inst.size();
  SA_CUDA_TRY(cudaMalloc(&b->d_inst, ni * sizeof(InstDesc)));
  SA_CUDA_TRY(cudaMalloc(&b->d_state, ni * sizeof(InstState)));
  SA_CUDA_TRY(cudaMalloc(&b->d_order, ni * sizeof(int32_t)));
  SA_CUDA_TRY(cudaMalloc(&b->d_work, std::max<size_t>(b->groups.size(), 1) * sizeof(int32_t)));
  SA_CUDA_TRY(cudaMalloc(&b->d_spins, std::max<int64_t>(spin_off, 1) * sizeof(word_t)));
  SA_CUDA_TRY(cudaMalloc(&b->d_J, std::max<int64_t>(J_off, 1) * sizeof(word_t)));
  SA_CUDA_TRY(cudaMalloc(&b->d_thr, std::max<size_t>(thr.size(), 1) * sizeof(BThr)));
  SA_CUDA_TRY(cudaMalloc(&b->d_acc, std::max<int64_t>(pair_off, 1) * sizeof(int64_t)));
  SA_CUDA_TRY(cudaMalloc(&b->d_att, std::max<int64_t>(pair_off, 1) * sizeof(int64_t)));
  SA_CUDA_TRY(cudaMalloc(&b->d_E, 64 * sizeof(int64_t)));
  int64_t maxN = 0;
  for (const InstDesc& d : b->inst) maxN = std::max(maxN, d.N);
  SA_CUDA_TRY(cudaMalloc(&b->d_stage, maxN * sizeof(word_t)));
  SA_CUDA_TRY(cudaMemsetAsync(b->d_state, 0, ni * sizeof(InstState), b->stream));
  SA_CUDA_TRY(cudaMemsetAsync(b->d_acc, 0, std::max<int64_t>(pair_off, 1) * sizeof(int64_t), b->stream));
  SA_CUDA_TRY(cudaMemsetAsync(b->d_att, 0, std::max<int64_t>(pair_off, 1) * sizeof(int64_t), b->stream));
  SA_CUDA_TRY(cudaMemcpyAsync(b->d_order, order.data(), ni * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream));
  if (!thr.empty())
    SA_CUDA_TRY(cudaMemcpyAsync(b->d_thr, thr.data(), thr.size() * sizeof(BThr), cudaMemcpyHostToDevice, b->stream));
  SA_CUDA_TRY(cudaMemcpyAsync(b->d_inst, b->inst.data(), ni * sizeof(InstDesc), cudaMemcpyHostToDevice, b->stream));
  uint64_t* d_seedJ = nullptr;
  SA_CUDA_TRY(cudaMalloc(&d_seedJ, ni * sizeof(uint64_t)));
  SA_CUDA_TRY(cudaMemcpyAsync(d_seedJ, b->seed_J.data(), ni * sizeof(uint64_t), cudaMemcpyHostToDevice, b->stream));
  dim3 g((unsigned)((maxN + 255) / 256), (unsigned)std::min<size_t>(ni, 65535));
  k_batch_init<<<g, 256, 0, b->stream>>>(b->d_inst, d_seedJ, (int)ni, b->d_spins, b->d_J);
  SA_CUDA_TRY(cudaGetLastError());
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  cudaFree(d_seedJ);
  b->h_sweeps.assign(ni, 0);
  b->h_xsteps.assign(ni, 0);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  const unsigned ev_flags = b->group_timing ? cudaEventDefault : cudaEventDisableTiming;
  SA_CUDA_TRY(cudaEventCreateWithFlags(&b->fork, ev_flags));
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    sa_batch::Group& g = b->groups[gi];
    SA_CUDA_TRY(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    SA_CUDA_TRY(cudaEventCreateWithFlags(&g.done, ev_flags));
    if (g.resident) {
      int mc = 0;
      int st = dispatch(b, g, (int)gi, 0, 1, &mc);
      if (st) return st;
      g.grid = mc;
    } else {
      g.grid = (int)std::min<int64_t>((int64_t)sms, (int64_t)g.count);  // one 512-thread CTA per SM
    }
  }
  b->finalized = true;
  // the ladders' first exchanges
  std::vector<int64_t> need(b->ladders.size(), 1);
  return ensure_decisions(b, need);
}

int sa_batch_set_exchange_interval(sa_batch_t b, int k) {
  if (!b || k < 1) return fail(SA_ERR_INVALID, "interval must be >= 1");
  b->xinterval = k;
  return SA_OK;
}

int sa_batch_set_histograms(sa_batch_t b, int stride) {
  if (!b || stride < 0) return fail(SA_ERR_INVALID, "stride must be >= 0");
  if (b->finalized) return fail(SA_ERR_INVALID, "enable histograms before finalize");
  b->hstride = stride;
  return SA_OK;
}

int sa_batch_histogram(sa_batch_t b, int id, int slot, int32_t* out, long cap, long* nbins) {
  if (!b || !nbins) return fail(SA_ERR_INVALID, "null argument");
  if (!b->finalized) return fail(SA_ERR_INVALID, "finalize the batch first");
  if (id < 0 || id >= (int)b->inst.size()) return fail(SA_ERR_INVALID, "instance id out of range");
  const InstDesc& d = b->inst[id];
  if (d.hist_off < 0) return fail(SA_ERR_INVALID, "no histograms for this instance");
  if (slot < 0 || slot >= d.nslots) return fail(SA_ERR_INVALID, "bad slot");
  *nbins = (long)(d.nbonds + 1);
  if (!out) return SA_OK;
  if (cap < *nbins) return fail(SA_ERR_BUFFER, "histogram buffer too small");
  SA_CUDA_TRY(cudaMemcpyAsync(out, b->d_hist + d.hist_off + (long)slot * (d.nbonds + 1),
                              (size_t)(d.nbonds + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  return SA_OK;
}

int sa_batch_set_kernel(sa_batch_t b, int kernel) {
  if (!b || kernel < 0 || kernel > 2)
    return fail(SA_ERR_INVALID, "kernel must be 0 (auto), 1 (global) or 2 (auto without the wide form)");
  if (b->finalized) return fail(SA_ERR_INVALID, "choose the kernel before finalize");
  b->force_global = (kernel == 1);
  b->no_wide = (kernel == 2);
  return SA_OK;
}

int sa_batch_set_group_timing(sa_batch_t b, int on) {
  if (!b) return fail(SA_ERR_INVALID, "null batch");
  if (b->finalized) return fail(SA_ERR_INVALID, "set group timing before finalize");
  b->group_timing = on != 0;
  return SA_OK;
}

int sa_batch_group_times(sa_batch_t b, int32_t* info, float* ms, int cap, int* n) {
  if (!b || !n) return fail(SA_ERR_INVALID, "null argument");
  if (!b->finalized || !b->group_timing) return fail(SA_ERR_INVALID, "enable group timing before finalize");
  *n = (int)b->groups.size();
  if (!info && !ms) return SA_OK;
  if (cap < *n) return fail(SA_ERR_BUFFER, "group buffer too small");
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    const sa_batch::Group& g = b->groups[gi];
    if (info) {
      const int32_t v[5] = {g.lattice, g.L, g.count, g.wide ? -1 : (g.resident ? g.C : 0), g.threads / 32};
      memcpy(info + 5 * gi, v, sizeof v);
    }
    if (ms) {
      SA_CUDA_TRY(cudaEventSynchronize(g.done));
      SA_CUDA_TRY(cudaEventElapsedTime(&ms[gi], b->fork, g.done));
    }
  }
  return SA_OK;
}

int sa_batch_set_spread(sa_batch_t b, int on) {
  if (!b) return fail(SA_ERR_INVALID, "null batch");
  if (b->finalized) return fail(SA_ERR_INVALID, "set spreading before finalize");
  b->no_spread = !on;
  return SA_OK;
}

int sa_batch_set_tuning(sa_batch_t b, const int32_t* entries, int n) {
  if (!b) return fail(SA_ERR_INVALID, "null batch");
  if (b->finalized) return fail(SA_ERR_INVALID, "set the tuning before finalize");
  if (n < 0) {
    b->tuning.clear();
    b->tuning_set = false;
    return SA_OK;
  }
  if (n > 0 && !entries) return fail(SA_ERR_INVALID, "null tuning entries");
  b->tuning.assign(n, TuneEntry{});
  for (int i = 0; i < n; ++i) {
    const int32_t* e = entries + 7 * i;
    b->tuning[i] = TuneEntry{e[0], e[1], e[2], e[3], e[4], e[5], e[6]};
  }
  b->tuning_set = true;
  return SA_OK;
}

int sa_tuning_table(int32_t* out, int cap, int* n) {
  if (!n) return fail(SA_ERR_INVALID, "null count");
  const std::vector<TuneEntry>& t = builtin_tuning();
  *n = (int)t.size();
  if (!out) return SA_OK;
  if (cap < (int)t.size()) return fail(SA_ERR_BUFFER, "tuning buffer too small");
  for (size_t i = 0; i < t.size(); ++i) {
    const TuneEntry& e = t[i];
    const int32_t v[7] = {e.lattice, e.L, e.nslots, e.C, e.SL, e.warps, e.hr};
    memcpy(out + 7 * i, v, sizeof v);
  }
  return SA_OK;
}

int sa_batch_instance_shape(sa_batch_t b, int id, int32_t* out) {
  if (!b || !out) return fail(SA_ERR_INVALID, "null argument");
  if (!b->finalized) return fail(SA_ERR_INVALID, "finalize first");
  if (id < 0 || id >= (int)b->inst.size()) return fail(SA_ERR_INVALID, "no such instance");
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    const sa_batch::Group& g = b->groups[gi];
    for (int k = g.begin; k < g.begin + g.count; ++k) {
      if (b->h_order[k] != id) continue;
      const InstDesc& d = b->inst[id];
      const int32_t v[7] = {d.lattice, d.L, d.nslots, g.wide ? -1 : (g.resident ? g.C : 0), g.SL, g.threads / 32,
                            g.hr ? 1 : 0};
      memcpy(out, v, sizeof v);
      return SA_OK;
    }
  }
  return fail(SA_ERR_INVALID, "instance not in a launch group");
}

int sa_batch_launches_per_run(sa_batch_t b, int* n) {
  if (!b || !n) return fail(SA_ERR_INVALID, "null argument");
  *n = (int)b->groups.size();
  return SA_OK;
}

int sa_batch_set_measure_stride(sa_batch_t b, int stride) {
  if (!b || stride < 0) return fail(SA_ERR_INVALID, "stride must be >= 0");
  b->mstride = stride;
  return SA_OK;
}

int sa_batch_record_exchanges(sa_batch_t b, long cap) {
  if (!b || cap < 0) return fail(SA_ERR_INVALID, "bad capacity");
  if (!b->finalized) return fail(SA_ERR_INVALID, "finalize the batch first");
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  cudaFree(b->d_rec_pair);
  cudaFree(b->d_rec_mask);
  b->d_rec_pair = nullptr;
  b->d_rec_mask = nullptr;
  b->rec_cap = cap;
  if (cap > 0) {
    size_t n = (size_t)cap * b->inst.size();
    SA_CUDA_TRY(cudaMalloc(&b->d_rec_pair, n * sizeof(int32_t)));
    SA_CUDA_TRY(cudaMalloc(&b->d_rec_mask, n * sizeof(uint64_t)));
    SA_CUDA_TRY(cudaMemset(b->d_rec_pair, 0xFF, n * sizeof(int32_t)));
    SA_CUDA_TRY(cudaMemset(b->d_rec_mask, 0, n * sizeof(uint64_t)));
  }
  return SA_OK;
}

int sa_batch_run(sa_batch_t b, long nsweeps) {
  if (!b) return fail(SA_ERR_INVALID, "null batch");
  if (!b->finalized) return fail(SA_ERR_INVALID, "finalize the batch first");
  if (nsweeps < 0) return fail(SA_ERR_INVALID, "nsweeps < 0");
  if (nsweeps == 0) return SA_OK;
  // host mirror of the counters -> exchange-table lengths this launch needs
  b->run_start = b->h_sweeps;
  std::vector<int64_t> need(b->ladders.size(), 0);
  for (size_t i = 0; i < b->inst.size(); ++i) {
    const InstDesc& d = b->inst[i];
    int64_t n = nsweeps;
    if (d.sweep_limit >= 0) n = std::max<int64_t>(0, std::min<int64_t>(n, d.sweep_limit - b->h_sweeps[i]));
    const int64_t s1 = b->h_sweeps[i] + n;
    if (d.ladder >= 0 && d.nslots > 1) {
      const int64_t x1 = s1 / b->xinterval;
      b->h_xsteps[i] = x1;
      need[d.ladder] = std::max(need[d.ladder], x1);
    }
    b->h_sweeps[i] = s1;
  }
  b->h2d_bytes_last = 0;
  int st = ensure_decisions(b, need);
  if (st) return st;
  SA_CUDA_TRY(cudaMemsetAsync(b->d_work, 0, b->groups.size() * sizeof(int32_t), b->stream));
  // every group on its own stream, forked from and joined back into the
  // batch stream, so one group's tail overlaps the others' work
  SA_CUDA_TRY(cudaEventRecord(b->fork, b->stream));
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    SA_CUDA_TRY(cudaStreamWaitEvent(b->groups[gi].stream, b->fork, 0));
    st = dispatch(b, b->groups[gi], (int)gi, nsweeps, 0, nullptr);
    if (st) return st;
    SA_CUDA_TRY(cudaEventRecord(b->groups[gi].done, b->groups[gi].stream));
  }
  for (size_t gi = 0; gi < b->groups.size(); ++gi)
    SA_CUDA_TRY(cudaStreamWaitEvent(b->stream, b->groups[gi].done, 0));
  SA_CUDA_TRY(cudaGetLastError());
  return SA_OK;
}

int sa_batch_sync(sa_batch_t b) {
  if (!b) return fail(SA_ERR_INVALID, "null batch");
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  return SA_OK;
}

int sa_batch_set_stream(sa_batch_t b, void* stream) {
  if (!b) return fail(SA_ERR_INVALID, "null batch");
  b->stream = stream ? (cudaStream_t)stream : b->own_stream;
  return SA_OK;
}

int sa_batch_site_slots(sa_batch_t b, long long* n) {
  if (!b || !n) return fail(SA_ERR_INVALID, "null argument");
  long long s = 0;
  for (const InstDesc& d : b->inst) s += d.N * d.nslots;
  *n = s;
  return SA_OK;
}

int sa_batch_num_instances(sa_batch_t b, int* n) {
  if (!b || !n) return fail(SA_ERR_INVALID, "null argument");
  *n = (int)b->inst.size();
  return SA_OK;
}

static int check_inst(sa_batch* b, int id) {
  if (!b) return fail(SA_ERR_INVALID, "null batch");
  if (!b->finalized) return fail(SA_ERR_INVALID, "finalize the batch first");
  if (id < 0 || id >= (int)b->inst.size()) return fail(SA_ERR_INVALID, "instance id out of range");
  return SA_OK;
}

int sa_batch_get_spins(sa_batch_t b, int id, int slot, uint64_t* s) {
  int st = check_inst(b, id);
  if (st) return st;
  const InstDesc& d = b->inst[id];
  if (!s || slot < 0 || slot >= d.nslots) return fail(SA_ERR_INVALID, "bad slot / buffer");
  k_batch_gather<<<(unsigned)((d.N + 255) / 256), 256, 0, b->stream>>>(b->d_spins, b->d_inst, id, slot,
                                                                       b->d_stage);
  SA_CUDA_TRY(cudaGetLastError());
  SA_CUDA_TRY(cudaMemcpyAsync(s, b->d_stage, d.N * sizeof(word_t), cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  return SA_OK;
}

int sa_batch_get_J(sa_batch_t b, int id, uint64_t* jx, uint64_t* jy, uint64_t* jz) {
  int st = check_inst(b, id);
  if (st) return st;
  const InstDesc& d = b->inst[id];
  const int dim = lattice_dim(d.lattice);
  if (!jx || !jy || (dim == 3 && !jz)) return fail(SA_ERR_INVALID, "null buffer");
  std::vector<word_t> own(dim * d.N);
  SA_CUDA_TRY(cudaMemcpyAsync(own.data(), b->d_J + d.J_off, own.size() * sizeof(word_t), cudaMemcpyDeviceToHost,
                              b->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  const long L = d.L, L2 = L * L, N = d.N, hL = L / 2;
  auto split = [&](long i) {
    long r = i / L;
    int x = (int)(i - r * L), y = (int)(r % L), c = (x + y) & 1;
    return (long)c * d.half + r * hL + (x >> 1);
  };
  for (long i = 0; i < N; ++i) {
    long e = ((i + 1) % L == 0) ? i - L + 1 : i + 1;
    long s_ = ((i + L) % L2 < L) ? i - L2 + L : i + L;
    jx[2 * i] = own[split(i)];
    jx[2 * i + 1] = own[split(e)];
    jy[2 * i] = own[N + split(i)];
    jy[2 * i + 1] = own[N + split(s_)];
    if (dim == 3) {
      long dd = (i + L2 >= N) ? i - N + L2 : i + L2;
      jz[2 * i] = own[2 * N + split(i)];
      jz[2 * i + 1] = own[2 * N + split(dd)];
    }
  }
  return SA_OK;
}

int sa_batch_measure(sa_batch_t b, int id, int slot, int64_t* E) {
  int st = check_inst(b, id);
  if (st) return st;
  if (!E || slot < 0 || slot >= b->inst[id].nslots) return fail(SA_ERR_INVALID, "bad slot / buffer");
  BatchParams p;
  batch_params(b, 0, &p);
  k_batch_measure_one<<<1, kBatchThreads, 0, b->stream>>>(p, id, slot, b->d_E);
  SA_CUDA_TRY(cudaGetLastError());
  SA_CUDA_TRY(cudaMemcpyAsync(E, b->d_E, 64 * sizeof(int64_t), cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  return SA_OK;
}

int sa_batch_acceptance(sa_batch_t b, int id, int64_t* accepted, int64_t* attempts) {
  int st = check_inst(b, id);
  if (st) return st;
  const InstDesc& d = b->inst[id];
  const int np = std::max(0, d.nslots - 1);
  if (np == 0) return SA_OK;
  if (!accepted || !attempts) return fail(SA_ERR_INVALID, "null buffer");
  SA_CUDA_TRY(cudaMemcpyAsync(accepted, b->d_acc + d.pair_off, np * sizeof(int64_t), cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaMemcpyAsync(attempts, b->d_att + d.pair_off, np * sizeof(int64_t), cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  return SA_OK;
}

int sa_batch_exchanges(sa_batch_t b, int id, int* pairs, uint64_t* masks, long cap, long* count) {
  int st = check_inst(b, id);
  if (st) return st;
  if (!count) return fail(SA_ERR_INVALID, "null count");
  long n = std::min<long>((long)b->h_xsteps[id], b->rec_cap);
  *count = n;
  if (!pairs || !masks || n == 0) return SA_OK;
  if (cap < n) return fail(SA_ERR_BUFFER, "buffer smaller than the recorded exchanges");
  SA_CUDA_TRY(cudaMemcpyAsync(pairs, b->d_rec_pair + (long)id * b->rec_cap, n * sizeof(int32_t),
                              cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaMemcpyAsync(masks, b->d_rec_mask + (long)id * b->rec_cap, n * sizeof(uint64_t),
                              cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  return SA_OK;
}

int sa_batch_energies(sa_batch_t b, int64_t* E) {
  if (!b || !E) return fail(SA_ERR_INVALID, "null argument");
  if (!b->finalized) return fail(SA_ERR_INVALID, "finalize the batch first");
  if (!b->d_Eall) {
    std::vector<int64_t> off(b->inst.size());
    int64_t o = 0;
    for (size_t i = 0; i < b->inst.size(); ++i) {
      off[i] = o;
      o += (int64_t)b->inst[i].nslots * 64;
    }
    b->e_count = o;
    SA_CUDA_TRY(cudaMalloc(&b->d_Eall, (o + (int64_t)off.size()) * sizeof(int64_t)));
    SA_CUDA_TRY(cudaMemcpy(b->d_Eall + o, off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  }
  BatchParams p;
  batch_params(b, 0, &p);
  k_batch_energies<<<(unsigned)b->inst.size(), kBatchThreads, 0, b->stream>>>(p, b->d_Eall + b->e_count,
                                                                                b->d_Eall);
  SA_CUDA_TRY(cudaGetLastError());
  SA_CUDA_TRY(cudaMemcpyAsync(E, b->d_Eall, b->e_count * sizeof(int64_t), cudaMemcpyDeviceToHost, b->stream));
  return SA_OK;
}

int sa_batch_energy_count(sa_batch_t b, long long* n) {
  if (!b || !n) return fail(SA_ERR_INVALID, "null argument");
  long long o = 0;
  for (const InstDesc& d : b->inst) o += (long long)d.nslots * 64;
  *n = o;
  return SA_OK;
}

int sa_batch_last_h2d_bytes(sa_batch_t b, long long* n) {
  if (!b || !n) return fail(SA_ERR_INVALID, "null argument");
  *n = b->h2d_bytes_last;
  return SA_OK;
}

int sa_batch_acceptance_all(sa_batch_t b, int64_t* accepted, int64_t* attempts) {
  if (!b || !accepted || !attempts) return fail(SA_ERR_INVALID, "null argument");
  if (!b->finalized) return fail(SA_ERR_INVALID, "finalize the batch first");
  if (b->npairs == 0) return SA_OK;
  SA_CUDA_TRY(cudaMemcpyAsync(accepted, b->d_acc, b->npairs * sizeof(int64_t), cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaMemcpyAsync(attempts, b->d_att, b->npairs * sizeof(int64_t), cudaMemcpyDeviceToHost, b->stream));
  return SA_OK;
}

int sa_batch_num_pairs(sa_batch_t b, long long* n) {
  if (!b || !n) return fail(SA_ERR_INVALID, "null argument");
  *n = b->npairs;
  return SA_OK;
}

int sa_batch_anneal_result(sa_batch_t b, int id, int64_t* Emax, long* sweeps_done) {
  int st = check_inst(b, id);
  if (st) return st;
  InstState s;
  SA_CUDA_TRY(cudaMemcpyAsync(&s, b->d_state + id, sizeof s, cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  if (Emax) memcpy(Emax, s.emax, sizeof s.emax);
  if (sweeps_done) *sweeps_done = (long)s.sweeps;
  return SA_OK;
}

int sa_batch_sweeps_done(sa_batch_t b, int id, long* sweeps_done) {
  int st = check_inst(b, id);
  if (st) return st;
  if (!sweeps_done) return fail(SA_ERR_INVALID, "null argument");
  InstState s;
  SA_CUDA_TRY(cudaMemcpyAsync(&s, b->d_state + id, sizeof s, cudaMemcpyDeviceToHost, b->stream));
  SA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  *sweeps_done = (long)s.sweeps;
  return SA_OK;
}

}  // extern "C"

// ===========================================================================
// Serving: continuous batching of anneal requests.
//
// A serving object owns device pools sized from a memory budget: one word pool
// for spins and couplings (first-fit free list), a threshold pool (one entry
// per schedule step) and a table of per-request states. A request is admitted
// only when all three have room; it is initialised on the device (couplings
// from seed_J, spins from seed, like a batch instance) and stays resident until
// it has run its whole schedule. Every round rebuilds the instance table from
// the active requests, groups it by shape and launches the same kernels as
// sa_batch_run for a chunk of sweeps; requests that arrive meanwhile join at
// the next round. Each request's random stream is keyed by its own seed, so
// its result does not depend on what else runs beside it.
// ===========================================================================
namespace {

struct FreeList {
  std::map<int64_t, int64_t> free;  // offset -> length
  int64_t cap = 0;
  void init(int64_t n) {
    cap = n;
    free.clear();
    if (n > 0) free[0] = n;
  }
  int64_t alloc(int64_t n) {
    for (auto it = free.begin(); it != free.end(); ++it) {
      if (it->second >= n) {
        const int64_t off = it->first, len = it->second;
        free.erase(it);
        if (len > n) free[off + n] = len - n;
        return off;
      }
    }
    return -1;
  }
  void release(int64_t off, int64_t n) {
    auto it = free.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free.erase(nx);
    }
    if (it != free.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free.erase(it);
      }
    }
  }
};

struct ServeReq {
  InstDesc d;
  int64_t words;     // spin + coupling words held
  int64_t thr_n;     // threshold entries held
  int64_t sweeps;    // host mirror of the sweeps done
  bool fresh;        // needs device initialisation
  uint64_t seed_J;
};

}  // namespace

struct sa_serve {
  sa_batch b;  // kernel context: pools as d_spins/d_J/d_thr/d_state
  FreeList words, thr;
  std::vector<int> free_states;
  std::map<int64_t, ServeReq> active;  // by request id
  std::vector<int64_t> finished;
  int64_t next_id = 1;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  std::vector<BThr> thr_stage;
  size_t budget = 0;
};

extern "C" {

int sa_serve_create(size_t budget_bytes, int max_requests, sa_serve_t* out) {
  if (!out || max_requests < 1 || budget_bytes < (1u << 20)) return fail(SA_ERR_INVALID, "bad serving parameters");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SA_ERR_NO_DEVICE, "no CUDA device available");
  sa_serve* s = new sa_serve();
  sa_batch& b = s->b;
  cudaGetDevice(&b.device);
  auto bail = [&](cudaError_t e, const char* w) {
    int st = cuda_fail(e, w);
    sa_serve_destroy(s);
    return st;
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&b.own_stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
  b.stream = b.own_stream;
  // budget: 1/64 for thresholds (64 B per schedule step), the request states
  // (~1.1 KB each), the rest spin and coupling words
  const size_t state_bytes = (size_t)max_requests * sizeof(InstState);
  const size_t thr_bytes = budget_bytes / 64;
  if (state_bytes + thr_bytes >= budget_bytes) {
    delete s;
    return fail(SA_ERR_BUDGET, "budget too small for the request table");
  }
  const int64_t nwords = (int64_t)((budget_bytes - state_bytes - thr_bytes) / sizeof(word_t));
  const int64_t nthr = (int64_t)(thr_bytes / sizeof(BThr));
  if ((e = cudaMalloc(&b.d_spins, nwords * sizeof(word_t))) != cudaSuccess) return bail(e, "word pool");
  b.d_J = b.d_spins;
  if ((e = cudaMalloc(&b.d_thr, nthr * sizeof(BThr))) != cudaSuccess) return bail(e, "threshold pool");
  if ((e = cudaMalloc(&b.d_state, state_bytes)) != cudaSuccess) return bail(e, "state table");
  if ((e = cudaMalloc(&b.d_acc, sizeof(int64_t))) != cudaSuccess) return bail(e, "acc");
  if ((e = cudaMalloc(&b.d_att, sizeof(int64_t))) != cudaSuccess) return bail(e, "att");
  s->words.init(nwords);
  s->thr.init(nthr);
  for (int i = max_requests - 1; i >= 0; --i) s->free_states.push_back(i);
  for (int i = 0; i < 16; ++i) {
    cudaStream_t st;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    s->streams.push_back(st);
  }
  if ((e = cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
  b.finalized = true;
  s->budget = budget_bytes;
  *out = s;
  return SA_OK;
}

int sa_serve_destroy(sa_serve_t s) {
  if (!s) return SA_OK;
  sa_batch& b = s->b;
  if (b.stream) cudaStreamSynchronize(b.stream);
  for (auto st : s->streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (auto ev : s->events) cudaEventDestroy(ev);
  if (b.fork) cudaEventDestroy(b.fork);
  b.fork = nullptr;
  cudaFree(b.d_spins);
  cudaFree(b.d_thr);
  cudaFree(b.d_state);
  cudaFree(b.d_acc);
  cudaFree(b.d_att);
  cudaFree(b.d_inst);
  cudaFree(b.d_order);
  cudaFree(b.d_work);
  cudaFree(b.d_wide);
  b.d_wide = nullptr;
  b.d_spins = b.d_J = nullptr;
  b.d_thr = nullptr;
  b.d_state = nullptr;
  b.d_acc = b.d_att = nullptr;
  b.d_inst = nullptr;
  b.d_order = nullptr;
  b.d_work = nullptr;
  b.groups.clear();  // the group streams belong to s->streams
  if (b.own_stream) cudaStreamDestroy(b.own_stream);
  b.own_stream = nullptr;
  delete s;
  return SA_OK;
}

int sa_serve_set_stream(sa_serve_t s, void* stream) {
  if (!s) return fail(SA_ERR_INVALID, "null server");
  s->b.stream = stream ? (cudaStream_t)stream : s->b.own_stream;
  return SA_OK;
}

// Admits an anneal request if the pools have room now (SA_ERR_BUDGET if not).
int sa_serve_submit(sa_serve_t s, int lattice, int L, uint64_t seed_J, uint64_t seed, const double* T, int nsteps,
                    int sweeps_per_step, int64_t* id) {
  if (!s || !T || !id) return fail(SA_ERR_INVALID, "null argument");
  if (lattice < 0 || lattice > 2) return fail(SA_ERR_INVALID, "unknown lattice kind");
  if (L < 2) return fail(SA_ERR_INVALID, "L must be >= 2");
  if (L & 1) return fail(SA_ERR_ODD_L, "L must be even");
  if (nsteps < 1 || sweeps_per_step < 1) return fail(SA_ERR_INVALID, "empty schedule");
  InstDesc d;
  memset(&d, 0, sizeof d);
  const int dim = lattice_dim(lattice);
  d.lattice = lattice;
  d.L = L;
  d.N = (dim == 3) ? (int64_t)L * L * L : (int64_t)L * L;
  if (d.N > kBatchMaxN) return fail(SA_ERR_UNSUPPORTED, "request too large");
  d.half = d.N / 2;
  d.nbonds = dim * d.N - (lattice == SA_LATTICE_2D_OPEN_X ? L : 0);
  d.nslots = 1;
  d.P = 1;
  d.ladder = -1;
  d.sched = 0;
  d.seed = seed;
  d.sweeps_per_step = sweeps_per_step;
  d.thr_count = nsteps;
  d.sweep_limit = (int64_t)nsteps * sweeps_per_step;
  d.hist_off = -1;
  std::vector<BThr> thr(nsteps);
  for (int k = 0; k < nsteps; ++k) {
    if (!(T[k] > 0)) return fail(SA_ERR_INVALID, "temperatures must be > 0");
    thr[k] = to_bthr(lattice, T[k]);
  }
  if (s->free_states.empty()) return fail(SA_ERR_BUDGET, "request table full");
  const int64_t words = d.N + dim * d.N;
  const int64_t woff = s->words.alloc(words);
  if (woff < 0) return fail(SA_ERR_BUDGET, "memory budget full");
  const int64_t toff = s->thr.alloc(nsteps);
  if (toff < 0) {
    s->words.release(woff, words);
    return fail(SA_ERR_BUDGET, "threshold pool full");
  }
  const int st = s->free_states.back();
  s->free_states.pop_back();
  d.spin_off = woff;
  d.J_off = woff + d.N;
  d.thr_off = toff;
  d.state_idx = st;
  SA_CUDA_TRY(cudaMemcpyAsync(s->b.d_thr + toff, thr.data(), nsteps * sizeof(BThr), cudaMemcpyHostToDevice,
                              s->b.stream));
  SA_CUDA_TRY(cudaMemsetAsync(s->b.d_state + st, 0, sizeof(InstState), s->b.stream));
  ServeReq r;
  r.d = d;
  r.words = words;
  r.thr_n = nsteps;
  r.sweeps = 0;
  r.fresh = true;
  r.seed_J = seed_J;
  *id = s->next_id++;
  s->active.emplace(*id, r);
  SA_CUDA_TRY(cudaStreamSynchronize(s->b.stream));  // thresholds staged from pageable memory
  return SA_OK;
}

// One round: every active request advances by up to nsweeps sweeps.
int sa_serve_run(sa_serve_t s, long nsweeps) {
  if (!s || nsweeps < 1) return fail(SA_ERR_INVALID, "bad arguments");
  sa_batch& b = s->b;
  // device initialisation of the requests admitted since the last round
  std::vector<InstDesc> fresh;
  std::vector<uint64_t> fresh_seedJ;
  int64_t maxN = 0;
  for (auto& kv : s->active)
    if (kv.second.fresh) {
      fresh.push_back(kv.second.d);
      fresh_seedJ.push_back(kv.second.seed_J);
      maxN = std::max<int64_t>(maxN, kv.second.d.N);
      kv.second.fresh = false;
    }
  b.inst.clear();
  b.run_start.clear();
  for (auto& kv : s->active)
    if (kv.second.sweeps < kv.second.d.sweep_limit) {
      b.inst.push_back(kv.second.d);
      b.run_start.push_back(kv.second.sweeps);
    }
  const size_t ni = b.inst.size();
  const size_t need = std::max(ni, fresh.size());
  if (need > b.inst_cap) {
    SA_CUDA_TRY(cudaStreamSynchronize(b.stream));
    cudaFree(b.d_inst);
    cudaFree(b.d_order);
    cudaFree(b.d_seedJ);
    b.inst_cap = std::max<size_t>(need, 2 * b.inst_cap);
    SA_CUDA_TRY(cudaMalloc(&b.d_inst, b.inst_cap * sizeof(InstDesc)));
    SA_CUDA_TRY(cudaMalloc(&b.d_order, b.inst_cap * sizeof(int32_t)));
    SA_CUDA_TRY(cudaMalloc(&b.d_seedJ, b.inst_cap * sizeof(uint64_t)));
  }
  if (!fresh.empty()) {
    SA_CUDA_TRY(cudaMemcpyAsync(b.d_inst, fresh.data(), fresh.size() * sizeof(InstDesc), cudaMemcpyHostToDevice,
                                b.stream));
    SA_CUDA_TRY(cudaMemcpyAsync(b.d_seedJ, fresh_seedJ.data(), fresh.size() * sizeof(uint64_t),
                                cudaMemcpyHostToDevice, b.stream));
    dim3 g((unsigned)((maxN + 255) / 256), (unsigned)std::min<size_t>(fresh.size(), 65535));
    k_batch_init<<<g, 256, 0, b.stream>>>(b.d_inst, b.d_seedJ, (int)fresh.size(), b.d_spins, b.d_J);
    SA_CUDA_TRY(cudaGetLastError());
  }
  if (ni == 0) return SA_OK;
  std::vector<int32_t> order = build_groups(&b);
  if (int st = ensure_wide_scratch(&b)) return st;
  if (b.groups.size() > b.work_cap) {
    SA_CUDA_TRY(cudaStreamSynchronize(b.stream));
    cudaFree(b.d_work);
    b.work_cap = std::max<size_t>(b.groups.size(), 2 * b.work_cap);
    SA_CUDA_TRY(cudaMalloc(&b.d_work, b.work_cap * sizeof(int32_t)));
  }
  while (s->events.size() < b.groups.size()) {
    cudaEvent_t ev;
    SA_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    s->events.push_back(ev);
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b.device);
  for (size_t gi = 0; gi < b.groups.size(); ++gi) {
    sa_batch::Group& g = b.groups[gi];
    g.stream = s->streams[gi % s->streams.size()];
    g.done = s->events[gi];
    if (g.resident) {
      int mc = 0;
      int st = dispatch(&b, g, (int)gi, 0, 2, &mc);  // kernel attributes, once per variant
      if (st) return st;
    } else {
      g.grid = (int)std::min<int64_t>((int64_t)sms, (int64_t)g.count);
    }
  }
  // the pageable uploads below complete before the call returns
  SA_CUDA_TRY(cudaMemcpyAsync(b.d_inst, b.inst.data(), ni * sizeof(InstDesc), cudaMemcpyHostToDevice, b.stream));
  SA_CUDA_TRY(cudaMemcpyAsync(b.d_order, order.data(), ni * sizeof(int32_t), cudaMemcpyHostToDevice, b.stream));
  SA_CUDA_TRY(cudaMemsetAsync(b.d_work, 0, b.groups.size() * sizeof(int32_t), b.stream));
  SA_CUDA_TRY(cudaEventRecord(b.fork, b.stream));
  for (size_t gi = 0; gi < b.groups.size(); ++gi) {
    SA_CUDA_TRY(cudaStreamWaitEvent(b.groups[gi].stream, b.fork, 0));
    int st = dispatch(&b, b.groups[gi], (int)gi, nsweeps, 0, nullptr);
    if (st) return st;
    SA_CUDA_TRY(cudaEventRecord(b.groups[gi].done, b.groups[gi].stream));
  }
  for (size_t gi = 0; gi < b.groups.size(); ++gi) SA_CUDA_TRY(cudaStreamWaitEvent(b.stream, b.groups[gi].done, 0));
  SA_CUDA_TRY(cudaGetLastError());
  // host mirror of the progress; finished requests are reported by poll
  for (auto& kv : s->active) {
    ServeReq& r = kv.second;
    if (r.sweeps >= r.d.sweep_limit) continue;
    r.sweeps = std::min<int64_t>(r.d.sweep_limit, r.sweeps + nsweeps);
    if (r.sweeps >= r.d.sweep_limit) s->finished.push_back(kv.first);
  }
  return SA_OK;
}

int sa_serve_sync(sa_serve_t s) {
  if (!s) return fail(SA_ERR_INVALID, "null server");
  SA_CUDA_TRY(cudaStreamSynchronize(s->b.stream));
  return SA_OK;
}

// Requests that completed their schedule (their results are final once the
// rounds that finished them have completed: sync first).
int sa_serve_poll(sa_serve_t s, int64_t* ids, int cap, int* n) {
  if (!s || !n) return fail(SA_ERR_INVALID, "null argument");
  const int k = (int)std::min<size_t>((size_t)std::max(cap, 0), s->finished.size());
  for (int i = 0; i < k; ++i) ids[i] = s->finished[i];
  s->finished.erase(s->finished.begin(), s->finished.begin() + k);
  *n = k;
  return SA_OK;
}

// Result of a finished request: running max of -H per replica (int64[64]),
// the last measured -H per replica (may be NULL) and the final spins in
// row-major order (may be NULL); then frees everything it held.
int sa_serve_result(sa_serve_t s, int64_t id, int64_t* Emax, int64_t* Elast, uint64_t* spins) {
  if (!s) return fail(SA_ERR_INVALID, "null server");
  auto it = s->active.find(id);
  if (it == s->active.end()) return fail(SA_ERR_INVALID, "unknown request id");
  ServeReq& r = it->second;
  if (r.sweeps < r.d.sweep_limit) return fail(SA_ERR_INVALID, "request has not finished");
  sa_batch& b = s->b;
  InstState st;
  SA_CUDA_TRY(cudaMemcpyAsync(&st, b.d_state + r.d.state_idx, sizeof st, cudaMemcpyDeviceToHost, b.stream));
  if (spins) {
    std::vector<word_t> raw(r.d.N);
    SA_CUDA_TRY(cudaMemcpyAsync(raw.data(), b.d_spins + r.d.spin_off, r.d.N * sizeof(word_t), cudaMemcpyDeviceToHost,
                                b.stream));
    SA_CUDA_TRY(cudaStreamSynchronize(b.stream));
    const long L = r.d.L, hL = L / 2;
    for (long i = 0; i < r.d.N; ++i) {
      const long row = i / L;
      const int x = (int)(i - row * L), y = (int)(row % L), c = (x + y) & 1;
      spins[i] = raw[(long)c * r.d.half + row * hL + (x >> 1)];
    }
  }
  SA_CUDA_TRY(cudaStreamSynchronize(b.stream));
  if (Emax) memcpy(Emax, st.emax, sizeof st.emax);
  if (Elast) memcpy(Elast, st.elast, sizeof st.elast);
  s->words.release(r.d.spin_off, r.words);
  s->thr.release(r.d.thr_off, r.thr_n);
  s->free_states.push_back((int)r.d.state_idx);
  s->active.erase(it);
  return SA_OK;
}

int sa_serve_active(sa_serve_t s, int* n, long long* free_words) {
  if (!s) return fail(SA_ERR_INVALID, "null server");
  if (n) *n = (int)s->active.size();
  if (free_words) {
    long long f = 0;
    for (auto& kv : s->words.free) f += kv.second;
    *free_words = f;
  }
  return SA_OK;
}

}  // extern "C"

// ===========================================================================
// One lattice of a single system (sa_system: spins [colour][row][k] and
// couplings [axis][colour][row][k], the batch layout with one slot) run by the
// resident kernel: the whole schedule in one launch, the lattice in the shared
// memory of a cluster spread over up to 16 SMs. Zero field only (the batch
// threshold tables have no field term).
// ===========================================================================
namespace sa {

bool resident_ok(const sa_system* sy) {
  return sy->rng_mode == SA_RNG_PHILOX && sy->first_colour == 0 && !sy->split && sy->h == 0.0 && sy->L >= 4 &&
         sy->N <= kBatchMaxN;
}

int resident_run(sa_system* sy, const double* T, int nsteps, int sweeps, int stride, int64_t* Emax,
                 int64_t* step_E, int* measured) {
  if (!resident_ok(sy)) return fail(SA_ERR_UNSUPPORTED, "lattice not supported by the resident runner");
  if (nsteps < 1 || sweeps < 1 || stride < 0) return fail(SA_ERR_INVALID, "bad schedule");
  std::vector<BThr> thr(nsteps);
  for (int k = 0; k < nsteps; ++k) {
    if (!(T[k] > 0)) return fail(SA_ERR_INVALID, "temperatures must be > 0");
    thr[k] = to_bthr(sy->lattice, T[k]);
  }
  sa_batch tmp;
  tmp.device = sy->device;
  tmp.stream = sy->stream;
  InstDesc d;
  memset(&d, 0, sizeof d);
  d.lattice = sy->lattice;
  d.L = sy->L;
  d.nslots = 1;
  d.P = 1;
  d.ladder = -1;
  d.sched = 0;
  d.sweeps_per_step = sweeps;
  d.thr_count = nsteps;
  d.N = sy->N;
  d.half = sy->half;
  d.nbonds = sy->nbonds;
  d.hist_off = -1;
  d.seed = sy->seed;
  d.sweep_limit = (int64_t)nsteps * sweeps;
  tmp.inst.push_back(d);
  std::vector<int32_t> order = build_groups(&tmp);
  if (tmp.groups.size() != 1 || !(tmp.groups[0].resident || tmp.groups[0].wide))
    return fail(SA_ERR_UNSUPPORTED, "lattice does not fit a cluster's shared memory");
  // one device block: descriptor, state, order, work counter, pair counters,
  // thresholds, per-step record, wide-form scratch
  const size_t o_state = 256, o_order = o_state + ((sizeof(InstState) + 255) / 256) * 256;
  const size_t o_work = o_order + 256, o_acc = o_work + 256, o_thr = o_acc + 256;
  const size_t o_rec = o_thr + ((nsteps * sizeof(BThr) + 255) / 256) * 256;
  const size_t o_wide = o_rec + (((size_t)nsteps * 64 * sizeof(int64_t) + 255) / 256) * 256;
  const size_t bytes = o_wide + kWideScratch;
  char* blk = nullptr;
  SA_CUDA_TRY(cudaMalloc(&blk, bytes));
  auto release = [&]() { cudaFree(blk); };
  InstState st;
  memset(&st, 0, sizeof st);
  st.draw = sy->draw;
  tmp.d_inst = reinterpret_cast<InstDesc*>(blk);
  tmp.d_state = reinterpret_cast<InstState*>(blk + o_state);
  tmp.d_order = reinterpret_cast<int32_t*>(blk + o_order);
  tmp.d_work = reinterpret_cast<int32_t*>(blk + o_work);
  tmp.d_acc = reinterpret_cast<int64_t*>(blk + o_acc);
  tmp.d_att = tmp.d_acc + 1;
  tmp.d_thr = reinterpret_cast<BThr*>(blk + o_thr);
  tmp.d_spins = sy->d_s;
  tmp.d_J = sy->d_J;
  tmp.mstride = stride;
  int64_t* d_rec = reinterpret_cast<int64_t*>(blk + o_rec);
  cudaError_t e = cudaMemcpyAsync(tmp.d_inst, &d, sizeof d, cudaMemcpyHostToDevice, sy->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tmp.d_state, &st, sizeof st, cudaMemcpyHostToDevice, sy->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tmp.d_order, order.data(), sizeof(int32_t), cudaMemcpyHostToDevice, sy->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(tmp.d_work, 0, 256 + 256, sy->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tmp.d_thr, thr.data(), nsteps * sizeof(BThr), cudaMemcpyHostToDevice, sy->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_rec, 0, (size_t)nsteps * 64 * sizeof(int64_t), sy->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(blk + o_wide, 0, kWideScratch, sy->stream);
  if (e != cudaSuccess) {
    release();
    return cuda_fail(e, "resident_run set-up");
  }
  sa_batch::Group& g = tmp.groups[0];
  g.stream = sy->stream;
  int mc = 0;
  int status = SA_OK;
  if (g.wide) {
    tmp.d_wide = blk + o_wide;
    tmp.wide_cap = 1;
    tmp.run_start.assign(1, 0);
    status = launch_wide(&tmp, g, d.sweep_limit, d_rec);
    tmp.d_wide = nullptr;  // part of blk
    if (status == SA_OK) {
      e = cudaMemcpyAsync(&st, tmp.d_state, sizeof st, cudaMemcpyDeviceToHost, sy->stream);
      if (e == cudaSuccess && step_E)
        e = cudaMemcpyAsync(step_E, d_rec, (size_t)nsteps * 64 * sizeof(int64_t), cudaMemcpyDeviceToHost, sy->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(sy->stream);
      if (e != cudaSuccess) status = cuda_fail(e, "resident_run");
    }
  } else {
    status = dispatch(&tmp, g, 0, 0, 2, &mc);
  }
  if (status == SA_OK && !g.wide) {
    BatchParams prm;
    batch_params(&tmp, d.sweep_limit, &prm);
    prm.order = tmp.d_order;
    prm.ninst = 1;
    prm.work = tmp.d_work;
    prm.step_rec = d_rec;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)g.C, 1, 1);
    cfg.blockDim = dim3((unsigned)g.threads, 1, 1);
    cfg.dynamicSmemBytes = g.smem;
    cfg.stream = sy->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)g.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void (*kern)(BatchParams) = resident_kernel<1>(g);
    e = cudaLaunchKernelEx(&cfg, kern, prm);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&st, tmp.d_state, sizeof st, cudaMemcpyDeviceToHost, sy->stream);
    if (e == cudaSuccess && step_E)
      e = cudaMemcpyAsync(step_E, d_rec, (size_t)nsteps * 64 * sizeof(int64_t), cudaMemcpyDeviceToHost, sy->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sy->stream);
    if (e != cudaSuccess) status = cuda_fail(e, "resident_run");
  }
  release();
  if (status != SA_OK) return status;
  if (Emax) memcpy(Emax, st.emax, sizeof st.emax);
  if (measured) *measured = (int)st.measured;
  sy->draw = st.draw;
  return SA_OK;
}

}  // namespace sa
