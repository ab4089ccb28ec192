// sa_resident.cuh -- the shared-memory-resident batched kernel.
//
// One instance (all its slots) is held in the shared memory of a thread-block
// cluster of C CTAs for a whole launch: CTA q owns ny_q consecutive y-rows
// starting at y0_q (ny_q = L/C, plus one for the first L%C CTAs) of every
// z-plane and both colours, layout
//   [colour][z][y_local][k][slot]            (k = x/2, slot innermost)
// and reads the two halo rows it needs (y0-1, y0+ny) from the neighbouring
// CTAs' shared memory over DSMEM (whose layouts use their own row counts). Couplings stay in global memory (L2) and
// are shared by the slots of a site. Between half-sweeps the cluster
// synchronises; the replica exchange sums per-CTA energy partials over DSMEM,
// so every CTA reaches the same decision and swaps its own rows.
//
// Spins go HBM -> shared memory once at the start of a launch and back once at
// the end, so a launch of S sweeps moves 2*8 bytes per site and slot through
// HBM instead of ~24*S.
#pragma once
#include <cooperative_groups.h>

#include <type_traits>

#include "sa_batch.hpp"
#include "sa_device.cuh"

namespace sa {

namespace cg = cooperative_groups;

constexpr int kResMaxWarps = 20;  // 5 warps per SM sub-partition at <= 96 registers
constexpr int kResMaxThreads = kResMaxWarps * 32;
// the segmented single-slot 3D variant trades threads for registers (its
// segment maps stay in registers): 16 warps at up to 128 registers
constexpr int kSegMaxThreads = 512;
// the high-register form of the two-slot 3D walk: 12 warps, ~170 registers
constexpr int kHiRegThreads = 384;
// two-slot 2D lanes in clusters of two or more CTAs (the large 2D lattices):
// at most 8 warps, launched for two blocks per SM, so up to 128 registers and
// the walk's words stay in registers (at 96 registers they spilled)
constexpr int kRes2dClThreads = 256;

struct ResCtx {
  word_t* sm;           // this CTA's rows
  const word_t* smN;    // CTA owning row y0-1 (generic pointer; self when C == 1)
  const word_t* smS;    // CTA owning row y0+ny
  const word_t* J;      // instance couplings [axis][colour][row][k] (global)
  uint64_t seed;
  int L, hL, ny, y0, ns, zc;  // zc: z-planes (L in 3D, 1 in 2D)
  int nyN, nyS;               // rows held by the CTAs owning y0-1 and y0+ny
  uint32_t smNA, smSA;        // shared::cluster byte addresses of those CTAs' spins
  int swm, swsh;              // slot swizzle: slot s of site k sits at s ^ ((k << swsh) & swm)
  int half;                   // sites per colour of the instance (global J stride)
  int rowW;                   // words per local row: hL*ns
  uint32_t magic;             // floor(2^32/hL)+1, for division by hL
};

// t / hL for t < 2^20, hL <= 2^11, with one correction step.
__device__ __forceinline__ int div_hl(int t, const ResCtx& x) {
  int q = (int)__umulhi((unsigned)t, x.magic);
  if ((q + 1) * x.hL <= t) ++q;
  if (q * x.hL > t) --q;
  return q;
}

// local word offset of (colour, z, y_local) row start
__device__ __forceinline__ int lrow(const ResCtx& x, int c, int z, int yl) {
  return ((c * x.zc + z) * x.ny + yl) * x.rowW;
}

// Slot swizzle. Slots are innermost (a site's ns words are contiguous), so a
// warp reading ONE slot of many sites (the exchange energies, the swap) would
// hit the same two banks ns/2-fold. With a power-of-two slot count the slot
// index is XORed with the site's k (in pairs when lanes access two slots at
// once), which keeps a site's words in its own ns-word block while spreading
// one slot over all banks.
__device__ __forceinline__ int swz(const ResCtx& x, int k) { return (k << x.swsh) & x.swm; }

// the halo rows: last row of the north neighbour, first row of the south one
__device__ __forceinline__ int lrow_n(const ResCtx& x, int c, int z) {
  return ((c * x.zc + z) * x.nyN + x.nyN - 1) * x.rowW;
}
__device__ __forceinline__ int lrow_s(const ResCtx& x, int c, int z) {
  return ((c * x.zc + z) * x.nyS) * x.rowW;
}

// SL consecutive slot words of one site (SL = 2: one 16-byte access).
template <int SL>
struct SlotWords {
  word_t w[SL];
};

template <int SL>
__device__ __forceinline__ SlotWords<SL> ldw(const word_t* p) {
  SlotWords<SL> r;
  if (SL == 2) {
    const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(p);
    r.w[0] = v.x;
    r.w[SL - 1] = v.y;
  } else {
    r.w[0] = p[0];
  }
  return r;
}

template <int SL>
__device__ __forceinline__ void stw(word_t* p, const SlotWords<SL>& v) {
  if (SL == 2) *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(v.w[0], v.w[SL - 1]);
  else p[0] = v.w[0];
}

// Cluster shared-memory access. A neighbour row is read through its 32-bit
// shared::cluster address with ld.shared::cluster (a local row's shared::cta
// address is a valid cluster address of the executing CTA), so the loads keep
// 32-bit address arithmetic and never go through generic addressing.
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t cluster_addr(uint32_t a, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}

template <int SL>
__device__ __forceinline__ SlotWords<SL> ldc(uint32_t a) {
  SlotWords<SL> r;
  if (SL == 2) {
    unsigned long long v0, v1;
    asm volatile("ld.shared::cluster.v2.u64 {%0, %1}, [%2];" : "=l"(v0), "=l"(v1) : "r"(a));
    r.w[0] = v0;
    r.w[SL - 1] = v1;
  } else {
    unsigned long long v0;
    asm volatile("ld.shared::cluster.u64 %0, [%1];" : "=l"(v0) : "r"(a));
    r.w[0] = v0;
  }
  return r;
}

// A row of the other colour north or south of a site row: local, or (CL)
// possibly in the neighbouring CTA. off / step are in words.
template <bool CL>
struct NbRow;

template <>
struct NbRow<false> {
  const word_t* p;
  template <int SL>
  __device__ __forceinline__ SlotWords<SL> ld(int off) const { return ldw<SL>(p + off); }
  __device__ __forceinline__ void step(int words) { p += words; }
};

template <>
struct NbRow<true> {
  uint32_t a;
  template <int SL>
  __device__ __forceinline__ SlotWords<SL> ld(int off) const { return ldc<SL>(a + 8u * (uint32_t)off); }
  __device__ __forceinline__ void step(int words) { a += 8u * (uint32_t)words; }
};

// row y_local-1 (north) / y_local+1 (south) of colour oc in plane z
template <bool CL>
__device__ __forceinline__ NbRow<CL> north_row(const ResCtx& x, int oc, int z, int yl) {
  NbRow<CL> r;
  if constexpr (CL) {
    r.a = (yl > 0) ? smem_addr(x.sm + lrow(x, oc, z, yl - 1)) : x.smNA + 8u * (uint32_t)lrow_n(x, oc, z);
  } else {
    r.p = (yl > 0) ? x.sm + lrow(x, oc, z, yl - 1) : x.smN + lrow_n(x, oc, z);
  }
  return r;
}

template <bool CL>
__device__ __forceinline__ NbRow<CL> south_row(const ResCtx& x, int oc, int z, int yl) {
  NbRow<CL> r;
  if constexpr (CL) {
    r.a = (yl < x.ny - 1) ? smem_addr(x.sm + lrow(x, oc, z, yl + 1)) : x.smSA + 8u * (uint32_t)lrow_s(x, oc, z);
  } else {
    r.p = (yl < x.ny - 1) ? x.sm + lrow(x, oc, z, yl + 1) : x.smS + lrow_s(x, oc, z);
  }
  return r;
}

// Lanes: (site group lane/P, slots (lane%P)*SL .. +SL-1). All slots of a site
// share the coupling loads and the site's Philox draw; SL > 1 requires an
// even slot count (16-byte aligned slot pairs).
template <int P, int SL, bool OPEN_X, bool CL>
__device__ __forceinline__ void rhalf_2d(const ResCtx& x, int c, uint64_t draw, const uint32_t (*th)[8],
                                         const uint32_t (*tb)[8]) {
  constexpr int SPS = 32 / P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // Clustered instances (BF): a lane without a slot (or a site) updates
  // slot 0 (site 0) of the CTA, reading only, and drops its store, so the
  // update has no divergent branch (measured faster there, and slower for
  // single-CTA instances).
  constexpr bool BF = CL;
  const bool slot_ok = (lane % P) * SL < x.ns;
  const int slot = (BF && !slot_ok) ? 0 : (lane % P) * SL;
  const int tot = x.ny * x.hL;
  const int L = x.L, hL = x.hL, ns = x.ns;
  const int oc = 1 - c;
  const word_t* Jxc = x.J + (long)(0 + c) * x.half;
  const word_t* Jxo = x.J + (long)(1 - c) * x.half;
  const word_t* Jyc = x.J + (long)(2 + c) * x.half;
  const word_t* Jyo = x.J + (long)(3 - c) * x.half;
  for (int base = warp * 32; base < tot; base += nwarps * 32) {
    // Lane i of the warp prepares site base+i once: its Philox draw, its four
    // coupling words, its row offsets, its neighbours' swizzles and its border
    // flags. The P lanes updating that site's slots fetch them by shuffles
    // instead of each recomputing the indices and reloading the couplings.
    const bool have = base + lane < tot;
    const int my = (BF && !have) ? 0 : base + lane;
    uint32_t um = 0, pk = 0, nadr = 0, sadr = 0;
    int rowc = 0, roww = 0, rowe = 0;
    word_t bw = 0, be = 0, bn = 0, bs = 0;
    if (BF || have) {
      const int yl = div_hl(my, x);
      const int k = my - yl * hL, y = x.y0 + yl;
      const int par = (c + y) & 1, xx = 2 * k + par;
      int kw, ke;
      x_neighbours(k, par, hL, kw, ke);
      const int ys = (y == L - 1) ? 0 : y + 1;
      um = philox_draw(x.seed, (unsigned long long)(xx + L * y), draw);
      bw = __ldg(Jxc + y * hL + k);
      be = __ldg(Jxo + y * hL + ke);
      bn = __ldg(Jyc + y * hL + k);
      bs = __ldg(Jyo + ys * hL + k);
      rowc = lrow(x, c, 0, yl) + k * ns;
      roww = lrow(x, oc, 0, yl) + kw * ns;
      rowe = lrow(x, oc, 0, yl) + ke * ns;
      // swizzles (< 32) of k, kw, ke and the border flags in one word
      pk = (uint32_t)swz(x, k) | ((uint32_t)swz(x, kw) << 8) | ((uint32_t)swz(x, ke) << 16) |
           ((OPEN_X && xx == 0) ? (1u << 24) : 0u) | ((OPEN_X && xx == L - 1) ? (1u << 25) : 0u);
      const NbRow<CL> pn = north_row<CL>(x, oc, 0, yl), ps = south_row<CL>(x, oc, 0, yl);
      if constexpr (CL) {
        nadr = pn.a + 8u * (uint32_t)(k * ns);
        sadr = ps.a + 8u * (uint32_t)(k * ns);
      } else {
        nadr = (uint32_t)(pn.p - x.sm) + (uint32_t)(k * ns);  // word offsets in this CTA
        sadr = (uint32_t)(ps.p - x.sm) + (uint32_t)(k * ns);
      }
    }
    // A warp whose 32 sites all exist and whose lanes all have a slot (every
    // warp but the last of the batched ensembles) updates without the
    // per-lane test.
    const bool all_upd = base + 32 <= tot && __all_sync(0xffffffffu, slot_ok);
    auto subs = [&](auto check) {
    constexpr bool CHECK = decltype(check)::value;
#pragma unroll 1
    for (int sub = 0; sub < P; ++sub) {
      const int sl = sub * SPS + lane / P;
      // one lane per site (P = 1): the lane's own values
      auto share = [&](auto v) { return (P == 1) ? v : __shfl_sync(0xffffffffu, v, sl); };
      const uint32_t u = share(um);
      const word_t jw = share(bw), je = share(be), jn = share(bn), js = share(bs);
      const int rc = share(rowc), rw = share(roww), re = share(rowe);
      const uint32_t f = share(pk), na = share(nadr), sa = share(sadr);
      const int t = base + sl;
      const bool upd = t < tot && slot_ok;
      if (!CHECK || BF || upd) {
        const int sk = slot ^ (int)(f & 0xFFu);
        const int own = rc + sk;
        const SlotWords<SL> si = ldw<SL>(x.sm + own);
        const SlotWords<SL> sw = ldw<SL>(x.sm + rw + (slot ^ (int)((f >> 8) & 0xFFu)));
        const SlotWords<SL> se = ldw<SL>(x.sm + re + (slot ^ (int)((f >> 16) & 0xFFu)));
        SlotWords<SL> sn, ss;
        if constexpr (CL) {
          sn = ldc<SL>(na + 8u * (uint32_t)sk);
          ss = ldc<SL>(sa + 8u * (uint32_t)sk);
        } else {
          sn = ldw<SL>(x.sm + na + sk);
          ss = ldw<SL>(x.sm + sa + sk);
        }
        const bool bwest = OPEN_X && (f & (1u << 24));
        const bool beast = OPEN_X && (f & (1u << 25));
        const bool border = bwest || beast;
        SlotWords<SL> out;
#pragma unroll
        for (int q = 0; q < SL; ++q) {
          word_t mw = jw ^ sw.w[q] ^ si.w[q];
          word_t me = je ^ se.w[q] ^ si.w[q];
          const word_t mn = jn ^ sn.w[q] ^ si.w[q];
          const word_t ms = js ^ ss.w[q] ^ si.w[q];
          if (OPEN_X) {
            if (bwest) mw = ~0ULL;
            if (beast) me = ~0ULL;
          }
          word_t c0, c1, c2;
          count4(mw, me, mn, ms, c0, c1, c2);
          uint32_t m0, m1, m2;
          prefix_bits(u, border ? tb[q] : th[q], m0, m1, m2);
          out.w[q] = flip_below(si.w[q], c0, c1, c2, m0, m1, m2);
        }
        if (!CHECK || !BF || upd) stw<SL>(x.sm + own, out);
      }
    }
    };
    if (all_upd) subs(std::false_type{});
    else subs(std::true_type{});
  }
}

// DB (the high-register form, which has registers to spare): the next plane
// block's Philox draw and coupling words are fetched while this block walks,
// so the L2 round trip of every block but the first is hidden.
template <int P, int SL, bool CL, bool DB = false>
__device__ __forceinline__ void rhalf_3d(const ResCtx& x, int c, uint64_t draw, const uint32_t (*th)[8]) {
  constexpr int SPS = 32 / P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int slot = (lane % P) * SL, cl = lane / P;
  const bool slot_ok = slot < x.ns;
  const int L = x.L, hL = x.hL, ns = x.ns;
  const int cols = x.ny * hL;
  const int oc = 1 - c;
  const int zs = x.ny * x.rowW;   // local z stride
  const int zg = L * hL;          // global z stride of the coupling arrays
  const word_t* Jxc = x.J + (long)(0 + c) * x.half;
  const word_t* Jxo = x.J + (long)(1 - c) * x.half;
  const word_t* Jyc = x.J + (long)(2 + c) * x.half;
  const word_t* Jyo = x.J + (long)(3 - c) * x.half;
  const word_t* Jzc = x.J + (long)(4 + c) * x.half;
  for (int cb = warp * SPS; cb < cols; cb += nwarps * SPS) {
    const int col = cb + cl;
    const bool col_ok = col < cols;
    const bool valid = col_ok && slot_ok;
    const int yl = col_ok ? div_hl(col, x) : 0;
    const int k = col_ok ? col - yl * hL : 0;
    const int y = x.y0 + yl;
    const int par = (c + y) & 1, xx = 2 * k + par;
    int kw, ke;
    x_neighbours(k, par, hL, kw, ke);
    const int ys = (y == L - 1) ? 0 : y + 1;
    // z = 0 offsets; every z step adds zs (shared) or zg (couplings)
    const int sk = slot ^ swz(x, k);
    int own = lrow(x, c, 0, yl) + k * ns + sk;
    int ow = lrow(x, oc, 0, yl) + kw * ns + (slot ^ swz(x, kw));
    int oe = lrow(x, oc, 0, yl) + ke * ns + (slot ^ swz(x, ke));
    NbRow<CL> pn = north_row<CL>(x, oc, 0, yl), ps = south_row<CL>(x, oc, 0, yl);
    pn.step(k * ns + sk);
    ps.step(k * ns + sk);
    const int zsn = (yl > 0) ? zs : x.nyN * x.rowW;       // z stride of the north row's owner
    const int zss = (yl < x.ny - 1) ? zs : x.nyS * x.rowW;
    const int jo = y * hL + k, je = y * hL + ke, js = ys * hL + k;
    SlotWords<SL> prev = {};
    if (valid) prev = ldw<SL>(x.sm + own + (L - 1) * zs);
    SlotWords<SL> first = {};
    // the plane's own words: plane 0's loaded here, every later plane's as
    // the z+1 neighbour of the plane below (only this lane writes them)
    SlotWords<SL> cur = {};
    if (valid) cur = ldw<SL>(x.sm + own);
    word_t jnext = __ldg(Jzc + jo);  // the z-1 coupling of the next plane (plane 0: the wrapped bond)
    // Lane (column cl, i) draws the Philox number and loads the coupling
    // words of plane z0+i of a block; the column's P lanes share them by
    // shuffles, so each coupling word is loaded once per site instead of once
    // per slot. A plane's z-1 coupling is the z+1 coupling of the plane below;
    // plane 0's (the wrapped bond) every lane loads before the walk.
    auto fetch = [&](int z0, uint32_t& u_, word_t& w_, word_t& e_, word_t& n_, word_t& s_, word_t& d_) {
      const int zd = z0 + (lane % P);
      u_ = 0;
      w_ = e_ = n_ = s_ = d_ = 0;
      if (col_ok && zd < L) {
        const int zo = zd * zg;
        w_ = __ldg(Jxc + jo + zo);
        e_ = __ldg(Jxo + je + zo);
        n_ = __ldg(Jyc + jo + zo);
        s_ = __ldg(Jyo + js + zo);
        d_ = __ldg(Jzc + jo + ((zd == L - 1) ? 0 : zo + zg));
        u_ = philox_draw(x.seed, (unsigned long long)(xx + L * (y + L * zd)), draw);
      }
    };
    uint32_t um = 0;
    word_t bw = 0, be = 0, bn = 0, bs = 0, bd = 0;
    if constexpr (DB) fetch(0, um, bw, be, bn, bs, bd);
    // A warp whose lanes all have a site and a slot (every warp of the
    // batched ensembles) walks without the per-lane test.
    auto walk = [&](auto check) {
    constexpr bool CHECK = decltype(check)::value;
    for (int z0 = 0; z0 < L; z0 += P) {
      [[maybe_unused]] uint32_t um2 = 0;
      [[maybe_unused]] word_t bw2 = 0, be2 = 0, bn2 = 0, bs2 = 0, bd2 = 0;
      if constexpr (DB) {
        if (z0 + P < L) fetch(z0 + P, um2, bw2, be2, bn2, bs2, bd2);
      } else {
        fetch(z0, um, bw, be, bn, bs, bd);
      }
      // One plane. POS 1: plane 0 (its new words are the top plane's z+1
      // neighbours); 2: plane L-1 (its z+1 neighbour is the new plane 0);
      // 0: any other. The position is known where the step is placed, so a
      // step carries no test of z.
      auto step = [&](int zi, auto pos) {
        constexpr int POS = decltype(pos)::value;
        const int src = cl * P + zi;
        // one lane per site (P = 1): the lane's own draw and couplings
        const uint32_t u = (P == 1) ? um : __shfl_sync(0xffffffffu, um, src);
        const word_t jw = (P == 1) ? bw : __shfl_sync(0xffffffffu, bw, src);
        const word_t je_ = (P == 1) ? be : __shfl_sync(0xffffffffu, be, src);
        const word_t jn = (P == 1) ? bn : __shfl_sync(0xffffffffu, bn, src);
        const word_t js_ = (P == 1) ? bs : __shfl_sync(0xffffffffu, bs, src);
        const word_t ju = jnext;
        const word_t jd = (P == 1) ? bd : __shfl_sync(0xffffffffu, bd, src);
        jnext = jd;
        if (!CHECK || valid) {
          const SlotWords<SL> si = cur;
          const SlotWords<SL> sd = (POS == 2) ? first : ldw<SL>(x.sm + own + zs);
          const SlotWords<SL> sw = ldw<SL>(x.sm + ow);
          const SlotWords<SL> se = ldw<SL>(x.sm + oe);
          const SlotWords<SL> sn = pn.template ld<SL>(0);
          const SlotWords<SL> ss = ps.template ld<SL>(0);
          SlotWords<SL> nsw;
#pragma unroll
          for (int q = 0; q < SL; ++q) {
            word_t c0, c1, c2;
            count6(jw ^ sw.w[q] ^ si.w[q], je_ ^ se.w[q] ^ si.w[q], jn ^ sn.w[q] ^ si.w[q],
                   js_ ^ ss.w[q] ^ si.w[q], ju ^ prev.w[q] ^ si.w[q], jd ^ sd.w[q] ^ si.w[q], c0, c1, c2);
            uint32_t m0, m1, m2;
            prefix_bits(u, th[q], m0, m1, m2);
            nsw.w[q] = flip_below(si.w[q], c0, c1, c2, m0, m1, m2);
          }
          stw<SL>(x.sm + own, nsw);
          if (POS == 1) first = nsw;
          prev = nsw;
          cur = sd;
        }
        own += zs;
        ow += zs;
        oe += zs;
        pn.step(zsn);
        ps.step(zss);
      };
      const int nz = min(P, L - z0);             // planes in this block (warp-uniform)
      const bool top = (z0 + nz == L);           // the block holds plane L-1
      int zi = 0;
      if (z0 == 0) {
        step(0, std::integral_constant<int, 1>{});
        zi = 1;
      }
      const int zend = top ? nz - 1 : nz;
#pragma unroll 4
      for (; zi < zend; ++zi) step(zi, std::integral_constant<int, 0>{});
      if (top) step(nz - 1, std::integral_constant<int, 2>{});
      if constexpr (DB) {
        um = um2;
        bw = bw2;
        be = be2;
        bn = bn2;
        bs = bs2;
        bd = bd2;
      }
    }
    };
    if (__all_sync(0xffffffffu, valid)) walk(std::false_type{});
    else walk(std::true_type{});
  }
}

// Satisfied-bond count of five bond words, bit-sliced (c2 c1 c0, 0..5).
__device__ __forceinline__ void count5(word_t a, word_t b, word_t c, word_t d, word_t e, word_t& c0, word_t& c1,
                                       word_t& c2) {
  const word_t s1 = a ^ b ^ c;
  const word_t k1 = (a & b) | (c & (a ^ b));
  const word_t s2 = d ^ e;
  const word_t k2 = d & e;
  c0 = s1 ^ s2;
  const word_t k3 = s1 & s2;
  c1 = k1 ^ k2 ^ k3;
  c2 = (k1 & k2) | (k3 & (k1 ^ k2));
}

// Replicas whose bit-sliced count (c2 c1 c0) is below the scalar t (bits
// broadcast as masks m2 m1 m0).
__device__ __forceinline__ word_t below(word_t c0, word_t c1, word_t c2, uint32_t m0, uint32_t m1, uint32_t m2) {
  uint32_t r[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t a0 = (uint32_t)(c0 >> (32 * h)), a1 = (uint32_t)(c1 >> (32 * h));
    const uint32_t a2 = (uint32_t)(c2 >> (32 * h));
    const uint32_t g0 = a0 | ~m0;
    const uint32_t g1 = (a1 & ~m1) | (~(a1 ^ m1) & g0);
    r[h] = ~((a2 & ~m2) | (~(a2 ^ m2) & g1));
  }
  return (word_t)r[0] | ((word_t)r[1] << 32);
}

// Per-lane satisfied-bond counter of the fused single-slot measurement: a
// 5-plane counter (values < 32) that takes adds of at most 5 and flushes into
// an 11-plane one before it could overflow. A lane's count over one measured
// sweep stays below 2048 (the kernel checks the bound before fusing).
struct BondCount {
  VCount<5> sm;
  VCount<11> big;
  int cap;  // largest value sm can hold now
  __device__ __forceinline__ void clear() {
    sm.clear();
    big.clear();
    cap = 0;
  }
  __device__ __forceinline__ void flush() {
    word_t carry = 0;
#pragma unroll
    for (int b = 0; b < 11; ++b) {
      const word_t q = (b < 5) ? sm.p[b] : 0;
      const word_t a = big.p[b];
      big.p[b] = a ^ q ^ carry;
      carry = (a & q) | (carry & (a ^ q));
    }
    sm.clear();
    cap = 0;
  }
  // += the 3-plane count (q2 q1 q0) <= 5
  __device__ __forceinline__ void add3(word_t q0, word_t q1, word_t q2) {
    if (cap + 5 > 31) flush();
    const word_t s0 = sm.p[0] ^ q0, k0 = sm.p[0] & q0;
    const word_t t1 = sm.p[1] ^ q1, k1 = (sm.p[1] & q1) | (k0 & t1);
    const word_t t2 = sm.p[2] ^ q2, k2 = (sm.p[2] & q2) | (k1 & t2);
    sm.p[0] = s0;
    sm.p[1] = t1 ^ k0;
    sm.p[2] = t2 ^ k1;
    const word_t k3 = sm.p[3] & k2;
    sm.p[3] ^= k2;
    sm.p[4] ^= k3;
    cap += 5;
  }
  // += one bond bit
  __device__ __forceinline__ void add1(word_t q) {
    if (cap + 1 > 31) flush();
    sm.add(q);
    cap += 1;
  }
};

// Single-slot 3D half-sweep. Sites of one colour in one (x, y) column depend
// on each other along z (the colour is (x+y)%2, so a site's z-1 neighbour has
// its colour and is updated first). The walk is split in two phases per chunk
// of Z planes: first every site's update is reduced to an affine map of the
// one new value it depends on, the new z-1 spin x:
//   new = A ^ (x & B),   A = s ^ f0,  B = f0 ^ f1,
// with f0 / f1 the flips for x = 0 / 1 (the z-1 bond then counts g = J^s or
// its complement, so f0 = g ? hi : lo and B = lo ^ hi, where lo / hi are the
// flips with that bond unsatisfied / satisfied). The maps read only old
// values, so their loads and Philox draws are independent; the chain then
// applies Z maps at two logic operations each. The top plane's z+1
// neighbour is the new z = 0 spin, known once the first chunk is applied
// (requires L > Z).
//
// Fused measurement (bc != null): -H after a sweep is counted from values the
// walk already holds, every bond once. cmode 1 (the next sweep's colour-0
// half, before its updates): each colour-0 site adds its four in-plane bonds
// (all of them lead to colour 1) and its old bond to z+1, the top plane its
// in-plane bonds only and the bottom plane the wrapped bond to the old top.
// cmode 2 (the measured sweep's colour-1 half): each colour-1 site adds its
// new bond to z-1, the top plane also the new wrapped bond to z = 0.
template <int Z, bool CL>
__device__ __forceinline__ void rhalf_3d1(const ResCtx& x, int c, uint64_t draw, const uint32_t* th,
                                          BondCount* bc = nullptr, int cmode = 0) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int L = x.L, hL = x.hL;
  const int cols = x.ny * hL;
  const int oc = 1 - c;
  const int zs = x.ny * x.rowW;  // local z stride (rowW == hL)
  const int zg = L * hL;         // z stride of the coupling arrays
  const word_t* Jxc = x.J + (long)(0 + c) * x.half;
  const word_t* Jxo = x.J + (long)(1 - c) * x.half;
  const word_t* Jyc = x.J + (long)(2 + c) * x.half;
  const word_t* Jyo = x.J + (long)(3 - c) * x.half;
  const word_t* Jzc = x.J + (long)(4 + c) * x.half;
  for (int cb = warp * 32; cb < cols; cb += nwarps * 32) {
    const int col = cb + lane;
    if (col >= cols) break;  // the last columns; nothing below is warp-collective
    const int yl = div_hl(col, x);
    const int k = col - yl * hL;
    const int y = x.y0 + yl;
    const int par = (c + y) & 1, xx = 2 * k + par;
    int kw, ke;
    x_neighbours(k, par, hL, kw, ke);
    const int ys = (y == L - 1) ? 0 : y + 1;
    const word_t* own = x.sm + lrow(x, c, 0, yl) + k;
    const word_t* pw = x.sm + lrow(x, oc, 0, yl) + kw;
    const word_t* pe = x.sm + lrow(x, oc, 0, yl) + ke;
    NbRow<CL> pn = north_row<CL>(x, oc, 0, yl), ps = south_row<CL>(x, oc, 0, yl);
    pn.step(k);
    ps.step(k);
    const int zsn = (yl > 0) ? zs : x.nyN * x.rowW;
    const int zss = (yl < x.ny - 1) ? zs : x.nyS * x.rowW;
    const int jo = y * hL + k, je = y * hL + ke, js = ys * hL + k;
    const unsigned long long site0 = (unsigned long long)(xx + L * y), plane = (unsigned long long)L * L;
    word_t* own_w = const_cast<word_t*>(own);
    word_t prev = own[(L - 1) * zs];  // old top spin: the z-1 neighbour of z = 0
    word_t first = 0;
    word_t jlast = 0;  // coupling of the wrapped bond (L-1, 0)
    for (int z0 = 0; z0 < L; z0 += Z) {
      word_t A[Z], B[Z], JU[Z];
#pragma unroll
      for (int i = 0; i < Z; ++i) {
        const int z = z0 + i;
        A[i] = 0;
        B[i] = 0;
        JU[i] = 0;
        if (z < L) {
          const bool last = (z == L - 1);
          const int zn = last ? 0 : z + 1;
          const word_t si = own[z * zs];
          const word_t sd = last ? first : own[zn * zs];
          const word_t sw = pw[z * zs], se = pe[z * zs];
          const word_t sn = pn.template ld<1>(z * zsn).w[0], ss = ps.template ld<1>(z * zss).w[0];
          const word_t jw = __ldg(Jxc + jo + z * zg), jee = __ldg(Jxo + je + z * zg);
          const word_t jn = __ldg(Jyc + jo + z * zg), jss = __ldg(Jyo + js + z * zg);
          const word_t ju = __ldg(Jzc + jo + z * zg), jd = __ldg(Jzc + jo + zn * zg);
          const uint32_t u = philox_draw(x.seed, site0 + plane * (unsigned)z, draw);
          word_t c0, c1, c2;
          count5(jw ^ sw ^ si, jee ^ se ^ si, jn ^ sn ^ si, jss ^ ss ^ si, jd ^ sd ^ si, c0, c1, c2);
          uint32_t m0, m1, m2;
          prefix_bits(u, th, m0, m1, m2);
          // t - 1 (or 0): the prefix once the z-1 bond counts as satisfied
          const uint32_t t = (m0 & 1u) | (m1 & 2u) | (m2 & 4u);
          const uint32_t t1 = t ? t - 1 : 0;
          const word_t lo = below(c0, c1, c2, m0, m1, m2);
          const word_t hi = below(c0, c1, c2, (t1 & 1u) ? ~0u : 0u, (t1 & 2u) ? ~0u : 0u, (t1 & 4u) ? ~0u : 0u);
          const word_t g = ju ^ si;
          const word_t f0 = (g & hi) | (~g & lo);
          A[i] = si ^ f0;
          B[i] = lo ^ hi;
          JU[i] = ju;
          if (last) jlast = jd;
          if (cmode == 1) {
            if (!last) {
              bc->add3(c0, c1, c2);
            } else {
              word_t d0, d1, d2;
              count4(jw ^ sw ^ si, jee ^ se ^ si, jn ^ sn ^ si, jss ^ ss ^ si, d0, d1, d2);
              bc->add3(d0, d1, d2);
            }
            if (z == 0) bc->add1(g ^ prev);  // prev is still the old top spin
          }
        }
      }
#pragma unroll
      for (int i = 0; i < Z; ++i) {
        const int z = z0 + i;
        if (z < L) {
          const word_t v = A[i] ^ (prev & B[i]);
          if (cmode == 2) {
            if (z > 0) bc->add1(JU[i] ^ prev ^ v);
            if (z == L - 1) bc->add1(jlast ^ v ^ first);
          }
          prev = v;
          own_w[z * zs] = v;
          if (z == 0) first = v;
        }
      }
    }
  }
}

// Lanes per column of the segmented single-slot 3D half-sweep: the smallest
// power of two that leaves at most kSegMax planes per lane.
constexpr int kSegMax = 4;
__host__ __device__ constexpr int seg_lanes(int L) {
  return L <= kSegMax ? 1 : L <= 2 * kSegMax ? 2 : L <= 4 * kSegMax ? 4 : L <= 8 * kSegMax ? 8 : 16;
}

// Single-slot 3D half-sweep with every column's z-walk split over G lanes,
// for instances spread over many SMs (few instances: latency, not throughput,
// is the limit). Each site's update is an affine map of the new spin below it
// (see rhalf_3d1): new = A ^ (x & B). Lane g of a column forms the maps of
// its segment of planes (<= kSegMax, loads and draws independent), composes
// them into one segment map, and an exclusive scan over the column's G lanes
// (shuffles) gives every segment its input; the chain into segment 0 is the
// old top spin. The top plane's z+1 neighbour is the new z = 0 spin, which
// segment 0 knows after its first map and shares before the other maps are
// formed. A column's lanes are in one warp and all of them finish reading
// old values before the scan, so the writes after it cannot race with them.
template <bool CL>
__device__ __forceinline__ void rhalf_3d1s(const ResCtx& x, int c, uint64_t draw, const uint32_t* th) {
  const int G = seg_lanes(x.L);
  const int CPW = 32 / G;  // columns per warp pass
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane % G, cl = lane / G, lead = cl * G;
  const int L = x.L, hL = x.hL;
  const int cols = x.ny * hL;
  const int oc = 1 - c;
  const int zs = x.ny * x.rowW;  // local z stride (rowW == hL)
  const int zg = L * hL;         // z stride of the coupling arrays
  // segment g: planes [z0, z0 + ls), sizes as even as L allows (ls >= 2)
  const int sbase = L / G, srem = L % G;
  const int ls = sbase + (g < srem ? 1 : 0);
  const int z0 = g * sbase + min(g, srem);
  const word_t* Jxc = x.J + (long)(0 + c) * x.half;
  const word_t* Jxo = x.J + (long)(1 - c) * x.half;
  const word_t* Jyc = x.J + (long)(2 + c) * x.half;
  const word_t* Jyo = x.J + (long)(3 - c) * x.half;
  const word_t* Jzc = x.J + (long)(4 + c) * x.half;
  for (int cb = warp * CPW; cb < cols; cb += nwarps * CPW) {  // warp-uniform
    const int col = cb + cl;
    const bool col_ok = col < cols;
    const int cc = col_ok ? col : 0;
    const int yl = div_hl(cc, x);
    const int k = cc - yl * hL;
    const int y = x.y0 + yl;
    const int par = (c + y) & 1, xx = 2 * k + par;
    int kw, ke;
    x_neighbours(k, par, hL, kw, ke);
    const int ys = (y == L - 1) ? 0 : y + 1;
    word_t* own = x.sm + lrow(x, c, 0, yl) + k;
    const word_t* pw = x.sm + lrow(x, oc, 0, yl) + kw;
    const word_t* pe = x.sm + lrow(x, oc, 0, yl) + ke;
    NbRow<CL> pn = north_row<CL>(x, oc, 0, yl), ps = south_row<CL>(x, oc, 0, yl);
    pn.step(k);
    ps.step(k);
    const int zsn = (yl > 0) ? zs : x.nyN * x.rowW;
    const int zss = (yl < x.ny - 1) ? zs : x.nyS * x.rowW;
    const int jo = y * hL + k, je = y * hL + ke, js = ys * hL + k;
    const unsigned long long site0 = (unsigned long long)(xx + L * y), plane = (unsigned long long)L * L;
    // the old top spin: the chain's input below z = 0
    const word_t top = __shfl_sync(0xffffffffu, (col_ok && g == 0) ? own[(L - 1) * zs] : 0ULL, lead);
    word_t A[kSegMax], B[kSegMax];
    auto site_map = [&](int z, word_t sd, word_t& a, word_t& b) {
      const int zn = (z == L - 1) ? 0 : z + 1;
      const word_t si = own[z * zs];
      const word_t sw = pw[z * zs], se = pe[z * zs];
      const word_t sn = pn.template ld<1>(z * zsn).w[0], ss = ps.template ld<1>(z * zss).w[0];
      const word_t jw = __ldg(Jxc + jo + z * zg), jee = __ldg(Jxo + je + z * zg);
      const word_t jn = __ldg(Jyc + jo + z * zg), jss = __ldg(Jyo + js + z * zg);
      const word_t ju = __ldg(Jzc + jo + z * zg), jd = __ldg(Jzc + jo + zn * zg);
      const uint32_t u = philox_draw(x.seed, site0 + plane * (unsigned)z, draw);
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
    A[0] = 0;
    B[0] = 0;
    if (col_ok) site_map(z0, own[(z0 + 1) * zs], A[0], B[0]);
    const word_t first = __shfl_sync(0xffffffffu, A[0] ^ (top & B[0]), lead);
#pragma unroll
    for (int i = 1; i < kSegMax; ++i) {
      A[i] = 0;
      B[i] = 0;
      if (col_ok && i < ls) {
        const int z = z0 + i;
        site_map(z, (z == L - 1) ? first : own[(z + 1) * zs], A[i], B[i]);
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
    for (int d = 1; d < G; d <<= 1) {
      const word_t pA = __shfl_up_sync(0xffffffffu, SA, d, G);
      const word_t pB = __shfl_up_sync(0xffffffffu, SB, d, G);
      if (g >= d) {
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
    __syncwarp();
    if (col_ok) {
      word_t v = EA ^ (top & EB);
#pragma unroll
      for (int i = 0; i < kSegMax; ++i)
        if (i < ls) {
          v = A[i] ^ (v & B[i]);
          own[(z0 + i) * zs] = v;
        }
    }
  }
}

// big += small over the low W planes only (values stay below 2^W).
template <int W>
__device__ __forceinline__ void add_small_w(VCount<16>& big, const VCount<4>& sm) {
  word_t carry = 0;
#pragma unroll
  for (int b = 0; b < W; ++b) {
    const word_t q = (b < 4) ? sm.p[b] : 0;
    const word_t a = big.p[b];
    big.p[b] = a ^ q ^ carry;
    carry = (a & q) | (carry & (a ^ q));
  }
}

// Sum over the lanes that share (lane mod NSL) of counters below 2^W0 per
// lane: level l of the butterfly adds values below 2^(W0+l), so it touches
// W0+l+1 planes (capped at 16) instead of all of them.
template <int NSL, int W0>
__device__ __forceinline__ void warp_sum_grow(VCount<16>& v) {
  constexpr int NL = (NSL == 1) ? 5 : (NSL == 2) ? 4 : 3;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const int off = 16 >> l;
    word_t carry = 0;
#pragma unroll
    for (int b = 0; b < 16; ++b) {
      if (b < W0 + l + 1) {
        const word_t a = v.p[b];
        const word_t q = __shfl_xor_sync(0xffffffffu, a, off);
        v.p[b] = a ^ q ^ carry;
        carry = (a & q) | (carry & (a ^ q));
      }
    }
  }
}

// Partial satisfied-bond counts of slots a..a+NSL-1 over this CTA's sites
// (each bond counted once, from its site towards -x/-y/-z), added into
// cnt[q][j]. Lanes: NSL per site, 32/NSL sites per warp row. A unit is one
// warp row of sites in one (colour, z) plane; units are ordered (row tile,
// colour, z), so a warp re-derives a site's indices only when it enters a
// new (tile, colour) and otherwise steps by one plane. A lane counts into W0
// bit planes; after at most (2^W0 - 1) / bonds-per-site units the warp sums
// its lanes and adds the totals to cnt. UNR units are formed before any is
// added, so their loads are in flight together.
template <bool CL, int UNR, int NSL, int W0>
__device__ __forceinline__ void rmeasure_body(const ResCtx& x, bool d3, bool open, int a, unsigned (*cnt)[64]) {
  static_assert(W0 >= 5 && W0 <= 11, "counter width: chunks of at least one UNR round");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  constexpr int per = 32 / NSL;
  const int g = lane / NSL, slot = a + lane % NSL;
  const int L = x.L, hL = x.hL, ns = x.ns, zc = x.zc;
  const int cols = x.ny * hL;
  const int tiles = (cols + per - 1) / per;
  const int units = 2 * zc * tiles;
  const int zs = x.ny * x.rowW, zg = L * hL;
  const int u0 = (int)(((long)units * warp) / nwarps), u1 = (int)(((long)units * (warp + 1)) / nwarps);
  const int chunk = ((1 << W0) - 1) / (d3 ? 3 : 2);  // units per lane before a warp sum
  // the lane's site in the current (tile, colour): plane-0 offsets and strides
  int tcol = u0 / zc, z = u0 - tcol * zc;
  bool ok = false, wopen = false;
  int own0 = 0, w0 = 0, zsn = zs, jr0 = 0;
  const word_t* Jc = x.J;  // couplings of the site's colour; axis a at Jc + 2*a*half
  NbRow<CL> pn;
  auto enter = [&]() {
    const int tile = tcol >> 1, c = tcol & 1, oc = 1 - c;
    const int col = tile * per + g;
    ok = col < cols;
    const int cc = ok ? col : 0;
    const int yl = div_hl(cc, x);
    const int k = cc - yl * hL, y = x.y0 + yl;
    const int par = (c + y) & 1, xx = 2 * k + par;
    int kw, ke;
    x_neighbours(k, par, hL, kw, ke);
    const int sk = slot ^ swz(x, k);
    own0 = lrow(x, c, 0, yl) + k * ns + sk;
    w0 = lrow(x, oc, 0, yl) + kw * ns + (slot ^ swz(x, kw));
    pn = north_row<CL>(x, oc, 0, yl);
    pn.step(k * ns + sk);
    zsn = (yl > 0) ? zs : x.nyN * x.rowW;
    jr0 = y * hL + k;
    Jc = x.J + (long)c * x.half;
    wopen = open && xx == 0;
  };
  // satisfied-bond bits (q1 q0 = 0..3) of this lane's site in plane z
  // lanes past the last column read column 0 (in range) and count nothing:
  // the unit has no divergent branch
  auto unit_bits = [&](word_t& q0, word_t& q1) {
    const word_t okm = ok ? ~0ULL : 0ULL;
    const word_t* jp = Jc + (jr0 + z * zg);
    const word_t si = x.sm[own0 + z * zs];
    const word_t w = wopen ? 0 : (__ldg(jp) ^ si ^ x.sm[w0 + z * zs]);
    const word_t n = __ldg(jp + 2 * x.half) ^ si ^ pn.template ld<1>(z * zsn).w[0];
    if (d3) {
      const int zu = (z == 0) ? L - 1 : z - 1;
      const word_t uu = __ldg(jp + 4 * x.half) ^ si ^ x.sm[own0 + zu * zs];
      q0 = (w ^ n ^ uu) & okm;
      q1 = ((w & n) | (uu & (w ^ n))) & okm;
    } else {
      q0 = (w ^ n) & okm;
      q1 = (w & n) & okm;
    }
  };
  auto advance = [&]() {
    if (++z == zc) {
      z = 0;
      ++tcol;
      enter();
    }
  };
  if (u0 < u1) enter();
  const int q = lane % NSL;
  for (int un = u0; un < u1;) {  // warp-uniform
    const int ue = min(u1, un + chunk);
    VCount<4> sm4;
    VCount<16> big;
    sm4.clear();
    big.clear();
    if (UNR > 1) {
      // UNR <= 5 units of <= 3 bonds per round keep the small counter below 16
      static_assert(UNR <= 5, "small counter range");
      for (; un + UNR <= ue; un += UNR) {
        word_t b0[UNR], b1[UNR];
#pragma unroll
        for (int i = 0; i < UNR; ++i) {
          unit_bits(b0[i], b1[i]);
          advance();
        }
#pragma unroll
        for (int i = 0; i < UNR; ++i) add2_small(sm4, b0[i], b1[i]);
        add_small_w<W0>(big, sm4);
        sm4.clear();
      }
    }
    int it = 0;
    for (; un < ue; ++un) {
      word_t b0, b1;
      unit_bits(b0, b1);
      add2_small(sm4, b0, b1);
      advance();
      if (++it == 5) {
        add_small_w<W0>(big, sm4);
        sm4.clear();
        it = 0;
      }
    }
    add_small_w<W0>(big, sm4);
    warp_sum_grow<NSL, W0>(big);
    // planes the sum can reach: W0 per lane, one more per butterfly level
    constexpr int NBU = W0 + ((NSL == 1) ? 5 : (NSL == 2) ? 4 : 3);
#pragma unroll
    for (int m = 0; m < 2 * NSL; ++m) {
      const int j = (lane / NSL) + per * m;
      atomicAdd(&cnt[q][j], big.template count_low<NBU>(j));
    }
  }
}

// Partial satisfied-bond counts of slots a..a+nsl-1 (nsl 1 or 2) over this
// CTA's sites added into cnt[q][j] (zeroed here first when `clear`; else the
// caller zeroed it before a barrier). Five counter planes per lane: a
// batched ensemble's share of a warp fits in one chunk (one warp sum per
// measurement); a single-slot lattice spread over few warps takes a warp
// sum every 10 (3D) or 15 (2D) units, which keeps the counters in registers.
// UNR units are formed before any is added, so their loads (couplings from
// L2 above all) are in flight together.
template <bool CL, int UNR = 1>
__device__ __forceinline__ void rmeasure(const ResCtx& x, bool d3, bool open, int a, int nsl,
                                         unsigned (*cnt)[64], bool clear = true) {
  if (clear) {
    for (int i = threadIdx.x; i < 128; i += blockDim.x) (&cnt[0][0])[i] = 0;
    __syncthreads();
  }
  if (nsl == 2) rmeasure_body<CL, UNR, 2, 5>(x, d3, open, a, cnt);
  else rmeasure_body<CL, UNR, 1, 5>(x, d3, open, a, cnt);
}

// ---------------------------------------------------------------------------
// The 3D exchange pass. The decision needs only E(a+1) - E(a) per replica, so
// one counter takes, for every bond, b(a+1) + (1 - b(a)) (b = J ^ s_i ^ s_j,
// the bits rmeasure counts): its total D gives v(a+1) - v(a) = D - nbonds.
// One lane holds both slots of a site, so a site's three coupling words
// (west, north, z-1: each site counts the bonds stored at it) are loaded once
// for both, and a warp sums one counter instead of two. Lane t takes column
// task t % T of T = 2 * columns (consecutive lanes, consecutive columns: the
// slot swizzle spreads their words over the banks) and planes t / T, t / T +
// phases, ...; a CTA with fewer threads than tasks loops over them. D goes
// into cnt[0][replica].
// ---------------------------------------------------------------------------
template <int W0>
__device__ __forceinline__ void add3_plane(VCount<16>& big, word_t c0, word_t c1, word_t c2) {
  word_t carry = 0;
#pragma unroll
  for (int b = 0; b < W0; ++b) {
    const word_t q = (b == 0) ? c0 : (b == 1) ? c1 : (b == 2) ? c2 : 0;
    const word_t v = big.p[b];
    big.p[b] = v ^ q ^ carry;
    carry = (v & q) | (carry & (v ^ q));
  }
}

template <bool CL>
__device__ __forceinline__ void rmeasure_pair_3d(const ResCtx& x, int a, unsigned (*cnt)[64]) {
  constexpr int W0 = 5;  // a lane adds at most 6 per site: a warp sum every 5 sites
  const int lane = threadIdx.x & 31, t = threadIdx.x, nthr = blockDim.x;
  const int L = x.L, hL = x.hL, ns = x.ns, cols = x.ny * hL;
  const int T = 2 * cols;
  const int phases = max(1, nthr / T);
  const int rounds = (T + nthr - 1) / nthr;  // > 1 only when nthr < T
  const int iters = (L + phases - 1) / phases;
  const int zs = x.ny * x.rowW, zg = L * hL;
  const long hf = x.half;
  VCount<16> big;
  big.clear();
  int held = 0;  // sites added since the last warp sum (warp-uniform)
  auto flush = [&]() {
    warp_sum_grow<1, W0>(big);
    constexpr int NBU = W0 + 5;
    atomicAdd(&cnt[0][lane], big.template count_low<NBU>(lane));
    atomicAdd(&cnt[0][lane + 32], big.template count_low<NBU>(lane + 32));
    big.clear();
  };
  const int zi = (nthr >= T) ? t / T : 0;
  for (int r = 0; r < rounds; ++r) {
    const int task = (nthr >= T) ? t % T : t + r * nthr;
    const bool tok = (nthr >= T) ? t < phases * T : task < T;
    const int tk = tok ? task : 0;  // idle lanes read column 0 and count nothing
    const int c = tk >= cols ? 1 : 0, oc = 1 - c;
    const int col = tk - c * cols;
    const int yl = div_hl(col, x);
    const int k = col - yl * hL, y = x.y0 + yl;
    int kw, ke;
    x_neighbours(k, (c + y) & 1, hL, kw, ke);
    const int sa = a ^ swz(x, k), sb = (a + 1) ^ swz(x, k);
    const int wa = a ^ swz(x, kw), wb = (a + 1) ^ swz(x, kw);
    const int own = lrow(x, c, 0, yl) + k * ns;
    const int wrow = lrow(x, oc, 0, yl) + kw * ns;
    NbRow<CL> pn = north_row<CL>(x, oc, 0, yl);
    pn.step(k * ns);
    const int zsn = (yl > 0) ? zs : x.nyN * x.rowW;
    const word_t* Jc = x.J + (long)c * hf + (y * hL + k);
#pragma unroll 1
    for (int it = 0; it < iters; ++it) {  // warp-uniform
      const int z = zi + it * phases;
      const bool ok = tok && z < L;
      const int zz = ok ? z : 0, zu = (zz == 0) ? L - 1 : zz - 1;
      const word_t* jp = Jc + zz * zg;
      const word_t jw = __ldg(jp), jn = __ldg(jp + 2 * hf), ju = __ldg(jp + 4 * hf);
      const int o = own + zz * zs, ou = own + zu * zs, ow = wrow + zz * zs;
      const word_t ai = x.sm[o + sa], bi = x.sm[o + sb];
      const word_t aw = x.sm[ow + wa], bw = x.sm[ow + wb];
      const word_t an = pn.template ld<1>(zz * zsn + sa).w[0], bn = pn.template ld<1>(zz * zsn + sb).w[0];
      const word_t au = x.sm[ou + sa], bu = x.sm[ou + sb];
      const word_t okm = ok ? ~0ULL : 0ULL;
      word_t c0, c1, c2;
      count6((jw ^ bi ^ bw) & okm, (jn ^ bi ^ bn) & okm, (ju ^ bi ^ bu) & okm,
             ~(jw ^ ai ^ aw) & okm, ~(jn ^ ai ^ an) & okm, ~(ju ^ ai ^ au) & okm, c0, c1, c2);
      add3_plane<W0>(big, c0, c1, c2);
      if (++held == 5) {
        flush();
        held = 0;
      }
    }
  }
  if (held) flush();
}

// ---------------------------------------------------------------------------
// The 2D exchange counts, taken by each warp over its own sites right after
// its colour-1 walk, with no barrier and no separate pass; the same difference
// counter D as rmeasure_pair_3d, into cnt[0][replica]. Every 2D bond joins a
// colour-0 and a colour-1 site, so the colour-1 sites' four bonds (west and
// east across an open x edge excepted) cover the lattice once. They are final
// when this warp has walked its colour-1 tiles: colour 0 was final at the
// barrier before the colour-1 half, and only this warp writes the colour-1
// sites of its tiles (rhalf_2d's tiles: 32 sites from 32 * warp, stepping
// 32 * warps). Lane = site of the tile, both slots. (In 3D the same scheme
// needs the z-bonds of both colours and measured slower than a separate pass.)
// ---------------------------------------------------------------------------
template <bool OPEN_X, bool CL>
__device__ __forceinline__ void rmeasure_own_2d(const ResCtx& x, int a, unsigned (*cnt)[64]) {
  constexpr int W0 = 5;  // a lane adds at most 8 per site: a warp sum every 3 sites
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int L = x.L, hL = x.hL, ns = x.ns, tot = x.ny * hL;
  const word_t* J = x.J;
  VCount<16> big;
  big.clear();
  int held = 0;  // sites added since the last warp sum (warp-uniform)
  auto flush = [&]() {
    warp_sum_grow<1, W0>(big);
    constexpr int NBU = W0 + 5;
    atomicAdd(&cnt[0][lane], big.template count_low<NBU>(lane));
    atomicAdd(&cnt[0][lane + 32], big.template count_low<NBU>(lane + 32));
    big.clear();
  };
  for (int base = warp * 32; base < tot; base += nwarps * 32) {
    const int t = base + lane;
    const bool ok = t < tot;
    const int tt = ok ? t : base;  // lanes past the end read a real site and count nothing
    const int yl = div_hl(tt, x);
    const int k = tt - yl * hL, y = x.y0 + yl;
    const int par = (1 + y) & 1, xx = 2 * k + par;
    int kw, ke;
    x_neighbours(k, par, hL, kw, ke);
    const int ys = (y == L - 1) ? 0 : y + 1;
    const int sa = a ^ swz(x, k), sb = (a + 1) ^ swz(x, k);
    const int o1 = lrow(x, 1, 0, yl) + k * ns;
    const int ow = lrow(x, 0, 0, yl) + kw * ns, oe = lrow(x, 0, 0, yl) + ke * ns;
    const int wa = a ^ swz(x, kw), wb = (a + 1) ^ swz(x, kw);
    const int ea = a ^ swz(x, ke), eb = (a + 1) ^ swz(x, ke);
    NbRow<CL> pn = north_row<CL>(x, 0, 0, yl), ps = south_row<CL>(x, 0, 0, yl);
    pn.step(k * ns);
    ps.step(k * ns);
    const word_t ai = x.sm[o1 + sa], bi = x.sm[o1 + sb];
    const word_t aw = x.sm[ow + wa], bw = x.sm[ow + wb];
    const word_t ae = x.sm[oe + ea], be = x.sm[oe + eb];
    const word_t an = pn.template ld<1>(sa).w[0], bn = pn.template ld<1>(sb).w[0];
    const word_t as = ps.template ld<1>(sa).w[0], bs = ps.template ld<1>(sb).w[0];
    // couplings: west bond stored at the site (Jx of colour 1), east bond at
    // the east neighbour (Jx of colour 0), north bond at the site (Jy of
    // colour 1), south bond at the south neighbour (Jy of colour 0)
    const word_t jw = __ldg(J + 1 * x.half + y * hL + k), je = __ldg(J + 0 * x.half + y * hL + ke);
    const word_t jn = __ldg(J + 3 * x.half + y * hL + k), js = __ldg(J + 2 * x.half + ys * hL + k);
    const word_t okm = ok ? ~0ULL : 0ULL;
    const word_t mw = (OPEN_X && xx == 0) ? 0 : okm, me = (OPEN_X && xx == L - 1) ? 0 : okm;
    // b(a+1) and 1 - b(a) for each existing bond
    word_t p0, p1, p2, q0, q1, q2;
    count4((jw ^ bi ^ bw) & mw, (je ^ bi ^ be) & me, (jn ^ bi ^ bn) & okm, (js ^ bi ^ bs) & okm, p0, p1, p2);
    count4(~(jw ^ ai ^ aw) & mw, ~(je ^ ai ^ ae) & me, ~(jn ^ ai ^ an) & okm, ~(js ^ ai ^ as) & okm, q0, q1, q2);
    add3_plane<W0>(big, p0, p1, p2);
    add3_plane<W0>(big, q0, q1, q2);
    if (++held == 3) {
      flush();
      held = 0;
    }
  }
  if (held) flush();
}

}  // namespace sa
