// ntt2048.cuh -- the transforms of ntt.cuh at N = 2048 with register passes.
//
// Same mathematics, twiddle tables and orders as ntt.cuh (forward: natural ->
// transform position brv(slot); inverse: the reverse), so results are
// identical word for word.  What changes is the schedule:
//   * 11 stages run as three radix-8 passes and one radix-4 pass; a thread
//     keeps its 8 (or 4) values in registers across the stages of a pass, so a
//     transform costs 4 barriers and 4 shared-memory round trips instead of 6;
//   * the polynomials live in a padded layout (4 words after every 32:
//     logical word i at i + 4 (i >> 5), PS = 2304 words per polynomial), which
//     makes every pass free of bank conflicts (the radix-4 pass moves 16-byte
//     vectors);
//   * NT, the number of threads, is a compile-time constant, so each thread
//     owns the same butterfly groups of every polynomial in a pass: its
//     twiddles are loaded once per pass and factor, not once per polynomial.
// Forward stage s (distance 2^(10-s)) uses tw[2^s + block]; inverse stage s
// (distance 2^s) uses iw[2^(10-s) + block]: the tables of ntt.cuh.
#pragma once
#include <type_traits>

#include "ntt.cuh"

namespace dnspir {
namespace n2k {

constexpr int N = 2048;
constexpr int PS = N + N / 8;  // padded words per polynomial

__host__ __device__ __forceinline__ constexpr uint32_t phys(uint32_t i) { return i + ((i >> 5) << 2); }
__device__ __forceinline__ uint32_t brv11(uint32_t i) { return __brev(i) >> 21; }

using ntt_detail::canon;
using ntt_detail::ct;
using ntt_detail::gs;
using ntt_detail::lazy_mul;
using ntt_detail::red;

// how NT threads cover the G butterfly groups of each polynomial in a pass
template <int NT, int G>
struct Split {
  static_assert(G % NT == 0 || NT % G == 0, "thread count and group count must divide");
  static constexpr int GSUB = G > NT ? G / NT : 1;  // groups per thread and polynomial
  static constexpr int PPI = G > NT ? 1 : NT / G;   // polynomials in flight across the block
};

// Radix-8 pass, first stage s with M = 2^s sub-blocks: group g covers logical
// words blk * 8D + r + D k (k < 8), D = N / (8M), blk = g / D, r = g % D.
template <int M>
struct Geo8 {
  static constexpr int D = N / (8 * M);
  static constexpr int STR = D >= 32 ? D + D / 8 : D;  // padded spacing of the 8 words
  __device__ __forceinline__ static int blk(int g) { return g / D; }
  __device__ __forceinline__ static int base(int g) { return (int)phys((uint32_t)((g / D) * 8 * D + g % D)); }
};

struct Tw8 {
  uint32_t a, aq, b[2], bq[2], c[4], cq[4];
};
// The seven twiddles of a radix-8 group from the interleaved (w, companion)
// table: one 8-byte and three 16-byte loads (2M + 2 blk and 4M + 4 blk are
// even, so the pairs of pairs are 16-byte aligned).
__device__ __forceinline__ Tw8 load_tw8(const uint2* __restrict__ tw2, int M, int blk) {
  Tw8 t;
  const uint2 a = __ldg(tw2 + M + blk);
  const uint4 b = __ldg(reinterpret_cast<const uint4*>(tw2 + 2 * M + 2 * blk));
  const uint4 c0 = __ldg(reinterpret_cast<const uint4*>(tw2 + 4 * M + 4 * blk));
  const uint4 c1 = __ldg(reinterpret_cast<const uint4*>(tw2 + 4 * M + 4 * blk + 2));
  t.a = a.x, t.aq = a.y;
  t.b[0] = b.x, t.bq[0] = b.y, t.b[1] = b.z, t.bq[1] = b.w;
  t.c[0] = c0.x, t.cq[0] = c0.y, t.c[1] = c0.z, t.cq[1] = c0.w;
  t.c[2] = c1.x, t.cq[2] = c1.y, t.c[3] = c1.z, t.cq[3] = c1.w;
  return t;
}
// The three twiddles of the radix-4 pass on quad g: tw[512 + g] and the pair
// tw[1024 + 2g], tw[1024 + 2g + 1].
struct Tw4 {
  uint32_t a, aq, b0, b0q, b1, b1q;
};
__device__ __forceinline__ Tw4 load_tw4(const uint2* __restrict__ tw2, int g) {
  const uint2 a = __ldg(tw2 + 512 + g);
  const uint4 b = __ldg(reinterpret_cast<const uint4*>(tw2 + 1024 + 2 * g));
  return Tw4{a.x, a.y, b.x, b.y, b.z, b.w};
}

__device__ __forceinline__ void fwd8_bf(uint32_t (&v)[8], const Tw8& t, uint32_t p) {
  ct(v[0], v[4], t.a, t.aq, p);
  ct(v[1], v[5], t.a, t.aq, p);
  ct(v[2], v[6], t.a, t.aq, p);
  ct(v[3], v[7], t.a, t.aq, p);
  ct(v[0], v[2], t.b[0], t.bq[0], p);
  ct(v[1], v[3], t.b[0], t.bq[0], p);
  ct(v[4], v[6], t.b[1], t.bq[1], p);
  ct(v[5], v[7], t.b[1], t.bq[1], p);
  ct(v[0], v[1], t.c[0], t.cq[0], p);
  ct(v[2], v[3], t.c[1], t.cq[1], p);
  ct(v[4], v[5], t.c[2], t.cq[2], p);
  ct(v[6], v[7], t.c[3], t.cq[3], p);
}
__device__ __forceinline__ void inv8_bf(uint32_t (&v)[8], const Tw8& t, uint32_t p) {
  gs(v[0], v[1], t.c[0], t.cq[0], p);
  gs(v[2], v[3], t.c[1], t.cq[1], p);
  gs(v[4], v[5], t.c[2], t.cq[2], p);
  gs(v[6], v[7], t.c[3], t.cq[3], p);
  gs(v[0], v[2], t.b[0], t.bq[0], p);
  gs(v[1], v[3], t.b[0], t.bq[0], p);
  gs(v[4], v[6], t.b[1], t.bq[1], p);
  gs(v[5], v[7], t.b[1], t.bq[1], p);
  gs(v[0], v[4], t.a, t.aq, p);
  gs(v[1], v[5], t.a, t.aq, p);
  gs(v[2], v[6], t.a, t.aq, p);
  gs(v[3], v[7], t.a, t.aq, p);
}

// Default end of an inverse transform: scale by N^-1 into [0, p), in place.
struct ScaleStore {
  __device__ __forceinline__ void operator()(uint32_t* y, int /*poly*/, int /*r*/, uint32_t (&v)[8], uint32_t p,
                                             uint32_t ni, uint32_t niq) const {
#pragma unroll
    for (int k = 0; k < 8; k++) y[k * Geo8<1>::STR] = red(lazy_mul(v[k], ni, niq, p), p);
  }
};

// Ends a pass: SYNC = 0 synchronises the block; SYNC = 1 only the 256-thread
// group of the calling thread (named barrier 1 + threadIdx.x / 256), for
// blocks of 512 threads whose two halves work on one polynomial each.
template <int SYNC>
__device__ __forceinline__ void pass_sync() {
  if constexpr (SYNC == 0) {
    __syncthreads();
  } else {
    asm volatile("bar.sync %0, 256;" ::"r"(1 + (threadIdx.x >> 8)) : "memory");
  }
}

// One radix-8 pass over polynomials [0, cnt0) (factor 0) and [cnt0, cnt0 +
// cnt1) (factor 1) of x.  INV selects Gentleman-Sande with the iw tables; FIN
// (inverse, M = 1 only) receives the finished values instead of a store.
template <int NT, int M, bool INV, int SYNC = 0, class Fin>
__device__ __forceinline__ void pass8(uint32_t* x, int cnt0, int cnt1, const NttTables& T, const Fin& fin) {
  using S = Split<NT, 256>;
  using Gm = Geo8<M>;
  const int tid = threadIdx.x;
  const int po = S::PPI > 1 ? tid / 256 : 0;
#pragma unroll
  for (int gsub = 0; gsub < S::GSUB; gsub++) {
    const int g = S::PPI > 1 ? tid % 256 : tid + gsub * NT;
    const int blk = Gm::blk(g), base = Gm::base(g);
#pragma unroll
    for (int pi = 0; pi < 2; pi++) {
      const int lo = pi ? cnt0 : 0, hi = pi ? cnt0 + cnt1 : cnt0;
      if (lo >= hi) continue;
      const uint32_t p = prime_of(pi);
      const Tw8 t = load_tw8(INV ? T.iw2[pi] : T.fw2[pi], M, blk);
      // polynomials are dealt to the PPI thread groups by their global index
      // (poly mod PPI), so one polynomial per factor still spreads over all
      // groups
      const int first = lo + ((po - lo) % S::PPI + S::PPI) % S::PPI;
      for (int poly = first; poly < hi; poly += S::PPI) {
        uint32_t* y = x + poly * PS + base;
        uint32_t v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = y[k * Gm::STR];
        if (INV) {
          inv8_bf(v, t, p);
          if constexpr (M == 1 && !std::is_same<Fin, void*>::value) {
            fin(y, poly, g, v, p, T.ninv[pi][11], T.ninvq[pi][11]);
            continue;
          }
        } else {
          fwd8_bf(v, t, p);
        }
#pragma unroll
        for (int k = 0; k < 8; k++) y[k * Gm::STR] = v[k];
      }
    }
  }
  pass_sync<SYNC>();
}

// Radix-4 pass on the aligned quads 4g .. 4g + 3 (forward stages 9-10 with
// the final reduction to [0, p); inverse stages 0-1), as 16-byte vectors.
template <int NT, bool INV>
__device__ __forceinline__ void pass4(uint32_t* x, int cnt0, int cnt1, const NttTables& T) {
  using S = Split<NT, 512>;
  const int tid = threadIdx.x;
  const int po = S::PPI > 1 ? tid / 512 : 0;
#pragma unroll
  for (int gsub = 0; gsub < S::GSUB; gsub++) {
    const int g = S::PPI > 1 ? tid % 512 : tid + gsub * NT;
    const int base = (int)phys(4 * g);
#pragma unroll
    for (int pi = 0; pi < 2; pi++) {
      const int lo = pi ? cnt0 : 0, hi = pi ? cnt0 + cnt1 : cnt0;
      if (lo >= hi) continue;
      const uint32_t p = prime_of(pi);
      const Tw4 tw = load_tw4(INV ? T.iw2[pi] : T.fw2[pi], g);
      const uint32_t a = tw.a, aq = tw.aq, b0 = tw.b0, b0q = tw.b0q, b1 = tw.b1, b1q = tw.b1q;
      const int first = lo + ((po - lo) % S::PPI + S::PPI) % S::PPI;
      for (int poly = first; poly < hi; poly += S::PPI) {
        uint4* y = reinterpret_cast<uint4*>(x + poly * PS + base);
        uint4 v = *y;
        if (INV) {
          gs(v.x, v.y, b0, b0q, p);
          gs(v.z, v.w, b1, b1q, p);
          gs(v.x, v.z, a, aq, p);
          gs(v.y, v.w, a, aq, p);
        } else {
          ct(v.x, v.z, a, aq, p);
          ct(v.y, v.w, a, aq, p);
          ct(v.x, v.y, b0, b0q, p);
          ct(v.z, v.w, b1, b1q, p);
          v.x = canon(v.x, p), v.y = canon(v.y, p), v.z = canon(v.z, p), v.w = canon(v.w, p);
        }
        *y = v;
      }
    }
  }
  __syncthreads();
}

// Forward transform of cnt0 + cnt1 padded polynomials (factor 0 then factor
// 1): canonical natural-order input, canonical output at transform positions.
// All NT threads of the block call; ends with a barrier.
template <int NT>
__device__ __forceinline__ void fwd(uint32_t* x, int cnt0, int cnt1, const NttTables& T) {
  pass8<NT, 1, false>(x, cnt0, cnt1, T, (void*)nullptr);
  pass8<NT, 8, false>(x, cnt0, cnt1, T, (void*)nullptr);
  pass8<NT, 64, false>(x, cnt0, cnt1, T, (void*)nullptr);
  pass4<NT, false>(x, cnt0, cnt1, T);
}

// Inverse transform (canonical input at transform positions).  The last pass
// hands each thread's 8 values -- logical words r + 256 k of polynomial poly,
// unscaled, in [0, 2p) -- to fin(y, poly, r, v, p, N^-1, its Shoup companion),
// y pointing at word r of the polynomial (stride Geo8<1>::STR); the default
// stores them scaled into [0, p).
template <int NT, class Fin = ScaleStore>
__device__ __forceinline__ void inv(uint32_t* x, int cnt0, int cnt1, const NttTables& T, const Fin& fin = Fin()) {
  pass4<NT, true>(x, cnt0, cnt1, T);
  pass8<NT, 64, true>(x, cnt0, cnt1, T, (void*)nullptr);
  pass8<NT, 8, true>(x, cnt0, cnt1, T, (void*)nullptr);
  pass8<NT, 1, true>(x, cnt0, cnt1, T, fin);
}

}  // namespace n2k
}  // namespace dnspir
