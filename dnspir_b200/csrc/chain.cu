// chain.cu -- the key-switching chain of preprocess / partial_gal
// (crates/pir/src/base_pir.rs:496-594, 782-863) and its fusion with the
// secondary scan (double_pir.rs:195-218).
//
// A chain step on the a-part of a ciphertext is
//     t      = sigma_5(a)                        (the galois lookup of :509-515)
//     v      = centred CRT lift of iNTT(t)        (:544-555)
//     d1     = (v + 2^25) >> 26, d0 = v - 2^26 d1 (:557-570; the second digit's
//              own carry is always 0 since |v| < q/2 < 2^50)
//     a      = NTT(d0) gk_a0 + NTT(d1) gk_a1 + qry_a E_i
// and, for the secondary database evaluated on a query ciphertext (b-part),
//     b      = sigma_5(b) + NTT(d0) gk_b0 + NTT(d1) gk_b1 + qry_b E_i,
// which is the homomorphic evaluation whose b-part main_pir_loop computes
// from the stored digits (its sum/sum_new recurrence equals b up to the
// sigma_5 applied before the final permute, :1072-1073).
//
// Because d0 + 2^26 d1 = v exactly and v = t in each factor, NTT(d0) =
// t - 2^26 NTT(d1): one forward transform per factor and step instead of two.
//
// Layout: one 2-block cluster per chain, block rank p owning RNS factor p.
// The blocks exchange their iNTT outputs through distributed shared memory
// (double-buffered by step parity, one cluster barrier per step), each
// computes the CRT lift and the high digit, and transforms it in its own
// factor.  NTT-domain vectors hold slots in bit-reversed position order
// (position q <-> slot brv(q)); the constants are stored the same way.
#include <cooperative_groups.h>

#include <cstring>

#include "kernels.cuh"
#include "ntt2048.cuh"

namespace cg = cooperative_groups;

namespace dnspir {
namespace {

constexpr int CT = 512;  // threads per block of a chain cluster

// ---- Montgomery arithmetic, R = 2^32 (p < 2^26)
__host__ __device__ constexpr uint32_t neg_inv32(uint32_t p) {
  uint32_t x = p;  // Newton iteration for p^-1 mod 2^32
  for (int i = 0; i < 5; i++) x *= 2u - p * x;
  return 0u - x;
}
// x * y R^-1 mod p for products and sums below 2^64 whose result is < 3p; returns [0, p)
__device__ __forceinline__ uint32_t mont_reduce(uint64_t T, uint32_t p, uint32_t pinv) {
  const uint32_t m = (uint32_t)T * pinv;
  uint64_t u = (T + (uint64_t)m * p) >> 32;
  u = u >= p ? u - p : u;
  u = u >= p ? u - p : u;
  return (uint32_t)u;
}

struct ChainPrime {
  uint32_t p, pinv;      // factor and -p^-1 mod 2^32
  uint32_t r2;           // R^2 mod p (to enter Montgomery form)
  uint32_t c26;          // 2^26 R mod p
  uint32_t k1, k1q;      // q2^-1 N^-1 mod q1 with its Shoup companion (CRT, factor 1)
  uint32_t k2, k2q;      // q1^-1 N^-1 mod q2 (CRT, factor 2)
};

// radix-4 / radix-2 transforms of one length-2^logn vector by CT threads, with
// Harvey's lazy butterflies: values stay in [0, 4p) inside a transform (4p <
// 2^28) and are brought back to [0, p) when it ends.
// Forward: natural -> bit-reversed (CT butterflies), input in [0, p).
// Inverse: bit-reversed -> natural, NOT scaled by N^-1 (the caller folds N^-1
// into its next constant), input in [0, p).
__device__ __forceinline__ uint32_t shoup_lazy(uint32_t x, uint32_t w, uint32_t wq, uint32_t p) {
  return x * w - __umulhi(x, wq) * p;  // in [0, 2p) for any x < 2^32
}
__device__ __forceinline__ uint32_t red2p(uint32_t x, uint32_t p2) { return x >= p2 ? x - p2 : x; }
// CT butterfly on [0, 4p) inputs: (x, y) -> (x + w y, x - w y), outputs in [0, 4p)
__device__ __forceinline__ void ct_bf(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wq, uint32_t p) {
  const uint32_t a = red2p(x, 2 * p);
  const uint32_t t = shoup_lazy(y, w, wq, p);
  x = a + t;
  y = a - t + 2 * p;
}
// GS butterfly on [0, 2p) inputs: (x, y) -> (x + y, w (x - y)), outputs in [0, 2p)
__device__ __forceinline__ void gs_bf(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wq, uint32_t p) {
  const uint32_t a = x + y;
  const uint32_t d = x - y + 2 * p;
  x = red2p(a, 2 * p);
  y = shoup_lazy(d, w, wq, p);
}

// LN vectors `stride` words apart, transformed together: one barrier per pass,
// and each thread handles the same butterfly group of every vector with its
// loads issued before the arithmetic (twiddles loaded once).
// LOGN > 0 fixes the length at compile time (the stage loop unrolls and every
// index shift is a constant); LOGN = 0 takes logn_rt.
template <int LN, int LOGN>
__device__ __forceinline__ void fwd_multi(uint32_t* x0, int stride, int logn_rt, const uint32_t* __restrict__ tw,
                                          const uint32_t* __restrict__ twq, uint32_t p) {
  const int logn = LOGN ? LOGN : logn_rt;
  const int N = 1 << logn;
  int s = 0;
#pragma unroll
  for (; s + 1 < logn; s += 2) {
    const int logt2 = logn - s - 2;
    const int t2 = 1 << logt2, t = 2 * t2, m = 1 << s;
    for (int g = threadIdx.x; g < N / 4; g += CT) {
      const int blk = g >> logt2, r = g & (t2 - 1);
      const int j = (blk << (logt2 + 2)) + r;
      const uint32_t w = tw[m + blk], wq = twq[m + blk];
      const uint32_t w1 = tw[2 * m + 2 * blk], w1q = twq[2 * m + 2 * blk];
      const uint32_t w2 = tw[2 * m + 2 * blk + 1], w2q = twq[2 * m + 2 * blk + 1];
      uint32_t v[LN][4];
#pragma unroll
      for (int l = 0; l < LN; l++) {
        const uint32_t* x = x0 + l * stride;
        v[l][0] = x[j], v[l][1] = x[j + t2], v[l][2] = x[j + t], v[l][3] = x[j + t + t2];
      }
#pragma unroll
      for (int l = 0; l < LN; l++) {
        ct_bf(v[l][0], v[l][2], w, wq, p);
        ct_bf(v[l][1], v[l][3], w, wq, p);
        ct_bf(v[l][0], v[l][1], w1, w1q, p);
        ct_bf(v[l][2], v[l][3], w2, w2q, p);
      }
#pragma unroll
      for (int l = 0; l < LN; l++) {
        uint32_t* x = x0 + l * stride;
        x[j] = v[l][0], x[j + t2] = v[l][1], x[j + t] = v[l][2], x[j + t + t2] = v[l][3];
      }
    }
    __syncthreads();
  }
  if (s < logn) {  // last stage, t = 1
    for (int b = threadIdx.x; b < N / 2; b += CT) {
      const uint32_t w = tw[N / 2 + b], wq = twq[N / 2 + b];
      uint32_t u[LN], v[LN];
#pragma unroll
      for (int l = 0; l < LN; l++) u[l] = x0[l * stride + 2 * b], v[l] = x0[l * stride + 2 * b + 1];
#pragma unroll
      for (int l = 0; l < LN; l++) {
        ct_bf(u[l], v[l], w, wq, p);
        x0[l * stride + 2 * b] = red2p(red2p(u[l], 2 * p), p);
        x0[l * stride + 2 * b + 1] = red2p(red2p(v[l], 2 * p), p);
      }
    }
  } else {
    for (int b = threadIdx.x; b < N; b += CT)
#pragma unroll
      for (int l = 0; l < LN; l++) x0[l * stride + b] = red2p(red2p(x0[l * stride + b], 2 * p), p);
  }
  __syncthreads();
}

template <int LN, int LOGN>
__device__ __forceinline__ void inv_multi(uint32_t* x0, int stride, int logn_rt, const uint32_t* __restrict__ tw,
                                          const uint32_t* __restrict__ twq, uint32_t p) {
  const int logn = LOGN ? LOGN : logn_rt;
  const int N = 1 << logn;
  int s = 0;
#pragma unroll
  for (; s + 1 < logn; s += 2) {
    const int t = 1 << s;
    const int h0 = N >> (s + 1), h1 = N >> (s + 2);
    for (int g = threadIdx.x; g < N / 4; g += CT) {
      const int blk = g >> s, r = g & (t - 1);
      const int j = (blk << (s + 2)) + r;
      const uint32_t w0 = tw[h0 + 2 * blk], w0q = twq[h0 + 2 * blk];
      const uint32_t w1 = tw[h0 + 2 * blk + 1], w1q = twq[h0 + 2 * blk + 1];
      const uint32_t w = tw[h1 + blk], wq = twq[h1 + blk];
      uint32_t v[LN][4];
#pragma unroll
      for (int l = 0; l < LN; l++) {
        const uint32_t* x = x0 + l * stride;
        v[l][0] = x[j], v[l][1] = x[j + t], v[l][2] = x[j + 2 * t], v[l][3] = x[j + 3 * t];
      }
#pragma unroll
      for (int l = 0; l < LN; l++) {
        gs_bf(v[l][0], v[l][1], w0, w0q, p);
        gs_bf(v[l][2], v[l][3], w1, w1q, p);
        gs_bf(v[l][0], v[l][2], w, wq, p);
        gs_bf(v[l][1], v[l][3], w, wq, p);
      }
#pragma unroll
      for (int l = 0; l < LN; l++) {
        uint32_t* x = x0 + l * stride;
        x[j] = v[l][0], x[j + t] = v[l][1], x[j + 2 * t] = v[l][2], x[j + 3 * t] = v[l][3];
      }
    }
    __syncthreads();
  }
  if (s < logn) {  // last stage, t = N/2
    const uint32_t w = tw[1], wq = twq[1];
    for (int j = threadIdx.x; j < N / 2; j += CT) {
      uint32_t u[LN], v[LN];
#pragma unroll
      for (int l = 0; l < LN; l++) u[l] = x0[l * stride + j], v[l] = x0[l * stride + j + N / 2];
#pragma unroll
      for (int l = 0; l < LN; l++) {
        gs_bf(u[l], v[l], w, wq, p);
        x0[l * stride + j] = u[l];
        x0[l * stride + j + N / 2] = v[l];
      }
    }
    __syncthreads();
  }
  // outputs are in [0, 2p); the consumer (high_digit via Shoup) accepts any value < 2^32
}

// High digit of the centred CRT lift from the two factors' unscaled iNTT
// outputs: x = v - k q (v = x1 q2 + x2 q1 < 2q, k = round(v / q)), digit
// floor((x + 2^25) / 2^26).  Computed in double precision, exactly: x1 q2 and
// x2 q1 are below 2^51, v below 2^52 and q = q1 q2 below 2^51, so every sum,
// difference and comparison is exact in the 53-bit significand, and
// x 2^-26 + 1/2 (a power-of-two scaling of an integer below 2^51 in
// magnitude, plus one half) is exact too, leaving floor() the only rounding
// -- the same integer as the 64-bit formula, on the FP64 pipe instead of the
// integer pipes the transforms saturate.
__device__ __forceinline__ int32_t high_digit(uint32_t c1, uint32_t c2, const ChainPrime& P1c, const ChainPrime& P2c) {
  const uint32_t x1 = shoup_mul(c1, P1c.k1, P1c.k1q, P1);
  const uint32_t x2 = shoup_mul(c2, P2c.k2, P2c.k2q, P2);
  constexpr double Q = (double)QQ, HALF_Q = (double)(QQ / 2);  // QQ / 2 = (q - 1) / 2, exact
  double v = fma((double)x1, (double)P2, (double)x2 * (double)P1);
  v = v >= Q ? v - Q : v;
  v = v > HALF_Q ? v - Q : v;
  return __double2int_rd(fma(v, 1.0 / (double)(1u << LOG2_B), 0.5));
}

struct ChainArgs {
  Group g;
  // constants: gk_a digits [d][p][pos], qry_a halves [h][p][pos], sigma_5 map, canonical
  const uint32_t* gka;
  const uint32_t* qa;
  const uint32_t* galb;
  SlotMaps maps;
  NttTables T;
  ChainPrime cp[2];
  // secondary: entries in chain layout, query vectors [q][slot][p][pos], output
  const uint32_t* E;
  const uint32_t* qv;
  size_t qv_stride;
  int nl;
  uint32_t* out;
  // primary: slabs and a-part output
  uint32_t* const* slabs;
  uint32_t* a_out;
  uint32_t c_first, cinv_first, inv5;
};

// Primary chain (preprocessing), one lane per block.  Shared-memory plan (u32
// words, N = 2^logn):
//   A, TC, D           N each    state a, saved sigma_5(a), work vector
//   X[2]               2N        iNTT outputs published to the peer block
//   CG0, CG1, CQA      3N        gk_a0 R, gk_a1 R, qry_a R of this factor and half
//   FW, FWQ, IW, IWQ   4N        twiddles of this factor
template <int LOGN>
__device__ __forceinline__ void primary_body(const ChainArgs& a, int h, int lane, int s, uint32_t* sm) {
  cg::cluster_group cluster = cg::this_cluster();
  const int p = (int)cluster.block_rank();
  const int logn = LOGN ? LOGN : a.g.log2n;
  const int N = 1 << logn;
  const uint32_t mask = 2 * N - 1;
  const ChainPrime cp = a.cp[p];
  const uint32_t pr = cp.p;
  uint32_t* A = sm;
  uint32_t* TC = A + N;
  uint32_t* D = TC + N;
  uint32_t* X = D + N;
  uint32_t* CG0 = X + 2 * N;
  uint32_t* CG1 = CG0 + N;
  uint32_t* CQA = CG1 + N;
  uint32_t* FW = CQA + N;
  uint32_t* FWQ = FW + N;
  uint32_t* IW = FWQ + N;
  uint32_t* IWQ = IW + N;
  for (int b = threadIdx.x; b < N; b += CT) {
    A[b] = 0;
    const size_t o = (size_t)p * N + b;
    CG0[b] = mont_reduce((uint64_t)a.gka[o] * cp.r2, pr, cp.pinv);
    CG1[b] = mont_reduce((uint64_t)a.gka[2 * (size_t)N + o] * cp.r2, pr, cp.pinv);
    CQA[b] = mont_reduce((uint64_t)a.qa[(size_t)h * 2 * N + o] * cp.r2, pr, cp.pinv);
    FW[b] = a.T.fw[p][b];
    FWQ[b] = a.T.fwq[p][b];
    IW[b] = a.T.iw[p][b];
    IWQ[b] = a.T.iwq[p][b];
  }
  cluster.sync();
  uint32_t* peerX = cluster.map_shared_rank(X, p ^ 1);
  uint32_t* slab = a.slabs[s];
  uint32_t ci = a.c_first, cinv = a.cinv_first;
  constexpr int PER = N_MAX / CT;  // positions per thread (N <= N_MAX)
  for (uint32_t i = 0; i < a.g.L; i++) {
    // entries of row i for this thread's positions, consumed at the end of the step
    uint32_t e[PER];
#pragma unroll
    for (int c = 0; c < PER; c++) {
      const int pos = threadIdx.x + c * CT;
      e[c] = 0;
      if (pos < N) {
        const uint32_t j = brv(pos, logn);
        const uint32_t ks = gidx(cinv * (2 * j + 1), mask);
        e[c] = slab[slab_off(a.g, p, h, i, 0, __ldg(a.maps.uof + ks)) + lane];
      }
    }
    // sigma_5 on a
    uint32_t ra[PER];
#pragma unroll
    for (int c = 0; c < PER; c++) {
      const int pos = threadIdx.x + c * CT;
      if (pos < N) ra[c] = A[pos];
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < PER; c++) {
      const int pos = threadIdx.x + c * CT;
      if (pos < N) {
        const uint32_t dst = __ldg(a.galb + pos);
        TC[dst] = ra[c];
        D[dst] = ra[c];
      }
    }
    __syncthreads();
    inv_multi<1, LOGN>(D, 0, logn, IW, IWQ, pr);
    uint32_t* Xc = X + (i & 1) * N;
    for (int b = threadIdx.x; b < N; b += CT) Xc[b] = D[b];
    cluster.sync();
    const uint32_t* Pc = peerX + (i & 1) * N;
    for (int b = threadIdx.x; b < N; b += CT) {
      const uint32_t own = D[b], other = Pc[b];
      const int32_t hd = p == 0 ? high_digit(own, other, a.cp[0], a.cp[1]) : high_digit(other, own, a.cp[0], a.cp[1]);
      D[b] = hd < 0 ? (uint32_t)(hd + (int32_t)pr) : (uint32_t)hd;
    }
    __syncthreads();
    fwd_multi<1, LOGN>(D, 0, logn, FW, FWQ, pr);
#pragma unroll
    for (int c = 0; c < PER; c++) {
      const int pos = threadIdx.x + c * CT;
      if (pos < N) {
        const uint32_t n1 = D[pos];
        const uint32_t n0 = sub_mod(TC[pos], mont_reduce((uint64_t)n1 * cp.c26, pr, cp.pinv), pr);
        A[pos] = mont_reduce((uint64_t)n0 * CG0[pos] + (uint64_t)n1 * CG1[pos] + (uint64_t)e[c] * CQA[pos], pr,
                             cp.pinv);
        TC[pos] = n0;
      }
    }
    __syncthreads();
    // key digits of row i in the scan layout: position u (natural slot k with
    // 2k+1 = g[u]) holds G_i[idx(5^(L-1-i) g[u])]
    for (int u = threadIdx.x; u < N; u += CT) {
      const uint32_t jb = brv(gidx(ci * __ldg(a.maps.g + u), mask), logn);
      slab[slab_off(a.g, p, h, i, 1, u) + lane] = TC[jb];
      slab[slab_off(a.g, p, h, i, 2, u) + lane] = D[jb];
    }
    // TC and D are rewritten only after the next step's first barrier
    ci = (ci * a.inv5) & mask;
    cinv = (cinv * 5) & mask;
  }
  uint32_t* o = a.a_out + (((size_t)s * a.g.H + h) * SIMD + lane) * 2 * N;
  for (int b = threadIdx.x; b < N; b += CT) o[(size_t)p * N + b] = A[b];
  cluster.sync();  // keep this block's shared memory alive until the peer's last read
}

// Secondary chain: LN of the three parts of one query's secondary ciphertext
// at half h in one block (factor p = rank in the cluster), parts part0 ..
// part0 + LN - 1 (the library launches LN = 1: the block then needs 88 KiB and
// shares an SM with a scan block, so the chains of a few queries overlap the
// next scan; larger chunks use secondary_dual_kernel below).  The key constants gk_a0,
// gk_a1, qry_a, gk_b0, gk_b1, qry_b (Montgomery form) and the sigma_5
// destinations of a thread's positions live in its registers.  Each step's
// pointwise stage writes the next step's sigma_5-permuted a and b straight
// into the other buffer of a pair, and the inverse transform is published to
// the peer from its own buffer D[i mod 2] (the peer reads it between the
// cluster barriers of steps i and i + 1; this block rewrites it only at the end
// of step i + 1).  Shared memory (u32 words):
//   FW FWQ IW IWQ                    4N   twiddles of this factor
//   per part: TC[2] D[2] B[2] H      7N   sigma_5(a) kept, sigma_5(a) transformed
//                                         (published), sigma_5(b), high digit
// (4 + 7 LN) N words: 200 KiB for LN = 3, 88 KiB for LN = 1 at N = 2048.
constexpr int SEC_PART_WORDS = 7;  // x N
__host__ __device__ constexpr int sec_smem_words(int ln) { return 4 + ln * SEC_PART_WORDS; }

template <int LN, int LOGN>
__device__ __forceinline__ void secondary_body(const ChainArgs& a, int h, int q, int part0, uint32_t* sm) {
  cg::cluster_group cluster = cg::this_cluster();
  const int p = (int)cluster.block_rank();
  const int logn = LOGN ? LOGN : a.g.log2n;
  const int N = 1 << logn;
  const ChainPrime cp = a.cp[p];
  const uint32_t pr = cp.p;
  uint32_t* FW = sm;
  uint32_t* FWQ = FW + N;
  uint32_t* IW = FWQ + N;
  uint32_t* IWQ = IW + N;
  uint32_t* P0 = IWQ + N;  // part blocks
  const int PS = SEC_PART_WORDS * N;
  // per part: TC[2] at 0, N; D[2] at 2N, 3N; B[2] at 4N, 5N; H at 6N
  const int oTC = 0, oD = 2 * N, oB = 4 * N, oH = 6 * N;
  const uint32_t* qq = a.qv + (size_t)q * a.qv_stride;
  constexpr int PER = N_MAX / CT;  // positions per thread (N <= N_MAX)
  uint32_t kc[6][PER], dst[PER];
#pragma unroll
  for (int c = 0; c < PER; c++) {
    const int pos = threadIdx.x + c * CT;
    if (pos < N) {
      const size_t o = (size_t)p * N + pos;
      kc[0][c] = mont_reduce((uint64_t)a.gka[o] * cp.r2, pr, cp.pinv);
      kc[1][c] = mont_reduce((uint64_t)a.gka[2 * (size_t)N + o] * cp.r2, pr, cp.pinv);
      kc[2][c] = mont_reduce((uint64_t)a.qa[(size_t)h * 2 * N + o] * cp.r2, pr, cp.pinv);
      kc[3][c] = mont_reduce((uint64_t)qq[o] * cp.r2, pr, cp.pinv);
      kc[4][c] = mont_reduce((uint64_t)qq[2 * (size_t)N + o] * cp.r2, pr, cp.pinv);
      kc[5][c] = mont_reduce((uint64_t)qq[(size_t)(4 + h) * 2 * N + o] * cp.r2, pr, cp.pinv);
      dst[c] = __ldg(a.galb + pos);
    }
  }
  for (int b = threadIdx.x; b < N; b += CT) {
    FW[b] = a.T.fw[p][b];
    FWQ[b] = a.T.fwq[p][b];
    IW[b] = a.T.iw[p][b];
    IWQ[b] = a.T.iwq[p][b];
#pragma unroll
    for (int t = 0; t < LN; t++) {  // a = b = 0, so sigma_5(a) = sigma_5(b) = 0
      P0[t * PS + oTC + b] = 0;
      P0[t * PS + oD + b] = 0;
      P0[t * PS + oB + b] = 0;
    }
  }
  cluster.sync();
  const uint32_t* peer = cluster.map_shared_rank(P0, p ^ 1);
  for (uint32_t i = 0; i < a.g.L; i++) {
    const int cur = (int)(i & 1) * N, nxt = N - cur;
    // entries of row i (the three parts' lanes are adjacent), consumed at the end of the step
    const uint32_t* Ei = a.E + ((((size_t)p * a.g.H + h) * a.g.L + i) * a.nl + (size_t)q * CTXT_PARTS + part0) * N;
    uint32_t e[LN][PER];
#pragma unroll
    for (int t = 0; t < LN; t++)
#pragma unroll
      for (int c = 0; c < PER; c++) {
        const int pos = threadIdx.x + c * CT;
        e[t][c] = pos < N ? __ldg(Ei + (size_t)t * N + pos) : 0;
      }
    inv_multi<LN, LOGN>(P0 + oD + cur, PS, logn, IW, IWQ, pr);
    cluster.sync();
    for (int b = threadIdx.x; b < N; b += CT) {
      uint32_t own[LN], other[LN];
#pragma unroll
      for (int t = 0; t < LN; t++) own[t] = P0[t * PS + oD + cur + b], other[t] = peer[t * PS + oD + cur + b];
#pragma unroll
      for (int t = 0; t < LN; t++) {
        const int32_t hd = p == 0 ? high_digit(own[t], other[t], a.cp[0], a.cp[1])
                                  : high_digit(other[t], own[t], a.cp[0], a.cp[1]);
        P0[t * PS + oH + b] = hd < 0 ? (uint32_t)(hd + (int32_t)pr) : (uint32_t)hd;
      }
    }
    __syncthreads();
    fwd_multi<LN, LOGN>(P0 + oH, PS, logn, FW, FWQ, pr);
#pragma unroll
    for (int c = 0; c < PER; c++) {
      const int pos = threadIdx.x + c * CT;
      if (pos < N) {
        const uint32_t cg0 = kc[0][c], cg1 = kc[1][c], cqa = kc[2][c];
        const uint32_t qg0 = kc[3][c], qg1 = kc[4][c], qqb = kc[5][c];
#pragma unroll
        for (int t = 0; t < LN; t++) {
          uint32_t* P = P0 + t * PS;
          const uint32_t n1 = P[oH + pos];
          const uint32_t n0 = sub_mod(P[oTC + cur + pos], mont_reduce((uint64_t)n1 * cp.c26, pr, cp.pinv), pr);
          const uint32_t an =
              mont_reduce((uint64_t)n0 * cg0 + (uint64_t)n1 * cg1 + (uint64_t)e[t][c] * cqa, pr, cp.pinv);
          const uint32_t bn = mont_reduce(((uint64_t)P[oB + cur + pos] << 32) + (uint64_t)n0 * qg0 +
                                              (uint64_t)n1 * qg1 + (uint64_t)e[t][c] * qqb,
                                          pr, cp.pinv);
          // sigma_5 for the next step
          P[oTC + nxt + dst[c]] = an;
          P[oD + nxt + dst[c]] = an;
          P[oB + nxt + dst[c]] = bn;
        }
      }
    }
    __syncthreads();
  }
  // the state after the last step sits sigma_5-permuted in buffer L mod 2
  const int fin = (int)(a.g.L & 1) * N;
#pragma unroll
  for (int c = 0; c < PER; c++) {
    const int pos = threadIdx.x + c * CT;
    if (pos < N) {
#pragma unroll
      for (int t = 0; t < LN; t++) {
        uint32_t* o = a.out + ((((size_t)q * a.g.H + h) * CTXT_PARTS + part0 + t) * 2) * 2 * N;
        o[(size_t)p * N + pos] = P0[t * PS + oTC + fin + dst[c]];
        o[2 * (size_t)N + (size_t)p * N + pos] = P0[t * PS + oB + fin + dst[c]];
      }
    }
  }
  cluster.sync();  // keep this block's shared memory alive until the peer's last read
}

// ---- secondary chain without a cluster: one block carries one part at half h
// in BOTH factors.  Every transform pass handles the two factors' vectors
// (each with its own twiddles and prime), the high digit reads both inverse
// transforms from this block's shared memory (no cluster barrier, no remote
// reads), and each barrier covers twice the work of the clustered form.
// Shared memory (u32 words): twiddles FW FWQ IW IWQ of each factor (8N), per
// factor TC[2] D[2] B[2] H (7N): 22N = 176 KiB at N = 2048, one block per SM.
constexpr int SEC_DUAL_WORDS = 8 + 2 * SEC_PART_WORDS;  // x N

template <int LOGN>
__device__ __forceinline__ void fwd_dual(uint32_t* x0, uint32_t* x1, int logn_rt, const uint32_t* const* tw,
                                         const uint32_t* const* twq, uint32_t p0, uint32_t p1) {
  const int logn = LOGN ? LOGN : logn_rt;
  const int N = 1 << logn;
  uint32_t* xs[2] = {x0, x1};
  const uint32_t ps[2] = {p0, p1};
  int s = 0;
#pragma unroll
  for (; s + 1 < logn; s += 2) {
    const int logt2 = logn - s - 2;
    const int t2 = 1 << logt2, t = 2 * t2, m = 1 << s;
    for (int g = threadIdx.x; g < N / 4; g += CT) {
      const int blk = g >> logt2, r = g & (t2 - 1);
      const int j = (blk << (logt2 + 2)) + r;
      uint32_t v[2][4];
#pragma unroll
      for (int l = 0; l < 2; l++) {
        const uint32_t* x = xs[l];
        v[l][0] = x[j], v[l][1] = x[j + t2], v[l][2] = x[j + t], v[l][3] = x[j + t + t2];
      }
#pragma unroll
      for (int l = 0; l < 2; l++) {
        const uint32_t w = tw[l][m + blk], wq = twq[l][m + blk];
        ct_bf(v[l][0], v[l][2], w, wq, ps[l]);
        ct_bf(v[l][1], v[l][3], w, wq, ps[l]);
        ct_bf(v[l][0], v[l][1], tw[l][2 * m + 2 * blk], twq[l][2 * m + 2 * blk], ps[l]);
        ct_bf(v[l][2], v[l][3], tw[l][2 * m + 2 * blk + 1], twq[l][2 * m + 2 * blk + 1], ps[l]);
      }
#pragma unroll
      for (int l = 0; l < 2; l++) {
        uint32_t* x = xs[l];
        x[j] = v[l][0], x[j + t2] = v[l][1], x[j + t] = v[l][2], x[j + t + t2] = v[l][3];
      }
    }
    __syncthreads();
  }
  if (s < logn) {  // last stage, t = 1
    for (int b = threadIdx.x; b < N / 2; b += CT) {
#pragma unroll
      for (int l = 0; l < 2; l++) {
        uint32_t* x = xs[l];
        uint32_t u = x[2 * b], v = x[2 * b + 1];
        ct_bf(u, v, tw[l][N / 2 + b], twq[l][N / 2 + b], ps[l]);
        x[2 * b] = red2p(red2p(u, 2 * ps[l]), ps[l]);
        x[2 * b + 1] = red2p(red2p(v, 2 * ps[l]), ps[l]);
      }
    }
  } else {
    for (int b = threadIdx.x; b < N; b += CT)
#pragma unroll
      for (int l = 0; l < 2; l++) xs[l][b] = red2p(red2p(xs[l][b], 2 * ps[l]), ps[l]);
  }
  __syncthreads();
}

template <int LOGN>
__device__ __forceinline__ void inv_dual(uint32_t* x0, uint32_t* x1, int logn_rt, const uint32_t* const* tw,
                                         const uint32_t* const* twq, uint32_t p0, uint32_t p1) {
  const int logn = LOGN ? LOGN : logn_rt;
  const int N = 1 << logn;
  uint32_t* xs[2] = {x0, x1};
  const uint32_t ps[2] = {p0, p1};
  int s = 0;
#pragma unroll
  for (; s + 1 < logn; s += 2) {
    const int t = 1 << s;
    const int h0 = N >> (s + 1), h1 = N >> (s + 2);
    for (int g = threadIdx.x; g < N / 4; g += CT) {
      const int blk = g >> s, r = g & (t - 1);
      const int j = (blk << (s + 2)) + r;
      uint32_t v[2][4];
#pragma unroll
      for (int l = 0; l < 2; l++) {
        const uint32_t* x = xs[l];
        v[l][0] = x[j], v[l][1] = x[j + t], v[l][2] = x[j + 2 * t], v[l][3] = x[j + 3 * t];
      }
#pragma unroll
      for (int l = 0; l < 2; l++) {
        gs_bf(v[l][0], v[l][1], tw[l][h0 + 2 * blk], twq[l][h0 + 2 * blk], ps[l]);
        gs_bf(v[l][2], v[l][3], tw[l][h0 + 2 * blk + 1], twq[l][h0 + 2 * blk + 1], ps[l]);
        const uint32_t w = tw[l][h1 + blk], wq = twq[l][h1 + blk];
        gs_bf(v[l][0], v[l][2], w, wq, ps[l]);
        gs_bf(v[l][1], v[l][3], w, wq, ps[l]);
      }
#pragma unroll
      for (int l = 0; l < 2; l++) {
        uint32_t* x = xs[l];
        x[j] = v[l][0], x[j + t] = v[l][1], x[j + 2 * t] = v[l][2], x[j + 3 * t] = v[l][3];
      }
    }
    __syncthreads();
  }
  if (s < logn) {  // last stage, t = N/2
    for (int j = threadIdx.x; j < N / 2; j += CT) {
#pragma unroll
      for (int l = 0; l < 2; l++) {
        uint32_t* x = xs[l];
        uint32_t u = x[j], v = x[j + N / 2];
        gs_bf(u, v, tw[l][1], twq[l][1], ps[l]);
        x[j] = u;
        x[j + N / 2] = v;
      }
    }
    __syncthreads();
  }
}

template <int LOGN>
__device__ __forceinline__ void secondary_dual_body(const ChainArgs& a, int h, int q, int part, uint32_t* sm) {
  const int logn = LOGN ? LOGN : a.g.log2n;
  const int N = 1 << logn;
  const uint32_t pr0 = a.cp[0].p, pr1 = a.cp[1].p;
  const uint32_t* tws[2] = {sm, sm + 4 * N};
  const uint32_t* twqs[2] = {sm + N, sm + 5 * N};
  const uint32_t* itws[2] = {sm + 2 * N, sm + 6 * N};
  const uint32_t* itwqs[2] = {sm + 3 * N, sm + 7 * N};
  uint32_t* F0 = sm + 8 * N;  // factor blocks: TC[2] at 0, N; D[2] at 2N, 3N; B[2] at 4N, 5N; H at 6N
  const int FS = SEC_PART_WORDS * N;
  const int oTC = 0, oD = 2 * N, oB = 4 * N, oH = 6 * N;
  const uint32_t* qq = a.qv + (size_t)q * a.qv_stride;
  constexpr int PER = N_MAX / CT;
  uint32_t kc[2][6][PER], dst[PER];
#pragma unroll
  for (int c = 0; c < PER; c++) {
    const int pos = threadIdx.x + c * CT;
    if (pos < N) {
#pragma unroll
      for (int p = 0; p < 2; p++) {
        const ChainPrime& cp = a.cp[p];
        const size_t o = (size_t)p * N + pos;
        kc[p][0][c] = mont_reduce((uint64_t)a.gka[o] * cp.r2, cp.p, cp.pinv);
        kc[p][1][c] = mont_reduce((uint64_t)a.gka[2 * (size_t)N + o] * cp.r2, cp.p, cp.pinv);
        kc[p][2][c] = mont_reduce((uint64_t)a.qa[(size_t)h * 2 * N + o] * cp.r2, cp.p, cp.pinv);
        kc[p][3][c] = mont_reduce((uint64_t)qq[o] * cp.r2, cp.p, cp.pinv);
        kc[p][4][c] = mont_reduce((uint64_t)qq[2 * (size_t)N + o] * cp.r2, cp.p, cp.pinv);
        kc[p][5][c] = mont_reduce((uint64_t)qq[(size_t)(4 + h) * 2 * N + o] * cp.r2, cp.p, cp.pinv);
      }
      dst[c] = __ldg(a.galb + pos);
    }
  }
  for (int b = threadIdx.x; b < N; b += CT) {
#pragma unroll
    for (int p = 0; p < 2; p++) {
      sm[4 * p * N + b] = a.T.fw[p][b];
      sm[(4 * p + 1) * N + b] = a.T.fwq[p][b];
      sm[(4 * p + 2) * N + b] = a.T.iw[p][b];
      sm[(4 * p + 3) * N + b] = a.T.iwq[p][b];
      F0[p * FS + oTC + b] = 0;
      F0[p * FS + oD + b] = 0;
      F0[p * FS + oB + b] = 0;
    }
  }
  __syncthreads();
  for (uint32_t i = 0; i < a.g.L; i++) {
    const int cur = (int)(i & 1) * N, nxt = N - cur;
    uint32_t e[2][PER];
#pragma unroll
    for (int p = 0; p < 2; p++) {
      const uint32_t* Ei = a.E + ((((size_t)p * a.g.H + h) * a.g.L + i) * a.nl + (size_t)q * CTXT_PARTS + part) * N;
#pragma unroll
      for (int c = 0; c < PER; c++) {
        const int pos = threadIdx.x + c * CT;
        e[p][c] = pos < N ? __ldg(Ei + pos) : 0;
      }
    }
    inv_dual<LOGN>(F0 + oD + cur, F0 + FS + oD + cur, logn, itws, itwqs, pr0, pr1);
    for (int b = threadIdx.x; b < N; b += CT) {
      const int32_t hd = high_digit(F0[oD + cur + b], F0[FS + oD + cur + b], a.cp[0], a.cp[1]);
      F0[oH + b] = hd < 0 ? (uint32_t)(hd + (int32_t)pr0) : (uint32_t)hd;
      F0[FS + oH + b] = hd < 0 ? (uint32_t)(hd + (int32_t)pr1) : (uint32_t)hd;
    }
    __syncthreads();
    fwd_dual<LOGN>(F0 + oH, F0 + FS + oH, logn, tws, twqs, pr0, pr1);
#pragma unroll
    for (int c = 0; c < PER; c++) {
      const int pos = threadIdx.x + c * CT;
      if (pos < N) {
#pragma unroll
        for (int p = 0; p < 2; p++) {
          const ChainPrime& cp = a.cp[p];
          uint32_t* P = F0 + p * FS;
          const uint32_t n1 = P[oH + pos];
          const uint32_t n0 = sub_mod(P[oTC + cur + pos], mont_reduce((uint64_t)n1 * cp.c26, cp.p, cp.pinv), cp.p);
          const uint32_t an = mont_reduce(
              (uint64_t)n0 * kc[p][0][c] + (uint64_t)n1 * kc[p][1][c] + (uint64_t)e[p][c] * kc[p][2][c], cp.p,
              cp.pinv);
          const uint32_t bn = mont_reduce(((uint64_t)P[oB + cur + pos] << 32) + (uint64_t)n0 * kc[p][3][c] +
                                              (uint64_t)n1 * kc[p][4][c] + (uint64_t)e[p][c] * kc[p][5][c],
                                          cp.p, cp.pinv);
          P[oTC + nxt + dst[c]] = an;
          P[oD + nxt + dst[c]] = an;
          P[oB + nxt + dst[c]] = bn;
        }
      }
    }
    __syncthreads();
  }
  const int fin = (int)(a.g.L & 1) * N;
  uint32_t* o = a.out + ((((size_t)q * a.g.H + h) * CTXT_PARTS + part) * 2) * 2 * N;
#pragma unroll
  for (int c = 0; c < PER; c++) {
    const int pos = threadIdx.x + c * CT;
    if (pos < N) {
#pragma unroll
      for (int p = 0; p < 2; p++) {
        o[(size_t)p * N + pos] = F0[p * FS + oTC + fin + dst[c]];
        o[2 * (size_t)N + (size_t)p * N + pos] = F0[p * FS + oB + fin + dst[c]];
      }
    }
  }
}

// ---- N = 2048: one block per part and half carrying both factors, on the
// register transforms of ntt2048.cuh.  The block's two 256-thread halves
// work one RNS factor each: half f holds factor f's polynomials in every pass,
// and thread t of a half owns positions 8t .. 8t + 7 of its factor in the
// first inverse pass, the last forward pass and the pointwise stage, so those
// run from registers.  The halves meet once a step: between the last inverse
// pass and the first forward pass each takes the other's values at its
// positions for the CRT high digit (the one block-wide barrier); every other
// barrier is a named barrier of one half.  The inverse work space D is double
// buffered by step parity, so a half may run a step ahead of the other's reads
// of its last inverse pass.  The state a, b stays in natural position order:
// instead of scattering the next step's sigma_5(a), sigma_5(b) (which needs a
// second buffer of each), every step gathers them at its own positions through
// the inverse of galb.  Shared memory, padded polynomials of n2k::PS words:
// A[2] (a; also the forward transform's work space), B[2] (b), D[2][2]; then
// the six key constants (Montgomery form) of every position, [j][factor]
// [quad half][thread] as 16-byte vectors, each thread reading only its own.
constexpr int SEC2K_KC_WORDS = 6 * 2 * 2 * 256 * 4;
constexpr int SEC2K_WORDS = 8 * n2k::PS + SEC2K_KC_WORDS;

__device__ __forceinline__ void half_sync() {
  asm volatile("bar.sync %0, 256;" ::"r"(1 + (threadIdx.x >> 8)) : "memory");
}

__global__ void __launch_bounds__(CT, 1) secondary_chain2k_kernel(ChainArgs a) {
  extern __shared__ __align__(16) uint32_t sm[];
  using namespace n2k;
  static_assert(CT == 512 && N_MAX == N, "two quads per thread of one factor");
  const int h = blockIdx.x % a.g.H, part = blockIdx.x / a.g.H, q = blockIdx.y;
  uint32_t* const A = sm;
  uint32_t* const B = sm + 2 * PS;
  uint32_t* const D = sm + 4 * PS;  // [parity][factor]
  const int tid = threadIdx.x;
  const int f = tid >> 8, t = tid & 255;  // factor of this half, thread within the half
  const int qb = (int)phys(8 * t);       // positions 8t .. 8t + 7 sit in one padded row: qb .. qb + 7
  const ChainPrime cp = f ? a.cp[1] : a.cp[0];
  const uint32_t p = cp.p;
  // sigma_5 sources of the positions (galb inverted through D), a = b = 0
  for (int b = tid; b < N; b += CT) D[__ldg(a.galb + b)] = b;
  for (int b = tid; b < 4 * PS; b += CT) sm[b] = 0;
  __syncthreads();
  uint32_t src[4];  // two 16-bit padded positions per word (PS < 2^16)
#pragma unroll
  for (int m = 0; m < 4; m++) src[m] = phys(D[8 * t + 2 * m]) | (phys(D[8 * t + 2 * m + 1]) << 16);
  const uint32_t* qq = a.qv + (size_t)q * a.qv_stride;
  uint4* const KC = reinterpret_cast<uint4*>(sm + 8 * PS);  // [j][factor][quad half][t]
#pragma unroll
  for (int h4 = 0; h4 < 2; h4++) {
    uint32_t kc[6][4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const size_t o = (size_t)f * N + 8 * t + 4 * h4 + m;
      kc[0][m] = mont_reduce((uint64_t)a.gka[o] * cp.r2, cp.p, cp.pinv);
      kc[1][m] = mont_reduce((uint64_t)a.gka[2 * (size_t)N + o] * cp.r2, cp.p, cp.pinv);
      kc[2][m] = mont_reduce((uint64_t)a.qa[(size_t)h * 2 * N + o] * cp.r2, cp.p, cp.pinv);
      kc[3][m] = mont_reduce((uint64_t)qq[o] * cp.r2, cp.p, cp.pinv);
      kc[4][m] = mont_reduce((uint64_t)qq[2 * (size_t)N + o] * cp.r2, cp.p, cp.pinv);
      kc[5][m] = mont_reduce((uint64_t)qq[(size_t)(4 + h) * 2 * N + o] * cp.r2, cp.p, cp.pinv);
      // with t = sigma_5(a): NTT(d0) gk0 + NTT(d1) gk1 = t gk0 + NTT(d1) (gk1 - 2^26 gk0),
      // and likewise for the b-part keys, so the pointwise stage needs no d0
      kc[1][m] = sub_mod(kc[1][m], mont_reduce((uint64_t)kc[0][m] * cp.c26, cp.p, cp.pinv), cp.p);
      kc[4][m] = sub_mod(kc[4][m], mont_reduce((uint64_t)kc[3][m] * cp.c26, cp.p, cp.pinv), cp.p);
    }
#pragma unroll
    for (int j = 0; j < 6; j++)
      KC[((j * 2 + f) * 2 + h4) * 256 + t] = make_uint4(kc[j][0], kc[j][1], kc[j][2], kc[j][3]);
  }
  __syncthreads();  // the table in D is overwritten by the first step
  const size_t lane = (size_t)q * CTXT_PARTS + part;
  const uint4* Erow = reinterpret_cast<const uint4*>(a.E + (((size_t)f * a.g.H + h) * a.g.L * a.nl + lane) * N);
  const size_t erow_stride = (size_t)a.nl * N / 4;  // uint4 per row i
  for (uint32_t i = 0; i < a.g.L; i++) {
    uint32_t* const Dc = D + (i & 1) * 2 * PS;
    // sigma_5(a) (the inverse transform's input and the kept t) and sigma_5(b)
    uint32_t ta[8], tb[8];
#pragma unroll
    for (int m = 0; m < 8; m++) {
      const uint32_t sp = m & 1 ? src[m >> 1] >> 16 : src[m >> 1] & 0xFFFFu;
      ta[m] = A[f * PS + sp], tb[m] = B[f * PS + sp];
    }
    // inverse stages 0-1 from registers, two quads
#pragma unroll
    for (int h4 = 0; h4 < 2; h4++) {
      const Tw4 w = load_tw4(a.T.iw2[f], 2 * t + h4);
      uint4 v = make_uint4(ta[4 * h4], ta[4 * h4 + 1], ta[4 * h4 + 2], ta[4 * h4 + 3]);
      gs(v.x, v.y, w.b0, w.b0q, p);
      gs(v.z, v.w, w.b1, w.b1q, p);
      gs(v.x, v.z, w.a, w.aq, p);
      gs(v.y, v.w, w.a, w.aq, p);
      *reinterpret_cast<uint4*>(Dc + f * PS + qb + 4 * h4) = v;
    }
    half_sync();
    pass8<CT, 64, true, 1>(Dc, 1, 1, a.T, (void*)nullptr);
    pass8<CT, 8, true, 1>(Dc, 1, 1, a.T, (void*)nullptr);
    {
      // last inverse pass (unscaled: N^-1 sits in the CRT constants), the
      // other factor's values at the same positions, high digit, first
      // forward pass; group g = t, words g + 256 k
      const int base = (int)phys(t);
      constexpr int STR = Geo8<1>::STR;
      uint32_t v[8];
      uint32_t* y = Dc + f * PS + base;
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = y[k * STR];
      inv8_bf(v, load_tw8(a.T.iw2[f], 1, 0), p);
#pragma unroll
      for (int k = 0; k < 8; k++) y[k * STR] = v[k];
      __syncthreads();
      const uint32_t* z = Dc + (1 - f) * PS + base;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const uint32_t o = z[k * STR];
        const int32_t hd = f == 0 ? high_digit(v[k], o, a.cp[0], a.cp[1]) : high_digit(o, v[k], a.cp[0], a.cp[1]);
        v[k] = hd < 0 ? (uint32_t)(hd + (int32_t)p) : (uint32_t)hd;
      }
      fwd8_bf(v, load_tw8(a.T.fw2[f], 1, 0), p);
      uint32_t* w = A + f * PS + base;
#pragma unroll
      for (int k = 0; k < 8; k++) w[k * STR] = v[k];
      half_sync();
    }
    // entries of row i at the positions, consumed by the pointwise stage
    // (loaded here: the two forward passes cover their latency)
    const uint4 e0 = __ldg(Erow + i * erow_stride + 2 * t), e1 = __ldg(Erow + i * erow_stride + 2 * t + 1);
    pass8<CT, 8, false, 1>(A, 1, 1, a.T, (void*)nullptr);
    pass8<CT, 64, false, 1>(A, 1, 1, a.T, (void*)nullptr);
    // forward stages 9-10 and the pointwise stage at the two quads
#pragma unroll
    for (int h4 = 0; h4 < 2; h4++) {
      const Tw4 w = load_tw4(a.T.fw2[f], 2 * t + h4);
      uint4 v = *reinterpret_cast<const uint4*>(A + f * PS + qb + 4 * h4);
      ct(v.x, v.z, w.a, w.aq, p);
      ct(v.y, v.w, w.a, w.aq, p);
      ct(v.x, v.y, w.b0, w.b0q, p);
      ct(v.z, v.w, w.b1, w.b1q, p);
      const uint32_t n1s[4] = {canon(v.x, p), canon(v.y, p), canon(v.z, p), canon(v.w, p)};
      const uint4 e = h4 ? e1 : e0;
      const uint32_t es[4] = {e.x, e.y, e.z, e.w};
      uint32_t kc[6][4];
#pragma unroll
      for (int j = 0; j < 6; j++) {
        const uint4 c = KC[((j * 2 + f) * 2 + h4) * 256 + t];
        kc[j][0] = c.x, kc[j][1] = c.y, kc[j][2] = c.z, kc[j][3] = c.w;
      }
      uint32_t an[4], bn[4];
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const int j = 4 * h4 + m;
        const uint32_t n1 = n1s[m], tt = ta[j];
        an[m] = mont_reduce((uint64_t)tt * kc[0][m] + (uint64_t)n1 * kc[1][m] + (uint64_t)es[m] * kc[2][m], p,
                            cp.pinv);
        bn[m] = mont_reduce(((uint64_t)tb[j] << 32) + (uint64_t)tt * kc[3][m] + (uint64_t)n1 * kc[4][m] +
                                (uint64_t)es[m] * kc[5][m],
                            p, cp.pinv);
      }
      *reinterpret_cast<uint4*>(A + f * PS + qb + 4 * h4) = make_uint4(an[0], an[1], an[2], an[3]);
      *reinterpret_cast<uint4*>(B + f * PS + qb + 4 * h4) = make_uint4(bn[0], bn[1], bn[2], bn[3]);
    }
    half_sync();
  }
  uint32_t* o = a.out + ((((size_t)q * a.g.H + h) * CTXT_PARTS + part) * 2) * 2 * N;
#pragma unroll
  for (int h4 = 0; h4 < 2; h4++) {
    reinterpret_cast<uint4*>(o + (size_t)f * N)[2 * t + h4] = *reinterpret_cast<const uint4*>(A + f * PS + qb + 4 * h4);
    reinterpret_cast<uint4*>(o + 2 * (size_t)N + (size_t)f * N)[2 * t + h4] =
        *reinterpret_cast<const uint4*>(B + f * PS + qb + 4 * h4);
  }
}

// grid: x = part * H + half, y = query (no cluster)
template <int LOGN>
__global__ void __launch_bounds__(CT, 1) secondary_dual_kernel(ChainArgs a) {
  extern __shared__ uint32_t sm[];
  secondary_dual_body<LOGN>(a, blockIdx.x % a.g.H, blockIdx.y, blockIdx.x / a.g.H, sm);
}

// grid: x = factor (cluster of 2), y = (part group) * H + half, z = query
template <int LN, int LOGN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CT) secondary_chain_kernel(ChainArgs a) {
  extern __shared__ uint32_t sm[];
  secondary_body<LN, LOGN>(a, blockIdx.y % a.g.H, blockIdx.z, (blockIdx.y / a.g.H) * LN, sm);
}

// grid: x = factor (cluster of 2), y = lane * H + half, z = shard
template <int LOGN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CT) primary_chain_kernel(ChainArgs a) {
  extern __shared__ uint32_t sm[];
  const int h = blockIdx.y % a.g.H, lane = blockIdx.y / a.g.H;
  primary_body<LOGN>(a, h, lane, blockIdx.z, sm);
}

// reply_a = a_main + a_conj -> iNTT -> CRT; also the 17-bit mod switch
// (get_a, base_pir.rs:897-903, and double_pir.rs:164).
__global__ void primary_finalize_kernel(const uint32_t* __restrict__ a_out, uint64_t* __restrict__ a_zq,
                                        uint32_t* __restrict__ a_ms, Group g, NttTables T, CrtConst crtc) {
  extern __shared__ uint32_t sm[];  // [2][N]
  const int lane = blockIdx.x, s = blockIdx.y;
  const uint32_t N = g.n;
  for (uint32_t b = threadIdx.x; b < 2 * N; b += blockDim.x) {
    const uint32_t p = b / N;
    uint32_t v = a_out[(((size_t)s * g.H + 0) * SIMD + lane) * 2 * N + b];
    if (g.H == 2) v = add_mod(v, a_out[(((size_t)s * g.H + 1) * SIMD + lane) * 2 * N + b], prime_of(p));
    sm[b] = v;
  }
  __syncthreads();
  ntt_inv_smem2(sm, g.log2n, 1, 1, T);
  for (uint32_t n = threadIdx.x; n < N; n += blockDim.x) {
    const uint64_t v = crt(sm[n], sm[N + n], crtc);
    a_zq[((size_t)s * SIMD + lane) * N + n] = v;
    a_ms[((size_t)s * SIMD + lane) * N + n] = ms_encode(v, PRIM_A_BITS);
  }
}

}  // namespace

CrtConst host_crt_const();

static uint64_t pw(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  b %= m;
  while (e) {
    if (e & 1) r = (uint64_t)((unsigned __int128)r * b % m);
    b = (uint64_t)((unsigned __int128)b * b % m);
    e >>= 1;
  }
  return r;
}
static uint32_t pow_mod2n(uint32_t b, uint32_t e, uint32_t mask) {
  uint32_t r = 1;
  for (uint32_t k = 0; k < e; k++) r = (r * b) & mask;
  return r;
}
static uint32_t inv5_mod2n(uint32_t two_n) {
  for (uint32_t x = 1; x < two_n; x += 2)
    if ((5 * x) % two_n == 1) return x;
  return 1;
}

static ChainArgs chain_args(const Group& g, const ChainConsts& cc, const NttTables& T) {
  ChainArgs a;
  memset(&a, 0, sizeof(a));
  a.g = g;
  a.gka = cc.gka;
  a.qa = cc.qa;
  a.galb = cc.galb;
  a.maps = cc.maps;
  a.T = T;
  const uint64_t n = g.n;
  const CrtConst crtc = host_crt_const();
  for (int p = 0; p < 2; p++) {
    ChainPrime& c = a.cp[p];
    c.p = p ? P2 : P1;
    c.pinv = neg_inv32(c.p);
    c.r2 = (uint32_t)pw(pw(2, 64, c.p), 1, c.p);
    c.c26 = (uint32_t)((((unsigned __int128)1 << 26) << 32) % c.p);
    const uint64_t ninv1 = pw(n, P1 - 2, P1), ninv2 = pw(n, P2 - 2, P2);
    c.k1 = (uint32_t)((uint64_t)crtc.q2inv1 * ninv1 % P1);
    c.k1q = (uint32_t)(((uint64_t)c.k1 << 32) / P1);
    c.k2 = (uint32_t)((uint64_t)crtc.q1inv2 * ninv2 % P2);
    c.k2q = (uint32_t)(((uint64_t)c.k2 << 32) / P2);
  }
  return a;
}

static size_t chain_smem(const Group& g, int secondary_parts) {
  return (size_t)(secondary_parts ? sec_smem_words(secondary_parts) : 12) * g.n * 4;
}

void launch_primary_chain(uint32_t* const* slabs_dev, int nshards, uint32_t* a_out, const Group& g,
                          const ChainConsts& cc, const NttTables& T, cudaStream_t st) {
  ChainArgs a = chain_args(g, cc, T);
  a.slabs = slabs_dev;
  a.a_out = a_out;
  const uint32_t mask = 2 * g.n - 1;
  a.inv5 = inv5_mod2n(2 * g.n);
  a.c_first = pow_mod2n(5, g.L - 1, mask);
  a.cinv_first = pow_mod2n(a.inv5, g.L - 1, mask);
  const size_t smem = chain_smem(g, 0);
  dim3 grid(2, SIMD * g.H, nshards);
  if (g.log2n == LOG2_N_MAX) {
    set_smem(primary_chain_kernel<LOG2_N_MAX>, smem);
    primary_chain_kernel<LOG2_N_MAX><<<grid, CT, smem, st>>>(a);
  } else {
    set_smem(primary_chain_kernel<0>, smem);
    primary_chain_kernel<0><<<grid, CT, smem, st>>>(a);
  }
}

void launch_primary_finalize(const uint32_t* a_out, int nshards, uint64_t* a_zq, uint32_t* a_ms, const Group& g,
                             const NttTables& T, cudaStream_t st) {
  const size_t smem = (size_t)2 * g.n * 4;
  dim3 grid(SIMD, nshards);
  primary_finalize_kernel<<<grid, 256, smem, st>>>(a_out, a_zq, a_ms, g, T, host_crt_const());
}

void launch_secondary_chain(const uint32_t* E, const uint32_t* qv, size_t qv_stride, int nq, uint32_t* out,
                            const Group& g, const ChainConsts& cc, const NttTables& T, cudaStream_t st,
                            bool clustered) {
  ChainArgs a = chain_args(g, cc, T);
  a.E = E;
  a.qv = qv;
  a.qv_stride = qv_stride;
  a.nl = nq * CTXT_PARTS;
  a.out = out;
  // one part and factor per block in 2-block clusters (88 KiB, 64 registers;
  // for a few queries: the chains run on many SMs, and a block fits beside a
  // scan block) while the chunk needs at most one block per SM; beyond that one
  // block per part carrying both factors (no cluster barrier, twice the work
  // per barrier): at N = 2048 the register-transform kernel, else the generic one.
  // `clustered` asks for the cluster form at any chunk size (it shares SMs with
  // a running scan; the pipeline tuner picks it per group size when faster)
  int sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool full = g.log2n == LOG2_N_MAX;
  if (clustered || (long)nq * CTXT_PARTS * g.H * 2 <= sms) {
    const size_t smem = chain_smem(g, 1);
    const dim3 grid(2, CTXT_PARTS * g.H, nq);
    if (full) {
      set_smem(secondary_chain_kernel<1, LOG2_N_MAX>, smem);
      secondary_chain_kernel<1, LOG2_N_MAX><<<grid, CT, smem, st>>>(a);
    } else {
      set_smem(secondary_chain_kernel<1, 0>, smem);
      secondary_chain_kernel<1, 0><<<grid, CT, smem, st>>>(a);
    }
  } else if (full) {
    const size_t smem = (size_t)SEC2K_WORDS * 4;
    set_smem(secondary_chain2k_kernel, smem);
    secondary_chain2k_kernel<<<dim3(CTXT_PARTS * g.H, nq), CT, smem, st>>>(a);
  } else {
    const size_t smem = (size_t)SEC_DUAL_WORDS * g.n * 4;
    set_smem(secondary_dual_kernel<0>, smem);
    secondary_dual_kernel<0><<<dim3(CTXT_PARTS * g.H, nq), CT, smem, st>>>(a);
  }
}

}  // namespace dnspir
