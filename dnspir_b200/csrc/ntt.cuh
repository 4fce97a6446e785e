// ntt.cuh -- negacyclic NTT over Z/pZ, p in {q1, q2}, for shared-memory tiles.
//
// Semantics (weighted_ntt / inv_weighted_ntt of base_pir.rs:453-483): slot s
// of the transform of a(X) is a(zeta^-(2s+1)), zeta a primitive 2N-th root of
// unity.  The kernels use zeta = g^((p-1)/2N) with g the least quadratic
// non-residue; a length-n transform (n <= N) uses zeta^(N/n).  Any such root
// gives the same ring arithmetic, and the library's outputs are coefficients,
// so its choice never reaches a reply byte.
//
// The butterflies are Cooley-Tukey (forward, natural -> bit-reversed order)
// and Gentleman-Sande (inverse, bit-reversed -> natural) with merged
// negacyclic weights; twiddles are psi^brv(k), psi = zeta^-1, with Shoup
// companions.  One table of length N_MAX serves every length n <= N_MAX
// because the first n entries of the bit-reversed table are the table for n.
#pragma once
#include "common.cuh"

namespace dnspir {

struct NttTables {
  const uint32_t* fw[2];   // psi^brv(k)          k < N_MAX
  const uint32_t* fwq[2];  // shoup companions
  const uint32_t* iw[2];   // psi^-brv(k)
  const uint32_t* iwq[2];
  const uint2* fw2[2];     // (psi^brv(k), companion) pairs, for vector loads
  const uint2* iw2[2];
  uint32_t ninv[2][LOG2_N_MAX + 1];   // n^-1 mod p for n = 2^i
  uint32_t ninvq[2][LOG2_N_MAX + 1];
};

__device__ __forceinline__ uint32_t brv(uint32_t i, int logn) { return logn ? (__brev(i) >> (32 - logn)) : 0; }

__device__ __forceinline__ uint32_t prime_of(int pi) { return pi ? P2 : P1; }

namespace ntt_detail {

// Lazy butterflies with Shoup multiplication.  Inverse (Gentleman-Sande, as
// Harvey): values stay in [0, 2p).  Forward (Cooley-Tukey): the multiplied
// operand is brought to [0, 2p) by the Shoup product and nothing else is
// reduced, so each stage adds at most 2p to the bound of its outputs; a
// transform of at most 11 stages on inputs below 4p ends below 26p < 2^31
// (p < 2^26), and canon() brings the results to [0, p).
__device__ __forceinline__ uint32_t lazy_mul(uint32_t x, uint32_t w, uint32_t wq, uint32_t p) {
  return x * w - __umulhi(x, wq) * p;  // in [0, 2p) for any x < 2^32
}
__device__ __forceinline__ uint32_t red(uint32_t x, uint32_t m) { return x >= m ? x - m : x; }
// x mod p for any x < 2^32, p in {q1, q2}: the Shoup product x * 1 (companion
// floor(2^32 / p)) lands in [0, 2p), one conditional subtraction finishes
__device__ __forceinline__ uint32_t canon(uint32_t x, uint32_t p) {
  constexpr uint32_t ONE_Q1 = (uint32_t)((1ull << 32) / P1), ONE_Q2 = (uint32_t)((1ull << 32) / P2);
  return red(lazy_mul(x, 1u, p == P1 ? ONE_Q1 : ONE_Q2, p), p);
}
__device__ __forceinline__ void ct(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wq, uint32_t p) {
  const uint32_t t = lazy_mul(y, w, wq, p);
  y = x - t + 2 * p;
  x = x + t;
}
__device__ __forceinline__ void gs(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wq, uint32_t p) {
  const uint32_t a = x + y;
  const uint32_t d = x - y + 2 * p;
  x = red(a, 2 * p);
  y = lazy_mul(d, w, wq, p);
}

// cnt0 polynomials with factor 0 followed by cnt1 with factor 1, back to back,
// radix-4 passes (one barrier per two stages) and a radix-2 pass for odd logn.
// LOGN > 0 fixes the length at compile time (stage loops unroll, every index
// shift is a constant); the public entry points take that path for N = 2048.
template <int LOGN>
__device__ __forceinline__ void fwd_t(uint32_t* x, int logn_rt, int cnt0, int cnt1, const NttTables& T) {
  const int logn = LOGN ? LOGN : logn_rt;
  const int n = 1 << logn, cnt = cnt0 + cnt1;
  int s = 0;
#pragma unroll
  for (; s + 1 < logn; s += 2) {
    const int logt2 = logn - s - 2;
    const int t2 = 1 << logt2, t = 2 * t2, m = 1 << s;
    const int total = cnt << (logn - 2);
    for (int gg = threadIdx.x; gg < total; gg += blockDim.x) {
      const int poly = gg >> (logn - 2), g = gg & ((n >> 2) - 1);
      const int pi = poly >= cnt0;
      const uint32_t p = prime_of(pi);
      const uint32_t* __restrict__ tw = T.fw[pi];
      const uint32_t* __restrict__ twq = T.fwq[pi];
      const int blk = g >> logt2, r = g & (t2 - 1);
      uint32_t* a = x + (poly << logn) + (blk << (logt2 + 2)) + r;
      uint32_t v0 = a[0], v1 = a[t2], v2 = a[t], v3 = a[t + t2];
      const uint32_t w = __ldg(tw + m + blk), wq = __ldg(twq + m + blk);
      ct(v0, v2, w, wq, p);
      ct(v1, v3, w, wq, p);
      ct(v0, v1, __ldg(tw + 2 * m + 2 * blk), __ldg(twq + 2 * m + 2 * blk), p);
      ct(v2, v3, __ldg(tw + 2 * m + 2 * blk + 1), __ldg(twq + 2 * m + 2 * blk + 1), p);
      a[0] = v0, a[t2] = v1, a[t] = v2, a[t + t2] = v3;
    }
    __syncthreads();
  }
  if (s < logn) {  // last stage, t = 1; outputs brought to [0, p)
    const int total = cnt << (logn - 1);
    for (int bb = threadIdx.x; bb < total; bb += blockDim.x) {
      const int poly = bb >> (logn - 1), b = bb & ((n >> 1) - 1);
      const int pi = poly >= cnt0;
      const uint32_t p = prime_of(pi);
      uint32_t* a = x + (poly << logn) + 2 * b;
      uint32_t u = a[0], v = a[1];
      ct(u, v, __ldg(T.fw[pi] + n / 2 + b), __ldg(T.fwq[pi] + n / 2 + b), p);
      a[0] = canon(u, p);
      a[1] = canon(v, p);
    }
  } else {
    const int total = cnt << logn;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const uint32_t p = prime_of((b >> logn) >= cnt0);
      x[b] = canon(x[b], p);
    }
  }
  __syncthreads();
}

template <int LOGN>
__device__ __forceinline__ void inv_t(uint32_t* x, int logn_rt, int cnt0, int cnt1, const NttTables& T) {
  const int logn = LOGN ? LOGN : logn_rt;
  const int n = 1 << logn, cnt = cnt0 + cnt1;
  int s = 0;
#pragma unroll
  for (; s + 1 < logn; s += 2) {
    const int t = 1 << s;
    const int h0 = n >> (s + 1), h1 = n >> (s + 2);
    const int total = cnt << (logn - 2);
    for (int gg = threadIdx.x; gg < total; gg += blockDim.x) {
      const int poly = gg >> (logn - 2), g = gg & ((n >> 2) - 1);
      const int pi = poly >= cnt0;
      const uint32_t p = prime_of(pi);
      const uint32_t* __restrict__ tw = T.iw[pi];
      const uint32_t* __restrict__ twq = T.iwq[pi];
      const int blk = g >> s, r = g & (t - 1);
      uint32_t* a = x + (poly << logn) + (blk << (s + 2)) + r;
      uint32_t v0 = a[0], v1 = a[t], v2 = a[2 * t], v3 = a[3 * t];
      gs(v0, v1, __ldg(tw + h0 + 2 * blk), __ldg(twq + h0 + 2 * blk), p);
      gs(v2, v3, __ldg(tw + h0 + 2 * blk + 1), __ldg(twq + h0 + 2 * blk + 1), p);
      const uint32_t w = __ldg(tw + h1 + blk), wq = __ldg(twq + h1 + blk);
      gs(v0, v2, w, wq, p);
      gs(v1, v3, w, wq, p);
      a[0] = v0, a[t] = v1, a[2 * t] = v2, a[3 * t] = v3;
    }
    __syncthreads();
  }
  if (s < logn) {  // last stage, t = n/2
    const int total = cnt << (logn - 1);
    for (int jj = threadIdx.x; jj < total; jj += blockDim.x) {
      const int poly = jj >> (logn - 1), j = jj & ((n >> 1) - 1);
      const int pi = poly >= cnt0;
      const uint32_t p = prime_of(pi);
      uint32_t* a = x + (poly << logn) + j;
      uint32_t u = a[0], v = a[n / 2];
      gs(u, v, __ldg(T.iw[pi] + 1), __ldg(T.iwq[pi] + 1), p);
      a[0] = u;
      a[n / 2] = v;
    }
    __syncthreads();
  }
  // scale by n^-1 and bring to [0, p)
  const int total = cnt << logn;
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    const int pi = (b >> logn) >= cnt0;
    const uint32_t p = prime_of(pi);
    x[b] = red(lazy_mul(x[b], T.ninv[pi][logn], T.ninvq[pi][logn], p), p);
  }
  __syncthreads();
}

__device__ __forceinline__ void fwd(uint32_t* x, int logn, int cnt0, int cnt1, const NttTables& T) {
  if (logn == LOG2_N_MAX)
    fwd_t<LOG2_N_MAX>(x, logn, cnt0, cnt1, T);
  else
    fwd_t<0>(x, logn, cnt0, cnt1, T);
}
__device__ __forceinline__ void inv(uint32_t* x, int logn, int cnt0, int cnt1, const NttTables& T) {
  if (logn == LOG2_N_MAX)
    inv_t<LOG2_N_MAX>(x, logn, cnt0, cnt1, T);
  else
    inv_t<0>(x, logn, cnt0, cnt1, T);
}

}  // namespace ntt_detail

// Forward transform of `cnt` length-2^logn polynomials stored back to back in
// shared memory; input in [0, p), result slot s at position brv(s), in
// [0, p).  All threads of the block must call; ends with __syncthreads().
__device__ __forceinline__ void ntt_fwd_smem(uint32_t* x, int logn, int cnt, const NttTables& T, int pi) {
  if (pi)
    ntt_detail::fwd(x, logn, 0, cnt, T);
  else
    ntt_detail::fwd(x, logn, cnt, 0, T);
}

// Inverse of ntt_fwd_smem: input slot s at position brv(s), in [0, p); output
// natural coefficients scaled by n^-1, in [0, p).  Ends with __syncthreads().
__device__ __forceinline__ void ntt_inv_smem(uint32_t* x, int logn, int cnt, const NttTables& T, int pi) {
  if (pi)
    ntt_detail::inv(x, logn, 0, cnt, T);
  else
    ntt_detail::inv(x, logn, cnt, 0, T);
}

// The same two transforms with the prime chosen per polynomial: polys
// [0, cnt0) use factor 0 and [cnt0, cnt0 + cnt1) factor 1, in one set of
// passes (halves the number of barriers when both factors are transformed).
__device__ __forceinline__ void ntt_fwd_smem2(uint32_t* x, int logn, int cnt0, int cnt1, const NttTables& T) {
  ntt_detail::fwd(x, logn, cnt0, cnt1, T);
}
__device__ __forceinline__ void ntt_inv_smem2(uint32_t* x, int logn, int cnt0, int cnt1, const NttTables& T) {
  ntt_detail::inv(x, logn, cnt0, cnt1, T);
}

}  // namespace dnspir
