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
  uint32_t ninv[2][LOG2_N_MAX + 1];   // n^-1 mod p for n = 2^i
  uint32_t ninvq[2][LOG2_N_MAX + 1];
};

__device__ __forceinline__ uint32_t brv(uint32_t i, int logn) { return logn ? (__brev(i) >> (32 - logn)) : 0; }

__device__ __forceinline__ uint32_t prime_of(int pi) { return pi ? P2 : P1; }

// Forward transform of `cnt` length-2^logn polynomials stored back to back in
// shared memory; result slot s sits at position brv(s).  All threads of the
// block must call; ends with __syncthreads().
__device__ __forceinline__ void ntt_fwd_smem(uint32_t* x, int logn, int cnt, const NttTables& T, int pi) {
  const uint32_t p = prime_of(pi);
  const uint32_t* __restrict__ tw = T.fw[pi];
  const uint32_t* __restrict__ twq = T.fwq[pi];
  const int half = 1 << (logn - 1);
  const int total = cnt << (logn - 1);
  for (int s = 0; s < logn; s++) {
    const int logt = logn - 1 - s;
    const int t = 1 << logt;
    const int m = 1 << s;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int poly = b >> (logn - 1);
      const int k = b & (half - 1);
      const int i = k >> logt;
      const int j = (i << (logt + 1)) + (k & (t - 1));
      uint32_t* a = x + (poly << logn);
      const uint32_t w = __ldg(tw + m + i), wq = __ldg(twq + m + i);
      const uint32_t U = a[j];
      const uint32_t V = shoup_mul(a[j + t], w, wq, p);
      a[j] = add_mod(U, V, p);
      a[j + t] = sub_mod(U, V, p);
    }
    __syncthreads();
  }
}

// Inverse of ntt_fwd_smem: input slot s at position brv(s), output natural
// coefficients (scaled by n^-1).  Ends with __syncthreads().
__device__ __forceinline__ void ntt_inv_smem(uint32_t* x, int logn, int cnt, const NttTables& T, int pi) {
  const uint32_t p = prime_of(pi);
  const uint32_t* __restrict__ tw = T.iw[pi];
  const uint32_t* __restrict__ twq = T.iwq[pi];
  const int half = 1 << (logn - 1);
  const int total = cnt << (logn - 1);
  for (int s = 0; s < logn; s++) {
    const int t = 1 << s;
    const int h = half >> s;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int poly = b >> (logn - 1);
      const int k = b & (half - 1);
      const int i = k >> s;
      const int j = (i << (s + 1)) + (k & (t - 1));
      uint32_t* a = x + (poly << logn);
      const uint32_t w = __ldg(tw + h + i), wq = __ldg(twq + h + i);
      const uint32_t U = a[j], V = a[j + t];
      a[j] = add_mod(U, V, p);
      a[j + t] = shoup_mul(sub_mod(U, V, p), w, wq, p);
    }
    __syncthreads();
  }
  const uint32_t ni = T.ninv[pi][logn], niq = T.ninvq[pi][logn];
  const int n_all = cnt << logn;
  for (int b = threadIdx.x; b < n_all; b += blockDim.x) x[b] = shoup_mul(x[b], ni, niq, p);
  __syncthreads();
}

// The same two transforms with the prime chosen per polynomial: polys
// [0, cnt0) use factor 0 and [cnt0, cnt0 + cnt1) factor 1, in one set of
// stages (halves the number of barriers when both factors are transformed).
__device__ __forceinline__ void ntt_fwd_smem2(uint32_t* x, int logn, int cnt0, int cnt1, const NttTables& T) {
  const int half = 1 << (logn - 1);
  const int cnt = cnt0 + cnt1;
  const int total = cnt << (logn - 1);
  for (int s = 0; s < logn; s++) {
    const int logt = logn - 1 - s;
    const int t = 1 << logt;
    const int m = 1 << s;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int poly = b >> (logn - 1);
      const int pi = poly >= cnt0;
      const uint32_t p = prime_of(pi);
      const int k = b & (half - 1);
      const int i = k >> logt;
      const int j = (i << (logt + 1)) + (k & (t - 1));
      uint32_t* a = x + (poly << logn);
      const uint32_t w = __ldg(T.fw[pi] + m + i), wq = __ldg(T.fwq[pi] + m + i);
      const uint32_t U = a[j];
      const uint32_t V = shoup_mul(a[j + t], w, wq, p);
      a[j] = add_mod(U, V, p);
      a[j + t] = sub_mod(U, V, p);
    }
    __syncthreads();
  }
}
__device__ __forceinline__ void ntt_inv_smem2(uint32_t* x, int logn, int cnt0, int cnt1, const NttTables& T) {
  const int half = 1 << (logn - 1);
  const int cnt = cnt0 + cnt1;
  const int total = cnt << (logn - 1);
  for (int s = 0; s < logn; s++) {
    const int t = 1 << s;
    const int h = half >> s;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int poly = b >> (logn - 1);
      const int pi = poly >= cnt0;
      const uint32_t p = prime_of(pi);
      const int k = b & (half - 1);
      const int i = k >> s;
      const int j = (i << (s + 1)) + (k & (t - 1));
      uint32_t* a = x + (poly << logn);
      const uint32_t w = __ldg(T.iw[pi] + h + i), wq = __ldg(T.iwq[pi] + h + i);
      const uint32_t U = a[j], V = a[j + t];
      a[j] = add_mod(U, V, p);
      a[j + t] = shoup_mul(sub_mod(U, V, p), w, wq, p);
    }
    __syncthreads();
  }
  const int n_all = cnt << logn;
  for (int b = threadIdx.x; b < n_all; b += blockDim.x) {
    const int pi = (b >> logn) >= cnt0;
    x[b] = shoup_mul(x[b], T.ninv[pi][logn], T.ninvq[pi][logn], prime_of(pi));
  }
  __syncthreads();
}

}  // namespace dnspir
