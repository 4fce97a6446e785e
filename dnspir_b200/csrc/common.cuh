// common.cuh -- parameters and exact modular arithmetic shared by all kernels.
//
// Ring parameters follow crates/pir/src/base_pir.rs:72-78 (two RNS factors
// q1 = 2^26 - 2^12 + 1, q2 = 2^25 - 2^12 + 1, N = 2^11, two gadget digits of
// base 2^26), double_pir.rs:36-41 (t = 1025, 3 ciphertext parts) and
// pir_wrapper.rs:57-72 (wire bit widths).  Every device value in the NTT
// domain is kept canonical, in [0, p).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dnspir {

constexpr uint32_t P1 = (1u << 26) - (1u << 12) + 1;  // 67104769
constexpr uint32_t P2 = (1u << 25) - (1u << 12) + 1;  // 33550337
constexpr uint64_t QQ = (uint64_t)P1 * (uint64_t)P2;
constexpr int SIMD = 8;
constexpr int GK_DIGITS = 2;
constexpr int LOG2_B = 26;
constexpr uint32_t TPLAIN = 1025;
constexpr int CTXT_PARTS = 3;
constexpr int LOG2_N_MAX = 11;
constexpr int N_MAX = 1 << LOG2_N_MAX;
constexpr int PRIM_A_BITS = 17, PRIM_B_BITS = 12;
constexpr int SEC_A_BITS = 17, SEC_B_BITS = 12;
constexpr int GK_BITS = 50, PQ_BITS = 34, SQ_BITS = 34;

// Per-factor constants.  mu = floor(2^64 / p) for Barrett reduction of any
// 64-bit value; shoup companions of twiddles are floor(w 2^32 / p).
struct PrimeConst {
  uint32_t p;
  uint64_t mu;
};

__host__ __device__ constexpr uint64_t barrett_mu(uint32_t p) { return ~0ull / p; }

// x mod p for any 64-bit x (two correction steps cover the Barrett error).
__device__ __forceinline__ uint32_t reduce64(uint64_t x, uint32_t p, uint64_t mu) {
  uint64_t q = __umul64hi(x, mu);
  uint64_t r = x - q * p;
  r = r >= p ? r - p : r;
  r = r >= p ? r - p : r;
  return (uint32_t)r;
}
__device__ __forceinline__ uint32_t mul_mod(uint32_t a, uint32_t b, uint32_t p, uint64_t mu) {
  return reduce64((uint64_t)a * b, p, mu);
}
__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) {
  uint32_t s = a + b;
  return s >= p ? s - p : s;
}
__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
  return a >= b ? a - b : a + p - b;
}
// x * w mod p with the Shoup companion wq = floor(w 2^32 / p); x < 2^32, w < p.
__device__ __forceinline__ uint32_t shoup_mul(uint32_t x, uint32_t w, uint32_t wq, uint32_t p) {
  uint32_t q = __umulhi(x, wq);
  uint32_t r = x * w - q * p;
  return r >= p ? r - p : r;
}

// Signed integer -> [0, p).  Valid for |v| < 2^62.
__device__ __forceinline__ uint32_t smod(int64_t v, uint32_t p) {
  int64_t r = v % (int64_t)p;
  return (uint32_t)(r < 0 ? r + p : r);
}

// CRT of canonical residues to [0, q): v = (c1 q2^-1 mod q1) q2 + (c2 q1^-1 mod q2) q1
// (from_simd_element, base_pir.rs:905-935).
struct CrtConst {
  uint32_t q2inv1, q1inv2;  // q2^-1 mod q1, q1^-1 mod q2
};
__device__ __forceinline__ uint64_t crt(uint32_t c1, uint32_t c2, CrtConst cc) {
  uint32_t x1 = mul_mod(c1, cc.q2inv1, P1, barrett_mu(P1));
  uint32_t x2 = mul_mod(c2, cc.q1inv2, P2, barrett_mu(P2));
  uint64_t v = (uint64_t)x1 * P2 + (uint64_t)x2 * P1;
  return v >= QQ ? v - QQ : v;
}

// mod_switch_encode (bfv.rs:52-58) of a canonical v in [0, q):
// round(v 2^bits / q) mod 2^bits.  (Rounding the centred lift gives the same
// value mod 2^bits; q is odd, so no ties occur.)  A double estimate is
// corrected exactly with 128-bit integers.
__device__ __forceinline__ uint32_t ms_encode(uint64_t v, int bits) {
  double est = (double)v * ((double)(1ull << bits) * (1.0 / (double)QQ));  // within one of the result
  int64_t r = (int64_t)floor(est + 0.5);
  unsigned __int128 num = ((unsigned __int128)v << (bits + 1)) + QQ;
  unsigned __int128 two_q = (unsigned __int128)(2 * QQ);
  unsigned __int128 lo = two_q * (unsigned __int128)(r < 0 ? 0 : r);
  if (r > 0 && num < lo) r--;
  else if (num >= lo + two_q) r++;
  return (uint32_t)((uint64_t)r & ((1ull << bits) - 1));
}
// mod_switch_decode (bfv.rs:61-69): floor(x q / 2^bits), x < 2^bits, bits <= 63.
__device__ __forceinline__ uint64_t ms_decode(uint64_t x, int bits) {
  unsigned __int128 v = (unsigned __int128)x * QQ;
  return (uint64_t)(v >> bits);
}

// index of the odd residue g mod 2N (galois_to_index with group order N,
// base_pir.rs:189-191)
__host__ __device__ __forceinline__ uint32_t gidx(uint32_t g, uint32_t two_n_mask) { return (g & two_n_mask) >> 1; }

}  // namespace dnspir
