// dnspir_oracle.cpp -- CPU restatement of the server-side answer path of
// DNSPIR's two-level BFV PIR (reference: crates/pir of FeanorTheElf/dnspir).
//
// THIS IS TEST INFRASTRUCTURE.  It is the checker the CUDA library in
// dnspir_b200/ is compared against (bit-exact reply bytes), and it is also the
// timed CPU baseline ("port").  It is never linked into, called by, or used as
// a fallback of the product library.
//
// Parity status:
//   * pinned by the reference's own known-answer tests, restated in
//     tests/test_oracle.py: the N = 8 shard-layout tests
//     (crates/pir/src/base_pir.rs:1281-1411), the decrypt-equality tests at
//     N = 256 (base_pir.rs:1413-1537, double_pir.rs:328-451), the codec round
//     trip (pir_wrapper.rs:442-452) and the reduction test (simd_zn.rs:490-542);
//   * `expand` (seed -> uniform a-part) is PARITY UNPINNED: the reference draws
//     it with feanor-math 3.5.18's `random_element` over rand_chacha 0.3.1's
//     StdRng, neither of which is present.  `expand` below follows StdRng's
//     ChaCha12 word stream and samples each coefficient by masked rejection;
//     the sampler itself is this project's definition.  Callers can replace the
//     six a-parts wholesale (orc_set_aparts) if reference vectors are supplied.
//
// Every value here is kept canonical (in [0, p)); the reference keeps lazily
// reduced representatives (<= 2p, simd_zn.rs:44-47).  Every quantity that
// reaches an output of the reference passes through an exact reduction first
// (simd_zn.rs:206-218, 251-255; base_pir.rs:905-935), so the two agree bit for
// bit.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <atomic>
#include <thread>
#include <immintrin.h>

typedef unsigned __int128 u128;
typedef __int128 i128;

namespace orc {

// ---- constants: base_pir.rs:72-78, double_pir.rs:36-41, pir_wrapper.rs:57-72
static const int64_t Q1 = (1LL << 26) - (1LL << 12) + 1;
static const int64_t Q2 = (1LL << 25) - (1LL << 12) + 1;
static const int64_t QQ = Q1 * Q2;
static const int SIMD = 8;
static const int GK_DIGITS = 2;
static const int LOG2_B = 26;
static const int64_t TPLAIN = 1025;
static const int CTXT_PARTS = 3;
static const int BATCH = 2;
static const int PRIM_A_BITS = 17, PRIM_B_BITS = 12;
static const int SEC_A_BITS = 17, SEC_B_BITS = 12;
static const int GK_BITS = 50, PQ_BITS = 34, SQ_BITS = 34;
static const int SK_HWT = 128;
static const double SIGMA = 3.2;
static const int LOG2_N_WIRE = 11;

// SEEDS: base_pir.rs:64-71 (SHA-3 of the six Star Wars titles)
static const uint8_t SEEDS[6][32] = {
    {0xda, 0xd2, 0x0c, 0x14, 0x2d, 0xeb, 0x8b, 0xb4, 0xd6, 0x63, 0x20, 0xee, 0x07, 0xb1, 0xc1, 0x90,
     0xec, 0x25, 0xc0, 0xa1, 0x54, 0x1c, 0xca, 0xf5, 0x98, 0xfa, 0x22, 0xff, 0xdf, 0xdd, 0x68, 0xba},
    {0xd3, 0xc5, 0xf6, 0xee, 0xb3, 0x3a, 0x4c, 0xf3, 0x33, 0x51, 0x6c, 0xe2, 0x73, 0xd5, 0x74, 0x76,
     0xb5, 0x79, 0x6c, 0xce, 0x9c, 0xf3, 0x37, 0xa1, 0x9c, 0x84, 0xbc, 0xbe, 0xa4, 0x3d, 0x2c, 0xb5},
    {0x95, 0x27, 0xb8, 0x6c, 0x30, 0xdc, 0x30, 0xcf, 0x1b, 0xb1, 0x74, 0xc3, 0xcd, 0x6c, 0xd7, 0x50,
     0x72, 0x09, 0xda, 0xa5, 0x4b, 0xbd, 0xb9, 0x99, 0x04, 0x14, 0x00, 0x08, 0x3d, 0x68, 0x24, 0x8a},
    {0x4c, 0xa2, 0xf6, 0x47, 0x8a, 0x58, 0x11, 0x91, 0x67, 0x67, 0x41, 0x00, 0x2a, 0x00, 0xed, 0xd1,
     0xac, 0x97, 0xf9, 0x30, 0x98, 0x0b, 0x7f, 0xbe, 0xf0, 0x33, 0xb4, 0x48, 0x23, 0x4b, 0x21, 0x6b},
    {0x98, 0xfc, 0x62, 0xc5, 0x17, 0x52, 0x0e, 0x5d, 0x29, 0xfc, 0x30, 0x7e, 0x73, 0xef, 0xb1, 0x0e,
     0x14, 0x18, 0xaa, 0x07, 0x0e, 0x32, 0x36, 0x4f, 0x89, 0x3f, 0xa8, 0xbd, 0x92, 0x13, 0x03, 0x27},
    {0xb3, 0x61, 0xdc, 0x94, 0x34, 0xdb, 0xba, 0xe9, 0x28, 0xe5, 0xc9, 0x64, 0xdc, 0x18, 0x02, 0x54,
     0x02, 0xfe, 0x81, 0xaa, 0xf7, 0x49, 0x17, 0x20, 0x8a, 0x6e, 0x6f, 0xd9, 0x55, 0x70, 0x2a, 0x21}};

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
#define ORC_CHECK(cond, msg)                  \
  do {                                        \
    if (!(cond)) throw ::orc::Error(msg);     \
  } while (0)

// ------------------------------------------------------- thread pool-less parallel for
static int g_threads = 0;  // 0 = hardware_concurrency
static int num_threads() {
  int n = g_threads > 0 ? g_threads : (int)std::thread::hardware_concurrency();
  return n > 0 ? n : 1;
}
// Runs f(i) for i in [0, n) on up to num_threads() threads (dynamic scheduling).
// The first exception thrown by any f(i) is rethrown on the calling thread.
template <class F>
static void parallel_for(size_t n, F f) {
  int nt = std::min<size_t>((size_t)num_threads(), n);
  if (nt <= 1) {
    for (size_t i = 0; i < n; i++) f(i);
    return;
  }
  std::atomic<size_t> next(0);
  std::exception_ptr err;
  std::atomic<bool> failed(false);
  auto work = [&]() {
    for (;;) {
      size_t i = next.fetch_add(1);
      if (i >= n || failed.load()) return;
      try {
        f(i);
      } catch (...) {
        if (!failed.exchange(true)) err = std::current_exception();
        return;
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; t++) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
  if (err) std::rethrow_exception(err);
}

// ---------------------------------------------------------------- integers
static inline int64_t mod_floor(int64_t a, int64_t m) {
  int64_t r = a % m;
  return r < 0 ? r + m : r;
}
static inline int64_t i128_mod(i128 a, int64_t m) {
  i128 r = a % (i128)m;
  if (r < 0) r += m;
  return (int64_t)r;
}
static uint64_t powmod(uint64_t b, uint64_t e, uint64_t p) {
  uint64_t r = 1 % p;
  b %= p;
  while (e) {
    if (e & 1) r = (uint64_t)((u128)r * b % p);
    b = (uint64_t)((u128)b * b % p);
    e >>= 1;
  }
  return r;
}
static uint64_t invmod(uint64_t a, uint64_t p) {  // p need not be prime
  int64_t t = 0, nt = 1, r = (int64_t)p, nr = (int64_t)(a % p);
  while (nr) {
    int64_t qq = r / nr;
    int64_t tmp = t - qq * nt; t = nt; nt = tmp;
    tmp = r - qq * nr; r = nr; nr = tmp;
  }
  ORC_CHECK(r == 1, "not invertible");
  return (uint64_t)mod_floor(t, (int64_t)p);
}
// feanor-math smallest_lift for odd modulus: representative in [-(m-1)/2, (m-1)/2]
static inline int64_t smallest_lift(int64_t x, int64_t m) { return x > m / 2 ? x - m : x; }

// Barrett reduction for a modulus below 2^31 of any 64-bit value.
struct Mod {
  uint64_t p;
  uint64_t m;  // floor(2^64 / p)
  explicit Mod(uint64_t p_ = 1) : p(p_), m((uint64_t)(((u128)1 << 64) / p_)) {}
  inline uint64_t red(uint64_t x) const {
    uint64_t q = (uint64_t)(((u128)x * m) >> 64);
    uint64_t r = x - q * p;
    while (r >= p) r -= p;
    return r;
  }
  inline uint64_t mul(uint64_t a, uint64_t b) const { return red(a * b); }
  inline uint64_t add(uint64_t a, uint64_t b) const { uint64_t s = a + b; return s >= p ? s - p : s; }
  inline uint64_t sub(uint64_t a, uint64_t b) const { return a >= b ? a - b : a + p - b; }
};

// ------------------------------------------------ StdRng (rand 0.8.6 / rand_chacha 0.3.1)
// ChaCha12 keyed by the 32-byte seed, 64-bit block counter in state words 12-13,
// stream id 0 in words 14-15, four blocks buffered per refill, and rand_core's
// BlockRng next_u32 / next_u64 word-consumption rules.
struct StdRng {
  uint32_t key[8];
  uint64_t counter = 0;
  uint32_t buf[64];
  int idx = 64;
  explicit StdRng(const uint8_t seed[32]) {
    for (int i = 0; i < 8; i++)
      key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) |
               ((uint32_t)seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
  }
  static inline uint32_t rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
  void block(uint64_t ctr, uint32_t* out) const {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                      key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                      (uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u};
    uint32_t x[16];
    memcpy(x, s, sizeof(x));
#define QR(a, b, c, d)                  \
  x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl(x[d], 16); \
  x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl(x[b], 12); \
  x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl(x[d], 8);  \
  x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl(x[b], 7);
    for (int r = 0; r < 6; r++) {
      QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
      QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
    }
#undef QR
    for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
  }
  void refill() {
    for (int b = 0; b < 4; b++) block(counter + b, buf + 16 * b);
    counter += 4;
    idx = 0;
  }
  uint32_t next_u32() {
    if (idx >= 64) refill();
    return buf[idx++];
  }
  uint64_t next_u64() {
    if (idx < 63) {
      uint64_t r = (uint64_t)buf[idx] | ((uint64_t)buf[idx + 1] << 32);
      idx += 2;
      return r;
    } else if (idx >= 64) {
      refill();
      idx = 2;
      return (uint64_t)buf[0] | ((uint64_t)buf[1] << 32);
    } else {
      uint64_t x = buf[63];
      refill();
      idx = 1;
      return x | ((uint64_t)buf[0] << 32);
    }
  }
  // standard-normal sample for the client's error terms (Box-Muller; the
  // reference uses rand_distr's ziggurat, bfv.rs:74 -- client side only)
  double normal() {
    double u1 = ((double)((next_u64() >> 11) + 1)) * (1.0 / 9007199254740992.0);
    double u2 = ((double)(next_u64() >> 11)) * (1.0 / 9007199254740992.0);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

// ------------------------------------------------------------- DFT engine
// out[i] = sum_t x_t * w^(i t), natural order in and out, radix-2 DIT.
struct Dft {
  uint64_t p = 0;
  size_t n = 0;
  Mod md;
  std::vector<uint64_t> tw;  // tw[h + j] = w^((n / (2h)) * j), h = len/2
  std::vector<uint32_t> rev;
  Dft() {}
  Dft(uint64_t p_, size_t n_, uint64_t w) : p(p_), n(n_), md(p_) {
    int logn = 0;
    while (((size_t)1 << logn) < n) logn++;
    ORC_CHECK(((size_t)1 << logn) == n, "dft length must be a power of two");
    rev.resize(n);
    for (size_t i = 0; i < n; i++) {
      size_t r = 0;
      for (int b = 0; b < logn; b++)
        if (i >> b & 1) r |= (size_t)1 << (logn - 1 - b);
      rev[i] = (uint32_t)r;
    }
    tw.assign(n > 1 ? n : 1, 0);
    for (size_t h = 1; h < n; h <<= 1) {
      uint64_t wl = powmod(w, n / (2 * h), p), cur = 1;
      for (size_t j = 0; j < h; j++) {
        tw[h + j] = cur;
        cur = md.mul(cur, wl);
      }
    }
  }
  // x: n elements of `lanes` interleaved lanes (element i lane k at x[i*lanes+k])
  void apply(uint64_t* x, int lanes) const {
    for (size_t i = 0; i < n; i++) {
      size_t r = rev[i];
      if (r > i)
        for (int k = 0; k < lanes; k++) std::swap(x[i * lanes + k], x[r * lanes + k]);
    }
    for (size_t h = 1; h < n; h <<= 1)
      for (size_t i = 0; i < n; i += 2 * h)
        for (size_t j = 0; j < h; j++) {
          uint64_t w = tw[h + j];
          uint64_t* a = x + (i + j) * lanes;
          uint64_t* b = x + (i + j + h) * lanes;
          for (int k = 0; k < lanes; k++) {
            uint64_t v = md.mul(b[k], w);
            uint64_t u = a[k];
            a[k] = md.add(u, v);
            b[k] = md.sub(u, v);
          }
        }
  }
};

// smallest g >= 2 with g^((p-1)/2) != 1; zeta = g^((p-1)/2N) is then a primitive
// 2N-th root of unity (the reference takes feanor's get_prim_root_of_unity_pow2,
// base_pir.rs:325-332; the outputs do not depend on which root is used)
static uint64_t prim_root_2n(uint64_t p, size_t two_n) {
  ORC_CHECK((p - 1) % two_n == 0, "2N does not divide p-1");
  for (uint64_t g = 2;; g++)
    if (powmod(g, (p - 1) / 2, p) != 1) return powmod(g, (p - 1) / two_n, p);
}

// Per-ring-dimension context: both RNS factors, db.zeta and the weighted NTTs
// of base_pir.rs:453-483.
struct Ring {
  int log2n;
  size_t n;
  uint64_t p[2];
  Mod md[2];
  uint64_t zeta[2];
  std::vector<uint64_t> zneg[2], zpos[2];  // zeta^(-i), zeta^(i), i < N
  Dft fwd[2], inv[2];                      // fft(., zeta^2) and its inverse
  uint64_t ninv[2];
  explicit Ring(int log2n_) : log2n(log2n_), n((size_t)1 << log2n_) {
    p[0] = Q1;
    p[1] = Q2;
    for (int pi = 0; pi < 2; pi++) {
      md[pi] = Mod(p[pi]);
      zeta[pi] = prim_root_2n(p[pi], 2 * n);
      uint64_t zi = invmod(zeta[pi], p[pi]);
      zneg[pi].resize(n);
      zpos[pi].resize(n);
      uint64_t a = 1, b = 1;
      for (size_t i = 0; i < n; i++) {
        zneg[pi][i] = a;
        zpos[pi][i] = b;
        a = md[pi].mul(a, zi);
        b = md[pi].mul(b, zeta[pi]);
      }
      uint64_t z2 = md[pi].mul(zeta[pi], zeta[pi]);
      // feanor fft with root w: out[i] = sum_t x_t w^(-i t)
      fwd[pi] = Dft(p[pi], n, invmod(z2, p[pi]));
      inv[pi] = Dft(p[pi], n, z2);
      ninv[pi] = invmod(n, p[pi]);
    }
  }
  // weighted_ntt (base_pir.rs:453-466): slot i <- f(zeta^-(2i+1))
  void weighted_ntt(int pi, uint64_t* x, int lanes) const {
    const Mod& m = md[pi];
    for (size_t i = 0; i < n; i++)
      for (int k = 0; k < lanes; k++) x[i * lanes + k] = m.mul(x[i * lanes + k], zneg[pi][i]);
    fwd[pi].apply(x, lanes);
  }
  // inv_weighted_ntt (base_pir.rs:471-483)
  void inv_weighted_ntt(int pi, uint64_t* x, int lanes) const {
    const Mod& m = md[pi];
    inv[pi].apply(x, lanes);
    for (size_t i = 0; i < n; i++) {
      uint64_t s = m.mul(ninv[pi], zpos[pi][i]);
      for (int k = 0; k < lanes; k++) x[i * lanes + k] = m.mul(x[i * lanes + k], s);
    }
  }
};

static std::shared_ptr<Ring> get_ring(int log2n) {
  static std::shared_ptr<Ring> cache[12];
  ORC_CHECK(log2n >= 1 && log2n <= 11, "log2 N out of range");
  if (!cache[log2n]) cache[log2n] = std::make_shared<Ring>(log2n);
  return cache[log2n];
}

// ------------------------------------------------ IndexGroup (base_pir.rs:132-191)
struct IndexGroup {
  size_t N, l;
  size_t loop_len() const { return l < N ? l : N / 2; }
  size_t qbp() const { return N / 2 / loop_len(); }
  bool conj() const { return l == N; }
};
static IndexGroup make_group(size_t N, size_t l) {
  ORC_CHECK(l >= 1 && N % l == 0, "group order must divide N");
  ORC_CHECK(l == N || 2 * l <= N, "subgroup order must be at most N/2");  // base_pir.rs:150-154
  return IndexGroup{N, l};
}
// index_to_galois / galois_to_index with group_order = N (base_pir.rs:185-191)
static inline int64_t idx2gal(size_t /*N*/, int64_t i) { return 2 * i + 1; }
static inline size_t gal2idx(size_t N, int64_t g) {
  int64_t m = 2 * (int64_t)N;
  int64_t x = mod_floor(g, m);
  ORC_CHECK(x % 2 == 1, "galois element must be odd");
  return (size_t)((x - 1) / 2);
}

// ----------------------------------------------------------------- BFV (bfv.rs)
typedef std::vector<int64_t> Poly;  // coefficients in [0, q) (or [0, t))

// expand (bfv.rs:46-49): coefficient i = 0..N-1 in turn, each the low
// ceil(log2 q) = 51 bits of one StdRng next_u64, drawn again while >= q -- the
// uniform-below-bound rule feanor-math 3.5.18's random_element applies per
// coefficient, as this project restates it (the crate is not available here to
// confirm the restatement)
static Poly expand(size_t N, const uint8_t seed[32]) {
  StdRng rng(seed);
  Poly out(N);
  const uint64_t mask = ((uint64_t)1 << 51) - 1;
  for (size_t i = 0; i < N; i++) {
    uint64_t x;
    do x = rng.next_u64() & mask;
    while (x >= (uint64_t)QQ);
    out[i] = (int64_t)x;
  }
  return out;
}

// a-parts in effect (may be replaced wholesale): [gk0, gk1, qry1, qry1conj, qry2, qry2conj]
struct APartStore {
  std::vector<Poly> parts[12];  // per log2n; empty = use expand()
};
static APartStore g_aparts;
static const Poly& apart(size_t N, int which) {
  int log2n = 0;
  while (((size_t)1 << log2n) < N) log2n++;
  static std::vector<Poly> expanded[12];
  if (!g_aparts.parts[log2n].empty()) return g_aparts.parts[log2n][which];
  if (expanded[log2n].empty()) {
    expanded[log2n].resize(6);
    for (int s = 0; s < 6; s++) expanded[log2n][s] = expand(N, SEEDS[s]);
  }
  return expanded[log2n][which];
}
// UsedSeeds (base_pir.rs:193-205): FirstSet = 0, SecondSet = 1
static const Poly& gk_a(size_t N, int k) { return apart(N, k); }
static const Poly& qry_a(size_t N, int used_seeds, int conj) { return apart(N, 2 + 2 * used_seeds + conj); }

// multiplication by a ternary secret in Z_q[X]/(X^N+1)
static Poly mul_sk(const Poly& a, const std::vector<int8_t>& sk) {
  size_t N = a.size();
  std::vector<i128> acc(N, 0);
  for (size_t j = 0; j < N; j++) {
    if (!sk[j]) continue;
    for (size_t i = 0; i < N; i++) {
      size_t d = i + j;
      i128 v = (i128)a[i] * sk[j];
      if (d >= N) acc[d - N] -= v;
      else acc[d] += v;
    }
  }
  Poly out(N);
  for (size_t i = 0; i < N; i++) out[i] = i128_mod(acc[i], QQ);
  return out;
}

// gen_sk (bfv.rs:37-45)
static std::vector<int8_t> gen_sk(size_t N, StdRng& rng, int hwt) {
  std::vector<int8_t> s(N, 0);
  for (int i = 0; i < hwt; i++) {
    size_t idx = (size_t)(rng.next_u64() % N);
    s[idx] = (int8_t)((int)(rng.next_u32() % 3) - 1);
  }
  return s;
}

// mod_switch_encode (bfv.rs:52-58): round(lift(c) * 2^BITS / q) mod 2^BITS
static uint64_t ms_encode(int64_t c, int bits) {
  i128 num = (i128)smallest_lift(c, QQ) * ((i128)1 << bits);
  // rounded division; q is odd and num is a multiple of 2, so no ties occur
  i128 two_q = 2 * (i128)QQ;
  i128 t = 2 * num + QQ;
  i128 r = t / two_q;
  if ((t % two_q) != 0 && t < 0) r -= 1;  // floor
  i128 res = (r + ((i128)1 << bits)) % ((i128)1 << bits);
  if (res < 0) res += ((i128)1 << bits);
  return (uint64_t)res;
}
// mod_switch_decode (bfv.rs:61-69): floor(x * q / 2^BITS) mod q
static int64_t ms_decode(uint64_t x, int bits) {
  i128 v = ((i128)x * QQ) >> bits;
  return i128_mod(v, QQ);
}

// enc_sym_b (bfv.rs:72-87); m has coefficients in [0, t)
static Poly enc_sym_b(size_t N, int64_t t, const Poly& a, StdRng& rng, const std::vector<int8_t>& sk,
                      const Poly& m, double sigma) {
  Poly e(N);
  for (size_t i = 0; i < N; i++) e[i] = mod_floor((int64_t)std::llround(rng.normal() * sigma), QQ);
  int64_t tinv = (int64_t)invmod((uint64_t)t, (uint64_t)QQ);
  Poly as = mul_sk(a, sk);
  Poly b(N);
  for (size_t i = 0; i < N; i++) {
    int64_t c = smallest_lift(m[i], t);
    i128 up = (i128)c * QQ;
    int64_t delta = smallest_lift(i128_mod(up, t), t);
    int64_t down = (int64_t)(((u128)(uint64_t)i128_mod(up - delta, QQ) * (uint64_t)tinv) % (u128)QQ);
    b[i] = mod_floor(mod_floor(e[i] - as[i], QQ) + down, QQ);
  }
  return b;
}

// dec (bfv.rs:90-102): returns coefficients in [0, t)
static Poly dec(size_t N, int64_t t, const std::vector<int8_t>& sk, const Poly& a, const Poly& b) {
  Poly as = mul_sk(a, sk);
  int64_t qinv_t = (int64_t)invmod((uint64_t)(QQ % t), (uint64_t)t);
  Poly out(N);
  for (size_t i = 0; i < N; i++) {
    int64_t c = smallest_lift(mod_floor(as[i] + b[i], QQ), QQ);
    i128 up = (i128)c * t;
    int64_t delta = smallest_lift(i128_mod(up, QQ), QQ);
    int64_t v = i128_mod((up - delta) % t, t);
    out[i] = (v * qinv_t) % t;
  }
  return out;
}

// gen_gk_b (bfv.rs:105-125) with g = 5
static std::vector<Poly> gen_gk_b(size_t N, StdRng& rng, const std::vector<int8_t>& sk, int g, int digits,
                                  int log2b, double sigma) {
  int64_t m = 2 * (int64_t)N;
  int64_t inv_g = (int64_t)invmod((uint64_t)g, (uint64_t)m);
  Poly gal_s(N);
  for (size_t i = 0; i < N; i++) {
    int64_t ni = mod_floor((int64_t)i * inv_g, m);
    if (ni > (int64_t)N) gal_s[i] = mod_floor(-(int64_t)sk[ni - N], QQ);
    else gal_s[i] = mod_floor((int64_t)sk[ni], QQ);
  }
  std::vector<Poly> out;
  for (int d = 0; d < digits; d++) {
    const Poly& a = gk_a(N, d);
    Poly e(N);
    for (size_t i = 0; i < N; i++) e[i] = mod_floor((int64_t)std::llround(rng.normal() * sigma), QQ);
    Poly as = mul_sk(a, sk);
    int64_t scale = (int64_t)powmod(((uint64_t)1 << log2b) % QQ, d, QQ);
    Poly b(N);
    for (size_t i = 0; i < N; i++)
      b[i] = mod_floor(mod_floor(e[i] - as[i], QQ) + (int64_t)(((u128)gal_s[i] * (uint64_t)scale) % QQ), QQ);
    out.push_back(b);
  }
  return out;
}

// ------------------------------------------------------------- PIRDatabase
// One preprocessed shard (base_pir.rs:229-255).  Arrays are stored row-major
// as the reference's slab: [row i < loop_len][slot j < N][lane k < 8].
struct Shard {
  std::shared_ptr<Ring> R;
  IndexGroup ig;
  int used_seeds;
  std::vector<uint64_t> te[2][2];     // transformed_entries[conj][prime]
  std::vector<uint64_t> gk[2][2][2];  // inner_prod_gk[conj][digit][prime]
  std::vector<uint64_t> reply_a[2];   // [prime] N x 8
  bool has_reply_a = false;
};

// coset_ntt (base_pir.rs:397-444); values: l elements x 8 lanes mod q1
static void coset_ntt(const Ring& R, const IndexGroup& ig, int64_t zeta_power, uint64_t* values,
                      const Dft& fft_l) {
  const size_t N = ig.N, l = ig.l;
  const int64_t m = 2 * (int64_t)N;
  const Mod& md = R.md[0];
  int64_t zp = mod_floor(zeta_power, m);
  ORC_CHECK(zp % (int64_t)ig.qbp() == 0, "zeta_power must be divisible by query_base_power");
  int64_t coset = zp % (m / (int64_t)l);
  uint64_t z = powmod(R.zeta[0], (uint64_t)coset, R.p[0]);
  uint64_t zinv = invmod(z, R.p[0]);
  uint64_t cur = 1;
  for (size_t i = 0; i < l; i++) {
    for (int k = 0; k < SIMD; k++) values[i * SIMD + k] = md.mul(values[i * SIMD + k], cur);
    cur = md.mul(cur, zinv);
  }
  fft_l.apply(values, SIMD);
  // permute: new[i] = old[galois_to_index(x_i)], galois_to_index(x) = (lift(-x) - coset) / (m/l)
  auto g2i = [&](int64_t x) -> size_t {
    int64_t v = mod_floor(-x, m) - coset;
    ORC_CHECK(v % (m / (int64_t)l) == 0, "coset permutation not exact");
    return (size_t)(v / (m / (int64_t)l));
  };
  int64_t zpn = mod_floor(-zp, m);
  std::vector<uint64_t> old(values, values + l * SIMD);
  int64_t gpow = 1;
  for (size_t i = 0; i < l; i++) {
    size_t src;
    if (ig.conj()) {
      if (i == N / 2) gpow = 1;
      src = i < N / 2 ? g2i(zpn * gpow % m) : g2i(zp * gpow % m);
    } else {
      src = g2i(zpn * gpow % m);
    }
    gpow = gpow * 5 % m;
    for (int k = 0; k < SIMD; k++) values[i * SIMD + k] = old[src * SIMD + k];
  }
}

// set_transformed_entries (base_pir.rs:662-772).  entries: (8 l) x N plaintext
// coefficients in [0, t), entry index e = 8 j + k (column j, lane k).
static void set_transformed_entries(Shard& db, const uint16_t* entries) {
  const Ring& R = *db.R;
  const size_t N = R.n, l = db.ig.l, L = db.ig.loop_len();
  const int64_t m = 2 * (int64_t)N;
  const Mod& m1 = R.md[0];
  ORC_CHECK(2 * TPLAIN * (int64_t)N < Q1, "max_coeff >= q1");  // :668-670
  // STEP 1 (:675-684): M (N x l) of 8-lane values, M[i][j][k] = coeff i of entry 8j+k
  std::vector<uint64_t> M(N * l * SIMD);
  for (size_t j = 0; j < l; j++)
    for (int k = 0; k < SIMD; k++) {
      const uint16_t* e = entries + ((size_t)j * SIMD + k) * N;
      for (size_t i = 0; i < N; i++) {
        ORC_CHECK(e[i] < TPLAIN, "entry coefficient must be below t");
        M[(i * l + j) * SIMD + k] = e[i];
      }
    }
  // STEP 2 (:688-692): column-wise weighted NTT in q1
  parallel_for(l, [&](size_t j) {
    std::vector<uint64_t> c(N * SIMD);
    for (size_t i = 0; i < N; i++)
      for (int k = 0; k < SIMD; k++) c[i * SIMD + k] = M[(i * l + j) * SIMD + k];
    R.weighted_ntt(0, c.data(), SIMD);
    for (size_t i = 0; i < N; i++)
      for (int k = 0; k < SIMD; k++) M[(i * l + j) * SIMD + k] = c[i * SIMD + k];
  });
  // STEP 3 (:699-702): row-wise coset NTT, zeta_power = (2i+1) * (-query_base_power)
  {
    size_t logl = 0;
    while (((size_t)1 << logl) < l) logl++;
    uint64_t omega = powmod(R.zeta[0], (uint64_t)(m / (int64_t)l), R.p[0]);  // zeta^(2 << (log N - log l))
    Dft fft_l(R.p[0], l, invmod(omega, R.p[0]));
    int64_t base_power = mod_floor(-(int64_t)db.ig.qbp(), m);
    parallel_for(N, [&](size_t i) {
      coset_ntt(R, db.ig, mod_floor(idx2gal(N, (int64_t)i) * base_power, m), &M[i * l * SIMD], fft_l);
    });
  }
  // STEP 4 (:712-718): column j undergoes the automorphism g^-j
  {
    int64_t g_inv = (int64_t)invmod(5, (uint64_t)m);
    parallel_for(l, [&](size_t j) {
      int64_t aut = (int64_t)powmod((uint64_t)g_inv, j, (uint64_t)m);
      std::vector<uint64_t> c(N * SIMD);
      for (size_t i = 0; i < N; i++) {
        size_t src = gal2idx(N, aut * idx2gal(N, (int64_t)i) % m);
        for (int k = 0; k < SIMD; k++) c[i * SIMD + k] = M[(src * l + j) * SIMD + k];
      }
      for (size_t i = 0; i < N; i++)
        for (int k = 0; k < SIMD; k++) M[(i * l + j) * SIMD + k] = c[i * SIMD + k];
    });
  }
  // STEP 5 (:728-738): reverse each row within <g> and -<g>
  for (size_t i = 0; i < N; i++) {
    uint64_t* row = &M[i * l * SIMD];
    auto rev = [&](size_t a, size_t b) {  // reverse [a, b)
      while (b > a + 1) {
        b--;
        for (int k = 0; k < SIMD; k++) std::swap(row[a * SIMD + k], row[b * SIMD + k]);
        a++;
      }
    };
    if (db.ig.conj()) {
      rev(0, N / 2);
      rev(N / 2, N);
    } else {
      rev(0, l);
    }
  }
  // STEP 6 (:741-764): column c -> iNTT, lift, * l^-1 mod t, centred lift, NTT in q1 and q2
  for (int c = 0; c < 2; c++)
    for (int pi = 0; pi < 2; pi++) db.te[c][pi].assign(db.ig.conj() || c == 0 ? L * N * SIMD : 0, 0);
  int64_t scale = (int64_t)invmod((uint64_t)(l % TPLAIN), (uint64_t)TPLAIN);
  parallel_for(l, [&](size_t col) {
    std::vector<uint64_t> c(N * SIMD);
    for (size_t i = 0; i < N; i++)
      for (int k = 0; k < SIMD; k++) c[i * SIMD + k] = M[(i * l + col) * SIMD + k];
    R.inv_weighted_ntt(0, c.data(), SIMD);
    std::vector<uint64_t> r0(N * SIMD), r1(N * SIMD);
    for (size_t i = 0; i < N * SIMD; i++) {
      int64_t v = smallest_lift((int64_t)c[i], Q1);
      int64_t w = smallest_lift(mod_floor(mod_floor(v, TPLAIN) * scale, TPLAIN), TPLAIN);
      r0[i] = (uint64_t)mod_floor(w, Q1);
      r1[i] = (uint64_t)mod_floor(w, Q2);
    }
    R.weighted_ntt(0, r0.data(), SIMD);
    R.weighted_ntt(1, r1.data(), SIMD);
    int half = col < L ? 0 : 1;
    size_t row = col < L ? col : col - L;
    memcpy(&db.te[half][0][row * N * SIMD], r0.data(), N * SIMD * 8);
    memcpy(&db.te[half][1][row * N * SIMD], r1.data(), N * SIMD * 8);
  });
  (void)m1;
  db.has_reply_a = false;
}

// to_simd_element (base_pir.rs:865-878): 8 ring elements mod q -> per prime NTT (N x 8)
static void to_simd_element(const Ring& R, const Poly* els[SIMD], std::vector<uint64_t> out[2]) {
  const size_t N = R.n;
  for (int pi = 0; pi < 2; pi++) {
    out[pi].assign(N * SIMD, 0);
    for (size_t i = 0; i < N; i++)
      for (int k = 0; k < SIMD; k++)
        out[pi][i * SIMD + k] = (uint64_t)mod_floor(smallest_lift((*els[k])[i], QQ), (int64_t)R.p[pi]);
    R.weighted_ntt(pi, out[pi].data(), SIMD);
  }
}
static void to_simd_element_same(const Ring& R, const Poly& el, std::vector<uint64_t> out[2]) {
  const Poly* els[SIMD];
  for (int k = 0; k < SIMD; k++) els[k] = &el;
  to_simd_element(R, els, out);
}

// partial_gal (base_pir.rs:496-594).  current: [prime] N x `lanes`.  Returns
// reply_a = <Decomp(gal(a)), gk_a> and the two NTT'd digits.
// gka: [digit][prime] in the same N x `lanes` layout as `cur`.
static void partial_gal(const Ring& R, const std::vector<uint64_t> cur[2], const std::vector<uint64_t> gka[2][2],
                        std::vector<uint64_t> reply_a[2], std::vector<uint64_t> dig[2][2], int lanes) {
  const size_t N = R.n;
  const int64_t m = 2 * (int64_t)N;
  int64_t inv_g = (int64_t)invmod(5, (uint64_t)m);
  std::vector<uint64_t> gal[2];
  for (int pi = 0; pi < 2; pi++) {
    gal[pi].assign(N * lanes, 0);
    for (size_t i = 0; i < N; i++) {
      size_t out_i = gal2idx(N, inv_g * idx2gal(N, (int64_t)i) % m);
      for (int k = 0; k < lanes; k++) gal[pi][out_i * lanes + k] = cur[pi][i * lanes + k];
    }
    R.inv_weighted_ntt(pi, gal[pi].data(), lanes);
  }
  const uint64_t q2inv1 = invmod(Q2 % Q1, Q1), q1inv2 = invmod(Q1 % Q2, Q2);
  for (int d = 0; d < 2; d++)
    for (int pi = 0; pi < 2; pi++) dig[d][pi].assign(N * lanes, 0);
  for (size_t i = 0; i < N * (size_t)lanes; i++) {
    int64_t x1 = (int64_t)R.md[0].mul(gal[0][i], q2inv1);
    int64_t x2 = (int64_t)R.md[1].mul(gal[1][i], q1inv2);
    int64_t v = x1 * Q2 + x2 * Q1;  // :548-551
    if (v > QQ) v -= QQ;             // :552-553
    if (v > QQ / 2) v -= QQ;         // :554-555
    int64_t cur_v = v;
    for (int d = 0; d < 2; d++) {  // :557-570
      int64_t high = (cur_v + ((int64_t)1 << (LOG2_B - 1))) >> LOG2_B;  // arithmetic shift
      int64_t low = cur_v - high * ((int64_t)1 << LOG2_B);
      dig[d][0][i] = (uint64_t)mod_floor(low, Q1);
      dig[d][1][i] = (uint64_t)mod_floor(low, Q2);
      cur_v = high;
    }
  }
  for (int d = 0; d < 2; d++)
    for (int pi = 0; pi < 2; pi++) R.weighted_ntt(pi, dig[d][pi].data(), lanes);
  for (int pi = 0; pi < 2; pi++) {
    reply_a[pi].assign(N * lanes, 0);
    const Mod& md = R.md[pi];
    for (size_t i = 0; i < N; i++)
      for (int k = 0; k < lanes; k++) {
        size_t ix = i * lanes + k;
        reply_a[pi][ix] = md.add(md.mul(dig[0][pi][ix], gka[0][pi][ix]), md.mul(dig[1][pi][ix], gka[1][pi][ix]));
      }
  }
}

// preprocess + preprocess_loop (base_pir.rs:782-863).  The chain is strictly
// sequential in i; the 8 lanes are independent and are run in parallel here.
static void preprocess(Shard& db) {
  const Ring& R = *db.R;
  const size_t N = R.n, L = db.ig.loop_len();
  std::vector<uint64_t> gka[2][2];
  for (int d = 0; d < 2; d++) to_simd_element_same(R, gk_a(N, d), gka[d]);
  std::vector<uint64_t> qa[2][2];
  for (int c = 0; c < (db.ig.conj() ? 2 : 1); c++) to_simd_element_same(R, qry_a(N, db.used_seeds, c), qa[c]);
  for (int c = 0; c < 2; c++)
    for (int d = 0; d < 2; d++)
      for (int pi = 0; pi < 2; pi++) db.gk[c][d][pi].assign(db.ig.conj() || c == 0 ? L * N * SIMD : 0, 0);
  std::vector<uint64_t> sums[2][SIMD][2];
  const int halves = db.ig.conj() ? 2 : 1;
  parallel_for((size_t)halves * SIMD, [&](size_t ck) {
    {
      const int c = (int)(ck / SIMD), k = (int)(ck % SIMD);
      // single-lane chain for lane k of half c
      std::vector<uint64_t> sum[2], ra[2], dg[2][2], gka_k[2][2], qa_k[2];
      for (int pi = 0; pi < 2; pi++) {
        sum[pi].assign(N, 0);
        qa_k[pi].resize(N);
        for (size_t j = 0; j < N; j++) qa_k[pi][j] = qa[c][pi][j * SIMD + k];
        for (int d = 0; d < 2; d++) {
          gka_k[d][pi].resize(N);
          for (size_t j = 0; j < N; j++) gka_k[d][pi][j] = gka[d][pi][j * SIMD + k];
        }
      }
      for (size_t i = 0; i < L; i++) {
        partial_gal(R, sum, gka_k, ra, dg, 1);
        for (int d = 0; d < 2; d++)
          for (int pi = 0; pi < 2; pi++)
            for (size_t j = 0; j < N; j++) db.gk[c][d][pi][(i * N + j) * SIMD + k] = dg[d][pi][j];
        for (int pi = 0; pi < 2; pi++) {
          const Mod& md = R.md[pi];
          for (size_t j = 0; j < N; j++)
            sum[pi][j] = md.add(ra[pi][j], md.mul(qa_k[pi][j], db.te[c][pi][(i * N + j) * SIMD + k]));
        }
      }
      for (int pi = 0; pi < 2; pi++) sums[c][k][pi] = sum[pi];
    }
  });
  for (int pi = 0; pi < 2; pi++) {
    db.reply_a[pi].assign(N * SIMD, 0);
    for (size_t j = 0; j < N; j++)
      for (int k = 0; k < SIMD; k++) {
        uint64_t v = sums[0][k][pi][j];
        if (halves == 2) v = R.md[pi].add(v, sums[1][k][pi][j]);
        db.reply_a[pi][j * SIMD + k] = v;
      }
  }
  db.has_reply_a = true;
}

// from_simd_element (base_pir.rs:905-935): per prime iNTT, then CRT to Z_q
static void from_simd_element(const Ring& R, std::vector<uint64_t> el[2], Poly out[SIMD]) {
  const size_t N = R.n;
  for (int pi = 0; pi < 2; pi++) R.inv_weighted_ntt(pi, el[pi].data(), SIMD);
  const uint64_t q2inv1 = invmod(Q2 % Q1, Q1), q1inv2 = invmod(Q1 % Q2, Q2);
  for (int k = 0; k < SIMD; k++) out[k].assign(N, 0);
  for (size_t i = 0; i < N; i++)
    for (int k = 0; k < SIMD; k++) {
      int64_t x1 = smallest_lift((int64_t)R.md[0].mul(el[0][i * SIMD + k], q2inv1), Q1);
      int64_t x2 = smallest_lift((int64_t)R.md[1].mul(el[1][i * SIMD + k], q1inv2), Q2);
      i128 v = (i128)Q2 * x1 + (i128)Q1 * x2;
      out[k][i] = i128_mod(v, QQ);
    }
}

static void get_a(const Shard& db, Poly out[SIMD]) {
  ORC_CHECK(db.has_reply_a, "database not preprocessed");
  std::vector<uint64_t> el[2] = {db.reply_a[0], db.reply_a[1]};
  from_simd_element(*db.R, el, out);
}

struct QueryRef {
  const Poly* qry_b;
  const Poly* qry_conj_b;  // may be null
  const Poly* gk_b[2];
};

// main_pir_loop (base_pir.rs:1085-1247), faithful to its sum/sum_new swapping,
// the galois scatter and the reduction every `reduce_every` iterations.
static void main_pir_loop(size_t N, size_t len, size_t reduce_every, const Mod& md, std::vector<uint64_t>& sum,
                          const std::vector<size_t>& gal, const uint64_t* qry_b, const uint64_t* gk0,
                          const uint64_t* gk1, const uint64_t* ipg0, const uint64_t* ipg1, const uint64_t* te) {
  std::vector<uint64_t> sum_new(N * SIMD, 0);
  size_t index = 0;
  for (size_t io = 0; io < len; io += reduce_every) {
    size_t cnt = std::min(len - io, reduce_every);
    for (size_t ii = 0; ii < cnt; ii++) {
      for (size_t j = 0; j < N; j++) {
        uint64_t* dst = &sum_new[gal[j] * SIMD];
        const uint64_t* src = &sum[j * SIMD];
        const size_t e = (index + j) * SIMD;
        for (int k = 0; k < SIMD; k++)
          dst[k] = src[k] + ipg0[e + k] * gk0[j * SIMD + k] + ipg1[e + k] * gk1[j * SIMD + k] +
                   te[e + k] * qry_b[j * SIMD + k];
      }
      index += N;
      std::swap(sum, sum_new);
    }
    for (size_t j = 0; j < N * SIMD; j++) sum[j] = md.red(sum[j]);
  }
}

// perform_pir_split (base_pir.rs:958-1077)
static void perform_pir_split(const Shard& db, const QueryRef q[SIMD], Poly out[SIMD]) {
  const Ring& R = *db.R;
  const size_t N = R.n, L = db.ig.loop_len();
  const int64_t m = 2 * (int64_t)N;
  std::vector<uint64_t> qb[2], qcb[2], gkb[2][2];
  {
    const Poly* els[SIMD];
    for (int k = 0; k < SIMD; k++) els[k] = q[k].qry_b;
    to_simd_element(R, els, qb);
    if (db.ig.conj()) {
      for (int k = 0; k < SIMD; k++) {
        ORC_CHECK(q[k].qry_conj_b, "conjugate query must be given when index subgroup requires conjugation");
        els[k] = q[k].qry_conj_b;
      }
      to_simd_element(R, els, qcb);
    }
    for (int d = 0; d < 2; d++) {
      for (int k = 0; k < SIMD; k++) els[k] = q[k].gk_b[d];
      to_simd_element(R, els, gkb[d]);
    }
  }
  int64_t inv_g = (int64_t)invmod(5, (uint64_t)m);
  std::vector<size_t> gal(N);
  for (size_t i = 0; i < N; i++) gal[i] = (size_t)((mod_floor(inv_g * (2 * (int64_t)i + 1), m) - 1) / 2);
  std::vector<uint64_t> sum[2], sum_conj[2];
  for (int pi = 0; pi < 2; pi++) {
    // reduce_every_iterations (:1002-1005): min over both factors with repr_bound = 2p
    u128 rb0 = 2 * (u128)R.p[0], rb1 = 2 * (u128)R.p[1];
    size_t reduce_every = (size_t)std::min((u128)UINT64_MAX / rb0 / rb0 / (GK_DIGITS + 1),
                                           (u128)UINT64_MAX / rb1 / rb1 / (GK_DIGITS + 1));
    sum[pi].assign(N * SIMD, 0);
    main_pir_loop(N, L, reduce_every, R.md[pi], sum[pi], gal, qb[pi].data(), gkb[0][pi].data(), gkb[1][pi].data(),
                  db.gk[0][0][pi].data(), db.gk[0][1][pi].data(), db.te[0][pi].data());
    if (db.ig.conj()) {
      sum_conj[pi].assign(N * SIMD, 0);
      main_pir_loop(N, L, reduce_every, R.md[pi], sum_conj[pi], gal, qcb[pi].data(), gkb[0][pi].data(),
                    gkb[1][pi].data(), db.gk[1][0][pi].data(), db.gk[1][1][pi].data(), db.te[1][pi].data());
      for (size_t j = 0; j < N * SIMD; j++) sum[pi][j] += sum_conj[pi][j];
    }
    // permute(sum, |i| gal[i]): new[i] = sum[gal[i]]; then reduce_from_u64
    std::vector<uint64_t> pm(N * SIMD);
    for (size_t i = 0; i < N; i++)
      for (int k = 0; k < SIMD; k++) pm[i * SIMD + k] = R.md[pi].red(sum[pi][gal[i] * SIMD + k]);
    sum[pi].swap(pm);
  }
  from_simd_element(R, sum, out);
}

// ------------------------------------------------------------ double PIR
// encode_ciphertext_plaintext (double_pir.rs:70-81)
static void encode_ct_pt(uint64_t a, uint64_t b, int64_t out[CTXT_PARTS]) {
  uint64_t v = a * ((uint64_t)1 << PRIM_B_BITS) + b;
  for (int j = 0; j < CTXT_PARTS; j++) {
    out[j] = (int64_t)(v % TPLAIN);
    v /= TPLAIN;
  }
  ORC_CHECK(v == 0, "encode_ciphertext_plaintext overflow");
}
// decode_ciphertext_plaintext (double_pir.rs:83-93)
static void decode_ct_pt(const int64_t d[CTXT_PARTS], uint64_t* a, uint64_t* b) {
  uint64_t v = 0;
  for (int j = CTXT_PARTS - 1; j >= 0; j--) v = v * TPLAIN + (uint64_t)d[j];
  ORC_CHECK(v / ((uint64_t)1 << PRIM_B_BITS) < ((uint64_t)1 << PRIM_A_BITS), "decode_ciphertext_plaintext range");
  *b = v % ((uint64_t)1 << PRIM_B_BITS);
  *a = v / ((uint64_t)1 << PRIM_B_BITS);
}

struct DoubleQuery {
  const Poly* pq;
  const Poly* pqc;  // may be null
  const Poly* sq;
  const Poly* sqc;  // may be null
  const Poly* gk[2];
};

// perform_batched_double_pir (double_pir.rs:126-228).  dbs[b] is the fleet
// for batch slot b (ndb[b] shards); queries[b] may be null.
static void perform_batched_double_pir(const Shard* const* dbs[BATCH], const size_t ndb[BATCH],
                                       const DoubleQuery* queries[BATCH], const IndexGroup& ig2,
                                       std::vector<std::array<Poly, 2>> results[BATCH],
                                       double* primary_us = nullptr, double* secondary_us = nullptr) {
  const std::shared_ptr<Ring> R = dbs[0][0]->R;
  const size_t N = R->n;
  for (int b = 0; b < BATCH; b++) ORC_CHECK(ndb[b] * SIMD <= ig2.l, "too many databases for the secondary group");
  std::vector<std::vector<std::array<Poly, CTXT_PARTS>>> part(BATCH);  // [slot][shard*8+k][part]
  for (int b = 0; b < BATCH; b++) {
    if (!queries[b]) continue;
    part[b].resize(ndb[b] * SIMD);
    for (size_t i = 0; i < ndb[b]; i++)  // :160
      ORC_CHECK(dbs[b][i]->ig.conj() == (queries[b]->pqc != nullptr), "conjugate presence mismatch");
    parallel_for(ndb[b], [&](size_t i) {
      const Shard& db = *dbs[b][i];
      Poly a[SIMD], bb[SIMD];
      get_a(db, a);
      QueryRef qr[SIMD];
      for (int k = 0; k < SIMD; k++) qr[k] = QueryRef{queries[b]->pq, queries[b]->pqc, {queries[b]->gk[0], queries[b]->gk[1]}};
      perform_pir_split(db, qr, bb);
      for (int k = 0; k < SIMD; k++) {
        std::array<Poly, CTXT_PARTS>& pr = part[b][i * SIMD + k];
        for (int j = 0; j < CTXT_PARTS; j++) pr[j].assign(N, 0);
        for (size_t n = 0; n < N; n++) {
          int64_t d[CTXT_PARTS];
          encode_ct_pt(ms_encode(a[k][n], PRIM_A_BITS), ms_encode(bb[k][n], PRIM_B_BITS), d);
          for (int j = 0; j < CTXT_PARTS; j++) pr[j][n] = d[j];
        }
      }
    });
  }
  (void)primary_us;
  (void)secondary_us;
  // secondary database (:195-218)
  Shard sdb;
  sdb.R = R;
  sdb.ig = ig2;
  sdb.used_seeds = 1;
  std::vector<uint16_t> entries(ig2.l * SIMD * N, 0);
  for (size_t i = 0; i < ig2.l; i++)
    for (int j = 0; j < SIMD; j++) {
      if (j < CTXT_PARTS * BATCH && i < SIMD * ndb[j / CTXT_PARTS] && queries[j / CTXT_PARTS]) {
        const Poly& src = part[j / CTXT_PARTS][i][j % CTXT_PARTS];
        for (size_t n = 0; n < N; n++) entries[(i * SIMD + j) * N + n] = (uint16_t)src[n];
      }
    }
  set_transformed_entries(sdb, entries.data());
  preprocess(sdb);
  Poly a[SIMD], bb[SIMD];
  get_a(sdb, a);
  Poly zero(N, 0);
  QueryRef qr[SIMD];
  for (int k = 0; k < SIMD; k++) {
    const DoubleQuery* dq = (k / CTXT_PARTS < BATCH) ? queries[k / CTXT_PARTS] : nullptr;
    if (dq) qr[k] = QueryRef{dq->sq, dq->sqc, {dq->gk[0], dq->gk[1]}};
    else qr[k] = QueryRef{&zero, &zero, {&zero, &zero}};
  }
  perform_pir_split(sdb, qr, bb);
  for (int b = 0; b < BATCH; b++) {
    results[b].clear();
    if (!queries[b]) continue;
    for (int j = 0; j < CTXT_PARTS; j++) results[b].push_back({a[b * CTXT_PARTS + j], bb[b * CTXT_PARTS + j]});
  }
}

// enc_double_pir (double_pir.rs:245-289)
struct EncQuery {
  Poly pq, pqc, sq, sqc;
  bool has_pqc = false, has_sqc = false;
  Poly gk[2];
};
static Poly monomial(size_t N, int64_t t, int64_t e) {  // X^e in Z_t[X]/(X^N+1)
  Poly m(N, 0);
  int64_t ee = mod_floor(e, 2 * (int64_t)N);
  if (ee < (int64_t)N) m[ee] = 1;
  else m[ee - N] = t - 1;
  return m;
}
static EncQuery enc_double_pir(StdRng& rng, const IndexGroup& ig1, const IndexGroup& ig2,
                               const std::vector<int8_t>& sk, size_t primary_idx, size_t secondary_idx, double sigma) {
  const size_t N = ig1.N;
  ORC_CHECK(primary_idx < ig1.l * SIMD, "primary index out of range");
  ORC_CHECK(secondary_idx < ig2.l / SIMD, "secondary index out of range");
  size_t i = primary_idx / SIMD;
  size_t j = secondary_idx * SIMD + primary_idx % SIMD;
  EncQuery q;
  std::vector<Poly> gk = gen_gk_b(N, rng, sk, 5, GK_DIGITS, LOG2_B, sigma);
  q.gk[0] = gk[0];
  q.gk[1] = gk[1];
  q.pq = enc_sym_b(N, TPLAIN, qry_a(N, 0, 0), rng, sk, monomial(N, TPLAIN, (int64_t)(i * ig1.qbp())), sigma);
  if (ig1.conj()) {
    q.has_pqc = true;
    q.pqc = enc_sym_b(N, TPLAIN, qry_a(N, 0, 1), rng, sk, monomial(N, TPLAIN, 2 * (int64_t)N - (int64_t)(i * ig1.qbp())), sigma);
  }
  q.sq = enc_sym_b(N, TPLAIN, qry_a(N, 1, 0), rng, sk, monomial(N, TPLAIN, (int64_t)(j * ig2.qbp())), sigma);
  if (ig2.conj()) {
    q.has_sqc = true;
    q.sqc = enc_sym_b(N, TPLAIN, qry_a(N, 1, 1), rng, sk, monomial(N, TPLAIN, 2 * (int64_t)N - (int64_t)(j * ig2.qbp())), sigma);
  }
  return q;
}

// dec_double_pir (double_pir.rs:292-317)
static Poly dec_double_pir(size_t N, const std::vector<int8_t>& sk, const Poly ra[CTXT_PARTS], const Poly rb[CTXT_PARTS]) {
  Poly parts[CTXT_PARTS];
  for (int j = 0; j < CTXT_PARTS; j++) parts[j] = dec(N, TPLAIN, sk, ra[j], rb[j]);
  Poly a(N), b(N);
  for (size_t n = 0; n < N; n++) {
    int64_t d[CTXT_PARTS];
    for (int j = 0; j < CTXT_PARTS; j++) d[j] = parts[j][n];
    uint64_t aa, bb;
    decode_ct_pt(d, &aa, &bb);
    a[n] = ms_decode(aa, PRIM_A_BITS);
    b[n] = ms_decode(bb, PRIM_B_BITS);
  }
  return dec(N, TPLAIN, sk, a, b);
}

// ------------------------------------------------------------ wire (pir_wrapper.rs)
// condense (pir_wrapper.rs:84-113)
static void condense(int bits, const uint64_t* data, size_t n, std::vector<uint8_t>& out) {
  ORC_CHECK(n % 8 == 0, "condense expects a multiple of 8 values");
  for (int i = 0; i < bits / 8; i++)
    for (size_t t = 0; t < n; t++) out.push_back((uint8_t)(data[t] >> (8 * i)));
  if (bits % 8 >= 4) {
    int sh = (bits / 8) * 8;
    for (size_t t = 0; t < n; t += 2)
      out.push_back((uint8_t)((((data[t] >> sh) & 0xF) << 4) | ((data[t + 1] >> sh) & 0xF)));
  }
  if (bits % 4 >= 2) {
    int sh = (bits / 4) * 4;
    for (size_t t = 0; t < n; t += 4) {
      uint8_t v = 0;
      for (int u = 0; u < 4; u++) v |= (uint8_t)(((data[t + u] >> sh) & 3) << (6 - 2 * u));
      out.push_back(v);
    }
  }
  if (bits % 2 >= 1) {
    int sh = (bits / 2) * 2;
    for (size_t t = 0; t < n; t += 8) {
      uint8_t v = 0;
      for (int u = 0; u < 8; u++) v |= (uint8_t)(((data[t + u] >> sh) & 1) << (7 - u));
      out.push_back(v);
    }
  }
}
// uncondense (pir_wrapper.rs:120-158); returns bytes consumed, throws "not enough data"
static size_t uncondense(int bits, size_t n, const uint8_t* data, size_t len, uint64_t* out) {
  size_t pos = 0;
  auto next = [&]() -> uint8_t {
    if (pos >= len) throw Error("not enough data");
    return data[pos++];
  };
  for (size_t t = 0; t < n; t++) out[t] = 0;
  for (int i = 0; i < bits / 8; i++)
    for (size_t t = 0; t < n; t++) out[t] |= (uint64_t)next() << (8 * i);
  if (bits % 8 >= 4) {
    int sh = (bits / 8) * 8;
    for (size_t t = 0; t + 2 <= n; t += 2) {
      uint8_t s = next();
      out[t] |= (uint64_t)(s >> 4) << sh;
      out[t + 1] |= (uint64_t)(s & 0xF) << sh;
    }
  }
  if (bits % 4 >= 2) {
    int sh = (bits / 4) * 4;
    for (size_t t = 0; t + 4 <= n; t += 4) {
      uint8_t s = next();
      for (int u = 0; u < 4; u++) out[t + u] |= (uint64_t)((s >> (6 - 2 * u)) & 3) << sh;
    }
  }
  if (bits % 2 >= 1) {
    int sh = (bits / 2) * 2;
    for (size_t t = 0; t + 8 <= n; t += 8) {
      uint8_t s = next();
      for (int u = 0; u < 8; u++) out[t + u] |= (uint64_t)((s >> (7 - u)) & 1) << sh;
    }
  }
  return pos;
}

// choose_index_group_secondary (pir_wrapper.rs:166-175)
static IndexGroup choose_secondary(size_t num_shards) {
  const size_t N = (size_t)1 << LOG2_N_WIRE;
  ORC_CHECK(num_shards <= N / SIMD, "too many shards");
  size_t log2l = 0;
  while (((size_t)1 << log2l) < num_shards) log2l++;
  if (((size_t)SIMD << log2l) == N) return IndexGroup{N, N};
  return make_group(N, (size_t)SIMD << log2l);
}
// get_database_shape (pir_wrapper.rs:219-231)
static void get_database_shape(size_t num_entries, IndexGroup* ig1, IndexGroup* ig2) {
  const size_t N = (size_t)1 << LOG2_N_WIRE;
  ORC_CHECK(num_entries >= 1 && num_entries <= N * N, "num_entries out of range");
  const size_t half_max = N * N / 16;  // HALF_SIZE_PRIMARY_MAX_ENTRIES (:188)
  *ig1 = num_entries <= half_max ? make_group(N, N / 2) : IndexGroup{N, N};
  size_t shards = (num_entries + SIMD * ig1->l - 1) / (SIMD * ig1->l);
  *ig2 = choose_secondary(shards);
}

}  // namespace orc

// ====================================================================== C ABI
using namespace orc;

// ===================================================== vectorised restatement
// The same set_transformed_entries, preprocess (partial_gal chain) and
// perform_pir_split as above, on the reference's vector shape: the 8 SIMD
// lanes of a slot in one AVX-512 register of 8 x u64 (simd_zn.rs
// SpecialZnx8, avx.rs), products by _mm512_mul_epu32 and the reduction for
// p = 2^K - alpha of simd_zn.rs:197-230 (two shift-multiply-subtract steps,
// then one conditional subtraction, so every value is canonical as in the
// scalar code), the chain of each half run for all 8 lanes at once and the
// halves in parallel (the reference's parallelism).  Used to time the
// secondary phase of the CPU arm; tests check it equals the scalar code
// array for array.  Compiled for AVX-512 in these functions only; callers
// check orc_cpu_has_avx512 first.
#define ORC_AVX512 __attribute__((target("avx512f,avx512dq")))

namespace vec {

// 64-byte aligned array of n vectors (std::vector drops __m512i's alignment)
struct VBuf {
  __m512i* p;
  explicit VBuf(size_t n) : p(static_cast<__m512i*>(aligned_alloc(64, (n ? n : 1) * sizeof(__m512i)))) {
    if (!p) throw std::runtime_error("out of host memory");
  }
  ~VBuf() { free(p); }
  VBuf(const VBuf&) = delete;
  VBuf& operator=(const VBuf&) = delete;
  __m512i& operator[](size_t i) { return p[i]; }
  __m512i* data() { return p; }
};

template <int PI>
struct Pr {
  static constexpr uint64_t P = PI ? Q2 : Q1;
  static constexpr int K = PI ? 25 : 26;
};

// a * b mod p for a, b < p (canonical out)
template <int PI>
ORC_AVX512 static inline __m512i mulmod(__m512i a, __m512i b) {
  const __m512i p = _mm512_set1_epi64((long long)Pr<PI>::P);
  __m512i x = _mm512_mul_epu32(a, b);
  x = _mm512_sub_epi64(x, _mm512_mul_epu32(_mm512_srli_epi64(x, Pr<PI>::K), p));
  x = _mm512_sub_epi64(x, _mm512_mul_epu32(_mm512_srli_epi64(x, Pr<PI>::K), p));
  return _mm512_min_epu64(x, _mm512_sub_epi64(x, p));
}
template <int PI>
ORC_AVX512 static inline __m512i addmod(__m512i a, __m512i b) {
  const __m512i p = _mm512_set1_epi64((long long)Pr<PI>::P);
  const __m512i s = _mm512_add_epi64(a, b);
  return _mm512_min_epu64(s, _mm512_sub_epi64(s, p));
}
template <int PI>
ORC_AVX512 static inline __m512i submod(__m512i a, __m512i b) {
  const __m512i p = _mm512_set1_epi64((long long)Pr<PI>::P);
  const __m512i d = _mm512_sub_epi64(_mm512_add_epi64(a, p), b);
  return _mm512_min_epu64(d, _mm512_sub_epi64(d, p));
}

// Dft::apply on n vectors (the same radix-2 DIT with bit reversal)
template <int PI>
ORC_AVX512 static void dft8(const Dft& d, __m512i* x) {
  const size_t n = d.n;
  for (size_t i = 0; i < n; i++) {
    const size_t r = d.rev[i];
    if (r > i) std::swap(x[i], x[r]);
  }
  for (size_t h = 1; h < n; h <<= 1)
    for (size_t j = 0; j < h; j++) {
      const __m512i w = _mm512_set1_epi64((long long)d.tw[h + j]);
      for (size_t i = 0; i < n; i += 2 * h) {
        const __m512i u = x[i + j], v = mulmod<PI>(x[i + j + h], w);
        x[i + j] = addmod<PI>(u, v);
        x[i + j + h] = submod<PI>(u, v);
      }
    }
}
template <int PI>
ORC_AVX512 static void weighted_ntt8(const Ring& R, __m512i* x) {
  for (size_t i = 0; i < R.n; i++) x[i] = mulmod<PI>(x[i], _mm512_set1_epi64((long long)R.zneg[PI][i]));
  dft8<PI>(R.fwd[PI], x);
}
template <int PI>
ORC_AVX512 static void inv_weighted_ntt8(const Ring& R, __m512i* x) {
  dft8<PI>(R.inv[PI], x);
  for (size_t i = 0; i < R.n; i++) {
    const uint64_t s = R.md[PI].mul(R.ninv[PI], R.zpos[PI][i]);
    x[i] = mulmod<PI>(x[i], _mm512_set1_epi64((long long)s));
  }
}

ORC_AVX512 static inline __m512i ld(const uint64_t* p) { return _mm512_loadu_si512((const void*)p); }
ORC_AVX512 static inline void st(uint64_t* p, __m512i v) { _mm512_storeu_si512((void*)p, v); }

// STEP 2 of set_transformed_entries for column j
ORC_AVX512 static void col_ntt(const Ring& R, uint64_t* M, size_t l, size_t j) {
  const size_t N = R.n;
  VBuf c(N);
  for (size_t i = 0; i < N; i++) c[i] = ld(&M[(i * l + j) * SIMD]);
  weighted_ntt8<0>(R, c.data());
  for (size_t i = 0; i < N; i++) st(&M[(i * l + j) * SIMD], c[i]);
}
// coset_ntt of row i (the scalar function's steps on vectors)
ORC_AVX512 static void row_coset_ntt(const Ring& R, const IndexGroup& ig, int64_t zeta_power, uint64_t* values,
                                     const Dft& fft_l) {
  const size_t N = ig.N, l = ig.l;
  const int64_t m = 2 * (int64_t)N;
  const Mod& md = R.md[0];
  const int64_t zp = mod_floor(zeta_power, m);
  const int64_t coset = zp % (m / (int64_t)l);
  const uint64_t z = powmod(R.zeta[0], (uint64_t)coset, R.p[0]);
  const uint64_t zinv = invmod(z, R.p[0]);
  VBuf v(l), old(l);
  uint64_t cur = 1;
  for (size_t i = 0; i < l; i++) {
    v[i] = mulmod<0>(ld(&values[i * SIMD]), _mm512_set1_epi64((long long)cur));
    cur = md.mul(cur, zinv);
  }
  dft8<0>(fft_l, v.data());
  auto g2i = [&](int64_t x) -> size_t { return (size_t)((mod_floor(-x, m) - coset) / (m / (int64_t)l)); };
  const int64_t zpn = mod_floor(-zp, m);
  memcpy(old.data(), v.data(), l * sizeof(__m512i));
  int64_t gpow = 1;
  for (size_t i = 0; i < l; i++) {
    size_t src;
    if (ig.conj()) {
      if (i == N / 2) gpow = 1;
      src = i < N / 2 ? g2i(zpn * gpow % m) : g2i(zp * gpow % m);
    } else {
      src = g2i(zpn * gpow % m);
    }
    gpow = gpow * 5 % m;
    st(&values[i * SIMD], old[src]);
  }
}
// STEP 6 for column col: iNTT, lift, * l^-1 mod t, centred lift, NTT in q1 and q2
ORC_AVX512 static void col_lift(const Ring& R, Shard& db, const uint64_t* M, size_t l, size_t col, int64_t scale) {
  const size_t N = R.n, L = db.ig.loop_len();
  VBuf c(N), r0(N), r1(N);
  for (size_t i = 0; i < N; i++) c[i] = ld(&M[(i * l + col) * SIMD]);
  inv_weighted_ntt8<0>(R, c.data());
  alignas(64) uint64_t cv[SIMD], a0[SIMD], a1[SIMD];
  for (size_t i = 0; i < N; i++) {
    _mm512_store_si512((void*)cv, c[i]);
    for (int k = 0; k < SIMD; k++) {
      const int64_t vv = smallest_lift((int64_t)cv[k], Q1);
      const int64_t w = smallest_lift(mod_floor(mod_floor(vv, TPLAIN) * scale, TPLAIN), TPLAIN);
      a0[k] = (uint64_t)mod_floor(w, Q1);
      a1[k] = (uint64_t)mod_floor(w, Q2);
    }
    r0[i] = _mm512_load_si512((const void*)a0);
    r1[i] = _mm512_load_si512((const void*)a1);
  }
  weighted_ntt8<0>(R, r0.data());
  weighted_ntt8<1>(R, r1.data());
  const int half = col < L ? 0 : 1;
  const size_t row = col < L ? col : col - L;
  for (size_t i = 0; i < N; i++) {
    st(&db.te[half][0][(row * N + i) * SIMD], r0[i]);
    st(&db.te[half][1][(row * N + i) * SIMD], r1[i]);
  }
}

}  // namespace vec

// set_transformed_entries on vectors: STEP 1, 4 and 5 move data as the scalar
// code does; STEP 2, 3 and 6 are the vector transforms above
static void set_transformed_entries_vec(Shard& db, const uint16_t* entries) {
  const Ring& R = *db.R;
  const size_t N = R.n, l = db.ig.l, L = db.ig.loop_len();
  const int64_t m = 2 * (int64_t)N;
  ORC_CHECK(2 * TPLAIN * (int64_t)N < Q1, "max_coeff >= q1");
  std::vector<uint64_t> M(N * l * SIMD);
  parallel_for(l, [&](size_t j) {
    for (int k = 0; k < SIMD; k++) {
      const uint16_t* e = entries + ((size_t)j * SIMD + k) * N;
      for (size_t i = 0; i < N; i++) M[(i * l + j) * SIMD + k] = e[i];
    }
  });
  parallel_for(l, [&](size_t j) { vec::col_ntt(R, M.data(), l, j); });
  {
    size_t logl = 0;
    while (((size_t)1 << logl) < l) logl++;
    uint64_t omega = powmod(R.zeta[0], (uint64_t)(m / (int64_t)l), R.p[0]);
    Dft fft_l(R.p[0], l, invmod(omega, R.p[0]));
    int64_t base_power = mod_floor(-(int64_t)db.ig.qbp(), m);
    parallel_for(N, [&](size_t i) {
      vec::row_coset_ntt(R, db.ig, mod_floor(idx2gal(N, (int64_t)i) * base_power, m), &M[i * l * SIMD], fft_l);
    });
  }
  {
    int64_t g_inv = (int64_t)invmod(5, (uint64_t)m);
    parallel_for(l, [&](size_t j) {
      int64_t aut = (int64_t)powmod((uint64_t)g_inv, j, (uint64_t)m);
      std::vector<uint64_t> c(N * SIMD);
      for (size_t i = 0; i < N; i++) {
        size_t src = gal2idx(N, aut * idx2gal(N, (int64_t)i) % m);
        memcpy(&c[i * SIMD], &M[(src * l + j) * SIMD], SIMD * 8);
      }
      for (size_t i = 0; i < N; i++) memcpy(&M[(i * l + j) * SIMD], &c[i * SIMD], SIMD * 8);
    });
  }
  parallel_for(N, [&](size_t i) {
    uint64_t* row = &M[i * l * SIMD];
    auto rev = [&](size_t a, size_t b) {
      while (b > a + 1) {
        b--;
        for (int k = 0; k < SIMD; k++) std::swap(row[a * SIMD + k], row[b * SIMD + k]);
        a++;
      }
    };
    if (db.ig.conj()) {
      rev(0, N / 2);
      rev(N / 2, N);
    } else {
      rev(0, l);
    }
  });
  for (int c = 0; c < 2; c++)
    for (int pi = 0; pi < 2; pi++) db.te[c][pi].assign(db.ig.conj() || c == 0 ? L * N * SIMD : 0, 0);
  const int64_t scale = (int64_t)invmod((uint64_t)(l % TPLAIN), (uint64_t)TPLAIN);
  parallel_for(l, [&](size_t col) { vec::col_lift(R, db, M.data(), l, col, scale); });
  db.has_reply_a = false;
}

namespace vec {

// Spin barrier for the few threads that share one half's chain step.
struct TeamBarrier {
  std::atomic<int> count{0};
  std::atomic<int> gen{0};
  int n;
  explicit TeamBarrier(int n_) : n(n_) {}
  void wait() {
    const int g = gen.load(std::memory_order_acquire);
    if (count.fetch_add(1, std::memory_order_acq_rel) == n - 1) {
      count.store(0, std::memory_order_relaxed);
      gen.store(g + 1, std::memory_order_release);
    } else {
      while (gen.load(std::memory_order_acquire) == g) _mm_pause();
    }
  }
};

// One step of the chain of half c, thread t of 4, as the reference splits it
// (base_pir.rs:496-594): the two factors' inverse transforms side by side
// (join), the decomposition split over positions (par_iter), the four digit
// transforms side by side (par_iter over digits x join over factors), then the
// pointwise reply_a and the next sum, split over positions.
struct ChainTeam {
  Shard* db;
  int c;
  size_t N;
  std::vector<size_t> gmap;
  VBuf buf;
  __m512i *sum[2], *ra[2], *dig[2][2], *gal[2], *gk[2][2], *qa[2];
  TeamBarrier bar{4};
  ChainTeam(Shard* db_, int c_, size_t N_) : db(db_), c(c_), N(N_), gmap(N_), buf(16 * N_) {
    for (int pi = 0; pi < 2; pi++) {
      sum[pi] = &buf[(0 + pi) * N];
      ra[pi] = &buf[(2 + pi) * N];
      dig[0][pi] = &buf[(4 + pi) * N];
      dig[1][pi] = &buf[(6 + pi) * N];
      gal[pi] = &buf[(8 + pi) * N];
      gk[0][pi] = &buf[(10 + pi) * N];
      gk[1][pi] = &buf[(12 + pi) * N];
      qa[pi] = &buf[(14 + pi) * N];
    }
  }
};

ORC_AVX512 static void chain_thread(ChainTeam& T, int t) {
  Shard& db = *T.db;
  const Ring& R = *db.R;
  const size_t N = T.N, L = db.ig.loop_len();
  const size_t j0 = N * t / 4, j1 = N * (t + 1) / 4;
  const __m512i q2inv1 = _mm512_set1_epi64((long long)invmod(Q2 % Q1, Q1));
  const __m512i q1inv2 = _mm512_set1_epi64((long long)invmod(Q1 % Q2, Q2));
  const __m512i vq1 = _mm512_set1_epi64(Q1), vq2 = _mm512_set1_epi64(Q2), vqq = _mm512_set1_epi64(QQ);
  const __m512i vqq2 = _mm512_set1_epi64(QQ / 2), half = _mm512_set1_epi64((long long)1 << (LOG2_B - 1));
  const __m512i zero = _mm512_setzero_si512();
  for (size_t i = 0; i < L; i++) {
    // gal(sum) and its inverse transform, one factor per thread (base_pir.rs:509-519)
    if (t < 2) {
      for (size_t j = 0; j < N; j++) T.gal[t][T.gmap[j]] = T.sum[t][j];
      if (t == 0)
        inv_weighted_ntt8<0>(R, T.gal[0]);
      else
        inv_weighted_ntt8<1>(R, T.gal[1]);
    }
    T.bar.wait();
    // centred CRT lift and the two digits (base_pir.rs:541-571)
    for (size_t j = j0; j < j1; j++) {
      const __m512i x1 = mulmod<0>(T.gal[0][j], q2inv1);
      const __m512i x2 = mulmod<1>(T.gal[1][j], q1inv2);
      __m512i v = _mm512_add_epi64(_mm512_mul_epu32(x1, vq2), _mm512_mul_epu32(x2, vq1));
      v = _mm512_mask_sub_epi64(v, _mm512_cmpgt_epi64_mask(v, vqq), v, vqq);
      v = _mm512_mask_sub_epi64(v, _mm512_cmpgt_epi64_mask(v, vqq2), v, vqq);
      __m512i cur_v = v;
      for (int d = 0; d < 2; d++) {
        const __m512i high = _mm512_srai_epi64(_mm512_add_epi64(cur_v, half), LOG2_B);
        const __m512i low = _mm512_sub_epi64(cur_v, _mm512_slli_epi64(high, LOG2_B));
        T.dig[d][0][j] = _mm512_mask_add_epi64(low, _mm512_cmplt_epi64_mask(low, zero), low, vq1);
        __m512i r = _mm512_mask_add_epi64(low, _mm512_cmplt_epi64_mask(low, zero), low, vq2);
        r = _mm512_mask_add_epi64(r, _mm512_cmplt_epi64_mask(r, zero), r, vq2);
        r = _mm512_mask_sub_epi64(r, _mm512_cmpge_epi64_mask(r, vq2), r, vq2);
        T.dig[d][1][j] = r;
        cur_v = high;
      }
    }
    T.bar.wait();
    // the four digit transforms, one per thread (base_pir.rs:574-579)
    if (t % 2 == 0)
      weighted_ntt8<0>(R, T.dig[t / 2][0]);
    else
      weighted_ntt8<1>(R, T.dig[t / 2][1]);
    T.bar.wait();
    // reply_a, the stored digits and the next sum (preprocess_loop)
    for (size_t j = j0; j < j1; j++) {
      const __m512i r0 = addmod<0>(mulmod<0>(T.dig[0][0][j], T.gk[0][0][j]), mulmod<0>(T.dig[1][0][j], T.gk[1][0][j]));
      const __m512i r1 = addmod<1>(mulmod<1>(T.dig[0][1][j], T.gk[0][1][j]), mulmod<1>(T.dig[1][1][j], T.gk[1][1][j]));
      for (int d = 0; d < 2; d++)
        for (int pi = 0; pi < 2; pi++) st(&db.gk[T.c][d][pi][(i * N + j) * SIMD], T.dig[d][pi][j]);
      T.sum[0][j] = addmod<0>(r0, mulmod<0>(T.qa[0][j], ld(&db.te[T.c][0][(i * N + j) * SIMD])));
      T.sum[1][j] = addmod<1>(r1, mulmod<1>(T.qa[1][j], ld(&db.te[T.c][1][(i * N + j) * SIMD])));
    }
    T.bar.wait();
  }
}

// the chain of half c for all 8 lanes (preprocess_loop, base_pir.rs:782-863)
ORC_AVX512 static void chain_half(Shard& db, int c, const std::vector<uint64_t> gka[2][2],
                                  const std::vector<uint64_t> qa[2], std::vector<uint64_t> sums_out[2]) {
  const Ring& R = *db.R;
  const size_t N = R.n;
  const int64_t m = 2 * (int64_t)N;
  const int64_t inv_g = (int64_t)invmod(5, (uint64_t)m);
  ChainTeam T(&db, c, N);
  for (size_t i = 0; i < N; i++) T.gmap[i] = gal2idx(N, inv_g * idx2gal(N, (int64_t)i) % m);
  for (size_t j = 0; j < N; j++)
    for (int pi = 0; pi < 2; pi++) {
      T.sum[pi][j] = _mm512_setzero_si512();
      for (int d = 0; d < 2; d++) T.gk[d][pi][j] = ld(&gka[d][pi][j * SIMD]);
      T.qa[pi][j] = ld(&qa[pi][j * SIMD]);
    }
  std::vector<std::thread> th;
  for (int t = 1; t < 4; t++) th.emplace_back([&T, t]() { chain_thread(T, t); });
  chain_thread(T, 0);
  for (auto& x : th) x.join();
  for (int pi = 0; pi < 2; pi++) sums_out[pi].assign(N * SIMD, 0);
  for (size_t j = 0; j < N; j++) {
    st(&sums_out[0][j * SIMD], T.sum[0][j]);
    st(&sums_out[1][j * SIMD], T.sum[1][j]);
  }
}

// main_pir_loop on vectors (same recurrence, reduction every reduce_every rows)
ORC_AVX512 static void main_pir_loop8(size_t N, size_t len, size_t reduce_every, const Mod& md,
                                      std::vector<uint64_t>& sum, const std::vector<size_t>& gal,
                                      const uint64_t* qry_b, const uint64_t* gk0, const uint64_t* gk1,
                                      const uint64_t* ipg0, const uint64_t* ipg1, const uint64_t* te) {
  std::vector<uint64_t> sum_new(N * SIMD, 0);
  size_t index = 0;
  for (size_t io = 0; io < len; io += reduce_every) {
    const size_t cnt = std::min(len - io, reduce_every);
    for (size_t ii = 0; ii < cnt; ii++) {
      for (size_t j = 0; j < N; j++) {
        const size_t e = (index + j) * SIMD;
        __m512i acc = ld(&sum[j * SIMD]);
        acc = _mm512_add_epi64(acc, _mm512_mul_epu32(ld(&ipg0[e]), ld(&gk0[j * SIMD])));
        acc = _mm512_add_epi64(acc, _mm512_mul_epu32(ld(&ipg1[e]), ld(&gk1[j * SIMD])));
        acc = _mm512_add_epi64(acc, _mm512_mul_epu32(ld(&te[e]), ld(&qry_b[j * SIMD])));
        st(&sum_new[gal[j] * SIMD], acc);
      }
      index += N;
      std::swap(sum, sum_new);
    }
    for (size_t j = 0; j < N * SIMD; j++) sum[j] = md.red(sum[j]);
  }
}

}  // namespace vec

static void preprocess_vec(Shard& db) {
  const Ring& R = *db.R;
  const size_t N = R.n, L = db.ig.loop_len();
  std::vector<uint64_t> gka[2][2];
  for (int d = 0; d < 2; d++) to_simd_element_same(R, gk_a(N, d), gka[d]);
  std::vector<uint64_t> qa[2][2];
  for (int c = 0; c < (db.ig.conj() ? 2 : 1); c++) to_simd_element_same(R, qry_a(N, db.used_seeds, c), qa[c]);
  for (int c = 0; c < 2; c++)
    for (int d = 0; d < 2; d++)
      for (int pi = 0; pi < 2; pi++) db.gk[c][d][pi].assign(db.ig.conj() || c == 0 ? L * N * SIMD : 0, 0);
  const int halves = db.ig.conj() ? 2 : 1;
  std::vector<uint64_t> sums[2][2];
  parallel_for((size_t)halves, [&](size_t c) { vec::chain_half(db, (int)c, gka, qa[c], sums[c]); });
  for (int pi = 0; pi < 2; pi++) {
    db.reply_a[pi].assign(N * SIMD, 0);
    for (size_t j = 0; j < N * SIMD; j++)
      db.reply_a[pi][j] = halves == 2 ? R.md[pi].add(sums[0][pi][j], sums[1][pi][j]) : sums[0][pi][j];
  }
  db.has_reply_a = true;
}

// perform_pir_split with the vector scan (everything else as the scalar function)
static void perform_pir_split_vec(const Shard& db, const QueryRef q[SIMD], Poly out[SIMD]) {
  const Ring& R = *db.R;
  const size_t N = R.n, L = db.ig.loop_len();
  const int64_t m = 2 * (int64_t)N;
  std::vector<uint64_t> qb[2], qcb[2], gkb[2][2];
  {
    const Poly* els[SIMD];
    for (int k = 0; k < SIMD; k++) els[k] = q[k].qry_b;
    to_simd_element(R, els, qb);
    if (db.ig.conj()) {
      for (int k = 0; k < SIMD; k++) {
        ORC_CHECK(q[k].qry_conj_b, "conjugate query must be given when index subgroup requires conjugation");
        els[k] = q[k].qry_conj_b;
      }
      to_simd_element(R, els, qcb);
    }
    for (int d = 0; d < 2; d++) {
      for (int k = 0; k < SIMD; k++) els[k] = q[k].gk_b[d];
      to_simd_element(R, els, gkb[d]);
    }
  }
  const int64_t inv_g = (int64_t)invmod(5, (uint64_t)m);
  std::vector<size_t> gal(N);
  for (size_t i = 0; i < N; i++) gal[i] = (size_t)((mod_floor(inv_g * (2 * (int64_t)i + 1), m) - 1) / 2);
  std::vector<uint64_t> sum[2], sum_conj[2];
  const int halves = db.ig.conj() ? 2 : 1;
  u128 rb0 = 2 * (u128)R.p[0], rb1 = 2 * (u128)R.p[1];
  const size_t reduce_every = (size_t)std::min((u128)UINT64_MAX / rb0 / rb0 / (GK_DIGITS + 1),
                                               (u128)UINT64_MAX / rb1 / rb1 / (GK_DIGITS + 1));
  parallel_for((size_t)2 * halves, [&](size_t u) {
    const int pi = (int)(u % 2), c = (int)(u / 2);
    std::vector<uint64_t>& s = c ? sum_conj[pi] : sum[pi];
    s.assign(N * SIMD, 0);
    vec::main_pir_loop8(N, L, reduce_every, R.md[pi], s, gal, (c ? qcb : qb)[pi].data(), gkb[0][pi].data(),
                        gkb[1][pi].data(), db.gk[c][0][pi].data(), db.gk[c][1][pi].data(), db.te[c][pi].data());
  });
  for (int pi = 0; pi < 2; pi++) {
    if (halves == 2)
      for (size_t j = 0; j < N * SIMD; j++) sum[pi][j] += sum_conj[pi][j];
    std::vector<uint64_t> pm(N * SIMD);
    for (size_t i = 0; i < N; i++)
      for (int k = 0; k < SIMD; k++) pm[i * SIMD + k] = R.md[pi].red(sum[pi][gal[i] * SIMD + k]);
    sum[pi].swap(pm);
  }
  from_simd_element(R, sum, out);
}

struct orc_db {
  Shard s;
};
struct orc_rng {
  StdRng r;
  explicit orc_rng(const uint8_t* seed) : r(seed) {}
};

static thread_local std::string g_err;
#define ORC_TRY(...)                    \
  try {                                 \
    __VA_ARGS__;                        \
    return 0;                           \
  } catch (const std::exception& e) {   \
    g_err = e.what();                   \
    return -1;                          \
  }

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }
int orc_num_threads() { return num_threads(); }
void orc_set_num_threads(int n) { g_threads = n; }

// ring constants
uint64_t orc_q1() { return Q1; }
uint64_t orc_q2() { return Q2; }
uint64_t orc_q() { return QQ; }
uint64_t orc_zeta(int log2n, int prime) { return get_ring(log2n)->zeta[prime]; }

// rng
orc_rng* orc_rng_new(const uint8_t* seed32) { return new orc_rng(seed32); }
void orc_rng_free(orc_rng* r) { delete r; }
uint64_t orc_rng_next_u64(orc_rng* r) { return r->r.next_u64(); }
uint32_t orc_rng_next_u32(orc_rng* r) { return r->r.next_u32(); }

// a-parts: out = 6 x N coefficients in [0, q) (gk0, gk1, qry FirstSet main/conj, qry SecondSet main/conj)
int orc_get_aparts(int log2n, int64_t* out) {
  ORC_TRY({
    size_t N = (size_t)1 << log2n;
    for (int s = 0; s < 6; s++) memcpy(out + s * N, apart(N, s).data(), N * 8);
  })
}
int orc_set_aparts(int log2n, const int64_t* in) {
  ORC_TRY({
    size_t N = (size_t)1 << log2n;
    if (!in) {
      g_aparts.parts[log2n].clear();
    } else {
      g_aparts.parts[log2n].assign(6, Poly(N));
      for (int s = 0; s < 6; s++) memcpy(g_aparts.parts[log2n][s].data(), in + s * N, N * 8);
    }
  })
}
int orc_expand(int log2n, const uint8_t* seed32, int64_t* out) {
  ORC_TRY({
    Poly p = expand((size_t)1 << log2n, seed32);
    memcpy(out, p.data(), p.size() * 8);
  })
}

// shape helpers (pir_wrapper.rs:166-241, base_pir.rs:369)
int orc_get_database_shape(uint64_t num_entries, uint32_t* l1, uint32_t* l2, uint32_t* num_shards) {
  ORC_TRY({
    IndexGroup a, b;
    get_database_shape(num_entries, &a, &b);
    *l1 = (uint32_t)a.l;
    *l2 = (uint32_t)b.l;
    *num_shards = (uint32_t)((num_entries + SIMD * a.l - 1) / (SIMD * a.l));
  })
}
int orc_choose_secondary(uint32_t num_shards, uint32_t* l2) {
  ORC_TRY({ *l2 = (uint32_t)choose_secondary(num_shards).l; })
}
uint64_t orc_required_memory_general(uint32_t log2n, uint32_t l) {
  return (uint64_t)(GK_DIGITS + 1) * 2 * ((uint64_t)1 << log2n) * l;
}

// PIRDatabase
int orc_db_create(int log2n, uint32_t l, int used_seeds, orc_db** out) {
  ORC_TRY({
    std::unique_ptr<orc_db> d(new orc_db());
    d->s.R = get_ring(log2n);
    d->s.ig = make_group((size_t)1 << log2n, l);
    d->s.used_seeds = used_seeds;
    *out = d.release();
  })
}
void orc_db_free(orc_db* d) { delete d; }
// entries: (8 l) x N coefficients in [0, t)
int orc_db_set_db(orc_db* d, const uint16_t* entries) {
  ORC_TRY({
    set_transformed_entries(d->s, entries);
    preprocess(d->s);
  })
}
// the vectorised restatement (AVX-512; the caller checks orc_cpu_has_avx512)
int orc_db_set_db_vec(orc_db* d, const uint16_t* entries) {
  ORC_TRY({
    for (size_t i = 0; i < (size_t)SIMD * d->s.ig.l * d->s.R->n; i++)
      ORC_CHECK(entries[i] < TPLAIN, "entry coefficient must be below t");
    set_transformed_entries_vec(d->s, entries);
    preprocess_vec(d->s);
  })
}
int orc_db_set_transformed_entries(orc_db* d, const uint16_t* entries) {
  ORC_TRY({ set_transformed_entries(d->s, entries); })
}
uint32_t orc_db_loop_len(orc_db* d) { return (uint32_t)d->s.ig.loop_len(); }
// arrays: which = 0 transformed_entries, 1 inner_prod_gk digit 0, 2 digit 1; out: L x N x 8
int orc_db_array(orc_db* d, int which, int conj, int prime, uint64_t* out) {
  ORC_TRY({
    const std::vector<uint64_t>& v = which == 0 ? d->s.te[conj][prime] : d->s.gk[conj][which - 1][prime];
    ORC_CHECK(!v.empty(), "array not present");
    memcpy(out, v.data(), v.size() * 8);
  })
}
int orc_db_reply_a_ntt(orc_db* d, int prime, uint64_t* out) {
  ORC_TRY({
    ORC_CHECK(d->s.has_reply_a, "not preprocessed");
    memcpy(out, d->s.reply_a[prime].data(), d->s.reply_a[prime].size() * 8);
  })
}
// out: 8 x N coefficients mod q
int orc_db_get_a(orc_db* d, int64_t* out) {
  ORC_TRY({
    Poly a[SIMD];
    get_a(d->s, a);
    size_t N = d->s.R->n;
    for (int k = 0; k < SIMD; k++) memcpy(out + k * N, a[k].data(), N * 8);
  })
}
// queries: qry_b 8 x N, qry_conj_b 8 x N (or null), gk_b 8 x 2 x N; out 8 x N
int orc_db_perform_pir_split(orc_db* d, const int64_t* qry_b, const int64_t* qry_conj_b, const int64_t* gk_b,
                             int64_t* out) {
  ORC_TRY({
    size_t N = d->s.R->n;
    std::vector<Poly> qb(SIMD), qcb(SIMD), g0(SIMD), g1(SIMD);
    QueryRef qr[SIMD];
    for (int k = 0; k < SIMD; k++) {
      qb[k].assign(qry_b + k * N, qry_b + (k + 1) * N);
      if (qry_conj_b) qcb[k].assign(qry_conj_b + k * N, qry_conj_b + (k + 1) * N);
      g0[k].assign(gk_b + (2 * k) * N, gk_b + (2 * k + 1) * N);
      g1[k].assign(gk_b + (2 * k + 1) * N, gk_b + (2 * k + 2) * N);
      qr[k] = QueryRef{&qb[k], qry_conj_b ? &qcb[k] : nullptr, {&g0[k], &g1[k]}};
    }
    Poly o[SIMD];
    perform_pir_split(d->s, qr, o);
    for (int k = 0; k < SIMD; k++) memcpy(out + k * N, o[k].data(), N * 8);
  })
}

int orc_db_perform_pir_split_vec(orc_db* d, const int64_t* qry_b, const int64_t* qry_conj_b, const int64_t* gk_b,
                                 int64_t* out) {
  ORC_TRY({
    size_t N = d->s.R->n;
    std::vector<Poly> qb(SIMD), qcb(SIMD), g0(SIMD), g1(SIMD);
    QueryRef qr[SIMD];
    for (int k = 0; k < SIMD; k++) {
      qb[k].assign(qry_b + k * N, qry_b + (k + 1) * N);
      if (qry_conj_b) qcb[k].assign(qry_conj_b + k * N, qry_conj_b + (k + 1) * N);
      g0[k].assign(gk_b + (2 * k) * N, gk_b + (2 * k + 1) * N);
      g1[k].assign(gk_b + (2 * k + 1) * N, gk_b + (2 * k + 2) * N);
      qr[k] = QueryRef{&qb[k], qry_conj_b ? &qcb[k] : nullptr, {&g0[k], &g1[k]}};
    }
    Poly o[SIMD];
    perform_pir_split_vec(d->s, qr, o);
    for (int k = 0; k < SIMD; k++) memcpy(out + k * N, o[k].data(), N * 8);
  })
}

// perform_double_pir (double_pir.rs:104-123) on ring elements; out: 3 x (a, b) x N
int orc_perform_double_pir(orc_db** dbs, uint32_t ndb, uint32_t l2, const int64_t* pq, const int64_t* pqc,
                           const int64_t* sq, const int64_t* sqc, const int64_t* gk, int64_t* out) {
  ORC_TRY({
    ORC_CHECK(ndb >= 1, "empty fleet");
    size_t N = dbs[0]->s.R->n;
    Poly P(pq, pq + N), PC, S(sq, sq + N), SC, G0(gk, gk + N), G1(gk + N, gk + 2 * N);
    if (pqc) PC.assign(pqc, pqc + N);
    if (sqc) SC.assign(sqc, sqc + N);
    DoubleQuery dq{&P, pqc ? &PC : nullptr, &S, sqc ? &SC : nullptr, {&G0, &G1}};
    std::vector<const Shard*> sh(ndb);
    for (uint32_t i = 0; i < ndb; i++) sh[i] = &dbs[i]->s;
    const Shard* const* fleets[BATCH] = {sh.data(), sh.data()};
    size_t nd[BATCH] = {ndb, ndb};
    const DoubleQuery* qs[BATCH] = {&dq, nullptr};
    IndexGroup ig2 = make_group(N, l2);
    std::vector<std::array<Poly, 2>> res[BATCH];
    perform_batched_double_pir(fleets, nd, qs, ig2, res);
    for (int j = 0; j < CTXT_PARTS; j++) {
      memcpy(out + (2 * j) * N, res[0][j][0].data(), N * 8);
      memcpy(out + (2 * j + 1) * N, res[0][j][1].data(), N * 8);
    }
  })
}

// wire codec
int orc_condense(int bits, const uint64_t* data, uint64_t n, uint8_t* out, uint64_t* out_len) {
  ORC_TRY({
    std::vector<uint8_t> v;
    condense(bits, data, n, v);
    memcpy(out, v.data(), v.size());
    *out_len = v.size();
  })
}
int orc_uncondense(int bits, uint64_t n, const uint8_t* data, uint64_t len, uint64_t* out, uint64_t* consumed) {
  ORC_TRY({ *consumed = uncondense(bits, n, data, len, out); })
}
int orc_ms_encode(int bits, const int64_t* x, uint64_t n, uint64_t* out) {
  ORC_TRY({
    for (uint64_t i = 0; i < n; i++) out[i] = ms_encode(x[i], bits);
  })
}
int orc_ms_decode(int bits, const uint64_t* x, uint64_t n, int64_t* out) {
  ORC_TRY({
    for (uint64_t i = 0; i < n; i++) out[i] = ms_decode(x[i], bits);
  })
}

// process_queries (pir_wrapper.rs:349-409) for one query in batch slot 0;
// fleet = ndb shard handles (shard k of the fleet is dbs[k]).
// process_query with an explicit secondary group order (0: the shape rule's
// choose_index_group_secondary, pir_wrapper.rs:166-175), as the reference's
// perform_double_pir allows (double_pir.rs:104-123)
int orc_process_query_general(orc_db** dbs, uint32_t ndb, uint32_t l2, const uint8_t* query, uint64_t qlen,
                              uint8_t* reply, uint64_t* reply_len) {
  ORC_TRY({
    const size_t N = (size_t)1 << LOG2_N_WIRE;
    ORC_CHECK(ndb >= 1 && dbs[0]->s.R->n == N, "fleet must be built at N = 2048");
    IndexGroup ig1 = dbs[0]->s.ig;
    IndexGroup ig2 = l2 ? make_group(N, l2) : choose_secondary(ndb);
    ORC_CHECK((size_t)ndb * SIMD <= ig2.l, "secondary group too small for the number of shards");
    size_t pos = 0;
    std::vector<uint64_t> raw(N);
    auto take = [&](int bits) {
      pos += uncondense(bits, N, query + pos, qlen - pos, raw.data());
      Poly p(N);
      for (size_t i = 0; i < N; i++) p[i] = ms_decode(raw[i], bits);
      return p;
    };
    Poly G0 = take(GK_BITS), G1 = take(GK_BITS);
    Poly P = take(PQ_BITS), PC;
    if (ig1.conj()) PC = take(PQ_BITS);
    Poly S = take(SQ_BITS), SC;
    if (ig2.conj()) SC = take(SQ_BITS);
    DoubleQuery dq{&P, ig1.conj() ? &PC : nullptr, &S, ig2.conj() ? &SC : nullptr, {&G0, &G1}};
    std::vector<const Shard*> sh(ndb);
    for (uint32_t i = 0; i < ndb; i++) sh[i] = &dbs[i]->s;
    const Shard* const* fleets[BATCH] = {sh.data(), sh.data()};
    size_t nd[BATCH] = {ndb, ndb};
    const DoubleQuery* qs[BATCH] = {&dq, nullptr};
    std::vector<std::array<Poly, 2>> res[BATCH];
    perform_batched_double_pir(fleets, nd, qs, ig2, res);
    std::vector<uint8_t> out;
    std::vector<uint64_t> enc(N);
    for (int j = 0; j < CTXT_PARTS; j++) {
      for (size_t i = 0; i < N; i++) enc[i] = ms_encode(res[0][j][0][i], SEC_A_BITS);
      condense(SEC_A_BITS, enc.data(), N, out);
      for (size_t i = 0; i < N; i++) enc[i] = ms_encode(res[0][j][1][i], SEC_B_BITS);
      condense(SEC_B_BITS, enc.data(), N, out);
    }
    memcpy(reply, out.data(), out.size());
    *reply_len = out.size();
  })
}

int orc_process_query(orc_db** dbs, uint32_t ndb, const uint8_t* query, uint64_t qlen, uint8_t* reply,
                      uint64_t* reply_len) {
  return orc_process_query_general(dbs, ndb, 0, query, qlen, reply, reply_len);
}

// ---- client side (test only)
int orc_gen_sk(orc_rng* rng, int log2n, int8_t* sk) {
  ORC_TRY({
    std::vector<int8_t> s = gen_sk((size_t)1 << log2n, rng->r, SK_HWT);
    memcpy(sk, s.data(), s.size());
  })
}
// plaintext m: N coefficients in [0, t); out: b-part
int orc_enc_sym_b(orc_rng* rng, int log2n, int apart_index, const int8_t* sk, const int64_t* m, int64_t* out) {
  ORC_TRY({
    size_t N = (size_t)1 << log2n;
    std::vector<int8_t> s(sk, sk + N);
    Poly mm(m, m + N);
    Poly b = enc_sym_b(N, TPLAIN, apart(N, apart_index), rng->r, s, mm, SIGMA);
    memcpy(out, b.data(), N * 8);
  })
}
int orc_gen_gk_b(orc_rng* rng, int log2n, const int8_t* sk, int64_t* out /* 2 x N */) {
  ORC_TRY({
    size_t N = (size_t)1 << log2n;
    std::vector<int8_t> s(sk, sk + N);
    std::vector<Poly> g = gen_gk_b(N, rng->r, s, 5, GK_DIGITS, LOG2_B, SIGMA);
    memcpy(out, g[0].data(), N * 8);
    memcpy(out + N, g[1].data(), N * 8);
  })
}
int orc_dec(int log2n, const int8_t* sk, const int64_t* a, const int64_t* b, int64_t* out) {
  ORC_TRY({
    size_t N = (size_t)1 << log2n;
    std::vector<int8_t> s(sk, sk + N);
    Poly o = dec(N, TPLAIN, s, Poly(a, a + N), Poly(b, b + N));
    memcpy(out, o.data(), N * 8);
  })
}
// enc_double_pir; outputs: pq, pqc, sq, sqc (N each; conj only when the group needs it), gk (2 x N)
int orc_enc_double_pir(orc_rng* rng, int log2n, uint32_t l1, uint32_t l2, const int8_t* sk, uint64_t primary_idx,
                       uint64_t secondary_idx, int64_t* pq, int64_t* pqc, int64_t* sq, int64_t* sqc, int64_t* gk,
                       int* has_pqc, int* has_sqc) {
  ORC_TRY({
    size_t N = (size_t)1 << log2n;
    std::vector<int8_t> s(sk, sk + N);
    IndexGroup ig1 = make_group(N, l1), ig2 = make_group(N, l2);
    EncQuery q = enc_double_pir(rng->r, ig1, ig2, s, primary_idx, secondary_idx, SIGMA);
    memcpy(pq, q.pq.data(), N * 8);
    memcpy(sq, q.sq.data(), N * 8);
    if (q.has_pqc) memcpy(pqc, q.pqc.data(), N * 8);
    if (q.has_sqc) memcpy(sqc, q.sqc.data(), N * 8);
    memcpy(gk, q.gk[0].data(), N * 8);
    memcpy(gk + N, q.gk[1].data(), N * 8);
    *has_pqc = q.has_pqc;
    *has_sqc = q.has_sqc;
  })
}
// reply: 3 x (a, b) x N; out: N coefficients in [0, t)
int orc_dec_double_pir(int log2n, const int8_t* sk, const int64_t* reply, int64_t* out) {
  ORC_TRY({
    size_t N = (size_t)1 << log2n;
    std::vector<int8_t> s(sk, sk + N);
    Poly ra[CTXT_PARTS], rb[CTXT_PARTS];
    for (int j = 0; j < CTXT_PARTS; j++) {
      ra[j].assign(reply + (2 * j) * N, reply + (2 * j + 1) * N);
      rb[j].assign(reply + (2 * j + 1) * N, reply + (2 * j + 2) * N);
    }
    Poly o = dec_double_pir(N, s, ra, rb);
    memcpy(out, o.data(), N * 8);
  })
}
// prepare_query_general (pir_wrapper.rs:276-317): query bytes + sk seed
int orc_prepare_query(orc_rng* rng, uint64_t primary_idx, uint64_t secondary_idx, uint32_t l1, uint32_t l2,
                      uint8_t* query, uint64_t* qlen, uint8_t* sk_seed32) {
  ORC_TRY({
    const size_t N = (size_t)1 << LOG2_N_WIRE;
    IndexGroup ig1 = make_group(N, l1), ig2 = make_group(N, l2);
    uint8_t seed[32];
    for (int i = 0; i < 32; i++) seed[i] = (uint8_t)(rng->r.next_u32() & 0xFFFF);
    StdRng skr(seed);
    std::vector<int8_t> sk = gen_sk(N, skr, SK_HWT);
    EncQuery q = enc_double_pir(rng->r, ig1, ig2, sk, primary_idx, secondary_idx, SIGMA);
    std::vector<uint8_t> out;
    std::vector<uint64_t> enc(N);
    auto put = [&](const Poly& p, int bits) {
      for (size_t i = 0; i < N; i++) enc[i] = ms_encode(p[i], bits);
      condense(bits, enc.data(), N, out);
    };
    put(q.gk[0], GK_BITS);
    put(q.gk[1], GK_BITS);
    put(q.pq, PQ_BITS);
    if (ig1.conj()) put(q.pqc, PQ_BITS);
    put(q.sq, SQ_BITS);
    if (ig2.conj()) put(q.sqc, SQ_BITS);
    memcpy(query, out.data(), out.size());
    *qlen = out.size();
    memcpy(sk_seed32, seed, 32);
  })
}
// process_reply (pir_wrapper.rs:420-440): N coefficients in [0, t)
int orc_process_reply(const uint8_t* reply, uint64_t len, const uint8_t* sk_seed32, int64_t* out) {
  ORC_TRY({
    const size_t N = (size_t)1 << LOG2_N_WIRE;
    StdRng skr(sk_seed32);
    std::vector<int8_t> sk = gen_sk(N, skr, SK_HWT);
    size_t pos = 0;
    std::vector<uint64_t> raw(N);
    Poly ra[CTXT_PARTS], rb[CTXT_PARTS];
    for (int j = 0; j < CTXT_PARTS; j++) {
      pos += uncondense(SEC_A_BITS, N, reply + pos, len - pos, raw.data());
      ra[j].resize(N);
      for (size_t i = 0; i < N; i++) ra[j][i] = ms_decode(raw[i], SEC_A_BITS);
      pos += uncondense(SEC_B_BITS, N, reply + pos, len - pos, raw.data());
      rb[j].resize(N);
      for (size_t i = 0; i < N; i++) rb[j][i] = ms_decode(raw[i], SEC_B_BITS);
    }
    Poly o = dec_double_pir(N, sk, ra, rb);
    memcpy(out, o.data(), N * 8);
  })
}

// reduce_after_mul / reduce_from_2p of simd_zn.rs:197-239, restated for the
// exhaustive test (simd_zn.rs:490-542): out[i] for x = start + i
void orc_reduce_after_mul(int K, uint64_t start, uint64_t count, uint64_t* out_lazy, uint64_t* out_full) {
  const uint64_t p = ((uint64_t)1 << K) - ((1 << 12) - 1);
  for (uint64_t i = 0; i < count; i++) {
    uint64_t x = start + i;
    auto step = [&](uint64_t d) { return d - (uint64_t)(uint32_t)(d >> K) * p; };
    uint64_t r = step(step(x));
    out_lazy[i] = r;
    out_full[i] = r > p ? r - p : r;
  }
}

}  // extern "C"
