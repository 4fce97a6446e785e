// client.cpp -- client side of the wire protocol, host C++ (no device work):
// prepare_query (crates/pir/src/pir_wrapper.rs:259-317) and process_reply
// (:420-440) with the BFV primitives they use (bfv.rs:37-125,
// double_pir.rs:83-93, 245-317).  Used for load generation and to decrypt and
// check answers; the server path never calls it.
//
// Randomness: one StdRng-compatible ChaCha12 stream per query, keyed by a
// caller-provided 32-byte seed; the secret-key seed is 32 low bytes of
// next_u32 as in pir_wrapper.rs:289; error terms are rounded N(0, 3.2^2)
// samples (Box-Muller on 53-bit uniforms; the reference samples rand_distr's
// StandardNormal).  Only the server's answer has to be reproducible; the
// client's randomness is never part of a reply's correctness.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "dnspir.h"

namespace {

typedef __int128 i128;
typedef unsigned __int128 u128;

const int64_t CQ1 = (1LL << 26) - (1LL << 12) + 1;
const int64_t CQ2 = (1LL << 25) - (1LL << 12) + 1;
const int64_t CQ = CQ1 * CQ2;
const int64_t TP = 1025;
const int CN = 2048;
const int HWT = 128;
const double SIG = 3.2;

int64_t modf_(int64_t a, int64_t m) {
  int64_t r = a % m;
  return r < 0 ? r + m : r;
}
int64_t modi(i128 a, int64_t m) {
  i128 r = a % m;
  return (int64_t)(r < 0 ? r + m : r);
}
int64_t lift(int64_t x, int64_t m) { return x > m / 2 ? x - m : x; }
int64_t inv_mod(int64_t a, int64_t m) {
  int64_t t = 0, nt = 1, r = m, nr = modf_(a, m);
  while (nr) {
    int64_t q = r / nr, tmp = t - q * nt;
    t = nt;
    nt = tmp;
    tmp = r - q * nr;
    r = nr;
    nr = tmp;
  }
  return modf_(t, m);
}

struct Rng {  // ChaCha12 word stream of rand_chacha 0.3.1's StdRng
  uint32_t key[8];
  uint64_t ctr = 0;
  uint32_t buf[64];
  int idx = 64;
  explicit Rng(const uint8_t* seed) {
    for (int i = 0; i < 8; i++)
      key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
               ((uint32_t)seed[4 * i + 3] << 24);
  }
  static uint32_t rl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
  void refill() {
    for (int b = 0; b < 4; b++) {
      const uint64_t c = ctr + b;
      uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                        key[4],      key[5],      key[6],      key[7],      (uint32_t)c, (uint32_t)(c >> 32), 0, 0};
      uint32_t x[16];
      memcpy(x, s, sizeof(x));
      auto qr = [&](int a, int bb, int cc, int d) {
        x[a] += x[bb]; x[d] = rl(x[d] ^ x[a], 16);
        x[cc] += x[d]; x[bb] = rl(x[bb] ^ x[cc], 12);
        x[a] += x[bb]; x[d] = rl(x[d] ^ x[a], 8);
        x[cc] += x[d]; x[bb] = rl(x[bb] ^ x[cc], 7);
      };
      for (int r = 0; r < 6; r++) {
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
      }
      for (int i = 0; i < 16; i++) buf[16 * b + i] = x[i] + s[i];
    }
    ctr += 4;
    idx = 0;
  }
  uint32_t u32() {
    if (idx >= 64) refill();
    return buf[idx++];
  }
  uint64_t u64() {
    if (idx < 63) {
      uint64_t r = (uint64_t)buf[idx] | ((uint64_t)buf[idx + 1] << 32);
      idx += 2;
      return r;
    }
    if (idx >= 64) {
      refill();
      idx = 2;
      return (uint64_t)buf[0] | ((uint64_t)buf[1] << 32);
    }
    uint64_t lo = buf[63];
    refill();
    idx = 1;
    return lo | ((uint64_t)buf[0] << 32);
  }
  double normal() {
    double u1 = ((double)((u64() >> 11) + 1)) * (1.0 / 9007199254740992.0);
    double u2 = ((double)(u64() >> 11)) * (1.0 / 9007199254740992.0);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

typedef std::vector<int64_t> P;

std::vector<int8_t> gen_sk(Rng& r) {  // bfv.rs:37-45
  std::vector<int8_t> s(CN, 0);
  for (int i = 0; i < HWT; i++) {
    size_t idx = (size_t)(r.u64() % CN);
    s[idx] = (int8_t)((int)(r.u32() % 3) - 1);
  }
  return s;
}

P mul_sk(const P& a, const std::vector<int8_t>& sk) {
  std::vector<i128> acc(CN, 0);
  for (int j = 0; j < CN; j++) {
    if (!sk[j]) continue;
    for (int i = 0; i < CN; i++) {
      i128 v = (i128)a[i] * sk[j];
      if (i + j >= CN) acc[i + j - CN] -= v;
      else acc[i + j] += v;
    }
  }
  P out(CN);
  for (int i = 0; i < CN; i++) out[i] = modi(acc[i], CQ);
  return out;
}

// a-part `which` in effect (the seed expansion, or what dnspir_set_a_parts installed)
P apart(int which) {
  std::vector<uint64_t> v((size_t)6 * CN);
  dnspir_get_a_parts(11, v.data());
  return P(v.begin() + (size_t)which * CN, v.begin() + (size_t)(which + 1) * CN);
}

P enc_sym_b(const P& a, Rng& r, const std::vector<int8_t>& sk, const P& m) {  // bfv.rs:72-87
  P e(CN);
  for (int i = 0; i < CN; i++) e[i] = modf_((int64_t)std::llround(r.normal() * SIG), CQ);
  const int64_t tinv = inv_mod(TP, CQ);
  P as = mul_sk(a, sk);
  P b(CN);
  for (int i = 0; i < CN; i++) {
    i128 up = (i128)lift(m[i], TP) * CQ;
    int64_t delta = lift(modi(up, TP), TP);
    int64_t down = (int64_t)(((u128)(uint64_t)modi(up - delta, CQ) * (uint64_t)tinv) % (u128)CQ);
    b[i] = modf_(modf_(e[i] - as[i], CQ) + down, CQ);
  }
  return b;
}

P dec(const std::vector<int8_t>& sk, const P& a, const P& b) {  // bfv.rs:90-102
  P as = mul_sk(a, sk);
  const int64_t qinv = inv_mod(CQ % TP, TP);
  P out(CN);
  for (int i = 0; i < CN; i++) {
    int64_t c = lift(modf_(as[i] + b[i], CQ), CQ);
    i128 up = (i128)c * TP;
    int64_t delta = lift(modi(up, CQ), CQ);
    out[i] = (modi((up - delta) % TP, TP) * qinv) % TP;
  }
  return out;
}

uint64_t ms_enc(int64_t c, int bits) {  // bfv.rs:52-58
  i128 num = (i128)lift(c, CQ) * ((i128)1 << bits);
  i128 t = 2 * num + CQ, two_q = 2 * (i128)CQ;
  i128 q = t / two_q;
  if (t % two_q != 0 && t < 0) q -= 1;
  i128 r = (q + ((i128)1 << bits)) % ((i128)1 << bits);
  if (r < 0) r += (i128)1 << bits;
  return (uint64_t)r;
}
int64_t ms_dec(uint64_t x, int bits) { return modi(((i128)x * CQ) >> bits, CQ); }  // bfv.rs:61-69

void condense(int bits, const std::vector<uint64_t>& d, std::vector<uint8_t>& out) {  // pir_wrapper.rs:84-113
  const size_t n = d.size();
  for (int i = 0; i < bits / 8; i++)
    for (size_t t = 0; t < n; t++) out.push_back((uint8_t)(d[t] >> (8 * i)));
  if (bits % 8 >= 4)
    for (size_t t = 0; t + 2 <= n; t += 2)
      out.push_back((uint8_t)((((d[t] >> ((bits / 8) * 8)) & 0xF) << 4) | ((d[t + 1] >> ((bits / 8) * 8)) & 0xF)));
  if (bits % 4 >= 2)
    for (size_t t = 0; t + 4 <= n; t += 4) {
      uint8_t v = 0;
      for (int u = 0; u < 4; u++) v |= (uint8_t)(((d[t + u] >> ((bits / 4) * 4)) & 3) << (6 - 2 * u));
      out.push_back(v);
    }
  if (bits % 2 >= 1)
    for (size_t t = 0; t + 8 <= n; t += 8) {
      uint8_t v = 0;
      for (int u = 0; u < 8; u++) v |= (uint8_t)(((d[t + u] >> ((bits / 2) * 2)) & 1) << (7 - u));
      out.push_back(v);
    }
}
// uncondense (pir_wrapper.rs:120-158); false = "not enough data"
bool uncondense(int bits, size_t n, const uint8_t* d, size_t len, size_t& pos, std::vector<uint64_t>& out) {
  out.assign(n, 0);
  auto nx = [&](uint8_t& v) {
    if (pos >= len) return false;
    v = d[pos++];
    return true;
  };
  uint8_t s;
  for (int i = 0; i < bits / 8; i++)
    for (size_t t = 0; t < n; t++) {
      if (!nx(s)) return false;
      out[t] |= (uint64_t)s << (8 * i);
    }
  if (bits % 8 >= 4)
    for (size_t t = 0; t + 2 <= n; t += 2) {
      if (!nx(s)) return false;
      out[t] |= (uint64_t)(s >> 4) << ((bits / 8) * 8);
      out[t + 1] |= (uint64_t)(s & 0xF) << ((bits / 8) * 8);
    }
  if (bits % 4 >= 2)
    for (size_t t = 0; t + 4 <= n; t += 4) {
      if (!nx(s)) return false;
      for (int u = 0; u < 4; u++) out[t + u] |= (uint64_t)((s >> (6 - 2 * u)) & 3) << ((bits / 4) * 4);
    }
  if (bits % 2 >= 1)
    for (size_t t = 0; t + 8 <= n; t += 8) {
      if (!nx(s)) return false;
      for (int u = 0; u < 8; u++) out[t + u] |= (uint64_t)((s >> (7 - u)) & 1) << ((bits / 2) * 2);
    }
  return true;
}

P monomial(int64_t e) {
  P m(CN, 0);
  e = modf_(e, 2 * CN);
  if (e < CN) m[e] = 1;
  else m[e - CN] = TP - 1;
  return m;
}

// gen_gk_b (bfv.rs:105-125), g = 5, two digits of base 2^26
std::vector<P> gen_gk_b(Rng& r, const std::vector<int8_t>& sk) {
  const int64_t m = 2 * CN, ig = inv_mod(5, m);
  P gal(CN);
  for (int i = 0; i < CN; i++) {
    int64_t ni = modf_((int64_t)i * ig, m);
    gal[i] = ni > CN ? modf_(-(int64_t)sk[ni - CN], CQ) : modf_((int64_t)sk[ni], CQ);
  }
  std::vector<P> out;
  for (int d = 0; d < 2; d++) {
    P a = apart(d), e(CN);
    for (int i = 0; i < CN; i++) e[i] = modf_((int64_t)std::llround(r.normal() * SIG), CQ);
    P as = mul_sk(a, sk);
    const int64_t sc = d == 0 ? 1 : (int64_t)((1LL << 26) % CQ);
    P b(CN);
    for (int i = 0; i < CN; i++) b[i] = modf_(modf_(e[i] - as[i], CQ) + (int64_t)(((u128)gal[i] * (uint64_t)sc) % CQ), CQ);
    out.push_back(b);
  }
  return out;
}

thread_local std::string c_err;

}  // namespace

extern "C" {

/* prepare_query_general (pir_wrapper.rs:276-317) with rng = StdRng(rng_seed) */
int dnspir_client_prepare_query(const uint8_t* rng_seed, uint64_t primary_idx, uint64_t secondary_idx,
                                uint32_t primary_order, uint32_t secondary_order, uint8_t* query,
                                uint64_t* query_len, uint8_t* sk_seed_out) {
  if (!rng_seed || !query || !query_len || !sk_seed_out) return DNSPIR_ERR_BAD_ARG;
  if (!(primary_order == CN || primary_order == CN / 2) || secondary_order < 8 || secondary_order > (uint32_t)CN ||
      (secondary_order & (secondary_order - 1)))
    return DNSPIR_ERR_BAD_SHAPE;
  if (primary_idx >= (uint64_t)8 * primary_order || secondary_idx >= secondary_order / 8) return DNSPIR_ERR_BAD_ARG;
  Rng r(rng_seed);
  uint8_t seed[32];
  for (int i = 0; i < 32; i++) seed[i] = (uint8_t)(r.u32() & 0xFFFF);
  Rng skr(seed);
  std::vector<int8_t> sk = gen_sk(skr);
  // enc_double_pir (double_pir.rs:245-289)
  const uint32_t L1 = primary_order < (uint32_t)CN ? primary_order : CN / 2;
  const uint32_t L2 = secondary_order < (uint32_t)CN ? secondary_order : CN / 2;
  const int64_t qbp1 = CN / 2 / L1, qbp2 = CN / 2 / L2;
  const int64_t i = (int64_t)(primary_idx / 8), j = (int64_t)(secondary_idx * 8 + primary_idx % 8);
  std::vector<P> gk = gen_gk_b(r, sk);
  P pq = enc_sym_b(apart(2), r, sk, monomial(i * qbp1)), pqc, sq, sqc;
  if (primary_order == (uint32_t)CN) pqc = enc_sym_b(apart(3), r, sk, monomial(2 * CN - i * qbp1));
  sq = enc_sym_b(apart(4), r, sk, monomial(j * qbp2));
  if (secondary_order == (uint32_t)CN) sqc = enc_sym_b(apart(5), r, sk, monomial(2 * CN - j * qbp2));
  std::vector<uint8_t> out;
  std::vector<uint64_t> enc(CN);
  auto put = [&](const P& p, int bits) {
    for (int k = 0; k < CN; k++) enc[k] = ms_enc(p[k], bits);
    condense(bits, enc, out);
  };
  put(gk[0], 50);
  put(gk[1], 50);
  put(pq, 34);
  if (!pqc.empty()) put(pqc, 34);
  put(sq, 34);
  if (!sqc.empty()) put(sqc, 34);
  memcpy(query, out.data(), out.size());
  *query_len = out.size();
  memcpy(sk_seed_out, seed, 32);
  return DNSPIR_OK;
}

/* process_reply (pir_wrapper.rs:420-440): coeffs = the N coefficients of the entry */
int dnspir_client_process_reply(const uint8_t* reply, uint64_t len, const uint8_t* sk_seed, uint16_t* coeffs) {
  if (!reply || !sk_seed || !coeffs) return DNSPIR_ERR_BAD_ARG;
  Rng skr(sk_seed);
  std::vector<int8_t> sk = gen_sk(skr);
  size_t pos = 0;
  std::vector<uint64_t> raw;
  P part[3];
  for (int j = 0; j < 3; j++) {
    P a(CN), b(CN);
    if (!uncondense(17, CN, reply, len, pos, raw)) return DNSPIR_ERR_BAD_SIZE;
    for (int k = 0; k < CN; k++) a[k] = ms_dec(raw[k], 17);
    if (!uncondense(12, CN, reply, len, pos, raw)) return DNSPIR_ERR_BAD_SIZE;
    for (int k = 0; k < CN; k++) b[k] = ms_dec(raw[k], 12);
    part[j] = dec(sk, a, b);
  }
  // dec_double_pir (double_pir.rs:292-317)
  P a(CN), b(CN);
  for (int k = 0; k < CN; k++) {
    uint64_t v = 0;
    for (int j = 2; j >= 0; j--) v = v * TP + (uint64_t)part[j][k];
    if (v / 4096 >= (1u << 17)) return DNSPIR_ERR_BAD_SIZE;
    b[k] = ms_dec(v % 4096, 12);
    a[k] = ms_dec(v / 4096, 17);
  }
  P m = dec(sk, a, b);
  for (int k = 0; k < CN; k++) coeffs[k] = (uint16_t)m[k];
  return DNSPIR_OK;
}

}  // extern "C"
