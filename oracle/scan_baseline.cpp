// scan_baseline.cpp -- timed CPU baseline of the answer path (test/bench
// infrastructure, part of the oracle library).
//
// orc_scan_baseline times a restatement of main_pir_loop
// (crates/pir/src/base_pir.rs:1085-1247) with the reference's AVX-512 op
// sequence (avx.rs: cvtepi32_epi64 of the 32-bit lanes, mul_epu32, add_epi64,
// the galois scatter into sum_new, a full reduction every 341 iterations) over
// the reference's slab layout (base_pir.rs:312-324), run in parallel over
// (shard, prime, half) like the reference's rayon join/par_iter
// (double_pir.rs:157, base_pir.rs:1007-1064).  The data are random residues:
// the loop's cost does not depend on them.  Without AVX-512 the same loop runs
// in scalar C++ and the caller is told (orc_cpu_has_avx512 == 0).
//
// orc_time_secondary times the oracle's secondary phase at a given secondary
// group order (set_db of the per-query database + its scan; double_pir.rs:195-218).
#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

extern "C" int orc_db_create(int log2n, uint32_t l, int used_seeds, void** out);
extern "C" void orc_db_free(void* d);
extern "C" int orc_db_set_db(void* d, const uint16_t* entries);
extern "C" int orc_db_perform_pir_split(void* d, const int64_t* qry_b, const int64_t* qry_conj_b, const int64_t* gk_b,
                                        int64_t* out);
extern "C" int orc_db_get_a(void* d, int64_t* out);
extern "C" int orc_db_set_db_vec(void* d, const uint16_t* entries);
extern "C" int orc_db_perform_pir_split_vec(void* d, const int64_t* qry_b, const int64_t* qry_conj_b,
                                            const int64_t* gk_b, int64_t* out);

namespace {

const uint64_t BQ1 = (1ull << 26) - (1ull << 12) + 1;
const uint64_t BQ2 = (1ull << 25) - (1ull << 12) + 1;

struct Unit {
  const uint32_t* te;
  const uint32_t* g0;
  const uint32_t* g1;
  const uint32_t* qry;  // N x 8 lanes (compressed)
  const uint32_t* gk0;
  const uint32_t* gk1;
  uint64_t p;
};

__attribute__((target("avx512f"))) void loop_avx512(const Unit& u, size_t N, size_t len, size_t reduce_every,
                                                    const uint32_t* gal, __m512i* sum, __m512i* sum_new) {
  size_t index = 0;
  for (size_t io = 0; io < len; io += reduce_every) {
    const size_t cnt = std::min(len - io, reduce_every);
    for (size_t ii = 0; ii < cnt; ii++) {
      for (size_t j = 0; j < N; j++) {
        const size_t e = (index + j) * 8;
        __m512i cur = sum[j];
        __m512i x = _mm512_cvtepi32_epi64(_mm256_load_si256((const __m256i*)(u.g0 + e)));
        __m512i y = _mm512_cvtepi32_epi64(_mm256_load_si256((const __m256i*)(u.gk0 + j * 8)));
        cur = _mm512_add_epi64(cur, _mm512_mul_epu32(x, y));
        x = _mm512_cvtepi32_epi64(_mm256_load_si256((const __m256i*)(u.g1 + e)));
        y = _mm512_cvtepi32_epi64(_mm256_load_si256((const __m256i*)(u.gk1 + j * 8)));
        cur = _mm512_add_epi64(cur, _mm512_mul_epu32(x, y));
        x = _mm512_cvtepi32_epi64(_mm256_load_si256((const __m256i*)(u.te + e)));
        y = _mm512_cvtepi32_epi64(_mm256_load_si256((const __m256i*)(u.qry + j * 8)));
        cur = _mm512_add_epi64(cur, _mm512_mul_epu32(x, y));
        sum_new[gal[j]] = cur;
      }
      index += N;
      std::swap(sum, sum_new);
    }
    for (size_t j = 0; j < N; j++) {
      alignas(64) uint64_t v[8];
      _mm512_store_si512((void*)v, sum[j]);
      for (int k = 0; k < 8; k++) v[k] %= u.p;
      sum[j] = _mm512_load_si512((const void*)v);
    }
  }
}

void loop_scalar(const Unit& u, size_t N, size_t len, size_t reduce_every, const uint32_t* gal, uint64_t* sum,
                 uint64_t* sum_new) {
  size_t index = 0;
  for (size_t io = 0; io < len; io += reduce_every) {
    const size_t cnt = std::min(len - io, reduce_every);
    for (size_t ii = 0; ii < cnt; ii++) {
      for (size_t j = 0; j < N; j++) {
        const size_t e = (index + j) * 8;
        uint64_t* d = sum_new + gal[j] * 8;
        const uint64_t* s = sum + j * 8;
        for (int k = 0; k < 8; k++)
          d[k] = s[k] + (uint64_t)u.g0[e + k] * u.gk0[j * 8 + k] + (uint64_t)u.g1[e + k] * u.gk1[j * 8 + k] +
                 (uint64_t)u.te[e + k] * u.qry[j * 8 + k];
      }
      index += N;
      std::swap(sum, sum_new);
    }
    for (size_t j = 0; j < N * 8; j++) sum[j] %= u.p;
  }
}

bool has_avx512() { return __builtin_cpu_supports("avx512f"); }

}  // namespace

extern "C" {

int orc_cpu_has_avx512() { return has_avx512() ? 1 : 0; }

// Seconds per pass of main_pir_loop over `shards` shards of group order l
// (both primes, both halves when l == N), using `threads` threads (0 = all).
double orc_scan_baseline(int log2n, uint32_t l, uint32_t shards, int threads, int reps, int* used_threads) {
  const size_t N = (size_t)1 << log2n;
  const size_t L = l < N ? l : N / 2;
  const int H = l == N ? 2 : 1;
  const size_t arr = L * N * 8;  // u32 words of one array
  int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (used_threads) *used_threads = nt;
  // slabs: shards x 2 primes x H halves x 3 arrays, 64-byte aligned
  const size_t per_unit = 3 * arr;
  const size_t units = (size_t)shards * 2 * H;
  uint32_t* slab = (uint32_t*)aligned_alloc(64, units * per_unit * 4);
  if (!slab) return -1.0;
  {
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
      th.emplace_back([&, t]() {
        uint64_t x = 0x9e3779b97f4a7c15ull * (t + 1);
        const size_t total = units * per_unit;
        for (size_t i = (size_t)t * (total / nt); i < (t == nt - 1 ? total : (size_t)(t + 1) * (total / nt)); i++) {
          x ^= x << 13;
          x ^= x >> 7;
          x ^= x << 17;
          slab[i] = (uint32_t)(x % BQ2);
        }
      });
    for (auto& t : th) t.join();
  }
  std::vector<uint32_t> qv(4 * N * 8);
  for (size_t i = 0; i < qv.size(); i++) qv[i] = (uint32_t)((i * 2654435761u) % BQ2);
  std::vector<uint32_t> gal(N);
  for (size_t i = 0; i < N; i++) gal[i] = (uint32_t)((i * 5 + 3) % N);  // any permutation (cost only)
  const size_t reduce_every = 341;  // base_pir.rs:1002-1005 for q1 = 2^26 - 2^12 + 1
  const bool avx = has_avx512();
  double best = 1e30;
  for (int r = 0; r < (reps > 0 ? reps : 1); r++) {
    std::atomic<size_t> next(0);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
      th.emplace_back([&]() {
        uint64_t* bufs = (uint64_t*)aligned_alloc(64, 2 * N * 8 * 8);
        for (;;) {
          size_t k = next.fetch_add(1);
          if (k >= units) break;
          const uint32_t* base = slab + k * per_unit;
          Unit u{base, base + arr, base + 2 * arr, qv.data(), qv.data() + 2 * N * 8, qv.data() + 3 * N * 8,
                 (k / H) % 2 ? BQ2 : BQ1};
          memset(bufs, 0, 2 * N * 8 * 8);
          if (avx)
            loop_avx512(u, N, L, reduce_every, gal.data(), (__m512i*)bufs, (__m512i*)(bufs + N * 8));
          else
            loop_scalar(u, N, L, reduce_every, gal.data(), bufs, bufs + N * 8);
        }
        free(bufs);
      });
    for (auto& t : th) t.join();
    double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    best = std::min(best, s);
  }
  free(slab);
  return best;
}

// ---- one whole query on the CPU, timed for real (the reference arm of the
// bench): the primary scan of every logical shard (shard k reads distinct slab
// k mod distinct, as bench_wrapped_pir's preprocessed-db-count does,
// pir_wrapper.rs:578), run in parallel over (shard, prime, half) units on all
// threads, then the secondary phase (set_db of the per-query database and its
// scan, double_pir.rs:195-218) on the oracle library's vectorised restatement
// (the scalar oracle without AVX-512).
struct orc_bench {
  int log2n = 11;
  uint32_t l1 = 0, l2 = 0, shards = 0, distinct = 0;
  size_t N = 0, L = 0, arr = 0;
  int H = 1;
  uint32_t* slab = nullptr;  // distinct x 2 primes x H halves x 3 arrays
  std::vector<uint32_t> qv, gal;
  std::vector<uint16_t> sec_entries;
};

orc_bench* orc_bench_new(int log2n, uint32_t l1, uint32_t l2, uint32_t shards, uint32_t distinct) {
  orc_bench* b = new orc_bench();
  b->log2n = log2n;
  b->l1 = l1;
  b->l2 = l2;
  b->shards = shards;
  b->distinct = std::max<uint32_t>(1, std::min(distinct, shards));
  b->N = (size_t)1 << log2n;
  b->L = l1 < b->N ? l1 : b->N / 2;
  b->H = l1 == b->N ? 2 : 1;
  b->arr = b->L * b->N * 8;
  const size_t words = (size_t)b->distinct * 2 * b->H * 3 * b->arr;
  b->slab = (uint32_t*)aligned_alloc(64, words * 4);
  if (!b->slab) {
    delete b;
    return nullptr;
  }
  const int nt = std::max(1, (int)std::thread::hardware_concurrency());
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([&, t]() {
      uint64_t x = 0x9e3779b97f4a7c15ull * (t + 1);
      for (size_t i = (size_t)t * (words / nt); i < (t == nt - 1 ? words : (size_t)(t + 1) * (words / nt)); i++) {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        b->slab[i] = (uint32_t)(x % BQ2);
      }
    });
  for (auto& t : th) t.join();
  b->qv.resize(4 * b->N * 8);
  for (size_t i = 0; i < b->qv.size(); i++) b->qv[i] = (uint32_t)((i * 2654435761u) % BQ2);
  b->gal.resize(b->N);
  for (size_t i = 0; i < b->N; i++) b->gal[i] = (uint32_t)((i * 5 + 3) % b->N);  // any permutation (cost only)
  b->sec_entries.resize((size_t)8 * l2 * b->N);
  for (size_t i = 0; i < b->sec_entries.size(); i++) b->sec_entries[i] = (uint16_t)((i * 2654435761u) % 1025);
  return b;
}

void orc_bench_free(orc_bench* b) {
  if (!b) return;
  free(b->slab);
  delete b;
}

// One query: seconds of the primary scan and of the secondary phase.
// *scan_threads receives the threads that took scan units.
int orc_bench_step(orc_bench* b, int threads, double* scan_s, double* sec_s, int* scan_threads) {
  const size_t units = (size_t)b->shards * 2 * b->H;
  int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min<int>(nt, (int)units));
  if (scan_threads) *scan_threads = nt;
  const bool avx = has_avx512();
  const size_t per_unit = 3 * b->arr;
  std::atomic<size_t> next(0);
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([&]() {
      uint64_t* bufs = (uint64_t*)aligned_alloc(64, 2 * b->N * 8 * 8);
      for (;;) {
        const size_t k = next.fetch_add(1);
        if (k >= units) break;
        // unit k = (logical shard, prime, half); logical shard s reads distinct slab s mod distinct
        const size_t shard = k / (2 * b->H), ph = k % (2 * b->H);
        const uint32_t* base = b->slab + ((shard % b->distinct) * 2 * b->H + ph) * per_unit;
        Unit u{base, base + b->arr, base + 2 * b->arr, b->qv.data(), b->qv.data() + 2 * b->N * 8,
               b->qv.data() + 3 * b->N * 8, (ph / b->H) % 2 ? BQ2 : BQ1};
        memset(bufs, 0, 2 * b->N * 8 * 8);
        if (avx)
          loop_avx512(u, b->N, b->L, 341, b->gal.data(), (__m512i*)bufs, (__m512i*)(bufs + b->N * 8));
        else
          loop_scalar(u, b->N, b->L, 341, b->gal.data(), bufs, bufs + b->N * 8);
      }
      free(bufs);
    });
  for (auto& t : th) t.join();
  auto t1 = std::chrono::steady_clock::now();
  void* db = nullptr;
  int rc = orc_db_create(b->log2n, b->l2, 1, &db);
  std::vector<int64_t> q(8 * b->N, 1), gk(16 * b->N, 1), out(8 * b->N);
  // the secondary phase on the vectorised restatement (8 lanes per AVX-512
  // register and the reference's thread split), else on the scalar oracle
  if (!rc) rc = avx ? orc_db_set_db_vec(db, b->sec_entries.data()) : orc_db_set_db(db, b->sec_entries.data());
  if (!rc) rc = orc_db_get_a(db, out.data());
  if (!rc)
    rc = avx ? orc_db_perform_pir_split_vec(db, q.data(), b->l2 == b->N ? q.data() : nullptr, gk.data(), out.data())
             : orc_db_perform_pir_split(db, q.data(), b->l2 == b->N ? q.data() : nullptr, gk.data(), out.data());
  auto t2 = std::chrono::steady_clock::now();
  if (db) orc_db_free(db);
  if (scan_s) *scan_s = std::chrono::duration<double>(t1 - t0).count();
  if (sec_s) *sec_s = std::chrono::duration<double>(t2 - t1).count();
  return rc;
}

// Seconds of one secondary phase at N = 2^log2n and secondary order l2:
// set_db of the per-query database (8 l2 entries) and perform_pir_split.
double orc_time_secondary(int log2n, uint32_t l2) {
  const size_t N = (size_t)1 << log2n;
  void* db = nullptr;
  if (orc_db_create(log2n, l2, 1, &db)) return -1.0;
  std::vector<uint16_t> entries((size_t)8 * l2 * N);
  for (size_t i = 0; i < entries.size(); i++) entries[i] = (uint16_t)((i * 2654435761u) % 1025);
  std::vector<int64_t> q(8 * N, 1), gk(16 * N, 1), out(8 * N);
  auto t0 = std::chrono::steady_clock::now();
  int rc = orc_db_set_db(db, entries.data());
  if (!rc) rc = orc_db_get_a(db, out.data());
  if (!rc) rc = orc_db_perform_pir_split(db, q.data(), l2 == N ? q.data() : nullptr, gk.data(), out.data());
  double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  orc_db_free(db);
  return rc ? -1.0 : s;
}

}  // extern "C"
