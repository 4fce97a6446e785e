// api.cu -- host side of the C ABI in include/dnspir.h: device context
// (twiddles, expanded a-parts), shards (PIRDatabase), fleets and the
// two-level answer pipeline (perform_batched_double_pir, double_pir.rs:126-228;
// process_queries, pir_wrapper.rs:349-409).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "dnspir.h"
#include "kernels.cuh"

using namespace dnspir;

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;
static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
#define CK(call)                                                                                           \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess) {                                                                               \
      cudaGetLastError();                                                                                  \
      return fail(e_ == cudaErrorMemoryAllocation ? DNSPIR_ERR_OOM : DNSPIR_ERR_CUDA,                      \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                                     \
    }                                                                                                      \
  } while (0)
#define CKR(expr)             \
  do {                        \
    int r_ = (expr);          \
    if (r_ != DNSPIR_OK) return r_; \
  } while (0)

// ------------------------------------------------------------- host maths
typedef unsigned __int128 u128;
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
static uint64_t invmod(uint64_t a, uint64_t p) { return powmod(a, p - 2, p); }  // p prime
static uint32_t brv_host(uint32_t i, int logn) {
  uint32_t r = 0;
  for (int b = 0; b < logn; b++)
    if (i >> b & 1) r |= 1u << (logn - 1 - b);
  return r;
}
// least quadratic non-residue g; g^((p-1)/2N) is a primitive 2N-th root of unity
static uint64_t prim_root_2n(uint64_t p, uint64_t two_n) {
  for (uint64_t g = 2;; g++)
    if (powmod(g, (p - 1) / 2, p) != 1) return powmod(g, (p - 1) / two_n, p);
}

namespace dnspir {
CrtConst host_crt_const() {
  CrtConst c;
  c.q2inv1 = (uint32_t)invmod(P2 % P1, P1);
  c.q1inv2 = (uint32_t)invmod(P1 % P2, P2);
  return c;
}
}  // namespace dnspir

// ---- seed expansion (bfv.rs:46-49).  The six a-parts are drawn from a
// ChaCha12 word stream keyed by the 32-byte seed (rand_chacha 0.3.1 StdRng:
// 64-bit block counter in words 12-13, stream 0, four blocks per refill,
// rand_core's next_u64 = low word then high word); each coefficient is the
// low 51 bits of next_u64, redrawn while >= q.  The seeds are the SHA-3
// hashes of base_pir.rs:64-71.
namespace {
const uint8_t SEEDS[6][32] = {
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

struct ChaCha12 {
  uint32_t key[8];
  uint64_t ctr = 0;
  uint32_t buf[64];
  int idx = 64;
  explicit ChaCha12(const uint8_t* seed) {
    for (int i = 0; i < 8; i++) memcpy(&key[i], seed + 4 * i, 4);  // little endian host
  }
  static uint32_t rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
  void block(uint64_t c, uint32_t* out) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                      key[4],      key[5],      key[6],      key[7],      (uint32_t)c, (uint32_t)(c >> 32), 0, 0};
    uint32_t x[16];
    memcpy(x, s, sizeof(x));
    auto qr = [&](int a, int b, int c2, int d) {
      x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 16);
      x[c2] += x[d]; x[b] = rotl(x[b] ^ x[c2], 12);
      x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 8);
      x[c2] += x[d]; x[b] = rotl(x[b] ^ x[c2], 7);
    };
    for (int r = 0; r < 6; r++) {
      qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
      qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
    }
    for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
  }
  void refill() {
    for (int b = 0; b < 4; b++) block(ctr + b, buf + 16 * b);
    ctr += 4;
    idx = 0;
  }
  uint64_t next_u64() {
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
};

void expand(uint32_t n, const uint8_t* seed, uint64_t* out) {
  ChaCha12 r(seed);
  const uint64_t mask = (1ull << 51) - 1;
  for (uint32_t i = 0; i < n; i++) {
    uint64_t x;
    do x = r.next_u64() & mask;
    while (x >= QQ);
    out[i] = x;
  }
}
}  // namespace

// ------------------------------------------------------------ device context
struct DeviceCtx {
  int device = -1;
  uint32_t* tables = nullptr;
  NttTables T;
  uint32_t* consts[LOG2_N_MAX + 1] = {};  // a-parts in NTT form: [6][2][N], bit-reversed positions
  uint32_t* galb[LOG2_N_MAX + 1] = {};
  std::mutex mu;
};

static std::mutex g_ctx_mu;
static DeviceCtx* g_ctx[64];

static int build_tables(DeviceCtx& c) {
  const int n = N_MAX;
  std::vector<uint32_t> h(8 * n);
  for (int pi = 0; pi < 2; pi++) {
    const uint64_t p = pi ? P2 : P1;
    const uint64_t zeta = prim_root_2n(p, 2 * n);
    const uint64_t psi = invmod(zeta, p);
    for (int k = 0; k < n; k++) {
      const uint32_t e = brv_host(k, LOG2_N_MAX);
      const uint64_t f = powmod(psi, e, p), iv = powmod(zeta, e, p);
      h[(0 + pi) * n + k] = (uint32_t)f;
      h[(2 + pi) * n + k] = (uint32_t)(((u128)f << 32) / p);
      h[(4 + pi) * n + k] = (uint32_t)iv;
      h[(6 + pi) * n + k] = (uint32_t)(((u128)iv << 32) / p);
    }
    for (int lg = 0; lg <= LOG2_N_MAX; lg++) {
      const uint64_t ni = invmod((1ull << lg) % p, p);
      c.T.ninv[pi][lg] = (uint32_t)ni;
      c.T.ninvq[pi][lg] = (uint32_t)(((u128)ni << 32) / p);
    }
  }
  CK(cudaMalloc(&c.tables, h.size() * 4));
  CK(cudaMemcpy(c.tables, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
  for (int pi = 0; pi < 2; pi++) {
    c.T.fw[pi] = c.tables + (0 + pi) * n;
    c.T.fwq[pi] = c.tables + (2 + pi) * n;
    c.T.iw[pi] = c.tables + (4 + pi) * n;
    c.T.iwq[pi] = c.tables + (6 + pi) * n;
  }
  return DNSPIR_OK;
}

static int get_ctx(int device, DeviceCtx** out) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(DNSPIR_ERR_CUDA, "no CUDA device available (this library has no CPU path)");
  }
  if (device < 0 || device >= count || device >= 64) return fail(DNSPIR_ERR_BAD_ARG, "device index out of range");
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (!g_ctx[device]) {
    CK(cudaSetDevice(device));
    std::unique_ptr<DeviceCtx> c(new DeviceCtx());
    c->device = device;
    CKR(build_tables(*c));
    g_ctx[device] = c.release();
  }
  *out = g_ctx[device];
  return DNSPIR_OK;
}

// a-parts and the sigma_5 position map for ring dimension 2^log2n
static int ctx_consts(DeviceCtx* c, int log2n) {
  std::lock_guard<std::mutex> lk(c->mu);
  if (c->consts[log2n]) return DNSPIR_OK;
  const uint32_t n = 1u << log2n;
  std::vector<uint64_t> ap(6 * (size_t)n);
  for (int s = 0; s < 6; s++) expand(n, SEEDS[s], ap.data() + (size_t)s * n);
  uint64_t* dz = nullptr;
  uint32_t* dc = nullptr;
  uint32_t* dg = nullptr;
  CK(cudaMalloc(&dz, ap.size() * 8));
  CK(cudaMalloc(&dc, (size_t)6 * 2 * n * 4));
  CK(cudaMalloc(&dg, (size_t)n * 4));
  CK(cudaMemcpy(dz, ap.data(), ap.size() * 8, cudaMemcpyHostToDevice));
  launch_ring_to_ntt(dz, 6, nullptr, dc, log2n, c->T, 0);
  CK(cudaGetLastError());
  std::vector<uint32_t> gb(n);
  const uint32_t two_n = 2 * n;
  uint32_t inv5 = 1;
  for (uint32_t x = 1; x < two_n; x += 2)
    if ((5 * x) % two_n == 1) inv5 = x;
  for (uint32_t pos = 0; pos < n; pos++) {
    const uint32_t j = brv_host(pos, log2n);
    const uint32_t g = (uint32_t)(((uint64_t)inv5 * (2 * j + 1)) % two_n);
    gb[pos] = brv_host((g - 1) / 2, log2n);
  }
  CK(cudaMemcpy(dg, gb.data(), n * 4, cudaMemcpyHostToDevice));
  CK(cudaDeviceSynchronize());
  CK(cudaFree(dz));
  device_pow5(log2n, false);
  device_pow5(log2n, true);
  c->galb[log2n] = dg;
  c->consts[log2n] = dc;
  return DNSPIR_OK;
}

static ChainConsts chain_consts(DeviceCtx* c, int log2n, int used_seeds) {
  const size_t n2 = (size_t)2 << log2n;
  ChainConsts cc;
  cc.gka = c->consts[log2n];
  cc.qa = c->consts[log2n] + (2 + 2 * used_seeds) * n2;
  cc.galb = c->galb[log2n];
  return cc;
}

// RAII device buffer
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DBuf() {
    if (p) cudaFree(p);
  }
  int ensure(size_t b) {
    if (b <= bytes) return DNSPIR_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    CK(cudaMalloc(&p, b));
    bytes = b;
    return DNSPIR_OK;
  }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

static int check_group(uint32_t log2n, uint32_t l) {
  if (log2n < 3 || log2n > LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_SHAPE, "log2_n must be in [3, 11]");
  const uint32_t n = 1u << log2n;
  if (l == 0 || n % l != 0) return fail(DNSPIR_ERR_BAD_SHAPE, "group order must divide N");
  if (l != n && 2 * l > n) return fail(DNSPIR_ERR_BAD_SHAPE, "a subgroup order must be at most N/2");
  if (2ull * TPLAIN * n >= P1) return fail(DNSPIR_ERR_BAD_SHAPE, "max_coeff >= q1");
  return DNSPIR_OK;
}

// -------------------------------------------------------------- shard state
// Device buffers shared by set_db and the secondary phase.
struct EncodeWs {
  DBuf A, Ahat, in16, a_out, slab_ptrs;
};

// Encodes `count` shards' entries (device u16, one shard after another) into
// their slabs, runs the preprocessing chain and the a-part finalisation.
static int preprocess_shards(DeviceCtx* c, const Group& g, int used_seeds, uint32_t* const* slabs_host, int count,
                             const uint16_t* entries_dev, uint64_t* a_zq, uint32_t* a_ms, EncodeWs& ws,
                             cudaStream_t st) {
  const size_t per_shard = (size_t)SIMD * g.l * g.n;
  CKR(ws.A.ensure((size_t)g.l * SIMD * g.n * 4));
  CKR(ws.Ahat.ensure((size_t)g.H * g.L * SIMD * g.n * 4));
  CKR(ws.a_out.ensure((size_t)count * g.H * SIMD * 2 * g.n * 4));
  CKR(ws.slab_ptrs.ensure((size_t)count * sizeof(uint32_t*)));
  for (int s = 0; s < count; s++) {
    launch_encode_cols(entries_dev + s * per_shard, ws.A.as<uint32_t>(), g, g.l, SIMD, c->T, st);
    launch_encode_rows(ws.A.as<uint32_t>(), ws.Ahat.as<uint32_t>(), g, g.l, SIMD, c->T, st);
    launch_encode_lift(ws.Ahat.as<uint32_t>(), slabs_host[s], g, SIMD, 0, c->T, st);
  }
  CK(cudaMemcpyAsync(ws.slab_ptrs.p, slabs_host, (size_t)count * sizeof(uint32_t*), cudaMemcpyHostToDevice, st));
  launch_primary_chain(ws.slab_ptrs.as<uint32_t*>(), count, ws.a_out.as<uint32_t>(), g,
                       chain_consts(c, g.log2n, used_seeds), c->T, st);
  launch_primary_finalize(ws.a_out.as<uint32_t>(), count, a_zq, a_ms, g, c->T, st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return DNSPIR_OK;
}

struct dnspir_db {
  int device = 0;
  DeviceCtx* ctx = nullptr;
  Group g;
  int used_seeds = 0;
  bool ready = false;
  cudaStream_t st = nullptr;
  uint32_t* slab = nullptr;
  DBuf a_zq, a_ms, qz, qlane, part, out, slab_ptr;
  EncodeWs ws;
  std::mutex mu;
  ~dnspir_db() {
    if (slab) cudaFree(slab);
    if (st) cudaStreamDestroy(st);
  }
};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    cudaGetDevice(&prev);
    cudaSetDevice(d);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// RAII pinned host buffer (asynchronous copies need page-locked memory)
struct HBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~HBuf() {
    if (p) cudaFreeHost(p);
  }
  int ensure(size_t b) {
    if (b <= bytes) return DNSPIR_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    CK(cudaMallocHost(&p, b));
    bytes = b;
    return DNSPIR_OK;
  }
};

// ------------------------------------------------------------------ fleet
// Buffers of one query in flight.  Two slots alternate by query parity so that
// the primary phase of query k+1 (main stream) overlaps the secondary phase of
// query k (secondary stream); events order the reuse of a slot.
struct QSlot {
  DBuf qbytes, qnat, qbrv, sec_in, reply_dev;
  HBuf qpin;  // host staging of the query bytes
  cudaEvent_t prim_done = nullptr, sec_done = nullptr;
  bool sec_pending = false, prim_recorded = false;
};

struct dnspir_fleet {
  int device = 0;
  DeviceCtx* ctx = nullptr;
  Group g1, g2;
  uint32_t S = 0, D = 0;
  cudaStream_t own = nullptr, st = nullptr, sec = nullptr;
  std::vector<uint32_t*> slabs;
  std::vector<bool> ready;
  DBuf slabs_dev, distinct_dev, a_zq, a_ms;
  EncodeWs ws;
  QSlot slot[2];
  DBuf part, secE, chain_out, qzq, reply_zq;  // used by one stream at a time
  HBuf rpin;                                  // host staging of the replies of one call
  int R = 1;
  std::vector<cudaEvent_t> tev;  // 6 timing events per query of the last call
  std::vector<int> tev_ok;
  uint32_t tev_n = 0;
  std::mutex mu;
  ~dnspir_fleet() {
    for (uint32_t* s : slabs)
      if (s) cudaFree(s);
    for (auto& e : tev)
      if (e) cudaEventDestroy(e);
    for (auto& s : slot) {
      if (s.prim_done) cudaEventDestroy(s.prim_done);
      if (s.sec_done) cudaEventDestroy(s.sec_done);
    }
    if (sec) cudaStreamDestroy(sec);
    if (own) cudaStreamDestroy(own);
  }
};

// Read-only view of a shard for the no-allocation entry point (noalloc.cu).
namespace dnspir {
int db_view(const dnspir_db* db, DbView* out) {
  out->device = db->device;
  out->ready = db->ready;
  out->g = db->g;
  out->slab = db->slab;
  out->T = db->ctx->T;
  return DNSPIR_OK;
}
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace dnspir

// ============================================================== C ABI
extern "C" {

const char* dnspir_last_error(void) { return g_err.c_str(); }
const char* dnspir_version(void) { return "dnspir_b200 0.1 (sm_100a)"; }

int dnspir_choose_secondary_order(uint32_t num_shards, uint32_t* secondary_order) {
  const uint32_t n = N_MAX;
  if (!secondary_order) return fail(DNSPIR_ERR_BAD_ARG, "null output");
  if (num_shards > n / SIMD) return fail(DNSPIR_ERR_BAD_SHAPE, "more shards than one fleet can address");
  uint32_t lg = 0;
  while ((1u << lg) < num_shards) lg++;
  *secondary_order = (uint32_t)SIMD << lg;
  return DNSPIR_OK;
}

int dnspir_get_database_shape(uint64_t num_entries, uint32_t* primary_order, uint32_t* secondary_order,
                              uint32_t* num_shards) {
  const uint64_t n = N_MAX;
  if (!primary_order || !secondary_order || !num_shards) return fail(DNSPIR_ERR_BAD_ARG, "null output");
  if (num_entries < 1 || num_entries > n * n) return fail(DNSPIR_ERR_BAD_SHAPE, "num_entries must be in [1, N^2]");
  const uint64_t half_max = n * n / 16;  // HALF_SIZE_PRIMARY_MAX_ENTRIES (pir_wrapper.rs:188)
  const uint32_t l1 = num_entries <= half_max ? (uint32_t)(n / 2) : (uint32_t)n;
  const uint32_t shards = (uint32_t)((num_entries + SIMD * (uint64_t)l1 - 1) / (SIMD * (uint64_t)l1));
  CKR(dnspir_choose_secondary_order(shards, secondary_order));
  *primary_order = l1;
  *num_shards = shards;
  return DNSPIR_OK;
}

uint64_t dnspir_required_memory_general(uint32_t log2_n, uint32_t group_order) {
  return (uint64_t)(GK_DIGITS + 1) * 2 * (1ull << log2_n) * group_order;
}

uint64_t dnspir_query_bytes(uint32_t primary_order, uint32_t secondary_order) {
  const uint64_t n = N_MAX;
  uint64_t b = 2 * n * GK_BITS / 8 + n * PQ_BITS / 8 + n * SQ_BITS / 8;
  if (primary_order == n) b += n * PQ_BITS / 8;
  if (secondary_order == n) b += n * SQ_BITS / 8;
  return b;
}
uint64_t dnspir_reply_bytes(void) { return (uint64_t)CTXT_PARTS * N_MAX * (SEC_A_BITS + SEC_B_BITS) / 8; }

int dnspir_expand_seed(uint32_t log2_n, int which, uint64_t* out) {
  if (!out || which < 0 || which >= 6 || log2_n < 1 || log2_n > LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_ARG, "bad argument");
  expand(1u << log2_n, SEEDS[which], out);
  return DNSPIR_OK;
}

int dnspir_pack_payloads(int device, const uint8_t* bytes, uint64_t entries, uint16_t* coeffs) {
  if (!bytes || !coeffs) return fail(DNSPIR_ERR_BAD_ARG, "null buffer");
  DeviceCtx* c = nullptr;
  CKR(get_ctx(device, &c));
  DeviceGuard dg(device);
  launch_pack_bytes(bytes, coeffs, entries, LOG2_N_MAX, 0);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  return DNSPIR_OK;
}

// ---------------------------------------------------------------- shards
int dnspir_db_create(int device, uint32_t log2_n, uint32_t group_order, int used_seeds, dnspir_db** out) {
  if (!out) return fail(DNSPIR_ERR_BAD_ARG, "null output");
  *out = nullptr;
  CKR(check_group(log2_n, group_order));
  if (used_seeds != 0 && used_seeds != 1) return fail(DNSPIR_ERR_BAD_ARG, "used_seeds must be 0 or 1");
  DeviceCtx* c = nullptr;
  CKR(get_ctx(device, &c));
  DeviceGuard dg(device);
  CKR(ctx_consts(c, log2_n));
  std::unique_ptr<dnspir_db> d(new dnspir_db());
  d->device = device;
  d->ctx = c;
  d->g = make_group(log2_n, group_order);
  d->used_seeds = used_seeds;
  CK(cudaStreamCreateWithFlags(&d->st, cudaStreamNonBlocking));
  CK(cudaMalloc(&d->slab, slab_words(d->g) * 4));
  CKR(d->a_zq.ensure((size_t)SIMD * d->g.n * 8));
  CKR(d->a_ms.ensure((size_t)SIMD * d->g.n * 4));
  *out = d.release();
  return DNSPIR_OK;
}

int dnspir_db_set_db(dnspir_db* db, const uint16_t* entries, uint64_t count, int entries_on_device) {
  if (!db || !entries) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(db->mu);
  const uint64_t want = (uint64_t)SIMD * db->g.l * db->g.n;
  if (count != want) return fail(DNSPIR_ERR_BAD_SIZE, "set_db needs exactly 8 * group_order entries of N coefficients");
  DeviceGuard dg(db->device);
  const uint16_t* src = entries;
  if (!entries_on_device) {
    CKR(db->ws.in16.ensure(want * 2));
    CK(cudaMemcpyAsync(db->ws.in16.p, entries, want * 2, cudaMemcpyHostToDevice, db->st));
    src = db->ws.in16.as<uint16_t>();
  }
  uint32_t* slabs[1] = {db->slab};
  db->ready = false;
  CKR(preprocess_shards(db->ctx, db->g, db->used_seeds, slabs, 1, src, db->a_zq.as<uint64_t>(),
                        db->a_ms.as<uint32_t>(), db->ws, db->st));
  db->ready = true;
  return DNSPIR_OK;
}

int dnspir_db_get_a(dnspir_db* db, uint64_t* out) {
  if (!db || !out) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(db->mu);
  if (!db->ready) return fail(DNSPIR_ERR_NOT_READY, "database not preprocessed");
  DeviceGuard dg(db->device);
  CK(cudaMemcpy(out, db->a_zq.p, (size_t)SIMD * db->g.n * 8, cudaMemcpyDeviceToHost));
  return DNSPIR_OK;
}

static bool reduced(const uint64_t* v, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (v[i] >= QQ) return false;
  return true;
}

int dnspir_db_perform_pir_split(dnspir_db* db, const uint64_t* qry_b, const uint64_t* qry_conj_b, const uint64_t* gk_b,
                                uint64_t* out_b) {
  if (!db || !qry_b || !gk_b || !out_b) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(db->mu);
  if (!db->ready) return fail(DNSPIR_ERR_NOT_READY, "database not preprocessed");
  const Group& g = db->g;
  if ((g.H == 2) != (qry_conj_b != nullptr))
    return fail(DNSPIR_ERR_BAD_SHAPE, "conjugate query must be given exactly when the group requires it");
  const size_t n = g.n;
  // [lane][v][N], v = qry, qry_conj, gk0, gk1
  std::vector<uint64_t> z((size_t)SIMD * 4 * n, 0);
  for (int k = 0; k < SIMD; k++) {
    memcpy(&z[((size_t)k * 4 + 0) * n], qry_b + k * n, n * 8);
    if (qry_conj_b) memcpy(&z[((size_t)k * 4 + 1) * n], qry_conj_b + k * n, n * 8);
    memcpy(&z[((size_t)k * 4 + 2) * n], gk_b + (2 * k) * n, n * 8);
    memcpy(&z[((size_t)k * 4 + 3) * n], gk_b + (2 * k + 1) * n, n * 8);
  }
  if (!reduced(z.data(), z.size())) return fail(DNSPIR_ERR_BAD_ARG, "ring element coefficients must be below q");
  DeviceGuard dg(db->device);
  const int R = scan_chunks(g, 1);
  CKR(db->qz.ensure(z.size() * 8));
  CKR(db->qlane.ensure(z.size() * 2 * 4));
  CKR(db->part.ensure((size_t)g.H * R * 2 * n * SIMD * 4));
  CKR(db->out.ensure((size_t)SIMD * n * 8));
  CK(cudaMemcpyAsync(db->qz.p, z.data(), z.size() * 8, cudaMemcpyHostToDevice, db->st));
  launch_ring_to_ntt(db->qz.as<uint64_t>(), SIMD * 4, db->qlane.as<uint32_t>(), nullptr, g.log2n, db->ctx->T, db->st);
  launch_scan_lanes(db->slab, db->qlane.as<uint32_t>(), db->part.as<uint32_t>(), g, R, db->st);
  launch_epilogue_zq(db->part.as<uint32_t>(), g.H * R, db->out.as<uint64_t>(), g, db->ctx->T, db->st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out_b, db->out.p, (size_t)SIMD * n * 8, cudaMemcpyDeviceToHost, db->st));
  CK(cudaStreamSynchronize(db->st));
  return DNSPIR_OK;
}

int dnspir_db_destroy(dnspir_db* db) {
  if (!db) return DNSPIR_OK;
  DeviceGuard dg(db->device);
  delete db;
  return DNSPIR_OK;
}

// ---------------------------------------------------------------- fleets
int dnspir_fleet_create_general(int device, uint32_t log2_n, uint32_t primary_order, uint32_t secondary_order,
                                uint32_t num_shards, uint32_t num_distinct, dnspir_fleet** out) {
  if (!out) return fail(DNSPIR_ERR_BAD_ARG, "null output");
  *out = nullptr;
  CKR(check_group(log2_n, primary_order));
  CKR(check_group(log2_n, secondary_order));
  if (num_shards == 0 || num_distinct == 0 || num_distinct > num_shards)
    return fail(DNSPIR_ERR_BAD_ARG, "need 1 <= num_distinct <= num_shards");
  if ((uint64_t)num_shards * SIMD > secondary_order)
    return fail(DNSPIR_ERR_BAD_SHAPE, "secondary group too small for the number of shards (double_pir.rs:152)");
  DeviceCtx* c = nullptr;
  CKR(get_ctx(device, &c));
  DeviceGuard dg(device);
  CKR(ctx_consts(c, log2_n));
  std::unique_ptr<dnspir_fleet> f(new dnspir_fleet());
  f->device = device;
  f->ctx = c;
  f->g1 = make_group(log2_n, primary_order);
  f->g2 = make_group(log2_n, secondary_order);
  f->S = num_shards;
  f->D = num_distinct;
  CK(cudaStreamCreateWithFlags(&f->own, cudaStreamNonBlocking));
  {
    // the secondary phase runs at the highest priority so that its few,
    // long-lived chain blocks are dispatched ahead of pending scan blocks
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&f->sec, cudaStreamNonBlocking, hi));
  }
  f->st = f->own;
  for (auto& s : f->slot) {
    CK(cudaEventCreateWithFlags(&s.prim_done, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&s.sec_done, cudaEventDisableTiming));
  }
  f->slabs.assign(num_distinct, nullptr);
  f->ready.assign(num_distinct, false);
  const size_t words = slab_words(f->g1);
  for (uint32_t d = 0; d < num_distinct; d++) CK(cudaMalloc(&f->slabs[d], words * 4));
  std::vector<uint32_t*> ptrs(num_shards);
  std::vector<int> dist(num_shards);
  for (uint32_t s = 0; s < num_shards; s++) {
    ptrs[s] = f->slabs[s % num_distinct];
    dist[s] = (int)(s % num_distinct);
  }
  CKR(f->slabs_dev.ensure(num_shards * sizeof(uint32_t*)));
  CKR(f->distinct_dev.ensure(num_shards * sizeof(int)));
  CK(cudaMemcpy(f->slabs_dev.p, ptrs.data(), num_shards * sizeof(uint32_t*), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(f->distinct_dev.p, dist.data(), num_shards * sizeof(int), cudaMemcpyHostToDevice));
  CKR(f->a_zq.ensure((size_t)num_distinct * SIMD * f->g1.n * 8));
  CKR(f->a_ms.ensure((size_t)num_distinct * SIMD * f->g1.n * 4));
  f->R = scan_chunks(f->g1, num_shards);
  *out = f.release();
  return DNSPIR_OK;
}

int dnspir_fleet_create(int device, uint64_t num_entries, uint32_t num_distinct, dnspir_fleet** out) {
  uint32_t l1 = 0, l2 = 0, s = 0;
  CKR(dnspir_get_database_shape(num_entries, &l1, &l2, &s));
  return dnspir_fleet_create_general(device, LOG2_N_MAX, l1, l2, s, num_distinct, out);
}

int dnspir_fleet_set_shards(dnspir_fleet* f, uint32_t first, uint32_t count, const uint16_t* entries,
                            int entries_on_device) {
  if (!f || !entries) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(f->mu);
  if ((uint64_t)first + count > f->D) return fail(DNSPIR_ERR_BAD_ARG, "distinct shard index out of range");
  DeviceGuard dg(f->device);
  const size_t per = (size_t)SIMD * f->g1.l * f->g1.n;
  const uint32_t batch = 16;
  for (uint32_t b0 = 0; b0 < count; b0 += batch) {
    const uint32_t cnt = count - b0 < batch ? count - b0 : batch;
    const uint16_t* src = entries + (size_t)b0 * per;
    if (!entries_on_device) {
      CKR(f->ws.in16.ensure((size_t)cnt * per * 2));
      CK(cudaMemcpyAsync(f->ws.in16.p, src, (size_t)cnt * per * 2, cudaMemcpyHostToDevice, f->st));
      src = f->ws.in16.as<uint16_t>();
    }
    for (uint32_t i = 0; i < cnt; i++) f->ready[first + b0 + i] = false;
    CKR(preprocess_shards(f->ctx, f->g1, 0, &f->slabs[first + b0], (int)cnt, src,
                          f->a_zq.as<uint64_t>() + (size_t)(first + b0) * SIMD * f->g1.n,
                          f->a_ms.as<uint32_t>() + (size_t)(first + b0) * SIMD * f->g1.n, f->ws, f->st));
    for (uint32_t i = 0; i < cnt; i++) f->ready[first + b0 + i] = true;
  }
  return DNSPIR_OK;
}

static int fleet_ready(dnspir_fleet* f) {
  for (uint32_t d = 0; d < f->D; d++)
    if (!f->ready[d]) return fail(DNSPIR_ERR_NOT_READY, "fleet shard not preprocessed");
  return DNSPIR_OK;
}

// Timing events of query i of the current call (created on demand).
static int query_events(dnspir_fleet* f, uint32_t i, cudaEvent_t** out) {
  while (f->tev.size() < 6 * (size_t)(i + 1)) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    f->tev.push_back(e);
  }
  if (f->tev_ok.size() < (size_t)i + 1) f->tev_ok.resize(i + 1, 0);
  *out = &f->tev[6 * (size_t)i];
  return DNSPIR_OK;
}

static int slot_workspace(dnspir_fleet* f, QSlot& s) {
  const uint32_t n = f->g1.n;
  CKR(s.qnat.ensure((size_t)6 * 2 * n * 4));
  CKR(s.qbrv.ensure((size_t)6 * 2 * n * 4));
  CKR(s.sec_in.ensure((size_t)f->g2.l * CTXT_PARTS * n * 2));
  return DNSPIR_OK;
}

// Primary phase of one query on the main stream: the slot's decoded vectors
// (already written by `load`, which runs first) -> scan of every shard ->
// epilogue into the slot's secondary entries.  Events: t[1] scan start,
// t[2] scan end, t[3] primary end.
static int stage_primary(dnspir_fleet* f, QSlot& s, cudaEvent_t* t) {
  const Group& g1 = f->g1;
  const uint32_t n = g1.n;
  cudaStream_t st = f->st;
  const int chunks = g1.H * f->R;
  CKR(f->part.ensure((size_t)chunks * f->S * 2 * n * SIMD * 4));
  if (t) CK(cudaEventRecord(t[1], st));
  launch_scan_plain(f->slabs_dev.as<uint32_t*>(), f->S, s.qnat.as<uint32_t>(), f->part.as<uint32_t>(), g1, f->R, st);
  if (t) CK(cudaEventRecord(t[2], st));
  launch_primary_epilogue(f->part.as<uint32_t>(), chunks, f->S, f->a_ms.as<uint32_t>(), f->distinct_dev.as<int>(),
                          s.sec_in.as<uint16_t>(), CTXT_PARTS, 0, g1, f->ctx->T, st);
  if (t) CK(cudaEventRecord(t[3], st));
  CK(cudaEventRecord(s.prim_done, st));
  s.prim_recorded = true;
  CK(cudaGetLastError());
  return DNSPIR_OK;
}

// Secondary phase on the secondary stream: encode the per-query database,
// run the fused key-switch chain, write the reply (bytes, or Z_q ciphertexts),
// and copy reply bytes to the host when host_reply is given.  Events: t[4]
// secondary start, t[5] end.
static int stage_secondary(dnspir_fleet* f, QSlot& s, cudaEvent_t* t, uint8_t* reply_dev, uint64_t* reply_zq,
                           uint8_t* host_reply) {
  const Group& g2 = f->g2;
  const uint32_t n = g2.n;
  cudaStream_t st = f->sec;
  CKR(f->ws.A.ensure((size_t)g2.l * CTXT_PARTS * n * 4));
  CKR(f->ws.Ahat.ensure((size_t)g2.H * g2.L * CTXT_PARTS * n * 4));
  CKR(f->secE.ensure((size_t)2 * g2.H * g2.L * CTXT_PARTS * n * 4));
  CKR(f->chain_out.ensure((size_t)g2.H * CTXT_PARTS * 2 * 2 * n * 4));
  CK(cudaStreamWaitEvent(st, s.prim_done, 0));
  if (t) CK(cudaEventRecord(t[4], st));
  const uint32_t l_in = f->S * SIMD;
  launch_encode_cols(s.sec_in.as<uint16_t>(), f->ws.A.as<uint32_t>(), g2, l_in, CTXT_PARTS, f->ctx->T, st);
  launch_encode_rows(f->ws.A.as<uint32_t>(), f->ws.Ahat.as<uint32_t>(), g2, l_in, CTXT_PARTS, f->ctx->T, st);
  launch_encode_lift(f->ws.Ahat.as<uint32_t>(), f->secE.as<uint32_t>(), g2, CTXT_PARTS, 1, f->ctx->T, st);
  launch_secondary_chain(f->secE.as<uint32_t>(), s.qbrv.as<uint32_t>(), (size_t)6 * 2 * n, 1,
                         f->chain_out.as<uint32_t>(), g2, chain_consts(f->ctx, g2.log2n, 1), f->ctx->T, st);
  launch_reply(f->chain_out.as<uint32_t>(), 1, g2.H, reply_dev, 0, reply_zq, g2.log2n, f->ctx->T, st);
  if (host_reply) CK(cudaMemcpyAsync(host_reply, reply_dev, dnspir_reply_bytes(), cudaMemcpyDeviceToHost, st));
  if (t) CK(cudaEventRecord(t[5], st));
  CK(cudaEventRecord(s.sec_done, st));
  s.sec_pending = true;
  CK(cudaGetLastError());
  return DNSPIR_OK;
}

// Before a slot is reused, the main stream waits for the slot's previous
// secondary phase (it reads the slot's decoded vectors and entries).
static int slot_acquire(dnspir_fleet* f, QSlot& s) {
  if (s.sec_pending) CK(cudaStreamWaitEvent(f->st, s.sec_done, 0));
  s.sec_pending = false;
  return DNSPIR_OK;
}

// End of a call: the main stream waits for every secondary phase, then the host.
static int fleet_drain(dnspir_fleet* f) {
  for (auto& s : f->slot)
    if (s.sec_pending) CK(cudaStreamWaitEvent(f->st, s.sec_done, 0));
  CK(cudaStreamSynchronize(f->st));
  for (auto& s : f->slot) s.sec_pending = false;
  return DNSPIR_OK;
}

static PolySpec wire_spec(const Group& g1, const Group& g2) {
  PolySpec spec;
  memset(&spec, 0, sizeof(spec));
  uint32_t off = 0;
  auto add = [&](int slot, int bits) {
    spec.off[spec.npoly] = off;
    spec.bits[spec.npoly] = bits;
    spec.slot[spec.npoly] = slot;
    spec.npoly++;
    off += g1.n * bits / 8;
  };
  add(0, GK_BITS);
  add(1, GK_BITS);
  add(2, PQ_BITS);
  if (g1.H == 2) add(3, PQ_BITS);
  add(4, SQ_BITS);
  if (g2.H == 2) add(5, SQ_BITS);
  return spec;
}

int dnspir_fleet_process_queries(dnspir_fleet* f, const uint8_t* const* queries, const uint64_t* query_lens,
                                 uint32_t nq, uint8_t* replies, uint64_t reply_stride, int32_t* status,
                                 int on_device) {
  if (!f || (!queries && nq) || (!query_lens && nq) || (!replies && nq)) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  if (nq && reply_stride < dnspir_reply_bytes()) return fail(DNSPIR_ERR_BAD_ARG, "reply stride too small");
  std::lock_guard<std::mutex> lk(f->mu);
  CKR(fleet_ready(f));
  const Group& g1 = f->g1;
  const Group& g2 = f->g2;
  if (g1.log2n != LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_SHAPE, "the wire format is defined for N = 2048");
  DeviceGuard dg(f->device);
  const uint64_t want = dnspir_query_bytes(g1.l, g2.l);
  const PolySpec spec = wire_spec(g1, g2);
  f->tev_n = 0;
  std::fill(f->tev_ok.begin(), f->tev_ok.end(), 0);
  const size_t RB = dnspir_reply_bytes();
  if (!on_device) CKR(f->rpin.ensure((size_t)nq * RB));
  int first_err = DNSPIR_OK;
  std::string first_msg;
  uint32_t k = 0;  // answered queries so far (slot parity)
  for (uint32_t i = 0; i < nq; i++) {
    int r = DNSPIR_OK;
    if (!queries[i]) r = fail(DNSPIR_ERR_BAD_ARG, "null query");
    else if (query_lens[i] != want) r = fail(DNSPIR_ERR_BAD_SIZE, "query length does not match the database shape");
    cudaEvent_t* t = nullptr;
    if (r == DNSPIR_OK) r = query_events(f, i, &t);
    if (r == DNSPIR_OK) {
      QSlot& s = f->slot[k & 1];
      r = slot_acquire(f, s);
      if (r == DNSPIR_OK) r = slot_workspace(f, s);
      if (r == DNSPIR_OK && !on_device) {
        r = s.qbytes.ensure(want);
        if (r == DNSPIR_OK) r = s.qpin.ensure(want);
        if (r == DNSPIR_OK) r = s.reply_dev.ensure(RB);
        // the slot's staging buffer may still feed the copy of the query two back
        if (r == DNSPIR_OK && s.prim_recorded && cudaEventSynchronize(s.prim_done) != cudaSuccess)
          r = fail(DNSPIR_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
        if (r == DNSPIR_OK) memcpy(s.qpin.p, queries[i], want);
      }
      if (r == DNSPIR_OK) {
        cudaError_t e = cudaEventRecord(t[0], f->st);
        const uint8_t* src = queries[i];
        if (e == cudaSuccess && !on_device) {
          e = cudaMemcpyAsync(s.qbytes.p, s.qpin.p, want, cudaMemcpyHostToDevice, f->st);
          src = s.qbytes.as<uint8_t>();
        }
        if (e != cudaSuccess) r = fail(DNSPIR_ERR_CUDA, cudaGetErrorString(e));
        else launch_decode_query(src, spec, s.qnat.as<uint32_t>(), s.qbrv.as<uint32_t>(), g1.log2n, f->ctx->T, f->st);
      }
      if (r == DNSPIR_OK) r = stage_primary(f, s, t);
      if (r == DNSPIR_OK)
        r = on_device ? stage_secondary(f, s, t, replies + (size_t)i * reply_stride, nullptr, nullptr)
                      : stage_secondary(f, s, t, s.reply_dev.as<uint8_t>(), nullptr, (uint8_t*)f->rpin.p + i * RB);
      if (r == DNSPIR_OK) k++;
      f->tev_ok[i] = r == DNSPIR_OK;
      f->tev_n = i + 1;
    }
    if (status) status[i] = r;
    if (r == DNSPIR_ERR_CUDA || r == DNSPIR_ERR_OOM) return r;
    if (r != DNSPIR_OK && first_err == DNSPIR_OK) {
      first_err = r;
      first_msg = g_err;
    }
  }
  CKR(fleet_drain(f));
  if (!on_device)
    for (uint32_t i = 0; i < nq; i++)
      if (i < f->tev_ok.size() && f->tev_ok[i] && i < f->tev_n)
        memcpy(replies + (size_t)i * reply_stride, (uint8_t*)f->rpin.p + i * RB, RB);
  if (first_err != DNSPIR_OK) g_err = first_msg;
  return first_err;
}

int dnspir_fleet_process_query(dnspir_fleet* f, const uint8_t* query, uint64_t query_len, uint8_t* reply,
                               uint64_t* reply_len) {
  int32_t st = 0;
  const uint8_t* qs[1] = {query};
  uint64_t ls[1] = {query_len};
  CKR(dnspir_fleet_process_queries(f, qs, ls, 1, reply, dnspir_reply_bytes(), &st, 0));
  if (reply_len) *reply_len = dnspir_reply_bytes();
  return DNSPIR_OK;
}

int dnspir_fleet_perform_double_pir(dnspir_fleet* f, const uint64_t* pq, const uint64_t* pqc, const uint64_t* sq,
                                    const uint64_t* sqc, const uint64_t* gk, uint64_t* out) {
  if (!f || !pq || !sq || !gk || !out) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(f->mu);
  CKR(fleet_ready(f));
  if ((f->g1.H == 2) != (pqc != nullptr))
    return fail(DNSPIR_ERR_BAD_SHAPE, "conjugate primary query must be given exactly when required (double_pir.rs:160)");
  if ((f->g2.H == 2) != (sqc != nullptr))
    return fail(DNSPIR_ERR_BAD_SHAPE, "conjugate secondary query must be given exactly when required");
  const size_t n = f->g1.n;
  std::vector<uint64_t> z(6 * n, 0);
  memcpy(&z[0], gk, n * 8);
  memcpy(&z[n], gk + n, n * 8);
  memcpy(&z[2 * n], pq, n * 8);
  if (pqc) memcpy(&z[3 * n], pqc, n * 8);
  memcpy(&z[4 * n], sq, n * 8);
  if (sqc) memcpy(&z[5 * n], sqc, n * 8);
  if (!reduced(z.data(), z.size())) return fail(DNSPIR_ERR_BAD_ARG, "ring element coefficients must be below q");
  DeviceGuard dg(f->device);
  QSlot& s = f->slot[0];
  cudaEvent_t* t = nullptr;
  CKR(query_events(f, 0, &t));
  CKR(slot_acquire(f, s));
  CKR(slot_workspace(f, s));
  CKR(f->qzq.ensure(z.size() * 8));
  CKR(f->reply_zq.ensure((size_t)CTXT_PARTS * 2 * n * 8));
  CK(cudaEventRecord(t[0], f->st));
  CK(cudaMemcpyAsync(f->qzq.p, z.data(), z.size() * 8, cudaMemcpyHostToDevice, f->st));
  launch_ring_to_ntt(f->qzq.as<uint64_t>(), 6, s.qnat.as<uint32_t>(), s.qbrv.as<uint32_t>(), f->g1.log2n, f->ctx->T,
                     f->st);
  CKR(stage_primary(f, s, t));
  CKR(stage_secondary(f, s, t, nullptr, f->reply_zq.as<uint64_t>(), nullptr));
  f->tev_ok[0] = 1;
  f->tev_n = 1;
  CKR(fleet_drain(f));
  CK(cudaMemcpy(out, f->reply_zq.p, (size_t)CTXT_PARTS * 2 * n * 8, cudaMemcpyDeviceToHost));
  return DNSPIR_OK;
}

int dnspir_fleet_batch_timings(dnspir_fleet* f, uint32_t max, double* latency_ms, double* primary_ms,
                               double* secondary_ms, double* scan_ms) {
  if (!f) return -fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  std::lock_guard<std::mutex> lk(f->mu);
  DeviceGuard dg(f->device);
  const uint32_t n = f->tev_n < max ? f->tev_n : max;
  for (uint32_t i = 0; i < n; i++) {
    double v[4] = {-1, -1, -1, -1};
    if (f->tev_ok[i]) {
      cudaEvent_t* t = &f->tev[6 * (size_t)i];
      float a = 0, b = 0, c = 0, d = 0;
      if (cudaEventSynchronize(t[5]) != cudaSuccess || cudaEventElapsedTime(&a, t[0], t[5]) != cudaSuccess ||
          cudaEventElapsedTime(&b, t[0], t[3]) != cudaSuccess || cudaEventElapsedTime(&c, t[4], t[5]) != cudaSuccess ||
          cudaEventElapsedTime(&d, t[1], t[2]) != cudaSuccess) {
        cudaGetLastError();
        return -fail(DNSPIR_ERR_CUDA, "timing events unavailable");
      }
      v[0] = a, v[1] = b, v[2] = c, v[3] = d;
    }
    if (latency_ms) latency_ms[i] = v[0];
    if (primary_ms) primary_ms[i] = v[1];
    if (secondary_ms) secondary_ms[i] = v[2];
    if (scan_ms) scan_ms[i] = v[3];
  }
  return (int)n;
}

int dnspir_fleet_last_timings(dnspir_fleet* f, double* primary_ms, double* secondary_ms, double* scan_ms) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  uint32_t n = 0;
  {
    std::lock_guard<std::mutex> lk(f->mu);
    n = f->tev_n;
    if (!n || !f->tev_ok[n - 1]) return fail(DNSPIR_ERR_NOT_READY, "no query answered yet");
  }
  std::vector<double> p(n), s(n), c(n);
  const int got = dnspir_fleet_batch_timings(f, n, nullptr, p.data(), s.data(), c.data());
  if (got < 0) return -got;
  if (primary_ms) *primary_ms = p[n - 1];
  if (secondary_ms) *secondary_ms = s[n - 1];
  if (scan_ms) *scan_ms = c[n - 1];
  return DNSPIR_OK;
}

int dnspir_fleet_set_stream(dnspir_fleet* f, void* s) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  std::lock_guard<std::mutex> lk(f->mu);
  f->st = s ? (cudaStream_t)s : f->own;
  return DNSPIR_OK;
}

uint64_t dnspir_fleet_slab_bytes(dnspir_fleet* f) { return f ? (uint64_t)f->D * slab_words(f->g1) * 4 : 0; }

int dnspir_fleet_destroy(dnspir_fleet* f) {
  if (!f) return DNSPIR_OK;
  DeviceGuard dg(f->device);
  cudaStreamSynchronize(f->st);
  cudaStreamSynchronize(f->sec);
  delete f;
  return DNSPIR_OK;
}

}  // extern "C"
