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

#include "host.h"

using namespace dnspir;

namespace dnspir {

// ------------------------------------------------------------------ errors
thread_local std::string g_err;
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
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

CrtConst host_crt_const() {
  CrtConst c;
  c.q2inv1 = (uint32_t)invmod(P2 % P1, P1);
  c.q1inv2 = (uint32_t)invmod(P1 % P2, P2);
  return c;
}

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
  const uint64_t mask = (1ull << 51) - 1;  // ceil(log2 q) = 51 bits
  for (uint32_t i = 0; i < n; i++) {
    uint64_t x;
    do x = r.next_u64() & mask;
    while (x >= QQ);
    out[i] = x;
  }
}

// The six a-parts in effect per ring dimension: the seed expansion above, or
// polynomials installed by dnspir_set_a_parts.  `version` changes with every
// installation, so shards preprocessed under other a-parts can be recognised.
std::mutex g_ap_mu;
std::vector<uint64_t> g_ap_override[LOG2_N_MAX + 1];
uint64_t g_ap_version[LOG2_N_MAX + 1];
}  // namespace

uint64_t a_parts_version(int log2n) {
  std::lock_guard<std::mutex> lk(g_ap_mu);
  return g_ap_version[log2n];
}

void a_parts_host(int log2n, uint64_t* out, uint64_t* version) {
  const uint32_t n = 1u << log2n;
  {
    std::lock_guard<std::mutex> lk(g_ap_mu);
    if (version) *version = g_ap_version[log2n];
    if (!g_ap_override[log2n].empty()) {
      memcpy(out, g_ap_override[log2n].data(), (size_t)6 * n * 8);
      return;
    }
  }
  for (int s = 0; s < 6; s++) expand(n, SEEDS[s], out + (size_t)s * n);
}

// ------------------------------------------------------------ device context
static std::mutex g_ctx_mu;
static DeviceCtx* g_ctx[64];

static int build_tables(DeviceCtx& c) {
  const int n = N_MAX;
  // 8 scalar tables (fw, fwq, iw, iwq of each factor), then the pairs
  // (w, Shoup companion) interleaved: fw2 of each factor, iw2 of each factor
  std::vector<uint32_t> h(16 * n);
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
      h[(8 + 2 * pi) * n + 2 * k] = h[(0 + pi) * n + k];
      h[(8 + 2 * pi) * n + 2 * k + 1] = h[(2 + pi) * n + k];
      h[(12 + 2 * pi) * n + 2 * k] = h[(4 + pi) * n + k];
      h[(12 + 2 * pi) * n + 2 * k + 1] = h[(6 + pi) * n + k];
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
    c.T.fw2[pi] = reinterpret_cast<const uint2*>(c.tables + (8 + 2 * pi) * n);
    c.T.iw2[pi] = reinterpret_cast<const uint2*>(c.tables + (12 + 2 * pi) * n);
  }
  return DNSPIR_OK;
}

int get_ctx(int device, DeviceCtx** out) {
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
// a-parts in NTT form for the a-parts now in effect (rebuilt after
// dnspir_set_a_parts; earlier buffers are kept, a kernel queued before the
// change may still read them)
static int ctx_a_parts(DeviceCtx* c, int log2n, uint64_t* version) {
  const uint32_t n = 1u << log2n;
  uint64_t ver = 0;
  std::vector<uint64_t> ap(6 * (size_t)n);
  a_parts_host(log2n, ap.data(), &ver);
  if (version) *version = ver;
  if (c->consts[log2n] && c->consts_ver[log2n] == ver) return DNSPIR_OK;
  uint64_t* dz = nullptr;
  uint32_t* dc = nullptr;
  CK(cudaMalloc(&dz, ap.size() * 8));
  CK(cudaMalloc(&dc, (size_t)6 * 2 * n * 4));
  CK(cudaMemcpy(dz, ap.data(), ap.size() * 8, cudaMemcpyHostToDevice));
  launch_ring_to_ntt(dz, 6, nullptr, dc, log2n, c->T, 0);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  CK(cudaFree(dz));
  if (c->consts[log2n]) c->retired.push_back(c->consts[log2n]);
  c->consts[log2n] = dc;
  c->consts_ver[log2n] = ver;
  return DNSPIR_OK;
}

int ctx_consts(DeviceCtx* c, int log2n, uint64_t* version) {
  std::lock_guard<std::mutex> lk(c->mu);
  if (c->galb[log2n]) return ctx_a_parts(c, log2n, version);
  const uint32_t n = 1u << log2n;
  uint32_t* dg = nullptr;
  CK(cudaMalloc(&dg, (size_t)n * 4));
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
  {
    // (sign, e) order of the scan: position u = sign * N/2 + e <-> residue +-5^e mod 2N
    std::vector<uint32_t> gt(n), uo(n);
    uint32_t p5 = 1;
    for (uint32_t e = 0; e < n / 2; e++) {
      gt[e] = p5;
      gt[n / 2 + e] = two_n - p5;
      p5 = (uint32_t)(((uint64_t)p5 * 5) % two_n);
    }
    for (uint32_t u = 0; u < n; u++) uo[(gt[u] - 1) / 2] = u;
    uint32_t *dgt = nullptr, *duo = nullptr;
    CK(cudaMalloc(&dgt, n * 4));
    CK(cudaMalloc(&duo, n * 4));
    CK(cudaMemcpy(dgt, gt.data(), n * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(duo, uo.data(), n * 4, cudaMemcpyHostToDevice));
    c->gtab[log2n] = dgt;
    c->uof[log2n] = duo;
  }
  CK(cudaDeviceSynchronize());
  device_pow5(log2n, false);
  device_pow5(log2n, true);
  c->galb[log2n] = dg;
  return ctx_a_parts(c, log2n, version);
}

SlotMaps slot_maps(DeviceCtx* c, int log2n) {
  SlotMaps m;
  m.g = c->gtab[log2n];
  m.uof = c->uof[log2n];
  return m;
}

ChainConsts chain_consts(DeviceCtx* c, int log2n, int used_seeds) {
  const size_t n2 = (size_t)2 << log2n;
  ChainConsts cc;
  cc.gka = c->consts[log2n];
  cc.qa = c->consts[log2n] + (2 + 2 * used_seeds) * n2;
  cc.galb = c->galb[log2n];
  cc.maps = slot_maps(c, log2n);
  return cc;
}

int check_group(uint32_t log2n, uint32_t l) {
  if (log2n < 3 || log2n > LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_SHAPE, "log2_n must be in [3, 11]");
  const uint32_t n = 1u << log2n;
  if (l == 0 || n % l != 0) return fail(DNSPIR_ERR_BAD_SHAPE, "group order must divide N");
  if (l != n && 2 * l > n) return fail(DNSPIR_ERR_BAD_SHAPE, "a subgroup order must be at most N/2");
  if (2ull * TPLAIN * n >= P1) return fail(DNSPIR_ERR_BAD_SHAPE, "max_coeff >= q1");
  return DNSPIR_OK;
}

// Encodes `count` shards' entries (device u16, one shard after another) into
// their slabs, runs the preprocessing chain and the a-part finalisation.
int preprocess_shards(DeviceCtx* c, const Group& g, int used_seeds, uint32_t* const* slabs_host, int count,
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
    launch_encode_lift(ws.Ahat.as<uint32_t>(), slabs_host[s], g, SIMD, 0, slot_maps(c, g.log2n), c->T, st);
  }
  CK(cudaMemcpyAsync(ws.slab_ptrs.p, slabs_host, (size_t)count * sizeof(uint32_t*), cudaMemcpyHostToDevice, st));
  launch_primary_chain(ws.slab_ptrs.as<uint32_t*>(), count, ws.a_out.as<uint32_t>(), g,
                       chain_consts(c, g.log2n, used_seeds), c->T, st);
  launch_primary_finalize(ws.a_out.as<uint32_t>(), count, a_zq, a_ms, g, c->T, st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return DNSPIR_OK;
}

bool reduced(const uint64_t* v, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (v[i] >= QQ) return false;
  return true;
}

}  // namespace dnspir

struct dnspir_db {
  int device = 0;
  DeviceCtx* ctx = nullptr;
  Group g;
  int used_seeds = 0;
  bool ready = false;
  uint64_t ap_ver = 0;  // a-parts version the slab was preprocessed under
  cudaStream_t st = nullptr;
  cudaEvent_t noalloc_done = nullptr;  // recorded on the caller's stream after each no-allocation call
  uint32_t* slab = nullptr;
  DBuf a_zq, a_ms, qz, qlane, part, out, slab_ptr;
  EncodeWs ws;
  std::mutex mu;
  ~dnspir_db() {
    if (noalloc_done) cudaEventDestroy(noalloc_done);
    if (slab) cudaFree(slab);
    if (st) cudaStreamDestroy(st);
  }
};

namespace dnspir {
int noalloc_reserve(int device);  // noalloc.cu

static int db_ready(const dnspir_db* db) {
  if (!db->ready) return fail(DNSPIR_ERR_NOT_READY, "database not preprocessed");
  if (db->ap_ver != a_parts_version(db->g.log2n))
    return fail(DNSPIR_ERR_NOT_READY, "the a-parts changed since the database was preprocessed: call set_db again");
  return DNSPIR_OK;
}

// The no-allocation entry point (noalloc.cu) holds the shard's lock from the
// view until its work is queued; the event recorded on its stream lets set_db
// and destroy wait for that work before they touch the slab.
int db_noalloc_begin(dnspir_db* db, DbView* out) {
  db->mu.lock();
  const int rc = db_ready(db);
  if (rc != DNSPIR_OK) {
    db->mu.unlock();
    return rc;
  }
  out->device = db->device;
  out->ready = db->ready;
  out->g = db->g;
  out->slab = db->slab;
  out->T = db->ctx->T;
  out->maps = slot_maps(db->ctx, db->g.log2n);
  return DNSPIR_OK;
}
int db_noalloc_end(dnspir_db* db, cudaStream_t st) {
  const cudaError_t e = cudaEventRecord(db->noalloc_done, st);
  db->mu.unlock();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(DNSPIR_ERR_CUDA, std::string("cudaEventRecord: ") + cudaGetErrorString(e));
  }
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

int dnspir_set_a_parts(uint32_t log2_n, const uint64_t* coeffs) {
  if (log2_n < 3 || log2_n > LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_ARG, "log2_n must be in [3, 11]");
  const size_t n = (size_t)1 << log2_n;
  if (coeffs && !reduced(coeffs, 6 * n)) return fail(DNSPIR_ERR_BAD_ARG, "a-part coefficients must be below q");
  std::lock_guard<std::mutex> lk(g_ap_mu);
  if (coeffs) g_ap_override[log2_n].assign(coeffs, coeffs + 6 * n);
  else g_ap_override[log2_n].clear();
  g_ap_version[log2_n]++;
  return DNSPIR_OK;
}

int dnspir_get_a_parts(uint32_t log2_n, uint64_t* out) {
  if (!out || log2_n < 3 || log2_n > LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_ARG, "bad argument");
  a_parts_host((int)log2_n, out, nullptr);
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
  CK(cudaEventCreateWithFlags(&d->noalloc_done, cudaEventDisableTiming));
  // the no-allocation entry point's static region is loaded now, before the
  // slab takes the memory (module loading is lazy)
  CKR(noalloc_reserve(device));
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
  // a no-allocation call queued on another stream may still read the slab
  CK(cudaStreamWaitEvent(db->st, db->noalloc_done, 0));
  uint64_t ver = 0;
  CKR(ctx_consts(db->ctx, db->g.log2n, &ver));
  CKR(preprocess_shards(db->ctx, db->g, db->used_seeds, slabs, 1, src, db->a_zq.as<uint64_t>(),
                        db->a_ms.as<uint32_t>(), db->ws, db->st));
  db->ap_ver = ver;
  db->ready = true;
  return DNSPIR_OK;
}

int dnspir_db_get_a(dnspir_db* db, uint64_t* out) {
  if (!db || !out) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(db->mu);
  CKR(db_ready(db));
  DeviceGuard dg(db->device);
  CK(cudaMemcpy(out, db->a_zq.p, (size_t)SIMD * db->g.n * 8, cudaMemcpyDeviceToHost));
  return DNSPIR_OK;
}

int dnspir_db_perform_pir_split(dnspir_db* db, const uint64_t* qry_b, const uint64_t* qry_conj_b, const uint64_t* gk_b,
                                uint64_t* out_b) {
  if (!db || !qry_b || !gk_b || !out_b) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(db->mu);
  CKR(db_ready(db));
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
  launch_scan_lanes(db->slab, db->qlane.as<uint32_t>(), db->part.as<uint32_t>(), g, R, slot_maps(db->ctx, g.log2n),
                    db->st);
  launch_epilogue_zq(db->part.as<uint32_t>(), g.H * R, db->out.as<uint64_t>(), g, slot_maps(db->ctx, g.log2n),
                     db->ctx->T, db->st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out_b, db->out.p, (size_t)SIMD * n * 8, cudaMemcpyDeviceToHost, db->st));
  CK(cudaStreamSynchronize(db->st));
  return DNSPIR_OK;
}

int dnspir_db_destroy(dnspir_db* db) {
  if (!db) return DNSPIR_OK;
  DeviceGuard dg(db->device);
  {
    // no-allocation calls still queued on the caller's stream read the slab
    std::lock_guard<std::mutex> lk(db->mu);
    cudaEventSynchronize(db->noalloc_done);
  }
  delete db;
  return DNSPIR_OK;
}

}  // extern "C"
