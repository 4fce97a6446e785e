// fleet.cu -- a fleet of primary shards and the two-level answer pipeline
// (perform_batched_double_pir, crates/pir/src/double_pir.rs:126-228;
// process_queries, pir_wrapper.rs:349-409).
//
// Queries are answered in groups of up to `batch` (1, 2, 4, 8 or 16): one pass
// of the scan over every shard serves the whole group (the slab is read once
// per group), then each query's secondary database is encoded and evaluated.
// Two buffer slots alternate between groups: the primary phase of group k+1
// (main stream) runs while the secondary phase of group k runs on a second,
// high-priority stream; events order the reuse of a slot.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "host.h"

using namespace dnspir;

namespace {

// Buffers of one group of queries in flight.
struct QSlot {
  DBuf qbytes, qnat, qbrv, fin, sec_in, reply_dev;
  HBuf qpin;  // host staging of the query bytes
  cudaEvent_t prim_done = nullptr, sec_done = nullptr;
  bool sec_pending = false, prim_recorded = false;
};

}  // namespace

struct dnspir_fleet {
  int device = 0;
  DeviceCtx* ctx = nullptr;
  Group g1, g2;
  uint32_t S = 0, D = 0;
  cudaStream_t own = nullptr, st = nullptr, sec = nullptr;
  std::vector<uint32_t*> slabs;
  std::vector<bool> ready;
  DBuf slabs_dev, distinct_dev, a_zq, a_ms, counter;
  EncodeWs ws;
  QSlot slot[2];
  DBuf secE, chain_out, qzq, reply_zq;  // used by one stream at a time
  HBuf rpin;                            // host staging of the replies of one call
  int batch = 1;
  std::vector<cudaEvent_t> tev;  // 6 timing events per group of the last call
  std::vector<int> q_group;      // per query of the last call: its group, or -1
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

namespace {

const size_t QV_WORDS_PER_QUERY = 6 * 2;  // decoded slots x factors, times N

int fleet_ready(dnspir_fleet* f) {
  for (uint32_t d = 0; d < f->D; d++)
    if (!f->ready[d]) return fail(DNSPIR_ERR_NOT_READY, "fleet shard not preprocessed");
  return DNSPIR_OK;
}

int group_events(dnspir_fleet* f, uint32_t gi, cudaEvent_t** out) {
  while (f->tev.size() < 6 * (size_t)(gi + 1)) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    f->tev.push_back(e);
  }
  *out = &f->tev[6 * (size_t)gi];
  return DNSPIR_OK;
}

int kernel_batch(int nb) {
  int b = 1;
  while (b < nb) b <<= 1;
  return b;
}

int slot_acquire(dnspir_fleet* f, QSlot& s) {
  if (s.sec_pending) CK(cudaStreamWaitEvent(f->st, s.sec_done, 0));
  s.sec_pending = false;
  return DNSPIR_OK;
}

int slot_workspace(dnspir_fleet* f, QSlot& s, int Bk, int nb) {
  const size_t n = f->g1.n;
  CKR(s.qnat.ensure((size_t)Bk * QV_WORDS_PER_QUERY * n * 4));
  CKR(s.qbrv.ensure((size_t)Bk * QV_WORDS_PER_QUERY * n * 4));
  CKR(s.fin.ensure((size_t)Bk * f->S * 2 * n * SIMD * 4));
  CKR(s.sec_in.ensure((size_t)f->g2.l * CTXT_PARTS * nb * n * 2));
  return DNSPIR_OK;
}

// Primary phase of a group on the main stream (decoded vectors already in the
// slot): one scan pass for Bk queries, epilogue of the first nb.
// Events: t[1] scan start, t[2] scan end, t[3] primary end.
int stage_primary(dnspir_fleet* f, QSlot& s, int nb, int Bk, cudaEvent_t* t) {
  const Group& g1 = f->g1;
  const size_t n = g1.n;
  cudaStream_t st = f->st;
  if (Bk > nb)  // unused query positions of the kernel batch compute on zeros
    CK(cudaMemsetAsync(s.qnat.as<uint32_t>() + (size_t)nb * QV_WORDS_PER_QUERY * n, 0,
                       (size_t)(Bk - nb) * QV_WORDS_PER_QUERY * n * 4, st));
  CK(cudaEventRecord(t[1], st));
  if (launch_scan_batch(f->slabs_dev.as<uint32_t*>(), f->S, s.qnat.as<uint32_t>(), QV_WORDS_PER_QUERY * n, Bk,
                        s.fin.as<uint32_t>(), g1, slot_maps(f->ctx, g1.log2n), f->counter.as<uint32_t>(), st))
    return fail(DNSPIR_ERR_BAD_ARG, "unsupported scan batch");
  CK(cudaEventRecord(t[2], st));
  launch_primary_epilogue(s.fin.as<uint32_t>(), nb, f->S, f->a_ms.as<uint32_t>(), f->distinct_dev.as<int>(),
                          s.sec_in.as<uint16_t>(), g1, slot_maps(f->ctx, g1.log2n), f->ctx->T, st);
  CK(cudaEventRecord(t[3], st));
  CK(cudaEventRecord(s.prim_done, st));
  s.prim_recorded = true;
  CK(cudaGetLastError());
  return DNSPIR_OK;
}

// Secondary phase of a group on the secondary stream: encode the nb per-query
// databases (3 lanes each), run the fused key-switch chains, write the replies
// (bytes at reply_dev + q * reply_stride, or Z_q ciphertexts) and copy reply
// bytes to host_reply when given.  Events: t[4] start, t[5] end.
int stage_secondary(dnspir_fleet* f, QSlot& s, int nb, cudaEvent_t* t, uint8_t* reply_dev, size_t reply_stride,
                    uint64_t* reply_zq, uint8_t* host_reply) {
  const Group& g2 = f->g2;
  const size_t n = g2.n;
  const int nl = CTXT_PARTS * nb;
  cudaStream_t st = f->sec;
  CKR(f->ws.A.ensure((size_t)g2.l * nl * n * 4));
  CKR(f->ws.Ahat.ensure((size_t)g2.H * g2.L * nl * n * 4));
  CKR(f->secE.ensure((size_t)2 * g2.H * g2.L * nl * n * 4));
  CKR(f->chain_out.ensure((size_t)nb * g2.H * CTXT_PARTS * 2 * 2 * n * 4));
  CK(cudaStreamWaitEvent(st, s.prim_done, 0));
  CK(cudaEventRecord(t[4], st));
  const uint32_t l_in = f->S * SIMD;
  const SlotMaps maps = slot_maps(f->ctx, g2.log2n);
  launch_encode_cols(s.sec_in.as<uint16_t>(), f->ws.A.as<uint32_t>(), g2, l_in, nl, f->ctx->T, st);
  launch_encode_rows(f->ws.A.as<uint32_t>(), f->ws.Ahat.as<uint32_t>(), g2, l_in, nl, f->ctx->T, st);
  launch_encode_lift(f->ws.Ahat.as<uint32_t>(), f->secE.as<uint32_t>(), g2, nl, 1, maps, f->ctx->T, st);
  launch_secondary_chain(f->secE.as<uint32_t>(), s.qbrv.as<uint32_t>(), QV_WORDS_PER_QUERY * n, nb,
                         f->chain_out.as<uint32_t>(), g2, chain_consts(f->ctx, g2.log2n, 1), f->ctx->T, st);
  launch_reply(f->chain_out.as<uint32_t>(), nb, g2.H, reply_dev, reply_stride, reply_zq, g2.log2n, f->ctx->T, st);
  if (host_reply)
    CK(cudaMemcpyAsync(host_reply, reply_dev, (size_t)nb * dnspir_reply_bytes(), cudaMemcpyDeviceToHost, st));
  CK(cudaEventRecord(t[5], st));
  CK(cudaEventRecord(s.sec_done, st));
  s.sec_pending = true;
  CK(cudaGetLastError());
  return DNSPIR_OK;
}

// End of a call: the main stream waits for every secondary phase, then the host.
int fleet_drain(dnspir_fleet* f) {
  for (auto& s : f->slot)
    if (s.sec_pending) CK(cudaStreamWaitEvent(f->st, s.sec_done, 0));
  CK(cudaStreamSynchronize(f->st));
  CK(cudaStreamSynchronize(f->sec));
  for (auto& s : f->slot) s.sec_pending = false;
  return DNSPIR_OK;
}

PolySpec wire_spec(const Group& g1, const Group& g2) {
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

}  // namespace

extern "C" {

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
  CKR(f->counter.ensure(sizeof(uint32_t)));
  CK(cudaMemcpy(f->slabs_dev.p, ptrs.data(), num_shards * sizeof(uint32_t*), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(f->distinct_dev.p, dist.data(), num_shards * sizeof(int), cudaMemcpyHostToDevice));
  CKR(f->a_zq.ensure((size_t)num_distinct * SIMD * f->g1.n * 8));
  CKR(f->a_ms.ensure((size_t)num_distinct * SIMD * f->g1.n * 4));
  *out = f.release();
  return DNSPIR_OK;
}

int dnspir_fleet_create(int device, uint64_t num_entries, uint32_t num_distinct, dnspir_fleet** out) {
  uint32_t l1 = 0, l2 = 0, s = 0;
  CKR(dnspir_get_database_shape(num_entries, &l1, &l2, &s));
  return dnspir_fleet_create_general(device, LOG2_N_MAX, l1, l2, s, num_distinct, out);
}

int dnspir_fleet_set_batch(dnspir_fleet* f, uint32_t max_batch) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  if (!scan_batch_supported((int)max_batch)) return fail(DNSPIR_ERR_BAD_ARG, "batch must be 1, 2, 4, 8 or 16");
  std::lock_guard<std::mutex> lk(f->mu);
  f->batch = (int)max_batch;
  return DNSPIR_OK;
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

int dnspir_fleet_process_queries(dnspir_fleet* f, const uint8_t* const* queries, const uint64_t* query_lens,
                                 uint32_t nq, uint8_t* replies, uint64_t reply_stride, int32_t* status,
                                 int on_device) {
  if (!f || (!queries && nq) || (!query_lens && nq) || (!replies && nq)) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  const size_t RB = dnspir_reply_bytes();
  if (nq && reply_stride < RB) return fail(DNSPIR_ERR_BAD_ARG, "reply stride too small");
  std::lock_guard<std::mutex> lk(f->mu);
  CKR(fleet_ready(f));
  const Group& g1 = f->g1;
  const Group& g2 = f->g2;
  if (g1.log2n != LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_SHAPE, "the wire format is defined for N = 2048");
  DeviceGuard dg(f->device);
  const uint64_t want = dnspir_query_bytes(g1.l, g2.l);
  const PolySpec spec = wire_spec(g1, g2);
  const size_t qv = QV_WORDS_PER_QUERY * g1.n;
  f->q_group.assign(nq, -1);
  // validate first: rejected queries are left out of the groups
  std::vector<uint32_t> ok;
  int first_err = DNSPIR_OK;
  std::string first_msg;
  for (uint32_t i = 0; i < nq; i++) {
    int r = DNSPIR_OK;
    if (!queries[i]) r = fail(DNSPIR_ERR_BAD_ARG, "null query");
    else if (query_lens[i] != want) r = fail(DNSPIR_ERR_BAD_SIZE, "query length does not match the database shape");
    if (status) status[i] = r;
    if (r == DNSPIR_OK) ok.push_back(i);
    else if (first_err == DNSPIR_OK) {
      first_err = r;
      first_msg = g_err;
    }
  }
  if (!on_device && !ok.empty()) CKR(f->rpin.ensure(ok.size() * RB));
  uint32_t gi = 0;
  for (size_t g0 = 0; g0 < ok.size(); g0 += f->batch, gi++) {
    const int nb = (int)std::min<size_t>(f->batch, ok.size() - g0);
    const int Bk = kernel_batch(nb);
    QSlot& s = f->slot[gi & 1];
    cudaEvent_t* t = nullptr;
    CKR(group_events(f, gi, &t));
    CKR(slot_acquire(f, s));
    CKR(slot_workspace(f, s, Bk, nb));
    if (!on_device) {
      CKR(s.qbytes.ensure((size_t)nb * want));
      CKR(s.qpin.ensure((size_t)nb * want));
      CKR(s.reply_dev.ensure((size_t)nb * RB));
      // the slot's staging buffer may still feed the copy of the group two back
      if (s.prim_recorded) CK(cudaEventSynchronize(s.prim_done));
      for (int q = 0; q < nb; q++) memcpy((uint8_t*)s.qpin.p + (size_t)q * want, queries[ok[g0 + q]], want);
    }
    CK(cudaEventRecord(t[0], f->st));
    if (!on_device) CK(cudaMemcpyAsync(s.qbytes.p, s.qpin.p, (size_t)nb * want, cudaMemcpyHostToDevice, f->st));
    for (int q = 0; q < nb; q++) {
      const uint8_t* src = on_device ? queries[ok[g0 + q]] : s.qbytes.as<uint8_t>() + (size_t)q * want;
      launch_decode_query(src, spec, s.qnat.as<uint32_t>() + q * qv, s.qbrv.as<uint32_t>() + q * qv, g1.log2n,
                          f->ctx->T, f->st);
    }
    CKR(stage_primary(f, s, nb, Bk, t));
    // replies of a group are contiguous in the caller's buffer only when its
    // queries are; otherwise (a rejected query inside the group) go through
    // the staging path
    bool contiguous = true;
    for (int q = 1; q < nb; q++) contiguous &= ok[g0 + q] == ok[g0] + q;
    if (on_device && contiguous) {
      CKR(stage_secondary(f, s, nb, t, replies + (size_t)ok[g0] * reply_stride, reply_stride, nullptr, nullptr));
    } else if (on_device) {
      CKR(s.reply_dev.ensure((size_t)nb * RB));
      CKR(stage_secondary(f, s, nb, t, s.reply_dev.as<uint8_t>(), RB, nullptr, nullptr));
      for (int q = 0; q < nb; q++)
        CK(cudaMemcpyAsync(replies + (size_t)ok[g0 + q] * reply_stride, s.reply_dev.as<uint8_t>() + q * RB, RB,
                           cudaMemcpyDeviceToDevice, f->sec));
    } else {
      CKR(stage_secondary(f, s, nb, t, s.reply_dev.as<uint8_t>(), RB, nullptr, (uint8_t*)f->rpin.p + g0 * RB));
    }
    for (int q = 0; q < nb; q++) f->q_group[ok[g0 + q]] = (int)gi;
  }
  CKR(fleet_drain(f));
  if (!on_device)
    for (size_t k = 0; k < ok.size(); k++) memcpy(replies + (size_t)ok[k] * reply_stride, (uint8_t*)f->rpin.p + k * RB, RB);
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
  CKR(group_events(f, 0, &t));
  CKR(slot_acquire(f, s));
  CKR(slot_workspace(f, s, 1, 1));
  CKR(f->qzq.ensure(z.size() * 8));
  CKR(f->reply_zq.ensure((size_t)CTXT_PARTS * 2 * n * 8));
  CK(cudaEventRecord(t[0], f->st));
  CK(cudaMemcpyAsync(f->qzq.p, z.data(), z.size() * 8, cudaMemcpyHostToDevice, f->st));
  launch_ring_to_ntt(f->qzq.as<uint64_t>(), 6, s.qnat.as<uint32_t>(), s.qbrv.as<uint32_t>(), f->g1.log2n, f->ctx->T,
                     f->st);
  CKR(stage_primary(f, s, 1, 1, t));
  CKR(stage_secondary(f, s, 1, t, nullptr, 0, f->reply_zq.as<uint64_t>(), nullptr));
  f->q_group.assign(1, 0);
  CKR(fleet_drain(f));
  CK(cudaMemcpy(out, f->reply_zq.p, (size_t)CTXT_PARTS * 2 * n * 8, cudaMemcpyDeviceToHost));
  return DNSPIR_OK;
}

int dnspir_fleet_batch_timings(dnspir_fleet* f, uint32_t max, double* latency_ms, double* primary_ms,
                               double* secondary_ms, double* scan_ms) {
  if (!f) return -fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  std::lock_guard<std::mutex> lk(f->mu);
  DeviceGuard dg(f->device);
  const uint32_t n = std::min<uint32_t>((uint32_t)f->q_group.size(), max);
  for (uint32_t i = 0; i < n; i++) {
    double v[4] = {-1, -1, -1, -1};
    const int gi = f->q_group[i];
    if (gi >= 0) {
      cudaEvent_t* t = &f->tev[6 * (size_t)gi];
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
    n = (uint32_t)f->q_group.size();
    while (n > 0 && f->q_group[n - 1] < 0) n--;
    if (!n) return fail(DNSPIR_ERR_NOT_READY, "no query answered yet");
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
