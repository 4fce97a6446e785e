// fleet.cu -- a fleet of primary shards and the two-level answer pipeline
// (perform_batched_double_pir, crates/pir/src/double_pir.rs:126-228;
// process_queries, pir_wrapper.rs:349-409).
//
// Queries are answered in groups of up to `batch`: one pass of the scan over
// every shard serves the whole group (the slab is read once per group), then
// the secondary databases are encoded and evaluated in chunks of one wave of
// chain clusters (two one-part blocks per SM: 2 SMs / (6 H) queries, capped by
// a memory budget).  Two scan
// engines: CUDA cores over the lane layout (groups of a power of two up to 256) and
// the tensor cores over the tensor layout (groups up to 256, tile shape per
// group size from a table or from dnspir_fleet_tune).  Two buffer slots
// alternate between groups: the primary phase of group k+1 (main stream) runs
// while the secondary phase of group k runs on a second, high-priority
// stream; events order the reuse of a slot.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "fleet_impl.h"

using namespace dnspir;

dnspir_fleet::~dnspir_fleet() {
  for (uint32_t* s : slabs)
    if (s) cudaFree(s);
  for (auto& e : tev)
    if (e) cudaEventDestroy(e);
  if (sec) cudaStreamDestroy(sec);
  if (own) cudaStreamDestroy(own);
}

namespace {

const size_t SEC_BUDGET = (size_t)6 << 30;  // secondary workspace of one chunk
const int TENSOR_MAX_BATCH = 256;

#define NOT_SERVING(f) \
  if ((f)->serving) return fail(DNSPIR_ERR_BAD_ARG, "the fleet is attached to a running server")

int group_events(dnspir_fleet* f, uint32_t gi, cudaEvent_t** out) {
  while (f->tev.size() < 6 * (size_t)(gi + 1)) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    f->tev.push_back(e);
  }
  *out = &f->tev[6 * (size_t)gi];
  return DNSPIR_OK;
}

int pow2_batch(int nb) {
  int b = 1;
  while (b < nb) b <<= 1;
  return b;
}

// Tile shape of the tensor scan for a group of nb queries, and the padded
// group size it implies.
const TScanShape& tensor_shape(dnspir_fleet* f, int nb, int* nb_pad) {
  int count = 0;
  const TScanShape* sh = tscan_shapes(&count);
  int idx;
  auto it = f->tuned.find(nb);
  if (it != f->tuned.end()) {
    idx = it->second;
  } else {
    // untuned: the narrowest query tile that holds the group, one m-tile,
    // the one-tile-per-CTA kernel
    const int want = nb <= 4 ? 16 : nb <= 8 ? 32 : nb <= 16 ? 64 : nb <= 32 ? 128 : nb <= 64 ? 256 : 512;
    idx = 0;
    for (int i = count - 1; i >= 0; i--)
      if (sh[i].nq == want && sh[i].mtpc == 1 && !sh[i].persistent) idx = i;
  }
  const int q = sh[idx].nq / 4;
  *nb_pad = (nb + q - 1) / q * q;
  return sh[idx];
}

int slot_acquire(dnspir_fleet* f, QSlot& s) {
  if (s.sec_pending) CK(cudaStreamWaitEvent(f->st, s.sec_done, 0));
  s.sec_pending = false;
  return DNSPIR_OK;
}

// End of a call: the main stream waits for every secondary phase, then the host.
int fleet_drain(dnspir_fleet* f) {
  for (auto& s : f->slot)
    if (s.sec_pending) CK(cudaStreamWaitEvent(f->st, s.sec_done, 0));
  CK(cudaStreamSynchronize(f->st));
  CK(cudaStreamSynchronize(f->sec));
  for (auto& s : f->slot) s.sec_pending = false;
  if (f->engine == DNSPIR_ENGINE_TENSOR) {
    uint32_t e = 0;
    CK(cudaMemcpy(&e, f->err_word.p, 4, cudaMemcpyDeviceToHost));
    if (e) {
      CK(cudaMemset(f->err_word.p, 0, 4));
      return fail(DNSPIR_ERR_TIMEOUT, "tensor scan: a pipeline wait gave up");
    }
  }
  return DNSPIR_OK;
}

// Scan of the decoded queries in s.qnat (kernel batch Bk) into s.fin.
int launch_scan(dnspir_fleet* f, QSlot& s, int nb, int Bk) {
  const Group& g1 = f->g1;
  const size_t qv = QV_WORDS_PER_QUERY * g1.n;
  if (f->engine == DNSPIR_ENGINE_TENSOR) {
    int nb_pad = 0;
    const TScanShape& shape = tensor_shape(f, nb, &nb_pad);
    if (nb_pad != Bk) return fail(DNSPIR_ERR_BAD_ARG, "tensor scan batch mismatch");
    if (launch_tscan(f->slabs_dev.as<uint8_t*>(), f->S, s.qnat.as<uint32_t>(), qv, nb, Bk, f->qb.as<uint8_t>(),
                     s.fin.as<uint32_t>(), f->err_word.as<uint32_t>(), g1, slot_maps(f->ctx, g1.log2n), shape, f->st,
                     f->limits, f->tmaps.p))
      return fail(DNSPIR_ERR_BAD_ARG, "tensor scan shape does not fit");
    f->launches += 2;  // query operand + scan
    return DNSPIR_OK;
  }
  if (Bk > nb)  // unused query positions of the kernel batch compute on zeros
    CK(cudaMemsetAsync(s.qnat.as<uint32_t>() + (size_t)nb * qv, 0, (size_t)(Bk - nb) * qv * 4, f->st));
  auto it = f->tuned_cc.find(nb);
  const int per_block = it == f->tuned_cc.end() ? 0 : std::min(it->second, Bk);
  if (launch_scan_batch(f->slabs_dev.as<uint32_t*>(), f->S, s.qnat.as<uint32_t>(), qv, Bk, per_block,
                        s.fin.as<uint32_t>(), g1, slot_maps(f->ctx, g1.log2n), f->st))
    return fail(DNSPIR_ERR_BAD_ARG, "unsupported scan batch");
  f->launches += 1;
  return DNSPIR_OK;
}

}  // namespace

namespace dnspir {

int fleet_ready(dnspir_fleet* f) {
  for (uint32_t d = 0; d < f->D; d++)
    if (!f->ready[d]) return fail(DNSPIR_ERR_NOT_READY, "fleet shard not preprocessed");
  if (f->ap_ver != a_parts_version(f->g1.log2n))
    return fail(DNSPIR_ERR_NOT_READY, "the a-parts changed since the shards were preprocessed: set the shards again");
  return DNSPIR_OK;
}

PolySpec fleet_wire_spec(const dnspir_fleet* f) {
  PolySpec spec;
  memset(&spec, 0, sizeof(spec));
  uint32_t off = 0;
  auto add = [&](int slot, int bits) {
    spec.off[spec.npoly] = off;
    spec.bits[spec.npoly] = bits;
    spec.slot[spec.npoly] = slot;
    spec.npoly++;
    off += f->g1.n * bits / 8;
  };
  add(0, GK_BITS);
  add(1, GK_BITS);
  add(2, PQ_BITS);
  if (f->g1.H == 2) add(3, PQ_BITS);
  add(4, SQ_BITS);
  if (f->g2.H == 2) add(5, SQ_BITS);
  return spec;
}

uint32_t fleet_gk_bytes(const dnspir_fleet* f) { return 2 * f->g1.n * GK_BITS / 8; }

int fleet_kernel_batch(dnspir_fleet* f, int nb) {
  int Bk = pow2_batch(nb);
  if (f->engine == DNSPIR_ENGINE_TENSOR) tensor_shape(f, nb, &Bk);
  return Bk;
}

int fleet_slot_workspace(dnspir_fleet* f, QSlot& s, int Bk, int nb, size_t qbytes) {
  const size_t n = f->g1.n;
  CKR(s.qnat.ensure((size_t)Bk * QV_WORDS_PER_QUERY * n * 4));
  CKR(s.qbrv.ensure((size_t)Bk * QV_WORDS_PER_QUERY * n * 4));
  CKR(s.fin.ensure((size_t)Bk * f->S * 2 * n * SIMD * 4));
  CKR(s.sec_in.ensure((size_t)f->g2.l * CTXT_PARTS * nb * n * 2));
  CKR(s.qdesc.ensure((size_t)nb * sizeof(QDesc)));
  CKR(s.dpin.ensure((size_t)nb * sizeof(QDesc)));
  if (qbytes) CKR(s.qbytes.ensure(qbytes));
  if (f->engine == DNSPIR_ENGINE_TENSOR) CKR(f->qb.ensure(tscan_query_bytes(f->g1, Bk)));
  return DNSPIR_OK;
}

int fleet_secondary_workspace(dnspir_fleet* f, int nb) {
  const Group& g2 = f->g2;
  const size_t n = g2.n;
  const int cmax = std::min(nb, f->sec_chunk);
  const int nlmax = CTXT_PARTS * cmax;
  // the encoder's column transforms (A) are dead before the lift writes secE:
  // A lives at the start of secE's buffer
  const size_t a_bytes = (size_t)g2.l * nlmax * n * 4, e_bytes = (size_t)2 * g2.H * g2.L * nlmax * n * 4;
  CKR(f->ws.Ahat.ensure((size_t)g2.H * g2.L * nlmax * n * 4));
  CKR(f->secE.ensure(std::max(a_bytes, e_bytes)));
  CKR(f->chain_out.ensure((size_t)cmax * g2.H * CTXT_PARTS * 2 * 2 * n * 4));
  return DNSPIR_OK;
}

int fleet_primary_kernels(dnspir_fleet* f, QSlot& s, int nb, int Bk, const uint32_t* sess_nat,
                          const uint32_t* sess_brv, cudaEvent_t scan0, cudaEvent_t scan1) {
  const Group& g1 = f->g1;
  const size_t qv = QV_WORDS_PER_QUERY * g1.n;
  if (s.qbytes.p) {
    launch_decode_query(s.qbytes.as<uint8_t>(), s.qdesc.as<QDesc>(), nb, fleet_wire_spec(f), fleet_gk_bytes(f),
                        s.qnat.as<uint32_t>(), s.qbrv.as<uint32_t>(), qv, sess_nat, sess_brv, g1.log2n, f->ctx->T,
                        f->st);
    f->launches += 1;
  }
  if (scan0) CK(cudaEventRecord(scan0, f->st));
  CKR(launch_scan(f, s, nb, Bk));
  if (scan1) CK(cudaEventRecord(scan1, f->st));
  CK(cudaGetLastError());
  return DNSPIR_OK;
}

int fleet_secondary_kernels(dnspir_fleet* f, QSlot& s, int nb, uint8_t* reply_dev, size_t reply_stride,
                            uint64_t* reply_zq, uint8_t* host_reply) {
  const Group& g2 = f->g2;
  const size_t n = g2.n;
  cudaStream_t st = f->sec;
  const uint32_t l_in = f->S * SIMD;
  // the primary epilogue (scan output -> secondary entries) runs here, on the
  // secondary stream, so that the next group's scan does not wait for it; it
  // reads and writes only this slot's buffers
  launch_primary_epilogue(s.fin.as<uint32_t>(), nb, f->S, f->a_ms.as<uint32_t>(), f->distinct_dev.as<int>(),
                          s.sec_in.as<uint16_t>(), f->sec_chunk, f->g1, slot_maps(f->ctx, f->g1.log2n), f->ctx->T, st);
  f->launches += 1;
  const SlotMaps maps = slot_maps(f->ctx, g2.log2n);
  const ChainConsts cc = chain_consts(f->ctx, g2.log2n, 1);
  const auto tc = f->tuned_chain.find(nb);
  const bool clustered = tc != f->tuned_chain.end() && tc->second;
  for (int c0 = 0; c0 < nb; c0 += f->sec_chunk) {
    const int nc = std::min(f->sec_chunk, nb - c0);
    const int nl = CTXT_PARTS * nc;
    // the last chunk's start: a later group's primary phase may wait for this
    // instead of the whole phase (it then shares the SMs the last chunk leaves idle)
    if (c0 + f->sec_chunk >= nb && s.sec_tail) CK(cudaEventRecord(s.sec_tail, st));
    const uint16_t* in = s.sec_in.as<uint16_t>() + (size_t)c0 * CTXT_PARTS * l_in * n;
    launch_encode_cols(in, f->secE.as<uint32_t>(), g2, l_in, nl, f->ctx->T, st);
    launch_encode_rows(f->secE.as<uint32_t>(), f->ws.Ahat.as<uint32_t>(), g2, l_in, nl, f->ctx->T, st);
    launch_encode_lift(f->ws.Ahat.as<uint32_t>(), f->secE.as<uint32_t>(), g2, nl, 1, maps, f->ctx->T, st);
    launch_secondary_chain(f->secE.as<uint32_t>(), s.qbrv.as<uint32_t>() + (size_t)c0 * QV_WORDS_PER_QUERY * n,
                           QV_WORDS_PER_QUERY * n, nc, f->chain_out.as<uint32_t>(), g2, cc, f->ctx->T, st, clustered);
    launch_reply(f->chain_out.as<uint32_t>(), nc, g2.H, reply_dev ? reply_dev + (size_t)c0 * reply_stride : nullptr,
                 reply_stride, reply_zq ? reply_zq + (size_t)c0 * CTXT_PARTS * 2 * n : nullptr, g2.log2n, f->ctx->T,
                 st);
    f->launches += 5;  // encoder columns, rows, lift; chains; replies
  }
  if (host_reply)
    CK(cudaMemcpyAsync(host_reply, reply_dev, (size_t)nb * dnspir_reply_bytes(), cudaMemcpyDeviceToHost, st));
  CK(cudaGetLastError());
  return DNSPIR_OK;
}

}  // namespace dnspir

namespace {

// One group through both phases with timing events: primary on f->st,
// secondary on f->sec after the primary.  Query bytes and descriptors (or
// decoded vectors) must already be queued on f->st.
int run_group(dnspir_fleet* f, QSlot& s, int nb, int Bk, cudaEvent_t* t, uint8_t* reply_dev, size_t reply_stride,
              uint64_t* reply_zq, uint8_t* host_reply) {
  CKR(fleet_primary_kernels(f, s, nb, Bk, nullptr, nullptr, t[1], t[2]));
  CK(cudaEventRecord(t[3], f->st));
  CK(cudaEventRecord(s.prim_done, f->st));
  s.prim_recorded = true;
  CKR(fleet_secondary_workspace(f, nb));
  CK(cudaStreamWaitEvent(f->sec, s.prim_done, 0));
  CK(cudaEventRecord(t[4], f->sec));
  CKR(fleet_secondary_kernels(f, s, nb, reply_dev, reply_stride, reply_zq, host_reply));
  CK(cudaEventRecord(t[5], f->sec));
  CK(cudaEventRecord(s.sec_done, f->sec));
  s.sec_pending = true;
  return DNSPIR_OK;
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
  uint64_t ap_ver = 0;
  CKR(ctx_consts(c, log2_n, &ap_ver));
  std::unique_ptr<dnspir_fleet> f(new dnspir_fleet());
  f->ap_ver = ap_ver;
  f->device = device;
  f->ctx = c;
  f->g1 = make_group(log2_n, primary_order);
  f->g2 = make_group(log2_n, secondary_order);
  f->S = num_shards;
  f->D = num_distinct;
  {
    // one wave of secondary chain clusters (one-part blocks, two per SM:
    // 2 x 3 x H blocks per query)
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const Group& g2 = f->g2;
    const size_t per_query = ((size_t)2 * g2.H * g2.L + (size_t)g2.H * g2.L) * CTXT_PARTS * g2.n * 4;
    const int wave = std::max(1, 2 * sms / (2 * CTXT_PARTS * (int)g2.H));
    f->sec_chunk = (int)std::max<size_t>(1, std::min<size_t>(wave, SEC_BUDGET / per_query));
  }
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
    CK(cudaEventCreateWithFlags(&s.sec_tail, cudaEventDisableTiming));
  }
  {
    // timing events of the first 64 groups of a call, made now rather than
    // between the launches of a call's first long run of groups
    cudaEvent_t* unused = nullptr;
    CKR(group_events(f.get(), 63, &unused));
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
  if (tensor_layout_supported(f->g1)) {
    // the slabs stay where they are: their tensor maps are made once
    CKR(f->tmaps.ensure(tscan_slab_map_bytes((int)num_shards)));
    std::vector<uint8_t*> hp(num_shards);
    for (uint32_t s = 0; s < num_shards; s++) hp[s] = reinterpret_cast<uint8_t*>(ptrs[s]);
    if (tscan_slab_maps(hp.data(), (int)num_shards, f->g1, f->tmaps.p) != 0) f->tmaps.release();
  }
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
  std::lock_guard<std::mutex> lk(f->mu);
  NOT_SERVING(f);
  if (f->engine == DNSPIR_ENGINE_TENSOR) {
    if (max_batch < 1 || max_batch > TENSOR_MAX_BATCH) return fail(DNSPIR_ERR_BAD_ARG, "batch must be 1..256");
  } else if (!scan_batch_supported((int)max_batch)) {
    return fail(DNSPIR_ERR_BAD_ARG, "batch must be a power of two up to 256");
  }
  f->batch = (int)max_batch;
  return DNSPIR_OK;
}

int dnspir_fleet_set_engine(dnspir_fleet* f, int engine) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  std::lock_guard<std::mutex> lk(f->mu);
  NOT_SERVING(f);
  if (engine != DNSPIR_ENGINE_CUDA_CORES && engine != DNSPIR_ENGINE_TENSOR)
    return fail(DNSPIR_ERR_BAD_ARG, "unknown scan engine");
  if (engine == DNSPIR_ENGINE_TENSOR && !tensor_layout_supported(f->g1))
    return fail(DNSPIR_ERR_BAD_SHAPE, "the tensor layout needs loop_len = N/2 and N >= 256");
  DeviceGuard dg(f->device);
  if (engine == DNSPIR_ENGINE_TENSOR) {
    CKR(f->err_word.ensure(4));
    CK(cudaMemset(f->err_word.p, 0, 4));
  }
  if (engine != f->engine)
    for (uint32_t d = 0; d < f->D; d++) f->ready[d] = false;  // the slab layout changes
  f->engine = engine;
  f->batch = 1;
  f->tuned.clear();
  f->tuned_cc.clear();
  f->tuned_serial.clear();
  f->tuned_chain.clear();
  return DNSPIR_OK;
}

int dnspir_fleet_tune(dnspir_fleet* f, uint32_t batch, double* ms_per_shape, int* chosen) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  std::lock_guard<std::mutex> lk(f->mu);
  NOT_SERVING(f);
  if (f->engine != DNSPIR_ENGINE_TENSOR) return fail(DNSPIR_ERR_BAD_ARG, "tuning applies to the tensor engine");
  if (batch < 1 || batch > (uint32_t)TENSOR_MAX_BATCH) return fail(DNSPIR_ERR_BAD_ARG, "batch must be 1..256");
  CKR(fleet_ready(f));
  DeviceGuard dg(f->device);
  const Group& g1 = f->g1;
  const size_t n = g1.n;
  int count = 0;
  const TScanShape* sh = tscan_shapes(&count);
  const int nb = (int)batch;
  int max_pad = nb;
  for (int i = 0; i < count; i++) {
    const int q = sh[i].nq / 4;
    max_pad = std::max(max_pad, (nb + q - 1) / q * q);
  }
  // zero queries: the scan's time does not depend on the values
  DBuf qnat, out, qb;
  CKR(qnat.ensure((size_t)max_pad * QV_WORDS_PER_QUERY * n * 4));
  CKR(out.ensure((size_t)nb * f->S * 2 * n * SIMD * 4));
  CKR(qb.ensure(tscan_query_bytes(g1, max_pad)));
  CK(cudaMemsetAsync(qnat.p, 0, (size_t)max_pad * QV_WORDS_PER_QUERY * n * 4, f->st));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double best = 1e30;
  int best_i = -1;
  for (int i = 0; i < count; i++) {
    const int q = sh[i].nq / 4;
    const int pad = (nb + q - 1) / q * q;
    double ms = -1;
    // the shape is a candidate when the padding costs at most a factor 2
    if (pad <= 2 * nb || q <= 4) {
      bool ok = true;
      float t = 0, tot = 0;
      for (int r = 0; r < 3 && ok; r++) {
        cudaEventRecord(e0, f->st);
        ok = launch_tscan(f->slabs_dev.as<uint8_t*>(), f->S, qnat.as<uint32_t>(), QV_WORDS_PER_QUERY * n, nb, pad,
                          qb.as<uint8_t>(), out.as<uint32_t>(), f->err_word.as<uint32_t>(), g1,
                          slot_maps(f->ctx, g1.log2n), sh[i], f->st, TScanLimits(), f->tmaps.p) == 0;
        cudaEventRecord(e1, f->st);
        if (ok && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) {
          if (r > 0) tot += t;  // the first run warms up
        } else {
          ok = false;
        }
      }
      cudaGetLastError();
      if (ok) ms = tot / 2;
    }
    if (ms_per_shape) ms_per_shape[i] = ms;
    if (ms > 0 && ms < best) {
      best = ms;
      best_i = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaStreamSynchronize(f->st));
  uint32_t e = 0;
  CK(cudaMemcpy(&e, f->err_word.p, 4, cudaMemcpyDeviceToHost));
  if (e) {
    CK(cudaMemset(f->err_word.p, 0, 4));
    return fail(DNSPIR_ERR_TIMEOUT, "tensor scan: a pipeline wait gave up");
  }
  if (best_i < 0) return fail(DNSPIR_ERR_CUDA, "no tile shape ran");
  f->tuned[nb] = best_i;
  if (chosen) *chosen = best_i;
  return DNSPIR_OK;
}

int dnspir_fleet_tune_pipeline(dnspir_fleet* f, uint32_t batch, double* ms_per_shape, int* chosen) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  uint64_t qlen = 0;
  {
    std::lock_guard<std::mutex> lk(f->mu);
    NOT_SERVING(f);
    if (f->engine != DNSPIR_ENGINE_TENSOR) return fail(DNSPIR_ERR_BAD_ARG, "tuning applies to the tensor engine");
    if (batch < 1 || batch > (uint32_t)TENSOR_MAX_BATCH) return fail(DNSPIR_ERR_BAD_ARG, "batch must be 1..256");
    if (f->g1.log2n != LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_SHAPE, "the wire format is defined for N = 2048");
    CKR(fleet_ready(f));
    qlen = dnspir_query_bytes(f->g1.l, f->g2.l);
  }
  DeviceGuard dg(f->device);
  // zero query bytes (valid wire data) answered in three groups per shape:
  // the first warms up, the other two are timed through both phases
  const int nb = (int)batch, groups = 3;
  const size_t RB = dnspir_reply_bytes();
  DBuf q, r;
  CKR(q.ensure((size_t)nb * groups * qlen));
  CKR(r.ensure((size_t)nb * groups * RB));
  CK(cudaMemset(q.p, 0, (size_t)nb * groups * qlen));
  std::vector<const uint8_t*> ptrs(nb * groups);
  std::vector<uint64_t> lens(nb * groups, qlen);
  for (int i = 0; i < nb * groups; i++) ptrs[i] = q.as<uint8_t>() + (size_t)i * qlen;
  const int old_batch = f->batch;
  const auto old_tuned = f->tuned;
  f->batch = nb;
  int count = 0;
  const TScanShape* sh = tscan_shapes(&count);
  double best = 1e30;
  int best_i = -1;
  int rc = DNSPIR_OK;
  std::vector<std::pair<double, int>> ranked;  // overlap-schedule time per shape that ran
  for (int i = 0; i < count && rc == DNSPIR_OK; i++) {
    const int qg = sh[i].nq / 4;
    const int pad = (nb + qg - 1) / qg * qg;
    double ms = -1;
    // candidates: padding at most a factor 2, and at most 8 query groups per m-tile
    if ((pad <= 2 * nb || qg <= 4) && qg * 8 >= nb) {
      f->tuned[nb] = i;
      rc = dnspir_fleet_process_queries(f, ptrs.data(), lens.data(), (uint32_t)(nb * groups), r.as<uint8_t>(), RB,
                                        nullptr, 1);
      if (rc == DNSPIR_OK) {
        std::lock_guard<std::mutex> lk(f->mu);
        float t = 0;
        cudaEvent_t* t1 = &f->tev[6];
        cudaEvent_t* t2 = &f->tev[12];
        if (cudaEventElapsedTime(&t, t1[0], t2[5]) == cudaSuccess) ms = t / 2;
        cudaGetLastError();
      }
    }
    if (ms_per_shape) ms_per_shape[i] = ms;
    if (ms > 0) ranked.emplace_back(ms, i);
    if (ms > 0 && ms < best) {
      best = ms;
      best_i = i;
    }
  }
  // schedule: the three best shapes again with each group's primary phase
  // waiting for the previous group's secondary phase (1), or for its last
  // chunk (2); keep the fastest shape and schedule (a shape whose small CTAs
  // share SMs well with an overlapping secondary phase is not always the best
  // one when the phases run one after the other)
  int serial = 0;
  std::sort(ranked.begin(), ranked.end());
  for (size_t r0 = 0; r0 < ranked.size() && r0 < 3 && rc == DNSPIR_OK; r0++) {
    const int i = ranked[r0].second;
    for (int sched = 1; sched <= 2 && rc == DNSPIR_OK; sched++) {
      f->tuned[nb] = i;
      f->tuned_serial[nb] = sched;
      rc = dnspir_fleet_process_queries(f, ptrs.data(), lens.data(), (uint32_t)(nb * groups), r.as<uint8_t>(), RB,
                                        nullptr, 1);
      if (rc == DNSPIR_OK) {
        std::lock_guard<std::mutex> lk(f->mu);
        float t = 0;
        if (cudaEventElapsedTime(&t, f->tev[6], f->tev[17]) == cudaSuccess && t / 2 < best) {
          serial = sched;
          best = t / 2;
          best_i = i;
          if (ms_per_shape) ms_per_shape[i] = best;
        }
        cudaGetLastError();
      }
    }
  }
  // chain form: the best shape and schedule again with the two-block-cluster
  // chains at every chunk size (they can share SMs with the next group's scan)
  bool clustered = false;
  if (rc == DNSPIR_OK && best_i >= 0) {
    f->tuned[nb] = best_i;
    f->tuned_serial[nb] = serial;
    f->tuned_chain[nb] = 1;
    rc = dnspir_fleet_process_queries(f, ptrs.data(), lens.data(), (uint32_t)(nb * groups), r.as<uint8_t>(), RB,
                                      nullptr, 1);
    if (rc == DNSPIR_OK) {
      std::lock_guard<std::mutex> lk(f->mu);
      float t = 0;
      if (cudaEventElapsedTime(&t, f->tev[6], f->tev[17]) == cudaSuccess && t / 2 < best) {
        clustered = true;
        best = t / 2;
        if (ms_per_shape) ms_per_shape[best_i] = best;
      }
      cudaGetLastError();
    }
  }
  f->batch = old_batch;
  f->tuned = old_tuned;
  f->tuned_serial.erase(nb);
  f->tuned_chain.erase(nb);
  if (rc != DNSPIR_OK) return rc;
  if (best_i < 0) return fail(DNSPIR_ERR_CUDA, "no tile shape ran");
  f->tuned[nb] = best_i;
  f->tuned_serial[nb] = serial;
  f->tuned_chain[nb] = clustered ? 1 : 0;
  if (chosen) *chosen = best_i;
  return DNSPIR_OK;
}

int dnspir_fleet_tune_cuda_cores(dnspir_fleet* f, uint32_t batch, double* ms_per_tile, int* chosen) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  std::lock_guard<std::mutex> lk(f->mu);
  NOT_SERVING(f);
  if (f->engine != DNSPIR_ENGINE_CUDA_CORES) return fail(DNSPIR_ERR_BAD_ARG, "this tuner applies to the CUDA-core engine");
  if (!scan_batch_supported((int)batch)) return fail(DNSPIR_ERR_BAD_ARG, "batch must be a power of two up to 256");
  CKR(fleet_ready(f));
  DeviceGuard dg(f->device);
  const Group& g1 = f->g1;
  const size_t n = g1.n, qv = QV_WORDS_PER_QUERY * n;
  const int B = (int)batch;
  DBuf qnat, out;
  CKR(qnat.ensure((size_t)B * qv * 4));
  CKR(out.ensure((size_t)B * f->S * 2 * n * SIMD * 4));
  CK(cudaMemsetAsync(qnat.p, 0, (size_t)B * qv * 4, f->st));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  static const int tiles[5] = {1, 2, 4, 8, 16};
  double best = 1e30;
  int best_t = -1;
  for (int i = 0; i < 5; i++) {
    double ms = -1;
    if (tiles[i] <= B && tiles[i] * 16 >= B) {  // at most 16 groups per block row
      float t = 0, tot = 0;
      bool ok = true;
      for (int r = 0; r < 3 && ok; r++) {
        cudaEventRecord(e0, f->st);
        ok = launch_scan_batch(f->slabs_dev.as<uint32_t*>(), f->S, qnat.as<uint32_t>(), qv, B, tiles[i],
                               out.as<uint32_t>(), g1, slot_maps(f->ctx, g1.log2n), f->st) == 0;
        cudaEventRecord(e1, f->st);
        if (ok && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) {
          if (r > 0) tot += t;
        } else {
          ok = false;
        }
      }
      cudaGetLastError();
      if (ok) ms = tot / 2;
    }
    if (ms_per_tile) ms_per_tile[i] = ms;
    if (ms > 0 && ms < best) {
      best = ms;
      best_t = tiles[i];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaStreamSynchronize(f->st));
  if (best_t < 0) return fail(DNSPIR_ERR_CUDA, "no tile ran");
  f->tuned_cc[B] = best_t;
  if (chosen) *chosen = best_t;
  return DNSPIR_OK;
}

int dnspir_fleet_set_schedule(dnspir_fleet* f, uint32_t batch, int schedule) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  std::lock_guard<std::mutex> lk(f->mu);
  NOT_SERVING(f);
  if (batch < 1 || batch > (uint32_t)TENSOR_MAX_BATCH) return fail(DNSPIR_ERR_BAD_ARG, "batch must be 1..256");
  if (schedule < -1 || schedule > 6 || (schedule >= 0 && (schedule & 3) == 3))
    return fail(DNSPIR_ERR_BAD_ARG, "schedule must be -1 or 0, 1, 2 plus optionally 4");
  if (schedule < 0) {
    f->tuned_serial.erase((int)batch);
    f->tuned_chain.erase((int)batch);
  } else {
    f->tuned_serial[(int)batch] = schedule & 3;
    f->tuned_chain[(int)batch] = schedule >> 2;
  }
  return DNSPIR_OK;
}

int dnspir_fleet_get_schedule(dnspir_fleet* f, uint32_t batch, int* schedule) {
  if (!f || !schedule) return fail(DNSPIR_ERR_BAD_ARG, "null fleet or output");
  std::lock_guard<std::mutex> lk(f->mu);
  const auto so = f->tuned_serial.find((int)batch);
  const auto tc = f->tuned_chain.find((int)batch);
  *schedule = (so == f->tuned_serial.end() ? 0 : so->second) + (tc != f->tuned_chain.end() && tc->second ? 4 : 0);
  return DNSPIR_OK;
}

int dnspir_fleet_set_tile(dnspir_fleet* f, uint32_t batch, int shape_index) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  std::lock_guard<std::mutex> lk(f->mu);
  NOT_SERVING(f);
  if (f->engine != DNSPIR_ENGINE_TENSOR) return fail(DNSPIR_ERR_BAD_ARG, "tiles apply to the tensor engine");
  if (batch < 1 || batch > (uint32_t)TENSOR_MAX_BATCH) return fail(DNSPIR_ERR_BAD_ARG, "batch must be 1..256");
  int count = 0;
  tscan_shapes(&count);
  if (shape_index < 0) {
    f->tuned.erase((int)batch);
    return DNSPIR_OK;
  }
  if (shape_index >= count) return fail(DNSPIR_ERR_BAD_ARG, "no such tile shape");
  f->tuned[(int)batch] = shape_index;
  return DNSPIR_OK;
}

int dnspir_fleet_scan(dnspir_fleet* f, const uint32_t* qnat_dev, uint32_t nq, uint32_t* out_dev) {
  if (!f || (nq && (!qnat_dev || !out_dev))) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(f->mu);
  NOT_SERVING(f);
  CKR(fleet_ready(f));
  DeviceGuard dg(f->device);
  const Group& g1 = f->g1;
  const size_t n = g1.n, qv = QV_WORDS_PER_QUERY * n;
  const size_t per_out = (size_t)f->S * 2 * n * SIMD;
  QSlot& s = f->slot[0];
  CKR(slot_acquire(f, s));
  for (uint32_t g0 = 0; g0 < nq; g0 += f->batch) {
    const int nb = (int)std::min<uint32_t>(f->batch, nq - g0);
    const int Bk = fleet_kernel_batch(f, nb);
    CKR(fleet_slot_workspace(f, s, Bk, nb, 0));
    CK(cudaMemcpyAsync(s.qnat.p, qnat_dev + g0 * qv, (size_t)nb * qv * 4, cudaMemcpyDeviceToDevice, f->st));
    CKR(launch_scan(f, s, nb, Bk));
    CK(cudaMemcpyAsync(out_dev + g0 * per_out, s.fin.p, (size_t)nb * per_out * 4, cudaMemcpyDeviceToDevice, f->st));
  }
  CK(cudaGetLastError());
  return fleet_drain(f);
}

int dnspir_fleet_set_wait_limit(dnspir_fleet* f, uint64_t wait_ns, int withhold_chunk) {
  if (!f) return fail(DNSPIR_ERR_BAD_ARG, "null fleet");
  std::lock_guard<std::mutex> lk(f->mu);
  NOT_SERVING(f);
  if (withhold_chunk < -1) return fail(DNSPIR_ERR_BAD_ARG, "withhold_chunk must be -1 or a chunk index");
  f->limits.wait_ns = wait_ns;
  f->limits.withhold = withhold_chunk;
  return DNSPIR_OK;
}

int dnspir_tscan_shapes(int* nq, int* mtpc, int* stages, int* persistent, int max) {
  int count = 0;
  const TScanShape* sh = tscan_shapes(&count);
  for (int i = 0; i < count && i < max; i++) {
    if (nq) nq[i] = sh[i].nq;
    if (mtpc) mtpc[i] = sh[i].mtpc;
    if (stages) stages[i] = sh[i].stages;
    if (persistent) persistent[i] = sh[i].persistent;
  }
  return count;
}

int dnspir_fleet_set_shards(dnspir_fleet* f, uint32_t first, uint32_t count, const uint16_t* entries,
                            int entries_on_device) {
  if (!f || !entries) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(f->mu);
  NOT_SERVING(f);
  if ((uint64_t)first + count > f->D) return fail(DNSPIR_ERR_BAD_ARG, "distinct shard index out of range");
  DeviceGuard dg(f->device);
  {
    // shards preprocessed under other a-parts cannot be mixed with these
    uint64_t ver = 0;
    CKR(ctx_consts(f->ctx, f->g1.log2n, &ver));
    if (ver != f->ap_ver)
      for (uint32_t d = 0; d < f->D; d++) f->ready[d] = false;
    f->ap_ver = ver;
  }
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
    if (f->engine == DNSPIR_ENGINE_TENSOR) {
      // preprocess into lane-layout scratch, then re-tile into the fleet slab
      const uint32_t tb = 4;
      const size_t words = slab_words(f->g1);
      CKR(f->tmp_lane.ensure((size_t)std::min(cnt, tb) * words * 4));
      for (uint32_t c0 = 0; c0 < cnt; c0 += tb) {
        const uint32_t cc = std::min(tb, cnt - c0);
        std::vector<uint32_t*> tmp(cc);
        for (uint32_t i = 0; i < cc; i++) tmp[i] = f->tmp_lane.as<uint32_t>() + i * words;
        CKR(preprocess_shards(f->ctx, f->g1, 0, tmp.data(), (int)cc, src + (size_t)c0 * per,
                              f->a_zq.as<uint64_t>() + (size_t)(first + b0 + c0) * SIMD * f->g1.n,
                              f->a_ms.as<uint32_t>() + (size_t)(first + b0 + c0) * SIMD * f->g1.n, f->ws, f->st));
        for (uint32_t i = 0; i < cc; i++)
          launch_retile(tmp[i], reinterpret_cast<uint8_t*>(f->slabs[first + b0 + c0 + i]), f->g1, f->st);
      }
      CK(cudaStreamSynchronize(f->st));
      f->tmp_lane.release();
    } else {
      CKR(preprocess_shards(f->ctx, f->g1, 0, &f->slabs[first + b0], (int)cnt, src,
                            f->a_zq.as<uint64_t>() + (size_t)(first + b0) * SIMD * f->g1.n,
                            f->a_ms.as<uint32_t>() + (size_t)(first + b0) * SIMD * f->g1.n, f->ws, f->st));
    }
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
  NOT_SERVING(f);
  CKR(fleet_ready(f));
  const Group& g1 = f->g1;
  const Group& g2 = f->g2;
  if (g1.log2n != LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_SHAPE, "the wire format is defined for N = 2048");
  DeviceGuard dg(f->device);
  const uint64_t want = dnspir_query_bytes(g1.l, g2.l);
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
    const int Bk = fleet_kernel_batch(f, nb);
    QSlot& s = f->slot[gi & 1];
    cudaEvent_t* t = nullptr;
    CKR(group_events(f, gi, &t));
    CKR(slot_acquire(f, s));
    // schedule: unless this group size overlaps, its primary phase waits for
    // the previous group's secondary phase (the two phases then do not share
    // SMs), or for that phase to reach its last chunk
    auto so = f->tuned_serial.find(nb);
    const QSlot& prev = f->slot[(gi & 1) ^ 1];
    if (so != f->tuned_serial.end() && so->second && prev.sec_pending)
      CK(cudaStreamWaitEvent(f->st, so->second == 2 ? prev.sec_tail : prev.sec_done, 0));
    CKR(fleet_slot_workspace(f, s, Bk, nb, (size_t)nb * want));
    // host staging of the slot may still feed the copies of the group two back
    if (s.prim_recorded) CK(cudaEventSynchronize(s.prim_done));
    QDesc* d = s.dpin.as<QDesc>();
    for (int q = 0; q < nb; q++) d[q] = QDesc{(uint32_t)(q * want), -1};
    if (!on_device) {
      CKR(s.qpin.ensure((size_t)nb * want));
      CKR(s.reply_dev.ensure((size_t)nb * RB));
      for (int q = 0; q < nb; q++) memcpy((uint8_t*)s.qpin.p + (size_t)q * want, queries[ok[g0 + q]], want);
    }
    CK(cudaEventRecord(t[0], f->st));
    CK(cudaMemcpyAsync(s.qdesc.p, s.dpin.p, (size_t)nb * sizeof(QDesc), cudaMemcpyHostToDevice, f->st));
    if (!on_device) {
      CK(cudaMemcpyAsync(s.qbytes.p, s.qpin.p, (size_t)nb * want, cudaMemcpyHostToDevice, f->st));
    } else {
      for (int q = 0; q < nb; q++)
        CK(cudaMemcpyAsync(s.qbytes.as<uint8_t>() + (size_t)q * want, queries[ok[g0 + q]], want,
                           cudaMemcpyDeviceToDevice, f->st));
    }
    // replies of a group are contiguous in the caller's buffer only when its
    // queries are; otherwise (a rejected query inside the group) go through
    // the staging path
    bool contiguous = true;
    for (int q = 1; q < nb; q++) contiguous &= ok[g0 + q] == ok[g0] + q;
    if (on_device && contiguous) {
      CKR(run_group(f, s, nb, Bk, t, replies + (size_t)ok[g0] * reply_stride, reply_stride, nullptr, nullptr));
    } else if (on_device) {
      CKR(s.reply_dev.ensure((size_t)nb * RB));
      CKR(run_group(f, s, nb, Bk, t, s.reply_dev.as<uint8_t>(), RB, nullptr, nullptr));
      for (int q = 0; q < nb; q++)
        CK(cudaMemcpyAsync(replies + (size_t)ok[g0 + q] * reply_stride, s.reply_dev.as<uint8_t>() + q * RB, RB,
                           cudaMemcpyDeviceToDevice, f->sec));
    } else {
      CKR(run_group(f, s, nb, Bk, t, s.reply_dev.as<uint8_t>(), RB, nullptr, (uint8_t*)f->rpin.p + g0 * RB));
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
  NOT_SERVING(f);
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
  // a private slot without query bytes: the ring elements go straight to the
  // decoded vectors
  QSlot s;
  CK(cudaEventCreateWithFlags(&s.prim_done, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&s.sec_done, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&s.sec_tail, cudaEventDisableTiming));
  for (auto& o : f->slot) CKR(slot_acquire(f, o));
  const int Bk = fleet_kernel_batch(f, 1);
  cudaEvent_t* t = nullptr;
  CKR(group_events(f, 0, &t));
  CKR(fleet_slot_workspace(f, s, Bk, 1, 0));
  CKR(f->qzq.ensure(z.size() * 8));
  CKR(f->reply_zq.ensure((size_t)CTXT_PARTS * 2 * n * 8));
  CK(cudaEventRecord(t[0], f->st));
  CK(cudaMemcpyAsync(f->qzq.p, z.data(), z.size() * 8, cudaMemcpyHostToDevice, f->st));
  launch_ring_to_ntt(f->qzq.as<uint64_t>(), 6, s.qnat.as<uint32_t>(), s.qbrv.as<uint32_t>(), f->g1.log2n, f->ctx->T,
                     f->st);
  CKR(run_group(f, s, 1, Bk, t, nullptr, 0, f->reply_zq.as<uint64_t>(), nullptr));
  f->q_group.assign(1, 0);
  CK(cudaStreamWaitEvent(f->st, s.sec_done, 0));
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
  NOT_SERVING(f);
  f->st = s ? (cudaStream_t)s : f->own;
  return DNSPIR_OK;
}

int dnspir_fleet_launch_count(dnspir_fleet* f, uint64_t* count) {
  if (!f || !count) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(f->mu);
  *count = f->launches;
  return DNSPIR_OK;
}

uint64_t dnspir_fleet_slab_bytes(dnspir_fleet* f) { return f ? (uint64_t)f->D * slab_words(f->g1) * 4 : 0; }

int dnspir_fleet_destroy(dnspir_fleet* f) {
  if (!f) return DNSPIR_OK;
  if (f->serving) return fail(DNSPIR_ERR_BAD_ARG, "the fleet is attached to a running server");
  DeviceGuard dg(f->device);
  cudaStreamSynchronize(f->st);
  cudaStreamSynchronize(f->sec);
  delete f;
  return DNSPIR_OK;
}

}  // extern "C"
