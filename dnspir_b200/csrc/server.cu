// server.cu -- the serving loop: continuous batching of queries over several
// resident databases (fleets) on one device.
//
// The reference answers each connection on its own OS thread with
// process_query (dns/server.rs:789, pir_wrapper.rs:328); here one worker
// thread owns the device work of every database:
//   * requests are queued per database as they are submitted;
//   * whenever one of a database's two buffer slots is free, the worker takes
//     every pending request of that database up to its admitted group size
//     (continuous batching: requests that arrive while other groups are on the
//     device join the next group), stages their bytes in pinned memory and
//     launches the group: primary phase on the fleet's main stream, secondary
//     phase on its high-priority stream, so groups of one database pipeline
//     and groups of different databases overlap on the device;
//   * each group size's primary and secondary launch sequences are captured
//     once as CUDA graphs (the first group of a size runs directly, which also
//     performs every lazy initialisation) and replayed afterwards;
//   * completion is observed with event queries; replies are copied out of
//     the slot's pinned buffer and the request is marked done.
// Group sizes are admitted by free device memory: a database's group size is
// halved until its two slots and the secondary workspace fit.  Each database
// gets its own pair of streams for the session, prioritised by database size
// (smaller databases first, and within a database the secondary phase above
// the scans), so short groups of small databases are dispatched between the
// blocks of long scans of large ones.  An optional batching window per
// database holds a group until it has min_batch queries or its oldest query
// has waited max_wait, so that cheap databases do not launch near-empty groups.  Sessions keep
// a client's decoded Galois keys on the device; a query of a session omits the
// two key polynomials from its bytes.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fleet_impl.h"

using namespace dnspir;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  uint32_t db = 0;
  int32_t session = -1;
  std::vector<uint8_t> bytes;
  std::vector<uint8_t> reply;
  int status = -1;  // -1 pending, else a DNSPIR status
  double t_submit = 0, t_done = 0;
};

struct InFlight {
  bool busy = false;
  std::vector<uint64_t> tickets;
};

struct Db {
  dnspir_fleet* f = nullptr;
  cudaStream_t saved_st = nullptr, saved_sec = nullptr;  // the fleet's own streams, restored at stop
  cudaStream_t st = nullptr, sec = nullptr;              // serving streams (priority by database size)
  int min_batch = 1;                                     // batching window: launch at this many pending
  double max_wait_s = 0;                                 // ... or when the oldest has waited this long
  int max_batch = 1;  // requested
  int admitted = 1;   // after memory admission
  int bk_max = 1;
  std::deque<uint64_t> pending;
  InFlight inflight[2];
  int next_slot = 0;
  std::vector<double> lat_ms;
  uint64_t completed = 0;
  uint64_t groups = 0, graph_groups = 0;
};

}  // namespace

struct dnspir_server {
  int device = 0;
  std::vector<std::unique_ptr<Db>> dbs;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::atomic<bool> running{false};
  bool use_graphs = true;
  std::unordered_map<uint64_t, Request> reqs;
  uint64_t next_ticket = 1;
  // session cache: decoded Galois keys [session][slot 0,1][factor][N], natural and bit-reversed
  DBuf sess_nat, sess_brv, sess_desc;
  std::vector<int> sess_refs;  // -1 free, else requests in flight + 1 while open
  std::vector<bool> sess_closing;
  uint32_t sess_cap = 0;
  cudaStream_t sess_stream = nullptr;
  uint32_t rr = 0;  // round-robin position over databases
  ~dnspir_server() {
    if (sess_stream) cudaStreamDestroy(sess_stream);
  }
};

namespace {

const uint32_t N_WIRE = 1u << LOG2_N_MAX;

uint64_t full_query_bytes(const dnspir_fleet* f) { return dnspir_query_bytes(f->g1.l, f->g2.l); }

// Workspace of both slots and the secondary phase for groups up to nb.
size_t group_bytes(dnspir_fleet* f, int nb, int Bk) {
  const size_t n = f->g1.n;
  const Group& g2 = f->g2;
  size_t slot = (size_t)2 * Bk * QV_WORDS_PER_QUERY * n * 4 + (size_t)Bk * f->S * 2 * n * SIMD * 4 +
                (size_t)g2.l * CTXT_PARTS * nb * n * 2 + (size_t)nb * (full_query_bytes(f) + dnspir_reply_bytes());
  const int cmax = std::min(nb, f->sec_chunk);
  const size_t sec = (size_t)CTXT_PARTS * cmax * n * 4 *
                     ((size_t)g2.H * g2.L + std::max<size_t>(g2.l, (size_t)2 * g2.H * g2.L) + (size_t)g2.H * 4);
  size_t qb = f->engine == DNSPIR_ENGINE_TENSOR ? tscan_query_bytes(f->g1, Bk) : 0;
  return 2 * slot + sec + qb;
}

int bk_max_of(dnspir_fleet* f, int nb) {
  int m = 1;
  for (int b = 1; b <= nb; b++) m = std::max(m, fleet_kernel_batch(f, b));
  return m;
}

// Size every buffer a group of up to db.admitted queries touches, so that
// captured graphs never see a reallocation.
int presize(Db& db) {
  dnspir_fleet* f = db.f;
  const int nb = db.admitted;
  const size_t RB = dnspir_reply_bytes();
  for (auto& s : f->slot) {
    CKR(fleet_slot_workspace(f, s, db.bk_max, nb, (size_t)nb * full_query_bytes(f)));
    CKR(s.qpin.ensure((size_t)nb * full_query_bytes(f)));
    CKR(s.reply_dev.ensure((size_t)nb * RB));
    CKR(s.rpin.ensure((size_t)nb * RB));
  }
  CKR(fleet_secondary_workspace(f, nb));
  return DNSPIR_OK;
}

// Group sizes come from a fixed set -- 1, 2, 3, 4, 6, 8, 12, ... (powers of
// two and 1.5 times powers of two) and the admitted maximum -- so that at most
// about 2 log2(max) sizes ever run, each captured once per slot: the first
// group of a size runs directly and holds the worker while its graphs are
// captured and instantiated.  The smallest member not below n (n <= cap); a
// group is padded up to it rather than leaving queries for the next group,
// since a group's pass over the slabs costs the same whatever its size.
int group_size_ceil(int n, int cap) {
  for (int p = 1; p < cap; p *= 2) {
    if (p >= n) return p;
    if (p >= 2 && p + p / 2 >= n && p + p / 2 < cap) return p + p / 2;
  }
  return cap;
}

// Launch one group of db on slot k: staging, H2D, primary and secondary
// phases (graphs when captured), completion event.
int launch_group(dnspir_server* sv, Db& db, int k, const std::vector<Request*>& rq) {
  dnspir_fleet* f = db.f;
  QSlot& s = f->slot[k];
  const int nb = (int)rq.size();
  const int Bk = fleet_kernel_batch(f, nb);
  const size_t RB = dnspir_reply_bytes();
  QDesc* d = s.dpin.as<QDesc>();
  size_t off = 0;
  for (int q = 0; q < nb; q++) {
    memcpy((uint8_t*)s.qpin.p + off, rq[q]->bytes.data(), rq[q]->bytes.size());
    d[q] = QDesc{(uint32_t)off, rq[q]->session};
    off += rq[q]->bytes.size();
  }
  CK(cudaMemcpyAsync(s.qdesc.p, s.dpin.p, (size_t)nb * sizeof(QDesc), cudaMemcpyHostToDevice, f->st));
  CK(cudaMemcpyAsync(s.qbytes.p, s.qpin.p, off, cudaMemcpyHostToDevice, f->st));
  const uint32_t* sn = sv->sess_nat.as<uint32_t>();
  const uint32_t* sb = sv->sess_brv.as<uint32_t>();
  auto gp = s.gprim.find(nb);
  auto gs = s.gsec.find(nb);
  const bool graphs = sv->use_graphs && gp != s.gprim.end() && gs != s.gsec.end();
  if (graphs) {
    CK(cudaGraphLaunch(gp->second, f->st));
    CK(cudaEventRecord(s.prim_done, f->st));
    CK(cudaStreamWaitEvent(f->sec, s.prim_done, 0));
    CK(cudaGraphLaunch(gs->second, f->sec));
    db.graph_groups++;
  } else {
    CKR(fleet_primary_kernels(f, s, nb, Bk, sn, sb, nullptr, nullptr));
    CK(cudaEventRecord(s.prim_done, f->st));
    CK(cudaStreamWaitEvent(f->sec, s.prim_done, 0));
    CKR(fleet_secondary_kernels(f, s, nb, s.reply_dev.as<uint8_t>(), RB, nullptr, s.rpin.as<uint8_t>()));
  }
  CK(cudaEventRecord(s.sec_done, f->sec));
  db.groups++;
  if (sv->use_graphs && !graphs) {
    // capture this size for the next groups (the direct run above performed
    // every lazy initialisation; capture records without executing)
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    CK(cudaStreamBeginCapture(f->st, cudaStreamCaptureModeRelaxed));
    const int r1 = fleet_primary_kernels(f, s, nb, Bk, sn, sb, nullptr, nullptr);
    CK(cudaStreamEndCapture(f->st, &g));
    CKR(r1);
    CK(cudaGraphInstantiate(&ge, g, 0));
    cudaGraphDestroy(g);
    s.gprim[nb] = ge;
    CK(cudaStreamBeginCapture(f->sec, cudaStreamCaptureModeRelaxed));
    const int r2 = fleet_secondary_kernels(f, s, nb, s.reply_dev.as<uint8_t>(), RB, nullptr, s.rpin.as<uint8_t>());
    CK(cudaStreamEndCapture(f->sec, &g));
    CKR(r2);
    CK(cudaGraphInstantiate(&ge, g, 0));
    cudaGraphDestroy(g);
    s.gsec[nb] = ge;
  }
  return DNSPIR_OK;
}

void finish_group(dnspir_server* sv, Db& db, int k, int status) {
  dnspir_fleet* f = db.f;
  QSlot& s = f->slot[k];
  const size_t RB = dnspir_reply_bytes();
  const double t = now_s();
  std::lock_guard<std::mutex> lk(sv->mu);
  auto& inf = db.inflight[k];
  for (size_t q = 0; q < inf.tickets.size(); q++) {
    auto it = sv->reqs.find(inf.tickets[q]);
    if (it == sv->reqs.end()) continue;
    Request& r = it->second;
    if (status == DNSPIR_OK) r.reply.assign(s.rpin.as<uint8_t>() + q * RB, s.rpin.as<uint8_t>() + (q + 1) * RB);
    r.status = status;
    r.t_done = t;
    r.bytes.clear();
    r.bytes.shrink_to_fit();
    if (r.session >= 0 && sv->sess_refs[r.session] > 0) {
      sv->sess_refs[r.session]--;
      if (sv->sess_refs[r.session] == 0 && sv->sess_closing[r.session]) {
        sv->sess_refs[r.session] = -1;
        sv->sess_closing[r.session] = false;
      }
    }
    db.lat_ms.push_back((t - r.t_submit) * 1e3);
    db.completed++;
  }
  inf.tickets.clear();
  inf.busy = false;
  sv->done_cv.notify_all();
}

void worker_main(dnspir_server* sv) {
  cudaSetDevice(sv->device);
  for (;;) {
    bool progress = false, idle = true;
    // completions
    for (auto& dbp : sv->dbs) {
      Db& db = *dbp;
      for (int k = 0; k < 2; k++) {
        if (!db.inflight[k].busy) continue;
        idle = false;
        const cudaError_t e = cudaEventQuery(db.f->slot[k].sec_done);
        if (e == cudaErrorNotReady) continue;
        int status = DNSPIR_OK;
        if (e != cudaSuccess) {
          cudaGetLastError();
          status = DNSPIR_ERR_CUDA;
        } else if (db.f->engine == DNSPIR_ENGINE_TENSOR) {
          uint32_t w = 0;
          if (cudaMemcpy(&w, db.f->err_word.p, 4, cudaMemcpyDeviceToHost) != cudaSuccess || w) {
            cudaMemset(db.f->err_word.p, 0, 4);
            status = DNSPIR_ERR_TIMEOUT;
          }
        }
        finish_group(sv, db, k, status);
        progress = true;
      }
    }
    // admissions, round robin over databases
    const uint32_t nd = (uint32_t)sv->dbs.size();
    for (uint32_t i = 0; i < nd; i++) {
      Db& db = *sv->dbs[(sv->rr + i) % nd];
      const int k = db.next_slot;
      if (db.inflight[k].busy) continue;
      std::vector<Request*> rq;
      std::vector<uint64_t> tk;
      {
        std::lock_guard<std::mutex> lk(sv->mu);
        // batching window: wait for min_batch pending queries unless the
        // oldest has waited max_wait_s (or the server is draining)
        if ((int)db.pending.size() < std::min(db.min_batch, db.admitted) && sv->running.load()) {
          auto it = db.pending.empty() ? sv->reqs.end() : sv->reqs.find(db.pending.front());
          if (it == sv->reqs.end() || now_s() - it->second.t_submit < db.max_wait_s) continue;
        }
        while (!db.pending.empty() && (int)rq.size() < db.admitted) {
          const uint64_t t = db.pending.front();
          db.pending.pop_front();
          auto it = sv->reqs.find(t);
          if (it == sv->reqs.end()) continue;
          rq.push_back(&it->second);
          tk.push_back(t);
        }
      }
      if (rq.empty()) continue;
      // fill the group up to the next size of the set with copies of its last
      // query; their replies go to ticket 0, which no request has
      for (int target = group_size_ceil((int)rq.size(), db.admitted); (int)rq.size() < target;) {
        rq.push_back(rq.back());
        tk.push_back(0);
      }
      idle = false;
      db.inflight[k].busy = true;
      db.inflight[k].tickets = tk;
      db.next_slot ^= 1;
      const int r = launch_group(sv, db, k, rq);
      if (r != DNSPIR_OK) {
        cudaGetLastError();
        cudaStreamSynchronize(db.f->st);
        cudaStreamSynchronize(db.f->sec);
        finish_group(sv, db, k, r);
      }
      progress = true;
    }
    sv->rr++;
    if (!progress) {
      std::unique_lock<std::mutex> lk(sv->mu);
      bool pending = false;
      for (auto& dbp : sv->dbs) pending |= !dbp->pending.empty();
      if (!sv->running.load() && !pending && idle) break;
      // wake on a submission, or poll the device again shortly
      sv->cv.wait_for(lk, std::chrono::microseconds(idle && !pending ? 2000 : 50));
    }
  }
}

}  // namespace

extern "C" {

int dnspir_server_create(int device, uint32_t max_sessions, dnspir_server** out) {
  if (!out) return fail(DNSPIR_ERR_BAD_ARG, "null output");
  *out = nullptr;
  DeviceCtx* c = nullptr;
  CKR(get_ctx(device, &c));
  DeviceGuard dg(device);
  std::unique_ptr<dnspir_server> sv(new dnspir_server());
  sv->device = device;
  sv->sess_cap = max_sessions;
  if (max_sessions) {
    CKR(sv->sess_nat.ensure((size_t)max_sessions * 4 * N_WIRE * 4));
    CKR(sv->sess_brv.ensure((size_t)max_sessions * 4 * N_WIRE * 4));
  }
  CKR(sv->sess_desc.ensure(sizeof(QDesc)));
  sv->sess_refs.assign(max_sessions, -1);
  sv->sess_closing.assign(max_sessions, false);
  CK(cudaStreamCreateWithFlags(&sv->sess_stream, cudaStreamNonBlocking));
  *out = sv.release();
  return DNSPIR_OK;
}

int dnspir_server_add_db(dnspir_server* sv, dnspir_fleet* f, uint32_t max_batch, uint32_t* db_id) {
  if (!sv || !f || !db_id) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  if (sv->running.load()) return fail(DNSPIR_ERR_BAD_ARG, "add databases before dnspir_server_start");
  if (f->device != sv->device) return fail(DNSPIR_ERR_BAD_ARG, "the fleet lives on another device");
  if (f->g1.log2n != LOG2_N_MAX) return fail(DNSPIR_ERR_BAD_SHAPE, "the wire format is defined for N = 2048");
  for (auto& d : sv->dbs)
    if (d->f == f) return fail(DNSPIR_ERR_BAD_ARG, "fleet already added");
  {
    std::lock_guard<std::mutex> lk(f->mu);
    CKR(fleet_ready(f));
  }
  const int maxb = 256;
  if (max_batch < 1 || (int)max_batch > maxb) return fail(DNSPIR_ERR_BAD_ARG, "max_batch out of range for the engine");
  if (f->engine == DNSPIR_ENGINE_CUDA_CORES && (max_batch & (max_batch - 1)))
    return fail(DNSPIR_ERR_BAD_ARG, "the CUDA-core engine takes power-of-two groups");
  std::unique_ptr<Db> db(new Db());
  db->f = f;
  db->max_batch = (int)max_batch;
  *db_id = (uint32_t)sv->dbs.size();
  sv->dbs.push_back(std::move(db));
  return DNSPIR_OK;
}

int dnspir_server_set_batching(dnspir_server* sv, uint32_t db_id, uint32_t min_batch, uint32_t max_wait_us) {
  if (!sv) return fail(DNSPIR_ERR_BAD_ARG, "null server");
  if (db_id >= sv->dbs.size()) return fail(DNSPIR_ERR_BAD_ARG, "no such database");
  if (min_batch < 1) return fail(DNSPIR_ERR_BAD_ARG, "min_batch must be at least 1");
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->dbs[db_id]->min_batch = (int)min_batch;
  sv->dbs[db_id]->max_wait_s = max_wait_us * 1e-6;
  return DNSPIR_OK;
}

int dnspir_server_start(dnspir_server* sv, int use_graphs) {
  if (!sv) return fail(DNSPIR_ERR_BAD_ARG, "null server");
  if (sv->running.load()) return fail(DNSPIR_ERR_BAD_ARG, "already running");
  if (sv->dbs.empty()) return fail(DNSPIR_ERR_BAD_ARG, "no database added");
  DeviceGuard dg(sv->device);
  sv->use_graphs = use_graphs != 0;
  // admission by device memory: halve a database's group size until its
  // workspace fits beside what the others already hold (1 GiB kept free)
  for (auto& dbp : sv->dbs) {
    Db& db = *dbp;
    dnspir_fleet* f = db.f;
    std::lock_guard<std::mutex> lk(f->mu);
    for (int nb = db.max_batch;; nb = nb / 2) {
      if (nb < 1) return fail(DNSPIR_ERR_OOM, "no group size fits in device memory");
      const int bk = bk_max_of(f, nb);
      size_t fr = 0, tot = 0;
      CK(cudaMemGetInfo(&fr, &tot));
      if (group_bytes(f, nb, bk) + ((size_t)1 << 30) <= fr || nb == 1) {
        db.admitted = nb;
        db.bk_max = bk;
        break;
      }
    }
    CKR(presize(db));
    for (auto& s : f->slot) s.drop_graphs();
  }
  {
    // serving streams: rank databases by slab words per query (smallest first);
    // each database's secondary phase above its own scans
    int least = 0, greatest = 0;
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    std::vector<size_t> order(sv->dbs.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    auto work = [&](size_t i) { return (double)sv->dbs[i]->f->S * slab_words(sv->dbs[i]->f->g1); };
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return work(a) < work(b); });
    for (size_t k = 0; k < order.size(); k++) {
      Db& db = *sv->dbs[order[k]];
      const int p_sec = std::min(least, greatest + 2 * (int)k), p_st = std::min(least, greatest + 2 * (int)k + 1);
      CK(cudaStreamCreateWithPriority(&db.sec, cudaStreamNonBlocking, p_sec));
      CK(cudaStreamCreateWithPriority(&db.st, cudaStreamNonBlocking, p_st));
      db.saved_st = db.f->st;
      db.saved_sec = db.f->sec;
      db.f->st = db.st;
      db.f->sec = db.sec;
      db.f->serving = true;
    }
  }
  CK(cudaDeviceSynchronize());
  sv->running = true;
  sv->worker = std::thread(worker_main, sv);
  return DNSPIR_OK;
}

int dnspir_server_open_session(dnspir_server* sv, const uint8_t* gk_bytes, uint64_t len, uint64_t* session) {
  if (!sv || !gk_bytes || !session) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  const uint64_t want = 2ull * N_WIRE * GK_BITS / 8;
  if (len != want) return fail(DNSPIR_ERR_BAD_SIZE, "Galois-key bytes: two 50-bit polynomials of N = 2048");
  int idx = -1;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    for (uint32_t i = 0; i < sv->sess_cap; i++)
      if (sv->sess_refs[i] < 0) {
        idx = (int)i;
        sv->sess_refs[i] = 0;  // reserved, not yet open
        break;
      }
  }
  if (idx < 0) return fail(DNSPIR_ERR_OOM, "no free session slot");
  DeviceGuard dg(sv->device);
  DeviceCtx* c = nullptr;
  CKR(get_ctx(sv->device, &c));
  // decode the two key polynomials straight into the session's cache entry
  PolySpec spec;
  memset(&spec, 0, sizeof(spec));
  spec.npoly = 2;
  spec.off[1] = N_WIRE * GK_BITS / 8;
  spec.bits[0] = spec.bits[1] = GK_BITS;
  spec.slot[0] = 0;
  spec.slot[1] = 1;
  DBuf bytes;
  CKR(bytes.ensure(want));
  const QDesc d{0, -1};
  CK(cudaMemcpyAsync(bytes.p, gk_bytes, want, cudaMemcpyHostToDevice, sv->sess_stream));
  CK(cudaMemcpyAsync(sv->sess_desc.p, &d, sizeof(d), cudaMemcpyHostToDevice, sv->sess_stream));
  launch_decode_query(bytes.as<uint8_t>(), sv->sess_desc.as<QDesc>(), 1, spec, 0,
                      sv->sess_nat.as<uint32_t>() + (size_t)idx * 4 * N_WIRE,
                      sv->sess_brv.as<uint32_t>() + (size_t)idx * 4 * N_WIRE, 4 * N_WIRE, nullptr, nullptr,
                      LOG2_N_MAX, c->T, sv->sess_stream);
  CK(cudaStreamSynchronize(sv->sess_stream));
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->sess_refs[idx] = 1;  // open
  }
  *session = (uint64_t)idx;
  return DNSPIR_OK;
}

int dnspir_server_close_session(dnspir_server* sv, uint64_t session) {
  if (!sv) return fail(DNSPIR_ERR_BAD_ARG, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  if (session >= sv->sess_cap || sv->sess_refs[session] < 1 || sv->sess_closing[session])
    return fail(DNSPIR_ERR_BAD_ARG, "no such open session");
  sv->sess_refs[session]--;  // drop the open reference; in-flight requests keep theirs
  if (sv->sess_refs[session] == 0)
    sv->sess_refs[session] = -1;
  else
    sv->sess_closing[session] = true;
  return DNSPIR_OK;
}

int dnspir_server_submit(dnspir_server* sv, uint32_t db_id, int64_t session, const uint8_t* query, uint64_t len,
                         uint64_t* ticket) {
  if (!sv || !query || !ticket) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  if (db_id >= sv->dbs.size()) return fail(DNSPIR_ERR_BAD_ARG, "no such database");
  Db& db = *sv->dbs[db_id];
  const uint64_t full = full_query_bytes(db.f);
  const uint64_t want = session >= 0 ? full - fleet_gk_bytes(db.f) : full;
  if (len != want) return fail(DNSPIR_ERR_BAD_SIZE, "query length does not match the database shape");
  Request r;
  r.db = db_id;
  r.session = (int32_t)session;
  r.bytes.assign(query, query + len);
  r.t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (!sv->running.load()) return fail(DNSPIR_ERR_NOT_READY, "server not running");
    if (session >= 0) {
      if ((uint64_t)session >= sv->sess_cap || sv->sess_refs[session] < 1 || sv->sess_closing[session])
        return fail(DNSPIR_ERR_BAD_ARG, "no such open session");
      sv->sess_refs[session]++;
    }
    const uint64_t t = sv->next_ticket++;
    sv->reqs.emplace(t, std::move(r));
    db.pending.push_back(t);
    *ticket = t;
  }
  sv->cv.notify_one();
  return DNSPIR_OK;
}

int dnspir_server_poll(dnspir_server* sv, uint64_t ticket, uint8_t* reply, uint64_t reply_cap, int* done) {
  if (!sv || !done) return fail(DNSPIR_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return fail(DNSPIR_ERR_BAD_ARG, "unknown ticket");
  Request& r = it->second;
  *done = r.status >= 0;
  if (!*done) return DNSPIR_OK;
  const int st = r.status;
  if (st == DNSPIR_OK) {
    if (!reply || reply_cap < r.reply.size()) return fail(DNSPIR_ERR_BAD_ARG, "reply buffer too small");
    memcpy(reply, r.reply.data(), r.reply.size());
  }
  sv->reqs.erase(it);
  return st == DNSPIR_OK ? DNSPIR_OK : fail(st, "the request failed on the device");
}

int dnspir_server_wait(dnspir_server* sv, uint64_t ticket, uint8_t* reply, uint64_t reply_cap, uint32_t timeout_ms) {
  if (!sv) return fail(DNSPIR_ERR_BAD_ARG, "null server");
  {
    std::unique_lock<std::mutex> lk(sv->mu);
    auto ready = [&] {
      auto it = sv->reqs.find(ticket);
      return it == sv->reqs.end() || it->second.status >= 0;
    };
    if (!sv->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
      return fail(DNSPIR_ERR_TIMEOUT, "request not answered within the timeout");
  }
  int done = 0;
  return dnspir_server_poll(sv, ticket, reply, reply_cap, &done);
}

int dnspir_server_db_stats(dnspir_server* sv, uint32_t db_id, uint64_t* completed, uint32_t* admitted_batch,
                           uint64_t* groups, uint64_t* graph_groups, double* latencies_ms, uint32_t max_latencies,
                           uint32_t* n_latencies) {
  if (!sv) return fail(DNSPIR_ERR_BAD_ARG, "null server");
  if (db_id >= sv->dbs.size()) return fail(DNSPIR_ERR_BAD_ARG, "no such database");
  std::lock_guard<std::mutex> lk(sv->mu);
  Db& db = *sv->dbs[db_id];
  if (completed) *completed = db.completed;
  if (admitted_batch) *admitted_batch = (uint32_t)db.admitted;
  if (groups) *groups = db.groups;
  if (graph_groups) *graph_groups = db.graph_groups;
  const uint32_t n = (uint32_t)std::min<size_t>(db.lat_ms.size(), max_latencies);
  if (latencies_ms)
    for (uint32_t i = 0; i < n; i++) latencies_ms[i] = db.lat_ms[i];
  if (n_latencies) *n_latencies = n;
  return DNSPIR_OK;
}

int dnspir_server_stop(dnspir_server* sv) {
  if (!sv) return fail(DNSPIR_ERR_BAD_ARG, "null server");
  if (!sv->running.load()) return DNSPIR_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->running = false;
  }
  sv->cv.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  DeviceGuard dg(sv->device);
  for (auto& dbp : sv->dbs) {
    dnspir_fleet* f = dbp->f;
    cudaStreamSynchronize(f->st);
    cudaStreamSynchronize(f->sec);
    for (auto& s : f->slot) {
      s.drop_graphs();
      s.sec_pending = false;
      s.prim_recorded = false;
    }
    if (dbp->saved_st) {
      f->st = dbp->saved_st;
      f->sec = dbp->saved_sec;
      cudaStreamDestroy(dbp->st);
      cudaStreamDestroy(dbp->sec);
      dbp->st = dbp->sec = dbp->saved_st = dbp->saved_sec = nullptr;
    }
    f->serving = false;
  }
  return DNSPIR_OK;
}

int dnspir_server_destroy(dnspir_server* sv) {
  if (!sv) return DNSPIR_OK;
  dnspir_server_stop(sv);
  DeviceGuard dg(sv->device);
  delete sv;
  return DNSPIR_OK;
}

}  // extern "C"
