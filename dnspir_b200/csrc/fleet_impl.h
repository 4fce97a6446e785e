// fleet_impl.h -- the fleet object and its group pipeline, shared by fleet.cu
// (the synchronous answer calls) and server.cu (the serving loop).
#pragma once
#include <map>
#include <mutex>
#include <vector>

#include "host.h"

namespace dnspir {

// Buffers of one group of queries in flight.
struct QSlot {
  DBuf qbytes, qdesc, qnat, qbrv, fin, sec_in, reply_dev;
  HBuf qpin, dpin, rpin;  // host staging: query bytes, descriptors, reply bytes
  cudaEvent_t prim_done = nullptr, sec_done = nullptr;
  cudaEvent_t sec_tail = nullptr;  // the secondary phase has reached its last chunk
  bool sec_pending = false, prim_recorded = false;
  // captured launch sequences of the serving loop, per group size
  std::map<int, cudaGraphExec_t> gprim, gsec;
  void drop_graphs() {
    for (auto& kv : gprim) cudaGraphExecDestroy(kv.second);
    for (auto& kv : gsec) cudaGraphExecDestroy(kv.second);
    gprim.clear();
    gsec.clear();
  }
  ~QSlot() {
    drop_graphs();
    if (prim_done) cudaEventDestroy(prim_done);
    if (sec_done) cudaEventDestroy(sec_done);
    if (sec_tail) cudaEventDestroy(sec_tail);
  }
};

const size_t QV_WORDS_PER_QUERY = 6 * 2;  // decoded slots x factors, times N

}  // namespace dnspir

struct dnspir_fleet {
  int device = 0;
  dnspir::DeviceCtx* ctx = nullptr;
  dnspir::Group g1, g2;
  uint32_t S = 0, D = 0;
  cudaStream_t own = nullptr, st = nullptr, sec = nullptr;
  std::vector<uint32_t*> slabs;
  std::vector<bool> ready;
  uint64_t ap_ver = 0;  // a-parts version every ready shard was preprocessed under
  dnspir::DBuf slabs_dev, distinct_dev, a_zq, a_ms;
  dnspir::DBuf tmaps;  // tensor maps of the slabs (CTA-pair tensor-map scan); empty when unavailable
  dnspir::EncodeWs ws;
  dnspir::QSlot slot[2];
  dnspir::DBuf secE, chain_out, qzq, reply_zq;  // used by one stream at a time
  dnspir::HBuf rpin;                            // host staging of the replies of one call
  int batch = 1;
  int sec_chunk = 1;  // queries per secondary launch sequence
  int engine = DNSPIR_ENGINE_CUDA_CORES;
  bool serving = false;                       // attached to a running server
  dnspir::DBuf qb, err_word, tmp_lane;        // tensor engine: query operand, wait-error word, preprocessing scratch
  dnspir::TScanLimits limits;                 // tensor engine: wait limit (and the timeout-test hook)
  std::map<int, int> tuned;                   // tensor engine: group size -> tile shape index
  std::map<int, int> tuned_cc;                // CUDA-core engine: group size -> queries per block
  std::map<int, int> tuned_chain;             // group size -> 1: two-block-cluster chains at every chunk size
  std::map<int, int> tuned_serial;            // group size -> schedule: 0 the primary phase overlaps the previous
                                              // group's secondary, 1 waits for all of it, 2 waits until it
                                              // reaches its last chunk
  std::vector<cudaEvent_t> tev;               // 6 timing events per group of the last call
  std::vector<int> q_group;                   // per query of the last call: its group, or -1
  uint64_t launches = 0;                      // kernels launched by the answer pipeline so far
  std::mutex mu;
  ~dnspir_fleet();
};

namespace dnspir {

// Wire layout of a full query for this fleet's shapes (pir_wrapper.rs:259-317).
PolySpec fleet_wire_spec(const dnspir_fleet* f);
// Bytes of the two Galois-key polynomials at the start of a query.
uint32_t fleet_gk_bytes(const dnspir_fleet* f);
// Padded kernel batch of a group of nb queries.
int fleet_kernel_batch(dnspir_fleet* f, int nb);
int fleet_ready(dnspir_fleet* f);
// Workspace of a slot for groups of up to nb queries (kernel batch Bk) and
// qbytes of query bytes.
int fleet_slot_workspace(dnspir_fleet* f, QSlot& s, int Bk, int nb, size_t qbytes);
// Secondary workspace for groups of up to nb queries.
int fleet_secondary_workspace(dnspir_fleet* f, int nb);
// Primary kernels of a group on f->st: decode (bytes and descriptors already
// in s.qbytes / s.qdesc) and scan.  scan0/scan1: optional events around the
// scan.
int fleet_primary_kernels(dnspir_fleet* f, QSlot& s, int nb, int Bk, const uint32_t* sess_nat,
                          const uint32_t* sess_brv, cudaEvent_t scan0, cudaEvent_t scan1);
// Secondary kernels of a group on f->sec: primary epilogue, encode, chains, replies (bytes at
// reply_dev + q * reply_stride, or Z_q ciphertexts at reply_zq), and the copy
// of nb reply bytes to host_reply when given.
int fleet_secondary_kernels(dnspir_fleet* f, QSlot& s, int nb, uint8_t* reply_dev, size_t reply_stride,
                            uint64_t* reply_zq, uint8_t* host_reply);

}  // namespace dnspir
