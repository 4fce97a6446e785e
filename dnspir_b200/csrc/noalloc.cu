// noalloc.cu -- perform_pir_split for callers that cannot allocate device memory.
//
// dnspir_db_perform_pir_split allocates (and grows) per-shard device
// workspaces on demand.  Some callers cannot let a request do that: a server
// that has committed all of HBM to shard slabs has no headroom left, and a
// request handler must not call cudaMalloc, which can fail under memory
// pressure and synchronizes the whole device.  dnspir_db_perform_pir_split_noalloc
// gives them the same answer with every intermediate buffer in one
// fixed-size region of device memory that is part of this library's module:
// the caller passes device inputs and outputs, the call allocates nothing.
//
// The region is a file-scope __device__ array (NOALLOC_SCRATCH_BYTES).  The
// CUDA runtime loads this library's device code lazily, so the region is
// reserved on a device when dnspir_db_create first runs there: that call looks
// its address up with cudaGetSymbolAddress while the device is current (before
// the shard's slab takes the memory) and keeps it; from then on the device
// holds the region until the process exits.  Host code cannot use the array's
// name as a device address; only the looked-up address is passed to kernels.
// All calls on a device share the region: two calls whose work overlaps on
// the GPU (different streams, no ordering between them) race and corrupt each
// other's answers; order them on one stream or synchronize between them.
// The call holds the shard's lock while it queues its work and records an
// event on the caller's stream; dnspir_db_set_db and dnspir_db_destroy wait
// for that event before they touch the slab.
// Nothing in the region has to start at zero: each call writes every byte of
// it that it later reads.
#include <cstdio>
#include <mutex>
#include <string>

#include "dnspir.h"
#include "kernels.cuh"

namespace dnspir {

// Query ring elements, 8 lanes x (qry, qry_conj, gk0, gk1), Z_q:   512 KiB
constexpr size_t NOALLOC_ZQ_BYTES = (size_t)SIMD * 4 * N_MAX * 8;
// their NTTs in both factors:                                        512 KiB
constexpr size_t NOALLOC_NTT_BYTES = (size_t)SIMD * 4 * 2 * N_MAX * 4;
// scan partial sums: 2 halves x at most 16 row chunks x 2 factors x N x 8 lanes: 4 MiB
constexpr int NOALLOC_MAX_CHUNKS = 16;
constexpr size_t NOALLOC_PART_BYTES = (size_t)2 * NOALLOC_MAX_CHUNKS * 2 * N_MAX * SIMD * 4;
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_ZQ_BYTES + NOALLOC_NTT_BYTES + NOALLOC_PART_BYTES;

// What the entry point needs from a shard (defined in api.cu): begin locks
// the shard and fills the view (unlocked again on failure); end records the
// shard's completion event on the stream and unlocks.
int db_noalloc_begin(dnspir_db* db, DbView* out);
int db_noalloc_end(dnspir_db* db, cudaStream_t st);
void set_last_error(const std::string& msg);

}  // namespace dnspir

static __device__ __align__(256) unsigned char g_noalloc_scratch[dnspir::NOALLOC_SCRATCH_BYTES];

using namespace dnspir;

static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_dev[64];

// Device address of the scratch region on `device` (which must be current).
static int noalloc_scratch(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (device < 0 || device >= 64) {
    set_last_error("device index out of range");
    return DNSPIR_ERR_BAD_ARG;
  }
  if (!g_noalloc_dev[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      set_last_error(std::string("cudaGetSymbolAddress of the no-allocation scratch region failed: ") +
                     cudaGetErrorString(e));
      return DNSPIR_ERR_CUDA;
    }
    g_noalloc_dev[device] = (unsigned char*)p;
  }
  *out = g_noalloc_dev[device];
  return DNSPIR_OK;
}

namespace dnspir {
// Reserves the region on `device` (which must be current): loads it, looks
// its address up and loads the kernels the entry point launches, so that its
// calls need no device memory of their own.  Called by dnspir_db_create.
int noalloc_reserve(int device) {
  unsigned char* p = nullptr;
  const int rc = noalloc_scratch(device, &p);
  if (rc != DNSPIR_OK) return rc;
  if (preload_pir_split_kernels() != 0) {
    set_last_error("cannot load the single-shard scan kernels");
    return DNSPIR_ERR_CUDA;
  }
  return DNSPIR_OK;
}
}  // namespace dnspir

static int noalloc_queue(const DbView& v, const uint64_t* qry_b, const uint64_t* qry_conj_b, const uint64_t* gk_b,
                         uint64_t* out_b, cudaStream_t st);

extern "C" int dnspir_db_perform_pir_split_noalloc(dnspir_db* db, const uint64_t* qry_b, const uint64_t* qry_conj_b,
                                                   const uint64_t* gk_b, uint64_t* out_b, void* cuda_stream) {
  if (!db || !qry_b || !gk_b || !out_b) {
    set_last_error("null argument");
    return DNSPIR_ERR_BAD_ARG;
  }
  DbView v;
  int rc = db_noalloc_begin(db, &v);  // locks the shard
  if (rc != DNSPIR_OK) return rc;
  cudaStream_t st = (cudaStream_t)cuda_stream;
  rc = noalloc_queue(v, qry_b, qry_conj_b, gk_b, out_b, st);
  const int rc_end = db_noalloc_end(db, st);  // unlocks
  return rc != DNSPIR_OK ? rc : rc_end;
}

static int noalloc_queue(const DbView& v, const uint64_t* qry_b, const uint64_t* qry_conj_b, const uint64_t* gk_b,
                         uint64_t* out_b, cudaStream_t st) {
  int rc = DNSPIR_OK;
  const Group& g = v.g;
  if ((g.H == 2) != (qry_conj_b != nullptr)) {
    set_last_error("conjugate query must be given exactly when the group requires it");
    return DNSPIR_ERR_BAD_SHAPE;
  }
  const size_t n = g.n;
  int chunks = scan_chunks(g, 1);
  if (chunks > NOALLOC_MAX_CHUNKS) chunks = NOALLOC_MAX_CHUNKS;
  const size_t zq_bytes = (size_t)SIMD * 4 * n * 8;
  const size_t ntt_bytes = (size_t)SIMD * 4 * 2 * n * 4;
  const size_t part_bytes = (size_t)g.H * chunks * 2 * n * SIMD * 4;
  if (zq_bytes > NOALLOC_ZQ_BYTES || ntt_bytes > NOALLOC_NTT_BYTES || part_bytes > NOALLOC_PART_BYTES) {
    char msg[200];
    snprintf(msg, sizeof(msg), "shard needs %zu bytes of scratch; the static no-allocation region holds %zu",
             zq_bytes + ntt_bytes + part_bytes, NOALLOC_SCRATCH_BYTES);
    set_last_error(msg);
    return DNSPIR_ERR_BAD_SIZE;
  }
  int prev = -1;
  cudaError_t e = cudaGetDevice(&prev);
  if (e == cudaSuccess && prev != v.device) e = cudaSetDevice(v.device);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_last_error(std::string("no-allocation perform_pir_split: cannot make the shard's device current: ") +
                   cudaGetErrorString(e));
    return DNSPIR_ERR_CUDA;
  }
  unsigned char* scratch = nullptr;
  rc = noalloc_scratch(v.device, &scratch);
  if (rc == DNSPIR_OK) {
    uint64_t* zq = (uint64_t*)scratch;
    uint32_t* ntt = (uint32_t*)(scratch + NOALLOC_ZQ_BYTES);
    uint32_t* part = (uint32_t*)(scratch + NOALLOC_ZQ_BYTES + NOALLOC_NTT_BYTES);
    // gather: lane k's polynomials land at slots 4k + {0: qry, 1: qry_conj, 2: gk0, 3: gk1}
    const size_t row = n * 8, pitch = 4 * row;
    e = cudaMemcpy2DAsync(zq, pitch, qry_b, row, row, SIMD, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
      e = qry_conj_b ? cudaMemcpy2DAsync((char*)zq + row, pitch, qry_conj_b, row, row, SIMD, cudaMemcpyDeviceToDevice, st)
                     : cudaMemset2DAsync((char*)zq + row, pitch, 0, row, SIMD, st);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync((char*)zq + 2 * row, pitch, gk_b, 2 * row, 2 * row, SIMD, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) {
      launch_ring_to_ntt(zq, SIMD * 4, ntt, nullptr, g.log2n, v.T, st);
      launch_scan_lanes(v.slab, ntt, part, g, chunks, v.maps, st);
      launch_epilogue_zq(part, g.H * chunks, out_b, g, v.maps, v.T, st);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_last_error(std::string("no-allocation perform_pir_split: ") + cudaGetErrorString(e));
      rc = DNSPIR_ERR_CUDA;
    }
  }
  if (prev >= 0 && prev != v.device) cudaSetDevice(prev);
  return rc;
}
