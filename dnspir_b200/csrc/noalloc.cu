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
// The region is a file-scope __device__ array, so every GPU that loads the
// library holds it (NOALLOC_SCRATCH_BYTES) until the process exits.  Host code
// cannot use the array's name as a device address; the first call on each
// device looks its address up with cudaGetSymbolAddress while that device is
// current (make that first call before any stream capture) and keeps it.
// All calls on a device share the region: two calls whose work overlaps on
// the GPU (different streams, no ordering between them) race and corrupt each
// other's answers; order them on one stream or synchronize between them.
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

// What the entry point needs from a shard (defined in api.cu).
int db_view(const dnspir_db* db, DbView* out);
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

extern "C" int dnspir_db_perform_pir_split_noalloc(dnspir_db* db, const uint64_t* qry_b, const uint64_t* qry_conj_b,
                                                   const uint64_t* gk_b, uint64_t* out_b, void* cuda_stream) {
  if (!db || !qry_b || !gk_b || !out_b) {
    set_last_error("null argument");
    return DNSPIR_ERR_BAD_ARG;
  }
  DbView v;
  int rc = db_view(db, &v);
  if (rc != DNSPIR_OK) return rc;
  if (!v.ready) {
    set_last_error("database not preprocessed");
    return DNSPIR_ERR_NOT_READY;
  }
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
  cudaGetDevice(&prev);
  if (prev != v.device) cudaSetDevice(v.device);
  unsigned char* scratch = nullptr;
  rc = noalloc_scratch(v.device, &scratch);
  if (rc == DNSPIR_OK) {
    cudaStream_t st = (cudaStream_t)cuda_stream;
    uint64_t* zq = (uint64_t*)scratch;
    uint32_t* ntt = (uint32_t*)(scratch + NOALLOC_ZQ_BYTES);
    uint32_t* part = (uint32_t*)(scratch + NOALLOC_ZQ_BYTES + NOALLOC_NTT_BYTES);
    // gather: lane k's polynomials land at slots 4k + {0: qry, 1: qry_conj, 2: gk0, 3: gk1}
    const size_t row = n * 8, pitch = 4 * row;
    cudaError_t e = cudaMemcpy2DAsync(zq, pitch, qry_b, row, row, SIMD, cudaMemcpyDeviceToDevice, st);
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
