// host.h -- host-side helpers shared by api.cu (device context, shards,
// shape rules) and fleet.cu (fleets and the answer pipeline).
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "dnspir.h"
#include "kernels.cuh"

namespace dnspir {

extern thread_local std::string g_err;
int fail(int code, const std::string& msg);

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

struct DeviceCtx {
  int device = -1;
  uint32_t* tables = nullptr;
  NttTables T;
  uint32_t* consts[LOG2_N_MAX + 1] = {};  // a-parts in NTT form: [6][2][N], bit-reversed positions
  uint64_t consts_ver[LOG2_N_MAX + 1] = {};  // a-parts version they were built from
  std::vector<uint32_t*> retired;            // a-part buffers replaced by dnspir_set_a_parts
  uint32_t* galb[LOG2_N_MAX + 1] = {};
  uint32_t* gtab[LOG2_N_MAX + 1] = {};  // scan slot order: position -> odd residue
  uint32_t* uof[LOG2_N_MAX + 1] = {};   // natural slot -> position
  std::mutex mu;
};

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
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
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
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

// -------------------------------------------------------------- shard state
// Device buffers shared by set_db and the secondary phase.
struct EncodeWs {
  DBuf A, Ahat, in16, a_out, slab_ptrs;
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

int get_ctx(int device, DeviceCtx** out);
// Per-dimension constants of a device; also brings the a-parts in NTT form up
// to the a-parts now in effect, whose version goes to *version.
int ctx_consts(DeviceCtx* c, int log2n, uint64_t* version = nullptr);
// The six a-parts in effect for dimension 2^log2n (6 x N coefficients in
// [0, q): gk0, gk1, FirstSet query, its conjugate, SecondSet query, its
// conjugate) and their version.
void a_parts_host(int log2n, uint64_t* out, uint64_t* version);
uint64_t a_parts_version(int log2n);
SlotMaps slot_maps(DeviceCtx* c, int log2n);
ChainConsts chain_consts(DeviceCtx* c, int log2n, int used_seeds);
int check_group(uint32_t log2n, uint32_t l);
bool reduced(const uint64_t* v, size_t n);
int preprocess_shards(DeviceCtx* c, const Group& g, int used_seeds, uint32_t* const* slabs_host, int count,
                      const uint16_t* entries_dev, uint64_t* a_zq, uint32_t* a_ms, EncodeWs& ws, cudaStream_t st);

}  // namespace dnspir
