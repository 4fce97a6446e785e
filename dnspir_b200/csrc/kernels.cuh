// kernels.cuh -- launch wrappers of the device kernels (host side declarations).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ntt.cuh"

namespace dnspir {

// Raises a kernel's dynamic shared-memory limit when a launch needs more than
// the default 48 KB (the attribute is per function and per device).
template <class K>
inline void set_smem(K* kernel, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Shape of one PIR database (IndexGroup, base_pir.rs:132-183).
struct Group {
  int log2n;    // ring dimension N = 2^log2n
  uint32_t n;   // N
  uint32_t l;   // group order
  uint32_t L;   // loop_len: l if l < N else N/2
  uint32_t H;   // halves: 2 if l == N (requires_conj) else 1
  uint32_t qbp; // query_base_power = N / 2 / L
};
Group make_group(int log2n, uint32_t l);

// Output slots of the scan are ordered by (sign, e): position u = sign * N/2 + e
// holds the slot k with 2k + 1 = (sign ? -1 : 1) 5^e mod 2N.  g[u] is that odd
// residue and uof[k] the position of natural slot k (device tables per N).
struct SlotMaps {
  const uint32_t* g;
  const uint32_t* uof;
};

// Scan-layout offset (in u32 words) of array a (0 = entries E, 1/2 = key digits
// G0/G1) of row i, half h, factor p, output position u, lane 0 inside one shard slab.
__host__ __device__ __forceinline__ size_t slab_off(const Group& g, int p, int h, uint32_t i, int a, uint32_t k) {
  return (((((size_t)p * g.H + h) * g.L + i) * 3 + a) * g.n + k) * SIMD;
}
__host__ __device__ __forceinline__ size_t slab_words(const Group& g) { return (size_t)2 * g.H * g.L * 3 * g.n * SIMD; }

// ---- DB encoding (set_transformed_entries, base_pir.rs:662-772)
// in: coefficients [t < l_in][lane < nl][n < N] (< t); A: [t][lane][x] (q1, transform
// position x = slot brv(x))
void launch_encode_cols(const uint16_t* in, uint32_t* A, const Group& g, uint32_t l_in, int nl, const NttTables& T,
                        cudaStream_t st);
// A -> Ahat[h][r][lane][x] (q1, position x = slot brv(x)): evaluations of column polys at the Galois orbit
void launch_encode_rows(const uint32_t* A, uint32_t* Ahat, const Group& g, uint32_t l_in, int nl, const NttTables& T,
                        cudaStream_t st);
// Ahat -> transformed entries.  frame 0: scan layout in `slab` (nl == 8);
// frame 1: chain layout out[((p*H + h)*L + c)*nl + lane][pos] in bit-reversed slot order.
void launch_encode_lift(const uint32_t* Ahat, uint32_t* out, const Group& g, int nl, int frame, const SlotMaps& maps,
                        const NttTables& T, cudaStream_t st);

// ---- key-switch chain (preprocess / partial_gal, base_pir.rs:496-594, 782-863)
struct ChainConsts {
  const uint32_t* gka;    // [digit][p][pos]  (bit-reversed slot order)
  const uint32_t* qa;     // [half][p][pos]   (qry_a for the database's seed set)
  const uint32_t* galb;   // [pos] -> destination position of sigma_5 (bit-reversed coordinates)
  SlotMaps maps;          // scan-layout slot order
};
// Primary preprocessing chain for `nshards` shards (slabs[s] already hold E);
// writes G0/G1 into the slabs and a_out[s][h][lane][p][pos].
void launch_primary_chain(uint32_t* const* slabs_dev, int nshards, uint32_t* a_out, const Group& g,
                          const ChainConsts& cc, const NttTables& T, cudaStream_t st);
// Sums the halves of a_out, returns reply_a as Z_q coefficients (u64) and the
// 17-bit mod-switched a-part (u32) per shard: [s][lane][n].
void launch_primary_finalize(const uint32_t* a_out, int nshards, uint64_t* a_zq, uint32_t* a_ms, const Group& g,
                             const NttTables& T, cudaStream_t st);

// Secondary chain fused with the secondary scan (homomorphic evaluation of
// the secondary database on each query's ciphertext).  E: chain layout from
// launch_encode_lift(frame 1) with nl = 3 * nq lanes; qv: per query decoded
// vectors [q][slot][p][pos] (bit-reversed), slots 0 gk0, 1 gk1, 2 pq, 3 pqc, 4 sq, 5 sqc.
// out: [q][h][part][a/b][p][pos].
void launch_secondary_chain(const uint32_t* E, const uint32_t* qv, size_t qv_stride, int nq, uint32_t* out,
                            const Group& g, const ChainConsts& cc, const NttTables& T, cudaStream_t st,
                            bool clustered = false);

// ---- primary scan (main_pir_loop, base_pir.rs:1085-1247)
// B queries (a power of two up to 256) in one launch over all shards, each
// block serving per_block of them (1, 2, 4, 8 or 16; 0: min(B, 16)), the other
// groups of per_block on grid.y.  qnat: per query [slot][p][N] natural order
// (slots 0 gk0, 1 gk1, 2 pq, 3 pqc), q_stride words apart.  out:
// [b][s][p][u][lane] reduced mod p.
int scan_batch_supported(int B);
int launch_scan_batch(uint32_t* const* slabs_dev, int nshards, const uint32_t* qnat, size_t q_stride, int B,
                      int per_block, uint32_t* out, const Group& g, const SlotMaps& maps, cudaStream_t st);
// ---- primary scan on the tensor cores (tscan.cu): 8-bit limbs, kind::i8
// Tensor layout: the slab indexed by query slot, bytes in 128 x 128 blocks
// [p][sign][m-tile][k-chunk] (same size as the lane layout).  Needs loop_len
// = N/2 and N >= 256.
struct TScanShape {
  int nq;          // rows of the query operand per CTA (4 limbs x queries)
  int mtpc;        // 128-row m-tiles per CTA
  int stages;      // shared-memory pipeline depth
  int persistent;  // 1: persistent warp-specialised kernel; 2: CTA pair (relayed bulk copies); 3: CTA pair (tensor maps)
};
int tensor_layout_supported(const Group& g);
void tensor_dims(const Group& g, uint32_t* mt_total, uint32_t* kc_total);
void launch_retile(const uint32_t* lane_slab, uint8_t* tensor_slab, const Group& g, cudaStream_t st);
const TScanShape* tscan_shapes(int* count);
size_t tscan_query_bytes(const Group& g, int nb_pad);
// Limits of the tensor scan's pipeline waits: wait_ns (0: the default, 2 s)
// and, for tests of the timeout path, a chunk that CTA 0's producer never
// copies (withhold >= 0), so that its MMA thread's wait runs out.
struct TScanLimits {
  uint64_t wait_ns = 0;
  int withhold = -1;
};
// nb queries (decoded, qnat) padded to nb_pad (a multiple of shape.nq / 4);
// qb: tscan_query_bytes of workspace; out as launch_scan_batch; err: one
// device word set to 1 when a bounded wait gave up.  Returns -1 for a shape
// that does not fit.
// slab_maps: tscan_slab_maps of the shards (device), required by the
// tensor-map pair shapes (persistent 3), which are refused (-1) without it.
int launch_tscan(uint8_t* const* slabs_dev, int nshards, const uint32_t* qnat, size_t q_stride, int nb, int nb_pad,
                 uint8_t* qb, uint32_t* out, uint32_t* err, const Group& g, const SlotMaps& maps,
                 const TScanShape& shape, cudaStream_t st, const TScanLimits& lim = TScanLimits(),
                 const void* slab_maps = nullptr);
// Tensor maps of the shards' tensor-layout slabs (host pointers; one map of
// tscan_slab_map_bytes(1) bytes per shard) written to dev_maps; -1 when the
// driver cannot encode them.
size_t tscan_slab_map_bytes(int nshards);
int tscan_slab_maps(uint8_t* const* host_slabs, int nshards, const Group& g, void* dev_maps);
// Per-lane queries (perform_pir_split): qlane [(lane*4 + v)*2 + p][N] natural order;
// part: [chunk][p][u][lane], chunks = H * R.
int scan_chunks(const Group& g, int nshards);
// Loads the kernels of launch_scan_lanes and launch_epilogue_zq on the current
// device (0, or -1 on a CUDA error).
int preload_pir_split_kernels();
void launch_scan_lanes(const uint32_t* slab, const uint32_t* qlane, uint32_t* part, const Group& g, int R,
                       const SlotMaps& maps, cudaStream_t st);
// Primary epilogue for nq queries: scan output -> b (iNTT, CRT), mod-switch,
// combine with the shard's a-part, three base-1025 digits -> secondary
// entries.  Queries are grouped in chunks of `chunk`; chunk c starts at
// c * chunk * 3 * nshards * 8 * N and holds [t = s*8+lane][q*3 + part][n].
void launch_primary_epilogue(const uint32_t* fin, int nq, int nshards, const uint32_t* a_ms, const int* distinct_of,
                             uint16_t* sec_in, int chunk, const Group& g, const SlotMaps& maps, const NttTables& T,
                             cudaStream_t st);
// Epilogue returning b as Z_q coefficients [lane][n] (shard-level perform_pir_split).
void launch_epilogue_zq(const uint32_t* part, int chunks, uint64_t* out, const Group& g, const SlotMaps& maps,
                        const NttTables& T, cudaStream_t st);

// ---- wire codec (pir_wrapper.rs:84-158, 370-408)
// Decodes one query's polynomials: poly_off/poly_bits per polynomial (npoly),
// writes natural-order vectors qnat[poly][p][u] and bit-reversed qbrv[poly][p][pos].
struct PolySpec {
  uint32_t off[6];   // byte offset of each polynomial in the query
  uint32_t bits[6];  // its wire width
  int slot[6];       // destination slot: 0 gk0, 1 gk1, 2 pq, 3 pqc, 4 sq, 5 sqc
  int npoly;
};
// Per query of a group: offset of its bytes, and its session slot (-1: the
// query carries its own Galois keys; otherwise they come from the session
// cache and the bytes omit them, gk_bytes shorter).
struct QDesc {
  uint32_t byte_off;
  int32_t session;
};
// nq queries, outputs at q * q_stride words.
void launch_decode_query(const uint8_t* bytes, const QDesc* desc, int nq, const PolySpec& spec, uint32_t gk_bytes,
                         uint32_t* qnat, uint32_t* qbrv, size_t q_stride, const uint32_t* sess_nat,
                         const uint32_t* sess_brv, int log2n, const NttTables& T, cudaStream_t st);
// Ring elements (Z_q, u64) -> NTT vectors, natural [i][p][u] and bit-reversed [i][p][pos].
void launch_ring_to_ntt(const uint64_t* zq, int count, uint32_t* qnat, uint32_t* qbrv, int log2n, const NttTables& T,
                        cudaStream_t st);
// Secondary chain output -> reply bytes (3 x (17-bit a, 12-bit b)) or Z_q ciphertexts.
void launch_reply(const uint32_t* chain_out, int nq, int H, uint8_t* reply_bytes, size_t reply_stride,
                  uint64_t* reply_zq, int log2n, const NttTables& T, cudaStream_t st);

// Device table of 5^r (inverse: 5^-r) mod 2N for r <= N/2.
const uint32_t* device_pow5(int log2n, bool inverse);

// Read-only view of a shard (api.cu) for the no-allocation entry point (noalloc.cu).
struct DbView {
  int device;
  bool ready;
  Group g;
  const uint32_t* slab;
  NttTables T;
  SlotMaps maps;
};

// Payload helpers for synthetic databases (dns/bucket.rs:289-303 packing).
void launch_pack_bytes(const uint8_t* bytes, uint16_t* coeffs, size_t entries, int log2n, cudaStream_t st);

}  // namespace dnspir
