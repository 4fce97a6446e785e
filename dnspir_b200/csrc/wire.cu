// wire.cu -- query unpacking and reply packing on the device
// (process_queries, crates/pir/src/pir_wrapper.rs:370-408; uncondense :120-158,
// condense :84-113; mod_switch_decode / mod_switch_encode, bfv.rs:52-69).
#include "kernels.cuh"

namespace dnspir {
namespace {

// One coefficient of a condense<bits> stream of N values (pir_wrapper.rs:84-113):
// whole bytes first (one plane of N bytes per byte), then a nibble plane,
// a 2-bit plane and a 1-bit plane, each only when the width needs it.
__device__ __forceinline__ uint64_t unpack_one(const uint8_t* __restrict__ b, int bits, uint32_t N, uint32_t n) {
  uint64_t x = 0;
  size_t pos = 0;
  for (int i = 0; i < bits / 8; i++) {
    x |= (uint64_t)b[pos + n] << (8 * i);
    pos += N;
  }
  if (bits % 8 >= 4) {
    const uint8_t s = b[pos + n / 2];
    x |= (uint64_t)((n & 1) ? (s & 0xF) : (s >> 4)) << ((bits / 8) * 8);
    pos += N / 2;
  }
  if (bits % 4 >= 2) {
    const uint8_t s = b[pos + n / 4];
    x |= (uint64_t)((s >> (6 - 2 * (n % 4))) & 3) << ((bits / 4) * 4);
    pos += N / 4;
  }
  if (bits % 2 >= 1) {
    const uint8_t s = b[pos + n / 8];
    x |= (uint64_t)((s >> (7 - n % 8)) & 1) << ((bits / 2) * 2);
  }
  return x;
}

// grid: x = polynomial of the query, y = factor, z = query of the group.
// Outputs natural-order qnat[slot][p][u] and bit-reversed qbrv[slot][p][pos]
// at q * q_stride.  A query with a session takes its Galois-key slots 0 and 1
// from the session cache ([session][slot][p][N], natural and bit-reversed)
// and its bytes start with the first polynomial after the keys.
__global__ void decode_query_kernel(const uint8_t* __restrict__ bytes, const QDesc* __restrict__ desc, PolySpec spec,
                                    uint32_t gk_bytes, uint32_t* __restrict__ qnat, uint32_t* __restrict__ qbrv,
                                    size_t q_stride, const uint32_t* __restrict__ sess_nat,
                                    const uint32_t* __restrict__ sess_brv, int log2n, NttTables T) {
  extern __shared__ uint32_t sm[];
  const int poly = blockIdx.x, p = blockIdx.y, q = blockIdx.z;
  const uint32_t N = 1u << log2n;
  const uint32_t pr = prime_of(p);
  const int bits = spec.bits[poly];
  const QDesc d = desc[q];
  const int slot = spec.slot[poly];
  qnat += (size_t)q * q_stride;
  qbrv += (size_t)q * q_stride;
  if (d.session >= 0 && slot < 2) {
    const size_t o = (((size_t)d.session * 2 + slot) * 2 + p) * N;
    for (uint32_t u = threadIdx.x; u < N; u += blockDim.x) {
      qnat[((size_t)slot * 2 + p) * N + u] = sess_nat[o + u];
      qbrv[((size_t)slot * 2 + p) * N + u] = sess_brv[o + u];
    }
    return;
  }
  const uint8_t* src = bytes + d.byte_off + spec.off[poly] - (d.session >= 0 ? gk_bytes : 0);
  for (uint32_t n = threadIdx.x; n < N; n += blockDim.x) {
    const uint64_t v = ms_decode(unpack_one(src, bits, N, n), bits);
    sm[n] = reduce64(v, pr, barrett_mu(pr));
  }
  __syncthreads();
  ntt_fwd_smem(sm, log2n, 1, T, p);
  uint32_t* on = qnat + ((size_t)slot * 2 + p) * N;
  uint32_t* ob = qbrv + ((size_t)slot * 2 + p) * N;
  for (uint32_t u = threadIdx.x; u < N; u += blockDim.x) {
    on[u] = sm[brv(u, log2n)];
    ob[u] = sm[u];
  }
}

__global__ void ring_to_ntt_kernel(const uint64_t* __restrict__ zq, uint32_t* __restrict__ qnat,
                                   uint32_t* __restrict__ qbrv, int log2n, NttTables T) {
  extern __shared__ uint32_t sm[];
  const int i = blockIdx.x, p = blockIdx.y;
  const uint32_t N = 1u << log2n;
  const uint32_t pr = prime_of(p);
  for (uint32_t n = threadIdx.x; n < N; n += blockDim.x) sm[n] = reduce64(zq[(size_t)i * N + n], pr, barrett_mu(pr));
  __syncthreads();
  ntt_fwd_smem(sm, log2n, 1, T, p);
  for (uint32_t u = threadIdx.x; u < N; u += blockDim.x) {
    if (qnat) qnat[((size_t)i * 2 + p) * N + u] = sm[brv(u, log2n)];
    if (qbrv) qbrv[((size_t)i * 2 + p) * N + u] = sm[u];
  }
}

// grid: x = ciphertext part, y = query.  Sums the two halves of the secondary
// chain, returns to coefficients, CRT, and either stores Z_q values or the
// mod-switched, condensed reply (pir_wrapper.rs:401-408).
__global__ void reply_kernel(const uint32_t* __restrict__ chain_out, int H, uint8_t* __restrict__ reply_bytes,
                             size_t reply_stride, uint64_t* __restrict__ reply_zq, int log2n, NttTables T,
                             CrtConst crtc) {
  extern __shared__ uint32_t sm[];  // [a q1 | b q1 | a q2 | b q2]
  const int part = blockIdx.x, q = blockIdx.y;
  const uint32_t N = 1u << log2n;
  for (uint32_t b = threadIdx.x; b < 4 * N; b += blockDim.x) {
    const uint32_t poly = b >> log2n, pos = b & (N - 1);
    const uint32_t p = poly >> 1, ab = poly & 1;
    const uint32_t pr = prime_of(p);
    uint32_t v = 0;
    for (int h = 0; h < H; h++)
      v = add_mod(v, chain_out[((((size_t)q * H + h) * CTXT_PARTS + part) * 2 + ab) * 2 * N + p * N + pos], pr);
    sm[b] = v;
  }
  __syncthreads();
  ntt_inv_smem2(sm, log2n, 2, 2, T);
  for (uint32_t n = threadIdx.x; n < N; n += blockDim.x) {
    const uint64_t va = crt(sm[n], sm[2 * N + n], crtc);
    const uint64_t vb = crt(sm[N + n], sm[3 * N + n], crtc);
    if (reply_zq) {
      reply_zq[(((size_t)q * CTXT_PARTS + part) * 2 + 0) * N + n] = va;
      reply_zq[(((size_t)q * CTXT_PARTS + part) * 2 + 1) * N + n] = vb;
    } else {
      sm[n] = ms_encode(va, SEC_A_BITS);
      sm[N + n] = ms_encode(vb, SEC_B_BITS);
    }
  }
  if (reply_zq) return;
  __syncthreads();
  const uint32_t abytes = N * SEC_A_BITS / 8, bbytes = N * SEC_B_BITS / 8;
  uint8_t* out = reply_bytes + (size_t)q * reply_stride + (size_t)part * (abytes + bbytes);
  const uint32_t* ea = sm;
  const uint32_t* eb = sm + N;
  for (uint32_t n = threadIdx.x; n < N; n += blockDim.x) {
    out[n] = (uint8_t)ea[n];
    out[N + n] = (uint8_t)(ea[n] >> 8);
    uint8_t* ob = out + abytes;
    ob[n] = (uint8_t)eb[n];
  }
  for (uint32_t m = threadIdx.x; m < N / 8; m += blockDim.x) {
    uint8_t v = 0;
    for (int u = 0; u < 8; u++) v |= (uint8_t)(((ea[8 * m + u] >> 16) & 1) << (7 - u));
    out[2 * N + m] = v;
  }
  for (uint32_t m = threadIdx.x; m < N / 2; m += blockDim.x) {
    out[abytes + N + m] = (uint8_t)((((eb[2 * m] >> 8) & 0xF) << 4) | ((eb[2 * m + 1] >> 8) & 0xF));
  }
}

}  // namespace

CrtConst host_crt_const();

void launch_decode_query(const uint8_t* bytes, const QDesc* desc, int nq, const PolySpec& spec, uint32_t gk_bytes,
                         uint32_t* qnat, uint32_t* qbrv, size_t q_stride, const uint32_t* sess_nat,
                         const uint32_t* sess_brv, int log2n, const NttTables& T, cudaStream_t st) {
  if (nq <= 0) return;
  dim3 grid(spec.npoly, 2, nq);
  decode_query_kernel<<<grid, 256, (size_t)4 << log2n, st>>>(bytes, desc, spec, gk_bytes, qnat, qbrv, q_stride,
                                                              sess_nat, sess_brv, log2n, T);
}

void launch_ring_to_ntt(const uint64_t* zq, int count, uint32_t* qnat, uint32_t* qbrv, int log2n, const NttTables& T,
                        cudaStream_t st) {
  if (count <= 0) return;
  dim3 grid(count, 2);
  ring_to_ntt_kernel<<<grid, 256, (size_t)4 << log2n, st>>>(zq, qnat, qbrv, log2n, T);
}

void launch_reply(const uint32_t* chain_out, int nq, int H, uint8_t* reply_bytes, size_t reply_stride,
                  uint64_t* reply_zq, int log2n, const NttTables& T, cudaStream_t st) {
  dim3 grid(CTXT_PARTS, nq);
  const size_t smem = (size_t)16 << log2n;
  set_smem(reply_kernel, smem);
  reply_kernel<<<grid, 256, smem, st>>>(chain_out, H, reply_bytes, reply_stride, reply_zq, log2n, T, host_crt_const());
}

}  // namespace dnspir
