// scan.cu -- the primary-phase scan (main_pir_loop, crates/pir/src/base_pir.rs:
// 1085-1247) and its epilogue (perform_pir_split :1066-1077, from_simd_element
// :905-935, double_pir.rs:161-175).
//
// main_pir_loop is the recurrence  sum'[gal(j)] = sum[j] + G0[i,j] gk0[j] +
// G1[i,j] gk1[j] + E[i,j] q[j]  followed by the inverse permutation.  Unrolled,
// output slot k receives from row i the terms at slot j = idx(5^(L-1-i) (2k+1)).
// The slab stores every row permuted that way (slab_off), so a thread that owns
// output slot k streams its rows contiguously and gathers only the query
// vectors, which sit in shared memory.  Products of canonical residues are
// below 2^52, so one 64-bit accumulator per lane absorbs a whole half
// (3 * L <= 3072 products) without reduction; halves and row chunks are
// reduced mod p and summed in the epilogue.
#include "kernels.cuh"

namespace dnspir {
namespace {

constexpr int SCAN_THREADS = 256;

__device__ __forceinline__ uint4 ld_stream(const uint32_t* p) {
  return __ldcs(reinterpret_cast<const uint4*>(p));
}

__device__ __forceinline__ void mac8(uint64_t acc[8], const uint4& x0, const uint4& x1, uint32_t w) {
  acc[0] += (uint64_t)x0.x * w;
  acc[1] += (uint64_t)x0.y * w;
  acc[2] += (uint64_t)x0.z * w;
  acc[3] += (uint64_t)x0.w * w;
  acc[4] += (uint64_t)x1.x * w;
  acc[5] += (uint64_t)x1.y * w;
  acc[6] += (uint64_t)x1.z * w;
  acc[7] += (uint64_t)x1.w * w;
}

// grid: x = slot tile, y = shard, z = p * (H * R) + h * R + rc
__global__ void __launch_bounds__(SCAN_THREADS) scan_plain_kernel(uint32_t* const* __restrict__ slabs,
                                                                 const uint32_t* __restrict__ qnat,
                                                                 uint32_t* __restrict__ part, Group g, int nshards,
                                                                 int R, const uint32_t* __restrict__ pow5,
                                                                 uint32_t inv5) {
  extern __shared__ uint32_t qs[];  // [qry | qry_conj | gk0 | gk1] for factor p
  const uint32_t N = g.n, mask = 2 * N - 1;
  const int HR = g.H * R;
  const int p = blockIdx.z / HR;
  const int ch = blockIdx.z % HR;
  const int h = ch / R, rc = ch % R;
  const int s = blockIdx.y;
  // decoded slots: 0 gk0, 1 gk1, 2 pq, 3 pqc
  const int slot_of[4] = {2, 3, 0, 1};
  for (uint32_t b = threadIdx.x; b < 4 * N; b += SCAN_THREADS) {
    const uint32_t v = b / N, u = b % N;
    qs[b] = qnat[((size_t)slot_of[v] * 2 + p) * N + u];
  }
  __syncthreads();
  const uint32_t k = blockIdx.x * SCAN_THREADS + threadIdx.x;
  if (k >= N) return;
  const uint32_t rows = (g.L + R - 1) / R;
  const uint32_t i0 = rc * rows;
  const uint32_t i1 = min(g.L, i0 + rows);
  if (i0 >= i1) {
    // empty chunk still writes zeros so the epilogue can sum all chunks
    uint4* o = reinterpret_cast<uint4*>(part + ((((size_t)ch * nshards + s) * 2 + p) * N + k) * SIMD);
    o[0] = make_uint4(0, 0, 0, 0);
    o[1] = make_uint4(0, 0, 0, 0);
    return;
  }
  const uint32_t* qv = qs + (h ? N : 0);
  const uint32_t* g0 = qs + 2 * N;
  const uint32_t* g1 = qs + 3 * N;
  const uint32_t tk1 = 2 * k + 1;
  uint32_t c = pow5[g.L - 1 - i0];
  const uint32_t* row = slabs[s] + slab_off(g, p, h, i0, 0, k);
  const size_t row_stride = (size_t)3 * N * SIMD;
  const size_t arr = (size_t)N * SIMD;
  uint64_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 2
  for (uint32_t i = i0; i < i1; i++) {
    const uint32_t j = ((c * tk1) & mask) >> 1;
    const uint4 e0 = ld_stream(row), e1 = ld_stream(row + 4);
    const uint4 a0 = ld_stream(row + arr), a1 = ld_stream(row + arr + 4);
    const uint4 b0 = ld_stream(row + 2 * arr), b1 = ld_stream(row + 2 * arr + 4);
    mac8(acc, e0, e1, qv[j]);
    mac8(acc, a0, a1, g0[j]);
    mac8(acc, b0, b1, g1[j]);
    c = (c * inv5) & mask;
    row += row_stride;
  }
  const uint32_t pr = prime_of(p);
  const uint64_t mu = barrett_mu(pr);
  uint4 r0, r1;
  r0.x = reduce64(acc[0], pr, mu);
  r0.y = reduce64(acc[1], pr, mu);
  r0.z = reduce64(acc[2], pr, mu);
  r0.w = reduce64(acc[3], pr, mu);
  r1.x = reduce64(acc[4], pr, mu);
  r1.y = reduce64(acc[5], pr, mu);
  r1.z = reduce64(acc[6], pr, mu);
  r1.w = reduce64(acc[7], pr, mu);
  uint4* o = reinterpret_cast<uint4*>(part + ((((size_t)ch * nshards + s) * 2 + p) * N + k) * SIMD);
  o[0] = r0;
  o[1] = r1;
}

// Per-lane queries (perform_pir_split): qlane[(lane*4 + v)*2 + p][N], v = qry, qry_conj, gk0, gk1.
__global__ void scan_lanes_kernel(const uint32_t* __restrict__ slab, const uint32_t* __restrict__ qlane,
                                  uint32_t* __restrict__ part, Group g, int R, const uint32_t* __restrict__ pow5,
                                  uint32_t inv5) {
  const uint32_t N = g.n, mask = 2 * N - 1;
  const int HR = g.H * R;
  const int p = blockIdx.z / HR;
  const int ch = blockIdx.z % HR;
  const int h = ch / R, rc = ch % R;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const uint32_t rows = (g.L + R - 1) / R;
  const uint32_t i0 = rc * rows;
  const uint32_t i1 = min(g.L, i0 + rows);
  uint64_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (i0 < i1) {
    uint32_t c = pow5[g.L - 1 - i0];
    for (uint32_t i = i0; i < i1; i++) {
      const uint32_t j = ((c * (2 * k + 1)) & mask) >> 1;
      const uint32_t* row = slab + slab_off(g, p, h, i, 0, k);
      for (int l = 0; l < SIMD; l++) {
        const uint32_t qv = qlane[(((size_t)l * 4 + h) * 2 + p) * N + j];
        const uint32_t gv0 = qlane[(((size_t)l * 4 + 2) * 2 + p) * N + j];
        const uint32_t gv1 = qlane[(((size_t)l * 4 + 3) * 2 + p) * N + j];
        acc[l] += (uint64_t)row[l] * qv + (uint64_t)row[N * SIMD + l] * gv0 + (uint64_t)row[2 * N * SIMD + l] * gv1;
      }
      c = (c * inv5) & mask;
    }
  }
  const uint32_t pr = prime_of(p);
  for (int l = 0; l < SIMD; l++)
    part[(((size_t)ch * 2 + p) * N + k) * SIMD + l] = reduce64(acc[l], pr, barrett_mu(pr));
}

// Sum of the partials of (s, p, k, lane) mod p.
__device__ __forceinline__ uint32_t sum_partials(const uint32_t* __restrict__ part, int chunks, int nshards, int s,
                                                 int p, uint32_t k, int lane, uint32_t N) {
  uint64_t sum = 0;
  for (int c = 0; c < chunks; c++) sum += part[((((size_t)c * nshards + s) * 2 + p) * N + k) * SIMD + lane];
  const uint32_t pr = prime_of(p);
  return reduce64(sum, pr, barrett_mu(pr));
}

// grid: x = shard, y = lane pair.  b = sum of partials -> iNTT -> CRT ->
// mod switch to 12 bits; with the shard's 17-bit a-part, three base-1025
// digits (encode_ciphertext_plaintext, double_pir.rs:70-81).
__global__ void primary_epilogue_kernel(const uint32_t* __restrict__ part, int chunks, int nshards,
                                        const uint32_t* __restrict__ a_ms, const int* __restrict__ distinct_of,
                                        uint16_t* __restrict__ sec_in, int sec_lanes, int sec_lane0, Group g,
                                        NttTables T, CrtConst crtc) {
  extern __shared__ uint32_t sm[];  // [l0 q1, l1 q1, l0 q2, l1 q2]
  const int s = blockIdx.x, l0 = blockIdx.y * 2;
  const int logn = g.log2n;
  const uint32_t N = g.n;
  for (uint32_t b = threadIdx.x; b < 4 * N; b += blockDim.x) {
    const uint32_t poly = b >> logn, k = b & (N - 1);
    const int p = poly >> 1, ll = poly & 1;
    sm[(poly << logn) + brv(k, logn)] = sum_partials(part, chunks, nshards, s, p, k, l0 + ll, N);
  }
  __syncthreads();
  ntt_inv_smem2(sm, logn, 2, 2, T);
  const int ds = distinct_of[s];
  for (uint32_t b = threadIdx.x; b < 2 * N; b += blockDim.x) {
    const uint32_t ll = b >> logn, n = b & (N - 1);
    const uint64_t v = crt(sm[(ll << logn) + n], sm[((2 + ll) << logn) + n], crtc);
    const uint32_t bq = ms_encode(v, PRIM_B_BITS);
    const uint32_t aq = a_ms[((size_t)ds * SIMD + l0 + ll) * N + n];
    uint32_t w = (aq << PRIM_B_BITS) + bq;
    const uint32_t d0 = w % TPLAIN;
    w /= TPLAIN;
    const uint32_t d1 = w % TPLAIN;
    const uint32_t d2 = w / TPLAIN;
    const size_t t = (size_t)s * SIMD + l0 + ll;
    uint16_t* o = sec_in + (t * sec_lanes + sec_lane0) * N + n;
    o[0] = (uint16_t)d0;
    o[N] = (uint16_t)d1;
    o[2 * N] = (uint16_t)d2;
  }
}

__global__ void epilogue_zq_kernel(const uint32_t* __restrict__ part, int chunks, uint64_t* __restrict__ out,
                                   Group g, NttTables T, CrtConst crtc) {
  extern __shared__ uint32_t sm[];
  const int l0 = blockIdx.x * 2;
  const int logn = g.log2n;
  const uint32_t N = g.n;
  for (uint32_t b = threadIdx.x; b < 4 * N; b += blockDim.x) {
    const uint32_t poly = b >> logn, k = b & (N - 1);
    const int p = poly >> 1, ll = poly & 1;
    sm[(poly << logn) + brv(k, logn)] = sum_partials(part, chunks, 1, 0, p, k, l0 + ll, N);
  }
  __syncthreads();
  ntt_inv_smem2(sm, logn, 2, 2, T);
  for (uint32_t b = threadIdx.x; b < 2 * N; b += blockDim.x) {
    const uint32_t ll = b >> logn, n = b & (N - 1);
    out[(size_t)(l0 + ll) * N + n] = crt(sm[(ll << logn) + n], sm[((2 + ll) << logn) + n], crtc);
  }
}

}  // namespace

CrtConst host_crt_const();
const uint32_t* device_pow5(int log2n, bool inverse);

static uint32_t inv5_of(uint32_t two_n) {
  for (uint32_t x = 1; x < two_n; x += 2)
    if ((5 * x) % two_n == 1) return x;
  return 1;
}

int scan_chunks(const Group& g, int nshards) {
  // enough independent (slot, row chunk) threads to keep every SM streaming
  const double target = 1.5e6;
  const double per_chunk = (double)nshards * 2 * g.n * g.H;
  int R = (int)((target + per_chunk - 1) / per_chunk);
  if (R < 1) R = 1;
  const int rmax = (int)(g.L / 8 > 0 ? g.L / 8 : 1);
  if (R > rmax) R = rmax;
  return R;
}

void launch_scan_plain(uint32_t* const* slabs_dev, int nshards, const uint32_t* qnat, uint32_t* part, const Group& g,
                       int R, cudaStream_t st) {
  dim3 grid((g.n + SCAN_THREADS - 1) / SCAN_THREADS, nshards, 2 * g.H * R);
  const size_t smem = (size_t)4 * g.n * 4;
  set_smem(scan_plain_kernel, smem);
  scan_plain_kernel<<<grid, SCAN_THREADS, smem, st>>>(slabs_dev, qnat, part, g, nshards, R,
                                                      device_pow5(g.log2n, false), inv5_of(2 * g.n));
}

void launch_scan_lanes(const uint32_t* slab, const uint32_t* qlane, uint32_t* part, const Group& g, int R,
                       cudaStream_t st) {
  const int nt = 128;
  dim3 grid((g.n + nt - 1) / nt, 1, 2 * g.H * R);
  scan_lanes_kernel<<<grid, nt, 0, st>>>(slab, qlane, part, g, R, device_pow5(g.log2n, false), inv5_of(2 * g.n));
}

void launch_primary_epilogue(const uint32_t* part, int chunks, int nshards, const uint32_t* a_ms,
                             const int* distinct_of, uint16_t* sec_in, int sec_lanes, int sec_lane0, const Group& g,
                             const NttTables& T, cudaStream_t st) {
  const size_t smem = (size_t)4 * g.n * 4;
  dim3 grid(nshards, SIMD / 2);
  set_smem(primary_epilogue_kernel, smem);
  primary_epilogue_kernel<<<grid, 256, smem, st>>>(part, chunks, nshards, a_ms, distinct_of, sec_in, sec_lanes,
                                                   sec_lane0, g, T, host_crt_const());
}

void launch_epilogue_zq(const uint32_t* part, int chunks, uint64_t* out, const Group& g, const NttTables& T,
                        cudaStream_t st) {
  const size_t smem = (size_t)4 * g.n * 4;
  set_smem(epilogue_zq_kernel, smem);
  epilogue_zq_kernel<<<SIMD / 2, 256, smem, st>>>(part, chunks, out, g, T, host_crt_const());
}

}  // namespace dnspir
