// scan.cu -- the primary-phase scan (main_pir_loop, crates/pir/src/base_pir.rs:
// 1085-1247) for B queries at once, and its epilogue (perform_pir_split
// :1066-1077, from_simd_element :905-935, double_pir.rs:161-175).
//
// main_pir_loop is the recurrence  sum'[gal(j)] = sum[j] + G0[i,j] gk0[j] +
// G1[i,j] gk1[j] + E[i,j] q[j]  followed by the inverse permutation.  Unrolled,
// output slot k receives from row i the terms at slot j = idx(5^(L-1-i) (2k+1)).
// The slab orders slots by (sign, e) with 2k+1 = +-5^e mod 2N (SlotMaps), so
// sigma_5 is e -> e+1 and output u = (sign, e) reads, at row i, the query
// entry (sign, e + L-1-i mod N/2): for a tile of consecutive e and a chunk of
// rows the query entries needed form one contiguous (cyclic) window, which is
// staged in shared memory for all B queries.  Every row is stored permuted so
// that the data for output u sits at position u (slab_off), so a block streams
// its rows contiguously.  Products of canonical residues are below 2^52, so one
// 64-bit accumulator per (lane, query) absorbs a half (3 * L <= 3072 products)
// without reduction; it is reduced once between halves and once at the end.
// One block per (shard, factor, sign, tile) item, consecutive blocks sharing a
// shard; blocks retire after their item so that the higher-priority secondary
// stream can take SMs while a scan is running.
#include "kernels.cuh"
#include "ntt2048.cuh"

namespace dnspir {
namespace {

constexpr int SCAN_NT = 256;

struct ScanArgs {
  Group g;
  uint32_t* const* slabs;
  int nshards;
  const uint32_t* qnat;  // per query [slot][p][N] natural order
  size_t q_stride;       // words between queries
  const uint32_t* gtab;  // (sign, e) position -> odd residue
  uint32_t* out;         // [b][s][p][u][lane], reduced mod p
  int rows;              // rows per window chunk
};

__device__ __forceinline__ void ld_lanes(const uint32_t* p, uint32_t* v, int lpt) {
  if (lpt == 8) {
    const uint4 a = __ldcs(reinterpret_cast<const uint4*>(p));
    const uint4 b = __ldcs(reinterpret_cast<const uint4*>(p + 4));
    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
  } else if (lpt == 4) {
    const uint4 a = __ldcs(reinterpret_cast<const uint4*>(p));
    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
  } else {
    const uint2 a = __ldcs(reinterpret_cast<const uint2*>(p));
    v[0] = a.x, v[1] = a.y;
  }
}

// 16 queries per block: two blocks per SM (128 registers, 16 warps: the
// kernel is latency-bound at one block of 8 warps); the other shapes would
// spill under that bound and keep the compiler's own register choice (a
// minimum of 0 blocks leaves it as with no minimum)
template <int B, int LPT>
__global__ void __launch_bounds__(SCAN_NT, B == 16 ? 2 : 0) scan_batch_kernel(ScanArgs a) {
  constexpr int LG = SIMD / LPT;     // lane groups per slot
  constexpr int TS = SCAN_NT / LG;   // slots per tile
  extern __shared__ uint32_t win[];  // [3][B][W]: x fastest, so a warp's slots hit distinct banks
  const Group& g = a.g;
  const uint32_t N = g.n, half = N / 2, L = g.L;
  const uint32_t R = (uint32_t)a.rows;
  const uint32_t W = TS + R - 1;
  const uint32_t tiles = (half + TS - 1) / TS;
  const int slot = threadIdx.x / LG, lg = threadIdx.x % LG;
  const size_t arr = (size_t)N * SIMD, row_stride = 3 * arr;
  // item = ((s * 2 + p) * 2 + sgn) * tiles + tile
  const uint32_t item = blockIdx.x;
  // grid.y: which group of B queries of the kernel batch this block serves
  const size_t qbase = (size_t)blockIdx.y * B;
  const uint32_t tile = item % tiles;
  const uint32_t sgn = (item / tiles) & 1;
  const int p = (item / (2 * tiles)) & 1;
  const int s = item / (4 * tiles);
  const uint32_t e0 = tile * TS;
  const uint32_t e = e0 + slot;
  const bool active = e < half;
  const uint32_t u = sgn * half + e;
  const uint32_t pr = prime_of(p);
  const uint64_t mu = barrett_mu(pr);
  const uint32_t* slab = a.slabs[s];
  uint64_t acc[LPT][B];
#pragma unroll
  for (int l = 0; l < LPT; l++)
#pragma unroll
    for (int b = 0; b < B; b++) acc[l][b] = 0;
  for (uint32_t h = 0; h < g.H; h++) {
    // decoded slots: 0 gk0, 1 gk1, 2 pq, 3 pqc -> window vectors (query of this half, gk0, gk1)
    const int vslot[3] = {2 + (int)h, 0, 1};
    for (uint32_t i0 = 0; i0 < L; i0 += R) {
      const uint32_t i1 = min(L, i0 + R);
      const uint32_t Wr = TS + (i1 - i0) - 1;
      const uint32_t w0 = (e0 + L - i1) % half;
      for (uint32_t idx = threadIdx.x; idx < 3 * Wr * B; idx += SCAN_NT) {
        const uint32_t x = idx % Wr, b = (idx / Wr) % B, v = idx / (B * Wr);
        const uint32_t uu = sgn * half + (w0 + x) % half;
        const uint32_t kk = (__ldg(a.gtab + uu) - 1) >> 1;
        win[(v * B + b) * W + x] = __ldg(a.qnat + (qbase + b) * a.q_stride + ((size_t)vslot[v] * 2 + p) * N + kk);
      }
      __syncthreads();
      if (active) {
        const uint32_t* row = slab + slab_off(g, p, h, i0, 0, u) + lg * LPT;
        uint32_t x = slot + (i1 - 1 - i0);
#pragma unroll 2
        for (uint32_t i = i0; i < i1; i++) {
          uint32_t ev[LPT], av[LPT], bv[LPT];
          ld_lanes(row, ev, LPT);
          ld_lanes(row + arr, av, LPT);
          ld_lanes(row + 2 * arr, bv, LPT);
#pragma unroll
          for (int b = 0; b < B; b++) {
            const uint32_t q = win[b * W + x], g0 = win[(B + b) * W + x], g1 = win[(2 * B + b) * W + x];
#pragma unroll
            for (int l = 0; l < LPT; l++)
              acc[l][b] += (uint64_t)ev[l] * q + (uint64_t)av[l] * g0 + (uint64_t)bv[l] * g1;
          }
          row += row_stride;
          x--;
        }
      }
      __syncthreads();
    }
    if (h + 1 < g.H) {
#pragma unroll
      for (int l = 0; l < LPT; l++)
#pragma unroll
        for (int b = 0; b < B; b++) acc[l][b] = reduce64(acc[l][b], pr, mu);
    }
  }
  if (active) {
#pragma unroll
    for (int b = 0; b < B; b++) {
      uint32_t* o = a.out + ((((qbase + b) * a.nshards + s) * 2 + p) * N + u) * SIMD + lg * LPT;
#pragma unroll
      for (int l = 0; l < LPT; l++) o[l] = reduce64(acc[l][b], pr, mu);
    }
  }
}

// Per-lane queries (perform_pir_split): qlane[(lane*4 + v)*2 + p][N] natural
// order, v = qry, qry_conj, gk0, gk1.  Partials [chunk][p][u][lane].
__global__ void scan_lanes_kernel(const uint32_t* __restrict__ slab, const uint32_t* __restrict__ qlane,
                                  uint32_t* __restrict__ part, Group g, int R, const uint32_t* __restrict__ pow5,
                                  const uint32_t* __restrict__ gtab, uint32_t inv5) {
  const uint32_t N = g.n, mask = 2 * N - 1;
  const int HR = g.H * R;
  const int p = blockIdx.z / HR;
  const int ch = blockIdx.z % HR;
  const int h = ch / R, rc = ch % R;
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= N) return;
  const uint32_t rows = (g.L + R - 1) / R;
  const uint32_t i0 = rc * rows;
  const uint32_t i1 = min(g.L, i0 + rows);
  const uint32_t gu = gtab[u];
  uint64_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (i0 < i1) {
    uint32_t c = pow5[g.L - 1 - i0];
    for (uint32_t i = i0; i < i1; i++) {
      const uint32_t j = ((c * gu) & mask) >> 1;
      const uint32_t* row = slab + slab_off(g, p, h, i, 0, u);
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
    part[(((size_t)ch * 2 + p) * N + u) * SIMD + l] = reduce64(acc[l], pr, barrett_mu(pr));
}

// grid: x = shard, y = lane pair, z = query.  b = the query's scan output ->
// iNTT -> CRT -> mod switch to 12 bits; with the shard's 17-bit a-part,
// three base-1025 digits (encode_ciphertext_plaintext, double_pir.rs:70-81).
__global__ void primary_epilogue_kernel(const uint32_t* __restrict__ fin, int nshards,
                                        const uint32_t* __restrict__ a_ms, const int* __restrict__ distinct_of,
                                        uint16_t* __restrict__ sec_in, int nq, int chunk, Group g,
                                        const uint32_t* __restrict__ uof, NttTables T, CrtConst crtc) {
  extern __shared__ uint32_t sm[];  // [l0 q1, l1 q1, l0 q2, l1 q2]
  const int s = blockIdx.x, l0 = blockIdx.y * 2, b = blockIdx.z;
  const int logn = g.log2n;
  const uint32_t N = g.n;
  // position x of factor p holds natural slot brv(x) of both lanes (one 8-byte
  // load per pair; iterating over positions keeps the stores conflict-free)
  for (uint32_t x = threadIdx.x; x < 2 * N; x += blockDim.x) {
    const uint32_t p = x >> logn, xx = x & (N - 1);
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(
        fin + ((((size_t)b * nshards + s) * 2 + p) * N + __ldg(uof + brv(xx, logn))) * SIMD + l0));
    sm[((2 * p) << logn) + xx] = v.x;
    sm[((2 * p + 1) << logn) + xx] = v.y;
  }
  __syncthreads();
  ntt_inv_smem2(sm, logn, 2, 2, T);
  const int ds = distinct_of[s];
  for (uint32_t x = threadIdx.x; x < 2 * N; x += blockDim.x) {
    const uint32_t ll = x >> logn, n = x & (N - 1);
    const uint64_t v = crt(sm[(ll << logn) + n], sm[((2 + ll) << logn) + n], crtc);
    const uint32_t bq = ms_encode(v, PRIM_B_BITS);
    const uint32_t aq = a_ms[((size_t)ds * SIMD + l0 + ll) * N + n];
    uint32_t w = (aq << PRIM_B_BITS) + bq;
    const uint32_t d0 = w % TPLAIN;
    w /= TPLAIN;
    const uint32_t d1 = w % TPLAIN;
    const uint32_t d2 = w / TPLAIN;
    // the secondary input of queries [c * chunk, ...) is one [t][lanes_c][N] block
    const int c = b / chunk, bl = b % chunk;
    const size_t lanes_c = (size_t)CTXT_PARTS * min(chunk, nq - c * chunk);
    const size_t t = (size_t)s * SIMD + l0 + ll;
    uint16_t* o = sec_in + (size_t)c * chunk * CTXT_PARTS * nshards * SIMD * N + (t * lanes_c + (size_t)bl * CTXT_PARTS) * N + n;
    o[0] = (uint16_t)d0;
    o[N] = (uint16_t)d1;
    o[2 * N] = (uint16_t)d2;
  }
}

// ---- N = 2048: the same epilogue on the register transforms of
// ntt2048.cuh.  Grid: x = shard, y = four lanes, z = query.  One 16-byte
// gather per position and factor brings four lanes (half a 32-byte sector; the
// other half is the neighbouring block's), the eight inverse transforms run
// together, the CRT uses Shoup companions of its two constants and the 12-bit
// switch an exact 64-bit rounding (v 2^13 + q < 2^64 for v < q).
constexpr int EPI_NT = 512;

__device__ __forceinline__ uint32_t ms_encode12(uint64_t v) {
  // round(v 2^12 / q) = floor((v 2^13 + q) / 2q): a double estimate (v times
  // the rounded constant 2^12 / q, within one of the result), then one exact
  // correction (r <= 2^12, so r 2q < 2^64)
  constexpr double SCALE = (double)(1u << PRIM_B_BITS) / (double)QQ;
  const uint64_t num = (v << (PRIM_B_BITS + 1)) + QQ;
  int64_t r = (int64_t)floor((double)v * SCALE + 0.5);
  r = r < 0 ? 0 : r;
  const uint64_t lo = (uint64_t)r * (2 * QQ);
  if (num < lo) r--;
  else if (num - lo >= 2 * QQ) r++;
  return (uint32_t)r & ((1u << PRIM_B_BITS) - 1);
}

__global__ void __launch_bounds__(EPI_NT, 3) primary_epilogue2k_kernel(
    const uint32_t* __restrict__ fin, int nshards, const uint32_t* __restrict__ a_ms,
    const int* __restrict__ distinct_of, uint16_t* __restrict__ sec_in, int nq, int chunk,
    const uint32_t* __restrict__ uof, NttTables T, uint32_t k1, uint32_t k1q, uint32_t k2, uint32_t k2q) {
  extern __shared__ __align__(16) uint32_t sm[];  // [q1 lanes l0 .. l0 + 3][q2 lanes], padded
  using namespace n2k;
  const int s = blockIdx.x, l0 = blockIdx.y * 4, b = blockIdx.z;
  // position x of factor p holds natural slot brv(x)
  for (int x = threadIdx.x; x < 2 * N; x += EPI_NT) {
    const int p = x >> 11, xx = x & (N - 1);
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(
        fin + ((((size_t)b * nshards + s) * 2 + p) * N + __ldg(uof + brv11(xx))) * SIMD + l0));
    uint32_t* o = sm + 4 * p * PS + phys(xx);
    o[0] = v.x, o[PS] = v.y, o[2 * PS] = v.z, o[3 * PS] = v.w;
  }
  __syncthreads();
  inv<EPI_NT>(sm, 4, 4, T);
  const int ds = distinct_of[s];
  // the secondary input of queries [c * chunk, ...) is one [t][lanes_c][N] block
  const int c = b / chunk, bl = b % chunk;
  const size_t lanes_c = (size_t)CTXT_PARTS * min(chunk, nq - c * chunk);
  uint16_t* const base = sec_in + (size_t)c * chunk * CTXT_PARTS * nshards * SIMD * N;
  for (int x = threadIdx.x; x < 4 * N; x += EPI_NT) {
    const int ll = x >> 11, n = x & (N - 1);
    const uint32_t o = phys(n);
    const uint32_t x1 = shoup_mul(sm[ll * PS + o], k1, k1q, P1);
    const uint32_t x2 = shoup_mul(sm[(4 + ll) * PS + o], k2, k2q, P2);
    uint64_t v = (uint64_t)x1 * P2 + (uint64_t)x2 * P1;
    v = v >= QQ ? v - QQ : v;
    const uint32_t aq = __ldg(a_ms + ((size_t)ds * SIMD + l0 + ll) * N + n);
    uint32_t w = (aq << PRIM_B_BITS) + ms_encode12(v);
    const uint32_t d0 = w % TPLAIN;
    w /= TPLAIN;
    const uint32_t d1 = w % TPLAIN;
    const uint32_t d2 = w / TPLAIN;
    uint16_t* op = base + (((size_t)s * SIMD + l0 + ll) * lanes_c + (size_t)bl * CTXT_PARTS) * N + n;
    op[0] = (uint16_t)d0;
    op[N] = (uint16_t)d1;
    op[2 * N] = (uint16_t)d2;
  }
}

__global__ void epilogue_zq_kernel(const uint32_t* __restrict__ part, int chunks, uint64_t* __restrict__ out,
                                   Group g, const uint32_t* __restrict__ uof, NttTables T, CrtConst crtc) {
  extern __shared__ uint32_t sm[];
  const int l0 = blockIdx.x * 2;
  const int logn = g.log2n;
  const uint32_t N = g.n;
  for (uint32_t x = threadIdx.x; x < 4 * N; x += blockDim.x) {
    const uint32_t poly = x >> logn, k = x & (N - 1);
    const int p = poly >> 1, ll = poly & 1;
    const uint32_t u = __ldg(uof + k);
    uint64_t sum = 0;
    for (int c = 0; c < chunks; c++) sum += part[(((size_t)c * 2 + p) * N + u) * SIMD + l0 + ll];
    const uint32_t pr = prime_of(p);
    sm[(poly << logn) + brv(k, logn)] = reduce64(sum, pr, barrett_mu(pr));
  }
  __syncthreads();
  ntt_inv_smem2(sm, logn, 2, 2, T);
  for (uint32_t x = threadIdx.x; x < 2 * N; x += blockDim.x) {
    const uint32_t ll = x >> logn, n = x & (N - 1);
    out[(size_t)(l0 + ll) * N + n] = crt(sm[(ll << logn) + n], sm[((2 + ll) << logn) + n], crtc);
  }
}

template <int B, int LPT>
void launch_batch(const ScanArgs& a, int groups, cudaStream_t st) {
  constexpr int TS = SCAN_NT / (SIMD / LPT);
  const size_t smem = (size_t)3 * (TS + a.rows - 1) * B * 4;
  set_smem(scan_batch_kernel<B, LPT>, smem);
  const uint32_t tiles = (a.g.n / 2 + TS - 1) / TS;
  const uint32_t items = (uint32_t)a.nshards * 4 * tiles;
  scan_batch_kernel<B, LPT><<<dim3(items, groups), SCAN_NT, smem, st>>>(a);
}

}  // namespace

CrtConst host_crt_const();
const uint32_t* device_pow5(int log2n, bool inverse);

static uint32_t inv5_of(uint32_t two_n) {
  for (uint32_t x = 1; x < two_n; x += 2)
    if ((5 * x) % two_n == 1) return x;
  return 1;
}

int scan_batch_supported(int B) { return B >= 1 && B <= 256 && (B & (B - 1)) == 0; }

int launch_scan_batch(uint32_t* const* slabs_dev, int nshards, const uint32_t* qnat, size_t q_stride, int B,
                      int per_block, uint32_t* out, const Group& g, const SlotMaps& maps, cudaStream_t st) {
  if (!scan_batch_supported(B)) return -1;
  if (per_block <= 0) per_block = B < 16 ? B : 16;
  if (per_block > B || B % per_block) return -1;
  const int groups = B / per_block;
  ScanArgs a;
  a.g = g;
  a.slabs = slabs_dev;
  a.nshards = nshards;
  a.qnat = qnat;
  a.q_stride = q_stride;
  a.gtab = maps.g;
  a.out = out;
  a.rows = (int)(g.L < 256 ? g.L : 256);
  switch (per_block) {
    case 1: launch_batch<1, 8>(a, groups, st); break;
    case 2: launch_batch<2, 8>(a, groups, st); break;
    case 4: launch_batch<4, 8>(a, groups, st); break;
    case 8: launch_batch<8, 4>(a, groups, st); break;
    case 16: launch_batch<16, 2>(a, groups, st); break;
    default: return -1;
  }
  return 0;
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

void launch_scan_lanes(const uint32_t* slab, const uint32_t* qlane, uint32_t* part, const Group& g, int R,
                       const SlotMaps& maps, cudaStream_t st) {
  const int nt = 128;
  dim3 grid((g.n + nt - 1) / nt, 1, 2 * g.H * R);
  scan_lanes_kernel<<<grid, nt, 0, st>>>(slab, qlane, part, g, R, device_pow5(g.log2n, false), maps.g,
                                         inv5_of(2 * g.n));
}

void launch_primary_epilogue(const uint32_t* fin, int nq, int nshards, const uint32_t* a_ms, const int* distinct_of,
                             uint16_t* sec_in, int chunk, const Group& g, const SlotMaps& maps, const NttTables& T,
                             cudaStream_t st) {
  if (g.log2n == 11) {
    const CrtConst cc = host_crt_const();
    const uint32_t k1q = (uint32_t)(((uint64_t)cc.q2inv1 << 32) / P1);
    const uint32_t k2q = (uint32_t)(((uint64_t)cc.q1inv2 << 32) / P2);
    const size_t smem = (size_t)8 * n2k::PS * 4;
    set_smem(primary_epilogue2k_kernel, smem);
    primary_epilogue2k_kernel<<<dim3(nshards, SIMD / 4, nq), EPI_NT, smem, st>>>(
        fin, nshards, a_ms, distinct_of, sec_in, nq, chunk, maps.uof, T, cc.q2inv1, k1q, cc.q1inv2, k2q);
    return;
  }
  const size_t smem = (size_t)4 * g.n * 4;
  dim3 grid(nshards, SIMD / 2, nq);
  set_smem(primary_epilogue_kernel, smem);
  primary_epilogue_kernel<<<grid, 256, smem, st>>>(fin, nshards, a_ms, distinct_of, sec_in, nq, chunk, g,
                                                   maps.uof, T, host_crt_const());
}

int preload_pir_split_kernels() {
  // the runtime loads kernels lazily, at their first launch; this loads the
  // single-shard scan kernels now (cudaFuncGetAttributes forces the load)
  cudaFuncAttributes a;
  if (cudaFuncGetAttributes(&a, (const void*)scan_lanes_kernel) != cudaSuccess ||
      cudaFuncGetAttributes(&a, (const void*)epilogue_zq_kernel) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return 0;
}

void launch_epilogue_zq(const uint32_t* part, int chunks, uint64_t* out, const Group& g, const SlotMaps& maps,
                        const NttTables& T, cudaStream_t st) {
  const size_t smem = (size_t)4 * g.n * 4;
  set_smem(epilogue_zq_kernel, smem);
  epilogue_zq_kernel<<<SIMD / 2, 256, smem, st>>>(part, chunks, out, g, maps.uof, T, host_crt_const());
}

}  // namespace dnspir
