// chain.cu -- the key-switching chain of preprocess / partial_gal
// (crates/pir/src/base_pir.rs:496-594, 782-863) and its fusion with the
// secondary scan (double_pir.rs:195-218).
//
// One block owns one (database, half, lane) chain; the ciphertext state stays
// in shared memory for all loop_len steps.  A step is
//     t      = sigma_5(a)                     (the galois lookup of :509-515)
//     d0, d1 = balanced base-2^26 digits of the centred CRT lift of iNTT(t)
//              (:541-571, copied exactly)
//     a      = NTT(d0) gk_a0 + NTT(d1) gk_a1 + qry_a E_i
// and, for the secondary database evaluated on a query ciphertext,
//     b      = sigma_5(b) + NTT(d0) gk_b0 + NTT(d1) gk_b1 + qry_b E_i,
// which is the homomorphic evaluation whose b-part main_pir_loop computes
// from the stored digits (its sum/sum_new recurrence equals b up to the
// sigma_5 applied before the final permute, :1072-1073).
//
// Shared-memory vectors hold NTT slots in bit-reversed position order
// (position q <-> slot brv(q)); constants are stored the same way.
#include "kernels.cuh"

namespace dnspir {
namespace {

constexpr int CHAIN_THREADS = 512;
constexpr int PERM_REGS = (4 * N_MAX) / CHAIN_THREADS;

// t = sigma_5(x) for `npoly` length-N vectors starting at sm (in place).
__device__ __forceinline__ void galois_inplace(uint32_t* sm, int npoly, int logn, const uint32_t* __restrict__ galb) {
  const int N = 1 << logn;
  const int total = npoly << logn;
  uint32_t regs[PERM_REGS];
#pragma unroll
  for (int c = 0; c < PERM_REGS; c++) {
    const int e = threadIdx.x + c * CHAIN_THREADS;
    if (e < total) regs[c] = sm[e];
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < PERM_REGS; c++) {
    const int e = threadIdx.x + c * CHAIN_THREADS;
    if (e < total) sm[(e & ~(N - 1)) + __ldg(galb + (e & (N - 1)))] = regs[c];
  }
  __syncthreads();
}

// digits of the centred CRT lift: src q1/q2 coefficient vectors -> dst[4][N]
// ordered (d0 q1, d1 q1, d0 q2, d1 q2)
__device__ __forceinline__ void decompose(const uint32_t* src1, const uint32_t* src2, uint32_t* dst, int logn,
                                          CrtConst cc) {
  const int N = 1 << logn;
  for (int n = threadIdx.x; n < N; n += CHAIN_THREADS) {
    const uint64_t v = crt(src1[n], src2[n], cc);
    int64_t x = (int64_t)v;
    if (v > QQ / 2) x -= (int64_t)QQ;
    int64_t cur = x;
    int64_t d[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const int64_t high = (cur + ((int64_t)1 << (LOG2_B - 1))) >> LOG2_B;
      d[k] = cur - high * ((int64_t)1 << LOG2_B);
      cur = high;
    }
    dst[n] = smod(d[0], P1);
    dst[N + n] = smod(d[1], P1);
    dst[2 * N + n] = smod(d[0], P2);
    dst[3 * N + n] = smod(d[1], P2);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(CHAIN_THREADS) primary_chain_kernel(uint32_t* const* __restrict__ slabs,
                                                                     uint32_t* __restrict__ a_out, Group g,
                                                                     ChainConsts cc, NttTables T, CrtConst crtc,
                                                                     uint32_t c_first, uint32_t cinv_first,
                                                                     uint32_t inv5) {
  extern __shared__ uint32_t sm[];  // [0,2N): a / t ; [2N,6N): digits
  const int lane = blockIdx.x, h = blockIdx.y, s = blockIdx.z;
  uint32_t* slab = slabs[s];
  const int logn = g.log2n;
  const uint32_t N = g.n, mask = 2 * N - 1;
  uint32_t* dg = sm + 2 * N;
  for (uint32_t b = threadIdx.x; b < 2 * N; b += CHAIN_THREADS) sm[b] = 0;
  __syncthreads();
  uint32_t ci = c_first;       // 5^(L-1-i) mod 2N
  uint32_t cinv = cinv_first;  // 5^-(L-1-i) mod 2N
  const uint32_t* gka0 = cc.gka;
  const uint32_t* gka1 = cc.gka + 2 * N;
  const uint32_t* qa = cc.qa + (size_t)h * 2 * N;
  for (uint32_t i = 0; i < g.L; i++) {
    galois_inplace(sm, 2, logn, cc.galb);
    ntt_inv_smem2(sm, logn, 1, 1, T);
    decompose(sm, sm + N, dg, logn, crtc);
    ntt_fwd_smem2(dg, logn, 2, 2, T);
    // key digits of row i in the scan layout: G'[i][k] = G_i[idx(5^(L-1-i) (2k+1))]
    for (uint32_t b = threadIdx.x; b < 4 * N; b += CHAIN_THREADS) {
      const uint32_t which = b >> logn, k = b & (N - 1);
      const uint32_t p = which >> 1, d = which & 1;
      const uint32_t j = gidx(ci * (2 * k + 1), mask);
      slab[slab_off(g, p, h, i, 1 + d, k) + lane] = dg[(which << logn) + brv(j, logn)];
    }
    // a = d0 gk_a0 + d1 gk_a1 + qry_a E_i  (E_i read back from the scan layout)
    for (uint32_t b = threadIdx.x; b < 2 * N; b += CHAIN_THREADS) {
      const uint32_t p = b >> logn, pos = b & (N - 1);
      const uint32_t j = brv(pos, logn);
      const uint32_t ks = gidx(cinv * (2 * j + 1), mask);
      const uint32_t e = slab[slab_off(g, p, h, i, 0, ks) + lane];
      const uint32_t d0 = dg[((2 * p) << logn) + pos], d1 = dg[((2 * p + 1) << logn) + pos];
      const uint32_t pr = prime_of(p);
      const uint64_t acc = (uint64_t)d0 * __ldg(gka0 + b) + (uint64_t)d1 * __ldg(gka1 + b) +
                           (uint64_t)e * __ldg(qa + b);
      sm[b] = reduce64(acc, pr, barrett_mu(pr));
    }
    __syncthreads();
    ci = (ci * inv5) & mask;
    cinv = (cinv * 5) & mask;
  }
  uint32_t* o = a_out + (((size_t)s * g.H + h) * SIMD + lane) * 2 * N;
  for (uint32_t b = threadIdx.x; b < 2 * N; b += CHAIN_THREADS) o[b] = sm[b];
}

// reply_a = a_main + a_conj -> iNTT -> CRT; also the 17-bit mod switch
// (get_a, base_pir.rs:897-903, and double_pir.rs:164).
__global__ void primary_finalize_kernel(const uint32_t* __restrict__ a_out, uint64_t* __restrict__ a_zq,
                                        uint32_t* __restrict__ a_ms, Group g, NttTables T, CrtConst crtc) {
  extern __shared__ uint32_t sm[];  // [2][N]
  const int lane = blockIdx.x, s = blockIdx.y;
  const uint32_t N = g.n;
  for (uint32_t b = threadIdx.x; b < 2 * N; b += blockDim.x) {
    const uint32_t p = b / N;
    uint32_t v = a_out[(((size_t)s * g.H + 0) * SIMD + lane) * 2 * N + b];
    if (g.H == 2) v = add_mod(v, a_out[(((size_t)s * g.H + 1) * SIMD + lane) * 2 * N + b], prime_of(p));
    sm[b] = v;
  }
  __syncthreads();
  ntt_inv_smem2(sm, g.log2n, 1, 1, T);
  for (uint32_t n = threadIdx.x; n < N; n += blockDim.x) {
    const uint64_t v = crt(sm[n], sm[N + n], crtc);
    a_zq[((size_t)s * SIMD + lane) * N + n] = v;
    a_ms[((size_t)s * SIMD + lane) * N + n] = ms_encode(v, PRIM_A_BITS);
  }
}

// Secondary database evaluated on each query ciphertext.  Block: (query,
// half, part).  State a, b and digits in shared memory: [0,2N) a, [2N,4N) b,
// [4N,8N) digits.
__global__ void __launch_bounds__(CHAIN_THREADS) secondary_chain_kernel(const uint32_t* __restrict__ E,
                                                                       const uint32_t* __restrict__ qv,
                                                                       size_t qv_stride, int nl,
                                                                       uint32_t* __restrict__ out, Group g,
                                                                       ChainConsts cc, NttTables T, CrtConst crtc) {
  extern __shared__ uint32_t sm[];
  const int part = blockIdx.x, h = blockIdx.y, q = blockIdx.z;
  const int lane = q * CTXT_PARTS + part;
  const int logn = g.log2n;
  const uint32_t N = g.n;
  uint32_t* a = sm;
  uint32_t* bb = sm + 2 * N;
  uint32_t* dg = sm + 4 * N;
  for (uint32_t b = threadIdx.x; b < 4 * N; b += CHAIN_THREADS) sm[b] = 0;
  __syncthreads();
  const uint32_t* gka0 = cc.gka;
  const uint32_t* gka1 = cc.gka + 2 * N;
  const uint32_t* qa = cc.qa + (size_t)h * 2 * N;
  // decoded query vectors, slots [gk0, gk1, pq, pqc, sq, sqc] each [p][pos]
  const uint32_t* qq = qv + (size_t)q * qv_stride;
  const uint32_t* gkb0 = qq;
  const uint32_t* gkb1 = qq + 2 * N;
  const uint32_t* qb = qq + (size_t)(4 + h) * 2 * N;
  for (uint32_t i = 0; i < g.L; i++) {
    galois_inplace(sm, 4, logn, cc.galb);
    ntt_inv_smem2(a, logn, 1, 1, T);
    decompose(a, a + N, dg, logn, crtc);
    ntt_fwd_smem2(dg, logn, 2, 2, T);
    const uint32_t* Ei = E + ((((size_t)0 * g.H + h) * g.L + i) * nl + lane) * N;
    const size_t pstride = (size_t)g.H * g.L * nl * N;
    for (uint32_t b = threadIdx.x; b < 2 * N; b += CHAIN_THREADS) {
      const uint32_t p = b >> logn, pos = b & (N - 1);
      const uint32_t e = __ldg(Ei + p * pstride + pos);
      const uint32_t d0 = dg[((2 * p) << logn) + pos], d1 = dg[((2 * p + 1) << logn) + pos];
      const uint32_t pr = prime_of(p);
      const uint64_t mu = barrett_mu(pr);
      const uint64_t acc_a = (uint64_t)d0 * __ldg(gka0 + b) + (uint64_t)d1 * __ldg(gka1 + b) +
                             (uint64_t)e * __ldg(qa + b);
      const uint64_t acc_b = (uint64_t)bb[b] + (uint64_t)d0 * __ldg(gkb0 + b) + (uint64_t)d1 * __ldg(gkb1 + b) +
                             (uint64_t)e * __ldg(qb + b);
      a[b] = reduce64(acc_a, pr, mu);
      bb[b] = reduce64(acc_b, pr, mu);
    }
    __syncthreads();
  }
  uint32_t* o = out + ((((size_t)q * g.H + h) * CTXT_PARTS + part) * 2) * 2 * N;
  for (uint32_t b = threadIdx.x; b < 4 * N; b += CHAIN_THREADS) o[b] = sm[b];
}

}  // namespace

static uint32_t pow_mod2n(uint32_t b, uint32_t e, uint32_t mask) {
  uint32_t r = 1;
  for (uint32_t k = 0; k < e; k++) r = (r * b) & mask;
  return r;
}
static uint32_t inv5_mod2n(uint32_t two_n) {
  for (uint32_t x = 1; x < two_n; x += 2)
    if ((5 * x) % two_n == 1) return x;
  return 1;
}

CrtConst host_crt_const();

void launch_primary_chain(uint32_t* const* slabs_dev, int nshards, uint32_t* a_out, const Group& g,
                          const ChainConsts& cc, const NttTables& T, cudaStream_t st) {
  const uint32_t mask = 2 * g.n - 1;
  const uint32_t inv5 = inv5_mod2n(2 * g.n);
  const uint32_t c_first = pow_mod2n(5, g.L - 1, mask);
  const uint32_t cinv_first = pow_mod2n(inv5, g.L - 1, mask);
  const size_t smem = (size_t)6 * g.n * 4;
  set_smem(primary_chain_kernel, smem);
  dim3 grid(SIMD, g.H, nshards);
  primary_chain_kernel<<<grid, CHAIN_THREADS, smem, st>>>(slabs_dev, a_out, g, cc, T, host_crt_const(), c_first,
                                                          cinv_first, inv5);
}

void launch_primary_finalize(const uint32_t* a_out, int nshards, uint64_t* a_zq, uint32_t* a_ms, const Group& g,
                             const NttTables& T, cudaStream_t st) {
  const size_t smem = (size_t)2 * g.n * 4;
  dim3 grid(SIMD, nshards);
  primary_finalize_kernel<<<grid, 256, smem, st>>>(a_out, a_zq, a_ms, g, T, host_crt_const());
}

void launch_secondary_chain(const uint32_t* E, const uint32_t* qv, size_t qv_stride, int nq, uint32_t* out,
                            const Group& g, const ChainConsts& cc, const NttTables& T, cudaStream_t st) {
  const size_t smem = (size_t)8 * g.n * 4;
  set_smem(secondary_chain_kernel, smem);
  dim3 grid(CTXT_PARTS, g.H, nq);
  secondary_chain_kernel<<<grid, CHAIN_THREADS, smem, st>>>(E, qv, qv_stride, nq * CTXT_PARTS, out, g, cc, T,
                                                            host_crt_const());
}

}  // namespace dnspir
