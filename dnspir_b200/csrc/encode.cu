// encode.cu -- database encoding on the GPU (set_transformed_entries,
// crates/pir/src/base_pir.rs:662-772).
//
// For a database of group order l with columns a_t (t < l, each a ring element
// per lane), row c of the reference's transformed entries is
//     E_c = lift_t( l^-1 * sigma_{5^-r}( A^_r ) ),   r = L-1-c,
//     A^_r = sum_t a_t X^(-qbp 5^r t)          (main half)
//     A~_r = sum_t a_t X^(+qbp 5^r t)          (conjugate half, l = N only)
// (base_pir.rs STEP 3-6).  The reference reaches this with a column NTT, a
// coset NTT per row, a Galois permutation per column, a reversal, and a lift
// through the coefficient domain.  Here:
//   cols: A_t = NTT_N(a_t)                                   (q1)
//   rows: for each slot u, W_u = NTT_{N/qbp}(A_.[u]) (zero-padded over t);
//         A^_r[u] and A~_r[u] are entries of W_u at the orbit of (2u+1) under 5
//   lift: iNTT_N, centred lift, * l^-1 mod t, centred lift, NTT_N in q1 and q2.
// The scan stores E_c permuted by the slot map it reads with, which cancels
// sigma_{5^-r}: in the scan layout row c of the entries is NTT(lift(l^-1 A^_r))
// in natural slot order.  The exactness argument is the reference's: every
// coefficient of A^_r is below l * t < q1 / 2 in magnitude (:668-670).
#include <vector>

#include "kernels.cuh"
#include "ntt2048.cuh"

namespace dnspir {

Group make_group(int log2n, uint32_t l) {
  Group g;
  g.log2n = log2n;
  g.n = 1u << log2n;
  g.l = l;
  g.L = l < g.n ? l : g.n / 2;
  g.H = l == g.n ? 2 : 1;
  g.qbp = g.n / 2 / g.L;
  return g;
}

namespace {

__global__ void encode_cols_kernel(const uint16_t* __restrict__ in, uint32_t* __restrict__ A, int log2n,
                                   uint32_t total, int ppc, NttTables T) {
  extern __shared__ uint32_t sm[];
  const uint32_t n = 1u << log2n;
  const uint32_t first = blockIdx.x * ppc;
  const int cnt = min((uint32_t)ppc, total - first);
  for (uint32_t b = threadIdx.x; b < (uint32_t)cnt * n; b += blockDim.x) sm[b] = in[(size_t)first * n + b];
  __syncthreads();
  ntt_fwd_smem(sm, log2n, cnt, T, 0);
  // transform-position order: position x holds slot brv(x)
  for (uint32_t b = threadIdx.x; b < (uint32_t)cnt * n; b += blockDim.x) A[(size_t)first * n + b] = sm[b];
}

// One block: U consecutive slots u of one lane.  Transforms the length-l
// vector over t (zero-padded to n2 = N / qbp) and scatters the orbit values.
__global__ void encode_rows_kernel(const uint32_t* __restrict__ A, uint32_t* __restrict__ Ahat, Group g,
                                   uint32_t l_in, int nl, int U, int logn2, const uint32_t* __restrict__ pow5,
                                   NttTables T) {
  extern __shared__ uint32_t sm[];
  const int k = blockIdx.y;
  const uint32_t x0 = blockIdx.x * U;  // first transform position of the block
  const uint32_t n2 = 1u << logn2;
  const uint32_t N = g.n;
  if (U == 8) {
    // one thread per t: the 8 slots are one 32-byte sector, and a warp's
    // stores to each slot's row hit 32 consecutive banks
    for (uint32_t t = threadIdx.x; t < n2; t += blockDim.x) {
      uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
      if (t < l_in) {
        const uint4* src = reinterpret_cast<const uint4*>(A + ((size_t)t * nl + k) * N + x0);
        lo = __ldg(src);
        hi = __ldg(src + 1);
      }
      sm[0 * n2 + t] = lo.x, sm[1 * n2 + t] = lo.y, sm[2 * n2 + t] = lo.z, sm[3 * n2 + t] = lo.w;
      sm[4 * n2 + t] = hi.x, sm[5 * n2 + t] = hi.y, sm[6 * n2 + t] = hi.z, sm[7 * n2 + t] = hi.w;
    }
  } else {
    for (uint32_t b = threadIdx.x; b < (uint32_t)U * n2; b += blockDim.x) {
      const uint32_t t = b / U, uu = b % U;
      uint32_t v = 0;
      if (t < l_in) v = A[((size_t)t * nl + k) * N + x0 + uu];
      sm[uu * n2 + t] = v;
    }
  }
  __syncthreads();
  ntt_fwd_smem(sm, logn2, U, T, 0);
  const uint32_t mask = 2 * n2 - 1;
  const uint32_t outs = g.H * g.L * U;
  for (uint32_t b = threadIdx.x; b < outs; b += blockDim.x) {
    const uint32_t uu = b % U;
    const uint32_t r = (b / U) % g.L;
    const uint32_t h = b / (U * g.L);
    // A and Ahat are in transform-position order: position x holds slot brv(x)
    const uint32_t x = x0 + uu;
    const uint32_t u = brv(x, g.log2n);
    const uint32_t g5 = ((2 * u + 1) * pow5[r]) & mask;
    // slot s of W holds V(zeta^(-qbp (2s+1))): main needs exponent (2u+1) qbp 5^r
    const uint32_t s = h == 0 ? ((mask + 1 - g5) & mask) >> 1 : g5 >> 1;
    Ahat[(((size_t)h * g.L + r) * nl + k) * N + x] = sm[uu * n2 + brv(s, logn2)];
  }
}

// One block: column r of half h for up to 8 lanes.
constexpr int LIFT_LANES_CHAIN = 4;

__global__ void encode_lift_kernel(const uint32_t* __restrict__ Ahat, uint32_t* __restrict__ out, Group g, int nl,
                                   int frame, uint32_t scale, const uint32_t* __restrict__ pow5inv,
                                   const uint32_t* __restrict__ gtab, NttTables T) {
  extern __shared__ uint32_t sm[];
  const uint32_t r = blockIdx.x, h = blockIdx.y;
  const int lpb = frame == 0 ? 8 : LIFT_LANES_CHAIN;  // lanes per block
  const int lane0 = blockIdx.z * lpb;
  const int nlg = min(lpb, nl - lane0);
  const uint32_t N = g.n;
  const int logn = g.log2n;
  uint32_t* x1 = sm;
  uint32_t* x2 = sm + nlg * N;
  // Ahat rows are in transform-position order, the inverse transform's input order
  for (uint32_t b = threadIdx.x; b < (uint32_t)nlg * N; b += blockDim.x) {
    const uint32_t kk = b >> logn;
    x1[b] = Ahat[(((size_t)h * g.L + r) * nl + lane0 + kk) * N + (b & (N - 1))];
  }
  __syncthreads();
  ntt_inv_smem(x1, logn, nlg, T, 0);
  for (uint32_t b = threadIdx.x; b < (uint32_t)nlg * N; b += blockDim.x) {
    const uint32_t v = x1[b];
    const int32_t c = v > P1 / 2 ? (int32_t)v - (int32_t)P1 : (int32_t)v;
    int32_t m = c % (int32_t)TPLAIN;
    if (m < 0) m += TPLAIN;
    m = (int32_t)(((uint32_t)m * scale) % TPLAIN);
    const int32_t y = m > (int32_t)(TPLAIN / 2) ? m - (int32_t)TPLAIN : m;
    x1[b] = y < 0 ? (uint32_t)(y + (int32_t)P1) : (uint32_t)y;
    x2[b] = y < 0 ? (uint32_t)(y + (int32_t)P2) : (uint32_t)y;
  }
  __syncthreads();
  ntt_fwd_smem2(sm, logn, nlg, nlg, T);
  const uint32_t c = g.L - 1 - r;
  if (frame == 0) {
    // scan layout: 8 lanes interleaved, (sign, e) position u holds natural slot (g[u]-1)/2
    for (uint32_t b = threadIdx.x; b < 2 * N * SIMD; b += blockDim.x) {
      const uint32_t p = b / (N * SIMD);
      const uint32_t rem = b % (N * SIMD);
      const uint32_t u = rem / SIMD, kk = rem % SIMD;
      const uint32_t k = (__ldg(gtab + u) - 1) >> 1;
      out[slab_off(g, p, h, c, 0, u) + kk] = sm[((p * nlg + kk) << logn) + brv(k, logn)];
    }
  } else {
    // chain layout, bit-reversed positions, E_c[j] = E^_r[idx(5^-r (2j+1))]
    const uint32_t mask = 2 * N - 1;
    for (uint32_t b = threadIdx.x; b < 2 * (uint32_t)nlg * N; b += blockDim.x) {
      const uint32_t p = b / (nlg * N);
      const uint32_t rem = b % (nlg * N);
      const uint32_t kk = rem >> logn, pos = rem & (N - 1);
      const uint32_t j = brv(pos, logn);
      const uint32_t src = gidx(pow5inv[r] * (2 * j + 1), mask);
      out[((((size_t)p * g.H + h) * g.L + c) * nl + lane0 + kk) * N + pos] =
          sm[((p * nlg + kk) << logn) + brv(src, logn)];
    }
  }
}

// ---- N = 2048: the same three steps on the register transforms of
// ntt2048.cuh (padded shared layout, 512 threads, 16-byte global accesses).
constexpr int NT2K = 512;
constexpr uint32_t LIFT_M = TPLAIN << 15;  // a multiple of t above q1 / 2

__global__ void __launch_bounds__(NT2K) encode_cols2k_kernel(const uint16_t* __restrict__ in,
                                                             uint32_t* __restrict__ A, uint32_t total, int ppc,
                                                             NttTables T) {
  extern __shared__ __align__(16) uint32_t sm[];
  using namespace n2k;
  const uint32_t first = blockIdx.x * ppc;
  const int cnt = min((uint32_t)ppc, total - first);
  for (int b = threadIdx.x; b < cnt * (N / 4); b += NT2K) {
    const int kk = b >> 9, q = b & (N / 4 - 1);
    const uint2 w = __ldg(reinterpret_cast<const uint2*>(in + ((size_t)first + kk) * N) + q);
    *reinterpret_cast<uint4*>(sm + kk * PS + phys(4 * q)) =
        make_uint4(w.x & 0xffffu, w.x >> 16, w.y & 0xffffu, w.y >> 16);
  }
  __syncthreads();
  fwd<NT2K>(sm, cnt, 0, T);
  // transform-position order: position x holds slot brv(x)
  for (int b = threadIdx.x; b < cnt * (N / 4); b += NT2K) {
    const int kk = b >> 9, q = b & (N / 4 - 1);
    reinterpret_cast<uint4*>(A + ((size_t)first + kk) * N)[q] =
        *reinterpret_cast<const uint4*>(sm + kk * PS + phys(4 * q));
  }
}

// One block: 8 consecutive transform positions x0 .. x0 + 7 of one lane, the
// length-2048 transform over t (qbp = 1), both halves' orbit values written.
__global__ void __launch_bounds__(NT2K) encode_rows2k_kernel(const uint32_t* __restrict__ A,
                                                             uint32_t* __restrict__ Ahat, Group g, uint32_t l_in,
                                                             int nl, const uint32_t* __restrict__ pow5,
                                                             NttTables T) {
  extern __shared__ __align__(16) uint32_t sm[];
  using namespace n2k;
  const int k = blockIdx.y;
  const uint32_t x0 = blockIdx.x * 8;
  for (uint32_t t = threadIdx.x; t < (uint32_t)N; t += NT2K) {
    uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
    if (t < l_in) {
      const uint4* src = reinterpret_cast<const uint4*>(A + ((size_t)t * nl + k) * N + x0);
      lo = __ldg(src);
      hi = __ldg(src + 1);
    }
    const uint32_t o = phys(t);
    sm[0 * PS + o] = lo.x, sm[1 * PS + o] = lo.y, sm[2 * PS + o] = lo.z, sm[3 * PS + o] = lo.w;
    sm[4 * PS + o] = hi.x, sm[5 * PS + o] = hi.y, sm[6 * PS + o] = hi.z, sm[7 * PS + o] = hi.w;
  }
  __syncthreads();
  fwd<NT2K>(sm, 8, 0, T);
  constexpr uint32_t mask = 2 * N - 1;
  const int uu = threadIdx.x & 7;
  const uint32_t x = x0 + uu;
  const uint32_t odd = 2 * brv11(x) + 1;  // A and Ahat are in transform-position order
  const uint32_t* w = sm + uu * PS;
  for (uint32_t r = threadIdx.x >> 3; r < g.L; r += NT2K / 8) {
    // slot s of W holds V(zeta^(-(2s+1))): the main half needs exponent (2u+1) 5^r
    const uint32_t g5 = (odd * __ldg(pow5 + r)) & mask;
    Ahat[((size_t)r * nl + k) * N + x] = w[phys(brv11(((mask + 1 - g5) & mask) >> 1))];
    if (g.H == 2) Ahat[(((size_t)g.L + r) * nl + k) * N + x] = w[phys(brv11(g5 >> 1))];
  }
}

// Ends the inverse transform of the lift: coefficient v (mod q1, unscaled)
// -> c = centred(v N^-1), y = centred((c l^-1) mod t), written as y mod q1 in
// place and y mod q2 into polynomial cnt + poly.  (c l^-1) mod t is taken as
// (u s) mod t with u = c + LIFT_M > 0 and a Shoup quotient for s = l^-1 mod t.
struct LiftFin {
  int cnt;
  uint32_t s, sq;  // l^-1 mod t and floor(s 2^32 / t)
  __device__ __forceinline__ void operator()(uint32_t* y, int, int, uint32_t (&v)[8], uint32_t p, uint32_t ni,
                                             uint32_t niq) const {
    using namespace n2k;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const uint32_t c = red(lazy_mul(v[k], ni, niq, p), p);
      const uint32_t u = c + (c > P1 / 2 ? LIFT_M - P1 : LIFT_M);
      uint32_t m = u * s - __umulhi(u, sq) * TPLAIN;  // in [0, 2t)
      m = m >= TPLAIN ? m - TPLAIN : m;
      const bool neg = m > TPLAIN / 2;
      y[k * Geo8<1>::STR] = neg ? m + (P1 - TPLAIN) : m;
      y[cnt * PS + k * Geo8<1>::STR] = neg ? m + (P2 - TPLAIN) : m;
    }
  }
};

// One block: column r of half h for up to LIFT_LANES_CHAIN lanes, chain layout.
__global__ void __launch_bounds__(NT2K) encode_lift2k_kernel(const uint32_t* __restrict__ Ahat,
                                                             uint32_t* __restrict__ out, Group g, int nl,
                                                             uint32_t scale, uint32_t scale_q,
                                                             const uint32_t* __restrict__ pow5inv, NttTables T) {
  extern __shared__ __align__(16) uint32_t sm[];
  using namespace n2k;
  const uint32_t r = blockIdx.x, h = blockIdx.y;
  const int lane0 = blockIdx.z * LIFT_LANES_CHAIN;
  const int nlg = min(LIFT_LANES_CHAIN, nl - lane0);
  for (int b = threadIdx.x; b < nlg * (N / 4); b += NT2K) {
    const int kk = b >> 9, q = b & (N / 4 - 1);
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(Ahat + (((size_t)h * g.L + r) * nl + lane0 + kk) * N) + q);
    *reinterpret_cast<uint4*>(sm + kk * PS + phys(4 * q)) = v;
  }
  __syncthreads();
  inv<NT2K>(sm, nlg, 0, T, LiftFin{nlg, scale, scale_q});
  fwd<NT2K>(sm, nlg, nlg, T);
  // E_c[j] = E^_r[idx(5^-r (2j+1))] at bit-reversed position brv(j)
  const uint32_t c = g.L - 1 - r;
  const uint32_t pw = __ldg(pow5inv + r);
  constexpr uint32_t mask = 2 * N - 1;
  for (int q = threadIdx.x; q < N / 4; q += NT2K) {
    uint32_t idx[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const uint32_t j = brv11(4 * q + m);
      idx[m] = phys(brv11(((pw * (2 * j + 1)) & mask) >> 1));
    }
    for (int pk = 0; pk < 2 * nlg; pk++) {
      const int pp = pk >= nlg, kk = pk - pp * nlg;
      const uint32_t* s = sm + pk * PS;
      reinterpret_cast<uint4*>(out + ((((size_t)pp * g.H + h) * g.L + c) * nl + lane0 + kk) * N)[q] =
          make_uint4(s[idx[0]], s[idx[1]], s[idx[2]], s[idx[3]]);
    }
  }
}

__global__ void pack_bytes_kernel(const uint8_t* __restrict__ bytes, uint16_t* __restrict__ coeffs, size_t groups) {
  // pack_bytes_into_coeffs (dns/bucket.rs:289-303): 5 bytes -> 4 ten-bit coefficients
  const size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= groups) return;
  const uint8_t* s = bytes + gi * 5;
  const uint64_t v = (uint64_t)s[0] | ((uint64_t)s[1] << 8) | ((uint64_t)s[2] << 16) | ((uint64_t)s[3] << 24) |
                     ((uint64_t)s[4] << 32);
  uint16_t* o = coeffs + gi * 4;
  o[0] = (uint16_t)(v & 1023);
  o[1] = (uint16_t)((v >> 10) & 1023);
  o[2] = (uint16_t)((v >> 20) & 1023);
  o[3] = (uint16_t)((v >> 30) & 1023);
}

// Device tables of 5^r and 5^-r mod 2N (r < N/2), one per log2n.
struct PowTables {
  uint32_t* pow5[LOG2_N_MAX + 1] = {};
  uint32_t* pow5inv[LOG2_N_MAX + 1] = {};
};

}  // namespace

// Host copies of the powers of 5 (computed once per process and device).
static const uint32_t* pow_table(int log2n, bool inverse) {
  static PowTables tabs[64];
  int dev = 0;
  cudaGetDevice(&dev);
  PowTables& pt = tabs[dev & 63];
  uint32_t*& slot = inverse ? pt.pow5inv[log2n] : pt.pow5[log2n];
  if (!slot) {
    const uint32_t two_n = 2u << log2n;
    std::vector<uint32_t> h(two_n / 4 + 1);
    uint32_t inv5 = 1;
    for (uint32_t x = 1; x < two_n; x += 2)
      if ((5 * x) % two_n == 1) inv5 = x;
    uint32_t base = inverse ? inv5 : 5, cur = 1;
    for (size_t r = 0; r < h.size(); r++) {
      h[r] = cur;
      cur = (cur * base) % two_n;
    }
    uint32_t* d = nullptr;
    if (cudaMalloc(&d, h.size() * 4) != cudaSuccess) return nullptr;
    cudaMemcpy(d, h.data(), h.size() * 4, cudaMemcpyHostToDevice);
    slot = d;
  }
  return slot;
}

void launch_encode_cols(const uint16_t* in, uint32_t* A, const Group& g, uint32_t l_in, int nl, const NttTables& T,
                        cudaStream_t st) {
  const uint32_t total = l_in * nl;
  if (!total) return;
  if (g.log2n == 11) {
    const int ppc = 4;
    const size_t smem = (size_t)ppc * n2k::PS * 4;
    set_smem(encode_cols2k_kernel, smem);
    encode_cols2k_kernel<<<(total + ppc - 1) / ppc, NT2K, smem, st>>>(in, A, total, ppc, T);
    return;
  }
  const int ppc = g.n >= 1024 ? 4 : 8;
  const size_t smem = (size_t)ppc * g.n * 4;
  const uint32_t blocks = (total + ppc - 1) / ppc;
  set_smem(encode_cols_kernel, smem);
  encode_cols_kernel<<<blocks, 256, smem, st>>>(in, A, g.log2n, total, ppc, T);
}

void launch_encode_rows(const uint32_t* A, uint32_t* Ahat, const Group& g, uint32_t l_in, int nl, const NttTables& T,
                        cudaStream_t st) {
  const int logn2 = g.log2n - __builtin_ctz(g.qbp);
  const uint32_t n2 = 1u << logn2;
  if (g.log2n == 11 && logn2 == 11) {
    const size_t smem = (size_t)8 * n2k::PS * 4;
    set_smem(encode_rows2k_kernel, smem);
    encode_rows2k_kernel<<<dim3(g.n / 8, nl), NT2K, smem, st>>>(A, Ahat, g, l_in, nl, pow_table(g.log2n, false), T);
    return;
  }
  int U = 8;
  while (U > 1 && (uint32_t)U > g.n) U >>= 1;
  const size_t smem = (size_t)U * n2 * 4;
  dim3 grid(g.n / U, nl);
  set_smem(encode_rows_kernel, smem);
  encode_rows_kernel<<<grid, 256, smem, st>>>(A, Ahat, g, l_in, nl, U, logn2, pow_table(g.log2n, false), T);
}

void launch_encode_lift(const uint32_t* Ahat, uint32_t* out, const Group& g, int nl, int frame, const SlotMaps& maps,
                        const NttTables& T, cudaStream_t st) {
  uint32_t linv = 1;
  for (uint32_t x = 1; x < TPLAIN; x++)
    if ((x * (g.l % TPLAIN)) % TPLAIN == 1) linv = x;
  if (g.log2n == 11 && frame == 1) {
    const uint32_t sq = (uint32_t)(((uint64_t)linv << 32) / TPLAIN);
    const int nlg = nl < LIFT_LANES_CHAIN ? nl : LIFT_LANES_CHAIN;
    const size_t smem = (size_t)2 * nlg * n2k::PS * 4;
    dim3 grid(g.L, g.H, (nl + LIFT_LANES_CHAIN - 1) / LIFT_LANES_CHAIN);
    set_smem(encode_lift2k_kernel, smem);
    encode_lift2k_kernel<<<grid, NT2K, smem, st>>>(Ahat, out, g, nl, linv, sq, pow_table(g.log2n, true), T);
    return;
  }
  // frame 0 writes the 8 lanes of a slot together; frame 1 (chain layout)
  // takes fewer lanes per block so that three blocks fit on an SM
  const int lpb = frame == 0 ? 8 : LIFT_LANES_CHAIN;
  const int nlg = nl < lpb ? nl : lpb;
  const size_t smem = (size_t)2 * nlg * g.n * 4;
  dim3 grid(g.L, g.H, (nl + lpb - 1) / lpb);
  set_smem(encode_lift_kernel, smem);
  encode_lift_kernel<<<grid, 512, smem, st>>>(Ahat, out, g, nl, frame, linv, pow_table(g.log2n, true), maps.g, T);
}

void launch_pack_bytes(const uint8_t* bytes, uint16_t* coeffs, size_t entries, int log2n, cudaStream_t st) {
  const size_t groups = entries * ((size_t)1 << log2n) / 4;
  pack_bytes_kernel<<<(unsigned)((groups + 255) / 256), 256, 0, st>>>(bytes, coeffs, groups);
}

const uint32_t* device_pow5(int log2n, bool inverse) { return pow_table(log2n, inverse); }

}  // namespace dnspir
