// tscan.cu -- the primary scan (main_pir_loop, crates/pir/src/base_pir.rs:
// 1085-1247) for a batch of queries on the tensor cores, exact over 8-bit limbs.
//
// With loop_len L = N/2 (every primary group at N = 2048, IndexGroup,
// base_pir.rs:168-174) each output slot u = (sign, e) meets every query slot
// d = (e + L - 1 - i) mod L of its sign exactly once, at row i.  Indexing the
// slab by d instead of i turns the scan, per (shard, factor p, sign), into a
// product of integer matrices
//     out[(e, lane), b] = sum_{K = (h, a, d)} A[(e, lane), K] * V[K, b]
// with A the slab (E, G0, G1 of each half h) and V the B queries (the query of
// half h, gk0, gk1 at slot (sign, d)).  Both factors are below 2^32 and split
// into four 8-bit limbs (the bytes of the word): tcgen05.mma kind::i8 forms the
// 16 limb products with u8 x u8 -> s32 accumulation, at most
// K * 255^2 <= 6144 * 65025 < 2^31 per entry, so no partial sum overflows;
// the epilogue recombines sum_{k,j} D_kj * (2^(8(k+j)) mod p) < 2^59 in 64 bits
// and reduces it mod p.  The result is the same residue as the CUDA-core scan.
//
// Tensor layout of one shard (bytes), blocks [p][sign][mt][kc] of 16 KiB: each
// block is 128 rows x 128 bytes in the 128-byte-swizzled K-major form the MMA
// reads (16-byte unit c of row r stored at unit c ^ (r mod 8)).  Row r of
// m-tile mt is limb r mod 4 of lane (r / 4) mod 8 of slot e = 4 mt + r / 32;
// byte kb of K-chunk kc is K index kk = 128 kc + kb = (h * 3 + a) * L + d.
// The query operand has the same form: [p][sign][kc][n = 4 b + j][128 bytes].
//
// One CTA of 128 threads per (shard, p, sign, m-tiles, query group): thread 0
// streams A and V chunks into a ring of shared-memory stages with bulk copies,
// thread 32 issues the MMAs into a TMEM accumulator, then all four warps read
// their 32 TMEM lanes and write the reduced residues.  Every wait is bounded;
// a wait that gives up sets an error word, and the CTA still waits for its
// copies in flight and frees its TMEM before returning.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <string.h>

#include <algorithm>
#include <vector>

#include "kernels.cuh"

namespace dnspir {
namespace {

constexpr uint32_t TBLK = 16384;  // one 128 x 128-byte block
constexpr int TSCAN_NT = 128;
constexpr uint64_t WAIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t sa(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sa(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(sa(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// The same test, but a thread whose phase is not complete may stay suspended
// up to hint_ns (instead of the system's shorter default) before it returns
// false: long waits (an epilogue warp waiting out a tile's MMAs) then issue
// almost nothing while they wait.
__device__ __forceinline__ bool mbar_try_sleep(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(sa(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}
constexpr uint32_t SLEEP_HINT_NS = 20000;

// Wait for the phase of `parity` to complete; false after limit_ns.
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  while (!mbar_try_sleep(bar, parity, SLEEP_HINT_NS))
    if (gtimer() - t0 > limit_ns) return false;
  return true;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   sa(dst)),
               "l"(src), "r"(bytes), "r"(sa(bar))
               : "memory");
}

// Tensor-map copy of the box at (x, y) into this CTA's shared memory, issued
// by either CTA of a pair: the byte count completes on the barrier at
// shared::cluster address mbar, which .cta_group::2 allows to be the peer's
// (here always the leader's), so the leader learns of both CTAs' data from
// one barrier.
__device__ __forceinline__ void tma_load_pair(void* dst, const CUtensorMap* map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(sa(dst)),
      "l"(map), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

// The same with an L2 cache policy (createpolicy): the query operand, which
// every CTA re-reads for every slab tile, is kept in L2 with evict_last --
// without it the tensor-map copies of the query operand went back to DRAM
// (at 256 queries the pair kernel read 2.9 x the slab bytes from DRAM).
__device__ __forceinline__ void tma_load_pair_hint(void* dst, const CUtensorMap* map, int x, int y, uint32_t mbar,
                                                   uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], "
      "[%1, {%2, %3}], [%4], %5;" ::"r"(sa(dst)),
      "l"(map), "r"(x), "r"(y), "r"(mbar), "l"(policy)
      : "memory");
}
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major, 128-byte swizzle, 8-row groups 1024 bytes apart (tcgen05 shared
// memory descriptor: start >> 4, LBO >> 4, SBO >> 4, version 1, layout 2).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor, kind::i8: D s32, A and B unsigned 8-bit, both K-major.
__host__ __device__ constexpr uint32_t idesc_u8(int M, int N) {
  return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_u8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sa(bar))
               : "memory");
}

// TMEM columns taddr .. taddr + 15 of this warp's 32 lanes; the wait is in the
// same asm statement, so no use of v can be scheduled before the data is there
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}
// TMEM columns taddr .. taddr + 63 of this warp's 32 lanes; the wait is in the
// same asm statement, so no use of v can be scheduled before the data is there
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
      : "r"(taddr)
      : "memory");
}

struct TScanArgs {
  const uint8_t* const* slabs;  // per shard, tensor layout
  int nshards;
  const uint8_t* qb;  // query operand [p][sign][kc][nq_rows][128]
  uint32_t nq_rows;   // rows of the query operand: 4 x padded batch
  uint32_t nvalid;    // queries whose results are written
  uint32_t* out;      // [b][s][p][u][lane]
  uint32_t* err;      // set to 1 when a wait gives up
  uint32_t half, mt_total, kc_total, groups, stages;
  uint64_t wait_ns;   // limit of every pipeline wait
  uint32_t withhold;  // test hook: CTA 0's producer stops before this chunk (~0u: never)
  const CUtensorMap* tmaps;  // per shard: the slab as rows of 128 bytes (tensor-map pair kernel)
};

// c_w = 2^(8w) mod p (< 2^26) for w = k .. k + 3: the weights of limb product
// D_kj (j = 0..3) in the recombination
__device__ __forceinline__ void limb_weights(uint32_t pr, uint64_t mu, int k, uint32_t (&c)[4]) {
  const uint32_t w3 = (uint32_t)reduce64(1ull << 24, pr, mu);
  const uint64_t c32 = reduce64(1ull << 32, pr, mu);
  const uint64_t c40 = reduce64(c32 << 8, pr, mu);
  const uint64_t c48 = reduce64(c40 << 8, pr, mu);
  c[0] = k == 0 ? 1u : k == 1 ? 256u : k == 2 ? 65536u : w3;
  c[1] = k == 0 ? 256u : k == 1 ? 65536u : k == 2 ? w3 : (uint32_t)c32;
  c[2] = k == 0 ? 65536u : k == 1 ? w3 : k == 2 ? (uint32_t)c32 : (uint32_t)c40;
  c[3] = k == 0 ? w3 : k == 1 ? (uint32_t)c32 : k == 2 ? (uint32_t)c40 : (uint32_t)c48;
}

// Epilogue of one m-tile: the warp's 32 TMEM lanes (rows (slot, lane, limb k)
// of output slot u) x NQ columns (query-operand rows 4 b + j of query group
// grp) starting at TMEM address taddr.  Each query's 16 limb products are
// recombined with the weights c and reduced mod pr; lanes 4 l8 .. 4 l8 + 3
// hold the four limbs k of SIMD lane l8, so three of every four lanes sum the
// others' partial recombinations with shuffles and lane k keeps query
// 4 q4 + k's sum.  The warp reads columns c_lo .. c_hi - 1 (multiples of the
// load width), 64 (16 for NQ = 16) per TMEM load.
template <int NQ>
__device__ __forceinline__ void epilogue_tile(const TScanArgs& a, uint32_t taddr, const uint32_t (&c)[4], uint32_t pr,
                                              uint64_t mu, uint32_t grp, uint32_t u, int s, int p, int k, int l8,
                                              int c_lo = 0, int c_hi = NQ) {
  constexpr int CW = NQ >= 64 ? 64 : 16;  // columns per TMEM load
  const uint32_t N = 2 * a.half;
#pragma unroll 1
  for (int c0 = c_lo; c0 < c_hi; c0 += CW) {
    uint32_t v[CW];
    if constexpr (CW == 64)
      tmem_ld64(taddr + c0, v);
    else
      tmem_ld16(taddr + c0, v);
#pragma unroll
    for (int q4 = 0; q4 < CW / 16; q4++) {
      uint64_t tot[4];
#pragma unroll
      for (int qq = 0; qq < 4; qq++) {
        const uint32_t* w = v + 16 * q4 + 4 * qq;
        uint64_t x = (uint64_t)w[0] * c[0] + (uint64_t)w[1] * c[1] + (uint64_t)w[2] * c[2] + (uint64_t)w[3] * c[3];
        x += __shfl_xor_sync(0xffffffffu, x, 1);
        x += __shfl_xor_sync(0xffffffffu, x, 2);
        tot[qq] = x;
      }
      const uint64_t mine = k == 0 ? tot[0] : k == 1 ? tot[1] : k == 2 ? tot[2] : tot[3];
      const uint32_t bq = grp * (NQ / 4) + (c0 / 16 + q4) * 4 + k;
      if (bq < a.nvalid) a.out[((((size_t)bq * a.nshards + s) * 2 + p) * N + u) * SIMD + l8] = reduce64(mine, pr, mu);
    }
  }
}

template <int NQ, int MTPC>
__global__ void __launch_bounds__(TSCAN_NT, 1) tscan_kernel(TScanArgs a) {
  constexpr uint32_t A_BYTES = MTPC * TBLK;
  constexpr uint32_t STAGE = A_BYTES + NQ * 128;
  constexpr uint32_t COLS = (MTPC * NQ) <= 32 ? 32 : (MTPC * NQ);
  constexpr int NSPLIT = NQ > 256 ? NQ / 256 : 1;
  constexpr int NMMA = NQ / NSPLIT;
  static_assert(STAGE % 1024 == 0 && COLS <= 512 && (COLS & (COLS - 1)) == 0, "tile shape");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const uint32_t S_ = a.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + S_ * STAGE);
  uint64_t* empty = full + S_;
  uint64_t* accb = empty + S_;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(accb + 1);
  volatile uint32_t* issued_s = tslot + 1;
  volatile uint32_t* consumed_s = tslot + 2;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

  // item = (((s * 2 + p) * 2 + sign) * mtc + mtc_i) * groups + grp
  uint32_t item = blockIdx.x;
  const uint32_t grp = item % a.groups;
  item /= a.groups;
  const uint32_t mtc = a.mt_total / MTPC;
  const uint32_t mt0 = (item % mtc) * MTPC;
  item /= mtc;
  const uint32_t sgn = item & 1;
  const int p = (item >> 1) & 1;
  const int s = item >> 2;
  const uint32_t KC = a.kc_total;
  const size_t ps = (size_t)p * 2 + sgn;
  const uint8_t* abase = a.slabs[s] + (ps * a.mt_total + mt0) * KC * TBLK;
  const uint8_t* bbase = a.qb + ps * KC * a.nq_rows * 128 + (size_t)grp * NQ * 128;

  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < S_; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(accb, 1);
    *issued_s = 0;
    *consumed_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa(tslot)), "r"(COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  if (threadIdx.x == 0) {
    // producer: chunk kc of every m-tile and of the query group into stage kc % S_
    uint32_t issued = 0;
    for (uint32_t kc = 0; kc < KC; kc++) {
      const uint32_t st = kc % S_, n = kc / S_;
      if (blockIdx.x == 0 && kc == a.withhold) break;  // test hook: a chunk that never arrives
      if (n > 0 && !mbar_wait(&empty[st], (n - 1) & 1, a.wait_ns)) {
        atomicOr(a.err, 1u);
        break;
      }
      uint8_t* dst = sm + st * STAGE;
      mbar_expect_tx(&full[st], STAGE);
#pragma unroll
      for (int t = 0; t < MTPC; t++) bulk_g2s(dst + t * TBLK, abase + ((size_t)t * KC + kc) * TBLK, TBLK, &full[st]);
      bulk_g2s(dst + A_BYTES, bbase + (size_t)kc * a.nq_rows * 128, NQ * 128, &full[st]);
      issued = kc + 1;
    }
    *issued_s = issued;
  } else if (threadIdx.x == 32) {
    // MMA issuer
    constexpr uint32_t idesc = idesc_u8(128, NMMA);
    uint32_t consumed = 0;
    for (uint32_t kc = 0; kc < KC; kc++) {
      const uint32_t st = kc % S_, n = kc / S_;
      if (!mbar_wait(&full[st], n & 1, a.wait_ns)) {
        atomicOr(a.err, 1u);
        break;
      }
      tc_fence_after();
      const uint32_t s0 = sa(sm + st * STAGE);
#pragma unroll
      for (int k = 0; k < 4; k++) {
#pragma unroll
        for (int t = 0; t < MTPC; t++) {
#pragma unroll
          for (int ns = 0; ns < NSPLIT; ns++)
            mma_u8(tmem + t * NQ + ns * NMMA, sw128_desc(s0 + t * TBLK + 32 * k),
                   sw128_desc(s0 + A_BYTES + ns * NMMA * 128 + 32 * k), idesc, (kc | k) != 0);
        }
      }
      mma_commit(&empty[st]);
      consumed = kc + 1;
    }
    *consumed_s = consumed;
    mma_commit(accb);
  }
  __syncwarp();

  // epilogue: warp w holds TMEM lanes 32w..32w+31 = rows of slot e = 4 mt + w
  const bool acc_ok = mbar_wait(accb, 0, a.wait_ns);
  tc_fence_after();
  if (acc_ok) {
    const uint32_t pr = prime_of(p);
    const uint64_t mu = barrett_mu(pr);
    const int k = lane & 3, l8 = lane >> 2;
    uint32_t c[4];
    limb_weights(pr, mu, k, c);
    for (int t = 0; t < MTPC; t++)
      epilogue_tile<NQ>(a, tmem + ((uint32_t)(32 * warp) << 16) + t * NQ, c, pr, mu, grp,
                        sgn * a.half + 4 * (mt0 + t) + warp, s, p, k, l8);
  } else if (threadIdx.x == 0) {
    atomicOr(a.err, 1u);
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    // copies issued but never consumed (only after a wait gave up) must land
    // before the shared memory is released
    for (uint32_t kc = *consumed_s; kc < *issued_s; kc++) mbar_wait(&full[kc % S_], (kc / S_) & 1, a.wait_ns);
  }
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(COLS) : "memory");
  }
}

// ---- persistent, warp-specialised variant.  Warp 0 streams the A and V
// chunks of every tile the CTA owns (tiles blockIdx.x, + gridDim.x, ...)
// through the stage ring; warp 1 issues the MMAs of tile j into TMEM
// accumulator j mod 2; warps 2 .. 2 + 4 EW - 1 read accumulator j mod 2 (TMEM
// lane quarter warp mod 4; the EW warps of a quarter split the columns, 64
// each) and write the residues, then release it, so the epilogue of tile j
// overlaps the main loop of tile j + 1.  With 2 x MTPC x NQ > 512 TMEM columns
// there is one accumulator and the MMAs of a tile wait for the previous
// tile's epilogue: the EW warps per quarter keep that wait short (one warp per
// quarter leaves each scheduler one dependent chain of TMEM loads, shuffles
// and reductions).  Waits are bounded as in tscan_kernel; a role that gives
// up raises the abort flag, and the CTA still waits for its MMAs and copies
// in flight before it frees TMEM.
template <int NQ>
constexpr int tscanp_ew() {
  return NQ >= 256 ? 4 : NQ >= 128 ? 2 : 1;
}
template <int NQ>
constexpr int tscanp_nt() {
  return 64 + 128 * tscanp_ew<NQ>();
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sa(bar)) : "memory");
}

template <int NQ, int MTPC>
__global__ void __launch_bounds__(tscanp_nt<NQ>(), 1) tscanp_kernel(TScanArgs a) {
  constexpr uint32_t A_BYTES = MTPC * TBLK;
  constexpr uint32_t STAGE = A_BYTES + NQ * 128;
  constexpr uint32_t ACC = MTPC * NQ;  // TMEM columns of one accumulator
  // two accumulators when they fit the SM's 512 columns; with one, the MMAs of
  // a tile wait for the previous tile's epilogue, but its chunks still stream in
  constexpr uint32_t BUFS = 2 * ACC <= 512 ? 2 : 1;
  constexpr uint32_t COLS = BUFS * ACC;
  constexpr int EW = tscanp_ew<NQ>();  // epilogue warps per TMEM lane quarter
  static_assert(STAGE % 1024 == 0 && ACC >= 16 && COLS <= 512 && (COLS & (COLS - 1)) == 0, "tile shape");
  static_assert(NQ % EW == 0 && (EW == 1 || NQ / EW == 64), "columns per epilogue warp");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const uint32_t S_ = a.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + S_ * STAGE);
  uint64_t* empty = full + S_;
  uint64_t* accf = empty + S_;  // [2] accumulator ready (MMA commit)
  uint64_t* acce = accf + 2;    // [2] accumulator drained (4 epilogue warps)
  uint64_t* done = acce + 2;    // every MMA of the CTA complete
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  volatile uint32_t* issued_s = tslot + 1;
  volatile uint32_t* consumed_s = tslot + 2;
  volatile uint32_t* abort_s = tslot + 3;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const uint32_t mtc = a.mt_total / MTPC;
  const uint32_t items = (uint32_t)a.nshards * 4 * mtc * a.groups;
  const uint32_t KC = a.kc_total;

  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < S_; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4 * EW);
    }
    mbar_init(done, 1);
    *issued_s = 0;
    *consumed_s = 0;
    *abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa(tslot)), "r"(COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  auto tile_of = [&](uint32_t item, uint32_t& grp, uint32_t& mt0, uint32_t& sgn, int& p, int& s) {
    grp = item % a.groups;
    item /= a.groups;
    mt0 = (item % mtc) * MTPC;
    item /= mtc;
    sgn = item & 1;
    p = (item >> 1) & 1;
    s = item >> 2;
  };

  if (warp == 0) {
    if (lane == 0) {
      uint32_t g = 0;
      bool withheld = false;
      for (uint32_t item = blockIdx.x; item < items && !*abort_s && !withheld; item += gridDim.x) {
        uint32_t grp, mt0, sgn;
        int p, s;
        tile_of(item, grp, mt0, sgn, p, s);
        const size_t ps = (size_t)p * 2 + sgn;
        const uint8_t* abase = a.slabs[s] + (ps * a.mt_total + mt0) * KC * TBLK;
        const uint8_t* bbase = a.qb + ps * KC * a.nq_rows * 128 + (size_t)grp * NQ * 128;
        for (uint32_t kc = 0; kc < KC; kc++, g++) {
          const uint32_t st = g % S_, n = g / S_;
          if (blockIdx.x == 0 && g == a.withhold) {  // test hook: a chunk that never arrives
            withheld = true;
            break;
          }
          if (n > 0 && !mbar_wait(&empty[st], (n - 1) & 1, a.wait_ns)) {
            *abort_s = 1;
            atomicOr(a.err, 1u);
            break;
          }
          uint8_t* dst = sm + st * STAGE;
          mbar_expect_tx(&full[st], STAGE);
#pragma unroll
          for (int t = 0; t < MTPC; t++)
            bulk_g2s(dst + t * TBLK, abase + ((size_t)t * KC + kc) * TBLK, TBLK, &full[st]);
          bulk_g2s(dst + A_BYTES, bbase + (size_t)kc * a.nq_rows * 128, NQ * 128, &full[st]);
          *issued_s = g + 1;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_u8(128, NQ);
      uint32_t g = 0, j = 0;
      for (uint32_t item = blockIdx.x; item < items && !*abort_s; item += gridDim.x, j++) {
        const uint32_t buf = j % BUFS, use = j / BUFS;
        if (use > 0 && !mbar_wait(&acce[buf], (use - 1) & 1, a.wait_ns)) {
          *abort_s = 1;
          atomicOr(a.err, 1u);
          break;
        }
        tc_fence_after();
        bool ok = true;
        for (uint32_t kc = 0; kc < KC; kc++, g++) {
          const uint32_t st = g % S_, n = g / S_;
          if (!mbar_wait(&full[st], n & 1, a.wait_ns)) {
            *abort_s = 1;
            atomicOr(a.err, 1u);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t s0 = sa(sm + st * STAGE);
#pragma unroll
          for (int k = 0; k < 4; k++)
#pragma unroll
            for (int t = 0; t < MTPC; t++)
              mma_u8(tmem + buf * ACC + t * NQ, sw128_desc(s0 + t * TBLK + 32 * k), sw128_desc(s0 + A_BYTES + 32 * k),
                     idesc, (kc | k) != 0);
          mma_commit(&empty[st]);
          *consumed_s = g + 1;
        }
        if (!ok) break;
        mma_commit(&accf[buf]);
      }
      mma_commit(done);
    }
  } else {
    const int q = warp & 3;  // TMEM lane quarter = slot e mod 4 of the m-tile
    const int k = lane & 3, l8 = lane >> 2;
    const int c_lo = ((warp - 2) >> 2) * (NQ / EW);  // this warp's columns of every m-tile
    uint32_t j = 0;
    for (uint32_t item = blockIdx.x; item < items; item += gridDim.x, j++) {
      const uint32_t buf = j % BUFS, use = j / BUFS;
      if (!mbar_wait(&accf[buf], use & 1, a.wait_ns)) {
        if (lane == 0) {
          *abort_s = 1;
          atomicOr(a.err, 1u);
        }
        break;
      }
      tc_fence_after();
      uint32_t grp, mt0, sgn;
      int p, s;
      tile_of(item, grp, mt0, sgn, p, s);
      const uint32_t pr = prime_of(p);
      const uint64_t mu = barrett_mu(pr);
      uint32_t c[4];
      limb_weights(pr, mu, k, c);
      for (int t = 0; t < MTPC; t++)
        epilogue_tile<NQ>(a, tmem + ((uint32_t)(32 * q) << 16) + buf * ACC + t * NQ, c, pr, mu, grp,
                          sgn * a.half + 4 * (mt0 + t) + q, s, p, k, l8, c_lo, c_lo + NQ / EW);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[buf]);
    }
  }
  __syncthreads();
  if (threadIdx.x == 32) mbar_wait(done, 0, a.wait_ns);  // every MMA issued by the CTA has completed
  if (threadIdx.x == 0) {
    // copies issued but never consumed (only after a wait gave up) must land
    // before the shared memory is released
    for (uint32_t g = *consumed_s; g < *issued_s; g++) mbar_wait(&full[g % S_], (g / S_) & 1, a.wait_ns);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(COLS) : "memory");
  }
}

// ---- CTA-pair variant: tcgen05.mma.cta_group::2, persistent, warp-specialised.
// A cluster of two CTAs works on one item at a time: 2 x MTPC m-tiles of one
// (shard, factor, sign) against one query group.  CTA r keeps m-tiles
// mt0 + r MTPC + t (t < MTPC) in its shared memory and half of the group's
// query-operand rows (grp NQ + r NQ/2 ..); the leader (rank 0) issues M = 256
// MMAs that read both CTAs' operands, and each CTA's TMEM receives its own 128
// rows x NQ columns per m-tile.  Compared with the one-CTA kernels every SM
// stages only half of the query operand per chunk, so a ring of the same size
// holds more chunks.  Roles, in each CTA: warp 0 lane 0 streams the CTA's
// chunks into its ring (bulk copies, local full barrier); warp 1 lane 0 is the
// MMA issuer in the leader and, in the follower, the relay that forwards each
// completed stage to the leader's pfull barrier; the 4 EW warps after them
// read the TMEM accumulators and write the residues (EW per lane quarter, as
// in tscanp_kernel).  The leader's commits arrive on both
// CTAs' barriers (multicast commit); the epilogue warps of both CTAs release
// an accumulator on the leader's acce barrier.  Accumulators are
// double-buffered when 2 MTPC NQ <= 512 TMEM columns.  Every wait is bounded
// and also gives up once either CTA has raised the pair's abort flag; a CTA
// then waits (bounded) for its MMAs and copies in flight before it frees TMEM.

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_idx() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_count() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
// shared::cluster address of the same shared-memory offset in CTA `rank`
__device__ __forceinline__ uint32_t peer_addr(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(sa(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_arrive_peer(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ bool mbar_try_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, "
      "p;\n}\n"
      : "=r"(ok)
      : "r"(sa(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// The phase of `parity` completed (true), or limit_ns passed or the pair's
// abort flag was raised (false).
__device__ bool mbar_wait_pair(uint64_t* bar, uint32_t parity, uint64_t limit_ns, volatile uint32_t* abort_flag,
                               bool cluster_scope) {
  auto done = [&] { return cluster_scope ? mbar_try_cluster(bar, parity) : mbar_try(bar, parity); };
  if (done()) return true;
  const uint64_t t0 = gtimer();
  for (;;) {
    if (done()) return true;
    if (*abort_flag) return false;
    if (gtimer() - t0 > limit_ns) return false;
  }
}
// raise the abort flag of both CTAs of the pair and the error word
__device__ __forceinline__ void pair_abort(volatile uint32_t* abort_flag, uint32_t* err) {
  *abort_flag = 1;
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(peer_addr((const void*)abort_flag, cluster_rank() ^ 1)),
               "r"(1u)
               : "memory");
  atomicOr(err, 1u);
}
__device__ __forceinline__ void mma2_u8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive on the barrier at this offset in both CTAs once the leader's MMAs issued so far complete
__device__ __forceinline__ void mma2_commit_both(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          sa(bar)),
      "h"((uint16_t)3)
      : "memory");
}

template <int NQ, int MTPC, bool TMA>
__global__ void __launch_bounds__(tscanp_nt<NQ>(), 1) tscan2_kernel(const __grid_constant__ TScanArgs a,
                                                                    const __grid_constant__ CUtensorMap qmap) {
  constexpr int EW = tscanp_ew<NQ>();  // epilogue warps per TMEM lane quarter, as in tscanp_kernel
  constexpr uint32_t A_BYTES = MTPC * TBLK;
  constexpr uint32_t V_BYTES = NQ / 2 * 128;  // this CTA's half of the group's query rows
  constexpr uint32_t STAGE = A_BYTES + V_BYTES;
  constexpr uint32_t ACC = MTPC * NQ;  // TMEM columns of one accumulator
  constexpr uint32_t BUFS = 2 * ACC <= 512 ? 2 : 1;
  constexpr uint32_t COLS = BUFS * ACC < 32 ? 32 : BUFS * ACC;
  static_assert(NQ >= 32 && NQ <= 256 && NQ % 32 == 0, "pair MMA: N in 32..256, a multiple of 32");
  static_assert(STAGE % 1024 == 0 && ACC <= 512 && (COLS & (COLS - 1)) == 0, "tile shape");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const uint32_t S_ = a.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + S_ * STAGE);
  uint64_t* empty = full + S_;
  uint64_t* pfull = empty + S_;  // leader: the follower's stage landed
  uint64_t* accf = pfull + S_;   // [2] accumulator ready (multicast commit)
  uint64_t* acce = accf + 2;     // [2] accumulator drained (leader: 4 EW local + 4 EW remote warps)
  uint64_t* done = acce + 2;     // every MMA of the pair complete (multicast commit)
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  volatile uint32_t* issued_s = tslot + 1;
  volatile uint32_t* abort_s = tslot + 2;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const uint32_t rank = cluster_rank();
  const uint32_t mtc = a.mt_total / (2 * MTPC);  // m-tile groups of a pair
  const uint32_t items = (uint32_t)a.nshards * 4 * mtc * a.groups;
  const uint32_t KC = a.kc_total;
  const uint32_t cid = cluster_idx(), ncl = cluster_count();

  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < S_; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
      mbar_init(&pfull[i], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 8 * EW);
    }
    mbar_init(done, 1);
    *issued_s = 0;
    *abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa(tslot)), "r"(COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // both CTAs' barriers exist before any remote arrive or MMA
  tc_fence_after();
  const uint32_t tmem = *tslot;

  auto tile_of = [&](uint32_t item, uint32_t& grp, uint32_t& mt0, uint32_t& sgn, int& p, int& s) {
    grp = item % a.groups;
    item /= a.groups;
    mt0 = (item % mtc) * 2 * MTPC;
    item /= mtc;
    sgn = item & 1;
    p = (item >> 1) & 1;
    s = item >> 2;
  };

  if (warp == 0) {
    if (lane == 0) {
      uint32_t g = 0;
      bool stop = false;
      const uint64_t vpol = TMA ? l2_evict_last_policy() : 0;
      for (uint32_t item = cid; item < items && !stop; item += ncl) {
        uint32_t grp, mt0, sgn;
        int p, s;
        tile_of(item, grp, mt0, sgn, p, s);
        const size_t ps = (size_t)p * 2 + sgn;
        const uint8_t* abase = a.slabs[s] + (ps * a.mt_total + mt0 + rank * MTPC) * KC * TBLK;
        const uint8_t* bbase = a.qb + ps * KC * a.nq_rows * 128 + ((size_t)grp * NQ + rank * (NQ / 2)) * 128;
        for (uint32_t kc = 0; kc < KC; kc++, g++) {
          const uint32_t st = g % S_, n = g / S_;
          if (blockIdx.x == 0 && g == a.withhold) {  // test hook: a chunk that never arrives
            stop = true;
            break;
          }
          if (n > 0 && !mbar_wait_pair(&empty[st], (n - 1) & 1, a.wait_ns, abort_s, false)) {
            if (!*abort_s) pair_abort(abort_s, a.err);
            stop = true;
            break;
          }
          uint8_t* dst = sm + st * STAGE;
          if constexpr (TMA) {
            // both CTAs' copies complete on the leader's barrier, which the
            // leader arms with the pair's bytes (a copy may land before it is
            // armed: the transaction count may run below zero meanwhile)
            if (rank == 0) mbar_expect_tx(&full[st], 2 * STAGE);
            const uint32_t fb = peer_addr(&full[st], 0);
            const int arow = (int)(((ps * a.mt_total + mt0 + rank * MTPC) * KC + kc) * 128);
#pragma unroll
            for (int t = 0; t < MTPC; t++) tma_load_pair(dst + t * TBLK, a.tmaps + s, 0, arow + t * (int)KC * 128, fb);
            tma_load_pair_hint(dst + A_BYTES, &qmap, 0,
                               (int)((ps * KC + kc) * a.nq_rows + (size_t)grp * NQ + rank * (NQ / 2)), fb, vpol);
          } else {
            mbar_expect_tx(&full[st], STAGE);
#pragma unroll
            for (int t = 0; t < MTPC; t++)
              bulk_g2s(dst + t * TBLK, abase + ((size_t)t * KC + kc) * TBLK, TBLK, &full[st]);
            bulk_g2s(dst + A_BYTES, bbase + (size_t)kc * a.nq_rows * 128, V_BYTES, &full[st]);
          }
          *issued_s = g + 1;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank != 0) {
      if constexpr (!TMA) {
        // relay: each stage of this CTA that lands is announced to the leader
        // (with tensor-map copies the follower's copies signal the leader)
        const uint32_t total = ((items > cid ? (items - cid + ncl - 1) / ncl : 0)) * KC;
        for (uint32_t g = 0; g < total; g++) {
          const uint32_t st = g % S_, n = g / S_;
          if (!mbar_wait_pair(&full[st], n & 1, a.wait_ns, abort_s, false)) {
            if (!*abort_s) pair_abort(abort_s, a.err);
            break;
          }
          mbar_arrive_peer(peer_addr(&pfull[st], 0));
        }
      }
    } else if (lane == 0) {
      constexpr uint32_t idesc = idesc_u8(256, NQ);
      uint32_t g = 0, j = 0;
      bool stop = false;
      for (uint32_t item = cid; item < items && !stop; item += ncl, j++) {
        const uint32_t buf = j % BUFS, use = j / BUFS;
        if (use > 0 && !mbar_wait_pair(&acce[buf], (use - 1) & 1, a.wait_ns, abort_s, true)) {
          if (!*abort_s) pair_abort(abort_s, a.err);
          break;
        }
        tc_fence_after();
        for (uint32_t kc = 0; kc < KC; kc++, g++) {
          const uint32_t st = g % S_, n = g / S_;
          const bool landed = TMA ? mbar_wait_pair(&full[st], n & 1, a.wait_ns, abort_s, true)
                                  : mbar_wait_pair(&full[st], n & 1, a.wait_ns, abort_s, false) &&
                                        mbar_wait_pair(&pfull[st], n & 1, a.wait_ns, abort_s, true);
          if (!landed) {
            if (!*abort_s) pair_abort(abort_s, a.err);
            stop = true;
            break;
          }
          tc_fence_after();
          const uint32_t s0 = sa(sm + st * STAGE);
#pragma unroll
          for (int k = 0; k < 4; k++)
#pragma unroll
            for (int t = 0; t < MTPC; t++)
              mma2_u8(tmem + buf * ACC + t * NQ, sw128_desc(s0 + t * TBLK + 32 * k),
                      sw128_desc(s0 + A_BYTES + 32 * k), idesc, (kc | k) != 0);
          mma2_commit_both(&empty[st]);
        }
        if (stop) break;
        mma2_commit_both(&accf[buf]);
      }
      mma2_commit_both(done);
    }
  } else {
    const int q = warp & 3;  // TMEM lane quarter = slot e mod 4 of the m-tile
    const int k = lane & 3, l8 = lane >> 2;
    const uint32_t acce_leader = peer_addr(&acce[0], 0);
    const int c_lo = ((warp - 2) >> 2) * (NQ / EW);  // this warp's columns of every m-tile
    uint32_t j = 0;
    for (uint32_t item = cid; item < items; item += ncl, j++) {
      const uint32_t buf = j % BUFS, use = j / BUFS;
      if (!mbar_wait_pair(&accf[buf], use & 1, a.wait_ns, abort_s, false)) {
        if (lane == 0 && !*abort_s) pair_abort(abort_s, a.err);
        break;
      }
      tc_fence_after();
      uint32_t grp, mt0, sgn;
      int p, s;
      tile_of(item, grp, mt0, sgn, p, s);
      const uint32_t pr = prime_of(p);
      const uint64_t mu = barrett_mu(pr);
      uint32_t c[4];
      limb_weights(pr, mu, k, c);
      for (int t = 0; t < MTPC; t++)
        epilogue_tile<NQ>(a, tmem + ((uint32_t)(32 * q) << 16) + buf * ACC + t * NQ, c, pr, mu, grp,
                          sgn * a.half + 4 * (mt0 + rank * MTPC + t) + q, s, p, k, l8, c_lo, c_lo + NQ / EW);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        if (rank == 0)
          mbar_arrive(&acce[buf]);
        else
          mbar_arrive_peer(acce_leader + buf * 8);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 32) mbar_wait(done, 0, a.wait_ns);  // every MMA of the pair has completed
  if (threadIdx.x == 0 && *abort_s) {
    // copies issued but perhaps never consumed must land before the shared
    // memory is released (only after a wait gave up)
    const uint32_t iss = *issued_s;
    if (!TMA || rank == 0)
      for (uint32_t g = iss > S_ ? iss - S_ : 0; g < iss; g++) mbar_wait(&full[g % S_], (g / S_) & 1, a.wait_ns);
    if (TMA) {
      // a tensor-map copy completes on the leader's barrier, which may never
      // see its phase when the two CTAs stopped at different chunks: give the
      // copies in flight a fixed 50 us (they take a few) before either CTA
      // leaves
      const uint64_t t0 = gtimer();
      while (gtimer() - t0 < 50000) {
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // neither CTA leaves while the peer may still touch its barriers
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(COLS) : "memory");
  }
}

// Lane layout (slab_off) -> tensor layout; one thread per 16-byte unit.
__global__ void retile_kernel(const uint32_t* __restrict__ src, uint8_t* __restrict__ dst, Group g, uint32_t mt_total,
                              uint32_t kc_total) {
  const uint32_t half = g.n / 2;
  const size_t total = (size_t)4 * mt_total * kc_total * 1024;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const uint32_t c = idx & 7, r = (idx >> 3) & 127;
  size_t blk = idx >> 10;
  const uint32_t kc = blk % kc_total;
  blk /= kc_total;
  const uint32_t mt = blk % mt_total;
  blk /= mt_total;
  const uint32_t sgn = blk & 1;
  const int p = (int)(blk >> 1);
  const uint32_t e = 4 * mt + r / 32, lane = (r / 4) & 7, limb = r & 3;
  const uint32_t u = sgn * half + e;
  const uint32_t kk0 = kc * 128 + c * 16;  // 16 consecutive K indices of one (h, a)
  const uint32_t ha = kk0 / half, d0 = kk0 % half;
  const uint32_t h = ha / 3, a = ha % 3;
  uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
  for (int x = 0; x < 16; x++) {
    const uint32_t d = d0 + x;
    const uint32_t i = (e + 2 * half - 1 - d) % half;  // row i meets slot d (loop_len = N/2)
    const uint32_t v = __ldg(src + slab_off(g, p, h, i, a, u) + lane);
    w[x >> 2] |= ((v >> (8 * limb)) & 0xFFu) << (8 * (x & 3));
  }
  uint8_t* o = dst + ((((size_t)p * 2 + sgn) * mt_total + mt) * kc_total + kc) * TBLK + r * 128 + ((c ^ (r & 7)) << 4);
  *reinterpret_cast<uint4*>(o) = make_uint4(w[0], w[1], w[2], w[3]);
}

// Query operand: one thread per (p, sign, query, 16-byte K unit); writes the
// four limb rows 4b + j.  Queries b >= nb are zero.
__global__ void tquery_kernel(const uint32_t* __restrict__ qnat, size_t q_stride, uint32_t nb, uint32_t nb_pad,
                              uint8_t* __restrict__ qb, Group g, const uint32_t* __restrict__ gtab,
                              uint32_t kc_total) {
  const uint32_t half = g.n / 2, N = g.n;
  const uint32_t units = kc_total * 8;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)4 * nb_pad * units) return;
  const uint32_t cu = idx % units;
  const uint32_t b = (idx / units) % nb_pad;
  const uint32_t ps = (uint32_t)(idx / ((size_t)units * nb_pad));
  const uint32_t sgn = ps & 1;
  const int p = (int)(ps >> 1);
  const uint32_t kk0 = cu * 16;
  const uint32_t ha = kk0 / half, d0 = kk0 % half;
  const uint32_t h = ha / 3, a = ha % 3;
  const uint32_t slot = a == 0 ? 2 + h : a - 1;  // decoded slots: 0 gk0, 1 gk1, 2 pq, 3 pqc
  uint32_t w[4][4];
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int q = 0; q < 4; q++) w[j][q] = 0;
  if (b < nb) {
    const uint32_t* src = qnat + (size_t)b * q_stride + ((size_t)slot * 2 + p) * N;
#pragma unroll
    for (int x = 0; x < 16; x++) {
      const uint32_t k = (__ldg(gtab + sgn * half + d0 + x) - 1) >> 1;
      const uint32_t v = __ldg(src + k);
#pragma unroll
      for (int j = 0; j < 4; j++) w[j][x >> 2] |= ((v >> (8 * j)) & 0xFFu) << (8 * (x & 3));
    }
  }
  const uint32_t kc = cu / 8, c = cu % 8;
  const uint32_t rows = 4 * nb_pad;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const uint32_t r = 4 * b + j;
    uint8_t* o = qb + (((size_t)ps * kc_total + kc) * rows + r) * 128 + ((c ^ (r & 7)) << 4);
    *reinterpret_cast<uint4*>(o) = make_uint4(w[j][0], w[j][1], w[j][2], w[j][3]);
  }
}

template <int NQ, int MTPC>
int launch_t(const TScanArgs& a0, int stages, cudaStream_t st) {
  TScanArgs a = a0;
  a.stages = (uint32_t)stages;
  constexpr uint32_t STAGE = MTPC * TBLK + NQ * 128;
  const size_t smem = 1024 + (size_t)stages * STAGE + (2 * stages + 1) * 8 + 16;
  if (smem > 227 * 1024) return -1;
  set_smem(tscan_kernel<NQ, MTPC>, smem);
  // resident CTAs must not ask for more TMEM columns than the SM has
  constexpr int COLS = (MTPC * NQ) <= 32 ? 32 : (MTPC * NQ);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tscan_kernel<NQ, MTPC>, TSCAN_NT, smem);
  if (per_sm * COLS > 512) return -1;
  const size_t items = (size_t)a.nshards * 4 * (a.mt_total / MTPC) * a.groups;
  tscan_kernel<NQ, MTPC><<<(unsigned)items, TSCAN_NT, smem, st>>>(a);
  return 0;
}

template <int NQ, int MTPC>
int launch_tp(const TScanArgs& a0, int stages, cudaStream_t st) {
  TScanArgs a = a0;
  a.stages = (uint32_t)stages;
  constexpr uint32_t STAGE = MTPC * TBLK + NQ * 128;
  const size_t smem = 1024 + (size_t)stages * STAGE + (2 * stages + 5) * 8 + 16;
  if (smem > 227 * 1024) return -1;
  set_smem(tscanp_kernel<NQ, MTPC>, smem);
  constexpr int COLS = (2 * MTPC * NQ <= 512 ? 2 : 1) * MTPC * NQ;
  int per_sm = 0, dev = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tscanp_kernel<NQ, MTPC>, tscanp_nt<NQ>(), smem);
  // resident CTAs must not ask for more TMEM columns than the SM has (a CTA
  // whose allocation waits would hold its SM until a neighbour finishes)
  if (per_sm < 1 || per_sm * COLS > 512) return -1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t items = (size_t)a.nshards * 4 * (a.mt_total / MTPC) * a.groups;
  size_t grid = std::min(items, (size_t)sms * per_sm);
  // a multiple of the query-group count, so that the CTAs sharing a slab
  // tile are the same in every round (as for the CTA pairs below)
  if (grid >= a.groups) grid -= grid % a.groups;
  tscanp_kernel<NQ, MTPC><<<(unsigned)grid, tscanp_nt<NQ>(), smem, st>>>(a);
  return 0;
}

// cuTensorMapEncodeTiled, from the driver through the runtime (no link
// against the driver library); null when unavailable.
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// `rows` rows of 128 bytes at base, copied box_rows rows at a time, as they
// lie (the data is stored pre-swizzled, so no swizzle mode).
bool encode_rows(CUtensorMap* m, const void* base, uint64_t rows, uint32_t box_rows) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc || rows == 0 || rows > (1ull << 31) || box_rows == 0 || box_rows > 256 ||
      (reinterpret_cast<uintptr_t>(base) & 15))
    return false;
  const cuuint64_t dims[2] = {128, rows};
  const cuuint64_t strides[1] = {128};
  const cuuint32_t box[2] = {128, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NQ, int MTPC, bool TMA>
int launch_t2(const TScanArgs& a0, int stages, cudaStream_t st) {
  TScanArgs a = a0;
  a.stages = (uint32_t)stages;
  constexpr uint32_t STAGE = MTPC * TBLK + NQ / 2 * 128;
  const size_t smem = 1024 + (size_t)stages * STAGE + (3 * stages + 5) * 8 + 16;
  if (smem > 227 * 1024 || a.mt_total % (2 * MTPC)) return -1;
  CUtensorMap qmap;
  memset(&qmap, 0, sizeof(qmap));
  if (TMA && (!a.tmaps || !encode_rows(&qmap, a.qb, (uint64_t)4 * a.kc_total * a.nq_rows, NQ / 2))) return -1;
  set_smem(tscan2_kernel<NQ, MTPC, TMA>, smem);
  const size_t items = (size_t)a.nshards * 4 * (a.mt_total / (2 * MTPC)) * a.groups;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(tscanp_nt<NQ>());
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(2);
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, tscan2_kernel<NQ, MTPC, TMA>, &cfg) != cudaSuccess || clusters < 1) {
    cudaGetLastError();
    return -1;
  }
  // one CTA per SM: TMEM columns of a resident CTA never exceed the SM's 512
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  clusters = std::min(clusters, sms / 2);
  // the query groups of one slab tile are consecutive items: with a cluster
  // count that is a multiple of the group count, the same clusters share a
  // slab tile in every round and stay in step, so the tile comes from HBM
  // once and from L2 for the other groups (74 clusters at 4 groups drifted
  // apart and read the slabs three times over)
  if (clusters >= (int)a.groups) clusters -= clusters % (int)a.groups;
  cfg.gridDim = dim3((unsigned)(2 * std::min<size_t>(items, (size_t)clusters)));
  return cudaLaunchKernelEx(&cfg, tscan2_kernel<NQ, MTPC, TMA>, a, qmap) == cudaSuccess ? 0 : -1;
}

}  // namespace

int tensor_layout_supported(const Group& g) { return g.log2n >= 8 && g.L == g.n / 2 && g.H >= 1; }

void tensor_dims(const Group& g, uint32_t* mt_total, uint32_t* kc_total) {
  *mt_total = (g.n / 2) * SIMD * 4 / 128;
  *kc_total = 3 * g.H * (g.n / 2) / 128;
}

void launch_retile(const uint32_t* lane_slab, uint8_t* tensor_slab, const Group& g, cudaStream_t st) {
  uint32_t mt, kc;
  tensor_dims(g, &mt, &kc);
  const size_t total = (size_t)4 * mt * kc * 1024;
  retile_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(lane_slab, tensor_slab, g, mt, kc);
}

// The tile shapes: queries per CTA (NQ / 4) and m-tiles per CTA.
const TScanShape* tscan_shapes(int* count) {
  // stages chosen so that most shapes fit two CTAs per SM (one CTA's TMEM
  // epilogue then overlaps the other's main loop); a few deeper one-per-SM
  // variants for the tuner to compare
  // (last field 1: the persistent warp-specialised kernel, stages sized so
  // that resident CTAs never exceed the SM's 512 TMEM columns)
  static const TScanShape shapes[] = {
      {16, 1, 5, 0},  {16, 1, 10, 0}, {32, 1, 5, 0},  {64, 1, 4, 0},  {64, 2, 3, 0},  {64, 2, 2, 0},
      {128, 1, 3, 0}, {128, 2, 2, 0}, {128, 2, 3, 0}, {256, 1, 2, 0}, {256, 1, 3, 0}, {256, 1, 4, 0},
      {256, 2, 2, 0}, {256, 2, 3, 0}, {512, 1, 2, 0}, {16, 1, 6, 1},  {64, 1, 5, 1},  {64, 2, 4, 1},
      {128, 1, 4, 1}, {128, 2, 3, 1}, {256, 1, 3, 1}, {256, 1, 4, 1}, {256, 2, 3, 1},
      // CTA pairs (tcgen05.mma.cta_group::2): rows are the pair's query
      // operand rows (each CTA stages half of them)
      {64, 1, 8, 2},  {128, 1, 6, 2}, {128, 2, 4, 2}, {256, 1, 6, 2}, {256, 2, 4, 2},
      // CTA pairs loading with tensor maps: both CTAs' copies complete on the
      // leader's barrier (no relay)
      {64, 1, 8, 3},  {128, 1, 6, 3}, {128, 2, 4, 3}, {256, 1, 6, 3}, {256, 2, 4, 3},
      // a deeper persistent ring for 16-query groups, whose scan is HBM-bound
      // (30.1 ms per group at 2^22 against 29.5-30.9 for the one-tile-per-CTA
      // shapes; (64, 1, 8-9) and (128, 1, 6-7) measured 35-37 ms)
      {64, 2, 5, 1},
  };
  *count = (int)(sizeof(shapes) / sizeof(shapes[0]));
  return shapes;
}

size_t tscan_query_bytes(const Group& g, int nb_pad) {
  uint32_t mt, kc;
  tensor_dims(g, &mt, &kc);
  return (size_t)4 * kc * 4 * nb_pad * 128;
}

int tscan_slab_maps(uint8_t* const* host_slabs, int nshards, const Group& g, void* dev_maps) {
  uint32_t mt, kc;
  tensor_dims(g, &mt, &kc);
  std::vector<CUtensorMap> maps((size_t)nshards);
  for (int s = 0; s < nshards; s++)
    if (!encode_rows(&maps[s], host_slabs[s], (uint64_t)4 * mt * kc * 128, 128)) return -1;
  return cudaMemcpy(dev_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice) == cudaSuccess
             ? 0
             : -1;
}

size_t tscan_slab_map_bytes(int nshards) { return (size_t)nshards * sizeof(CUtensorMap); }

int launch_tscan(uint8_t* const* slabs_dev, int nshards, const uint32_t* qnat, size_t q_stride, int nb, int nb_pad,
                 uint8_t* qb, uint32_t* out, uint32_t* err, const Group& g, const SlotMaps& maps,
                 const TScanShape& shape, cudaStream_t st, const TScanLimits& lim, const void* slab_maps) {
  uint32_t mt, kc;
  tensor_dims(g, &mt, &kc);
  const int qpc = shape.nq / 4;
  if (nb_pad % qpc || nb_pad < qpc || mt % shape.mtpc) return -1;
  {
    const size_t threads = (size_t)4 * nb_pad * kc * 8;
    tquery_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(qnat, q_stride, nb, nb_pad, qb, g, maps.g, kc);
  }
  TScanArgs a;
  a.slabs = slabs_dev;
  a.nshards = nshards;
  a.qb = qb;
  a.nq_rows = 4 * nb_pad;
  a.nvalid = nb;
  a.out = out;
  a.err = err;
  a.half = g.n / 2;
  a.mt_total = mt;
  a.kc_total = kc;
  a.groups = nb_pad / qpc;
  a.stages = 0;
  a.wait_ns = lim.wait_ns ? lim.wait_ns : WAIT_NS;
  a.withhold = lim.withhold < 0 ? ~0u : (uint32_t)lim.withhold;
  a.tmaps = static_cast<const CUtensorMap*>(slab_maps);
  const int stg = shape.stages;
  if (shape.persistent == 2) {
    switch (shape.nq * 10 + shape.mtpc) {
      case 641: return launch_t2<64, 1, false>(a, stg, st);
      case 1281: return launch_t2<128, 1, false>(a, stg, st);
      case 1282: return launch_t2<128, 2, false>(a, stg, st);
      case 2561: return launch_t2<256, 1, false>(a, stg, st);
      case 2562: return launch_t2<256, 2, false>(a, stg, st);
      default: return -1;
    }
  }
  if (shape.persistent == 3) {
    switch (shape.nq * 10 + shape.mtpc) {
      case 641: return launch_t2<64, 1, true>(a, stg, st);
      case 1281: return launch_t2<128, 1, true>(a, stg, st);
      case 1282: return launch_t2<128, 2, true>(a, stg, st);
      case 2561: return launch_t2<256, 1, true>(a, stg, st);
      case 2562: return launch_t2<256, 2, true>(a, stg, st);
      default: return -1;
    }
  }
  if (shape.persistent) {
    switch (shape.nq * 10 + shape.mtpc) {
      case 161: return launch_tp<16, 1>(a, stg, st);
      case 641: return launch_tp<64, 1>(a, stg, st);
      case 642: return launch_tp<64, 2>(a, stg, st);
      case 1281: return launch_tp<128, 1>(a, stg, st);
      case 1282: return launch_tp<128, 2>(a, stg, st);
      case 2561: return launch_tp<256, 1>(a, stg, st);
      case 2562: return launch_tp<256, 2>(a, stg, st);
      default: return -1;
    }
  }
  switch (shape.nq * 10 + shape.mtpc) {
    case 161: return launch_t<16, 1>(a, stg, st);
    case 321: return launch_t<32, 1>(a, stg, st);
    case 641: return launch_t<64, 1>(a, stg, st);
    case 642: return launch_t<64, 2>(a, stg, st);
    case 1281: return launch_t<128, 1>(a, stg, st);
    case 1282: return launch_t<128, 2>(a, stg, st);
    case 2561: return launch_t<256, 1>(a, stg, st);
    case 2562: return launch_t<256, 2>(a, stg, st);
    case 5121: return launch_t<512, 1>(a, stg, st);
    default: return -1;
  }
}

}  // namespace dnspir
