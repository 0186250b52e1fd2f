// Beta contraction of the forward transform on the 5th-generation tensor cores
// (tcgen05), FP32 plans.
//
// After the alpha/gamma stage (k_anal_ag) the forward transform of
// fftSO3R.m:89-106 (MEX fftSO3R/kernel.cu:11-195) is, for each (m, n) pair, one
// real GEMM over the quadrature nodes beta_b:
//
//   F^l_mn[w] = sum_b  w_b d^l_mn(beta_b) Q_b[m][n][w],   l = max(|m|,|n|)..lmax,
//
// with Q complex and w_b d real.  Here a CTA owns one pair and a run of omega
// tiles; a tile is M = 128 real rows (64 complex omega points, real and
// imaginary parts as separate rows), K = the 2B nodes (padded to a multiple of
// 8), N = the pair's l values (padded to 16 or 32):
//
//   D[r][j] = sum_b A[r][b] W[j][b],   A[r][b] = (float view of Q_b)[r],  W = w_b d.
//
// Precision: FP32 through three TF32 products.  Each operand x is split into
// hi = x rounded to TF32 (low 13 mantissa bits cleared) and lo = x - hi (exact
// in FP32), and D accumulates A_hi W_hi + A_hi W_lo + A_lo W_hi in FP32 in
// tensor memory; the dropped A_lo W_lo term and the tensor core's truncation of
// lo are below 2^-21 relative per product.  W's split is taken from the FP64
// table (lo = x64 - hi), so W carries ~34 significant bits.
//
// Precision, second form: BF16x3 (kind::f16 with BF16 operands, FP32
// accumulation).  Each operand is split three ways, x = b0 + b1 + b2 with
// b0 = bf16(x), b1 = bf16(x - b0), b2 = bf16(x - b0 - b1) (each remainder is
// exact in FP32), and D accumulates the six products of order <= 2,
// A0W0 + A0W1 + A1W0 + A0W2 + A2W0 + A1W1; the dropped terms are of order
// 2^-24 relative.  Products of two BF16 values are exact in FP32.  W's split
// is again taken from the FP64 table.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout: core
// matrices of 8 rows x 16 bytes (4 TF32 or 8 BF16 values), the K chunks of one
// 8-row group 128 bytes apart (leading byte offset) and the 8-row groups
// KC*128 bytes apart (stride byte offset), KC = the 16-byte chunks of a row.  One thread issues the MMAs and commits
// them to an mbarrier; every warp then reads its 32 TMEM lanes
// (tcgen05.ld 32x32b) and writes the rows straight into the [row][omega]
// coefficient layout.
#include <stdint.h>
#include <algorithm>
#include <cuda.h>
#include <cuda_bf16.h>
#include "common.cuh"
#include "plan.hpp"

namespace hp {
namespace {

__device__ __forceinline__ float tf32_rn(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
// three-way BF16 split of x (bits of b0 | b1 << 16 and of b2), remainders exact in FP32
__device__ __forceinline__ void bf16x3_split(float x, uint32_t& b0, uint32_t& b1, uint32_t& b2) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h0);
  const __nv_bfloat16 h1 = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(h1);
  const __nv_bfloat16 h2 = __float2bfloat16_rn(r2);
  b0 = (uint32_t)__bfloat16_as_ushort(h0);
  b1 = (uint32_t)__bfloat16_as_ushort(h1);
  b2 = (uint32_t)__bfloat16_as_ushort(h2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, no swizzle, sm_100 version bits
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor of kind::tf32: F32 accumulator, TF32 A and B, both
// K-major, no negation, N >> 3 at bit 17, M >> 4 at bit 24
template <int M, int N> __host__ __device__ constexpr uint32_t idesc_tf32() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// kind::f16 with BF16 A and B (format 1 in both type fields), F32 accumulator
template <int M, int N> __host__ __device__ constexpr uint32_t idesc_bf16() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(done)
      : "r"(mbar), "r"(parity)
      : "memory");
  return done != 0;
}
// bounded wait: gives up after ~2^31 SM cycles (about a second)
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(mbar, parity))
    if (clock64() - t0 > (1LL << 31)) return false;
  return true;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

constexpr int TC_M = 128;        // real rows per tile (64 complex omega points)
constexpr int TC_TMEM_COLS = 32; // accumulator columns allocated (N <= 32)

// Grid: (omega-tile runs, pairs).  Q: the stage-1 tiles as floats,
// [(mi*2B + q)*2B + b][2*nwc]; tab: per row, the split parts of w_b d (zero for
// b >= 2B): TF32 [row][2][KP] floats, BF16 [row][3][KP] bf16 values;
// out: [row][nx] complex as floats.  err: counts the blocks whose wait on the
// tensor cores gave up.
// STAGED: the raw tile [b][128 rows] of Q arrives in shared memory by 16-byte
// cp.async copies issued while the previous tile's MMAs and epilogue run (the
// whole tile in flight at once, no registers held); the split pass then reads
// it from shared memory.  Requires nwc even (16-byte aligned rows), which every
// omega chunk of a plan satisfies (nx = (2Bx)^ndim is even and full chunks are
// multiples of 32 points); for an odd chunk length the kernel instead loads
// each row's values into registers, 32 at a time (the GPU tests run only the
// staged form, since no plan produces an odd chunk).
// BF16: the BF16x3 form (KP a multiple of 16); else the 3xTF32 form (KP a
// multiple of 8).
template <int KP, int NP, bool STAGED, bool BF16>
__global__ void __launch_bounds__(128) k_tc_beta(const float* __restrict__ Q, const void* __restrict__ tabv,
                                                 const int2* __restrict__ pairs, int NB2, long long nwc,
                                                 int tiles_per_cta, float* __restrict__ out, long long nx,
                                                 long long w0, int* __restrict__ err) {
  constexpr int ES = BF16 ? 2 : 4;                 // operand element bytes
  constexpr int NPL = BF16 ? 3 : 2;                // split planes per operand
  static_assert(KP % (BF16 ? 16 : 8) == 0 && KP <= 64, "K: multiple of one MMA's K, at most 64");
  static_assert(NP == 16 || NP == 32, "N: 16 or 32");
  constexpr int KC = KP * ES / 16;                 // 16-byte K chunks per row
  constexpr int EC = 16 / ES;                      // elements per chunk
  constexpr uint32_t LBO = 128, SBO = KC * 128;    // bytes
  constexpr uint32_t A_BYTES = TC_M * KP * ES, B_BYTES = NP * KP * ES;
  constexpr uint32_t S_BYTES = STAGED ? TC_M * KP * 4 : 0;
  constexpr uint32_t IDESC = BF16 ? idesc_bf16<TC_M, NP>() : idesc_tf32<TC_M, NP>();
  extern __shared__ __align__(1024) unsigned char tc_sm[];
  unsigned char* sA = tc_sm;                                   // NPL planes of A_BYTES
  unsigned char* sB = tc_sm + NPL * A_BYTES;                   // NPL planes of B_BYTES
  float* sS = reinterpret_cast<float*>(tc_sm + NPL * (A_BYTES + B_BYTES));   // raw tile [KP][128]
  uint64_t* mbar_p = reinterpret_cast<uint64_t*>(tc_sm + NPL * (A_BYTES + B_BYTES) + S_BYTES);
  uint32_t* tmem_p = reinterpret_cast<uint32_t*>(mbar_p + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int2 pe = pairs[blockIdx.y];
  const int s = pe.x, len = pe.y & 0xff, mi = (pe.y >> 8) & 0xff, q = (pe.y >> 16) & 0xff;
  const uint32_t mbar = smem_u32(mbar_p);
  const float* Qp = Q + (size_t)(mi * NB2 + q) * NB2 * 2 * nwc;
  const long long ntiles = (nwc + TC_M / 2 - 1) / (TC_M / 2);
  const long long t_begin = (long long)blockIdx.x * tiles_per_cta;
  const long long t_end = t_begin + tiles_per_cta < ntiles ? t_begin + tiles_per_cta : ntiles;
  // raw tile t: row b < NB2 of Q in 32 pieces of 16 bytes; pieces past the
  // chunk's 2*nwc real rows are zero-filled by the copy itself
  auto stage = [&](long long t) {
    const long long r0 = t * TC_M;
    for (int e = tid; e < NB2 * 32; e += 128) {
      const int b = e >> 5, pc = e & 31;
      const long long r = r0 + pc * 4;
      const bool in = r < 2 * nwc;
      cp_async16_n(sS + b * TC_M + pc * 4, Qp + (size_t)b * 2 * nwc + (in ? r : 0), in ? 16 : 0);
    }
  };

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_p)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) mbar_init(mbar, 1);
  if (STAGED) {
    for (int e = tid; e < (KP - NB2) * TC_M; e += 128) sS[NB2 * TC_M + e] = 0.f;   // K padding rows
    if (t_begin < t_end) stage(t_begin);
  }
  // W tile planes: item (j, K chunk), rows j >= len zero
  for (int it = tid; it < NP * KC; it += 128) {
    const int j = it / KC, kc = it % KC;
    const uint32_t off = (j >> 3) * SBO + kc * 128 + (j & 7) * 16;
#pragma unroll
    for (int pl = 0; pl < NPL; ++pl) {
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (j < len)
        v = *reinterpret_cast<const uint4*>(static_cast<const unsigned char*>(tabv) +
                                            ((size_t)(s + j) * NPL + pl) * KP * ES + kc * 16);
      *reinterpret_cast<uint4*>(sB + pl * B_BYTES + off) = v;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_p;

  // split of this thread's row (r = tid) into the A planes: K chunk kc from x[EC]
  const uint32_t aoff = (tid >> 3) * SBO + (tid & 7) * 16;   // this thread's row r = tid
  auto put_chunk = [&](int kc, const float (&x)[EC]) {
    if constexpr (BF16) {
      uint32_t w[3][4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        uint32_t a0, a1, a2, c0, c1, c2;
        bf16x3_split(x[2 * u], a0, a1, a2);
        bf16x3_split(x[2 * u + 1], c0, c1, c2);
        w[0][u] = a0 | (c0 << 16);
        w[1][u] = a1 | (c1 << 16);
        w[2][u] = a2 | (c2 << 16);
      }
#pragma unroll
      for (int pl = 0; pl < 3; ++pl)
        *reinterpret_cast<uint4*>(sA + pl * A_BYTES + aoff + kc * 128) = make_uint4(w[pl][0], w[pl][1], w[pl][2], w[pl][3]);
    } else {
      float4 h, l;
      h.x = tf32_rn(x[0]); l.x = x[0] - h.x;
      h.y = tf32_rn(x[1]); l.y = x[1] - h.y;
      h.z = tf32_rn(x[2]); l.z = x[2] - h.z;
      h.w = tf32_rn(x[3]); l.w = x[3] - h.w;
      *reinterpret_cast<float4*>(sA + aoff + kc * 128) = h;
      *reinterpret_cast<float4*>(sA + A_BYTES + aoff + kc * 128) = l;
    }
  };

  uint32_t phase = 0;
  bool ok = true;
  for (long long t = t_begin; t < t_end && ok; ++t) {
    const long long r0 = t * TC_M;                          // first real row of the tile
    const long long rows = 2 * nwc - r0 < TC_M ? 2 * nwc - r0 : TC_M;
    const bool rv = tid < rows;
    if (STAGED) {
      cp_async_wait_all();
      __syncthreads();                                      // tile t is in sS
#pragma unroll
      for (int kc = 0; kc < KC; ++kc) {
        float x[EC];
#pragma unroll
        for (int u = 0; u < EC; ++u) x[u] = sS[(kc * EC + u) * TC_M + tid];
        put_chunk(kc, x);
      }
    } else {
      // A tile: row r = tid, all K chunks; 32 loads in flight at a time
      constexpr int CB = 32 / EC;                           // chunks per batch
#pragma unroll
      for (int k0 = 0; k0 < KC; k0 += CB) {
        float v[CB][EC];
#pragma unroll
        for (int c = 0; c < CB; ++c)
#pragma unroll
          for (int u = 0; u < EC; ++u) {
            const int b = (k0 + c) * EC + u;
            v[c][u] = (k0 + c < KC && rv && b < NB2) ? __ldg(Qp + (size_t)b * 2 * nwc + r0 + tid) : 0.f;
          }
#pragma unroll
        for (int c = 0; c < CB; ++c)
          if (k0 + c < KC) put_chunk(k0 + c, v[c]);
      }
    }
    fence_async_smem();   // generic-proxy smem writes -> visible to the tensor core
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
      for (int kk = 0; kk < KC / 2; ++kk) {                 // one MMA consumes two K chunks
        const uint32_t o = kk * 2 * 128;
        auto ad = [&](int pl) { return umma_desc(a0 + pl * A_BYTES + o, LBO, SBO); };
        auto bd = [&](int pl) { return umma_desc(b0 + pl * B_BYTES + o, LBO, SBO); };
        if constexpr (BF16) {
          umma_bf16(tmem, ad(0), bd(0), IDESC, kk > 0 ? 1u : 0u);
          umma_bf16(tmem, ad(0), bd(1), IDESC, 1u);
          umma_bf16(tmem, ad(1), bd(0), IDESC, 1u);
          umma_bf16(tmem, ad(0), bd(2), IDESC, 1u);
          umma_bf16(tmem, ad(2), bd(0), IDESC, 1u);
          umma_bf16(tmem, ad(1), bd(1), IDESC, 1u);
        } else {
          umma_tf32(tmem, ad(0), bd(0), IDESC, kk > 0 ? 1u : 0u);
          umma_tf32(tmem, ad(0), bd(1), IDESC, 1u);
          umma_tf32(tmem, ad(1), bd(0), IDESC, 1u);
        }
      }
      umma_commit(mbar);
    }
    // the raw tile was consumed before the barrier: the next one streams in
    // while the tensor core and the epilogue work on this one
    if (STAGED && t + 1 < t_end) stage(t + 1);
    // every thread takes the same branch (a wait that gave up anywhere ends the block's loop)
    ok = __syncthreads_and(mbar_wait(mbar, phase)) != 0;
    phase ^= 1u;
    if (!ok) {
      if (tid == 0) atomicAdd(err, 1);   // one count per block whose wait gave up
      break;
    }
    tc_fence_after();
    // epilogue: warp w reads TMEM lanes 32w..32w+31 = rows r0 + 32w + lane
    float* orow = out + ((size_t)s * nx + w0) * 2 + r0 + tid;
#pragma unroll
    for (int c0 = 0; c0 < NP; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (rv && c0 + j < len) orow[(size_t)(c0 + j) * nx * 2] = v[j];
    }
    tc_fence_before();
    __syncthreads();      // every TMEM read done before the next tile's MMAs overwrite D
    tc_fence_after();
  }
  if (!ok) {
    // the tensor core did not signal: wait once more (bounded) before
    // releasing the accumulator it may still be writing
    mbar_wait(mbar, phase ^ 1u);
  }
  if (STAGED) cp_async_wait_all();   // no copy into this block's shared memory outlives it
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                 : "memory");
}

// ---------------------------------------------- warp-specialised form ----
// The same contraction as k_tc_beta, with its stages overlapped across tiles:
//   warp 0 (one lane)  loads raw tiles of Q by TMA (cp.async.bulk.tensor, 2-D
//                      tiled, no multicast) into a ring of S stages, completion
//                      counted in bytes on an mbarrier per stage;
//   warp 1 (one lane)  issues the MMAs of tile t into the TMEM accumulator of
//                      tile t's group (32 columns each) and commits them;
//   warps 2-5, 6-9     two groups of four warps taking alternate tiles: split
//                      the raw tile (TF32 hi/lo or BF16 x3 operands, one
//                      operand buffer per group), then read the accumulator
//                      (each warp its 32-lane TMEM quadrant) and store the
//                      rows, so one group's split and stores overlap the other
//                      group's, the tensor core and the next copies.
// Barriers: raw_full/raw_free per stage, a_full/mma_done/acc_free per group;
// the phase of use k is k & 1.  Every wait is bounded; a wait that gives up
// sets a shared abort flag (counted once in err), every role leaves its loop,
// the block waits (bounded) for its own copies and MMAs in flight, and frees
// its TMEM.
constexpr int WS_THREADS = 320;

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
// 2-D tiled TMA load of the box at (x, y) into shared memory, completion on mbar
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void* tmap, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

template <int KP, bool BF16> __host__ __device__ constexpr int ws_stages() {
  // as many raw stages (up to 4) as fit beside the two operand buffers and W
  constexpr long long ES = BF16 ? 2 : 4, NPL = BF16 ? 3 : 2;
  constexpr long long fixed = 2 * NPL * 128 * KP * ES + NPL * 32 * KP * ES + 1024;
  constexpr long long raw = 128LL * KP * 4;
  constexpr long long n = (227LL * 1024 - fixed) / raw;
  return n >= 4 ? 4 : (n < 2 ? 2 : (int)n);
}

template <int KP, int NP, bool BF16>
__global__ void __launch_bounds__(WS_THREADS, 1) k_tc_beta_ws(const __grid_constant__ CUtensorMap tmQ,
                                                              const void* __restrict__ tabv,
                                                              const int2* __restrict__ pairs, int NB2, long long nwc,
                                                              int tiles_per_cta, float* __restrict__ out, long long nx,
                                                              long long w0, int* __restrict__ err) {
  constexpr int S = ws_stages<KP, BF16>();
  constexpr int ES = BF16 ? 2 : 4, NPL = BF16 ? 3 : 2;
  static_assert(KP % (BF16 ? 16 : 8) == 0 && KP <= 64, "K: multiple of one MMA's K, at most 64");
  constexpr int KC = KP * ES / 16, EC = 16 / ES;
  constexpr uint32_t LBO = 128, SBO = KC * 128;
  constexpr uint32_t A_BYTES = TC_M * KP * ES, B_BYTES = NP * KP * ES;
  constexpr uint32_t RAW_BYTES = KP * TC_M * 4;
  constexpr uint32_t IDESC = BF16 ? idesc_bf16<TC_M, NP>() : idesc_tf32<TC_M, NP>();
  extern __shared__ __align__(1024) unsigned char tc_sm[];
  float* raw = reinterpret_cast<float*>(tc_sm);                                   // [S][KP][128]
  unsigned char* sA = tc_sm + S * RAW_BYTES;                                       // [2][NPL][A_BYTES]
  unsigned char* sB = sA + 2 * NPL * A_BYTES;                                      // [NPL][B_BYTES]
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + NPL * B_BYTES);
  // raw_full[S], raw_free[S], a_full[2], mma_done[2], acc_free[2]
  uint32_t* tmem_p = reinterpret_cast<uint32_t*>(bars + 2 * S + 6);
  volatile int* abort_p = reinterpret_cast<volatile int*>(tmem_p + 1);
  volatile int* nload_p = abort_p + 1;   // TMA loads issued
  volatile int* nmma_p = abort_p + 2;    // MMA groups committed
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int2 pe = pairs[blockIdx.y];
  const int s = pe.x, len = pe.y & 0xff, mi = (pe.y >> 8) & 0xff, q = (pe.y >> 16) & 0xff;
  const int ycoord = (mi * NB2 + q) * NB2;
  const long long ntiles = (nwc + TC_M / 2 - 1) / (TC_M / 2);
  const long long t_begin = (long long)blockIdx.x * tiles_per_cta;
  const long long t_end = t_begin + tiles_per_cta < ntiles ? t_begin + tiles_per_cta : ntiles;
  const int nt = (int)(t_end > t_begin ? t_end - t_begin : 0);
  auto bar = [&](int i) { return smem_u32(bars + i); };
  auto raw_full = [&](int i) { return bar(i); };
  auto raw_free = [&](int i) { return bar(S + i); };
  auto a_full = [&](int j) { return bar(2 * S + j); };
  auto mma_done = [&](int j) { return bar(2 * S + 2 + j); };
  auto acc_free = [&](int j) { return bar(2 * S + 4 + j); };
  auto give_up = [&]() {
    if (atomicExch((int*)abort_p, 1) == 0) atomicAdd(err, 1);
  };

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_p)), "r"(64)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(raw_full(i), 1);
      mbar_init(raw_free(i), 128);
    }
    for (int j = 0; j < 2; ++j) {
      mbar_init(a_full(j), 128);
      mbar_init(mma_done(j), 1);
      mbar_init(acc_free(j), 128);
    }
    *abort_p = 0;
    *nload_p = 0;
    *nmma_p = 0;
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmQ)) : "memory");
  }
  // K padding rows of every raw stage (the TMA box writes rows < NB2 only)
  for (int e = tid; e < S * (KP - NB2) * TC_M; e += WS_THREADS) {
    const int st = e / ((KP - NB2) * TC_M), o = e % ((KP - NB2) * TC_M);
    raw[(size_t)st * KP * TC_M + NB2 * TC_M + o] = 0.f;
  }
  // W tile planes: item (j, K chunk), rows j >= len zero
  for (int it = tid; it < NP * KC; it += WS_THREADS) {
    const int j = it / KC, kc = it % KC;
    const uint32_t off = (j >> 3) * SBO + kc * 128 + (j & 7) * 16;
#pragma unroll
    for (int pl = 0; pl < NPL; ++pl) {
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (j < len)
        v = *reinterpret_cast<const uint4*>(static_cast<const unsigned char*>(tabv) +
                                            ((size_t)(s + j) * NPL + pl) * KP * ES + kc * 16);
      *reinterpret_cast<uint4*>(sB + pl * B_BYTES + off) = v;
    }
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_p;

  if (warp == 0) {
    // ---- producer: raw tile t into stage t % S once the split has released it
    if (lane == 0) {
      for (int k = 0; k < nt && !*abort_p; ++k) {
        const int i = k % S;
        if (k >= S && !mbar_wait(raw_free(i), (uint32_t)((k / S - 1) & 1))) { give_up(); break; }
        mbar_arrive_tx(raw_full(i), (uint32_t)(NB2 * TC_M * 4));
        tma_load_2d(smem_u32(raw + (size_t)i * KP * TC_M), &tmQ, (int)((t_begin + k) * TC_M), ycoord, raw_full(i));
        *nload_p = k + 1;
      }
    }
  } else if (warp == 1) {
    // ---- MMA issuer
    if (lane == 0) {
      const uint32_t b0 = smem_u32(sB);
      for (int k = 0; k < nt && !*abort_p; ++k) {
        const int j = k & 1, u = k >> 1;
        if (!mbar_wait(a_full(j), (uint32_t)(u & 1))) { give_up(); break; }
        if (u > 0 && !mbar_wait(acc_free(j), (uint32_t)((u - 1) & 1))) { give_up(); break; }
        tc_fence_after();
        const uint32_t a0 = smem_u32(sA + (size_t)j * NPL * A_BYTES);
        const uint32_t d = tmem + (uint32_t)(j * 32);
#pragma unroll
        for (int kk = 0; kk < KC / 2; ++kk) {
          const uint32_t o = kk * 2 * 128;
          auto ad = [&](int pl) { return umma_desc(a0 + pl * A_BYTES + o, LBO, SBO); };
          auto bd = [&](int pl) { return umma_desc(b0 + pl * B_BYTES + o, LBO, SBO); };
          if constexpr (BF16) {
            umma_bf16(d, ad(0), bd(0), IDESC, kk > 0 ? 1u : 0u);
            umma_bf16(d, ad(0), bd(1), IDESC, 1u);
            umma_bf16(d, ad(1), bd(0), IDESC, 1u);
            umma_bf16(d, ad(0), bd(2), IDESC, 1u);
            umma_bf16(d, ad(2), bd(0), IDESC, 1u);
            umma_bf16(d, ad(1), bd(1), IDESC, 1u);
          } else {
            umma_tf32(d, ad(0), bd(0), IDESC, kk > 0 ? 1u : 0u);
            umma_tf32(d, ad(0), bd(1), IDESC, 1u);
            umma_tf32(d, ad(1), bd(0), IDESC, 1u);
          }
        }
        umma_commit(mma_done(j));
        *nmma_p = k + 1;
      }
    }
  } else {
    // ---- two groups of 128 threads: group g splits and stores tiles k = g, g + 2, ...
    const int g = (warp - 2) >> 2;
    const int r = (tid - 64) & 127;                           // split row
    const uint32_t aoff = (r >> 3) * SBO + (r & 7) * 16;
    const int quad = warp & 3;                                // TMEM lanes 32 quad .. of this warp
    const int er = quad * 32 + lane;                          // epilogue row
    unsigned char* A = sA + (size_t)g * NPL * A_BYTES;
    for (int k = g; k < nt; k += 2) {
      if (__any_sync(0xffffffffu, *abort_p != 0)) break;
      const int i = k % S, u = k >> 1;
      // the warp agrees on every wait's outcome (the TMEM loads below are warp-collective)
      if (!__all_sync(0xffffffffu, mbar_wait(raw_full(i), (uint32_t)((k / S) & 1)))) {
        if (lane == 0) give_up();
        break;
      }
      const float* rs = raw + (size_t)i * KP * TC_M;
#pragma unroll
      for (int kc = 0; kc < KC; ++kc) {
        float x[EC];
#pragma unroll
        for (int u2 = 0; u2 < EC; ++u2) x[u2] = rs[(kc * EC + u2) * TC_M + r];
        if constexpr (BF16) {
          uint32_t w[3][4];
#pragma unroll
          for (int u2 = 0; u2 < 4; ++u2) {
            uint32_t p0, p1, p2, c0, c1, c2;
            bf16x3_split(x[2 * u2], p0, p1, p2);
            bf16x3_split(x[2 * u2 + 1], c0, c1, c2);
            w[0][u2] = p0 | (c0 << 16);
            w[1][u2] = p1 | (c1 << 16);
            w[2][u2] = p2 | (c2 << 16);
          }
#pragma unroll
          for (int pl = 0; pl < 3; ++pl)
            *reinterpret_cast<uint4*>(A + pl * A_BYTES + aoff + kc * 128) = make_uint4(w[pl][0], w[pl][1], w[pl][2], w[pl][3]);
        } else {
          float4 h, l;
          h.x = tf32_rn(x[0]); l.x = x[0] - h.x;
          h.y = tf32_rn(x[1]); l.y = x[1] - h.y;
          h.z = tf32_rn(x[2]); l.z = x[2] - h.z;
          h.w = tf32_rn(x[3]); l.w = x[3] - h.w;
          *reinterpret_cast<float4*>(A + aoff + kc * 128) = h;
          *reinterpret_cast<float4*>(A + A_BYTES + aoff + kc * 128) = l;
        }
      }
      fence_async_smem();            // the operand writes, visible to the tensor core
      mbar_arrive(raw_free(i));      // the raw stage can be refilled
      mbar_arrive(a_full(g));
      if (!__all_sync(0xffffffffu, mbar_wait(mma_done(g), (uint32_t)(u & 1)))) {
        if (lane == 0) give_up();
        break;
      }
      tc_fence_after();
      const long long r0 = (t_begin + k) * TC_M;
      const long long rows = 2 * nwc - r0 < TC_M ? 2 * nwc - r0 : TC_M;
      float* orow = out + ((size_t)s * nx + w0) * 2 + r0 + er;
#pragma unroll
      for (int c0 = 0; c0 < NP; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(g * 32 + c0), v);
#pragma unroll
        for (int jj = 0; jj < 16; ++jj)
          if (er < rows && c0 + jj < len) orow[(size_t)(c0 + jj) * nx * 2] = v[jj];
      }
      tc_fence_before();
      mbar_arrive(acc_free(g));
    }
  }
  __syncthreads();
  if (*abort_p && tid == 0) {
    // the last TMA load of each stage and the last MMA group of each
    // accumulator that were issued end before this block's shared and tensor
    // memory are released (bounded waits; their results are discarded)
    const int nl = *nload_p, nm = *nmma_p;
    for (int k = nl - S > 0 ? nl - S : 0; k < nl; ++k) mbar_wait(raw_full(k % S), (uint32_t)((k / S) & 1));
    for (int k = nm - 2 > 0 ? nm - 2 : 0; k < nm; ++k) mbar_wait(mma_done(k & 1), (uint32_t)((k >> 1) & 1));
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
}

// [row][3][KP]: BF16 parts b0, b1, b2 of w_b d^l_mn(beta_b), split from FP64
__global__ void k_dwtc_table_bf16(RowLayout L, const double* __restrict__ wig, const double* __restrict__ qw, int KP,
                                  __nv_bfloat16* __restrict__ tab) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.nrows * KP) return;
  const long long r = t / KP;
  const int b = (int)(t % KP);
  const int NB2 = 2 * L.B;
  const double x = b < NB2 ? qw[b] * wig[(size_t)b * L.nrows + r] : 0.0;
  const __nv_bfloat16 h0 = __double2bfloat16(x);
  const double r1 = x - (double)__bfloat162float(h0);
  const __nv_bfloat16 h1 = __double2bfloat16(r1);
  const double r2 = r1 - (double)__bfloat162float(h1);
  tab[(r * 3) * KP + b] = h0;
  tab[(r * 3 + 1) * KP + b] = h1;
  tab[(r * 3 + 2) * KP + b] = __double2bfloat16(r2);
}

// [row][2][KP]: TF32 hi and lo parts of w_b d^l_mn(beta_b), from FP64
__global__ void k_dwtc_table(RowLayout L, const double* __restrict__ wig, const double* __restrict__ qw, int KP,
                             float* __restrict__ tab) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.nrows * KP) return;
  const long long r = t / KP;
  const int b = (int)(t % KP);
  const int NB2 = 2 * L.B;
  const double x = b < NB2 ? qw[b] * wig[(size_t)b * L.nrows + r] : 0.0;
  const float hi = tf32_rn((float)x);
  tab[(r * 2) * KP + b] = hi;
  tab[(r * 2 + 1) * KP + b] = (float)(x - (double)hi);
}

template <int KP, int NP, bool BF16>
int tc_launch(hp_plan* p, const float2* Qg, const void* tab, const int2* pairs, int npairs, float2* out,
              long long w0, long long nwc, int* err, cudaStream_t s) {
  const bool staged = nwc % 2 == 0;
  constexpr size_t ES = BF16 ? 2 : 4, NPL = BF16 ? 3 : 2;
  const size_t smem = NPL * ((size_t)TC_M * KP * ES + (size_t)NP * KP * ES) + (staged ? (size_t)TC_M * KP * 4 : 0) + 16;
  auto kern = staged ? k_tc_beta<KP, NP, true, BF16> : k_tc_beta<KP, NP, false, BF16>;
  HP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long ntiles = (nwc + TC_M / 2 - 1) / (TC_M / 2);
  // about tc_waves (16 unless tuned) waves of CTAs over 148 SMs, at least 2 tiles per CTA
  const long long waves = p->tune.tc_waves;
  long long per = std::max(2LL, (ntiles * npairs + 148LL * 4 * waves - 1) / (148LL * 4 * waves));
  per = std::min(per, ntiles);
  const dim3 grid((unsigned)((ntiles + per - 1) / per), (unsigned)npairs);
  kern<<<grid, 128, smem, s>>>(reinterpret_cast<const float*>(Qg), tab, pairs, 2 * p->B, nwc, (int)per,
                               reinterpret_cast<float*>(out), p->nx, w0, err);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
    else
      cudaGetLastError();
  }
  return fn;
}

// The warp-specialised kernel on one omega chunk: a 2-D tensor map over the
// chunk's stage-1 tiles as floats, rows (m, n, b) of 2*nwc values, boxes of
// NB2 rows x 128 values (the raw tile of one pair); past the chunk's end the
// copy fills zeros.
template <int KP, int NP, bool BF16>
int tc_launch_ws(hp_plan* p, const float2* Qg, const void* tab, const int2* pairs, int npairs, float2* out,
                 long long w0, long long nwc, int* err, cudaStream_t s) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) { hp_set_error("cuTensorMapEncodeTiled is not available"); return HP_ERR_UNSUPPORTED; }
  const int NB2 = 2 * p->B;
  CUtensorMap tm;
  const cuuint64_t dims[2] = {(cuuint64_t)(2 * nwc), (cuuint64_t)p->nm * NB2 * NB2};
  const cuuint64_t strides[1] = {(cuuint64_t)(2 * nwc * sizeof(float))};
  const cuuint32_t box[2] = {(cuuint32_t)TC_M, (cuuint32_t)NB2};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float2*>(Qg), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { hp_set_error("tensor map encoding failed"); return HP_ERR_CUDA; }
  constexpr size_t ES = BF16 ? 2 : 4, NPL = BF16 ? 3 : 2;
  constexpr int S = ws_stages<KP, BF16>();
  const size_t smem = S * (size_t)KP * TC_M * 4 + 2 * NPL * (size_t)TC_M * KP * ES + NPL * (size_t)NP * KP * ES +
                      (2 * S + 6) * sizeof(uint64_t) + 16;
  auto kern = k_tc_beta_ws<KP, NP, BF16>;
  HP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long ntiles = (nwc + TC_M / 2 - 1) / (TC_M / 2);
  const int per_sm = std::max(1, (int)((227 * 1024) / (smem + 1024)));
  const long long waves = p->tune.tc_waves;
  long long per = std::max(4LL, (ntiles * npairs + 148LL * per_sm * waves - 1) / (148LL * per_sm * waves));
  per = std::min(per, ntiles);
  const dim3 grid((unsigned)((ntiles + per - 1) / per), (unsigned)npairs);
  kern<<<grid, WS_THREADS, smem, s>>>(tm, tab, pairs, NB2, nwc, (int)per, reinterpret_cast<float*>(out), p->nx, w0,
                                      err);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

template <int KP, int NP, bool BF16>
int tc_dispatch(hp_plan* p, const float2* Qg, const void* tab, const int2* pairs, int npairs, float2* out,
                long long w0, long long nwc, int* err, cudaStream_t s) {
  // the pipelined form (tc_form 1) needs 16-byte rows for the tensor map (nwc
  // even, true of every chunk of a plan); the staged form is the default, as
  // it measured faster (B=30, 24x24: 0.248 vs 0.281 ms per launch; B=15, 32x32:
  // 0.048 vs 0.056 ms), and hp_plan_autotune times both
  if (p->tune.tc_form == 1 && nwc % 2 == 0 && encode_tiled())
    return tc_launch_ws<KP, NP, BF16>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
  return tc_launch<KP, NP, BF16>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
}

}  // namespace

bool tc_beta_supported(const hp_plan* p) { return p->precision == HP_MIXED && p->B >= 2 && p->B <= 32; }

int tc_beta_forward(hp_plan* p, const float2* Qg, const int2* pairs, int npairs, float2* out, long long w0,
                    long long nwc, cudaStream_t s) {
  if (!tc_beta_supported(p)) {
    hp_set_error("tensor-core beta contraction: FP32 plans with B <= 32 only");
    return HP_ERR_UNSUPPORTED;
  }
  const bool bf16 = p->beta_engine == HP_BETA_TENSOR_BF16;
  // nodes padded to the kernels' K: multiples of 16 (BF16) or of 8 with 56
  // taken up to 64 (TF32); the padding rows of the operand tables are zero
  const int k8 = (2 * p->B + 7) / 8 * 8;
  const int KP = bf16 ? (2 * p->B + 15) / 16 * 16 : (k8 == 56 ? 64 : k8);
  int st = HP_OK;
  const char* tkey = bf16 ? "tf.dwtc16" : "tf.dwtc";
  bool have = false, have_err = false;
  for (auto& kv : p->ws) {
    if (kv.first == tkey) have = true;
    if (kv.first == "tf.tcerr") have_err = true;
  }
  void* tab = p->ws_get(tkey, (bf16 ? 3 * sizeof(__nv_bfloat16) : 2 * sizeof(float)) * (size_t)p->nrows * KP, &st);
  if (st) return st;
  int* err = (int*)p->ws_get("tf.tcerr", sizeof(int), &st);
  if (st) return st;
  if (!have_err) HP_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
  if (!have) {
    const long long n = p->nrows * KP;
    if (bf16)
      k_dwtc_table_bf16<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p->layout(), p->wig64, p->qw, KP,
                                                                     (__nv_bfloat16*)tab);
    else
      k_dwtc_table<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p->layout(), p->wig64, p->qw, KP, (float*)tab);
    HP_CUDA_TRY(cudaGetLastError());
  }
  ProfScope _ps(p, bf16 ? "tf.anal.beta.tc16" : "tf.anal.beta.tc", s);
  const bool n16 = p->B <= 16;
  if (bf16) {
    switch (KP) {
      case 16: return n16 ? tc_dispatch<16, 16, true>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s)
                          : tc_dispatch<16, 32, true>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
      case 32: return tc_dispatch<32, 16, true>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
      case 48: return tc_dispatch<48, 32, true>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
      case 64: return tc_dispatch<64, 32, true>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
      default:
        hp_set_error("tensor-core beta contraction: unsupported node count");
        return HP_ERR_UNSUPPORTED;
    }
  }
  switch (KP) {
    case 8: return n16 ? tc_dispatch<8, 16, false>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s)
                       : tc_dispatch<8, 32, false>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
    case 16: return tc_dispatch<16, 16, false>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
    case 24: return tc_dispatch<24, 16, false>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
    case 32: return tc_dispatch<32, 16, false>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
    case 40: return tc_dispatch<40, 32, false>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
    case 48: return tc_dispatch<48, 32, false>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
    case 64: return tc_dispatch<64, 32, false>(p, Qg, tab, pairs, npairs, out, w0, nwc, err, s);
    default:
      hp_set_error("tensor-core beta contraction: unsupported node count");
      return HP_ERR_UNSUPPORTED;
  }
}

int tc_beta_errors(hp_plan* p, int* count) {
  *count = 0;
  for (auto& kv : p->ws)
    if (kv.first == "tf.tcerr") {
      HP_CUDA_TRY(cudaMemcpy(count, kv.second.p, sizeof(int), cudaMemcpyDeviceToHost));
      HP_CUDA_TRY(cudaMemset(kv.second.p, 0, sizeof(int)));   // counted from the last read on
    }
  return HP_OK;
}

}  // namespace hp
