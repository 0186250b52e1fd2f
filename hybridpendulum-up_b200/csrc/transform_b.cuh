// Per-bandlimit kernels of the SO(3) transforms and their launchers: the
// synthesis (beta contraction, gamma and alpha FFTs; ifftSO3R.m:16-37) and the
// two-stage analysis (alpha/gamma FFTs, beta contraction; fftSO3R.m:89-106).
// Included by transform.cu (configurations and declarations only) and by
// transform_b0.cu .. transform_b3.cu, each of which instantiates the launchers
// for the bandlimits B with B mod 4 equal to its part number, so that the
// kernels compile in parallel.  Each translation unit holds its own twiddle
// table, which the launchers fill before their first launch (tw_init).
#pragma once
#include <algorithm>
#include <vector>
#include "common.cuh"
#include "plan.hpp"

using namespace hp;

static inline int smem_limit() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v;
}

// 16-byte global store of values read one by one from shared memory
__device__ __forceinline__ void store16(float* dst, const float* s) {
  *reinterpret_cast<float4*>(dst) = make_float4(s[0], s[1], s[2], s[3]);
}
__device__ __forceinline__ void store16(double* dst, const double* s) {
  *reinterpret_cast<double2*>(dst) = make_double2(s[0], s[1]);
}

// ------------------------------------------------------------ synthesis ----
// Real staging of the synthesis: one run of NB*2B values per (omega point p,
// gamma column c), runs RS elements apart.  FP32: RS = 4 (mod 32), and
// element i of run (p, c) sits at (i & ~3) | ((i + p) & 3), a rotation by p
// inside its 16-byte chunk.  The alpha-stage writers (lanes: p fastest, then
// c) then hit 32 distinct banks per scalar store, and the store loop reads
// whole 16-byte chunks (LDS.128, rotated back in registers).  FP64: runs
// padded by one element, no rotation.
template <typename T, int NB, int NB2> __host__ __device__ constexpr int synth_rs() {
  return sizeof(T) == 4 ? (NB * NB2 + 27) / 32 * 32 + 4 : NB * NB2 + 1;
}
__device__ __forceinline__ int synth_swz(int i, int rot) { return (i & ~3) | ((i + rot) & 3); }
// Bulk (TMA engine) copy of a contiguous shared-memory run to global memory:
// both addresses 16-byte aligned, size a multiple of 16 bytes.  The issuing
// thread later waits for the source to have been read (wait_group.read) before
// the buffer is rewritten, and for completion (wait_group) before exit.
__device__ __forceinline__ void bulk_s2g(void* gdst, const void* ssrc, unsigned bytes, uint64_t pol) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(ssrc);
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;" ::"l"(gdst), "r"(s),
               "r"(bytes), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// orders this thread's shared-memory writes before later bulk-copy reads of them
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// logical chunk from a physical one whose element k sits at (k + rot) & 3
__device__ __forceinline__ float4 unrotate4(float4 v, int rot) {
  switch (rot & 3) {
    case 0: return v;
    case 1: return make_float4(v.y, v.z, v.w, v.x);
    case 2: return make_float4(v.z, v.w, v.x, v.y);
    default: return make_float4(v.w, v.x, v.y, v.z);
  }
}

// Block = (group of NB consecutive beta indices, range of omega points), the
// (2l+1)-weighted d values of its betas resident in shared memory.  Input
// element (row s, omega point w) sits, for FP64, in the omega-blocked layout
// [w / P][row][w % P] (omega_block_index: one batch is one contiguous run of
// nrows * P values, the rows of an (m, n) pair P values apart) and, for FP32,
// in [row][omega] (rows nx values apart).  The P points of a row sit on
// consecutive lanes; the per-(omega, beta) intermediates G -> H live in shared
// memory as [bb][m][q][p].
// GD: the (2l+1) d table of the block's betas is read from a global table
// [group][row][NB] (large bandlimits, where it does not fit shared memory)
// instead of being staged from the d table `wig`.
// PT: omega points per beta-stage item (1, 2 or 4, dividing P): an item
// computes the NB x PT tile of one (m, n) pair, so each coefficient load (PT
// consecutive omega points, one vector load) feeds NB x PT complex FMAs and
// each d value PT of them.
// Two staging runs of N floats (the real and the imaginary parts of x), both
// starting LEAD floats (0 or 2) before a 16-byte boundary: an 8-byte store
// for the lead, 16-byte stores, an 8-byte store for an even remainder.
template <int N, int LEAD>
__device__ __forceinline__ void stage_run(float* st, float* st2, const float2 (&x)[N]) {
  static_assert(N % 2 == 0 && (LEAD == 0 || LEAD == 2), "even runs, 8-byte aligned");
  if constexpr (LEAD == 2) {
    *reinterpret_cast<float2*>(st) = make_float2(x[0].x, x[1].x);
    *reinterpret_cast<float2*>(st2) = make_float2(x[0].y, x[1].y);
  }
  constexpr int n4 = (N - LEAD) / 4;
#pragma unroll
  for (int i = 0; i < n4; ++i) {
    const int a = LEAD + 4 * i;
    *reinterpret_cast<float4*>(st + a) = make_float4(x[a].x, x[a + 1].x, x[a + 2].x, x[a + 3].x);
    *reinterpret_cast<float4*>(st2 + a) = make_float4(x[a].y, x[a + 1].y, x[a + 2].y, x[a + 3].y);
  }
  constexpr int a = LEAD + 4 * n4;
  if constexpr (a < N) {
    *reinterpret_cast<float2*>(st + a) = make_float2(x[a].x, x[a + 1].x);
    *reinterpret_cast<float2*>(st2 + a) = make_float2(x[a].y, x[a + 1].y);
  }
}

template <int B, typename T, int NB, int P, bool CPLX, bool GD, int PT = 1>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 1 : 2)
    k_synth(RowLayout L, const c2<T>* __restrict__ Fp, const T* __restrict__ wig, const int2* __restrict__ pairs,
            void* __restrict__ fout, int nbatch) {
  static_assert(P % PT == 0, "PT divides P");
  constexpr bool BLOCKED = sizeof(T) == 8;   // input layout (see above)
  using C = c2<T>;
  constexpr int NB2 = 2 * B, lmax = B - 1, D = 2 * lmax + 1;
  constexpr int NM = CPLX ? D : B;
  constexpr int MLO = CPLX ? -lmax : 0;
  constexpr int NPAIR = NM * D;
  // G/H stride per (bb, m): 2B q-bins x P omega points, padded by P so that
  // the P-wide groups of the gamma stage fall on distinct banks
  constexpr int GS = NB2 * P + P;
  constexpr int RS = synth_rs<T, NB, NB2>();
  // FP32 real plans with an even NB: every run (NB*2B or the last group's
  // nbv*2B floats) starts 16-byte aligned in f and in the staging buffer, so
  // the runs leave by bulk copies that drain while the next batch computes.
  // Otherwise FP32 uses the rotated staging and vector stores.
  constexpr bool BULK = sizeof(T) == 4 && !CPLX && NB % 2 == 0;
  constexpr bool SWZ = sizeof(T) == 4 && !BULK;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nrows = (int)L.nrows;
  T* sds = reinterpret_cast<T*>(smraw);
  int2* spairs = reinterpret_cast<int2*>(smraw + (GD ? 0 : ((size_t)NB * nrows * sizeof(T) + 15) / 16 * 16));
  C* sG = reinterpret_cast<C*>(reinterpret_cast<unsigned char*>(spairs) + ((size_t)NPAIR * sizeof(int2) + 15) / 16 * 16);
  // beta groups of one omega chunk are consecutive blocks, so they read the
  // same coefficient rows close together in time (L2 reuse)
  constexpr int NGROUPS = (NB2 + NB - 1) / NB;
  const int grp = blockIdx.x % NGROUPS;
  const int chunk = blockIdx.x / NGROUPS;
  const int b0 = grp * NB;
  const int nbv = min(NB, NB2 - b0);
  const int tid = threadIdx.x, nth = blockDim.x;
  const T* sd = GD ? wig + (size_t)grp * nrows * NB : sds;
  for (int e = tid; !GD && e < NB * nrows; e += nth) {   // interleaved [row][bb]
    const int r = e / NB, bb = e % NB;
    const T l2 = (T)(2 * L.rows[r].x + 1);
    sds[e] = (bb < nbv) ? l2 * wig[(size_t)(b0 + bb) * nrows + r] : (T)0;
  }
  for (int e = tid; e < NPAIR; e += nth) spairs[e] = pairs[e];
  const long long nx = L.nx;
  // vector and bulk stores need a 16-byte aligned density buffer
  const bool fout_al16 = (reinterpret_cast<unsigned long long>(fout) & 15ull) == 0;
  for (int bt = 0; bt < nbatch; ++bt) {
    const long long w0 = ((long long)chunk * nbatch + bt) * P;
    if (w0 >= nx) break;
    if (BULK && fout_al16) bulk_wait_read_all();   // the previous batch's runs have left the staging (aliases sG)
    __syncthreads();
    // beta stage: item (pair, p), p fastest.  Pairs come from the block's copy
    // of the pair table (longest l-runs first, so the lanes of a warp run
    // loops of similar length); the l-run is loaded in batches of 8 ahead of
    // its FMAs, each coefficient feeding NB FMAs per component.
    constexpr int NPG = P / PT;                 // omega groups of PT points per batch
    for (int it = tid; it < NPAIR * NPG; it += nth) {
      const int p0 = (it % NPG) * PT;
      const int2 pe = spairs[it / NPG];
      const int s = pe.x, len = pe.y & 0xff, mi = (pe.y >> 8) & 0xff, q = (pe.y >> 16) & 0xff;
      C acc[NB][PT];
#pragma unroll
      for (int bb = 0; bb < NB; ++bb)
#pragma unroll
        for (int pt = 0; pt < PT; ++pt) acc[bb][pt] = czero<C>();
      if (w0 + p0 < nx) {
        // row s at the item's first omega point; rows rs values apart
        const size_t rs = BLOCKED ? (size_t)P : (size_t)nx;
        const C* src = BLOCKED ? Fp + ((size_t)(w0 / P) * nrows + s) * P + p0 : Fp + (size_t)s * nx + w0 + p0;
        const T* dsrc = sd + (size_t)s * NB;
        // a vector load per row where the PT points are all inside the grid
        const bool full = w0 + p0 + PT <= nx;
        constexpr int JB = PT >= 4 ? 4 : 8;
#pragma unroll
        for (int j0 = 0; j0 < B; j0 += JB) {
          if (j0 < len) {
            C v[JB][PT];
#pragma unroll
            for (int u = 0; u < JB; ++u) {
              const bool ok = j0 + u < len;
              if constexpr (PT > 1 && sizeof(T) == 4) {
                if (ok && full) {
#pragma unroll
                  for (int h = 0; h < PT / 2; ++h) {
                    const float4 w4 = *reinterpret_cast<const float4*>(src + (size_t)(j0 + u) * rs + 2 * h);
                    v[u][2 * h] = mk(w4.x, w4.y);
                    v[u][2 * h + 1] = mk(w4.z, w4.w);
                  }
                } else {
#pragma unroll
                  for (int pt = 0; pt < PT; ++pt)
                    v[u][pt] = (ok && w0 + p0 + pt < nx) ? src[(size_t)(j0 + u) * rs + pt] : czero<C>();
                }
              } else {
#pragma unroll
                for (int pt = 0; pt < PT; ++pt)
                  v[u][pt] = (ok && (PT == 1 || w0 + p0 + pt < nx)) ? src[(size_t)(j0 + u) * rs + pt] : czero<C>();
              }
            }
#pragma unroll
            for (int u = 0; u < JB; ++u) {
              if (j0 + u < len) {
#pragma unroll
                for (int bb = 0; bb < NB; ++bb) {
                  const T dv = dsrc[(j0 + u) * NB + bb];
#pragma unroll
                  for (int pt = 0; pt < PT; ++pt) {
                    acc[bb][pt].x = fma(dv, v[u][pt].x, acc[bb][pt].x);
                    acc[bb][pt].y = fma(dv, v[u][pt].y, acc[bb][pt].y);
                  }
                }
              }
            }
          }
        }
      }
#pragma unroll
      for (int bb = 0; bb < NB; ++bb) {
#pragma unroll
        for (int pt = 0; pt < PT; ++pt) {
          C* g = sG + (bb * NM + mi) * GS + p0 + pt;
          g[q * P] = acc[bb][pt];
          if (pe.y >> 24) g[B * P] = czero<C>();
        }
      }
    }
    __syncthreads();
    // gamma stage: item (bb, mi, p): FFT over n -> c, in place
    for (int it = tid; it < NB * NM * P; it += nth) {
      C* g = sG + (it / P) * GS + it % P;
      C x[NB2];
#pragma unroll
      for (int j = 0; j < NB2; ++j) x[j] = g[j * P];
      fft<NB2, false>(x);
#pragma unroll
      for (int j = 0; j < NB2; ++j) g[j * P] = x[j];
    }
    __syncthreads();
    // alpha stage, one round (host guarantees the item count fits the block).
    // Real plans: f_c = Re FFT(w_m H[m][c]) = FFT(h_c) with h_c the Hermitian
    // extension of H[.][c] (h[0] = Re H[0]); two columns c, c+B share one complex
    // FFT, FFT(h_c + i h_c') = f_c + i f_c'.  Complex plans: one FFT per column.
    constexpr int NCOL = CPLX ? NB2 : B;   // FFTs per (bb, p)
    const bool act = tid < NB * NCOL * P;
    const int p = tid % P, c = (tid / P) % NCOL, bb = tid / (P * NCOL);
    C x[NB2];
    if (act) {
      const C* h = sG + bb * NM * GS + c * P + p;
#pragma unroll
      for (int q = 0; q < NB2; ++q) x[q] = czero<C>();
      if (CPLX) {
#pragma unroll
        for (int mi = 0; mi < NM; ++mi) {
          const int m = mi + MLO;
          x[m >= 0 ? m : m + NB2] = h[mi * GS];
        }
      } else {
        const C* h2 = h + B * P;   // column c + B
        {
          const C u = h[0], v = h2[0];
          x[0].x = u.x;
          x[0].y = v.x;
        }
#pragma unroll
        for (int m = 1; m < B; ++m) {
          const C u = h[m * GS], v = h2[m * GS];
          // z[m] = u + i v ; z[N-m] = conj(u) + i conj(v)
          x[m].x = u.x - v.y;
          x[m].y = u.y + v.x;
          x[NB2 - m].x = u.x + v.y;
          x[NB2 - m].y = -u.y + v.x;
        }
      }
      fft<NB2, false>(x);
    }
    __syncthreads();
    if (act) {  // staging [p][c][bb][a], aliasing sG
      if (CPLX) {
        C* st = sG + ((p * NB2 + c) * NB + bb) * NB2;
#pragma unroll
        for (int a = 0; a < NB2; ++a) st[a] = x[a];
      } else if constexpr (BULK) {
        // runs start on 4-float boundaries (RS is a multiple of 4): 16-byte
        // stores, after one 8-byte store where bb * 2B is 2 mod 4 (2B even)
        float* st = reinterpret_cast<float*>(sG) + (p * NB2 + c) * RS + bb * NB2;
        float* st2 = reinterpret_cast<float*>(sG) + (p * NB2 + c + B) * RS + bb * NB2;
        if (((bb * NB2) & 3) == 0) stage_run<NB2, 0>(st, st2, x);
        else stage_run<NB2, 2>(st, st2, x);
      } else {
        T* st = reinterpret_cast<T*>(sG) + (p * NB2 + c) * RS;
        T* st2 = reinterpret_cast<T*>(sG) + (p * NB2 + c + B) * RS;
        const int rot = SWZ ? (p & 3) : 0;
#pragma unroll
        for (int a = 0; a < NB2; ++a) {
          const int i = bb * NB2 + a;
          const int j = SWZ ? synth_swz(i, rot) : i;
          st[j] = x[a].x;
          st2[j] = x[a].y;
        }
      }
    }
    if (BULK && fout_al16) fence_proxy_async_smem();
    __syncthreads();
    // store: f[a + 2B (b + 2B (c + 2B w))]; the nbv*2B values of one (w, c) are
    // contiguous in f and in the staging buffer; a warp copies one run with
    // consecutive lanes on consecutive 16-byte pieces.
    const int pc = (int)min((long long)P, nx - w0);
    constexpr int RUN = NB * NB2;
    if (BULK && fout_al16) {
      const uint64_t pol = l2_policy_evict_first();   // the density is written once, read by later kernels
      for (int run = tid; run < pc * NB2; run += nth) {
        const int pp = run / NB2, cc = run % NB2;
        const size_t gi = ((size_t)(w0 + pp) * NB2 + cc) * NB2 * NB2 + (size_t)b0 * NB2;
        bulk_s2g(reinterpret_cast<T*>(fout) + gi, reinterpret_cast<const T*>(sG) + (pp * NB2 + cc) * RS,
                 (unsigned)(nbv * NB2 * sizeof(T)), pol);
      }
      bulk_commit();
      continue;
    }
    const int lane = tid & 31, warp = tid >> 5, nwarps = nth >> 5;
    for (int run = warp; run < pc * NB2; run += nwarps) {
      const int pp = run / NB2, cc = run % NB2;
      const size_t gi = ((size_t)(w0 + pp) * NB2 + cc) * NB2 * NB2 + (size_t)b0 * NB2;
      if (CPLX) {
        C* dst = reinterpret_cast<C*>(fout) + gi;
        const C* src = sG + (pp * NB2 + cc) * RUN;
        for (int o = lane; o < nbv * NB2; o += 32) dst[o] = src[o];
      } else {
        T* dst = reinterpret_cast<T*>(fout) + gi;
        const T* src = reinterpret_cast<const T*>(sG) + (pp * NB2 + cc) * RS;
        const int rot = SWZ ? (pp & 3) : 0;
        constexpr int VW = 16 / sizeof(T);   // elements per 16-byte vector
        if (fout_al16 && nbv == NB && (RUN % VW) == 0 && (gi % VW) == 0) {
          if constexpr (SWZ) {
            for (int o = lane * 4; o < RUN; o += 128)
              *reinterpret_cast<float4*>(dst + o) = unrotate4(*reinterpret_cast<const float4*>(src + o), rot);
          } else {
            for (int o = lane * VW; o < RUN; o += 32 * VW) store16(dst + o, src + o);
          }
        } else {
          for (int o = lane; o < nbv * NB2; o += 32) dst[o] = src[SWZ ? synth_swz(o, rot) : o];
        }
      }
    }
  }
  if (BULK && fout_al16) bulk_wait_all();   // shared memory must outlive the bulk copies reading it
}

// (NB, P) of the synthesis: betas per block and omega points per batch, chosen
// so that shared memory allows two resident blocks where possible and the
// alpha stage fits one round of 256 threads.
template <int B, typename T, bool CPLX> struct SynthCfg {
  static constexpr long long nrows = CPLX ? (long long)B * (2 * B - 1) * (2 * B + 1) / 3
                                          : (long long)B * (B + 1) * (4 * B - 1) / 6;
  static constexpr int NM = CPLX ? 2 * B - 1 : B;
  static constexpr int NCOL = CPLX ? 2 * B : B;
  // the d table of one beta above 64 KB: read it from a global table
  static constexpr bool GD = nrows * (long long)sizeof(T) > 64 * 1024;
  static constexpr long long bytes(int nb, int p) {
    const long long c = 2 * (long long)sizeof(T);
    const long long g = (long long)nb * NM * (2 * B * p + p) * c;                     // G/H, padded
    const long long rs = sizeof(T) == 4 ? ((long long)nb * 2 * B + 27) / 32 * 32 + 4   // synth_rs
                                        : (long long)nb * 2 * B + 1;
    const long long st = CPLX ? (long long)p * 2 * B * nb * 2 * B * c                 // f staging
                              : (long long)p * 2 * B * rs * (long long)sizeof(T);
    return (GD ? 0 : nb * nrows * (long long)sizeof(T)) + 32 + (long long)NM * (2 * B - 1) * 8 + (g > st ? g : st);
  }
  // two resident blocks (110 KB each) when a batch of 4 fits, else one (220 KB);
  // with the d table in global memory (large B) one block with two betas beat
  // two blocks with one (B = 30, FP32: 10.2 vs 11.2 ms per launch at 60x60)
  static constexpr long long budget() {
    return (!GD && bytes(1, 4) <= 110 * 1024) ? 110 * 1024 : 220 * 1024;
  }
  // betas per block: up to 4 (each coefficient then feeds 4 x P FMAs), as
  // many as keep a batch of 4 omega points within the budget
  static constexpr int pick_nb() {
    return bytes(4, 4) <= budget() && 4 * NCOL * 4 <= 256 ? 4
         : bytes(2, 4) <= budget() ? 2 : 1;
  }
  static constexpr int NB = pick_nb();
  static constexpr int pick_p() {
    int p = NB >= 4 ? 4 : 8;
    while (p > 1 && (bytes(NB, p) > budget() || NB * NCOL * p > 256)) p /= 2;
    return p;
  }
  static constexpr int P = pick_p();
};

// (m, n) pairs with their row start, l-run length, m slot and n bin, longest
// runs first (the order keeps the lanes of a warp on loops of similar length)
template <int B, bool CPLX>
static int build_pairs(hp_plan* p, int2* dpairs) {
  constexpr int NB2 = 2 * B, NM = CPLX ? 2 * B - 1 : B, NPAIR = NM * (2 * B - 1);
  std::vector<std::pair<int, int2>> v;
  const int lmax = B - 1, D = 2 * lmax + 1, mlo = CPLX ? -lmax : 0;
  for (int mi = 0; mi < NM; ++mi)
    for (int n = -lmax; n <= lmax; ++n) {
      const int m = mi + mlo;
      const int lmin = std::max(std::abs(m), std::abs(n));
      const int len = lmax - lmin + 1;
      const int q = n >= 0 ? n : n + NB2;
      int2 e;
      e.x = p->h_seg[(size_t)(m - p->m_lo) * D + n + lmax];
      e.y = len | (mi << 8) | (q << 16) | ((n == 0 ? 1 : 0) << 24);
      v.push_back({len, e});
    }
  std::stable_sort(v.begin(), v.end(), [](const std::pair<int, int2>& a, const std::pair<int, int2>& b) {
    return a.first > b.first;
  });
  std::vector<int2> h;
  for (auto& x : v) h.push_back(x.second);
  HP_CUDA_TRY(cudaMemcpy(dpairs, h.data(), sizeof(int2) * NPAIR, cudaMemcpyHostToDevice));
  return HP_OK;
}

template <typename T>
__global__ void k_sd_table(RowLayout L, const T* __restrict__ wig, T* __restrict__ out, int NB, int ngroups,
                           int synth, const double* __restrict__ qw = nullptr) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)ngroups * L.nrows * NB;
  if (t >= n) return;
  int bb;
  long long r;
  if (synth) { bb = (int)(t % NB); r = (t / NB) % L.nrows; }
  else { r = t % L.nrows; bb = (int)((t / L.nrows) % NB); }
  const int g = (int)(t / ((long long)NB * L.nrows));
  const int b = g * NB + bb;
  T v = (T)0;
  if (b < 2 * L.B)
    v = synth ? (T)(2 * L.rows[r].x + 1) * wig[(size_t)b * L.nrows + r]
              : (T)(qw[b] * (double)wig[(size_t)b * L.nrows + r]);
  out[t] = v;
}

template <int B, typename T, bool CPLX>
int synth_launch(hp_plan* p, const c2<T>* Fp, void* f, cudaStream_t s) {
  using C = c2<T>;
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  using Cfg = SynthCfg<B, T, CPLX>;
  constexpr int NB = Cfg::NB, P = Cfg::P, NB2 = 2 * B, NM = Cfg::NM;
  constexpr bool GD = Cfg::GD;
  static_assert(NB * Cfg::NCOL * P <= 256, "alpha stage must fit one round");
  const size_t sd_bytes = GD ? 0 : ((size_t)NB * p->nrows * sizeof(T) + 15) / 16 * 16;
  constexpr int RS = synth_rs<T, NB, NB2>();
  const size_t sg_bytes = std::max((size_t)NB * NM * (NB2 * P + P) * sizeof(C),
                                   CPLX ? (size_t)P * NB2 * NB * NB2 * sizeof(C)
                                        : (size_t)P * NB2 * RS * sizeof(T));
  constexpr int NPAIR = NM * (2 * B - 1);
  const size_t pr_bytes = ((size_t)NPAIR * sizeof(int2) + 15) / 16 * 16;
  const size_t smem = sd_bytes + pr_bytes + sg_bytes;
  if (smem > (size_t)smem_limit()) {
    hp_set_error("synthesis tables exceed shared memory for this bandlimit");
    return HP_ERR_UNSUPPORTED;
  }
  int st = HP_OK;
  const char* key = CPLX ? "tf.pairs_c" : "tf.pairs_r";
  bool have = false;
  for (auto& kv : p->ws) if (kv.first == key) have = true;
  int2* dpairs = (int2*)p->ws_get(key, sizeof(int2) * NPAIR, &st);
  if (st) return st;
  if (!have) {
    st = build_pairs<B, CPLX>(p, dpairs);
    if (st) return st;
  }
  const int ngroups = (NB2 + NB - 1) / NB;
  const T* dtab = sizeof(T) == 8 ? (const T*)(const void*)p->wig64 : (const T*)(const void*)p->wig32;
  if (GD) {   // (2l+1) d as [group][row][NB], built once per plan
    const char* gkey = sizeof(T) == 8 ? (CPLX ? "tf.sdg64c" : "tf.sdg64") : (CPLX ? "tf.sdg32c" : "tf.sdg32");
    bool hv = false;
    for (auto& kv : p->ws) if (kv.first == gkey) hv = true;
    const long long n = (long long)ngroups * p->nrows * NB;
    T* sdg = (T*)p->ws_get(gkey, sizeof(T) * n, &st);
    if (st) return st;
    if (!hv) {
      k_sd_table<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p->layout(), dtab, sdg, NB, ngroups, 1);
      HP_CUDA_TRY(cudaGetLastError());
    }
    dtab = sdg;
  }
  const long long nbatches = (p->nx + P - 1) / P;
  // synth_waves (8 unless tuned) resident waves of blocks over 148 SMs
  constexpr int NT = 256;
  long long gx = std::max(1LL, (148LL * (sizeof(T) == 8 ? 1 : 2) * p->tune.synth_waves) / ngroups);
  int nbatch = (int)std::max(1LL, (nbatches + gx - 1) / gx);
  gx = (nbatches + nbatch - 1) / nbatch;
  dim3 grid((unsigned)(gx * ngroups), 1);
  // omega points per beta-stage item: the plan's tuned choice (FP32 plans; 1 otherwise)
  const int pt = (sizeof(T) == 4 && P % p->tune.synth_pt == 0) ? p->tune.synth_pt : 1;
  auto launch = [&](auto kern) -> int {
    HP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ProfScope _ps(p, "tf.synth", s);
    kern<<<grid, NT, smem, s>>>(p->layout(), Fp, dtab, dpairs, f, nbatch);
    HP_CUDA_TRY(cudaGetLastError());
    return HP_OK;
  };
  if constexpr (sizeof(T) == 4) {
    if (pt == 2 && P % 2 == 0) return launch(k_synth<B, T, NB, P, CPLX, GD, (P % 2 == 0 ? 2 : 1)>);
    if (pt == 4 && P % 4 == 0) return launch(k_synth<B, T, NB, P, CPLX, GD, (P % 4 == 0 ? 4 : 1)>);
  }
  return launch(k_synth<B, T, NB, P, CPLX, GD, 1>);
}



// ----------------------------------------- analysis without atomics ----
// Stage 1 (k_anal_ag): block = (beta, chunk of PA omega points).  For each
// omega point the alpha FFT over a and the gamma FFT over c of f(., b, ., w)
// (times an optional grid multiplier) give Q_b[m][n]; it is written to
// Qg[(m, n bin)][b][w] with the chunk's omega points consecutive.
// Stage 2 (k_anal_beta): thread = ((m, n) pair, omega point), all l of the
// pair: F^l_mn[w] = sum_b w_b d^l_mn(beta_b) Q_b[m][n][w], written straight
// into the [row][omega] layout.  Every output has one owner: no atomics.
template <int B, typename T, int PA, bool CPLX>
__global__ void __launch_bounds__(B >= 24 ? 128 : 256, B >= 24 && sizeof(T) == 4 ? 3 : 1)
    k_anal_ag(const void* __restrict__ fin, const double* __restrict__ mult,
                                                 c2<T>* __restrict__ Qg, long long w0, long long nwc) {
  using C = c2<T>;
  constexpr int NB2 = 2 * B, lmax = B - 1, D = 2 * lmax + 1;
  constexpr int NM = CPLX ? D : B;
  constexpr int MLO = CPLX ? -lmax : 0;
  extern __shared__ __align__(16) unsigned char smraw[];
  // input tile [PA][c][a] (complex, or real values for real densities); the
  // alpha stage reads its lines into registers before a barrier, so its
  // output [PA][m][c or q] reuses the same shared memory
  C* sIn = reinterpret_cast<C*>(smraw);
  T* sInR = reinterpret_cast<T*>(smraw);
  C* sQ = reinterpret_cast<C*>(smraw);
  const int b = blockIdx.y;
  const long long wl0 = (long long)blockIdx.x * PA;                       // chunk-local omega
  const int pc = (int)min((long long)PA, nwc - wl0);
  const int tid = threadIdx.x, nth = blockDim.x;
  const int NG = NB2 * NB2;
  constexpr long long TILE = (long long)PA * (2LL * NM * NB2 > (long long)NB2 * NB2 * (CPLX ? 2 : 1)
                                               ? 2LL * NM * NB2 : (long long)NB2 * NB2 * (CPLX ? 2 : 1));
  T* smult = reinterpret_cast<T*>(smraw) + TILE;   // [c][a] multiplier of this beta (real densities)
  // Real densities whose 2B-runs are 16-byte aligned: every run of 2B
  // consecutive a arrives by 16-byte asynchronous copies (all in flight at
  // once), the grid multiplier slice of this beta is staged beside it and
  // applied when the alpha stage reads its lines.
  constexpr bool ASYNC = !CPLX && (NB2 * sizeof(T)) % 16 == 0;
  const bool async_ok = ASYNC && (reinterpret_cast<unsigned long long>(fin) & 15ull) == 0;
  if (async_ok) {
    constexpr int VPR = NB2 * (int)sizeof(T) / 16;                       // 16-byte pieces per run
    for (int e = tid; e < pc * NB2 * VPR; e += nth) {
      const int run = e / VPR, piece = e % VPR, pp = run / NB2, cc = run % NB2;
      const long long w = w0 + wl0 + pp;
      const long long gi = (long long)NB2 * ((long long)b + NB2 * ((long long)cc + NB2 * w));
      cp_async<16>(sInR + (size_t)run * NB2 + piece * (16 / sizeof(T)),
                   reinterpret_cast<const T*>(fin) + gi + piece * (16 / sizeof(T)), true);
    }
    for (int e = tid; e < NG; e += nth) {
      const int cc = e / NB2, a = e % NB2;
      smult[e] = mult ? (T)mult[a + NB2 * (b + NB2 * cc)] : (T)1;
    }
    cp_async_wait_all();
  } else
  // load f(a, b, c, w) for this beta: runs of 2B consecutive a
  for (int e = tid; e < pc * NG; e += nth) {
    const int pp = e / NG, r = e % NG, cc = r / NB2, a = r % NB2;
    const long long w = w0 + wl0 + pp;
    const long long gi = (long long)a + NB2 * ((long long)b + NB2 * ((long long)cc + NB2 * w));
    const T mv = mult ? (T)mult[a + NB2 * (b + NB2 * cc)] : (T)1;
    if (CPLX) {
      C v = reinterpret_cast<const C*>(fin)[gi];
      v.x *= mv;
      v.y *= mv;
      sIn[e] = v;
    } else {
      sInR[e] = reinterpret_cast<const T*>(fin)[gi] * mv;
    }
  }
  __syncthreads();
  // alpha, one item per thread (the host keeps the item count within the
  // block).  Real densities: item (p, c pair), columns c, c+1 share one complex
  // FFT, z = f_c + i f_{c+1}: X_c[m] = (Z[m] + conj Z[-m]) / 2,
  // X_{c+1}[m] = (Z[m] - conj Z[-m]) / 2i.  Complex densities: item (p, c).
  {
    const int nitems = CPLX ? pc * NB2 : pc * B;
    const bool act = tid < nitems;
    const int pp = CPLX ? tid / NB2 : tid / B;
    const int c0 = CPLX ? tid % NB2 : 2 * (tid % B);
    C x[NB2];
    if (act) {
      if (CPLX) {
        const C* src = sIn + (size_t)tid * NB2;
#pragma unroll
        for (int a = 0; a < NB2; ++a) x[a] = src[a];
      } else if (async_ok) {
        const T* r0 = sInR + ((size_t)pp * NB2 + c0) * NB2;
        const T* r1 = r0 + NB2;
        const T* m0 = smult + (size_t)c0 * NB2;
        const T* m1 = m0 + NB2;
#pragma unroll
        for (int a = 0; a < NB2; ++a) { x[a].x = r0[a] * m0[a]; x[a].y = r1[a] * m1[a]; }
      } else {
        const T* r0 = sInR + ((size_t)pp * NB2 + c0) * NB2;
        const T* r1 = r0 + NB2;
#pragma unroll
        for (int a = 0; a < NB2; ++a) { x[a].x = r0[a]; x[a].y = r1[a]; }
      }
    }
    __syncthreads();
    if (act) {
      fft<NB2, true>(x);
      C* dst = sQ + (size_t)pp * NM * NB2 + c0;
      if (CPLX) {
#pragma unroll
        for (int mi = 0; mi < NM; ++mi) {
          const int m = mi + MLO;
          dst[(size_t)mi * NB2] = x[m >= 0 ? m : m + NB2];
        }
      } else {
#pragma unroll
        for (int m = 0; m < NM; ++m) {
          const C zp = x[m], zm = x[(NB2 - m) % NB2];
          C u, v;
          u.x = (T)0.5 * (zp.x + zm.x);
          u.y = (T)0.5 * (zp.y - zm.y);
          v.x = (T)0.5 * (zp.y + zm.y);
          v.y = (T)0.5 * (zm.x - zp.x);
          dst[(size_t)m * NB2] = u;
          dst[(size_t)m * NB2 + 1] = v;
        }
      }
    }
  }
  __syncthreads();
  // gamma: item (p, m): FFT(+) over c, in place (bins n mod 2B)
  for (int it = tid; it < pc * NM; it += nth) {
    C* row = sQ + (size_t)it * NB2;
    C x[NB2];
#pragma unroll
    for (int j = 0; j < NB2; ++j) x[j] = row[j];
    fft<NB2, true>(x);
#pragma unroll
    for (int j = 0; j < NB2; ++j) row[j] = x[j];
  }
  __syncthreads();
  // store: Qg[((m * 2B + q) * 2B + b) * nwc + w], consecutive omega points
  for (int e = tid; e < NM * NB2 * pc; e += nth) {
    const int pp = e % pc, mq = e / pc;
    Qg[((long long)mq * NB2 + b) * nwc + wl0 + pp] = sQ[(size_t)pp * NM * NB2 + mq];
  }
}

template <int B, typename T, bool CPLX>
__global__ void __launch_bounds__(256) k_anal_beta(RowLayout L, const c2<T>* __restrict__ Qg,
                                                   const T* __restrict__ dw, const int2* __restrict__ pairs,
                                                   int npairs, c2<T>* __restrict__ out, long long w0, long long nwc) {
  using C = c2<T>;
  constexpr int NB2 = 2 * B;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int pi = blockIdx.y * (blockDim.x >> 5) + warp;
  if (pi >= npairs) return;
  const long long wl = (long long)blockIdx.x * 32 + lane;
  if (wl >= nwc) return;
  const int2 pe = pairs[pi];
  const int s = pe.x, len = pe.y & 0xff, mi = (pe.y >> 8) & 0xff, q = (pe.y >> 16) & 0xff;
  const C* qsrc = Qg + ((long long)(mi * NB2 + q) * NB2) * nwc + wl;
  const T* dsrc = dw + (size_t)s * NB2;
  C acc[B];
#pragma unroll
  for (int j = 0; j < B; ++j) acc[j] = czero<C>();
  for (int b0 = 0; b0 < NB2; b0 += 4) {
    C v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = (b0 + u < NB2) ? qsrc[(long long)(b0 + u) * nwc] : czero<C>();
#pragma unroll
    for (int j = 0; j < B; ++j) {
      if (j < len) {
        if constexpr (sizeof(T) == 4 && NB2 % 4 == 0) {
          // four consecutive betas of one row in one 16-byte load (the row
          // starts 16-byte aligned: NB2 and b0 are multiples of 4)
          const float4 d4 = __ldg(reinterpret_cast<const float4*>(dsrc + (size_t)j * NB2 + b0));
          const T dd[4] = {d4.x, d4.y, d4.z, d4.w};
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            acc[j].x = fma(dd[u], v[u].x, acc[j].x);
            acc[j].y = fma(dd[u], v[u].y, acc[j].y);
          }
        } else {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (b0 + u < NB2) {
              const T d = __ldg(dsrc + (size_t)j * NB2 + b0 + u);
              acc[j].x = fma(d, v[u].x, acc[j].x);
              acc[j].y = fma(d, v[u].y, acc[j].y);
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < B; ++j)
    if (j < len) out[(long long)(s + j) * L.nx + w0 + wl] = acc[j];
}

// dw[row][b] = w_b d^l_mn(beta_b)
template <typename T>
__global__ void k_dw_table(RowLayout L, const T* __restrict__ wig, const double* __restrict__ qw,
                           T* __restrict__ dw) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int NB2 = 2 * L.B;
  if (t >= L.nrows * NB2) return;
  const long long r = t / NB2;
  const int b = (int)(t % NB2);
  dw[t] = (T)(qw[b] * (double)wig[(size_t)b * L.nrows + r]);
}

// largest omega batch (16, 8, 4, 2, 1) whose stage-1 tiles fit the budget
template <int B, typename T, bool CPLX> struct AnalCfg {
  static constexpr int NM = CPLX ? 2 * B - 1 : B;
  static constexpr long long in_w = (long long)(2 * B) * (2 * B) * (CPLX ? 2 : 1);   // T elements per omega
  static constexpr long long q_w = 2LL * NM * (2 * B);
  // tiles for pa omega points, plus (real densities) this beta's grid multiplier slice
  static constexpr long long bytes(int pa) {
    return (long long)pa * (in_w > q_w ? in_w : q_w) * (long long)sizeof(T) +
           (CPLX ? 0 : (long long)(2 * B) * (2 * B) * (long long)sizeof(T));
  }
  static constexpr int items = CPLX ? 2 * B : B;    // alpha items per omega point
  // threads per block: from B = 24 the 2B-point register FFTs need ~170-255
  // registers, so two 128-thread blocks per SM overlap loads and FFTs
  static constexpr int NT = B >= 24 ? 128 : 256;
  // two resident blocks where a batch of 4 fits 110 KB, else one block of up to 220 KB
  static constexpr long long cap() { return bytes(4) <= 110 * 1024 ? 110 * 1024 : 220 * 1024; }
  static constexpr int pick() {
    int pa = 16;
    while (pa > 1 && (bytes(pa) > cap() || pa * items > NT)) pa /= 2;
    return pa;
  }
  static constexpr int PA = pick();
};

template <int B, typename T, bool CPLX>
int anal2_launch(hp_plan* p, const void* f, const double* mult, c2<T>* out, cudaStream_t s) {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  using C = c2<T>;
  using Cfg = AnalCfg<B, T, CPLX>;
  constexpr int PA = Cfg::PA, NB2 = 2 * B, NM = Cfg::NM;
  const size_t smem = (size_t)Cfg::bytes(PA);
  if (smem > (size_t)smem_limit()) { hp_set_error("analysis tiles exceed shared memory"); return HP_ERR_UNSUPPORTED; }
  int st = HP_OK;
  // pair table (shared with the synthesis) and the w_b d table
  constexpr int NPAIR = NM * (2 * B - 1);
  const char* key = CPLX ? "tf.pairs_c" : "tf.pairs_r";
  bool have = false;
  for (auto& kv : p->ws) if (kv.first == key) have = true;
  int2* dpairs = (int2*)p->ws_get(key, sizeof(int2) * NPAIR, &st);
  if (st) return st;
  if (!have) {
    st = build_pairs<B, CPLX>(p, dpairs);
    if (st) return st;
  }
  const char* dkey = sizeof(T) == 8 ? "tf.dw64" : "tf.dw32";
  have = false;
  for (auto& kv : p->ws) if (kv.first == dkey) have = true;
  T* dw = (T*)p->ws_get(dkey, sizeof(T) * p->nrows * NB2, &st);
  if (st) return st;
  if (!have) {
    const long long n = p->nrows * NB2;
    k_dw_table<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
        p->layout(), sizeof(T) == 8 ? (const T*)(const void*)p->wig64 : (const T*)(const void*)p->wig32, p->qw, dw);
    HP_CUDA_TRY(cudaGetLastError());
  }
  // omega chunks keep the staged tiles within 2 GB
  const long long per_w = (long long)NM * NB2 * NB2 * (long long)sizeof(C);
  long long nwc = std::max(32LL, (2LL << 30) / per_w / 32 * 32);
  nwc = std::min(nwc, (p->nx + 31) / 32 * 32);
  C* Qg = (C*)p->ws_get("tf.Q", (size_t)per_w * nwc, &st);
  if (st) return st;
  HP_CUDA_TRY(cudaFuncSetAttribute(k_anal_ag<B, T, PA, CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (long long w0 = 0; w0 < p->nx; w0 += nwc) {
    const long long nw = std::min(nwc, p->nx - w0);
    {
      ProfScope _ps(p, "tf.anal.ag", s);
      dim3 ga((unsigned)((nw + PA - 1) / PA), (unsigned)NB2);
      k_anal_ag<B, T, PA, CPLX><<<ga, Cfg::NT, smem, s>>>(f, mult, Qg, w0, nw);
      HP_CUDA_TRY(cudaGetLastError());
    }
    if constexpr (sizeof(T) == 4) {
      // AUTO: tensor cores from B = 15 (B=15, 32x32: 0.046 vs 0.052 ms; B=30: 0.24 vs
      // 0.50 ms), CUDA cores below (B=8: 0.015 vs 0.009 ms, set-up dominates)
      const bool tc = p->beta_engine == HP_BETA_TENSOR || p->beta_engine == HP_BETA_TENSOR_BF16 ||
                      (p->beta_engine == HP_BETA_AUTO && p->B >= 15);
      if (tc && tc_beta_supported(p)) {
        st = tc_beta_forward(p, reinterpret_cast<const float2*>(Qg), dpairs, NPAIR, reinterpret_cast<float2*>(out),
                             w0, nw, s);
        if (st) return st;
        continue;
      }
    }
    ProfScope _ps(p, "tf.anal.beta", s);
    dim3 gb((unsigned)((nw + 31) / 32), (unsigned)((NPAIR + 7) / 8));
    k_anal_beta<B, T, CPLX><<<gb, 256, 0, s>>>(p->layout(), Qg, dw, dpairs, NPAIR, out, w0, nw);
    HP_CUDA_TRY(cudaGetLastError());
  }
  return HP_OK;
}


// explicit instantiations of the launchers for one bandlimit (used by the
// part files)
#ifdef HP_TRANSFORM_PART
#define HP_INST_B(b)                                                                                   \
  template int synth_launch<b, float, false>(hp_plan*, const float2*, void*, cudaStream_t);        \
  template int synth_launch<b, float, true>(hp_plan*, const float2*, void*, cudaStream_t);         \
  template int synth_launch<b, double, false>(hp_plan*, const double2*, void*, cudaStream_t);      \
  template int synth_launch<b, double, true>(hp_plan*, const double2*, void*, cudaStream_t);       \
  template int anal2_launch<b, float, false>(hp_plan*, const void*, const double*, float2*, cudaStream_t);  \
  template int anal2_launch<b, float, true>(hp_plan*, const void*, const double*, float2*, cudaStream_t);   \
  template int anal2_launch<b, double, false>(hp_plan*, const void*, const double*, double2*, cudaStream_t); \
  template int anal2_launch<b, double, true>(hp_plan*, const void*, const double*, double2*, cudaStream_t);
#endif
