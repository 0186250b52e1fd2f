// SO(3) x R^n transforms (fftSO3R forward / backward) on the internal layout.
//
// Backward (ifftSO3R.m:16-37, pendulum.m:284-304):
//   1. inverse omega FFT of every coefficient row (plane pass over (k1,k2),
//      line pass over k3), normalised by 1/nx  -> rows x physical omega;
//   2. transpose to omega-major so each omega point's coefficients are contiguous;
//   3. synthesis per omega point and beta_b:
//        G_b[m][n] = sum_l (2l+1) d^l_mn(beta_b) F^l_mn
//        H_b[m][c] = sum_n G_b[m][n] e^{-i n gamma_c}          (2B-point FFT)
//        f[a][b][c] = sum_m H_b[m][c] e^{-i m alpha_a}          (2B-point FFT)
//      For HP_REAL plans only m >= 0 is stored and f = Re(H_0 + 2 sum_{m>0} ...),
//      the Hermitian reconstruction of ifftn(..., 'symmetric').
// Forward (fftSO3R.m:89-106) runs the same stages in reverse with the
// quadrature weights w_b.
#include <algorithm>
#include <vector>
#include "common.cuh"
#include "plan.hpp"
#include "transform_b.cuh"

using namespace hp;

// ------------------------------------------------------------ omega FFTs ----

// Omega-blocked layout of the synthesis input: blocks of blk consecutive omega
// points, each block holding every row's blk values contiguously,
// [w / blk][row][w % blk].  One synthesis batch (blk = P omega points) then
// reads a single contiguous run of nrows * P values, and the rows of one
// (m, n) pair (consecutive in l) sit P values apart.  FP64 synthesis reads
// this layout (B = 15, 32^3: 9.0 ms per synthesis against 10.0 from
// [row][omega], while the blocked omega-FFT stores cost 0.35 ms more); FP32
// synthesis reads [row][omega] (the same 2.85 ms either way, and the blocked
// stores would cost 0.5 ms more).
__host__ __device__ __forceinline__ long long omega_block_index(long long w, long long row, long long nrows, int blk) {
  return (w / blk * nrows + row) * blk + w % blk;
}

// Planes per block of k_wplane: enough that the N FFTs of each pass of every
// plane give the 128 threads one FFT each, within 64 KB of shared memory.
template <int N, typename T> __host__ __device__ constexpr int wplane_ppb() {
  constexpr int want = 128 / N > 1 ? 128 / N : 1;
  constexpr int fit = (int)((64 * 1024) / ((size_t)N * (N + 1) * sizeof(c2<T>)));
  return want < fit ? want : (fit > 1 ? fit : 1);
}

// 2-D FFT over (k1, k2) of every (row, k3) plane; PPB consecutive planes (one
// contiguous run of PPB N^2 values) per block.
// blk > 0: the output goes to the omega-blocked layout of the synthesis input
// (see omega_block_index), plane pl holding omega points pl_w0 .. pl_w0 + N^2 of
// row pl / planes_per_row.  in may equal out (a block reads all of its planes
// before it writes).
template <int N, typename Tin, typename T, bool INV>
__global__ void __launch_bounds__(128) k_wplane(const c2<Tin>* __restrict__ in, c2<T>* __restrict__ out,
                                                long long nplanes, T scale, int blk = 0, long long nrows = 0,
                                                int planes_per_row = 1) {
  using C = c2<T>;
  constexpr int PPB = wplane_ppb<N, T>();
  constexpr int PS = N * (N + 1);
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);   // [PPB][N][N+1]
  const long long pl0 = (long long)blockIdx.x * PPB;
  if (pl0 >= nplanes) return;
  const int np = (int)min((long long)PPB, nplanes - pl0);
  const int tot = np * N * N;
  const c2<Tin>* src = in + pl0 * N * N;
  if constexpr (sizeof(Tin) == sizeof(T)) {
    // no conversion: the block's whole run is in flight at once (cp.async,
    // no register round trip)
    for (int e = threadIdx.x; e < tot; e += blockDim.x)
      cp_async<sizeof(C)>(sm + (e / (N * N)) * PS + ((e / N) % N) * (N + 1) + e % N, src + e, true);
    cp_async_wait_all();
  } else {
    for (int e0 = threadIdx.x; e0 < tot; e0 += 4 * blockDim.x) {
      C v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * blockDim.x;
        v[u] = e < tot ? cvt<C, c2<Tin>>(src[e]) : czero<C>();
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * blockDim.x;
        if (e < tot) sm[(e / (N * N)) * PS + ((e / N) % N) * (N + 1) + e % N] = v[u];
      }
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < np * N; it += blockDim.x) {
    C* row = sm + (it / N) * PS + (it % N) * (N + 1);
    C x[N];
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = row[j];
    fft<N, INV>(x);
#pragma unroll
    for (int j = 0; j < N; ++j) row[j] = x[j];
  }
  __syncthreads();
  for (int it = threadIdx.x; it < np * N; it += blockDim.x) {
    C* col = sm + (it / N) * PS + it % N;
    C x[N];
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = col[j * (N + 1)];
    fft<N, INV>(x);
#pragma unroll
    for (int j = 0; j < N; ++j) col[j * (N + 1)] = scale * x[j];
  }
  __syncthreads();
  if (blk > 0) {
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      const long long pl = pl0 + e / (N * N);
      const int q = e % (N * N);
      const long long row = pl / planes_per_row, w0 = (pl % planes_per_row) * (long long)(N * N);
      out[omega_block_index(w0 + q, row, nrows, blk)] = sm[(e / (N * N)) * PS + (q / N) * (N + 1) + q % N];
    }
    return;
  }
  C* dst = out + pl0 * N * N;
  for (int e = threadIdx.x; e < tot; e += blockDim.x) dst[e] = sm[(e / (N * N)) * PS + ((e / N) % N) * (N + 1) + e % N];
}

// 1-D FFT along the last omega axis (stride N^2) of a [row][N^3] array.
// blk > 0: in and out are in the omega-blocked layout (N^2 a multiple of blk).
template <int N, typename T, bool INV>
__global__ void __launch_bounds__(128) k_wline(const c2<T>* __restrict__ in, c2<T>* __restrict__ out,
                                               long long nrows, T scale, int blk = 0) {
  using C = c2<T>;
  constexpr long long plane = (long long)N * N;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= nrows * plane) return;
  const long long row = t / plane, p = t % plane;
  C x[N];
  if (blk > 0) {
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = in[omega_block_index(j * plane + p, row, nrows, blk)];
    fft<N, INV>(x);
#pragma unroll
    for (int j = 0; j < N; ++j) out[omega_block_index(j * plane + p, row, nrows, blk)] = scale * x[j];
    return;
  }
  const C* src = in + row * plane * N + p;
#pragma unroll
  for (int j = 0; j < N; ++j) x[j] = src[j * plane];
  fft<N, INV>(x);
  C* dst = out + row * plane * N + p;
#pragma unroll
  for (int j = 0; j < N; ++j) dst[j * plane] = scale * x[j];
}

template <typename T>
__global__ void k_to_c64(const c2<T>* __restrict__ in, double2* __restrict__ out, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = cvt<double2, c2<T>>(in[i]);
}

// -------------------------------------------------------------- drivers ----


template <int N, typename Tin, typename T>
static int omega_fft(hp_plan* p, const c2<Tin>* in, c2<T>* out, bool inv, cudaStream_t s, int blk = 0) {
  // in/out [row][nx]; in may equal out only when Tin == T.  blk > 0 (inverse
  // only): out in the omega-blocked layout of the synthesis input.
  const T scale = inv ? (T)1 / (T)p->nx : (T)1;
  const int ppr = p->ndim == 3 ? N : 1;
  const long long nplanes = p->nrows * ppr;
  constexpr int PPB = wplane_ppb<N, T>();
  const size_t smem = sizeof(c2<T>) * PPB * N * (N + 1);
  const unsigned nblk = (unsigned)((nplanes + PPB - 1) / PPB);
  auto plane = [&](T sc) -> int {
    ProfScope _ps(p, "tf.wplane", s);
    if (inv) {
      HP_CUDA_TRY(cudaFuncSetAttribute(k_wplane<N, Tin, T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_wplane<N, Tin, T, true><<<nblk, 128, smem, s>>>(in, out, nplanes, sc, blk, p->nrows, ppr);
    } else {
      HP_CUDA_TRY(cudaFuncSetAttribute(k_wplane<N, Tin, T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_wplane<N, Tin, T, false><<<nblk, 128, smem, s>>>(in, out, nplanes, sc, blk, p->nrows, ppr);
    }
    HP_CUDA_TRY(cudaGetLastError());
    return HP_OK;
  };
  if (p->ndim == 3) {
    // plane pass (k1,k2) then line pass along k3, scale applied in the line pass
    int st = plane((T)1);
    if (st) return st;
    const long long nt = p->nrows * (long long)N * N;
    ProfScope _ps(p, "tf.wline", s);
    if (inv) k_wline<N, T, true><<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(out, out, p->nrows, scale, blk);
    else k_wline<N, T, false><<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(out, out, p->nrows, scale, blk);
    HP_CUDA_TRY(cudaGetLastError());
    return HP_OK;
  }
  return plane(scale);
}

template <typename Tin, typename T>
static int omega_fft_any(hp_plan* p, const c2<Tin>* in, c2<T>* out, bool inv, cudaStream_t s, int blk = 0) {
  switch (p->N) {
#define X(n) case n: return omega_fft<n, Tin, T>(p, in, out, inv, s, blk);
    HP_FOR_EACH_N(X)
#undef X
    default:
      hp_set_error("omega grid size 2Bx not supported (even, 4..64)");
      return HP_ERR_UNSUPPORTED;
  }
}

// Per-bandlimit synthesis and analysis launchers: defined in transform_b.cuh,
// instantiated in transform_b0.cu .. transform_b3.cu (bandlimits by B mod 4),
// so that their kernels compile in parallel.
#define X(b)                                                                                            \
  extern template int synth_launch<b, float, false>(hp_plan*, const float2*, void*, cudaStream_t);        \
  extern template int synth_launch<b, float, true>(hp_plan*, const float2*, void*, cudaStream_t);         \
  extern template int synth_launch<b, double, false>(hp_plan*, const double2*, void*, cudaStream_t);      \
  extern template int synth_launch<b, double, true>(hp_plan*, const double2*, void*, cudaStream_t);       \
  extern template int anal2_launch<b, float, false>(hp_plan*, const void*, const double*, float2*, cudaStream_t);  \
  extern template int anal2_launch<b, float, true>(hp_plan*, const void*, const double*, float2*, cudaStream_t);   \
  extern template int anal2_launch<b, double, false>(hp_plan*, const void*, const double*, double2*, cudaStream_t); \
  extern template int anal2_launch<b, double, true>(hp_plan*, const void*, const double*, double2*, cudaStream_t);
HP_FOR_EACH_B(X)
#undef X

// Omega block of the synthesis input (P of the synthesis configuration) for
// FP64 synthesis; 0 (the [row][omega] layout) for FP32.
template <typename T, bool CPLX>
static int synth_block(const hp_plan* p) {
  if (sizeof(T) == 4) return 0;
  switch (p->B) {
#define X(b) case b: return SynthCfg<b, T, CPLX>::P;
    HP_FOR_EACH_B(X)
#undef X
    default: return 1;
  }
}

template <typename T, bool CPLX>
static int synth_any(hp_plan* p, const c2<T>* Fp, void* f, cudaStream_t s) {
  switch (p->B) {
#define X(b) case b: return synth_launch<b, T, CPLX>(p, Fp, f, s);
    HP_FOR_EACH_B(X)
#undef X
    default:
      hp_set_error("bandlimit B not supported (2..32)");
      return HP_ERR_UNSUPPORTED;
  }
}


// Inverse omega FFT of every row into the synthesis input (a plan workspace;
// omega-blocked and sized for whole blocks for FP64, [row][omega] for FP32),
// then the synthesis.
template <typename Tin, typename T>
static int backward_rows(hp_plan* p, const c2<Tin>* Fint, void* f, int complex_out, cudaStream_t s) {
  using C = c2<T>;
  int st = HP_OK;
  const int blk = complex_out ? synth_block<T, true>(p) : synth_block<T, false>(p);
  const long long nxb = blk ? (p->nx + blk - 1) / blk * blk : p->nx;
  const size_t fb = sizeof(C) * (size_t)p->nrows * nxb;
  C* t1 = (C*)p->ws_get("tf.t1", fb, &st);
  if (st) return st;
  st = omega_fft_any<Tin, T>(p, Fint, t1, true, s, blk);
  if (st) return st;
  if (complex_out) return synth_any<T, true>(p, t1, f, s);
  return synth_any<T, false>(p, t1, f, s);
}

template <typename T>
static int backward_T(hp_plan* p, const double2* Fint, void* f, int complex_out, cudaStream_t s) {
  return backward_rows<double, T>(p, Fint, f, complex_out, s);
}

// Forward transform of (mult .) f into [row][omega] coefficients of type c2<T>.
template <typename T, bool CPLX>
static int anal2_any(hp_plan* p, const void* f, const double* mult, c2<T>* out, cudaStream_t s) {
  switch (p->B) {
#define X(b) case b: return anal2_launch<b, T, CPLX>(p, f, mult, out, s);
    HP_FOR_EACH_B(X)
#undef X
    default:
      hp_set_error("bandlimit B not supported (2..32)");
      return HP_ERR_UNSUPPORTED;
  }
}

template <typename T>
static int forward_rows_T(hp_plan* p, const void* f, int complex_in, const double* mult, c2<T>* out,
                          cudaStream_t s) {
  using C = c2<T>;
  int st = HP_OK;
  const size_t fb = sizeof(C) * (size_t)p->nrows * p->nx;
  C* t1 = (C*)p->ws_get("tf.t1", fb, &st);
  if (st) return st;
  C* t2 = (C*)p->ws_get("tf.t2", fb, &st);
  if (st) return st;
  (void)t1;
  st = complex_in ? anal2_any<T, true>(p, f, mult, t2, s) : anal2_any<T, false>(p, f, mult, t2, s);
  if (st) return st;
  return omega_fft_any<T, T>(p, t2, out, false, s);
}

template <typename T>
static int forward_T(hp_plan* p, const void* f, int complex_in, double2* Fint, cudaStream_t s) {
  using C = c2<T>;
  int st = HP_OK;
  C* t3 = (C*)p->ws_get("tf.t1", sizeof(C) * (size_t)p->nrows * p->nx, &st);  // free again after the transpose
  if (st) return st;
  st = forward_rows_T<T>(p, f, complex_in, nullptr, t3, s);
  if (st) return st;
  // to FP64 rows
  const long long n = p->nrows * p->nx;
  ProfScope _ps(p, "convert", s);
  k_to_c64<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(t3, Fint, n);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

int hp_backward_internal(hp_plan* p, const double2* Fint, void* f, int complex_out, cudaStream_t s) {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  if (p->precision == HP_FP64) return backward_T<double>(p, Fint, f, complex_out, s);
  return backward_T<float>(p, Fint, f, complex_out, s);
}

int hp_backward_internal32(hp_plan* p, const float2* Fint32, void* f, int complex_out, cudaStream_t s) {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  if (p->precision != HP_MIXED) { hp_set_error("FP32 coefficients need a mixed-precision plan"); return HP_ERR_INVALID; }
  return backward_rows<float, float>(p, Fint32, f, complex_out, s);
}

int hp_forward_internal(hp_plan* p, const void* f, int complex_in, double2* Fint, cudaStream_t s) {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  if (p->precision == HP_FP64) return forward_T<double>(p, f, complex_in, Fint, s);
  return forward_T<float>(p, f, complex_in, Fint, s);
}

int hp_forward_internal_T(hp_plan* p, const void* f, const double* mult, void* out, cudaStream_t s) {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  const int cplx = p->symmetry == HP_COMPLEX;
  if (p->precision == HP_FP64) return forward_rows_T<double>(p, f, cplx, mult, (double2*)out, s);
  return forward_rows_T<float>(p, f, cplx, mult, (float2*)out, s);
}

// Forward transform in FP64 whatever the plan's precision (initial densities).
int hp_forward_internal64(hp_plan* p, const double* f, double2* Fint, cudaStream_t s) {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  return forward_T<double>(p, f, 0, Fint, s);   // real density, HP_REAL plans
}

// Omega FFTs of all rows for the derivative's large-grid path (compute precision).
int hp_omega_ifft_rows(hp_plan* p, const double2* in, void* out, cudaStream_t s) {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  if (p->precision == HP_FP64) return omega_fft_any<double, double>(p, in, (double2*)out, true, s);
  return omega_fft_any<double, float>(p, in, (float2*)out, true, s);
}
int hp_omega_fft_rows(hp_plan* p, void* inout, cudaStream_t s) {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  if (p->precision == HP_FP64) return omega_fft_any<double, double>(p, (double2*)inout, (double2*)inout, false, s);
  return omega_fft_any<float, float>(p, (float2*)inout, (float2*)inout, false, s);
}
