// Common device/host helpers for the SO(3) x R^n Fokker-Planck kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/hp.h"

#define HP_CUDA_TRY(expr)                                                     \
  do {                                                                        \
    cudaError_t _e = (expr);                                                  \
    if (_e != cudaSuccess) {                                                  \
      hp_set_error(cudaGetErrorString(_e));                                   \
      return _e == cudaErrorMemoryAllocation ? HP_ERR_ALLOC : HP_ERR_CUDA;    \
    }                                                                         \
  } while (0)

void hp_set_error(const char* msg);

// Every device allocation of the library goes through these two, so that the
// process-wide budget of hp_set_device_budget applies to all of them: beyond
// the budget hp_dev_alloc fails with cudaErrorMemoryAllocation, as cudaMalloc
// does when the device is full.
cudaError_t hp_dev_alloc_raw(void** p, size_t bytes);
cudaError_t hp_dev_free(void* p);
template <typename T> inline cudaError_t hp_dev_alloc(T** p, size_t bytes) {
  return hp_dev_alloc_raw(reinterpret_cast<void**>(p), bytes);
}

namespace hp {

// ------------------------------------------------------------- complex ----
template <typename T> struct C2T;
template <> struct C2T<double> { using type = double2; };
template <> struct C2T<float> { using type = float2; };
template <typename T> using c2 = typename C2T<T>::type;

__host__ __device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__host__ __device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a + b * c
__device__ __forceinline__ double2 cfma(double2 b, double2 c, double2 a) {
  return make_double2(fma(b.x, c.x, fma(-b.y, c.y, a.x)), fma(b.x, c.y, fma(b.y, c.x, a.y)));
}
__device__ __forceinline__ float2 cfma(float2 b, float2 c, float2 a) {
  return make_float2(fmaf(b.x, c.x, fmaf(-b.y, c.y, a.x)), fmaf(b.x, c.y, fmaf(b.y, c.x, a.y)));
}
// i * a
template <typename C> __device__ __forceinline__ C cI(C a) { C r; r.x = -a.y; r.y = a.x; return r; }
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }

template <typename Cout, typename Cin> __device__ __forceinline__ Cout cvt(Cin a);
template <> __device__ __forceinline__ double2 cvt<double2, double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 cvt<float2, float2>(float2 a) { return a; }
template <> __device__ __forceinline__ float2 cvt<float2, double2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __device__ __forceinline__ double2 cvt<double2, float2>(float2 a) { return make_double2(a.x, a.y); }

template <typename C> __device__ __forceinline__ C czero() { C r; r.x = 0; r.y = 0; return r; }

// ------------------------------------------------------------ sizes ----
// Kernels are instantiated per bandlimit B (2..32) and per omega grid size N
// (even, 4..64; the plane kernels of the derivative for N <= 32).
#define HP_FOR_EACH_B(X) \
  X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) X(19) X(20) \
  X(21) X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31) X(32)
#define HP_FOR_EACH_N_TO_32(X) \
  X(4) X(6) X(8) X(10) X(12) X(14) X(16) X(18) X(20) X(22) X(24) X(26) X(28) X(30) X(32)
#define HP_FOR_EACH_N_ABOVE_32(X) \
  X(34) X(36) X(38) X(40) X(42) X(44) X(46) X(48) X(50) X(52) X(54) X(56) X(58) X(60) X(62) X(64)
#define HP_FOR_EACH_N(X) HP_FOR_EACH_N_TO_32(X) HP_FOR_EACH_N_ABOVE_32(X)

// ------------------------------------------------------------ twiddles ----
// Entries 0..959: W[k] = exp(-2 pi i k / 960), the twiddles of every length
// that divides 960 (all the 2/3/5 sizes).  Then one section per other length
// M that an FFT of at most 64 points can need (M <= 64 not dividing 960, even
// or at most 32): W_M^e, e = 0..M-1.  Each translation unit holds its own copy
// (no relocatable device code) and fills it once per device with tw_init()
// before its first launch.
constexpr int kTw960 = 960;
constexpr int kTwMaxM = 64;
__host__ __device__ constexpr bool tw_own_section(int M) {
  return kTw960 % M != 0 && (M % 2 == 0 || M <= 32);
}
__host__ __device__ constexpr int tw_section(int M) {   // first entry of length M's section
  int o = kTw960;
  for (int m = 1; m < M; ++m) o += tw_own_section(m) ? m : 0;
  return o;
}
constexpr int kTwN = tw_section(kTwMaxM + 1);
static __constant__ double2 c_tw64[kTwN];
static __constant__ float2 c_tw32[kTwN];

int tw_fill_host(double2* t64, float2* t32);  // defined in tables.cu

static inline int tw_init() {
  static unsigned long long done_mask = 0ULL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 4;
  if (dev < 64 && (done_mask >> dev) & 1ULL) return 0;
  static double2 t64[kTwN];
  static float2 t32[kTwN];
  tw_fill_host(t64, t32);
  if (cudaMemcpyToSymbol(c_tw64, t64, sizeof(t64)) != cudaSuccess) return 4;
  if (cudaMemcpyToSymbol(c_tw32, t32, sizeof(t32)) != cudaSuccess) return 4;
  if (dev < 64) done_mask |= 1ULL << dev;
  return 0;
}

template <typename C> __device__ __forceinline__ C tw_load(int idx);
template <> __device__ __forceinline__ double2 tw_load<double2>(int idx) { return c_tw64[idx]; }
template <> __device__ __forceinline__ float2 tw_load<float2>(int idx) { return c_tw32[idx]; }

// exp(-+ 2 pi i e / M) (INV selects +), e >= 0.  Lengths dividing 960 read
// the shared 960-entry part (equal twiddles of different lengths, W_8^1 and
// W_32^4, are one entry), the others their own section.
template <typename C, bool INV, int M>
__device__ __forceinline__ C twiddle(int e) {
  static_assert(M >= 1 && M <= kTwMaxM && (kTw960 % M == 0 || tw_own_section(M)), "twiddle length");
  int idx;
  if constexpr (kTw960 % M == 0) {
    idx = ((e % M) * (kTw960 / M)) % kTw960;
  } else {
    constexpr int off = tw_section(M);
    idx = off + e % M;
  }
  C w = tw_load<C>(idx);
  if (INV) w.y = -w.y;
  return w;
}

// ------------------------------------------------ asynchronous smem fill ----
// cp.async of one element (8 or 16 bytes) from global to shared memory without
// a register round trip; src_bytes = 0 writes zeros (the source is not read).
// Completion: cp_async_wait_all() by the issuing thread, then a block barrier.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, bool valid) {
  static_assert(BYTES == 8 || BYTES == 16, "cp.async of 8 or 16 bytes");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int nb = valid ? BYTES : 0;
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(nb) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(nb) : "memory");
}
// the same with an explicit source byte count (0..BYTES; the rest zero-filled)
__device__ __forceinline__ void cp_async16_n(void* smem, const void* gmem, int nbytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(nbytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// ------------------------------------------------------ L2 cache hints ----
// Streams written once and read only by a later kernel (density, updated
// coefficients) are stored with an evict-first L2 policy, so that they do not
// push out lines that blocks running at the same time still read (the
// synthesis blocks of one omega chunk share their coefficient rows, the plane
// tiles of one row their halo rows).
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void st_evict_first(double2* a, double2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(a), "d"(v.x), "d"(v.y), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_evict_first(float2* a, float2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(a), "f"(v.x), "f"(v.y), "l"(pol) : "memory");
}

// ------------------------------------------------- register-resident FFT ----
// Small DFT of radix R in registers (out-of-place on v).
template <int R, bool INV, typename C>
__device__ __forceinline__ void dft_small(C (&v)[R]) {
  if constexpr (R == 2) {
    C a = v[0], b = v[1];
    v[0] = a + b; v[1] = a - b;
  } else if constexpr (R == 4) {
    C t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3], t3 = v[1] - v[3];
    // forward: multiply t3 by -i ; inverse: by +i
    C t3r;
    if (INV) { t3r.x = -t3.y; t3r.y = t3.x; } else { t3r.x = t3.y; t3r.y = -t3.x; }
    v[0] = t0 + t2; v[2] = t0 - t2; v[1] = t1 + t3r; v[3] = t1 - t3r;
  } else if constexpr (R == 3) {
    // y0 = x0 + s, y1,2 = x0 - s/2 -+ i (sqrt3/2) d  (forward), s = x1 + x2, d = x1 - x2
    using T = decltype(v[0].x);
    const T h = (T)0.86602540378443864676;  // sin(pi/3)
    C s = v[1] + v[2], d = v[1] - v[2];
    C a;
    a.x = v[0].x - (T)0.5 * s.x;
    a.y = v[0].y - (T)0.5 * s.y;
    C t;  // -i h d (forward) or +i h d (inverse)
    if (INV) { t.x = -h * d.y; t.y = h * d.x; } else { t.x = h * d.y; t.y = -h * d.x; }
    v[0] = v[0] + s;
    v[1] = a + t;
    v[2] = a - t;
  } else if constexpr (R == 5) {
    using T = decltype(v[0].x);
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    const C s14 = v[1] + v[4], d14 = v[1] - v[4], s23 = v[2] + v[3], d23 = v[2] - v[3];
    C a1, a2, b1, b2;
    a1.x = v[0].x + c1 * s14.x + c2 * s23.x;  a1.y = v[0].y + c1 * s14.y + c2 * s23.y;
    a2.x = v[0].x + c2 * s14.x + c1 * s23.x;  a2.y = v[0].y + c2 * s14.y + c1 * s23.y;
    b1.x = s1 * d14.x + s2 * d23.x;            b1.y = s1 * d14.y + s2 * d23.y;
    b2.x = s2 * d14.x - s1 * d23.x;            b2.y = s2 * d14.y - s1 * d23.y;
    // forward: y1 = a1 - i b1, y4 = a1 + i b1, y2 = a2 - i b2, y3 = a2 + i b2
    C ib1, ib2;
    if (INV) { ib1.x = b1.y; ib1.y = -b1.x; ib2.x = b2.y; ib2.y = -b2.x; }   // -(i b)
    else { ib1.x = -b1.y; ib1.y = b1.x; ib2.x = -b2.y; ib2.y = b2.x; }      // +(i b)
    v[0] = v[0] + s14 + s23;
    v[1] = a1 - ib1;
    v[4] = a1 + ib1;
    v[2] = a2 - ib2;
    v[3] = a2 + ib2;
  } else {
    // any other prime factor (7, 11, ..., 31: bandlimits and grids off the
    // 2/3/5 sizes): a direct DFT, its outer loop kept rolled so that the code
    // stays small (the outputs go through a local array)
    C o[R];
#pragma unroll 1
    for (int q = 0; q < R; ++q) {
      C acc = v[0];
      int e = q;   // r q mod R
#pragma unroll
      for (int r = 1; r < R; ++r) {
        acc = cfma(v[r], twiddle<C, INV, R>(e), acc);
        e = e + q >= R ? e + q - R : e + q;
      }
      o[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = o[q];
  }
}

template <int N, int Ns>
struct FftRadix {
  static constexpr int rem = N / Ns;
  static constexpr int value = (rem % 4 == 0) ? 4 : (rem % 2 == 0 ? 2 : (rem % 3 == 0 ? 3 : (rem % 5 == 0 ? 5 : rem)));
};

// Stockham self-sorting FFT stages: unnormalised, X[k] = sum_j x[j] exp(-+2 pi i jk/N).
template <int N, int Ns, bool INV, typename C>
__device__ __forceinline__ void fft_stages(C (&x)[N]) {
  if constexpr (Ns < N) {
    constexpr int R = FftRadix<N, Ns>::value;
    C y[N];
#pragma unroll
    for (int j = 0; j < N / R; ++j) {
      const int k = j % Ns;
      C v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = x[j + r * (N / R)];
#pragma unroll
      for (int r = 1; r < R; ++r)
        if ((r * k) % (Ns * R) != 0) v[r] = cmul(v[r], twiddle<C, INV, Ns * R>(r * k));
      dft_small<R, INV>(v);
      const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) y[idxD + r * Ns] = v[r];
    }
#pragma unroll
    for (int i = 0; i < N; ++i) x[i] = y[i];
    fft_stages<N, Ns * R, INV>(x);
  }
}

// Prime-factor (Good-Thomas) FFT for N = N1 N2 N3 with pairwise coprime
// factors, no twiddle multiplies.  Input map n = (N/N1 n1 + N/N2 n2 + N/N3 n3)
// mod N; output map k = (M1 k1 + M2 k2 + M3 k3) mod N with Mi = N/Ni times the
// inverse of N/Ni modulo Ni (Chinese remainder), so that
// nk = (N/N1)M1 n1k1 + ... = N/N1 n1k1 + ... (mod N) and the N-point DFT is an
// N1 x N2 x N3 DFT over (n1, n2, n3); both maps are register permutations.
// Used for N = 30 (2*3*5, the 2B-point FFTs of B = 15) and N = 60 (4*3*5).
template <int A, int M> constexpr int inv_mod() {
  int r = 1;
  while ((A % M) * r % M != 1) ++r;
  return r;
}
template <int N1, int N2, int N3, bool INV, typename C>
__device__ __forceinline__ void fft_pfa3(C (&x)[N1 * N2 * N3]) {
  constexpr int N = N1 * N2 * N3;
  constexpr int Q1 = N / N1, Q2 = N / N2, Q3 = N / N3;
  constexpr int M1 = Q1 * inv_mod<Q1, N1>(), M2 = Q2 * inv_mod<Q2, N2>(), M3 = Q3 * inv_mod<Q3, N3>();
#pragma unroll
  for (int a = 0; a < N1 * N2; ++a) {   // length-N3 DFTs along n3
    const int n1 = a / N2, n2 = a % N2;
    C v[N3];
#pragma unroll
    for (int r = 0; r < N3; ++r) v[r] = x[(Q1 * n1 + Q2 * n2 + Q3 * r) % N];
    dft_small<N3, INV>(v);
#pragma unroll
    for (int r = 0; r < N3; ++r) x[(Q1 * n1 + Q2 * n2 + Q3 * r) % N] = v[r];
  }
  // x now holds, at input position (n1, n2, k3), the partial result; continue in place
#pragma unroll
  for (int a = 0; a < N1 * N3; ++a) {   // length-N2 DFTs along n2
    const int n1 = a / N3, k3 = a % N3;
    C v[N2];
#pragma unroll
    for (int r = 0; r < N2; ++r) v[r] = x[(Q1 * n1 + Q2 * r + Q3 * k3) % N];
    dft_small<N2, INV>(v);
#pragma unroll
    for (int r = 0; r < N2; ++r) x[(Q1 * n1 + Q2 * r + Q3 * k3) % N] = v[r];
  }
#pragma unroll
  for (int a = 0; a < N2 * N3; ++a) {   // length-N1 DFTs along n1
    const int k2 = a / N3, k3 = a % N3;
    C v[N1];
#pragma unroll
    for (int r = 0; r < N1; ++r) v[r] = x[(Q1 * r + Q2 * k2 + Q3 * k3) % N];
    dft_small<N1, INV>(v);
#pragma unroll
    for (int r = 0; r < N1; ++r) x[(Q1 * r + Q2 * k2 + Q3 * k3) % N] = v[r];
  }
  // result (k1, k2, k3) sits at input position (Q1 k1 + Q2 k2 + Q3 k3) % N and
  // belongs at output position (M1 k1 + M2 k2 + M3 k3) % N
  C y[N];
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2)
#pragma unroll
      for (int k3 = 0; k3 < N3; ++k3) y[(M1 * k1 + M2 * k2 + M3 * k3) % N] = x[(Q1 * k1 + Q2 * k2 + Q3 * k3) % N];
#pragma unroll
  for (int i = 0; i < N; ++i) x[i] = y[i];
}

template <int N, bool INV, typename C>
__device__ __forceinline__ void fft(C (&x)[N]) {
  if constexpr (N == 30) fft_pfa3<2, 3, 5, INV>(x);
  else if constexpr (N == 60) fft_pfa3<4, 3, 5, INV>(x);
  else fft_stages<N, 1, INV>(x);
}

// 2H-point DFT over a lane pair: lanes 2t and 2t+1 of a warp (threadIdx.x of
// a 1-D block) hold the same transform, lane h = threadIdx.x & 1 the inputs
// x[j] = input[2j + h], j < H.  Each lane transforms its half (even or odd
// samples), the odd half is twisted by W_2H^k, and one exchange by shuffles
// finishes the radix-2 step: on return lane h holds output[h H + k], k < H.
// The shuffles name the two lanes of the pair only, so pairs of one warp may
// take different paths; both lanes of a pair must call it together.
template <int H, bool INV, typename C>
__device__ __forceinline__ void fft_lane_pair(C (&x)[H], int h) {
  using T = decltype(x[0].x);
  const unsigned pm = 3u << (threadIdx.x & 30u);
  fft<H, INV>(x);
#pragma unroll
  for (int k = 1; k < H; ++k) {
    const C t = cmul(x[k], twiddle<C, INV, 2 * H>(k));
    x[k].x = h ? t.x : x[k].x;
    x[k].y = h ? t.y : x[k].y;
  }
  // lane 0 (even half E): E + W O ; lane 1 (holding W O, receiving E): E - W O
  const T sg = h ? (T)-1 : (T)1;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    const T ox = __shfl_xor_sync(pm, x[k].x, 1);
    const T oy = __shfl_xor_sync(pm, x[k].y, 1);
    x[k].x = fma(sg, x[k].x, ox);
    x[k].y = fma(sg, x[k].y, oy);
  }
}

// Fourier index k (FFT order) -> signed wavenumber with the Nyquist bin zeroed
// (the 2 pi i [0:Bx-1, 0, -Bx+1:-1] / L multiplier of the first derivative).
__host__ __device__ __forceinline__ int kappa_first(int k, int N) {
  return (k < N / 2) ? k : (k == N / 2 ? 0 : k - N);
}
// Signed wavenumber keeping the Nyquist bin as -N/2 (the diagonal diffusion term).
__host__ __device__ __forceinline__ int kappa_diag(int k, int N) { return (k < N / 2) ? k : k - N; }

}  // namespace hp
