// Pendulum Fokker-Planck derivative and integrator update on the internal
// coefficient layout (see plan.hpp).
//
// The reference forms every Omega-dependent term as an O(nx^2) circular
// convolution with X, bX or OJO (pendulum.m:396-466).  Here the same operators
// are applied exactly as 1-D maps along the omega axes: multiplication by the
// grid coordinate x_i in physical space is
//     M_i F = FFT_i( x_i . IFFT_i F )      (== (1/N) X_i (*) F along axis i),
// so with P3 = M_3 F the derivative is
//   dF = -(M_1F)u_1^T - (M_2F)u_2^T - (M_3F)u_3^T            Lie term   (pendulum.m:396-422)
//        + sum_i b_i D_i M_i F                               damping    (pendulum.m:424-446)
//        - g_1 D_1 M_2 P3 - g_2 D_2 M_1 P3 - g_3 D_3 M_1 M_2 F   gyroscopic (pendulum.m:448-466)
//        - sum_i D_i Grav_i(F)                               gravity    (pendulum.m:470-506)
//        + sum_ij G_ij c_ij F                                diffusion  (pendulum.m:510-523)
// with D_i = 2 pi i kappa_i / L (Nyquist zeroed) and (g_1, g_2, g_3) the
// coefficients of J^-1(-x cross Jx) = (g_1 x2 x3, g_2 x1 x3, g_3 x1 x2).
//
// Three passes (ndim = 3):
//   k_axis3   : P3 = M_3 F            (lines along k3, one thread per line, registers only)
//   k_local   : G  = gravity + noise  (pointwise in omega, all rows of an m group)
//   k_plane   : 2-D (k1, k2) work of every remaining term on one k3 plane of a
//               tile of n-consecutive rows, then out = F0 + a dF (+ acc += b dF).
// For ndim = 2 the plane pass covers the whole omega grid and k_axis3 is skipped.
#include <algorithm>
#include <atomic>
#include <vector>
#include "common.cuh"
#include "plan.hpp"

using namespace hp;

#define ST_CHECK(expr)          \
  do {                          \
    int _s = (expr);            \
    if (_s != HP_OK) return _s; \
  } while (0)

#define HP_CHECK_RET(expr)          \
  do {                              \
    int _s = (expr);                \
    if (_s != HP_OK) return _s;     \
  } while (0)


// -------------------------------------------------------- pass A: axis 3 ----
// Fc (may be null): the coefficients themselves in the compute precision, the
// input the local and plane passes then read instead of the FP64 state.  With
// TIN = T the input already is that copy (written by the previous step's plane
// pass) and Fc is null.
template <int N, typename T, typename TIN = double>
__global__ void __launch_bounds__(128) k_axis3(RowLayout L, const c2<TIN>* __restrict__ F,
                                               c2<T>* __restrict__ P3, T Llen, c2<T>* __restrict__ Fc) {
  using C = c2<T>;
  constexpr long long plane = (long long)N * N;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.nrows * plane) return;
  const long long row = t / plane, p = t % plane;
  const c2<TIN>* src = F + row * L.nx + p;
  C x[N];
#pragma unroll
  for (int j = 0; j < N; ++j) x[j] = cvt<C, c2<TIN>>(__ldg(src + j * plane));
  if (Fc) {
    C* fc = Fc + row * L.nx + p;
#pragma unroll
    for (int j = 0; j < N; ++j) fc[j * plane] = x[j];
  }
  fft<N, true>(x);
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const T xc = (-Llen / 2 + Llen * (T)j / (T)N) / (T)N;
    x[j] = xc * x[j];
  }
  fft<N, false>(x);
  C* dst = P3 + row * L.nx + p;
#pragma unroll
  for (int j = 0; j < N; ++j) dst[j * plane] = x[j];
}

// ------------------------------------------------ pass B: gravity + noise ----
// Block = one m group x cpb chunks of W consecutive omega points.  The
// group's real tap weights and tap sources are staged once per block, its
// rows once per chunk, in shared memory (taps stay inside the group because
// the gravity multiplier has m2 = 0); a warp handles one
// output row at a time, lanes are omega points, so the tap loop is
// warp-uniform and reads shared memory only.  Per omega point the model part
// of the weights folds into nu[n2] = -i sum_i D_i gs_i MR_i^1_{0 n2}, so
//   G = noise F + sum_{n2} nu[n2] sum_{l1} w(l1, n2) F^{l1}_{m, n-n2}.
template <typename T> __host__ __device__ constexpr size_t local_tile_bytes(int rmax, int W) {
  return ((size_t)rmax * W * sizeof(c2<T>) + 15) / 16 * 16;
}

template <typename T, int W, int NDIM, typename TIN>
__global__ void __launch_bounds__(256) k_local(RowLayout L, const c2<TIN>* __restrict__ F,
                                               c2<T>* __restrict__ G, const T* __restrict__ tap_wr,
                                               const c2<T>* __restrict__ Gx, const c2<T>* __restrict__ sdk,
                                               DerivParams prm, int cpb) {
  using C = c2<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int D = 2 * L.lmax + 1;
  const int rmax = (L.lmax + 1) * (L.lmax + 1);
  C* tile = reinterpret_cast<C*>(smraw);                                          // [R][W]
  T* sw = reinterpret_cast<T*>(smraw + local_tile_bytes<T>(rmax, W));             // [R][9]
  int* sseg = reinterpret_cast<int*>(smraw + local_tile_bytes<T>(rmax, W) +
                                     ((size_t)rmax * 9 * sizeof(T) + 15) / 16 * 16);  // [D]
  short* ssrc = reinterpret_cast<short*>(sseg + (D + 3) / 4 * 4);                 // [R][9]
  const int m = (int)blockIdx.y + L.m_lo;
  const int r0 = L.seg[(m - L.m_lo) * D];
  const int r1 = (m + 1 <= L.lmax) ? L.seg[(m + 1 - L.m_lo) * D] : (int)L.nrows;
  const int R = r1 - r0;
  const int tid = threadIdx.x, nth = blockDim.x;
  // per block, once for its cpb omega chunks: the group's tap weights and tap
  // sources
  for (int e = tid; e < R * 9; e += nth) sw[e] = tap_wr[(size_t)r0 * 9 + e];
  for (int e = tid; e < D; e += nth) sseg[e] = L.seg[(m - L.m_lo) * D + e] - r0;
  // tap t = (l1 - l + 1) * 3 + (n2 + 1) of row r reads group row ssrc[r][t]
  // (row 0 where the tap has no weight), so the tap loop below has no branches
  const int am = abs(m), lmax = L.lmax;
  for (int e = tid; e < R * 9; e += nth) {
    const char4 q = L.rows[r0 + e / 9];
    const int t = e % 9, l1 = q.x + t / 3 - 1, n1 = q.z - (t % 3 - 1), an1 = abs(n1);
    int src = 0;
    if (l1 >= 0 && l1 <= lmax && am <= l1 && an1 <= l1)
      src = L.seg[(m - L.m_lo) * D + n1 + lmax] - r0 + l1 - (am > an1 ? am : an1);
    ssrc[e] = (short)src;
  }
  const int N = L.N;
  const T tp = (T)(2.0 * M_PI / prm.L);
  const int w = tid % W, rl = tid / W, nrl = nth / W;
  const long long nchunks = (L.nx + W - 1) / W;
  const long long ch0 = (long long)blockIdx.x * cpb;
  const long long ch1 = ch0 + cpb < nchunks ? ch0 + cpb : nchunks;
  for (long long ch = ch0; ch < ch1; ++ch) {
    const long long w0 = ch * W;
    __syncthreads();   // the previous chunk's reads of the tile are done
    // group rows staged with 8 loads in flight per thread (asynchronous copies
    // into the tile measured no faster here)
    for (int e0 = tid; e0 < R * W; e0 += 8 * nth) {
      C v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * nth;
        const int r = e / W, ww = e % W;
        v[u] = (e < R * W && w0 + ww < L.nx) ? cvt<C, c2<TIN>>(F[(size_t)(r0 + r) * L.nx + w0 + ww]) : czero<C>();
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * nth;
        if (e < R * W) tile[e] = v[u];
      }
    }
    __syncthreads();
    if (ch + 1 < ch1) {   // the next chunk's rows into L2 while this one computes
      constexpr int EPL = 128 / (int)sizeof(c2<TIN>);           // elements per 128-byte line
      constexpr int LPR = (W + EPL - 1) / EPL;                   // lines per row segment
      const long long w1 = w0 + W;
      for (int e = tid; e < R * LPR; e += nth) {
        const long long ww = w1 + (long long)(e % LPR) * EPL;
        if (ww < L.nx) asm volatile("prefetch.global.L2 [%0];" ::"l"(F + (size_t)(r0 + e / LPR) * L.nx + ww));
      }
    }
    const long long wg = w0 + w;
    if (wg >= L.nx) continue;
    T d1[NDIM], dd[NDIM];
    {
      long long ww = wg;
#pragma unroll
      for (int a = 0; a < NDIM; ++a) {
        const int k = (int)(ww % N);
        ww /= N;
        d1[a] = tp * (T)kappa_first(k, N);
        dd[a] = tp * (T)kappa_diag(k, N);
      }
    }
    T noise = 0;
#pragma unroll
    for (int i = 0; i < NDIM; ++i)
#pragma unroll
      for (int j = 0; j < NDIM; ++j)
        noise -= (T)prm.G[i * 3 + j] * ((i == j) ? dd[i] * dd[i] : d1[i] * d1[j]);
    C nu[3];  // -i sum_i d1_i gs_i MR_i^1_{0 n2}
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      T mx = 0, my = 0;
#pragma unroll
      for (int i = 0; i < NDIM; ++i) {
        const T s = d1[i] * (T)prm.gs[i];
        mx += s * (T)prm.mr[q][i][0];
        my += s * (T)prm.mr[q][i][1];
      }
      nu[q].x = my;
      nu[q].y = -mx;
    }
    for (int r = rl; r < R; r += nrl) {
      const C f0 = tile[r * W + w];
      T ax = noise * f0.x, ay = noise * f0.y;
#pragma unroll
      for (int n2o = 0; n2o < 3; ++n2o) {
        T sx = 0, sy = 0;
#pragma unroll
        for (int l1o = 0; l1o < 3; ++l1o) {
          const int t = r * 9 + l1o * 3 + n2o;
          const T wt = sw[t];
          const C fs = tile[ssrc[t] * W + w];
          sx = fma(wt, fs.x, sx);
          sy = fma(wt, fs.y, sy);
        }
        ax += nu[n2o].x * sx - nu[n2o].y * sy;
        ay += nu[n2o].x * sy + nu[n2o].y * sx;
      }
      if (sdk) {  // attitude diffusion: sum_o K^l[n][n+o-2] F^l_{m, n+o-2} (gyro-bias model)
        const char4 q = L.rows[r0 + r];
        const int l = q.x, n = q.z;
        const c2<T>* kw = sdk + (size_t)(r0 + r) * 5;
#pragma unroll
        for (int o = 0; o < 5; ++o) {
          const int k = n + o - 2;
          if (k < -l || k > l) continue;
          const int ak = abs(k);
          const C fs = tile[(sseg[k + lmax] - (am > ak ? am : ak) + l) * W + w];
          const C wk = kw[o];
          ax += wk.x * fs.x - wk.y * fs.y;
          ay += wk.x * fs.y + wk.y * fs.x;
        }
      }
      if (Gx) {  // density-side gravity term (density-gravity models)
        const C gx = Gx[(size_t)(r0 + r) * L.nx + wg];
        ax += gx.x;
        ay += gx.y;
      }
      C o;
      o.x = ax;
      o.y = ay;
      G[(size_t)(r0 + r) * L.nx + wg] = o;
    }
  }
}

template <typename T> static size_t local_smem(const hp_plan* p, int W) {
  const int rmax = (p->lmax + 1) * (p->lmax + 1);
  return local_tile_bytes<T>(rmax, W) + ((size_t)rmax * 9 * sizeof(T) + 15) / 16 * 16 +
         sizeof(int) * ((p->D + 3) / 4 * 4) + sizeof(short) * (size_t)rmax * 9;
}
template <typename T> static const T* tap_table(const hp_plan* p);
template <> const double* tap_table<double>(const hp_plan* p) { return p->tap_wr; }
template <> const float* tap_table<float>(const hp_plan* p) { return p->tap_wr32; }
template <typename T> static const c2<T>* so3d_table(const hp_plan* p);
template <> const double2* so3d_table<double>(const hp_plan* p) { return p->so3d64; }
template <> const float2* so3d_table<float>(const hp_plan* p) { return p->so3d32; }

template <typename T> static constexpr int local_w() { return sizeof(T) == 8 ? 16 : 32; }

// --------------------------------------------------- pass C: plane pass ----

template <typename T> struct PlaneCfg;
template <> struct PlaneCfg<double> { static constexpr int C = 1; static constexpr int NT = 128; static constexpr int MINB = 2; };
template <> struct PlaneCfg<float> { static constexpr int C = 2; static constexpr int NT = 256; static constexpr int MINB = 2; };

__device__ __forceinline__ long long row_of(const RowLayout& L, int l, int m, int n) {
  const int am = abs(m), an = abs(n);
  return L.seg[(m - L.m_lo) * (2 * L.lmax + 1) + n + L.lmax] + l - (am > an ? am : an);
}

// smem planes (stride PS = N*(N+1)):
//   [0, C+2)           F~ rows n0-1 .. n0+C     (physical after the inverse FFTs)
//   [C+2, 2C+2)        P~ rows n0 .. n0+C-1     (ndim = 3)
//   [2C+2, 3C+2)       A  = FFT2(Y0) + D_2 FFT2(Y2), then FFT_1
//   [3C+2, 4C+2)       Y1' = FFT_2(Y1), then D_1 FFT_1
// One tile (tl) on one k3 plane: the body of k_plane, also run by the
// persistent batched plane pass (k_plane_batch) for tiles of many members.
template <int N, typename T, bool HAS_P3, typename TIN>
__device__ __forceinline__ void plane_body(const RowLayout& L, const PlaneTile tl, const int k3,
                                           const c2<TIN>* __restrict__ Fev, const c2<T>* __restrict__ P3,
                                           const c2<T>* __restrict__ Gl, const double2* __restrict__ F0, double a,
                                           double2* __restrict__ out, double2* __restrict__ acc, double bacc,
                                           const DerivParams& prm, c2<T>* __restrict__ out32, unsigned char* smraw) {
  using C = c2<T>;
  constexpr int CT = PlaneCfg<T>::C;
  constexpr int PS = N * (N + 1);
  constexpr int NP = HAS_P3 ? CT : 0;
  C* sm = reinterpret_cast<C*>(smraw);
  C* sF = sm;
  C* sP = sm + (CT + 2) * PS;
  C* sA = sm + (CT + 2 + NP) * PS;
  C* sY = sm + (CT + 2 + NP + CT) * PS;

  const long long pbase = (long long)k3 * N * N;  // plane offset inside a row
  const int tid = threadIdx.x, nth = blockDim.x;
  const T Ll = (T)prm.L;
  const T tp = (T)(2.0 * M_PI / prm.L);
  const T inv_n2 = (T)1 / (T)(N * N);

  // ---- S1: load F rows n0-1 .. n0+cnt and P3 rows n0 .. n0+cnt-1 ----
  // Input already in the compute precision: asynchronous copies straight into
  // the padded planes (every element's copy in flight at once, no register
  // staging; rows outside -l..l are zero-filled).  FP64 input of an FP32 plan:
  // loads in batches of 8 per thread, converted, then stored.
  const int nF = tl.cnt + 2;
  // element offsets of the tile's output rows in this plane, for S6
  __shared__ long long s_rb[CT];
  if (tid < CT) s_rb[tid] = tid < tl.cnt ? row_of(L, tl.l, tl.m, tl.n0 + tid) * L.nx + pbase : 0;
  if constexpr (sizeof(TIN) == sizeof(T)) {
    // one source row per loaded plane: its address once, then the plane's
    // N^2 elements (rows outside -l..l zero-filled)
    for (int sl = 0; sl < nF; ++sl) {
      const int n = tl.n0 - 1 + sl;
      const bool ok = n >= -tl.l && n <= tl.l;
      const c2<TIN>* src = ok ? Fev + row_of(L, tl.l, tl.m, n) * L.nx + pbase : Fev;
      C* dst = sF + sl * PS;
      for (int q = tid; q < N * N; q += nth) cp_async<sizeof(C)>(dst + (q / N) * (N + 1) + q % N, src + (ok ? q : 0), ok);
    }
    if (HAS_P3) {
      for (int sl = 0; sl < tl.cnt; ++sl) {
        const c2<T>* src = P3 + row_of(L, tl.l, tl.m, tl.n0 + sl) * L.nx + pbase;
        C* dst = sP + sl * PS;
        for (int q = tid; q < N * N; q += nth) cp_async<sizeof(C)>(dst + (q / N) * (N + 1) + q % N, src + q, true);
      }
    }
    cp_async_wait_all();
  } else {
    const int tot = nF * N * N;
    for (int e0 = tid; e0 < tot; e0 += 8 * nth) {
      C v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * nth;
        v[u] = czero<C>();
        if (e < tot) {
          const int sl = e / (N * N), q = e % (N * N);
          const int n = tl.n0 - 1 + sl;
          if (n >= -tl.l && n <= tl.l) v[u] = cvt<C, c2<TIN>>(Fev[row_of(L, tl.l, tl.m, n) * L.nx + pbase + q]);
        }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * nth;
        if (e < tot) {
          const int sl = e / (N * N), q = e % (N * N);
          sF[sl * PS + (q / N) * (N + 1) + q % N] = v[u];
        }
      }
    }
  if (HAS_P3) {
    const int tot = tl.cnt * N * N;
    for (int e0 = tid; e0 < tot; e0 += 8 * nth) {
      C v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * nth;
        v[u] = czero<C>();
        if (e < tot) {
          const int sl = e / (N * N), q = e % (N * N);
          v[u] = P3[row_of(L, tl.l, tl.m, tl.n0 + sl) * L.nx + pbase + q];
        }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * nth;
        if (e < tot) {
          const int sl = e / (N * N), q = e % (N * N);
          sP[sl * PS + (q / N) * (N + 1) + q % N] = v[u];
        }
      }
    }
  }
  }
  __syncthreads();

  // The update stage's loads (G, F0, acc) depend on nothing computed here:
  // their 128-byte lines are prefetched into L2 now and land during the FFT
  // stages (row offsets from s_rb, set before the barrier above).
  {
    const int tot = tl.cnt * N * N;
    constexpr int EG = 128 / (int)sizeof(C);   // elements of G per line
    for (int e = tid * EG; e < tot; e += nth * EG) {
      const long long gi = s_rb[e / (N * N)] + e % (N * N);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(Gl + gi));
    }
    for (int e = tid * 8; e < tot; e += nth * 8) {   // FP64: 8 elements per line
      const long long gi = s_rb[e / (N * N)] + e % (N * N);
      if (F0) asm volatile("prefetch.global.L2 [%0];" ::"l"(F0 + gi));
      if (acc) asm volatile("prefetch.global.L2 [%0];" ::"l"(acc + gi));
    }
  }

  // ---- S2/S3: inverse FFT along k1 (rows) then k2 (columns) of all loaded planes ----
  const int nLoaded = nF + (HAS_P3 ? tl.cnt : 0);
  auto plane_ptr = [&](int s) -> C* { return s < nF ? sF + s * PS : sP + (s - nF) * PS; };
  for (int it = tid; it < nLoaded * N; it += nth) {
    C* pl = plane_ptr(it / N);
    const int k2 = it % N;
    C x[N];
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = pl[k2 * (N + 1) + j];
    fft<N, true>(x);
#pragma unroll
    for (int j = 0; j < N; ++j) pl[k2 * (N + 1) + j] = x[j];
  }
  __syncthreads();
  for (int it = tid; it < nLoaded * N; it += nth) {
    C* pl = plane_ptr(it / N);
    const int k1 = it % N;
    C x[N];
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = pl[j * (N + 1) + k1];
    fft<N, true>(x);
#pragma unroll
    for (int j = 0; j < N; ++j) pl[j * (N + 1) + k1] = inv_n2 * x[j];
  }
  __syncthreads();

  // ---- S4: physical-space products, forward FFT along k2 ----
  // item (c, j1, kind): kind 0 -> A column, kind 1 -> Y1' column.  Each item
  // runs on a lane pair (fft_lane_pair): lane h forms the products at the rows
  // j2 = 2j + h and ends with the wavenumbers k2 = h N/2 + k, so both stages
  // give every thread of the block half an FFT.
  constexpr int H = N / 2;
  const int h = tid & 1, pr = tid >> 1, npr = nth >> 1;
  const T d3 = HAS_P3 ? tp * (T)kappa_first(k3, N) : (T)0;
  const T b1 = (T)prm.b[0], b2 = (T)prm.b[1], b3 = (T)prm.b[2];
  const T g1 = (T)prm.gyro[0], g2 = (T)prm.gyro[1], g3 = (T)prm.gyro[2];
  for (int it = pr; it < tl.cnt * N * 2; it += npr) {   // both lanes of a pair hold the same item
    const int kind = it / (tl.cnt * N);
    const int c = (it / N) % tl.cnt;
    const int j1 = it % N;
    const T x1 = -Ll / 2 + Ll * (T)j1 / (T)N;
    const C* f0 = sF + (c + 1) * PS;
    const C* fm = sF + c * PS;
    const C* fp = sF + (c + 2) * PS;
    const C* pp = sP + c * PS;
    const int n = tl.n0 + c, l = tl.l;
    const T lie = (T)prm.lie;
    const T ap = lie * sqrt((T)((l - n) * (l + n + 1))), am = lie * sqrt((T)((l + n) * (l - n + 1)));
    C x[H];
    if (kind == 0) {
      // Y0 = a+ F~+ (0.5i x1 - 0.5 x2) + a- F~- (0.5i x1 + 0.5 x2) - g3 D3 x1 x2 F~ + (i n + b3 D3) P~
#pragma unroll
      for (int j = 0; j < H; ++j) {
        const int j2 = 2 * j + h;
        const T x2 = -Ll / 2 + Ll * (T)j2 / (T)N;
        const int o = j2 * (N + 1) + j1;
        const C vp = fp[o], vm = fm[o];
        C y;
        // a+ vp * (0.5 i x1 - 0.5 x2) + a- vm * (0.5 i x1 + 0.5 x2)
        const T h1 = (T)0.5 * x1, h2 = (T)0.5 * x2;
        y.x = ap * (-h1 * vp.y - h2 * vp.x) + am * (-h1 * vm.y + h2 * vm.x);
        y.y = ap * (h1 * vp.x - h2 * vp.y) + am * (h1 * vm.x + h2 * vm.y);
        if (HAS_P3) {
          const C v0 = f0[o], pv = pp[o];
          // - g3 (i d3) x1 x2 v0
          const T sg = g3 * d3 * x1 * x2;
          y.x += sg * v0.y;
          y.y -= sg * v0.x;
          // (i n + b3 i d3) pv = i (n + b3 d3) pv
          const T q = lie * (T)n + b3 * d3;
          y.x -= q * pv.y;
          y.y += q * pv.x;
        }
        x[j] = y;
      }
      fft_lane_pair<H, false>(x, h);
#pragma unroll
      for (int k = 0; k < H; ++k) sA[c * PS + (h * H + k) * (N + 1) + j1] = x[k];
      // Y2 = b2 x2 F~ - g2 x1 P~  -> FFT_2 -> times D_2 = i d2(k2), added to A
#pragma unroll
      for (int j = 0; j < H; ++j) {
        const int j2 = 2 * j + h;
        const T x2 = -Ll / 2 + Ll * (T)j2 / (T)N;
        const int o = j2 * (N + 1) + j1;
        C y = (b2 * x2) * f0[o];
        if (HAS_P3) y = y - (g2 * x1) * pp[o];
        x[j] = y;
      }
      fft_lane_pair<H, false>(x, h);
#pragma unroll
      for (int k = 0; k < H; ++k) {
        const int k2 = h * H + k;
        const T dk = tp * (T)kappa_first(k2, N);
        C* dst = sA + c * PS + k2 * (N + 1) + j1;
        C v = *dst;
        v.x -= dk * x[k].y;
        v.y += dk * x[k].x;
        *dst = v;
      }
    } else {
      // Y1 = b1 x1 F~ - g1 x2 P~
#pragma unroll
      for (int j = 0; j < H; ++j) {
        const int j2 = 2 * j + h;
        const T x2 = -Ll / 2 + Ll * (T)j2 / (T)N;
        const int o = j2 * (N + 1) + j1;
        C y = (b1 * x1) * f0[o];
        if (HAS_P3) y = y - (g1 * x2) * pp[o];
        x[j] = y;
      }
      fft_lane_pair<H, false>(x, h);
#pragma unroll
      for (int k = 0; k < H; ++k) sY[c * PS + (h * H + k) * (N + 1) + j1] = x[k];
    }
  }
  __syncthreads();

  // ---- S5: forward FFT along k1 (lane pairs, in place); Y1' gets D_1 ----
  // The lanes of a pair read all of the row before their first exchange and
  // write it after, so the in-place update is safe.
  for (int it = pr; it < tl.cnt * N * 2; it += npr) {
    const int kind = it / (tl.cnt * N);
    const int c = (it / N) % tl.cnt;
    const int k2 = it % N;
    C* pl = (kind == 0 ? sA : sY) + c * PS + k2 * (N + 1);
    C x[H];
#pragma unroll
    for (int j = 0; j < H; ++j) x[j] = pl[2 * j + h];
    fft_lane_pair<H, false>(x, h);
    if (kind == 0) {
#pragma unroll
      for (int k = 0; k < H; ++k) pl[h * H + k] = x[k];
    } else {
#pragma unroll
      for (int k = 0; k < H; ++k) {
        const T dk = tp * (T)kappa_first(h * H + k, N);
        C v;
        v.x = -dk * x[k].y;
        v.y = dk * x[k].x;
        pl[h * H + k] = v;
      }
    }
  }
  __syncthreads();

  // ---- S6: dF = A + Y1' + G ; out = F0 + a dF ; acc += bacc dF ----
  {
    const uint64_t pol = l2_policy_evict_first();
    const int tot = tl.cnt * N * N;
    for (int e0 = tid; e0 < tot; e0 += 4 * nth) {
      C g[4];
      double2 f0[4], ac[4];
      long long gi[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * nth;
        gi[u] = -1;
        if (e < tot) {
          const int c = e / (N * N), q = e % (N * N);
          gi[u] = s_rb[c] + q;
          g[u] = Gl[gi[u]];
          f0[u] = F0 ? F0[gi[u]] : make_double2(0.0, 0.0);
          if (acc) ac[u] = acc[gi[u]];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * nth;
        if (e >= tot) continue;
        const int c = e / (N * N), q = e % (N * N), k1 = q % N, k2 = q / N;
        const C s = sA[c * PS + k2 * (N + 1) + k1] + sY[c * PS + k2 * (N + 1) + k1];
        const double dx = (double)s.x + (double)g[u].x, dy = (double)s.y + (double)g[u].y;
        double2 o = f0[u];
        o.x += a * dx;
        o.y += a * dy;
        // written once here and read by later kernels: evict first, so the
        // halo rows other tiles of this plane still read stay in L2
        st_evict_first(out + gi[u], o, pol);
        if (out32) st_evict_first(out32 + gi[u], cvt<C, double2>(o), pol);   // the next step's compute-precision input
        if (acc) {
          double2 v = ac[u];
          v.x += bacc * dx;
          v.y += bacc * dy;
          acc[gi[u]] = v;
        }
      }
    }
  }
}

template <int N, typename T, bool HAS_P3, typename TIN>
__global__ void __launch_bounds__(PlaneCfg<T>::NT, PlaneCfg<T>::MINB) k_plane(RowLayout L, const PlaneTile* __restrict__ tiles,
                                                  const c2<TIN>* __restrict__ Fev,
                                                  const c2<T>* __restrict__ P3,
                                                  const c2<T>* __restrict__ Gl,
                                                  const double2* __restrict__ F0, double a,
                                                  double2* __restrict__ out,
                                                  double2* __restrict__ acc, double bacc,
                                                  DerivParams prm, c2<T>* __restrict__ out32 = nullptr) {
  extern __shared__ __align__(16) unsigned char smraw[];
  plane_body<N, T, HAS_P3, TIN>(L, tiles[blockIdx.x], HAS_P3 ? (int)blockIdx.y : 0, Fev, P3, Gl, F0, a, out, acc, bacc,
                                prm, out32, smraw);
}

// ----------------------------------------- persistent batched plane pass ----
// The plane passes of several members (3-D plans of one compute precision,
// any bandlimit and omega grid) in one launch: every (member, tile, k3 plane)
// is an item of a work queue that the resident blocks drain through an atomic
// counter, larger grids first, so the uneven members share the GPU without a
// launch (and a tail) each.

// one grid size of the batched pass as a separate (not inlined) function, so
// that each keeps its own register allocation
template <int N, typename T>
__device__ __noinline__ void plane_item(const PlaneJob& jb, const PlaneTile tl, int k3, unsigned char* smraw) {
  using C = c2<T>;
  plane_body<N, T, true, T>(jb.L, tl, k3, (const C*)jb.Fev, (const C*)jb.P3, (const C*)jb.G, jb.F0, jb.a, jb.out,
                            jb.acc, jb.bacc, jb.prm, (C*)jb.out32, smraw);
}

template <typename T>
__global__ void __launch_bounds__(PlaneCfg<T>::NT, PlaneCfg<T>::MINB)
    k_plane_batch(const PlaneJob* __restrict__ jobs, int njobs, long long nitems, int* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ long long s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const long long it = s_item;
    if (it >= nitems) break;
    int j = 0;
    while (j + 1 < njobs && jobs[j + 1].item0 <= it) ++j;
    const PlaneJob& jb = jobs[j];
    const long long local = it - jb.item0;
    const PlaneTile tl = jb.tiles[local / jb.N];
    const int k3 = (int)(local % jb.N);
    switch (jb.N) {
      case 8: plane_item<8, T>(jb, tl, k3, smraw); break;
      case 12: plane_item<12, T>(jb, tl, k3, smraw); break;
      case 16: plane_item<16, T>(jb, tl, k3, smraw); break;
      case 20: plane_item<20, T>(jb, tl, k3, smraw); break;
      case 24: plane_item<24, T>(jb, tl, k3, smraw); break;
      case 30: plane_item<30, T>(jb, tl, k3, smraw); break;
      case 32: plane_item<32, T>(jb, tl, k3, smraw); break;
      default: break;
    }
    __syncthreads();   // shared memory and s_item are reused by the next item
  }
}

// Plane passes collected instead of launched while a batch step is being
// assembled (hp_plane_collect_begin / _end, batch.cu).
static thread_local std::vector<PlaneJob>* g_collect[2] = {nullptr, nullptr};   // [FP32, FP64]

static bool plane_batchable_N(int N) {
  return N == 8 || N == 12 || N == 16 || N == 20 || N == 24 || N == 30 || N == 32;
}

void hp_plane_collect_begin(std::vector<PlaneJob>* f32, std::vector<PlaneJob>* f64) {
  g_collect[0] = f32;
  g_collect[1] = f64;
}
void hp_plane_collect_end() { g_collect[0] = g_collect[1] = nullptr; }
size_t hp_plane_job_bytes() { return sizeof(PlaneJob); }
bool hp_plane_collecting() { return g_collect[0] || g_collect[1]; }

template <typename T> static size_t plane_smem_p3(int N) {
  constexpr int C = PlaneCfg<T>::C;
  return (size_t)((C + 2) + C + 2 * C) * N * (N + 1) * sizeof(c2<T>);
}
size_t hp_plane_batch_smem(int precision, int Nmax) {
  return precision == HP_FP64 ? plane_smem_p3<double>(Nmax) : plane_smem_p3<float>(Nmax);
}

// Runs the collected jobs of one precision in one persistent launch.
// d_jobs: device array of at least jobs.size() entries (filled by the caller);
// counter: device int.
// Orders jobs by grid size (largest first) and numbers their queue items.
void hp_plane_batch_prepare(std::vector<PlaneJob>& jobs) {
  std::stable_sort(jobs.begin(), jobs.end(), [](const PlaneJob& a, const PlaneJob& b) { return a.N > b.N; });
  long long it = 0;
  for (auto& j : jobs) {
    j.item0 = it;
    it += (long long)j.ntiles * j.N;
  }
}

int hp_plane_batch_launch(int precision, const std::vector<PlaneJob>& jobs, const PlaneJob* d_jobs, int* counter,
                          cudaStream_t s) {
  if (jobs.empty()) return HP_OK;
  long long nitems = 0;
  int nmax = 0;
  for (auto& j : jobs) {
    nitems = std::max(nitems, j.item0 + (long long)j.ntiles * j.N);
    nmax = std::max(nmax, j.N);
  }
  HP_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int), s));
  const size_t smem = hp_plane_batch_smem(precision, nmax);
  if (precision == HP_FP64) {
    HP_CUDA_TRY(cudaFuncSetAttribute(k_plane_batch<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_plane_batch<double><<<148 * PlaneCfg<double>::MINB, PlaneCfg<double>::NT, smem, s>>>(d_jobs, (int)jobs.size(),
                                                                                            nitems, counter);
  } else {
    HP_CUDA_TRY(cudaFuncSetAttribute(k_plane_batch<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_plane_batch<float><<<148 * PlaneCfg<float>::MINB, PlaneCfg<float>::NT, smem, s>>>(d_jobs, (int)jobs.size(),
                                                                                         nitems, counter);
  }
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// ------------------------------------------------------------ launcher ----
template <typename T> static size_t plane_smem(int N, bool p3) {
  const int C = PlaneCfg<T>::C;
  const int planes = (C + 2) + (p3 ? C : 0) + 2 * C;
  return (size_t)planes * N * (N + 1) * sizeof(c2<T>);
}


// k_local with the widest omega tile (32/16/8/4 points) whose group tile and
// tap weights fit 110 KB of shared memory (the m = 0 group has (lmax+1)^2 rows).
template <typename T, int W, typename TIN>
static int local_w_launch(hp_plan* p, const c2<TIN>* F, c2<T>* G, const c2<T>* Gx, const DerivParams& prm,
                          cudaStream_t s) {
  const size_t lsm = local_smem<T>(p, W);
  // omega chunks per block: the per-block staging of the tap tables amortised
  // over several chunks while about twelve blocks per SM remain
  const long long nchunks = (p->nx + W - 1) / W;
  const int cpb = (int)std::max(1LL, std::min(64LL, nchunks * p->nm / (148LL * 12)));
  dim3 grid((unsigned)((nchunks + cpb - 1) / cpb), (unsigned)p->nm);
  ProfScope _ps(p, "deriv.local", s);
  if (p->ndim == 3) {
    HP_CUDA_TRY(cudaFuncSetAttribute(k_local<T, W, 3, TIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsm));
    k_local<T, W, 3, TIN><<<grid, 256, lsm, s>>>(p->layout(), F, G, tap_table<T>(p), Gx, so3d_table<T>(p), prm, cpb);
  } else {
    HP_CUDA_TRY(cudaFuncSetAttribute(k_local<T, W, 2, TIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsm));
    k_local<T, W, 2, TIN><<<grid, 256, lsm, s>>>(p->layout(), F, G, tap_table<T>(p), Gx, so3d_table<T>(p), prm, cpb);
  }
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

template <typename T, typename TIN = double>
static int launch_local(hp_plan* p, const c2<TIN>* F, c2<T>* G, const c2<T>* Gx, const DerivParams& prm,
                        cudaStream_t s) {
  constexpr size_t budget = 110 * 1024;
  if (sizeof(T) == 4 && local_smem<T>(p, 32) <= budget) return local_w_launch<T, 32, TIN>(p, F, G, Gx, prm, s);
  if (local_smem<T>(p, 16) <= budget) return local_w_launch<T, 16, TIN>(p, F, G, Gx, prm, s);
  if (local_smem<T>(p, 8) <= budget) return local_w_launch<T, 8, TIN>(p, F, G, Gx, prm, s);
  if (local_smem<T>(p, 4) <= (size_t)200 * 1024) return local_w_launch<T, 4, TIN>(p, F, G, Gx, prm, s);
  hp_set_error("gravity pass tiles exceed shared memory for this bandlimit");
  return HP_ERR_UNSUPPORTED;
}

template <int N, typename T>
static int run_deriv_N(hp_plan* p, const double2* Fev, const double2* F0, double a, double2* out,
                       double2* acc, double bacc, cudaStream_t s, const DerivParams& prm, const void* Gx,
                       const void* fev32, void* out32) {
  using C = c2<T>;
  int st = HP_OK;
  const size_t fb = sizeof(C) * (size_t)p->nrows * p->nx;
  C* P3 = nullptr;
  if (p->ndim == 3) {
    P3 = (C*)p->ws_get("deriv.P3", fb, &st);
    if (st) return st;
  }
  C* G = (C*)p->ws_get("deriv.G", fb, &st);
  if (st) return st;
  // mixed 3-D plans: the axis-3 pass also leaves F in FP32 (Fc), which the
  // local and plane passes read in place of the FP64 state (the values they
  // convert to anyway), halving their coefficient traffic
  // When the caller already holds Fev in FP32 (fev32, from the previous step's
  // plane pass), the axis-3 pass reads that copy and writes none.
  const bool mixed3 = p->ndim == 3 && sizeof(T) == 4;
  C* Fc = nullptr;
  if (mixed3 && fev32) {
    Fc = (C*)const_cast<void*>(fev32);
  } else if (mixed3) {
    Fc = (C*)p->ws_get("deriv.F32", fb, &st);
    if (st) return st;
  }
  const RowLayout L = p->layout();
  if (p->ndim == 3) {
    const long long nt = p->nrows * (long long)N * N;
    ProfScope _ps(p, "deriv.axis3", s);
    if (mixed3 && fev32)
      k_axis3<N, T, T><<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(L, Fc, P3, (T)prm.L, (C*)nullptr);
    else
      k_axis3<N, T><<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(L, Fev, P3, (T)prm.L, Fc);
    HP_CUDA_TRY(cudaGetLastError());
  }
  if (Fc) {
    st = launch_local<T, T>(p, Fc, G, (const C*)Gx, prm, s);
  } else {
    st = launch_local<T>(p, Fev, G, (const C*)Gx, prm, s);
  }
  if (st) return st;
  // tiles: every (m, l) row split into chunks of CT consecutive n (built once per plan)
  constexpr int CT = PlaneCfg<T>::C;
  const char tkey[] = {'d', 'e', 'r', 'i', 'v', '.', 't', 'i', 'l', 'e', 's', (char)('0' + CT), 0};
  bool have = false;
  for (auto& kv : p->ws) if (kv.first == tkey) have = true;
  std::vector<PlaneTile> htiles;
  for (int m = p->m_lo; m <= p->lmax; ++m)
    for (int l = std::abs(m); l <= p->lmax; ++l)
      for (int n0 = -l; n0 <= l; n0 += CT) htiles.push_back({m, l, n0, std::min(CT, l - n0 + 1)});
  PlaneTile* dt = (PlaneTile*)p->ws_get(tkey, sizeof(PlaneTile) * htiles.size(), &st);
  if (st) return st;
  if (!have) {
    HP_CUDA_TRY(cudaMemcpy(dt, htiles.data(), sizeof(PlaneTile) * htiles.size(), cudaMemcpyHostToDevice));
  }
  const bool p3 = p->ndim == 3;
  // inside an assembled batch step the plane pass joins the batch's persistent launch
  std::vector<PlaneJob>* coll = g_collect[sizeof(T) == 8 ? 1 : 0];
  if (coll && p3 && plane_batchable_N(N) && (Fc || sizeof(T) == 8)) {
    PlaneJob jb{};
    jb.L = L;
    jb.tiles = dt;
    jb.ntiles = (int)htiles.size();
    jb.N = N;
    jb.Fev = Fc ? (const void*)Fc : (const void*)Fev;
    jb.P3 = P3;
    jb.G = G;
    jb.F0 = F0;
    jb.a = a;
    jb.out = out;
    jb.acc = acc;
    jb.bacc = bacc;
    jb.out32 = mixed3 ? out32 : nullptr;
    jb.prm = prm;
    coll->push_back(jb);
    return HP_OK;
  }
  const size_t smem = plane_smem<T>(N, p3);
  dim3 grid((unsigned)htiles.size(), p3 ? N : 1);
  ProfScope _ps(p, "deriv.plane", s);
  if (p3 && Fc) {
    HP_CUDA_TRY(cudaFuncSetAttribute(k_plane<N, T, true, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_plane<N, T, true, T><<<grid, PlaneCfg<T>::NT, smem, s>>>(L, dt, Fc, P3, G, F0, a, out, acc, bacc, prm,
                                                                (C*)(mixed3 ? out32 : nullptr));
  } else if (p3) {
    HP_CUDA_TRY(cudaFuncSetAttribute(k_plane<N, T, true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_plane<N, T, true, double><<<grid, PlaneCfg<T>::NT, smem, s>>>(L, dt, Fev, P3, G, F0, a, out, acc, bacc, prm);
  } else {
    HP_CUDA_TRY(cudaFuncSetAttribute(k_plane<N, T, false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_plane<N, T, false, double><<<grid, PlaneCfg<T>::NT, smem, s>>>(L, dt, Fev, P3, G, F0, a, out, acc, bacc, prm);
  }
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// ------------------------------------- large omega grids (2-D, N >= 40) ----
// The per-plane kernel's tiles do not fit shared memory beyond N = 32, so the
// 2-D derivative goes through whole-array omega FFTs:
//   Fp = IFFT(F);  Z = x1 S + x2 T with S = i/2 (a+ Fp_{n+1} + a- Fp_{n-1}),
//   T = 1/2 (a- Fp_{n-1} - a+ Fp_{n+1}) (the u_1, u_2 Lie terms), P1 = b1 x1 Fp,
//   P2 = b2 x2 Fp;  dF = FFT(Z) + D1 FFT(P1) + D2 FFT(P2) + G.
template <typename T>
__global__ void k_phys2d(RowLayout L, const c2<T>* __restrict__ Fp, c2<T>* __restrict__ Z, c2<T>* __restrict__ P1,
                         c2<T>* __restrict__ P2, DerivParams prm) {
  using C = c2<T>;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.nrows * L.nx) return;
  const long long row = t / L.nx, w = t % L.nx;
  const int N = L.N;
  const T Ll = (T)prm.L;
  const T x1 = -Ll / 2 + Ll * (T)(int)(w % N) / (T)N, x2 = -Ll / 2 + Ll * (T)(int)(w / N) / (T)N;
  const char4 q = L.rows[row];
  const int l = q.x, m = q.y, n = q.z;
  const T lie = (T)prm.lie;
  const T ap = lie * sqrt((T)((l - n) * (l + n + 1))), am = lie * sqrt((T)((l + n) * (l - n + 1)));
  const C vp = (n + 1 <= l) ? Fp[row_of(L, l, m, n + 1) * L.nx + w] : czero<C>();
  const C vm = (n - 1 >= -l) ? Fp[row_of(L, l, m, n - 1) * L.nx + w] : czero<C>();
  const T h1 = (T)0.5 * x1, h2 = (T)0.5 * x2;
  C y;
  y.x = ap * (-h1 * vp.y - h2 * vp.x) + am * (-h1 * vm.y + h2 * vm.x);
  y.y = ap * (h1 * vp.x - h2 * vp.y) + am * (h1 * vm.x + h2 * vm.y);
  Z[t] = y;
  const C f = Fp[t];
  P1[t] = ((T)prm.b[0] * x1) * f;
  P2[t] = ((T)prm.b[1] * x2) * f;
}

template <typename T>
__global__ void k_combine2d(RowLayout L, const c2<T>* __restrict__ Z, const c2<T>* __restrict__ P1,
                            const c2<T>* __restrict__ P2, const c2<T>* __restrict__ G,
                            const double2* __restrict__ F0, double a, double2* __restrict__ out,
                            double2* __restrict__ acc, double bacc, double tp) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.nrows * L.nx) return;
  const long long w = t % L.nx;
  const int N = L.N;
  const double d1 = tp * kappa_first((int)(w % N), N), d2 = tp * kappa_first((int)(w / N), N);
  const c2<T> z = Z[t], u = P1[t], v = P2[t], g = G[t];
  // dF = z + i d1 u + i d2 v + g
  const double dx = (double)z.x - d1 * (double)u.y - d2 * (double)v.y + (double)g.x;
  const double dy = (double)z.y + d1 * (double)u.x + d2 * (double)v.x + (double)g.y;
  double2 o = F0 ? F0[t] : make_double2(0.0, 0.0);
  o.x += a * dx;
  o.y += a * dy;
  out[t] = o;
  if (acc) {
    double2 c = acc[t];
    c.x += bacc * dx;
    c.y += bacc * dy;
    acc[t] = c;
  }
}

template <typename T>
static int run_deriv_lines(hp_plan* p, const double2* Fev, const double2* F0, double a, double2* out,
                           double2* acc, double bacc, cudaStream_t s, const DerivParams& prm, const void* Gx) {
  using C = c2<T>;
  if (p->ndim != 2) {
    hp_set_error("the derivative supports omega grids above 32 points per axis in 2-D only");
    return HP_ERR_UNSUPPORTED;
  }
  int st = HP_OK;
  const size_t fb = sizeof(C) * (size_t)p->nrows * p->nx;
  C* G = (C*)p->ws_get("deriv.G", fb, &st);
  if (st) return st;
  C* Fp = (C*)p->ws_get("deriv.Fp", fb, &st);
  if (st) return st;
  C* Z = (C*)p->ws_get("deriv.Z", fb, &st);
  if (st) return st;
  C* P1 = (C*)p->ws_get("deriv.P1", fb, &st);
  if (st) return st;
  C* P2 = (C*)p->ws_get("deriv.P2", fb, &st);
  if (st) return st;
  ST_CHECK(launch_local<T>(p, Fev, G, (const C*)Gx, prm, s));
  ST_CHECK(hp_omega_ifft_rows(p, Fev, Fp, s));
  const long long n = p->nrows * p->nx;
  const unsigned g = (unsigned)((n + 255) / 256);
  {
    ProfScope _ps(p, "deriv.phys", s);
    k_phys2d<T><<<g, 256, 0, s>>>(p->layout(), Fp, Z, P1, P2, prm);
    HP_CUDA_TRY(cudaGetLastError());
  }
  ST_CHECK(hp_omega_fft_rows(p, Z, s));
  ST_CHECK(hp_omega_fft_rows(p, P1, s));
  ST_CHECK(hp_omega_fft_rows(p, P2, s));
  ProfScope _ps(p, "deriv.combine", s);
  k_combine2d<T><<<g, 256, 0, s>>>(p->layout(), Z, P1, P2, G, F0, a, out, acc, bacc, 2.0 * M_PI / prm.L);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

template <typename T>
static int run_deriv(hp_plan* p, const double2* Fev, const double2* F0, double a, double2* out,
                     double2* acc, double bacc, cudaStream_t s, const DerivParams& prm, const void* Gx,
                     const void* fev32 = nullptr, void* out32 = nullptr) {
  switch (p->N) {
#define X(n) case n: return run_deriv_N<n, T>(p, Fev, F0, a, out, acc, bacc, s, prm, Gx, fev32, out32);
    HP_FOR_EACH_N_TO_32(X)
#undef X
#define X(n) case n:
    HP_FOR_EACH_N_ABOVE_32(X)
#undef X
      return run_deriv_lines<T>(p, Fev, F0, a, out, acc, bacc, s, prm, Gx);
    default:
      hp_set_error("omega grid size 2Bx not supported (even, 4..64)");
      return HP_ERR_UNSUPPORTED;
  }
}

// Density-side gravity of pendulum_reduced_den.m:449-516:
// Gx = -sum_i D_i fftSO3R(f . mR_i), with f the given grid density (first
// stage) or the backward transform of Feval (later stages, :454-475).
template <typename T>
__global__ void k_den_combine(const c2<T>* __restrict__ FMR, c2<T>* __restrict__ Gx, long long nrows, long long nx,
                              int N, int axis, double tp, int first) {
  using C = c2<T>;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= nrows * nx) return;
  const long long w = t % nx;
  const int k = (int)((axis == 0 ? w : w / N) % N);
  const T dk = (T)(tp * kappa_first(k, N));
  const C v = FMR[t];
  C g;                               // -(i dk) v
  g.x = dk * v.y;
  g.y = -dk * v.x;
  Gx[t] = first ? g : Gx[t] + g;
}

template <typename T>
static int den_gravity(hp_plan* p, const double2* Fev, const void* fgrid, cudaStream_t s, c2<T>** Gx_out) {
  using C = c2<T>;
  int st = HP_OK;
  const size_t fb = sizeof(C) * (size_t)p->nrows * p->nx;
  C* Gx = (C*)p->ws_get("deriv.Gden", fb, &st);
  if (st) return st;
  C* FMR = (C*)p->ws_get("deriv.FMR", fb, &st);
  if (st) return st;
  const void* f = fgrid;
  if (!f) {
    T* fg = (T*)p->ws_get("deriv.fden", sizeof(T) * (size_t)p->n_grid(), &st);
    if (st) return st;
    HP_CHECK_RET(hp_backward_internal(p, Fev, fg, 0, s));
    f = fg;
  }
  for (int i = 0; i < 2; ++i) {
    HP_CHECK_RET(hp_forward_internal_T(p, f, p->den_mR + (size_t)i * 8 * p->B * p->B * p->B, FMR, s));
    const long long n = p->nrows * p->nx;
    ProfScope _ps(p, "deriv.den", s);
    k_den_combine<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(FMR, Gx, p->nrows, p->nx, p->N, i,
                                                              2.0 * M_PI / p->model.L, i == 0);
    HP_CUDA_TRY(cudaGetLastError());
  }
  *Gx_out = Gx;
  return HP_OK;
}

// out = F0 + a * dF(Feval); if acc: acc += bacc * dF(Feval).  F0 may be null (zero).
// With a density-gravity model (hp_pendulum_propagate_den), fgrid is the grid
// density of Feval when the caller has it (else it is recomputed from Feval).
DerivParams hp_model_params(const hp_plan* p) {
  DerivParams prm;
  prm.L = p->model.L;
  for (int i = 0; i < 3; ++i) { prm.b[i] = p->model.b[i]; prm.gyro[i] = p->model.gyro[i]; prm.gs[i] = 1.0; }
  for (int i = 0; i < 9; ++i) prm.G[i] = p->model.G[i];
  prm.lie = 1.0;
  for (int q = 0; q < 3; ++q)
    for (int i = 0; i < 3; ++i) {
      prm.mr[q][i][0] = p->mr1[q][i].x;
      prm.mr[q][i][1] = p->mr1[q][i].y;
    }
  if (p->ndim == 2) { prm.b[2] = 0; prm.gyro[0] = prm.gyro[1] = prm.gyro[2] = 0; }
  return prm;
}

int hp_derivative_eval_prm(hp_plan* p, const DerivParams& prm, const double2* Fev, const double2* F0, double a,
                           double2* out, double2* acc, double bacc, cudaStream_t s, const void* fgrid,
                           const void* fev32, void* out32) {
  if (!p->has_model) { hp_set_error("no model: call hp_plan_set_model first"); return HP_ERR_NO_MODEL; }
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  const bool den = p->den_mR != nullptr && (prm.gs[0] != 0 || prm.gs[1] != 0);
  if (p->precision == HP_FP64) {
    double2* Gx = nullptr;
    if (den) HP_CHECK_RET(den_gravity<double>(p, Fev, fgrid, s, &Gx));
    return run_deriv<double>(p, Fev, F0, a, out, acc, bacc, s, prm, Gx);
  }
  float2* Gx = nullptr;
  if (den) HP_CHECK_RET(den_gravity<float>(p, Fev, fgrid, s, &Gx));
  return run_deriv<float>(p, Fev, F0, a, out, acc, bacc, s, prm, Gx, fev32, out32);
}

// out = F0 + a * dF(Feval); if acc: acc += bacc * dF(Feval).  F0 may be null (zero).
// With a density-gravity model (hp_pendulum_propagate_den), fgrid is the grid
// density of Feval when the caller has it (else it is recomputed from Feval).
int hp_gravity_noise_eval64(hp_plan* p, const DerivParams& prm, const double2* F, double2* out, cudaStream_t s) {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  return launch_local<double, double>(p, F, out, nullptr, prm, s);
}

int hp_derivative_eval(hp_plan* p, const double2* Fev, const double2* F0, double a, double2* out,
                       double2* acc, double bacc, cudaStream_t s, const void* fgrid, const void* fev32,
                       void* out32) {
  return hp_derivative_eval_prm(p, hp_model_params(p), Fev, F0, a, out, acc, bacc, s, fgrid, fev32, out32);
}

// ------------------------------------------ derivative without allocation ----
// Scratch of hp_pendulum_derivative_noalloc: a file-scope device array that every
// GPU loading the library holds until exit.  Holds, 256-byte aligned: the
// coefficients and the derivative in the internal layout, the two intermediate
// fields of the derivative (P3 = M_3 F and gravity + diffusion), and the plane
// tile list.  All of it is fully overwritten by each call, so nothing is cleared.
static constexpr size_t kNoAllocScratchBytes = (size_t)HP_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Address of the scratch array on each device (one context per device, the
// runtime's primary context), looked up once per device.  Threads that race on
// the first call store the same value; the atomics make that well defined.
static std::atomic<void*> g_noalloc_addr[64];

static int noalloc_scratch(void** out) {
  int dev = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { hp_set_error("device index out of range"); return HP_ERR_INVALID; }
  void* ptr = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (!ptr) {
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      hp_set_error(e != cudaSuccess ? cudaGetErrorString(e) : "scratch symbol has no device address");
      return HP_ERR_CUDA;
    }
    g_noalloc_addr[dev].store(ptr, std::memory_order_release);
  }
  *out = ptr;
  return HP_OK;
}

// Writes the plane-pass tile list (every (m, l) row cut into chunks of CT
// consecutive n) on the device, so no host buffer is needed: one thread per
// (m, l) row, its first tile at the count of the tiles of the rows before it.
__global__ void k_make_tiles(int m_lo, int lmax, int CT, PlaneTile* tiles) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int k = 0, r = 0;
  for (int m = m_lo; m <= lmax; ++m)
    for (int l = abs(m); l <= lmax; ++l, ++r) {
      if (r == t) {
        for (int n0 = -l; n0 <= l; n0 += CT) tiles[k++] = PlaneTile{m, l, n0, min(CT, l - n0 + 1)};
        return;
      }
      k += (2 * l + 1 + CT - 1) / CT;
    }
}

static size_t align256(size_t x) { return (x + 255) / 256 * 256; }

template <int N, typename T>
static int noalloc_N(hp_plan* p, const double2* Ffull, double2* dFfull, unsigned char* base,
                     const DerivParams& prm) {
  using C = c2<T>;
  constexpr int CT = PlaneCfg<T>::C;
  cudaStream_t s = p->stream;
  const size_t pts = (size_t)p->nrows * p->nx;
  int ntiles = 0, nml = 0;
  for (int m = p->m_lo; m <= p->lmax; ++m)
    for (int l = std::abs(m); l <= p->lmax; ++l, ++nml) ntiles += (2 * l + 1 + CT - 1) / CT;
  const bool p3 = p->ndim == 3;
  size_t off = 0;
  double2* Fi = reinterpret_cast<double2*>(base + off); off = align256(off + 16 * pts);
  double2* dFi = reinterpret_cast<double2*>(base + off); off = align256(off + 16 * pts);
  C* P3 = p3 ? reinterpret_cast<C*>(base + off) : nullptr; if (p3) off = align256(off + sizeof(C) * pts);
  C* G = reinterpret_cast<C*>(base + off); off = align256(off + sizeof(C) * pts);
  PlaneTile* tiles = reinterpret_cast<PlaneTile*>(base + off); off = align256(off + sizeof(PlaneTile) * ntiles);
  if (off > kNoAllocScratchBytes) {
    hp_set_error("problem too large for the fixed scratch of hp_pendulum_derivative_noalloc "
                 "(see HP_NOALLOC_SCRATCH_BYTES)");
    return HP_ERR_SHAPE;
  }
  const RowLayout L = p->layout();
  int st = hp_full_to_internal(p, Ffull, Fi, s);
  if (st) return st;
  k_make_tiles<<<(nml + 127) / 128, 128, 0, s>>>(p->m_lo, p->lmax, CT, tiles);
  HP_CUDA_TRY(cudaGetLastError());
  if (p3) {
    const long long nt = p->nrows * (long long)N * N;
    k_axis3<N, T><<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(L, Fi, P3, (T)prm.L, (c2<T>*)nullptr);
    HP_CUDA_TRY(cudaGetLastError());
  }
  ST_CHECK(launch_local<T>(p, Fi, G, (const c2<T>*)nullptr, prm, s));
  const size_t smem = plane_smem<T>(N, p3);
  dim3 grid((unsigned)ntiles, p3 ? N : 1);
  if (p3) {
    HP_CUDA_TRY(cudaFuncSetAttribute(k_plane<N, T, true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_plane<N, T, true, double><<<grid, PlaneCfg<T>::NT, smem, s>>>(L, tiles, Fi, P3, G, nullptr, 1.0, dFi, nullptr, 0.0, prm);
  } else {
    HP_CUDA_TRY(cudaFuncSetAttribute(k_plane<N, T, false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_plane<N, T, false, double><<<grid, PlaneCfg<T>::NT, smem, s>>>(L, tiles, Fi, P3, G, nullptr, 1.0, dFi, nullptr, 0.0, prm);
  }
  HP_CUDA_TRY(cudaGetLastError());
  return hp_internal_to_full(p, dFi, dFfull, s);
}

template <typename T>
static int noalloc_T(hp_plan* p, const double2* F, double2* dF, unsigned char* base, const DerivParams& prm) {
  switch (p->N) {
#define X(n) case n: return noalloc_N<n, T>(p, F, dF, base, prm);
    HP_FOR_EACH_N_TO_32(X)
#undef X
    default:
      hp_set_error("the allocation-free derivative covers omega grids of 4..32 points per axis");
      return HP_ERR_UNSUPPORTED;
  }
}

extern "C" int hp_pendulum_derivative_noalloc(hp_plan* p, const double* F, double* dF) {
  if (!p || !F || !dF) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (!p->has_model) { hp_set_error("no model: call hp_plan_set_model first"); return HP_ERR_NO_MODEL; }
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  void* base = nullptr;
  int st = noalloc_scratch(&base);
  if (st) return st;
  if (p->den_mR) {
    hp_set_error("the allocation-free derivative does not cover density-gravity models");
    return HP_ERR_UNSUPPORTED;
  }
  const DerivParams prm = hp_model_params(p);
  const double2* Fin = reinterpret_cast<const double2*>(F);
  double2* out = reinterpret_cast<double2*>(dF);
  unsigned char* b = static_cast<unsigned char*>(base);
  if (p->precision == HP_FP64) return noalloc_T<double>(p, Fin, out, b, prm);
  return noalloc_T<float>(p, Fin, out, b, prm);
}
