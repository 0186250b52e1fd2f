// Clebsch-Gordan product rule of fftSO3_prod.m:209-265 (complex branch):
//   FG^l_{mn} = sum_{l1,l2} (2l1+1)(2l2+1)/(2l+1)
//               sum_{m1,n1} F^{l1}_{m1 n1} G^{l2}_{m-m1, n-n1} <l1 m1; l2 m-m1|l m><l1 n1; l2 n-n1|l n>
// which is the entry-wise form of [CG^T kron(F^{l1}, G^{l2}) CG]_{l-block}.
// The dense CG table [l1][l2][l][m][m1] is built once per plan in FP64 on the
// device with the same tridiagonal solve as clebsch_gordan.m.
#include "common.cuh"
#include "plan.hpp"

using namespace hp;

#include "cg.cuh"

static __host__ __device__ __forceinline__ long long cgt_index(int B, int l1, int l2, int l, int m, int m1) {
  const int D = 2 * B - 1, lmax = B - 1;
  return ((((long long)l1 * B + l2) * B + l) * D + (m + lmax)) * D + (m1 + lmax);
}

__global__ void k_cg_table(int B, double* __restrict__ cgt) {
  const int lmax = B - 1, D = 2 * lmax + 1;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)B * B * B * D) return;
  const int m = (int)(t % D) - lmax;
  const int l = (int)((t / D) % B), l2 = (int)((t / D / B) % B), l1 = (int)(t / D / B / B);
  for (int m1 = -lmax; m1 <= lmax; ++m1) cgt[cgt_index(B, l1, l2, l, m, m1)] = 0.0;
  if (l < abs(l1 - l2) || l > l1 + l2 || abs(m) > l) return;
  double C[64], dd[64], du[64], dl[64], rb[64];
  const int nnz = cg_column(l1, l2, l, m, C, dd, du, dl, rb);
  const int m1lo = max(-l1, m - l2);
  for (int k = 0; k < nnz; ++k) cgt[cgt_index(B, l1, l2, l, m, m1lo + k)] = C[k];
}

// One thread per (output (m, n, l), batch element); full MATLAB layout.
__global__ void k_prod(int B, const double* __restrict__ cgt, const double2* __restrict__ F,
                       const double2* __restrict__ G, double2* __restrict__ FG, int batch) {
  const int lmax = B - 1, D = 2 * lmax + 1;
  const long long per = (long long)D * D * B;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= per * batch) return;
  const long long bidx = t / per, fi = t % per;
  const int m = (int)(fi % D) - lmax, n = (int)((fi / D) % D) - lmax, l = (int)(fi / (D * D));
  double2 acc = make_double2(0.0, 0.0);
  if (abs(m) <= l && abs(n) <= l) {
    const double2* Fb = F + bidx * per;
    const double2* Gb = G + bidx * per;
    for (int l1 = 0; l1 <= lmax; ++l1)
      for (int l2 = abs(l - l1); l2 <= lmax && l2 <= l + l1; ++l2) {
        const double cl = (2.0 * l1 + 1.0) * (2.0 * l2 + 1.0) / (2.0 * l + 1.0);
        double2 s = make_double2(0.0, 0.0);
        for (int m1 = max(-l1, m - l2); m1 <= min(l1, m + l2); ++m1) {
          const double cm = cgt[cgt_index(B, l1, l2, l, m, m1)];
          if (cm == 0.0) continue;
          const int m2 = m - m1;
          for (int n1 = max(-l1, n - l2); n1 <= min(l1, n + l2); ++n1) {
            const double cn = cgt[cgt_index(B, l1, l2, l, n, n1)];
            if (cn == 0.0) continue;
            const int n2 = n - n1;
            const double2 a = Fb[(m1 + lmax) + (long long)D * (n1 + lmax) + (long long)D * D * l1];
            const double2 b = Gb[(m2 + lmax) + (long long)D * (n2 + lmax) + (long long)D * D * l2];
            const double c = cm * cn;
            s.x += c * (a.x * b.x - a.y * b.y);
            s.y += c * (a.x * b.y + a.y * b.x);
          }
        }
        acc.x += cl * s.x;
        acc.y += cl * s.y;
      }
  }
  FG[t] = acc;
}

int hp_prod_launch(hp_plan* p, const double2* F, const double2* G, double2* FG, int batch, cudaStream_t s) {
  const int B = p->B, D = p->D;
  if (B > 32) { hp_set_error("fftSO3_prod supports B <= 32"); return HP_ERR_UNSUPPORTED; }
  int st = HP_OK;
  const size_t nb = sizeof(double) * (size_t)B * B * B * D * D;
  bool fresh = true;
  for (auto& kv : p->ws) if (kv.first == "prod.cgt") fresh = false;
  double* cgt = (double*)p->ws_get("prod.cgt", nb, &st);
  if (st) return st;
  if (fresh) {
    const long long nt = (long long)B * B * B * D;
    k_cg_table<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(B, cgt);
    HP_CUDA_TRY(cudaGetLastError());
  }
  const long long nt = (long long)D * D * B * batch;
  ProfScope _ps(p, "prod", s);
  k_prod<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(B, cgt, F, G, FG, batch);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}
