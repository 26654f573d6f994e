// Linear predictors E[i, j] = z_i . B_j (the dense columns' GEMM plus the cells' level
// coefficients) on the FP64 tensor pipe, for W / nu (getWForBeta, ggplvm.cu:468-514) and the
// gradient's predictions z_i . tilde-beta_j.
//
//   k_eta_pack   Bd[k, j] = B[dcol k, j]: the dense rows of B, gene-contiguous (n_d x Jpad)
//   k_eta_dmma   the GEMM D (N x n_d) . Bd (n_d x J) with K = n_d <= 136 held whole: each CTA
//                keeps one 64-gene panel of Bd in shared memory and streams 64-cell tiles of
//                D through a double buffer (cp.async, the next tile's copies in flight during
//                the current tile's MMAs); 8 warps as 2 (cells) x 4 (genes), warp tile 32 x 16.
//                Persistent: 148-ish CTAs walk the (gene panel, cell tile) units in
//                gene-panel-major order, reloading the panel only when it changes. The
//                epilogue adds the level coefficients and stores along the cells.
//                Work 2 N J n_d flops (DMMA-bound), 8 N J bytes written.
// Wider designs (n_d > 136) use the FFMA tile GEMM k_eta.
#include <algorithm>

#include "dmma_common.cuh"
#include "gpl_internal.cuh"

namespace gpl {

namespace {
constexpr int EBM = 64, EBN = 64, EKMAX = 136;
constexpr int ESA = EBM + 4;  // As[k][m]: rows 544 B (16-byte multiple, fragment loads conflict-free)
constexpr int ESB = EBN + 4;  // Bs[k][n]
}  // namespace

__global__ void k_eta_pack(int n_d, int J, int Jpad, int P, const int* __restrict__ dcol, const double* __restrict__ B,
                           double* __restrict__ Bd) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (j < Jpad) Bd[(size_t)k * Jpad + j] = j < J ? B[dcol[k] + (size_t)j * P] : 0.0;
}

__global__ void __launch_bounds__(256, 1)
    k_eta_dmma(int N, int ldN, int J, int Jpad, int P, int n_d, int KP, int n_cv, const double* __restrict__ D,
               const double* __restrict__ Bd, const int* __restrict__ cv_nh, const int* __restrict__ codes,
               const double* __restrict__ B, double* __restrict__ out) {
  extern __shared__ __align__(16) double esm[];
  double* Bs = esm;                  // [KP][ESB]
  double* As = esm + KP * ESB;       // [2][KP][ESA]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  const int CT = (N + EBM - 1) / EBM, GT = Jpad / EBN;
  const long long U = (long long)CT * GT;
  const int u0 = (int)(U * blockIdx.x / gridDim.x), u1 = (int)(U * (blockIdx.x + 1) / gridDim.x);

  auto loadB = [&](int gt) {
    for (int e = tid; e < KP * (EBN / 2); e += 256) {
      const int k = e / (EBN / 2), part = e - k * (EBN / 2);
      const double* src = k < n_d ? Bd + (size_t)k * Jpad + gt * EBN + part * 2 : Bd;
      cp_async16(Bs + k * ESB + part * 2, src, k < n_d ? 16 : 0);
    }
  };
  auto loadA = [&](int ct, int buf) {
    double* as = As + buf * KP * ESA;
    for (int e = tid; e < KP * (EBM / 2); e += 256) {
      const int k = e / (EBM / 2), part = e - k * (EBM / 2);
      const int i = ct * EBM + part * 2;
      const int nb = k < n_d ? 8 * max(0, min(2, N - i)) : 0;
      const double* src = k < n_d ? D + (size_t)k * ldN + min(i, ldN - 2) : D;
      cp_async16(as + k * ESA + part * 2, src, nb);
    }
  };

  if (u0 < u1) {
    loadB(u0 / CT);
    loadA(u0 % CT, 0);
  }
  cp_async_commit();
  for (int u = u0; u < u1; u++) {
    const int buf = (u - u0) & 1, gt = u / CT, ct = u - gt * CT;
    const bool next_same = u + 1 < u1 && (u + 1) / CT == gt;
    if (next_same) loadA((u + 1) % CT, buf ^ 1);
    cp_async_commit();
    cp_async_wait<1>();  // this unit's tiles landed
    __syncthreads();

    double acc[2][2][4];
#pragma unroll
    for (int x = 0; x < 2; x++)
#pragma unroll
      for (int y = 0; y < 2; y++)
#pragma unroll
        for (int w = 0; w < 4; w++) acc[x][y][w] = 0.0;
    const double* as = As + buf * KP * ESA + wm * 32 + g;
    const double* bs = Bs + wn * 16 + g;
    for (int kk = 0; kk < KP; kk += 4) {
      double a[2][2], b[2];
#pragma unroll
      for (int x = 0; x < 2; x++) {
        a[x][0] = as[(kk + t) * ESA + x * 16];
        a[x][1] = as[(kk + t) * ESA + x * 16 + 8];
      }
#pragma unroll
      for (int y = 0; y < 2; y++) b[y] = bs[(kk + t) * ESB + y * 8];
#pragma unroll
      for (int x = 0; x < 2; x++)
#pragma unroll
        for (int y = 0; y < 2; y++) dmma_16x8x4(acc[x][y], a[x][0], a[x][1], b[y]);
    }

    // epilogue: E = acc + the level coefficients of the cell, stored along the cells
#pragma unroll
    for (int x = 0; x < 2; x++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int i = ct * EBM + wm * 32 + x * 16 + g + 8 * h;
        if (i >= N) continue;
#pragma unroll
        for (int y = 0; y < 2; y++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int j = gt * EBN + wn * 16 + y * 8 + 2 * t + e;
            if (j >= J) continue;
            double s = acc[x][y][2 * h + e];
            for (int v = 0; v < n_cv; v++) s += B[cv_nh[v] + codes[(size_t)v * ldN + i] + (size_t)j * P];
            out[i + (size_t)j * ldN] = s;
          }
      }
    __syncthreads();  // every warp is done with this unit's tiles
    if (!next_same && u + 1 < u1) {  // a new gene panel: its own copy group
      loadB((u + 1) / CT);
      loadA((u + 1) % CT, buf ^ 1);
      cp_async_commit();
    }
  }
  cp_async_wait<0>();
}

int eta_dmma_smem(int n_d) {
  const int KP = (n_d + 3) / 4 * 4;
  return (int)sizeof(double) * (KP * ESB + 2 * KP * ESA);
}

// E = Z B for all J genes into out (ldN x J); GPL_ERR_ARG when the dense columns exceed the
// kernel's K (the caller then uses the FFMA tile GEMM).
int launch_eta_dmma(Ctx* c, const double* B, double* out) {
  const int n_d = c->n_d, KP = (n_d + 3) / 4 * 4;
  if (KP > EKMAX) return GPL_ERR_ARG;
  const int Jpad = (c->J + EBN - 1) / EBN * EBN;
  if (!c->eta_bd) {
    if (cudaMalloc((void**)&c->eta_bd, sizeof(double) * (size_t)n_d * Jpad) != cudaSuccess) {
      cudaGetLastError();
      c->err = "device allocation failed: predictor panel";
      return GPL_ERR_ALLOC;
    }
  }
  dim3 gp(div_up(Jpad, 256), n_d);
  k_eta_pack<<<gp, 256, 0, c->stream>>>(n_d, c->J, Jpad, c->P, c->dcol_d, B, c->eta_bd);
  GPL_LAUNCHED(c, "k_eta_pack");
  const int smem = eta_dmma_smem(n_d);
  GPL_TRY(c, cudaFuncSetAttribute(k_eta_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  k_eta_dmma<<<sms, 256, smem, c->stream>>>(c->N, c->ldN, c->J, Jpad, c->P, n_d, KP, c->n_cv, c->Dm, c->eta_bd,
                                             c->cv_nh_d, c->codes_d, B, out);
  GPL_LAUNCHED(c, "k_eta_dmma");
  return GPL_OK;
}

}  // namespace gpl
