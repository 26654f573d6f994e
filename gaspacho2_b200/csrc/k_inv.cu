// Batched inverse of the per-gene Psi_j from their Cholesky factors (solvePsi,
// ggplvm.cu:46-53, which runs cholsl chol.cu:45-56 on every column of the identity):
// Psi_j^{-1} = V^T V with V = L^{-1}, in 32-column panels with FP64 tensor-core (DMMA)
// block products.
//
//   k_trtri_panel  one CTA per (panel jb, gene): the columns [32 jb, 32 jb + 32) of V by
//                  forward substitution over 32-row blocks. Block i first takes the product of
//                  the finished rows, R = E - L[i, jb..i) Y[jb..i) (DMMA), then solves
//                  L[i,i] Y_i = R by column-oriented substitution: one warp per 4 right-hand
//                  sides, lanes over rows, y_q = r_q * (1/L[q,q]) broadcast by shuffle, each
//                  row's sum taken in increasing q as in cholsl. The panel stays in shared memory;
//                  L's rows stream through two 32-column buffers. Work: P^3/6 multiply-adds per gene.
//   k_lauum_panel  one CTA per (panel b, gene): S[a, b] = sum_{k >= a} V[k, a]^T V[k, b]
//                  for the blocks a >= b, written to both triangles; the rows of block column a
//                  stream through two 32-row buffers. Work: P^3/6 per gene.
// Both fit two CTAs per SM up to P = 256 (the panel's rows plus the two buffers).
//
// L is the lower triangle (with diagonal) of the factored Psi_j (column-major, ld P); V is
// written column-major (ld P) below and on the diagonal of each panel, the strict upper part of
// the diagonal blocks holding exact zeros. A factor zero-filled by a failed Cholesky gives
// infinities and NaNs, as in the reference.
#include <algorithm>

#include "dmma_common.cuh"
#include "gpl_internal.cuh"

namespace gpl {

namespace {
constexpr int IB = 32;  // block size
constexpr int IS = 36;  // shared row stride (doubles): conflict-free fragment loads
constexpr int LS = 33;  // shared row stride of the 32 x 32 diagonal and right-hand-side blocks
constexpr int CW = 8;   // finished columns per chunk of the Cholesky's panel update
// Largest P each kernel is launched for. k_potrf_panel's update covers 256 rows of a panel
// (8 warps x 2 row tiles of 16), so its panels below the first may hold at most 256 rows:
// P <= 288. The inverse panels hold any P their shared memory admits (P <= 640 within 220 KiB).
// tests/index_mirror/k_inv_mirror.c replays every shared- and global-memory index of the
// three kernels on the CPU for every P up to these limits.
constexpr int kPotrfMaxP = 288;
constexpr int kInverseMaxP = 640;
}  // namespace

__global__ void __launch_bounds__(256, 2)
    k_trtri_panel(const double* __restrict__ Psi, int P, int64_t stride, double* __restrict__ V) {
  extern __shared__ __align__(16) double sm[];
  const int nb = (P + IB - 1) / IB;
  const int jb = blockIdx.x;
  const double* L = Psi + (size_t)blockIdx.y * stride;
  double* Vm = V + (size_t)blockIdx.y * stride;
  const int r0 = jb * IB;
  double* Yp = sm;                            // [nb*32][IS], local row r = global row r0 + r
  double* As = Yp + (size_t)nb * IB * IS;     // [2][32][IS]: As[k][m] = L[rb + m][r0 + 32 ch + k]
  double* Ld = As + 2 * IB * IS;              // [32][LS] diagonal block
  double* Rs = Ld + IB * LS;                  // [32][LS] right-hand sides
  double* Rd = Rs + IB * LS;                  // [32] reciprocals of the diagonal
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int m0 = (warp >> 2) * 16, n0 = (warp & 3) * 8;

  for (int ib = jb; ib < nb; ib++) {
    const int rb = ib * IB;
    const int nch = ib - jb;  // 32-column chunks of the finished rows
    // L[rb.., r0 + 32 ch ..] streamed through two buffers, 32 columns at a time
    auto stage = [&](int ch, int buf) {
      double* dst = As + buf * IB * IS;
      for (int e = tid; e < IB * IB; e += blockDim.x) {
        const int k = e >> 5, m = e & 31;
        const int row = rb + m;
        cp_async8(dst + k * IS + m, L + (size_t)min(row, P - 1) + (size_t)(r0 + ch * IB + k) * P, row < P ? 8 : 0);
      }
      cp_async_commit();
    };
    if (nch > 0) stage(0, 0);
    for (int e = tid; e < IB * IB; e += blockDim.x) {
      const int q = e >> 5, m = e & 31;
      const int row = rb + m, col = rb + q;
      double v;
      if (row < P && col < P) v = q <= m ? L[row + (size_t)col * P] : 0.0;
      else v = (m == q) ? 1.0 : 0.0;
      Ld[m * LS + q] = v;
    }

    // two accumulators over alternating K steps break the DMMA chain; the K order is that of
    // one pass over all the finished rows
    double acc[4] = {0.0, 0.0, 0.0, 0.0}, acc2[4] = {0.0, 0.0, 0.0, 0.0};
    for (int ch = 0; ch < nch; ch++) {
      if (ch + 1 < nch) {
        stage(ch + 1, (ch + 1) & 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
      const double* as = As + (ch & 1) * IB * IS;
      const double* yp = Yp + (size_t)ch * IB * IS;
#pragma unroll
      for (int kb = 0; kb < IB; kb += 8) {
        dmma_16x8x4(acc, as[(kb + t) * IS + m0 + g], as[(kb + t) * IS + m0 + g + 8], yp[(kb + t) * IS + n0 + g]);
        dmma_16x8x4(acc2, as[(kb + 4 + t) * IS + m0 + g], as[(kb + 4 + t) * IS + m0 + g + 8],
                    yp[(kb + 4 + t) * IS + n0 + g]);
      }
      __syncthreads();  // the buffer is refilled two chunks on
    }
    __syncthreads();  // Ld complete
    const int K = nch * IB;
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int m = m0 + g + 8 * h, n = n0 + 2 * t + e;
        const double ev = (ib == jb && m == n) ? 1.0 : 0.0;
        Rs[m * LS + n] = ev - (acc[2 * h + e] + acc2[2 * h + e]);
      }
    if (tid < IB) Rd[tid] = 1.0 / Ld[tid * LS + tid];
    __syncthreads();

    // L[i,i] Y_i = R: warp owns columns 4*warp .. +3, lane = row
    double rr[4];
#pragma unroll
    for (int c = 0; c < 4; c++) rr[c] = Rs[lane * LS + 4 * warp + c];
    for (int q = 0; q < IB; q++) {
      const double rq = Rd[q];
      const double lrq = Ld[lane * LS + q];
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const double yq = __shfl_sync(0xffffffffu, rr[c], q) * rq;
        if (lane == q) rr[c] = yq;
        else if (lane > q) rr[c] = fma(-lrq, yq, rr[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < 4; c++) Yp[(K + lane) * IS + 4 * warp + c] = rr[c];
    __syncthreads();
  }
  // the panel out: rows r0 .. P-1, columns r0 .. min(r0 + 32, P) - 1
  const int ncol = min(IB, P - r0), nrow = P - r0;
  for (int e = tid; e < nrow * ncol; e += blockDim.x) {
    const int c = e / nrow, r = e - c * nrow;
    Vm[(size_t)(r0 + r) + (size_t)(r0 + c) * P] = Yp[r * IS + c];
  }
}

__global__ void __launch_bounds__(256, 2)
    k_lauum_panel(const double* __restrict__ V, int P, int64_t stride, double* __restrict__ S) {
  extern __shared__ __align__(16) double sm[];
  const int nb = (P + IB - 1) / IB;
  const int b = blockIdx.x;
  const double* Vm = V + (size_t)blockIdx.y * stride;
  double* Sm = S + (size_t)blockIdx.y * stride;
  const int c0 = b * IB;
  const int ncol = min(IB, P - c0);
  double* Vb = sm;                          // [nb*32][IS]: Vb[k][n] = V[c0 + k][c0 + n]
  double* Ak = Vb + (size_t)nb * IB * IS;   // [2][32][IS]: Ak[k][m] = V[a0 + 32 ch + k][a0 + m]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int m0 = (warp >> 2) * 16, n0 = (warp & 3) * 8;
  const int kb_rows = (P - c0 + 3) / 4 * 4;
  for (int e = tid; e < kb_rows * IB; e += blockDim.x) {  // rows fastest: coalesced columns
    const int n = e / kb_rows, k = e - n * kb_rows;
    const int row = c0 + k, col = c0 + n;
    const bool ok = row < P && col < P;
    cp_async8(Vb + k * IS + n, Vm + (ok ? (size_t)row + (size_t)col * P : 0), ok ? 8 : 0);
  }
  cp_async_commit();
  for (int a = b; a < nb; a++) {
    const int a0 = a * IB;
    const int K = (P - a0 + 3) / 4 * 4;
    const int nch = (K + IB - 1) / IB;
    // the rows of block column a streamed through two buffers, 32 rows at a time
    auto stage = [&](int ch, int buf) {
      double* dst = Ak + buf * IB * IS;
      const int k0 = ch * IB, kn = min(IB, K - k0);
      for (int e = tid; e < kn * IB; e += blockDim.x) {
        const int m = e / kn, k = e - m * kn;
        const int row = a0 + k0 + k, col = a0 + m;
        const bool ok = row < P && col < P;
        cp_async8(dst + k * IS + m, Vm + (ok ? (size_t)row + (size_t)col * P : 0), ok ? 8 : 0);
      }
      cp_async_commit();
    };
    stage(0, 0);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const int off = a0 - c0;
    for (int ch = 0; ch < nch; ch++) {
      if (ch + 1 < nch) {
        stage(ch + 1, (ch + 1) & 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
      const double* ak = Ak + (ch & 1) * IB * IS;
      const double* vb = Vb + (size_t)(off + ch * IB) * IS;
      const int kn = min(IB, K - ch * IB);  // a multiple of 4
      for (int kb = 0; kb < kn; kb += 4) {
        const double a0v = ak[(kb + t) * IS + m0 + g];
        const double a1v = ak[(kb + t) * IS + m0 + g + 8];
        const double b0v = vb[(kb + t) * IS + n0 + g];
        dmma_16x8x4(acc, a0v, a1v, b0v);
      }
      __syncthreads();  // the buffer is refilled two chunks on
    }
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int m = m0 + g + 8 * h, n = n0 + 2 * t + e;
        const int row = a0 + m, col = c0 + n;
        if (row < P && n < ncol) {
          Sm[(size_t)row + (size_t)col * P] = acc[2 * h + e];
          Sm[(size_t)col + (size_t)row * P] = acc[2 * h + e];
        }
      }
  }
}

// Batched Cholesky (cholPsi, ggplvm.cu:683-692), one CTA per gene, 32-column panels left to
// right (left-looking): the panel is loaded into shared memory, takes the product of the
// finished columns (DMMA, the finished part streamed through shared memory 8 columns at a
// time, so that two CTAs share an SM), then its 32 x 32 diagonal block is factored by one warp (lane = row; each entry's sum
// in increasing column order as in choldc) and the rows below solve against it (thread per
// row). A non-positive pivot zero-fills the matrix, as choldc does. Reads the lower triangle,
// writes the factor over it; the strict upper triangle is left as it was.
// The factorization of one matrix A (P x P, ld P) by the CTA (256 threads); `sm` is the dynamic
// shared memory (potrf_panel_smem(P) bytes), `fail` a shared flag. Used by k_potrf_panel (one
// matrix per CTA) and by the persistent IRLS tail (k_irls_tail, matrices from a queue).
__device__ __forceinline__ void potrf_panel_one(double* __restrict__ A, int P, double* sm, int& fail) {
  const int rows_pad = (P + 15) / 16 * 16;
  const int SA = rows_pad + 4;                 // La[q][r]: rows contiguous, 4 mod 16
  double* Ap = sm;                             // [rows_pad][IS]: the panel, Ap[r][c]
  double* La = Ap + (size_t)rows_pad * IS;     // [2][CW][SA]: finished columns, one CW-chunk
  double* Rd = La + 2 * (size_t)CW * SA;       // [32] reciprocals of the diagonal
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int nb = (P + IB - 1) / IB;
  if (tid == 0) fail = 0;
  for (int kp = 0; kp < nb; kp++) {
    const int c0 = kp * IB, rows = P - c0, ncol = min(IB, rows);
    const int rpad = (rows + 15) / 16 * 16;
    // the panel's lower part: rows c0.., columns c0..c0+ncol
    for (int e = tid; e < rpad * IB; e += blockDim.x) {  // rows fastest: coalesced columns
      const int cc = e / rpad, r = e - cc * rpad;
      Ap[r * IS + cc] = (r < rows && cc < ncol) ? A[(size_t)(c0 + r) + (size_t)(c0 + cc) * P] : 0.0;
    }
    if (kp > 0) {
      // Ap -= L[c0.., 0..c0) L[c0..c0+32, 0..c0)^T, CW finished columns per chunk
      double acc[2][4][4];
#pragma unroll
      for (int x = 0; x < 2; x++)
#pragma unroll
        for (int y = 0; y < 4; y++)
#pragma unroll
          for (int z = 0; z < 4; z++) acc[x][y][z] = 0.0;
      auto stage = [&](int ch, int buf) {
        double* dst = La + (size_t)buf * CW * SA;
        for (int e = tid; e < CW * rpad; e += blockDim.x) {
          const int q = e / rpad, r = e - q * rpad;
          const bool ok = r < rows;
          cp_async8(dst + q * SA + r, A + (ok ? (size_t)(c0 + r) + (size_t)(ch * CW + q) * P : 0), ok ? 8 : 0);
        }
        cp_async_commit();
      };
      stage(0, 0);
      const int nch = c0 / CW;
      for (int ch = 0; ch < nch; ch++) {
        if (ch + 1 < nch) {
          stage(ch + 1, (ch + 1) & 1);
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
        __syncthreads();
        const double* la = La + (size_t)(ch & 1) * CW * SA;
#pragma unroll
        for (int k4 = 0; k4 < CW / 4; k4++) {
          const double* lr = la + (k4 * 4 + t) * SA;
          double b[4];
#pragma unroll
          for (int y = 0; y < 4; y++) b[y] = lr[y * 8 + g];  // B[k][n] = L[c0 + n][q]
#pragma unroll
          for (int x = 0; x < 2; x++) {
            const int mt = warp + 8 * x;
            if (mt * 16 < rpad) {
              const double a0 = lr[mt * 16 + g], a1 = lr[mt * 16 + g + 8];
#pragma unroll
              for (int y = 0; y < 4; y++) dmma_16x8x4(acc[x][y], a0, a1, b[y]);
            }
          }
        }
        __syncthreads();
      }
#pragma unroll
      for (int x = 0; x < 2; x++) {
        const int mt = warp + 8 * x;
        if (mt * 16 >= rpad) continue;
#pragma unroll
        for (int y = 0; y < 4; y++)
#pragma unroll
          for (int h = 0; h < 2; h++)
#pragma unroll
            for (int e = 0; e < 2; e++) Ap[(mt * 16 + g + 8 * h) * IS + y * 8 + 2 * t + e] -= acc[x][y][2 * h + e];
      }
    }
    __syncthreads();
    // The diagonal block, one warp, right-looking with row `lane` in registers; then the rows
    // below it, thread per row, the same way. Entry (r, q) still takes its products
    // l_rk l_qk in increasing k and is scaled by 1/l_qq last, as choldc's sums: the same
    // operations in the same order as the entry-by-entry form, with independent FMAs in place
    // of one dependent chain per entry.
    if (warp == 0) {
      // rows past the panel (ncol < 32 only when P - c0 < 32, where the panel may hold 16 rows)
      // are zeros in registers and never touch shared memory
      double a[IB];
#pragma unroll
      for (int q = 0; q < IB; q++) a[q] = lane < ncol ? Ap[lane * IS + q] : 0.0;
#pragma unroll
      for (int cc = 0; cc < IB; cc++) {
        if (cc < ncol) {
          const double piv = __shfl_sync(0xffffffffu, a[cc], cc);
          const double l = sqrt(piv);
          const double rd = 1.0 / l;
          if (lane == cc) {
            if (piv <= 0.0) fail = 1;  // a NaN pivot passes, as in choldc
            a[cc] = l;
            Rd[cc] = rd;
          } else if (lane > cc) {
            a[cc] = a[cc] * rd;
          }
#pragma unroll
          for (int q = cc + 1; q < IB; q++) {
            const double lq = __shfl_sync(0xffffffffu, a[cc], q);
            a[q] -= a[cc] * lq;
          }
        }
      }
      if (lane < ncol)
#pragma unroll
        for (int q = 0; q < IB; q++) Ap[lane * IS + q] = a[q];
    }
    __syncthreads();
    for (int r = IB + tid; r < rows; r += blockDim.x) {
      double a[IB];
#pragma unroll
      for (int q = 0; q < IB; q++) a[q] = Ap[r * IS + q];
#pragma unroll
      for (int cc = 0; cc < IB; cc++) {
        if (cc < ncol) {
          const double x = a[cc] * Rd[cc];
          a[cc] = x;
#pragma unroll
          for (int q = cc + 1; q < IB; q++) a[q] -= x * Ap[q * IS + cc];
        }
      }
#pragma unroll
      for (int q = 0; q < IB; q++) Ap[r * IS + q] = a[q];
    }
    __syncthreads();
    for (int e = tid; e < rows * IB; e += blockDim.x) {
      const int cc = e / rows, r = e - cc * rows;
      if (cc < ncol && r >= cc) A[(size_t)(c0 + r) + (size_t)(c0 + cc) * P] = Ap[r * IS + cc];
    }
    __threadfence_block();
    __syncthreads();
  }
  if (fail)
    for (int e = tid; e < P * P; e += blockDim.x) A[e] = 0.0;
}

__global__ void __launch_bounds__(256, 2) k_potrf_panel(double* __restrict__ Psi, int P, int64_t stride) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int fail;
  potrf_panel_one(Psi + (size_t)blockIdx.x * stride, P, sm, fail);
}

int potrf_panel_smem(int P) {
  const int rows_pad = (P + 15) / 16 * 16;
  return (int)sizeof(double) * (rows_pad * IS + 2 * CW * (rows_pad + 4) + IB);
}

int launch_potrf_panels(Ctx* c, double* A, int n, int batch, int64_t stride) {
  const int smem = potrf_panel_smem(n);
  if (n > kPotrfMaxP || smem > 220 * 1024) return GPL_ERR_ARG;
  GPL_TRY(c, cudaFuncSetAttribute(k_potrf_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  GPL_TRY(c, cudaFuncSetAttribute(k_potrf_panel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  k_potrf_panel<<<batch, 256, smem, c->stream>>>(A, n, stride);
  GPL_LAUNCHED(c, "k_potrf_panel");
  return GPL_OK;
}

// trtri: the panel's rows, two 32-column chunks of L, the diagonal and right-hand-side blocks;
// lauum needs less (the panel's rows and two chunks). About 107 KB at P = 236: two CTAs per SM.
int inverse_panel_smem(int P) {
  const int nb = (P + IB - 1) / IB;
  return (int)sizeof(double) * (nb * IB * IS + 2 * IB * IS + 2 * IB * LS + IB);
}

// Returns GPL_ERR_ARG when P is beyond the panel kernels' checked range.
int launch_inverse_panels(Ctx* c) {
  const int P = c->P;
  const int smem = inverse_panel_smem(P);
  if (P > kInverseMaxP || smem > 220 * 1024) return GPL_ERR_ARG;
  GPL_TRY(c, cudaFuncSetAttribute(k_trtri_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  GPL_TRY(c, cudaFuncSetAttribute(k_lauum_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  GPL_TRY(c, cudaFuncSetAttribute(k_trtri_panel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  GPL_TRY(c, cudaFuncSetAttribute(k_lauum_panel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  const int64_t st = (int64_t)P * P;
  const int nb = (P + IB - 1) / IB;
  dim3 g(nb, c->J);
  k_trtri_panel<<<g, 256, smem, c->stream>>>(c->Psi, P, st, c->scratch);
  GPL_LAUNCHED(c, "k_trtri_panel");
  k_lauum_panel<<<g, 256, smem, c->stream>>>(c->scratch, P, st, c->PsiInv);
  GPL_LAUNCHED(c, "k_lauum_panel");
  return GPL_OK;
}

}  // namespace gpl

namespace gpl {

// The per-gene tail of one IRLS sweep as ONE persistent launch (getBetaPhi's cholPsi, cholsl and
// coefficient update, then getLkhdPois: ggplvm.cu:683-692, 418-464, 703-724). Each CTA takes
// genes from a queue (an atomic head over `order`, the genes by decreasing matched count, so that
// the genes with the most counts start first and the short ones fill the end) and for each gene:
//   1. factors Psi_j in place (potrf_panel_one, as k_potrf_panel);
//   2. solves L L^T x = b_j with one warp, in k_solve's operation order, and stores x (sol);
//   3. beta_j <- (1 - r) beta_j + r x and phi_j from nu^T diag(W/Omega) nu - |L^T beta_j|^2 with
//      the reference's clamps, in k_beta_phi's order;
//   4. the Poisson log-likelihood of the gene's matched counts, in k_lkhd_pois's order.
// Every sum is taken in the same per-thread order and reduced by the same block tree as in the
// separate kernels, so the results are the same bits; which CTA takes which gene changes nothing.
// The W and nu columns are read once for steps 3 and 4 together.
__global__ void __launch_bounds__(256, 2)
    k_irls_tail(int J, int N, int ldN, int P, int pvars, double r, double wt, double* __restrict__ Psi,
                const double* __restrict__ bvec, double* __restrict__ sol, double* __restrict__ Beta,
                double* __restrict__ phi, const double* __restrict__ W, const double* __restrict__ Nu,
                const double* __restrict__ Omega, const double* __restrict__ delta,
                const double* __restrict__ titsias, const int32_t* __restrict__ cell,
                const int64_t* __restrict__ gptr, const int32_t* __restrict__ gvalid,
                const double* __restrict__ cnt, double* __restrict__ lkhds, const int* __restrict__ order,
                int* __restrict__ head) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int fail, next;
  __shared__ double sh[32];
  const int rows_pad = (P + 15) / 16 * 16;
  double* y = sm + (size_t)rows_pad * IS + 2 * (size_t)CW * (rows_pad + 4) + IB;  // past the panel's space
  double* sb = y + P;
  double* dg = sb + P;  // the factor's diagonal
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  const int64_t PP = (int64_t)P * P;
  for (;;) {
    __syncthreads();  // the previous gene's shared values are no longer read
    if (tid == 0) next = atomicAdd(head, 1);
    __syncthreads();
    const int q = next;
    if (q >= J) break;
    const int j = order[q];
    double* L = Psi + (size_t)j * PP;
    potrf_panel_one(L, P, sm, fail);
    __syncthreads();
    // 2. (L L^T) x = b_j, one warp, in k_solve's operation order (lane l updates the rows
    // k + 1 + l + 32 m of column k, and sums the rows i + 1 + l + 32 m of row i's column); the
    // next column's entries are loaded into registers while the current one is applied, so the
    // dependent chain does not wait on a global load per step
    if (wid == 0) {
      constexpr int NR = (kPotrfMaxP + 31) / 32;  // rows per lane
      const double* rhs = bvec + (size_t)j * P;
      for (int i = lane; i < P; i += 32) {
        y[i] = rhs[i];
        dg[i] = L[i + (size_t)i * P];
      }
      __syncwarp();
      double cur[NR], nxt[NR];
#pragma unroll
      for (int m = 0; m < NR; m++) {
        const int i = 1 + lane + 32 * m;
        cur[m] = i < P ? L[i] : 0.0;
      }
      for (int k = 0; k < P; k++) {
        if (k + 1 < P) {
#pragma unroll
          for (int m = 0; m < NR; m++) {
            const int i = k + 2 + lane + 32 * m;
            nxt[m] = i < P ? L[i + (size_t)(k + 1) * P] : 0.0;
          }
        }
        const double xk = y[k] / dg[k];
        __syncwarp();
        if (lane == 0) y[k] = xk;
#pragma unroll
        for (int m = 0; m < NR; m++) {
          const int i = k + 1 + lane + 32 * m;
          if (i < P) y[i] -= cur[m] * xk;
        }
        __syncwarp();
#pragma unroll
        for (int m = 0; m < NR; m++) cur[m] = nxt[m];
      }
#pragma unroll
      for (int m = 0; m < NR; m++) cur[m] = 0.0;  // column P - 1 has no rows below the diagonal
      for (int i = P - 1; i >= 0; i--) {
        if (i > 0) {
#pragma unroll
          for (int m = 0; m < NR; m++) {
            const int k = i + lane + 32 * m;
            nxt[m] = k < P ? L[k + (size_t)(i - 1) * P] : 0.0;
          }
        }
        double part = 0.0;
#pragma unroll
        for (int m = 0; m < NR; m++) {
          const int k = i + 1 + lane + 32 * m;
          if (k < P) part += cur[m] * y[k];
        }
        part = warp_sum(part);
        const double xi = (y[i] - part) / dg[i];
        __syncwarp();
        if (lane == 0) y[i] = xi;
        __syncwarp();
#pragma unroll
        for (int m = 0; m < NR; m++) cur[m] = nxt[m];
      }
      double* x = sol + (size_t)j * P;
      for (int i = lane; i < P; i += 32) x[i] = y[i];
    }
    // 3. and 4.: one pass over the gene's cells for both per-cell sums
    const double* Wj = W + (size_t)j * ldN;
    const double* nj = Nu + (size_t)j * ldN;
    double qpart = 0.0, lpart = 0.0;
    for (int i = tid; i < N; i += blockDim.x) {
      qpart += nj[i] * nj[i] * Wj[i] / Omega[i];
      lpart -= Wj[i];
    }
    const int64_t b0 = gptr[j], b1 = gptr[j] + gvalid[j];
    const double dgp = delta[pvars - 1];
    for (int64_t l = b0 + tid; l < b1; l += blockDim.x) {
      const int i = cell[l];
      lpart += (log(Wj[i]) - dgp * titsias[i] * wt) * cnt[l];
    }
    const double quad = block_sum(qpart, sh);  // syncs: the solution y is complete
    double* bj = Beta + (size_t)j * P;
    for (int k = tid; k < P; k += blockDim.x) {
      const double nb = bj[k] * (1 - r) + y[k] * r;
      bj[k] = nb;
      sb[k] = nb;
    }
    __syncthreads();
    double sq = 0.0;
    for (int k = wid; k < P; k += nw) {
      double t = 0.0;
      for (int i = k + lane; i < P; i += 32) t += L[i + (size_t)k * P] * sb[i];
      t = warp_sum(t);
      sq += t * t;
    }
    if (lane != 0) sq = 0.0;
    const double s2 = block_sum(sq, sh);
    const double lk = block_sum(lpart, sh);
    if (tid == 0) {
      double ph = (quad - s2) / (double)N;
      if (isnan(ph)) ph = 1.0;
      if (ph < 0.0) ph = 1.0;
      if (ph < 0.01) ph = 0.01;
      if (ph > 1000.0) ph = 1000.0;
      phi[j] = ph;
      lkhds[j] = lk;
    }
  }
}

int irls_tail_smem(int P) { return potrf_panel_smem(P) + 3 * (int)sizeof(double) * P; }

// GPL_ERR_ARG when the fused tail does not apply (P beyond the panel Cholesky's range).
int launch_irls_tail(Ctx* c, int jtr, int ctas_per_sm) {
  const int P = c->P;
  const int smem = irls_tail_smem(P);
  if (P > kPotrfMaxP || smem > 220 * 1024 || !c->gene_order_d) return GPL_ERR_ARG;
  GPL_TRY(c, cudaFuncSetAttribute(k_irls_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  GPL_TRY(c, cudaFuncSetAttribute(k_irls_tail, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  double r = (double)(jtr + 1) / 100.0;  // the damping of getBetaPhi (ggplvm.cu:426)
  if (jtr > 100) r = 1.0;
  Tunable* tu = nullptr;
  ctas_per_sm = tune_pick(c, "irls_tail", {1, 2}, ctas_per_sm, &tu);
  const int grid = std::max(1, std::min(c->J, std::max(1, ctas_per_sm) * c->sm_count));
  GPL_TRY(c, cudaMemsetAsync(c->queue_head_d, 0, sizeof(int), c->stream));
  ProfScope ps(c, "irls_tail");
  TuneScope ts(c, tu);
  k_irls_tail<<<grid, 256, smem, c->stream>>>(c->J, c->N, c->ldN, P, c->p, r, c->vcomp ? 1.0 : kWt, c->Psi, c->bvec,
                                              c->sol, c->Beta, c->phi, c->W, c->Nu, c->Omega, c->delta,
                                              c->titsias, c->cell, c->gptr, c->gvalid, c->cnt, c->lkhds,
                                              c->gene_order_d, c->queue_head_d);
  GPL_LAUNCHED(c, "k_irls_tail");
  return GPL_OK;
}

}  // namespace gpl
