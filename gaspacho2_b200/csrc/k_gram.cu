// Per-gene Gram matrices and their factorisations (replaces getPsi ggplvm.cu:621-680,
// cholPsi :683-692, cholDeltaInv :695-700, cholKmm kernel_funcs.cu:139-143, solvePsi
// ggplvm.cu:46-53, choldc/cholsl chol.cu:19-97, initPsi init.cu:125-181).
//
//   k_gram      dense x dense block of Psi_j = Z^T diag(W_j / Omega) Z + DeltaInv over the
//               dense model columns (the categorical rows come from the group sums), all
//               genes, scattered to the model-column positions. A CTA owns a 32x32
//               block pair (upper triangle of blocks) for 8 genes and streams every cell:
//               Z column blocks and the weights for a 32-cell chunk go to shared memory,
//               each thread accumulates a 4x8 tile for one gene in registers.
//               Roofline: FP64 FMA, N*J*P^2/2 multiply-adds.
//   k_chol      batched in-place Cholesky, one CTA per matrix, left-looking by columns:
//               the update of column j reads row j of the factor (broadcast) and the rows
//               below it (coalesced). A non-positive pivot zero-fills the matrix, as
//               choldc does.
//   k_solve     batched (L L^T) x = b, one warp per system: forward substitution column-
//               oriented (coalesced), back substitution as warp dot products.
//   k_trtri     V = L^{-1} (row-major scratch), one thread per column of V.
//   k_lauum     Psi^{-1} = V^T V, full symmetric, column-major.
#include "gpl_internal.cuh"

namespace gpl {

namespace {
constexpr int GB = 32;   // column block
constexpr int GG = 8;    // genes per CTA
constexpr int GC = 32;   // cells per chunk
}  // namespace

__global__ void __launch_bounds__(256) k_gram(int N, int ldN, int n_d, int P, int J, const double* __restrict__ Z,
                                              const int* __restrict__ dcol, const double* __restrict__ W,
                                              const double* __restrict__ Omega, const double* __restrict__ Dinv,
                                              double* __restrict__ Psi, int unweighted) {
  __shared__ double sk[GC][GB + 1];
  __shared__ double sl[GC][GB + 1];
  __shared__ double sw[GC][GG];
  // blockIdx.x enumerates block pairs (kb <= lb) of the upper triangle
  int lbi = (int)((sqrt(8.0 * blockIdx.x + 1.0) - 1.0) * 0.5);
  while ((lbi + 1) * (lbi + 2) / 2 <= (int)blockIdx.x) lbi++;
  while (lbi * (lbi + 1) / 2 > (int)blockIdx.x) lbi--;
  const int kbi = (int)blockIdx.x - lbi * (lbi + 1) / 2;
  const int kb = kbi * GB, lb = lbi * GB;
  const int j0 = blockIdx.y * GG;
  const int tid = threadIdx.x;
  const int g = tid >> 5, kq = (tid & 31) >> 2, lq = tid & 3;
  double acc[4][8];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 8; b++) acc[a][b] = 0.0;

  for (int i0 = 0; i0 < N; i0 += GC) {
    // load 32 cells x 32 columns of each block (cell fastest in memory)
    for (int e = tid; e < GC * GB; e += 256) {
      const int r = e & (GC - 1), col = e >> 5;
      const int i = i0 + r;
      const int ck = kb + col, cl = lb + col;
      sk[r][col] = (i < N && ck < n_d) ? Z[(size_t)ck * ldN + i] : 0.0;
      sl[r][col] = (i < N && cl < n_d) ? Z[(size_t)cl * ldN + i] : 0.0;
    }
    {
      const int r = tid & (GC - 1), gg = tid >> 5;
      const int i = i0 + r, j = j0 + gg;
      double w = 0.0;
      if (i < N && j < J) w = unweighted ? 1.0 : W[(size_t)j * ldN + i] / Omega[i];
      sw[r][gg] = w;
    }
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < GC; r++) {
      const double w = sw[r][g];
      double a[4], b[8];
#pragma unroll
      for (int x = 0; x < 4; x++) a[x] = sk[r][kq * 4 + x] * w;
#pragma unroll
      for (int y = 0; y < 8; y++) b[y] = sl[r][lq * 8 + y];
#pragma unroll
      for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 8; y++) acc[x][y] = fma(a[x], b[y], acc[x][y]);
    }
    __syncthreads();
  }
  const int j = j0 + g;
  if (j >= J) return;
  double* Pj = Psi + (size_t)j * P * P;
#pragma unroll
  for (int x = 0; x < 4; x++) {
    const int k = kb + kq * 4 + x;
    if (k >= n_d) continue;
#pragma unroll
    for (int y = 0; y < 8; y++) {
      const int l = lb + lq * 8 + y;
      if (l >= n_d || k > l) continue;
      const size_t mk = dcol[k], ml = dcol[l];  // model columns, mk <= ml
      const double v = acc[x][y] + Dinv[mk + ml * P];
      Pj[mk + ml * P] = v;
      Pj[ml + mk * P] = v;
    }
  }
}

// Left-looking Cholesky of n x n matrices A_b = A + b*stride (col-major, ld n). The input is
// read from the upper triangle (src_upper) or the lower one; the factor overwrites the
// lower triangle and the diagonal; the strict upper triangle is left as it was.
__global__ void __launch_bounds__(256) k_chol(double* __restrict__ A, int n, int64_t stride, int src_upper) {
  __shared__ double sh[32];
  __shared__ int fail;
  double* a = A + (size_t)blockIdx.x * stride;
  const int tid = threadIdx.x;
  if (tid == 0) fail = 0;
  __syncthreads();
  for (int j = 0; j < n; j++) {
    // pivot: d = A(j,j) - sum_k L(j,k)^2
    double part = 0.0;
    for (int k = tid; k < j; k += blockDim.x) {
      const double l = a[j + (size_t)k * n];
      part = fma(l, l, part);
    }
    const double s = block_sum(part, sh);
    const double d = a[j + (size_t)j * n] - s;
    if (d <= 0.0) fail = 1;  // a NaN pivot passes, as in choldc, and yields a NaN factor
    __syncthreads();
    if (fail) break;
    const double ljj = sqrt(d);
    for (int i = j + 1 + tid; i < n; i += blockDim.x) {
      double acc = src_upper ? a[j + (size_t)i * n] : a[i + (size_t)j * n];
      for (int k = j - 1; k >= 0; k--) acc -= a[i + (size_t)k * n] * a[j + (size_t)k * n];
      a[i + (size_t)j * n] = acc / ljj;
    }
    __syncthreads();
    if (tid == 0) a[j + (size_t)j * n] = ljj;
    __syncthreads();
  }
  if (fail) {
    for (int e = tid; e < n * n; e += blockDim.x) a[e] = 0.0;
  }
}

// Single-matrix Cholesky in choldc's exact operation order (chol.cu:19-43): row i of the
// factor is finished before row i+1, each entry's sum runs k = i-1 .. 0, and no multiply-add
// is contracted, so identical inputs give the host reference's bits (sqrt and division are
// correctly rounded on both). Used for the small, often ill-conditioned matrices: Kmm (no
// jitter in the reference), the prior precision DeltaInv and the GLM initialisation Gram.
// Reads the upper triangle, writes the factor into the lower one; zero-fills on a
// non-positive pivot. One CTA.
__global__ void __launch_bounds__(256) k_chol_exact(double* __restrict__ a, int n) {
  __shared__ int fail;
  if (threadIdx.x == 0) fail = 0;
  __syncthreads();
  for (int i = 0; i < n; i++) {
    // sums for j = i .. n-1 (j = i is the pivot)
    double sums[4];
    int cnt = 0;
    for (int j = i + threadIdx.x; j < n && cnt < 4; j += blockDim.x, cnt++) {
      double sum = a[i + (size_t)j * n];
      for (int k = i - 1; k >= 0; k--) sum = __dsub_rn(sum, __dmul_rn(a[i + (size_t)k * n], a[j + (size_t)k * n]));
      sums[cnt] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (sums[0] <= 0.0) fail = 1;
      else a[i + (size_t)i * n] = __dsqrt_rn(sums[0]);
    }
    __syncthreads();
    if (fail) break;
    const double lii = a[i + (size_t)i * n];
    cnt = 0;
    for (int j = i + threadIdx.x; j < n && cnt < 4; j += blockDim.x, cnt++)
      if (j > i) a[j + (size_t)i * n] = __ddiv_rn(sums[cnt], lii);
    __syncthreads();
  }
  if (fail)
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) a[e] = 0.0;
}

// Columns of (L L^T)^{-1} in cholsl's order (chol.cu:45-56), thread per column, no
// contraction: the Kmm^{-1} of getC2 (ggplvm.cu:93-95). Y is an n x n scratch (col-major).
__global__ void k_cholinv_exact(const double* __restrict__ a, int n, double* __restrict__ Y) {
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < n; col += gridDim.x * blockDim.x) {
    double* x = Y + (size_t)col * n;
    for (int i = 0; i < n; i++) {
      double sum = (i == col) ? 1.0 : 0.0;
      for (int k = i - 1; k >= 0; k--) sum = __dsub_rn(sum, __dmul_rn(a[i + (size_t)k * n], x[k]));
      x[i] = __ddiv_rn(sum, a[i + (size_t)i * n]);
    }
    for (int i = n - 1; i >= 0; i--) {
      double sum = x[i];
      for (int k = i + 1; k < n; k++) sum = __dsub_rn(sum, __dmul_rn(a[k + (size_t)i * n], x[k]));
      x[i] = __ddiv_rn(sum, a[i + (size_t)i * n]);
    }
  }
}

// (L L^T) x = b for `batch` systems, one warp each; y in shared memory.
__global__ void k_solve(const double* __restrict__ L, int n, int64_t lstride, const double* __restrict__ B,
                        int64_t bstride, double* __restrict__ X, int64_t xstride, int batch) {
  extern __shared__ double sy[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * (blockDim.x >> 5) + warp;
  if (b >= batch) return;
  double* y = sy + (size_t)warp * n;
  const double* a = L + (size_t)b * lstride;
  const double* rhs = B + (size_t)b * bstride;
  double* x = X + (size_t)b * xstride;
  for (int i = lane; i < n; i += 32) y[i] = rhs[i];
  __syncwarp();
  for (int k = 0; k < n; k++) {
    const double xk = y[k] / a[k + (size_t)k * n];
    __syncwarp();
    if (lane == 0) y[k] = xk;
    for (int i = k + 1 + lane; i < n; i += 32) y[i] -= a[i + (size_t)k * n] * xk;
    __syncwarp();
  }
  for (int i = n - 1; i >= 0; i--) {
    double part = 0.0;
    for (int k = i + 1 + lane; k < n; k += 32) part += a[k + (size_t)i * n] * y[k];
    part = warp_sum(part);
    const double xi = (y[i] - part) / a[i + (size_t)i * n];
    __syncwarp();
    if (lane == 0) y[i] = xi;
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) x[i] = y[i];
}

// V = L^{-1}, row-major into Vrm (V[m][k] at m*n + k); thread per column k of V.
__global__ void k_trtri(const double* __restrict__ L, int n, int64_t stride, double* __restrict__ Vrm) {
  const double* a = L + (size_t)blockIdx.x * stride;
  double* v = Vrm + (size_t)blockIdx.x * stride;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    for (int i = 0; i < k; i++) v[(size_t)i * n + k] = 0.0;
    v[(size_t)k * n + k] = 1.0 / a[k + (size_t)k * n];
    for (int i = k + 1; i < n; i++) {
      double acc = 0.0;
      for (int m = k; m < i; m++) acc = fma(a[i + (size_t)m * n], v[(size_t)m * n + k], acc);
      v[(size_t)i * n + k] = -acc / a[i + (size_t)i * n];
    }
  }
}

// S = V^T V with V lower triangular (row-major); S full symmetric col-major.
__global__ void k_lauum(const double* __restrict__ Vrm, int n, int64_t stride, double* __restrict__ S) {
  const double* v = Vrm + (size_t)blockIdx.x * stride;
  double* s = S + (size_t)blockIdx.x * stride;
  for (int b = threadIdx.x; b < n; b += blockDim.x) {
    for (int a = 0; a <= b; a++) {
      double acc = 0.0;
      for (int i = b; i < n; i++) acc = fma(v[(size_t)i * n + a], v[(size_t)i * n + b], acc);
      s[a + (size_t)b * n] = acc;
      s[b + (size_t)a * n] = acc;
    }
  }
}

int launch_gram(Ctx* c, bool unweighted) {
  const int nb = div_up(c->n_d, GB);
  const int npairs = nb * (nb + 1) / 2;
  const int J = unweighted ? 1 : c->J;
  int rc = GPL_ERR_ARG;
  if (!unweighted) rc = c->precision == GPL_PREC_BF16X3 ? launch_tc_gram(c) : launch_pair_gram(c);
  if (rc != GPL_OK && !(rc == GPL_ERR_ARG && (unweighted || c->precision == GPL_PREC_FP64))) return rc;
  if (rc == GPL_ERR_ARG) {
    // the unweighted Gram of one gene (GLM initialisation), or more dense columns than the
    // staged pair contraction holds
    ProfScope ps(c, "gram");
    dim3 g(npairs, div_up(J, GG));
    k_gram<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->n_d, c->P, J, c->Dm, c->dcol_d, c->W, c->Omega, c->DeltaInv,
                                     c->Psi, unweighted ? 1 : 0);
    GPL_LAUNCHED(c, "k_gram");
  }
  rc = launch_group_sums(c, unweighted ? 1 : 0);
  if (rc) return rc;
  return launch_assemble_psi(c, J);
}

int launch_chol_batched(Ctx* c, double* A, int n, int batch, int64_t stride) {
  ProfScope ps(c, "chol");
  {
    const int rc = launch_potrf_panels(c, A, n, batch, stride);
    if (rc != GPL_ERR_ARG) return rc;  // GPL_ERR_ARG: n beyond the panel kernel's checked range
  }
  k_chol<<<batch, 256, 0, c->stream>>>(A, n, stride, 0);
  GPL_LAUNCHED(c, "k_chol");
  return GPL_OK;
}

int launch_chol_single(Ctx* c, double* A, int n) {
  ProfScope ps(c, "chol_small");
  if (n > 4 * 256) {  // wider than the exact kernel's per-thread row slots
    k_chol<<<1, 256, 0, c->stream>>>(A, n, 0, 1);
    GPL_LAUNCHED(c, "k_chol");
    return GPL_OK;
  }
  k_chol_exact<<<1, 256, 0, c->stream>>>(A, n);
  GPL_LAUNCHED(c, "k_chol_exact");
  return GPL_OK;
}

cudaError_t launch_chol_exact_raw(cudaStream_t st, double* A, int n) {
  void* args[] = {&A, &n};
  return cudaLaunchKernel((const void*)k_chol_exact, dim3(1), dim3(256), args, 0, st);
}

int launch_cholinv_exact(Ctx* c, const double* L, int n, double* out) {
  k_cholinv_exact<<<div_up(n, 64), 64, 0, c->stream>>>(L, n, out);
  GPL_LAUNCHED(c, "k_cholinv_exact");
  return GPL_OK;
}

int launch_solve_batched(Ctx* c, const double* L, int n, int64_t lstride, const double* B, int64_t bstride,
                         double* X, int64_t xstride, int batch) {
  ProfScope ps(c, "solve");
  const int warps = 4;
  const size_t shm = sizeof(double) * (size_t)n * warps;
  if (shm > 48 * 1024) {
    GPL_TRY(c, cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
  }
  k_solve<<<div_up(batch, warps), 32 * warps, shm, c->stream>>>(L, n, lstride, B, bstride, X, xstride, batch);
  GPL_LAUNCHED(c, "k_solve");
  return GPL_OK;
}

int launch_inverse_batched(Ctx* c) {
  const int64_t st = (int64_t)c->P * c->P;
  ProfScope ps(c, "inverse");
  {
    const int rc = launch_inverse_panels(c);
    if (rc != GPL_ERR_ARG) return rc;  // GPL_ERR_ARG: P beyond the panel kernels' checked range
  }
  k_trtri<<<c->J, 256, 0, c->stream>>>(c->Psi, c->P, st, c->scratch);
  GPL_LAUNCHED(c, "k_trtri");
  k_lauum<<<c->J, 256, 0, c->stream>>>(c->scratch, c->P, st, c->PsiInv);
  GPL_LAUNCHED(c, "k_lauum");
  return GPL_OK;
}

int launch_inverse_single(Ctx* c, const double* L, int n, double* tmp, double* out) {
  k_trtri<<<1, 256, 0, c->stream>>>(L, n, 0, tmp);
  GPL_LAUNCHED(c, "k_trtri");
  k_lauum<<<1, 256, 0, c->stream>>>(tmp, n, 0, out);
  GPL_LAUNCHED(c, "k_lauum");
  return GPL_OK;
}

}  // namespace gpl
