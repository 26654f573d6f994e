// Kernel matrices of the sparse GP (replaces kernel_funcs.cu:61-162 and util_cuda.cu:249-269).
//
//   k_knm        Knm[i, m] = exp(-(sin^2((x_i0 - t_m0)/2)/rho_0 + sum_q>=1 (x_iq - t_mq)^2/(2 rho_q)))
//                written into the model matrix's GP block (column-major, cell fastest); with
//                lv >= 0 only latent dimension lv enters (the DE driver's per-dimension models).
//                Bound: N*M*Q transcendental work, ~2% of one objective evaluation.
//   k_kmm        Kmm (upper, unit diagonal, zero lower) and its copy Kinv.
//   k_kinvkmn    per cell: x = Kmm^{-1} k_n by two triangular solves against the factor in
//                Kinv's lower triangle (cholslg order), titsias_n = (1 - k_n . x)/2.
//                One thread per cell; the factor is read by every thread at the same
//                address (broadcast), the solution lives in a cell-fastest scratch so the
//                per-step loads coalesce.
//   k_expand     DeltaInv = blockdiag(1/delta_k I, Kmm/delta_GP), upper + diagonal.
#include <algorithm>

#include "gpl_internal.cuh"

namespace gpl {

// Squared-distance sum of one point pair: all latent dimensions (periodic dim 0, ARD dims
// >= 1; getKernelMatsWithPer) when lv < 0, dimension lv alone otherwise
// (getKernelMatsWithPerSpecificLV, kernel_funcs.cu:101-135), in the reference's order.
__device__ __forceinline__ double kern_sum(const double* __restrict__ A, size_t lda, int a,
                                           const double* __restrict__ B, int ldb, int b,
                                           const double* __restrict__ rho, int Q, int lv) {
  double sum = 0.0, t;
  if (lv <= 0) {
    t = sin((A[a] - B[b]) / 2.0);
    sum += t * t / rho[0];
  }
  const int k0 = lv < 0 ? 1 : lv, k1 = lv < 0 ? Q : (lv == 0 ? 0 : lv + 1);
  for (int k = k0; k < k1; k++) {
    t = A[a + k * lda] - B[b + k * ldb];
    sum += t * t / 2.0 / rho[k];
  }
  return sum;
}

__global__ void k_knm(int N, int ldN, int M, int Q, int lv, const double* __restrict__ X,
                      const double* __restrict__ T, const double* __restrict__ rho, double* __restrict__ Knm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= N) return;
  Knm[i + (size_t)j * ldN] = exp(-kern_sum(X, (size_t)N, i, T, M, j, rho, Q, lv));
}

__global__ void k_kmm(int M, int Q, int lv, const double* __restrict__ T, const double* __restrict__ rho,
                      double* __restrict__ K, double* __restrict__ Kinv) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (ii >= M) return;
  double val;
  if (ii == j) val = 1.0;
  else if (ii > j) val = 0.0;
  else val = exp(-kern_sum(T, (size_t)M, ii, T, M, j, rho, Q, lv));
  K[ii + j * M] = val;
  if (Kinv) Kinv[ii + j * M] = val;  // no copy when the caller needs Kmm once (Kinv == nullptr)
}

// The DE driver's null model as a design whose GP block is inert: Knm = 0, Kmm = Kinv = I,
// Kmm^{-1} k_n = 0, titsias = 0 (initTitsias). The GP columns then decouple from the rest of
// every Psi_j (their Gram entries vanish, DeltaInv holds 1/delta_GP on their diagonal), and
// their coefficients stay 0.
__global__ void k_gp_null(int N, int ldN, int M, double* __restrict__ Knm, double* __restrict__ KinvKmn,
                          double* __restrict__ titsias, double* __restrict__ K, double* __restrict__ Kinv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ldN)
    for (int m = 0; m < M; m++) {
      Knm[i + (size_t)m * ldN] = 0.0;
      KinvKmn[i + (size_t)m * ldN] = 0.0;
    }
  if (i < N) titsias[i] = 0.0;
  if (i < M * M) K[i] = Kinv[i] = (i % M == i / M) ? 1.0 : 0.0;
}

// Two triangular solves per cell with the lower factor L (n x n, col-major) held in the
// lower triangle of Kinv; Knm and the solution Y are cell-fastest (ld ldN).
__global__ void k_kinvkmn(int N, int ldN, int M, const double* __restrict__ L, const double* __restrict__ Knm,
                          double* __restrict__ Y, double* __restrict__ titsias) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  // cholslg's order (chol.cu:86-97) without contracted multiply-adds: Kmm has no jitter in
  // the reference and is often nearly singular, so the solve keeps the reference's rounding
  for (int r = 0; r < M; r++) {
    double sum = Knm[i + (size_t)r * ldN];
    for (int k = r - 1; k >= 0; k--) sum = __dsub_rn(sum, __dmul_rn(L[r + k * M], Y[i + (size_t)k * ldN]));
    Y[i + (size_t)r * ldN] = __ddiv_rn(sum, L[r + r * M]);
  }
  for (int r = M - 1; r >= 0; r--) {
    double sum = Y[i + (size_t)r * ldN];
    for (int k = r + 1; k < M; k++) sum = __dsub_rn(sum, __dmul_rn(L[k + r * M], Y[i + (size_t)k * ldN]));
    Y[i + (size_t)r * ldN] = __ddiv_rn(sum, L[r + r * M]);
  }
  double d = 0.0;
  for (int k = 0; k < M; k++) d = __dadd_rn(d, __dmul_rn(Knm[i + (size_t)k * ldN], Y[i + (size_t)k * ldN]));
  titsias[i] = (1.0 - d) / 2.0;
}

__global__ void k_expand(int P, int p, int g0, int M, const int* __restrict__ mk, const double* __restrict__ delta,
                         const double* __restrict__ K, double* __restrict__ D) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = blockIdx.y;
  if (r >= P) return;
  double v = 0.0;
  if (r <= col) {
    if (r >= g0) v = K[(r - g0) + (col - g0) * M] / delta[p - 1];
    else if (r == col) v = 1.0 / delta[mk[r]];
  }
  D[r + (size_t)col * P] = v;
}

int launch_kernel_mats(Ctx* c) { return launch_kernel_mats_lv(c, c->kernel_lv); }

int launch_kernel_mats_lv(Ctx* c, int lv) {
  double* Knm = c->Dm + (size_t)c->dg0 * c->ldN;
  if (lv == kLvNone) {
    ProfScope ps(c, "kernel_mats");
    const int n = std::max(c->ldN, c->M * c->M);
    k_gp_null<<<div_up(n, 256), 256, 0, c->stream>>>(c->N, c->ldN, c->M, Knm, c->KinvKmn, c->titsias, c->Kmm,
                                                     c->Kinv);
    GPL_LAUNCHED(c, "k_gp_null");
    return GPL_OK;
  }
  {
    ProfScope ps(c, "kernel_mats");
    dim3 g(div_up(c->N, 128), c->M);
    k_knm<<<g, 128, 0, c->stream>>>(c->N, c->ldN, c->M, c->Q, lv, c->X, c->T, c->rho, Knm);
    GPL_LAUNCHED(c, "k_knm");
    dim3 g2(div_up(c->M, 64), c->M);
    k_kmm<<<g2, 64, 0, c->stream>>>(c->M, c->Q, lv, c->T, c->rho, c->Kmm, c->Kinv);
    GPL_LAUNCHED(c, "k_kmm");
  }
  int rc = launch_chol_single(c, c->Kinv, c->M);
  if (rc) return rc;
  ProfScope ps(c, "kinvkmn");
  k_kinvkmn<<<div_up(c->N, 128), 128, 0, c->stream>>>(c->N, c->ldN, c->M, c->Kinv, Knm, c->KinvKmn, c->titsias);
  GPL_LAUNCHED(c, "k_kinvkmn");
  return GPL_OK;
}

int launch_expand_delta(Ctx* c) {
  ProfScope ps(c, "expand_delta");
  dim3 g(div_up(c->P, 128), c->P);
  k_expand<<<g, 128, 0, c->stream>>>(c->P, c->p, c->nh[c->p - 1], c->M, c->mk_d, c->delta, c->Kmm, c->DeltaInv);
  GPL_LAUNCHED(c, "k_expand");
  return GPL_OK;
}

// The kernel-matrix sequence on caller-supplied buffers, without a context: Knm and the
// cell-fastest Kmm^{-1} k_n (both N x M, ld N), titsias (N), and an M x M work matrix that
// receives Kmm and then its factor. Each launch goes through cudaLaunchKernel, whose return
// value is that launch's own status (an error left on the thread by earlier, unrelated work is
// neither reported nor cleared). Returns the first failing launch's cudaError_t, else
// cudaSuccess.
int launch_kernel_mats_raw(cudaStream_t st, int N, int M, int Q, const double* X, const double* T,
                           const double* rho, double* Knm, double* KinvKmn, double* titsias, double* Lwork) {
  int ldN = N, lv = kLvAll;
  double* no_copy = nullptr;
  void* a_knm[] = {&N, &ldN, &M, &Q, &lv, &X, &T, &rho, &Knm};
  cudaError_t e = cudaLaunchKernel((const void*)k_knm, dim3(div_up(N, 128), M), dim3(128), a_knm, 0, st);
  if (e != cudaSuccess) return (int)e;
  void* a_kmm[] = {&M, &Q, &lv, &T, &rho, &Lwork, &no_copy};
  e = cudaLaunchKernel((const void*)k_kmm, dim3(div_up(M, 64), M), dim3(64), a_kmm, 0, st);
  if (e != cudaSuccess) return (int)e;
  e = launch_chol_exact_raw(st, Lwork, M);
  if (e != cudaSuccess) return (int)e;
  const double* L = Lwork;
  void* a_kk[] = {&N, &ldN, &M, &L, &Knm, &KinvKmn, &titsias};
  e = cudaLaunchKernel((const void*)k_kinvkmn, dim3(div_up(N, 128)), dim3(128), a_kk, 0, st);
  return (int)e;
}

}  // namespace gpl
