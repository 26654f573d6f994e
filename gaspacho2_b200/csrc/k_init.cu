// The starting point of a fit from the counts alone: latent coordinates X from the leading principal
// components of log1p(y / s), and inducing points T by k-means on X. The reference reads both from
// files (its X from argv[4], ggplvm.cu:1019-1022; T from initTaWithPer or --init-params,
// ggplvm.cu:1011,1103-1106) and ships PCA kernels that its driver never calls (init.cu:329-357);
// the start is computed here on the GPU so that the CLI can produce Xi.bin and Tau.bin itself.
//
//   k_dense_log1p   D[i, j] = log1p(y_ij / s_i) for every cell and gene (the counts the merge walk
//                   matches, as the fit reads them), cell fastest, zeros elsewhere
//   k_center_cols   D[:, j] -= mean_i D[i, j] (one block per gene, deterministic sum)
//   (FFMA GEMMs)    the gene covariance C = D^T D, the subspace iteration's C V, the scores D V
//   k_kmeans_assign each cell's nearest centre (ties to the lower index)
// The subspace iteration orthonormalises its J x Q block and solves its Q x Q Rayleigh quotient on
// the host (a few KB per iteration); the k-means centres are averaged on the host from the labels.
// Deterministic for a given seed; the principal directions are defined up to sign.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <random>
#include <vector>

#include "gpl_internal.cuh"

namespace gpl {

int launch_gemm_cm(Ctx* c, int m, int n, int K, const double* A, int lda, bool a_trans, const double* B, int ldb,
                   double* C, int ldc);  // k_gemm.cu

namespace {

__global__ void k_dense_log1p(int ldN, const int32_t* __restrict__ cell, const int64_t* __restrict__ gptr,
                              const int32_t* __restrict__ gvalid, const double* __restrict__ cnt,
                              const double* __restrict__ ls, double* __restrict__ D) {
  const int j = blockIdx.x;
  const int64_t b = gptr[j], e = gptr[j] + gvalid[j];
  for (int64_t l = b + threadIdx.x; l < e; l += blockDim.x) {
    const int i = cell[l];
    D[(size_t)j * ldN + i] = log1p(cnt[l] / ls[i]);
  }
}

__global__ void k_center_cols(int N, int ldN, double* __restrict__ D) {
  __shared__ double sh[32];
  double* col = D + (size_t)blockIdx.x * ldN;
  double s = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s += col[i];
  const double mean = block_sum(s, sh) / (double)N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) col[i] -= mean;
}

__global__ void k_kmeans_assign(int N, int Q, int M, const double* __restrict__ X, const double* __restrict__ C,
                                int* __restrict__ lab) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double best = 1e300;
  int bk = 0;
  for (int k = 0; k < M; k++) {
    double d = 0.0;
    for (int q = 0; q < Q; q++) {
      const double t = X[i + (size_t)q * N] - C[k + (size_t)q * M];
      d += t * t;
    }
    if (d < best) {
      best = d;
      bk = k;
    }
  }
  lab[i] = bk;
}

// Eigen-decomposition of a symmetric n x n matrix A (column-major, overwritten) by cyclic Jacobi
// rotations: eigenvalues on the diagonal, eigenvectors in the columns of V.
void jacobi_eig(int n, std::vector<double>& A, std::vector<double>& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[i + (size_t)i * n] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) off += A[p + (size_t)q * n] * A[p + (size_t)q * n];
    if (off < 1e-30) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = A[p + (size_t)q * n];
        if (fabs(apq) < 1e-300) continue;
        const double app = A[p + (size_t)p * n], aqq = A[q + (size_t)q * n];
        const double th = 0.5 * (aqq - app) / apq;
        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
        const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; k++) {  // A <- A R (columns p, q)
          const double akp = A[k + (size_t)p * n], akq = A[k + (size_t)q * n];
          A[k + (size_t)p * n] = cs * akp - sn * akq;
          A[k + (size_t)q * n] = sn * akp + cs * akq;
        }
        for (int k = 0; k < n; k++) {  // A <- R^T A (rows p, q)
          const double apk = A[p + (size_t)k * n], aqk = A[q + (size_t)k * n];
          A[p + (size_t)k * n] = cs * apk - sn * aqk;
          A[q + (size_t)k * n] = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = V[k + (size_t)p * n], vkq = V[k + (size_t)q * n];
          V[k + (size_t)p * n] = cs * vkp - sn * vkq;
          V[k + (size_t)q * n] = sn * vkp + cs * vkq;
        }
      }
  }
}

// Modified Gram-Schmidt on the columns of Z (rows x cols, column-major).
void orthonormalise(int rows, int cols, std::vector<double>& Z) {
  for (int a = 0; a < cols; a++) {
    double* za = &Z[(size_t)a * rows];
    for (int b = 0; b < a; b++) {
      const double* zb = &Z[(size_t)b * rows];
      double d = 0.0;
      for (int r = 0; r < rows; r++) d += za[r] * zb[r];
      for (int r = 0; r < rows; r++) za[r] -= d * zb[r];
    }
    double nr = 0.0;
    for (int r = 0; r < rows; r++) nr += za[r] * za[r];
    nr = sqrt(nr);
    if (nr > 0)
      for (int r = 0; r < rows; r++) za[r] /= nr;
  }
}

}  // namespace

int init_latent(Ctx* c, int pca_iters, int kmeans_iters, uint64_t seed, double* X_host, double* T_host) {
  const int N = c->N, J = c->J, Q = c->Q, M = c->M, ldN = c->ldN;
  if (Q > J || M > N) {
    c->err = "the start needs Q <= genes and M <= cells";
    return GPL_ERR_ARG;
  }
  double *C = nullptr, *V = nullptr, *Z = nullptr, *S = nullptr, *Cm = nullptr;
  int* lab = nullptr;
  auto cleanup = [&]() {
    void* b[] = {C, V, Z, S, Cm, lab};
    for (void* p : b)
      if (p) cudaFree(p);
  };
  if (cudaMalloc((void**)&C, sizeof(double) * (size_t)J * J) != cudaSuccess ||
      cudaMalloc((void**)&V, sizeof(double) * (size_t)J * Q) != cudaSuccess ||
      cudaMalloc((void**)&Z, sizeof(double) * (size_t)J * Q) != cudaSuccess ||
      cudaMalloc((void**)&S, sizeof(double) * (size_t)N * Q) != cudaSuccess ||
      cudaMalloc((void**)&Cm, sizeof(double) * (size_t)M * Q) != cudaSuccess ||
      cudaMalloc((void**)&lab, sizeof(int) * (size_t)N) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    c->err = "device allocation failed: start buffers";
    return GPL_ERR_ALLOC;
  }
  auto run = [&]() -> int {
    double* D = c->scratch;  // ldN x J, cell fastest
    GPL_TRY(c, cudaMemsetAsync(D, 0, sizeof(double) * (size_t)ldN * J, c->stream));
    k_dense_log1p<<<J, 256, 0, c->stream>>>(ldN, c->cell, c->gptr, c->gvalid, c->cnt, c->ls, D);
    GPL_LAUNCHED(c, "k_dense_log1p");
    k_center_cols<<<J, 256, 0, c->stream>>>(N, ldN, D);
    GPL_LAUNCHED(c, "k_center_cols");
    int rc = launch_gemm_cm(c, J, J, N, D, ldN, true, D, ldN, C, J);  // C = D^T D
    if (rc) return rc;
    // subspace iteration on C from a seeded Gaussian block
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<double> Vh((size_t)J * Q);
    for (auto& v : Vh) v = nd(rng);
    orthonormalise(J, Q, Vh);
    for (int it = 0; it < pca_iters; it++) {
      GPL_TRY(c, cudaMemcpyAsync(V, Vh.data(), sizeof(double) * Vh.size(), cudaMemcpyHostToDevice, c->stream));
      if ((rc = launch_gemm_cm(c, J, Q, J, C, J, false, V, J, Z, J))) return rc;
      GPL_TRY(c, cudaMemcpyAsync(Vh.data(), Z, sizeof(double) * Vh.size(), cudaMemcpyDeviceToHost, c->stream));
      GPL_TRY(c, cudaStreamSynchronize(c->stream));
      orthonormalise(J, Q, Vh);
    }
    // Rayleigh-Ritz: H = V^T C V (Q x Q), its eigenvectors order and rotate the block
    GPL_TRY(c, cudaMemcpyAsync(V, Vh.data(), sizeof(double) * Vh.size(), cudaMemcpyHostToDevice, c->stream));
    if ((rc = launch_gemm_cm(c, J, Q, J, C, J, false, V, J, Z, J))) return rc;
    std::vector<double> Zh((size_t)J * Q);
    GPL_TRY(c, cudaMemcpyAsync(Zh.data(), Z, sizeof(double) * Zh.size(), cudaMemcpyDeviceToHost, c->stream));
    GPL_TRY(c, cudaStreamSynchronize(c->stream));
    std::vector<double> H((size_t)Q * Q), E;
    for (int a = 0; a < Q; a++)
      for (int b = 0; b < Q; b++) {
        double s = 0.0;
        for (int r = 0; r < J; r++) s += Vh[r + (size_t)a * J] * Zh[r + (size_t)b * J];
        H[a + (size_t)b * Q] = s;
      }
    for (int a = 0; a < Q; a++)
      for (int b = a + 1; b < Q; b++) H[a + (size_t)b * Q] = H[b + (size_t)a * Q] =
          0.5 * (H[a + (size_t)b * Q] + H[b + (size_t)a * Q]);
    jacobi_eig(Q, H, E);
    std::vector<int> ord(Q);
    for (int a = 0; a < Q; a++) ord[a] = a;
    std::stable_sort(ord.begin(), ord.end(),
                     [&](int a, int b) { return H[a + (size_t)a * Q] > H[b + (size_t)b * Q]; });
    std::vector<double> R((size_t)J * Q, 0.0);
    for (int a = 0; a < Q; a++) {
      const int e = ord[a];
      // sign: the largest-magnitude loading positive (a fixed choice of the free sign)
      double big = 0.0;
      for (int r = 0; r < J; r++) {
        double s = 0.0;
        for (int b = 0; b < Q; b++) s += Vh[r + (size_t)b * J] * E[b + (size_t)e * Q];
        R[r + (size_t)a * J] = s;
        if (fabs(s) > fabs(big)) big = s;
      }
      if (big < 0)
        for (int r = 0; r < J; r++) R[r + (size_t)a * J] = -R[r + (size_t)a * J];
    }
    GPL_TRY(c, cudaMemcpyAsync(V, R.data(), sizeof(double) * R.size(), cudaMemcpyHostToDevice, c->stream));
    if ((rc = launch_gemm_cm(c, N, Q, J, D, ldN, false, V, J, S, N))) return rc;  // scores D V
    std::vector<double> Xs((size_t)N * Q);
    GPL_TRY(c, cudaMemcpyAsync(Xs.data(), S, sizeof(double) * Xs.size(), cudaMemcpyDeviceToHost, c->stream));
    GPL_TRY(c, cudaStreamSynchronize(c->stream));
    for (int q = 0; q < Q; q++) {  // centred, unit variance
      double* x = &Xs[(size_t)q * N];
      double m = 0.0;
      for (int i = 0; i < N; i++) m += x[i];
      m /= N;
      double v = 0.0;
      for (int i = 0; i < N; i++) v += (x[i] - m) * (x[i] - m);
      double sd = sqrt(v / N);
      if (sd == 0.0) sd = 1.0;
      for (int i = 0; i < N; i++) x[i] = (x[i] - m) / sd;
    }
    // k-means (Lloyd) on X from M distinct seeded cells
    std::vector<int> pick(N);
    for (int i = 0; i < N; i++) pick[i] = i;
    for (int k = 0; k < M; k++) {
      std::uniform_int_distribution<int> ud(k, N - 1);
      std::swap(pick[k], pick[ud(rng)]);
    }
    std::vector<double> Ch((size_t)M * Q);
    for (int k = 0; k < M; k++)
      for (int q = 0; q < Q; q++) Ch[k + (size_t)q * M] = Xs[pick[k] + (size_t)q * N];
    GPL_TRY(c, cudaMemcpyAsync(S, Xs.data(), sizeof(double) * Xs.size(), cudaMemcpyHostToDevice, c->stream));
    std::vector<int> labh(N);
    for (int it = 0; it < kmeans_iters; it++) {
      GPL_TRY(c, cudaMemcpyAsync(Cm, Ch.data(), sizeof(double) * Ch.size(), cudaMemcpyHostToDevice, c->stream));
      k_kmeans_assign<<<div_up(N, 128), 128, 0, c->stream>>>(N, Q, M, S, Cm, lab);
      GPL_LAUNCHED(c, "k_kmeans_assign");
      GPL_TRY(c, cudaMemcpyAsync(labh.data(), lab, sizeof(int) * N, cudaMemcpyDeviceToHost, c->stream));
      GPL_TRY(c, cudaStreamSynchronize(c->stream));
      std::vector<double> sum((size_t)M * Q, 0.0);
      std::vector<int> cnt(M, 0);
      for (int i = 0; i < N; i++) {
        cnt[labh[i]]++;
        for (int q = 0; q < Q; q++) sum[labh[i] + (size_t)q * M] += Xs[i + (size_t)q * N];
      }
      for (int k = 0; k < M; k++)
        if (cnt[k] > 0)
          for (int q = 0; q < Q; q++) Ch[k + (size_t)q * M] = sum[k + (size_t)q * M] / cnt[k];
    }
    memcpy(X_host, Xs.data(), sizeof(double) * Xs.size());
    memcpy(T_host, Ch.data(), sizeof(double) * Ch.size());
    return GPL_OK;
  };
  const int rc = run();
  cleanup();
  return rc;
}

}  // namespace gpl
