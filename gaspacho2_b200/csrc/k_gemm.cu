// Double-precision (cell x gene) contractions of the IRLS and the gradient, all built on
// one register-tiled FP64 GEMM (64x64 output tile, 16-deep K chunks in shared memory,
// 4x4 accumulators per thread) with element-wise prologues and epilogues. The model
// matrix enters as its dense columns D (ldN x n_d) plus per-cell level codes of the grouped
// categorical variables, so every product z_i . beta is D_i . beta[dcol] + the coefficients
// of the cell's levels.
//
//   W / Nu     eta = z_i . beta_j for every cell and gene (k_eta; k_eta_dmma in k_dgemm.cu on the
//              FP64 tensor cores with option eta_tc), then the getWForBeta element-wise pass
//              (ggplvm.cu:468-514): k_w_nu over cells x genes, then k_w_nu_counts. Bound:
//              FP64 FMA (N*J*n_d) for the predictor, HBM and FP64 exp() for the pass.
//   bvec       dense rows of Z^T diag(W_j/Omega) nu_j (getZtOinvjnj, util_cuda.cu:462-487)
//              and of the GLM initialisation right-hand sides Z^T y0_j (initBeta,
//              init.cu:193-221); the categorical rows come from the group sums.
//   E          z_i . tBeta_j (cell x gene predictions used by the Omega/X gradient).
//   C1 (part)  sum_j (tn_ij / phi_j) tBeta_j[GP] (ggplvm.cu:344).
#include <algorithm>

#include "gpl_internal.cuh"

namespace gpl {

namespace {
constexpr int TM = 64, TN = 64, TK = 16;
}

// A(r, k) and B(k, c) loaders. kFastK: the K index is contiguous in memory (load K-fastest).
struct LoadD {  // A(r = cell, k = dense column) = D[k*ldN + r]
  static constexpr bool kFastK = false;
  const double* D;
  int ldN, N, n_d;
  __device__ double operator()(int r, int k) const { return (r < N && k < n_d) ? D[(size_t)k * ldN + r] : 0.0; }
};
struct LoadDt {  // A(r = dense column, k = cell) = D[r*ldN + k]
  static constexpr bool kFastK = true;
  const double* D;
  int ldN, N, n_d;
  __device__ double operator()(int r, int k) const { return (r < n_d && k < N) ? D[(size_t)r * ldN + k] : 0.0; }
};
struct LoadBetaDense {  // B(k = dense column, c = gene) = B[dcol[k] + c*P]
  static constexpr bool kFastK = true;
  const double* B;
  const int* dcol;
  int P, n_d, J;
  __device__ double operator()(int k, int c) const { return (k < n_d && c < J) ? B[dcol[k] + (size_t)c * P] : 0.0; }
};
struct LoadOinvNu {  // B(k = cell, c = gene) = W/Omega * Nu
  static constexpr bool kFastK = true;
  const double *W, *Nu, *Omega;
  int ldN, N, J;
  __device__ double operator()(int k, int c) const {
    if (k >= N || c >= J) return 0.0;
    const size_t e = (size_t)c * ldN + k;
    return W[e] / Omega[k] * Nu[e];
  }
};
struct LoadCellGene {  // B(k = cell, c = gene) = S[c*ldN + k]
  static constexpr bool kFastK = true;
  const double* S;
  int ldN, N, J;
  __device__ double operator()(int k, int c) const { return (k < N && c < J) ? S[(size_t)c * ldN + k] : 0.0; }
};
struct LoadTn {  // A(r = cell, k = gene) = tn / phi, tn = O*nu - O*E, O = W/Omega
  static constexpr bool kFastK = false;
  const double *W, *Nu, *E, *Omega, *phi;
  int ldN, N, J;
  __device__ double operator()(int r, int k) const {
    if (r >= N || k >= J) return 0.0;
    const size_t e = (size_t)k * ldN + r;
    const double o = W[e] / Omega[r];
    const double tn = o * Nu[e] - o * E[e];
    return tn / phi[k];
  }
};
struct LoadCellGeneA {  // A(r = cell, k = gene) = S[k*ldN + r]
  static constexpr bool kFastK = false;
  const double* S;
  int ldN, N, J;
  __device__ double operator()(int r, int k) const { return (r < N && k < J) ? S[(size_t)k * ldN + r] : 0.0; }
};
struct LoadTBetaGP {  // B(k = gene, c = a) = tBeta[g0 + a + k*P]
  static constexpr bool kFastK = false;
  const double* tB;
  int P, g0, M, J;
  __device__ double operator()(int k, int c) const { return (k < J && c < M) ? tB[g0 + c + (size_t)k * P] : 0.0; }
};

template <class LA, class LB>
__device__ __forceinline__ void gemm_tile(int m0, int n0, int K, const LA& A, const LB& B, double (&acc)[4][4],
                                          double (*As)[TM + 1], double (*Bs)[TN + 1]) {
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
#pragma unroll
  for (int x = 0; x < 4; x++)
#pragma unroll
    for (int y = 0; y < 4; y++) acc[x][y] = 0.0;
  for (int k0 = 0; k0 < K; k0 += TK) {
#pragma unroll
    for (int t = 0; t < (TM * TK) / 256; t++) {
      const int e = tid + t * 256;
      int r, k;
      if (LA::kFastK) { k = e % TK; r = e / TK; }
      else { r = e % TM; k = e / TM; }
      As[k][r] = A(m0 + r, k0 + k);
    }
#pragma unroll
    for (int t = 0; t < (TN * TK) / 256; t++) {
      const int e = tid + t * 256;
      int k, cc;
      if (LB::kFastK) { k = e % TK; cc = e / TK; }
      else { cc = e % TN; k = e / TN; }
      Bs[k][cc] = B(k0 + k, n0 + cc);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < TK; k++) {
      double a[4], b[4];
#pragma unroll
      for (int x = 0; x < 4; x++) a[x] = As[k][tx + 16 * x];
#pragma unroll
      for (int y = 0; y < 4; y++) b[y] = Bs[k][ty + 16 * y];
#pragma unroll
      for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y] = fma(a[x], b[y], acc[x][y]);
    }
    __syncthreads();
  }
}

// z_i . B_j for a tile: the dense GEMM result plus the coefficients of the cell's levels
__device__ __forceinline__ double add_levels(double dense, int i, int j, int ldN, int P, int n_cv,
                                             const int* __restrict__ cv_nh, const int* __restrict__ codes,
                                             const double* __restrict__ B) {
  double s = dense;
  for (int v = 0; v < n_cv; v++) s += B[cv_nh[v] + codes[(size_t)v * ldN + i] + (size_t)j * P];
  return s;
}

// ---- W / Nu -----------------------------------------------------------------------------
// getWForBeta (ggplvm.cu:468-514) from the linear predictor eta = z_i . beta_j (k_eta_dmma or
// k_eta, written to a cell x gene buffer first). The per-cell factors exp(dgp titsias_i wt),
// dgp titsias_i wt and log s_i are computed once per pass (k_cell_factors); then every cell gets
// W = exp(eta) s_i exp(dgp titsias_i wt) and the working response of a zero count (k_w_nu), and
// the counts that the reference's merge walk matches (the first gvalid entries of each gene)
// replace their cells' working response (k_w_nu_counts, after it in stream order). The same
// expressions, in the same order, as the per-element form. The DE driver takes
// the Titsias factor at weight 1 and nu = z.(beta - zeta) + (y - W)/W (ggplvm_de.cu:442-486);
// the fit driver has zeta = 0.
__global__ void k_cell_factors(int N, int ldN, int pvars, int de, const double* __restrict__ delta,
                               const double* __restrict__ titsias, const double* __restrict__ ls,
                               double* __restrict__ f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double tt = delta[pvars - 1] * titsias[i] * (de ? 1.0 : kWt);
  f[i] = exp(tt);
  f[ldN + i] = tt;
  f[2 * (size_t)ldN + i] = log(ls[i]);
}

// Zero-count values of every cell and gene: a 2-D grid (cell pairs x gene quads), two cells and
// up to kWnuGenes genes per thread with 16-byte loads and stores (ldN is even, so a pair never
// straddles a column; past N the pair's second value is read from the column's padding and
// dropped). The quad's loads are issued before any exp(), so 64 bytes per thread are in flight.
// With a group order (gpos: each cell's position in it) W's group-ordered copy for the group-sum
// GEMMs is written here too, one 8-byte store per value, in place of a gather pass over W.
constexpr int kWnuGenes = 4;
__global__ void __launch_bounds__(256) k_w_nu(int N, int ldN, int J, const double* __restrict__ E,
                                              const double* __restrict__ ls, const double* __restrict__ f,
                                              int de, const double* __restrict__ e0,
                                              const int* __restrict__ gpos, double* __restrict__ W,
                                              double* __restrict__ Nu, double* __restrict__ Wg) {
  const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= N) return;
  const bool two = i + 1 < N;
  const double l0 = ls[i], f0 = f[i], l1 = two ? ls[i + 1] : 0.0, f1 = two ? f[i + 1] : 0.0;
  const double z0 = de ? e0[i] : 0.0, z1 = de && two ? e0[i + 1] : 0.0;
  const int p0 = Wg ? gpos[i] : 0, p1 = Wg && two ? gpos[i + 1] : 0;
  for (int jb = blockIdx.y * kWnuGenes; jb < J; jb += gridDim.y * kWnuGenes) {
    double2 eta[kWnuGenes];
#pragma unroll
    for (int u = 0; u < kWnuGenes; u++)
      if (jb + u < J) eta[u] = *reinterpret_cast<const double2*>(E + (size_t)(jb + u) * ldN + i);
#pragma unroll
    for (int u = 0; u < kWnuGenes; u++) {
      const int j = jb + u;
      if (j >= J) break;
      const size_t o = (size_t)j * ldN + i;
      double2 w, nu;
      w.x = exp(eta[u].x) * l0 * f0;
      nu.x = de ? (eta[u].x - z0) - 1.0 : eta[u].x - 1.0;
      if (two) {
        w.y = exp(eta[u].y) * l1 * f1;
        nu.y = de ? (eta[u].y - z1) - 1.0 : eta[u].y - 1.0;
        *reinterpret_cast<double2*>(W + o) = w;
        *reinterpret_cast<double2*>(Nu + o) = nu;
      } else {
        W[o] = w.x;
        Nu[o] = nu.x;
      }
      if (Wg) {
        Wg[(size_t)j * ldN + p0] = w.x;
        if (two) Wg[(size_t)j * ldN + p1] = w.y;
      }
    }
  }
}

// The working response of the counts that the reference's merge walk matches (the first gvalid
// entries of each gene), after k_w_nu wrote every cell's zero-count value (stream order). Each
// thread takes kCountsIlp entries per round, their index, count and eta loads issued before any
// exp(), so that the dependent gathers of several entries are in flight at once.
constexpr int kCountsIlp = 4;
__global__ void __launch_bounds__(256) k_w_nu_counts(int ldN, const double* __restrict__ E,
                                                     const double* __restrict__ ls, const double* __restrict__ f,
                                                     const int32_t* __restrict__ cell,
                                                     const int64_t* __restrict__ gptr,
                                                     const int32_t* __restrict__ gvalid,
                                                     const double* __restrict__ cnt, int de,
                                                     const double* __restrict__ e0, double* __restrict__ Nu) {
  const int j = blockIdx.x;
  const double* Ej = E + (size_t)j * ldN;
  double* Nj = Nu + (size_t)j * ldN;
  const int64_t b = gptr[j], e = gptr[j] + gvalid[j];
  for (int64_t l0 = b + threadIdx.x; l0 < e; l0 += (int64_t)kCountsIlp * blockDim.x) {
    int ic[kCountsIlp];
    double y[kCountsIlp], eta[kCountsIlp];
#pragma unroll
    for (int u = 0; u < kCountsIlp; u++) {
      const int64_t l = l0 + (int64_t)u * blockDim.x;
      ic[u] = l < e ? cell[l] : -1;
      y[u] = l < e ? cnt[l] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kCountsIlp; u++) eta[u] = ic[u] >= 0 ? Ej[ic[u]] : 0.0;
#pragma unroll
    for (int u = 0; u < kCountsIlp; u++) {
      const int i = ic[u];
      if (i < 0) continue;
      if (de) {
        const double w = exp(eta[u]) * ls[i] * f[i];
        Nj[i] = (eta[u] - e0[i]) + (y[u] - w) / w;
      } else {
        Nj[i] = eta[u] + exp(log(y[u]) - (eta[u] + f[2 * (size_t)ldN + i] + f[ldN + i])) - 1.0;
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_eta(int N, int ldN, int P, int J, int n_d, int n_cv,
                                             const double* __restrict__ D, const int* __restrict__ dcol,
                                             const int* __restrict__ cv_nh, const int* __restrict__ codes,
                                             const double* __restrict__ B, double* __restrict__ out);

// W / Nu: the linear predictor into the scratch buffer (on the FP64 tensor cores with option
// eta_tc), the per-cell factors, then k_w_nu.
int launch_w_nu(Ctx* c) {
  ProfScope ps(c, "w_nu");
  if (c->eta_tc) {
    const int rc = launch_eta_dmma(c, c->Beta, c->scratch);
    if (rc) return rc;
  } else {
    dim3 g(div_up(c->N, TM), div_up(c->J, TN));
    k_eta<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->P, c->J, c->n_d, c->n_cv, c->Dm, c->dcol_d, c->cv_nh_d,
                                    c->codes_d, c->Beta, c->scratch);
    GPL_LAUNCHED(c, "k_eta");
  }
  k_cell_factors<<<div_up(c->N, 256), 256, 0, c->stream>>>(c->N, c->ldN, c->p, c->de ? 1 : 0, c->delta, c->titsias,
                                                          c->ls, c->cellfac);
  GPL_LAUNCHED(c, "k_cell_factors");
  {
    // W's group-ordered copy for the group-sum GEMMs is written by k_w_nu (W changes only here)
    dim3 g(div_up(c->N, 512), std::min(div_up(c->J, kWnuGenes), 65535));
    k_w_nu<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->J, c->scratch, c->ls, c->cellfac, c->de ? 1 : 0, c->e0,
                                     c->gpos_d, c->W, c->Nu, c->Wg);
    GPL_LAUNCHED(c, "k_w_nu");
    k_w_nu_counts<<<c->J, 256, 0, c->stream>>>(c->ldN, c->scratch, c->ls, c->cellfac, c->cell, c->gptr, c->gvalid,
                                               c->cnt, c->de ? 1 : 0, c->e0, c->Nu);
    GPL_LAUNCHED(c, "k_w_nu_counts");
  }
  return GPL_OK;
}

// ---- E = z_i . B_j ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_eta(int N, int ldN, int P, int J, int n_d, int n_cv,
                                             const double* __restrict__ D, const int* __restrict__ dcol,
                                             const int* __restrict__ cv_nh, const int* __restrict__ codes,
                                             const double* __restrict__ B, double* __restrict__ out) {
  __shared__ double As[TK][TM + 1];
  __shared__ double Bs[TK][TN + 1];
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  double acc[4][4];
  gemm_tile(m0, n0, n_d, LoadD{D, ldN, N, n_d}, LoadBetaDense{B, dcol, P, n_d, J}, acc, As, Bs);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int x = 0; x < 4; x++) {
    const int i = m0 + tx + 16 * x;
    if (i >= N) continue;
#pragma unroll
    for (int y = 0; y < 4; y++) {
      const int j = n0 + ty + 16 * y;
      if (j < J) out[i + (size_t)j * ldN] = add_levels(acc[x][y], i, j, ldN, P, n_cv, cv_nh, codes, B);
    }
  }
}

int launch_zbeta(Ctx* c, const double* B, double* out) {
  ProfScope ps(c, "zbeta");
  if (c->eta_tc) return launch_eta_dmma(c, B, out);
  dim3 g(div_up(c->N, TM), div_up(c->J, TN));
  k_eta<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->P, c->J, c->n_d, c->n_cv, c->Dm, c->dcol_d, c->cv_nh_d,
                                  c->codes_d, B, out);
  GPL_LAUNCHED(c, "k_eta");
  return GPL_OK;
}

int launch_eta_one(Ctx* c, const double* b, double* out) {
  dim3 g(div_up(c->N, TM), 1);
  k_eta<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->P, 1, c->n_d, c->n_cv, c->Dm, c->dcol_d, c->cv_nh_d, c->codes_d,
                                  b, out);
  GPL_LAUNCHED(c, "k_eta");
  return GPL_OK;
}

// ---- generic GEMM with a column-major store; rows optionally mapped ------------------------
template <class LA, class LB>
__global__ void __launch_bounds__(256) k_gemm_store(int m, int n, int K, LA A, LB B, double* __restrict__ out,
                                                    int64_t ldo, const int* __restrict__ rowmap) {
  __shared__ double As[TK][TM + 1];
  __shared__ double Bs[TK][TN + 1];
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  double acc[4][4];
  gemm_tile(m0, n0, K, A, B, acc, As, Bs);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int x = 0; x < 4; x++) {
    const int r = m0 + tx + 16 * x;
    if (r >= m) continue;
    const int orow = rowmap ? rowmap[r] : r;
#pragma unroll
    for (int y = 0; y < 4; y++) {
      const int cc = n0 + ty + 16 * y;
      if (cc < n) out[orow + (size_t)cc * ldo] = acc[x][y];
    }
  }
}

// y0 for initBeta: log((y + 0.05)/ls) where a count is matched, log(0.05/ls) elsewhere.
__global__ void k_init_response(int N, int ldN, int J, const double* __restrict__ ls, double* __restrict__ out) {
  const int j = blockIdx.x;
  for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < N; i += gridDim.y * blockDim.x)
    out[(size_t)j * ldN + i] = log(0.05 / ls[i]);
}
__global__ void k_init_response_counts(int N, int ldN, int J, const double* __restrict__ ls,
                                       const int32_t* __restrict__ cell, const int64_t* __restrict__ gptr,
                                       const int32_t* __restrict__ gvalid, const double* __restrict__ cnt,
                                       double* __restrict__ out) {
  const int j = blockIdx.x;
  const int64_t b = gptr[j], e = gptr[j] + gvalid[j];
  for (int64_t l = b + threadIdx.x; l < e; l += blockDim.x) {
    const int i = cell[l];
    out[(size_t)j * ldN + i] = log((cnt[l] + 0.05) / ls[i]);
  }
}

int launch_init_response(Ctx* c) {
  ProfScope ps(c, "init_response");
  dim3 g(c->J, div_up(c->N, 256) > 64 ? 64 : div_up(c->N, 256));
  k_init_response<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->J, c->ls, c->scratch);
  GPL_LAUNCHED(c, "k_init_response");
  k_init_response_counts<<<c->J, 128, 0, c->stream>>>(c->N, c->ldN, c->J, c->ls, c->cell, c->gptr, c->gvalid,
                                                     c->cnt, c->scratch);
  GPL_LAUNCHED(c, "k_init_response_counts");
  return GPL_OK;
}

// Z^T u: dense rows by GEMM (mode 0: u = W/Omega nu; 1: u = y0), categorical rows from groups
int launch_zt_u(Ctx* c, int mode) { return launch_zt_u_ex(c, mode, mode == 0 ? c->Nu : c->scratch, c->bvec); }

int launch_zt_u_ex(Ctx* c, int mode, const double* u, double* out) {
  {
    ProfScope ps(c, "zt_u");
    dim3 g(div_up(c->n_d, TM), div_up(c->J, TN));
    LoadDt A{c->Dm, c->ldN, c->N, c->n_d};
    const int rc = dgen_zt_u(c, mode, u, out);
    if (rc != GPL_OK && rc != GPL_ERR_ARG) return rc;
    if (rc == GPL_ERR_ARG && mode == 2) {
      c->err = "per-cell Z^T u needs the DMMA form (at most 144 dense columns)";
      return GPL_ERR_ARG;
    }
    if (rc == GPL_ERR_ARG) {  // the FFMA form: more dense columns than one DMMA tile
      if (mode == 0)
        k_gemm_store<<<g, 256, 0, c->stream>>>(c->n_d, c->J, c->N, A,
                                               LoadOinvNu{c->W, u, c->Omega, c->ldN, c->N, c->J}, out,
                                               (int64_t)c->P, c->dcol_d);
      else
        k_gemm_store<<<g, 256, 0, c->stream>>>(c->n_d, c->J, c->N, A, LoadCellGene{u, c->ldN, c->N, c->J}, out,
                                               (int64_t)c->P, c->dcol_d);
      GPL_LAUNCHED(c, "k_gemm_store(zt_u)");
    }
  }
  c->zt_u_src = (mode == 2 || (mode == 0 && u != c->Nu)) ? u : nullptr;
  int rc = launch_group_sums(c, mode == 0 ? 3 : mode == 2 ? 4 : 2);
  c->zt_u_src = nullptr;
  if (rc) return rc;
  return launch_assemble_b(c, out);
}

// C1 <- sum_j (tn_ij/phi_j) tBeta_j[GP]   (stored cell-fastest, ld ldN)
int launch_c1_tn(Ctx* c) {
  ProfScope ps(c, "c1_tn");
  {
    const int rc = dgen_c1_tn(c);
    if (rc != GPL_ERR_ARG) return rc;  // GPL_ERR_ARG: more dense columns than one DMMA tile
  }
  const int g0 = c->nh[c->p - 1];
  dim3 g(div_up(c->N, TM), div_up(c->M, TN));
  k_gemm_store<<<g, 256, 0, c->stream>>>(c->N, c->M, c->J,
                                         LoadTn{c->W, c->Nu, c->scratch, c->Omega, c->phi, c->ldN, c->N, c->J},
                                         LoadTBetaGP{c->tBeta, c->P, g0, c->M, c->J}, c->C1, (int64_t)c->ldN,
                                         (const int*)nullptr);
  GPL_LAUNCHED(c, "k_gemm_store(c1_tn)");
  return GPL_OK;
}

}  // namespace gpl

namespace gpl {

// C (m x n, column-major, ld ldc) = op(A) B with op(A)(r, k) = A[k * lda + r] (a_trans = false)
// or A[r * lda + k] (a_trans = true), B(k, c) = B[c * ldb + k]; FFMA tile GEMM.
int launch_gemm_cm(Ctx* c, int m, int n, int K, const double* A, int lda, bool a_trans, const double* B, int ldb,
                   double* C, int ldc) {
  dim3 g(div_up(m, TM), div_up(n, TN));
  if (a_trans)
    k_gemm_store<<<g, 256, 0, c->stream>>>(m, n, K, LoadDt{A, lda, K, m}, LoadCellGene{B, ldb, K, n}, C,
                                           (int64_t)ldc, (const int*)nullptr);
  else
    k_gemm_store<<<g, 256, 0, c->stream>>>(m, n, K, LoadD{A, lda, m, K}, LoadCellGene{B, ldb, K, n}, C,
                                           (int64_t)ldc, (const int*)nullptr);
  GPL_LAUNCHED(c, "k_gemm_store(cm)");
  return GPL_OK;
}

// G[i, a] = sum_j R_ij B[g0 + a, j]: a cell x gene matrix R (cell fastest, ld ldN) against the GP
// block of coefficients (P x J), into G (cell fastest, ld ldN). FFMA tile GEMM.
int launch_resid_gp(Ctx* c, const double* R, const double* B, double* G) {
  const int g0 = c->nh[c->p - 1];
  dim3 g(div_up(c->N, TM), div_up(c->M, TN));
  k_gemm_store<<<g, 256, 0, c->stream>>>(c->N, c->M, c->J, LoadCellGeneA{R, c->ldN, c->N, c->J},
                                         LoadTBetaGP{B, c->P, g0, c->M, c->J}, G, (int64_t)c->ldN,
                                         (const int*)nullptr);
  GPL_LAUNCHED(c, "k_gemm_store(resid_gp)");
  return GPL_OK;
}

}  // namespace gpl
