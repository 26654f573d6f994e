// Cis genotype statistics per (gene, variant): the efficient score of adding one genotype column to
// a gene's fitted model, as getScoreStats of the reference's differential-expression driver computes
// it for genotype columns shared by all genes (ggplvm_de.cu:489-535), here for a separate set of
// variants per gene whose dosages are constant within a donor (genotypes are per donor; every cell
// carries its donor's). For gene j and a dosage column g (g_i = G[donor(i)]):
//     s = sum_i g_i (y_ij - W_ij) / Omega_i
//     v = g^T diag(W_j / Omega) g - t^T Psi_j^{-1} t,   t = Z^T diag(W_j / Omega) g
//     S = s / sqrt(phi_j v),   LR = S^2
// LR is the likelihood ratio of the IRLS working model (Gaussian in nu with weights W/Omega and
// dispersion phi) for adding the column with every other coefficient re-estimated: the
// per-(gene, variant) likelihood-ratio statistic against the fitted GP.
//
// Because g is constant within a donor, every sum over cells reduces to sums over the cell groups
// (the combinations of categorical levels, which include the donor):
//     s     = sum_g G[donor(g)] R_jg,          R_jg = sum_{i in g} (y_ij - W_ij) / Omega_i
//     t_a   = sum_g G[donor(g)] S_j[g][a]       (dense column a; S = the Gram's group sums)
//     t_c   = sum_{g at level c} G[donor(g)] S_j[g][intercept]   (categorical column c)
//     g^T diag(w) g = sum_g G[donor(g)]^2 S_j[g][intercept]
// and t^T Psi_j^{-1} t = |L_j^{-1} t|^2 with the factor L_j of Psi_j. The counts enter through W
// and nu of the last W/nu pass (y = W (nu - eta + 1) for the matched counts and 0 = W (nu - eta + 1)
// for the others, with eta = log W - log s - wt delta_GP titsias).
//
//   k_group_resid  R_jg, one warp per (gene, group), the group's cells in order
//   k_cis          one block per gene: t for all V variants of the gene, the forward substitution
//                  L^{-1} [t_1 .. t_V] (each factor entry read once), the statistics
#include <math.h>

#include <algorithm>
#include <vector>

#include "gpl_internal.cuh"

namespace gpl {

namespace {

__global__ void k_group_resid(int N, int ldN, int J, int n_grp, int pvars, const int* __restrict__ gcells,
                              const int* __restrict__ gstart, const double* __restrict__ W,
                              const double* __restrict__ Nu, const double* __restrict__ Omega,
                              const double* __restrict__ ls, const double* __restrict__ delta,
                              const double* __restrict__ titsias, double* __restrict__ R) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int j = warp / n_grp, g = warp - j * n_grp;
  if (j >= J) return;
  const double dgp = delta[pvars - 1];
  const double* Wj = W + (size_t)j * ldN;
  const double* nj = Nu + (size_t)j * ldN;
  double s = 0.0;
  for (int k = gstart[g] + lane; k < gstart[g + 1]; k += 32) {
    const int i = gcells[k];
    const double w = Wj[i];
    const double eta = log(w) - log(ls[i]) - dgp * titsias[i] * kWt;
    s += w * (nj[i] - eta) / Omega[i];  // (y - W) / Omega with y = W (nu - eta + 1)
  }
  s = warp_sum(s);
  if (lane == 0) R[(size_t)j * n_grp + g] = s;
}

// smem: Gg[n_grp], T[P][V] (row-major by column index then variant)
__global__ void __launch_bounds__(256) k_cis(int J, int P, int n_d, int n_grp, int n_cv, int V, int n_donors,
                                             const int* __restrict__ dcol, const int* __restrict__ cv_nh,
                                             const int* __restrict__ glev, const int* __restrict__ gdonor,
                                             const int8_t* __restrict__ dos, const double* __restrict__ gsum,
                                             const double* __restrict__ R, const double* __restrict__ Psi,
                                             const double* __restrict__ phi, double* __restrict__ S,
                                             double* __restrict__ LR) {
  extern __shared__ double sm[];
  double* Gg = sm;            // [n_grp]
  double* T = Gg + n_grp;     // [P][V]
  __shared__ double red[3][32];
  const int j = blockIdx.x;
  const int tid = threadIdx.x;
  const int ld = n_d + 1;
  const double* Sj = gsum + (size_t)j * n_grp * ld;
  const double* Rj = R + (size_t)j * n_grp;
  const double* L = Psi + (size_t)j * P * P;
  for (int e = tid; e < P * V; e += blockDim.x) T[e] = 0.0;
  __syncthreads();
  for (int v = 0; v < V; v++) {
    for (int g = tid; g < n_grp; g += blockDim.x)
      Gg[g] = (double)dos[((size_t)gdonor[g] * J + j) * V + v];
    __syncthreads();
    // dense rows of t: thread per dense column, groups in order
    for (int a = tid; a < n_d; a += blockDim.x) {
      double s = 0.0;
      for (int g = 0; g < n_grp; g++) s += Gg[g] * Sj[(size_t)g * ld + a];
      T[dcol[a] * V + v] = s;
    }
    __syncthreads();
    if (tid == 0) {  // categorical rows: each group adds to the columns of its levels
      for (int g = 0; g < n_grp; g++) {
        const double wg = Gg[g] * Sj[(size_t)g * ld];
        for (int c = 0; c < n_cv; c++) T[(cv_nh[c] + glev[(size_t)g * n_cv + c]) * V + v] += wg;
      }
    }
    // s and g^T diag(w) g
    double sp = 0.0, gw = 0.0;
    for (int g = tid; g < n_grp; g += blockDim.x) {
      sp += Gg[g] * Rj[g];
      gw += Gg[g] * Gg[g] * Sj[(size_t)g * ld];
    }
    sp = block_sum(sp, red[0]);
    gw = block_sum(gw, red[1]);
    if (tid == 0) {
      S[j + (size_t)v * J] = sp;   // numerator, finished below
      LR[j + (size_t)v * J] = gw;  // g^T diag(w) g, finished below
    }
    __syncthreads();
  }
  // forward substitution y = L^{-1} T for the V right-hand sides, each factor entry read once
  for (int k = 0; k < P; k++) {
    const double lkk = L[k + (size_t)k * P];
    if (tid < V) T[k * V + tid] /= lkk;
    __syncthreads();
    for (int e = tid; e < (P - k - 1) * V; e += blockDim.x) {
      const int i = k + 1 + e / V, v = e - (e / V) * V;
      T[i * V + v] -= L[i + (size_t)k * P] * T[k * V + v];
    }
    __syncthreads();
  }
  for (int v = 0; v < V; v++) {
    double q = 0.0;
    for (int k = tid; k < P; k += blockDim.x) q += T[k * V + v] * T[k * V + v];
    q = block_sum(q, red[2]);
    if (tid == 0) {
      const double var = LR[j + (size_t)v * J] - q;
      const double st = S[j + (size_t)v * J] / sqrt(phi[j] * var);
      S[j + (size_t)v * J] = st;
      LR[j + (size_t)v * J] = st * st;
    }
    __syncthreads();
  }
}

}  // namespace

int cis_stats(Ctx* c, int donor_var, int n_donors, int V, const int8_t* dos_host, double* S_host, double* LR_host) {
  if (c->n_grp == 0 || c->n_cv == 0) {
    c->err = "cis statistics need the categorical variables handled by cell groups";
    return GPL_ERR_ARG;
  }
  if (donor_var < 0 || donor_var >= c->n_var || c->vc[donor_var + 1] == 1) {
    c->err = "donor_var must name a categorical design variable";
    return GPL_ERR_ARG;
  }
  const int col = c->nh[donor_var + 1];
  int vd = -1;
  for (int v = 0; v < c->n_cv; v++)
    if (c->cv_nh[v] == col) vd = v;
  if (vd < 0 || n_donors != c->cv_nlev[vd]) {
    c->err = "n_donors must equal the donor variable's level count";
    return GPL_ERR_ARG;
  }
  const int J = c->J, n_grp = c->n_grp, n_cv = c->n_cv, P = c->P;
  const size_t smem = sizeof(double) * ((size_t)n_grp + (size_t)P * V);
  if (smem > 200 * 1024 || V < 1 || V > 256) {
    c->err = "too many variants or cell groups for the per-gene statistics";
    return GPL_ERR_ARG;
  }
  std::vector<int> glev((size_t)n_grp * n_cv), gdon(n_grp);
  GPL_TRY(c, cudaMemcpy(glev.data(), c->glev_d, sizeof(int) * glev.size(), cudaMemcpyDeviceToHost));
  for (int g = 0; g < n_grp; g++) gdon[g] = glev[(size_t)g * n_cv + vd];
  int* gdon_d = nullptr;
  int8_t* dos_d = nullptr;
  double *R = nullptr, *Sd = nullptr, *LRd = nullptr;
  auto cleanup = [&]() {
    void* b[] = {gdon_d, dos_d, R, Sd, LRd};
    for (void* p : b)
      if (p) cudaFree(p);
  };
  const size_t nd = (size_t)n_donors * J * V;
  if (cudaMalloc((void**)&gdon_d, sizeof(int) * n_grp) != cudaSuccess ||
      cudaMalloc((void**)&dos_d, nd) != cudaSuccess ||
      cudaMalloc((void**)&R, sizeof(double) * (size_t)J * n_grp) != cudaSuccess ||
      cudaMalloc((void**)&Sd, sizeof(double) * (size_t)J * V) != cudaSuccess ||
      cudaMalloc((void**)&LRd, sizeof(double) * (size_t)J * V) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    c->err = "device allocation failed: cis statistics";
    return GPL_ERR_ALLOC;
  }
  auto run = [&]() -> int {
    GPL_TRY(c, cudaMemcpyAsync(gdon_d, gdon.data(), sizeof(int) * n_grp, cudaMemcpyHostToDevice, c->stream));
    GPL_TRY(c, cudaMemcpyAsync(dos_d, dos_host, nd, cudaMemcpyHostToDevice, c->stream));
    int rc = launch_group_sums(c, 0);  // S_j[g][a] with w = W/Omega at the current state
    if (rc) return rc;
    const int64_t warps = (int64_t)J * n_grp;
    k_group_resid<<<div_up(warps * 32, 256), 256, 0, c->stream>>>(c->N, c->ldN, J, n_grp, c->p, c->gcells_d,
                                                                   c->gstart_d, c->W, c->Nu, c->Omega, c->ls,
                                                                   c->delta, c->titsias, R);
    GPL_LAUNCHED(c, "k_group_resid");
    if (smem > 48 * 1024) GPL_TRY(c, cudaFuncSetAttribute(k_cis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_cis<<<J, 256, smem, c->stream>>>(J, P, c->n_d, n_grp, n_cv, V, n_donors, c->dcol_d, c->cv_nh_d, c->glev_d,
                                       gdon_d, dos_d, c->gsum, R, c->Psi, c->phi, Sd, LRd);
    GPL_LAUNCHED(c, "k_cis");
    GPL_TRY(c, cudaMemcpyAsync(S_host, Sd, sizeof(double) * (size_t)J * V, cudaMemcpyDeviceToHost, c->stream));
    if (LR_host)
      GPL_TRY(c, cudaMemcpyAsync(LR_host, LRd, sizeof(double) * (size_t)J * V, cudaMemcpyDeviceToHost, c->stream));
    GPL_TRY(c, cudaStreamSynchronize(c->stream));
    return GPL_OK;
  };
  const int rc = run();
  cleanup();
  return rc;
}

}  // namespace gpl
