// The IRLS forms of the differential-expression driver (ggplvm_de.cu), which refits the GLM
// part for a null model, one GP model per latent dimension and the full model and keeps every
// model's per-gene log-likelihood ("BFs"). They differ from the fit driver's forms in:
//
//   k_de_zeta      zeta_k = sum_j Beta_kj / phi_j / sum_j 1/phi_j (getZeta, :34-47), recomputed
//                  after every coefficient update; the working response then needs
//                  e0_i = z_i . zeta (launch_eta_one) because nu = z_i.(beta_j - zeta) + ...
//   k_de_beta_phi  undamped beta_j = Psi_j^{-1} b_j + zeta and
//                  phi_j = (sum_i nu^2 W/Omega - b_j . Psi_j^{-1} b_j) / N with the clamps
//                  NaN -> 1, < 0 -> 100, < 0.01 -> 0.01, > 100 -> 100 (getBetaPhi, :413-438)
//   k_de_lkhd      l_j = (sum_i [((log W - delta_{p-1} titsias) y - W) / Omega]
//                         - sum_k log L_kk) / phi_j + P' log(2 pi') / 2
//                  with pi' = 3.1415926535 (getLkhdPois, :667-693); P' excludes the inert GP
//                  block of the null model.
//   (W and nu themselves: k_eta_dmma with the DE flag, k_dgemm.cu.)
//
// All are per-gene (or per-coefficient) reductions over HBM-resident W, nu: bandwidth-bound
// and small next to the Gram of each sweep.
#include "gpl_internal.cuh"

namespace gpl {

__global__ void __launch_bounds__(256) k_de_zeta(int J, int P, const double* __restrict__ Beta,
                                                 const double* __restrict__ phi, double* __restrict__ zeta) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  double s = 0.0, d = 0.0;
  for (int j = threadIdx.x; j < J; j += blockDim.x) {
    s += Beta[k + (size_t)j * P] / phi[j];
    d += 1.0 / phi[j];
  }
  const double ss = block_sum(s, sh);
  const double sd = block_sum(d, sh);
  if (threadIdx.x == 0) zeta[k] = ss / sd;
}

int launch_de_zeta(Ctx* c) {
  {
    ProfScope ps(c, "de_zeta");
    k_de_zeta<<<c->P, 256, 0, c->stream>>>(c->J, c->P, c->Beta, c->phi, c->zeta);
    GPL_LAUNCHED(c, "k_de_zeta");
  }
  ProfScope ps(c, "zbeta");  // e0 = Z zeta feeds the next working response
  return launch_eta_one(c, c->zeta, c->e0);
}

__global__ void __launch_bounds__(256) k_de_beta_phi(int N, int ldN, int P, const double* __restrict__ W,
                                                     const double* __restrict__ Nu, const double* __restrict__ Omega,
                                                     const double* __restrict__ b, const double* __restrict__ sol,
                                                     const double* __restrict__ zeta, double* __restrict__ Beta,
                                                     double* __restrict__ phi) {
  __shared__ double sh[32];
  const int j = blockIdx.x;
  const double* Wj = W + (size_t)j * ldN;
  const double* nj = Nu + (size_t)j * ldN;
  double q = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) q += nj[i] * nj[i] * Wj[i] / Omega[i];
  double bs = 0.0;
  const double* sj = sol + (size_t)j * P;
  const double* bj = b + (size_t)j * P;
  double* beta = Beta + (size_t)j * P;
  for (int k = threadIdx.x; k < P; k += blockDim.x) {
    bs += sj[k] * bj[k];
    beta[k] = sj[k] + zeta[k];
  }
  const double sq = block_sum(q, sh);
  const double sb = block_sum(bs, sh);
  if (threadIdx.x == 0) {
    double ph = (sq - sb) / (double)N;
    if (isnan(ph)) ph = 1.0;
    if (ph < 0.0) ph = 100.0;
    if (ph < 0.01) ph = 0.01;
    if (ph > 100.0) ph = 100.0;
    phi[j] = ph;
  }
}

int launch_de_beta_phi(Ctx* c) {
  const int64_t PP = (int64_t)c->P * c->P;
  const int rc = launch_solve_batched(c, c->Psi, c->P, PP, c->bvec, c->P, c->sol, c->P, c->J);
  if (rc) return rc;
  ProfScope ps(c, "beta_phi");
  k_de_beta_phi<<<c->J, 256, 0, c->stream>>>(c->N, c->ldN, c->P, c->W, c->Nu, c->Omega, c->bvec, c->sol,
                                             c->zeta, c->Beta, c->phi);
  GPL_LAUNCHED(c, "k_de_beta_phi");
  return GPL_OK;
}

// Every cell contributes -W/Omega; a matched count (the reference's merge walk: the first
// gvalid entries of the gene) turns its cell's term into ((log W - dgp t) y - W)/Omega.
__global__ void __launch_bounds__(256) k_de_lkhd(int N, int ldN, int P, int p_eff, int pvars, const double* __restrict__ W,
                                                 const double* __restrict__ Omega, const double* __restrict__ delta,
                                                 const double* __restrict__ titsias, const int32_t* __restrict__ cell,
                                                 const int64_t* __restrict__ gptr, const int32_t* __restrict__ gvalid,
                                                 const double* __restrict__ cnt, const double* __restrict__ Psi,
                                                 const double* __restrict__ phi, double* __restrict__ lkhds) {
  __shared__ double sh[32];
  const int j = blockIdx.x;
  const double* Wj = W + (size_t)j * ldN;
  double part = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) part -= Wj[i] / Omega[i];
  const double dgp = delta[pvars - 1];
  const int64_t b = gptr[j], e = gptr[j] + gvalid[j];
  for (int64_t l = b + threadIdx.x; l < e; l += blockDim.x) {
    const int i = cell[l];
    const double w = Wj[i], om = Omega[i];
    part += ((log(w) - dgp * titsias[i]) * cnt[l] - w) / om + w / om;
  }
  const double* Lj = Psi + (size_t)j * P * P;
  double ld = 0.0;
  for (int k = threadIdx.x; k < p_eff; k += blockDim.x) ld += log(Lj[k + (size_t)k * P]);
  const double s = block_sum(part, sh);
  const double sl = block_sum(ld, sh);
  if (threadIdx.x == 0) lkhds[j] = (s - sl) / phi[j] + log(2 * 3.1415926535) * ((double)p_eff) / 2.0;
}

int launch_de_lkhd(Ctx* c, int slot) {
  {
    ProfScope ps(c, "lkhd_pois");
    const int p_eff = c->kernel_lv == kLvNone ? c->P - c->M : c->P;
    k_de_lkhd<<<c->J, 256, 0, c->stream>>>(c->N, c->ldN, c->P, p_eff, c->p, c->W, c->Omega, c->delta, c->titsias,
                                           c->cell, c->gptr, c->gvalid, c->cnt, c->Psi, c->phi, c->lkhds);
    GPL_LAUNCHED(c, "k_de_lkhd");
  }
  return launch_collect_lkhd(c, 0, slot);
}

}  // namespace gpl
