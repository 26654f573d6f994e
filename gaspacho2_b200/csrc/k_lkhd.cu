// Per-gene likelihood pieces and the IRLS coefficient update (replaces getBetaPhi
// ggplvm.cu:418-464, getLkhdPois :703-724, getLkhd/getLkhdj :744-784, collectLkhd :788-815,
// getOinvt :284-294, initBeta init.cu:193-221). All reductions are block-deterministic:
// a fixed shuffle tree per warp, then the warps in order.
//
//   k_oinvt       Oinvt_i = sum_j W_ij / Omega_i (thread per cell, genes in order) -> W column J
//   k_beta_phi    per gene: damped beta <- (1-r) beta + r Psi^{-1} b, phi from the residual
//                 quadratic form nu^T (W/Omega) nu - |L^T beta|^2, clamped as the reference
//   k_lkhd_pois   per gene: sum over matched counts of (log W - delta_GP titsias wt) y, minus sum W
//   k_lkhd_genes  per gene: the Laplace/PQL marginal l_j
//   k_collect     sum_j l_j - wt delta_GP sum_i Oinvt_i titsias_i - inverse-gamma prior on Omega
//                 (and the variance-component driver's N(0, 1) priors on X and T)
#include "gpl_internal.cuh"

namespace gpl {

// sum_j W_ij / Omega_i as (sum_j W_ij) / Omega_i: one division per cell instead of per entry,
// four independent partial sums (genes j = 4q + r in order within each) to keep loads in flight.
__global__ void k_oinvt(int N, int ldN, int J, const double* __restrict__ Omega, double* __restrict__ W) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int j = 0;
  for (; j + 4 <= J; j += 4) {
    s0 += W[(size_t)j * ldN + i];
    s1 += W[(size_t)(j + 1) * ldN + i];
    s2 += W[(size_t)(j + 2) * ldN + i];
    s3 += W[(size_t)(j + 3) * ldN + i];
  }
  for (; j < J; j++) s0 += W[(size_t)j * ldN + i];
  W[(size_t)J * ldN + i] = ((s0 + s1) + (s2 + s3)) / Omega[i];
}

int launch_oinvt(Ctx* c) {
  ProfScope ps(c, "oinvt");
  k_oinvt<<<div_up(c->N, 256), 256, 0, c->stream>>>(c->N, c->ldN, c->J, c->Omega, c->W);
  GPL_LAUNCHED(c, "k_oinvt");
  return GPL_OK;
}

// sol_j = Psi_j^{-1} b_j was solved beforehand.
__global__ void __launch_bounds__(256) k_beta_phi(int N, int ldN, int P, double r, const double* __restrict__ W,
                                                  const double* __restrict__ Nu, const double* __restrict__ Omega,
                                                  const double* __restrict__ Psi, const double* __restrict__ sol,
                                                  double* __restrict__ Beta, double* __restrict__ phi) {
  __shared__ double sh[32];
  extern __shared__ double sb[];  // P
  const int j = blockIdx.x;
  const double* Wj = W + (size_t)j * ldN;
  const double* nj = Nu + (size_t)j * ldN;
  double part = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) part += nj[i] * nj[i] * Wj[i] / Omega[i];
  const double quad = block_sum(part, sh);
  double* bj = Beta + (size_t)j * P;
  for (int k = threadIdx.x; k < P; k += blockDim.x) {
    const double nb = bj[k] * (1 - r) + sol[(size_t)j * P + k] * r;
    bj[k] = nb;
    sb[k] = nb;
  }
  __syncthreads();
  // |L^T beta|^2: row k of L^T is column k of L (rows >= k), one warp per k
  const double* L = Psi + (size_t)j * P * P;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double sq = 0.0;
  for (int k = wid; k < P; k += nw) {
    double t = 0.0;
    for (int i = k + lane; i < P; i += 32) t += L[i + (size_t)k * P] * sb[i];
    t = warp_sum(t);
    sq += t * t;
  }
  if (lane != 0) sq = 0.0;
  const double s2 = block_sum(sq, sh);
  if (threadIdx.x == 0) {
    double ph = (quad - s2) / (double)N;
    if (isnan(ph)) ph = 1.0;
    if (ph < 0.0) ph = 1.0;
    if (ph < 0.01) ph = 0.01;
    if (ph > 1000.0) ph = 1000.0;
    phi[j] = ph;
  }
}

// r = b - Z^T diag(W/Omega) (Z x) - DeltaInv x for every gene (bx holds the first product), one
// CTA per gene. DeltaInv is read from its upper triangle and diagonal, or, once cholDeltaInv has
// overwritten its lower triangle and diagonal with the factor L (factored), as L (L^T x).
__global__ void __launch_bounds__(256) k_residual(int P, int J, const double* __restrict__ b,
                                                  const double* __restrict__ bx, const double* __restrict__ Dinv,
                                                  int factored, const double* __restrict__ x,
                                                  double* __restrict__ r) {
  extern __shared__ double xs[];  // x_j, then L^T x_j
  const int j = blockIdx.x;
  const double* xj = x + (size_t)j * P;
  double* ts = xs + P;
  for (int k = threadIdx.x; k < P; k += blockDim.x) xs[k] = xj[k];
  __syncthreads();
  if (factored) {
    for (int k = threadIdx.x; k < P; k += blockDim.x) {
      double t = 0.0;
      for (int l = k; l < P; l++) t = fma(Dinv[l + (size_t)k * P], xs[l], t);
      ts[k] = t;
    }
    __syncthreads();
  }
  for (int k = threadIdx.x; k < P; k += blockDim.x) {
    double s = 0.0;
    if (factored)
      for (int l = 0; l <= k; l++) s = fma(Dinv[k + (size_t)l * P], ts[l], s);
    else
      for (int l = 0; l < P; l++) s = fma(Dinv[k <= l ? k + (size_t)l * P : l + (size_t)k * P], xs[l], s);
    const size_t e = (size_t)j * P + k;
    r[e] = b[e] - bx[e] - s;
  }
}

__global__ void k_add_to(size_t n, const double* __restrict__ d, double* __restrict__ x) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) x[e] += d[e];
}

// Psi_j x = b for every gene. In the precision form Psi_j carries the tensor-core Gram's
// error, so the solution is refined against the exact FP64 operator, applied without forming
// it: x += Psi~^{-1} (b - Z^T diag(W/Omega) Z x - DeltaInv x). The reference solves once with
// its FP64 Psi (cholsl in getBetaPhi / getTildeBeta); the refined x converges to that solution.
int solve_refined(Ctx* c, const double* b, double* x, bool dinv_factored) {
  const int64_t PP = (int64_t)c->P * c->P;
  int rc = launch_solve_batched(c, c->Psi, c->P, PP, b, c->P, x, c->P, c->J);
  if (rc || c->precision != GPL_PREC_BF16X3) return rc;
  ProfScope ps(c, "refine");
  for (int it = 0; it < c->refine_steps; it++) {
    if ((rc = launch_zbeta(c, x, c->scratch))) return rc;
    if ((rc = launch_zt_u_ex(c, 0, c->scratch, c->bx))) return rc;
    k_residual<<<c->J, 256, 2 * sizeof(double) * c->P, c->stream>>>(c->P, c->J, b, c->bx, c->DeltaInv,
                                                                     dinv_factored ? 1 : 0, x, c->rres);
    GPL_LAUNCHED(c, "k_residual");
    if ((rc = launch_solve_batched(c, c->Psi, c->P, PP, c->rres, c->P, c->bx, c->P, c->J))) return rc;
    const size_t n = (size_t)c->P * c->J;
    k_add_to<<<div_up((int64_t)n, 256), 256, 0, c->stream>>>(n, c->bx, x);
    GPL_LAUNCHED(c, "k_add_to");
  }
  return GPL_OK;
}

// phi from the exact quadratic form (precision form): beta^T Psi beta =
// sum_i (W_ij/Omega_i) (z_i . beta_j)^2 + beta^T DeltaInv beta with E = Z beta given, instead of
// |L^T beta|^2 with the factor of the tensor-core Gram; the same clamps as k_beta_phi.
__global__ void __launch_bounds__(256) k_phi_exact(int N, int ldN, int P, const double* __restrict__ W,
                                                   const double* __restrict__ Nu, const double* __restrict__ E,
                                                   const double* __restrict__ Omega, const double* __restrict__ Dinv,
                                                   const double* __restrict__ Beta, double* __restrict__ phi) {
  __shared__ double sh[32];
  const int j = blockIdx.x;
  const double* Wj = W + (size_t)j * ldN;
  const double* nj = Nu + (size_t)j * ldN;
  const double* ej = E + (size_t)j * ldN;
  double q = 0.0, s = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const double w = Wj[i] / Omega[i];
    q += nj[i] * nj[i] * w;
    s += ej[i] * ej[i] * w;
  }
  const double* bj = Beta + (size_t)j * P;
  double d = 0.0;
  for (int k = threadIdx.x; k < P; k += blockDim.x) {
    double t = 0.0;
    for (int l = 0; l < P; l++) t += Dinv[k <= l ? k + (size_t)l * P : l + (size_t)k * P] * bj[l];
    d += bj[k] * t;
  }
  const double sq = block_sum(q, sh);
  const double ss = block_sum(s, sh);
  const double sd = block_sum(d, sh);
  if (threadIdx.x == 0) {
    double ph = (sq - (ss + sd)) / (double)N;
    if (isnan(ph)) ph = 1.0;
    if (ph < 0.0) ph = 1.0;
    if (ph < 0.01) ph = 0.01;
    if (ph > 1000.0) ph = 1000.0;
    phi[j] = ph;
  }
}

int launch_beta_phi(Ctx* c, int jtr) {
  int rc = solve_refined(c, c->bvec, c->sol);
  if (rc) return rc;
  double r = (double)(jtr + 1) / 100.0;
  if (jtr > 100) r = 1.0;
  ProfScope ps(c, "beta_phi");
  k_beta_phi<<<c->J, 256, sizeof(double) * c->P, c->stream>>>(c->N, c->ldN, c->P, r, c->W, c->Nu, c->Omega, c->Psi,
                                                              c->sol, c->Beta, c->phi);
  GPL_LAUNCHED(c, "k_beta_phi");
  if (c->precision == GPL_PREC_BF16X3) {
    if ((rc = launch_zbeta(c, c->Beta, c->scratch))) return rc;
    k_phi_exact<<<c->J, 256, 0, c->stream>>>(c->N, c->ldN, c->P, c->W, c->Nu, c->scratch, c->Omega, c->DeltaInv,
                                              c->Beta, c->phi);
    GPL_LAUNCHED(c, "k_phi_exact");
  }
  return GPL_OK;
}

__global__ void __launch_bounds__(256) k_lkhd_pois(int N, int ldN, int pvars, double wt, const double* __restrict__ W,
                                                   const double* __restrict__ delta, const double* __restrict__ titsias,
                                                   const int32_t* __restrict__ cell, const int64_t* __restrict__ gptr,
                                                   const int32_t* __restrict__ gvalid, const double* __restrict__ cnt,
                                                   double* __restrict__ lkhds) {
  __shared__ double sh[32];
  const int j = blockIdx.x;
  const double* Wj = W + (size_t)j * ldN;
  double part = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) part -= Wj[i];
  const int64_t b = gptr[j], e = gptr[j] + gvalid[j];
  const double dgp = delta[pvars - 1];
  for (int64_t l = b + threadIdx.x; l < e; l += blockDim.x) {
    const int i = cell[l];
    part += (log(Wj[i]) - dgp * titsias[i] * wt) * cnt[l];
  }
  const double s = block_sum(part, sh);
  if (threadIdx.x == 0) lkhds[j] = s;
}

int launch_lkhd_pois(Ctx* c) {
  ProfScope ps(c, "lkhd_pois");
  // the variance-component driver takes the Titsias factor at weight 1 (ggplvm_delta.cu:610-631)
  k_lkhd_pois<<<c->J, 256, 0, c->stream>>>(c->N, c->ldN, c->p, c->vcomp ? 1.0 : kWt, c->W, c->delta, c->titsias, c->cell, c->gptr,
                                           c->gvalid, c->cnt, c->lkhds);
  GPL_LAUNCHED(c, "k_lkhd_pois");
  return GPL_OK;
}

// l_j = -N/2 log phi - sum_i log(Omega/W)/2 - sum_k log L_kk + sum_k log LD_kk
//       - sum_i nu^2 (W/Omega) / (2 phi) + b^T Psi^{-1} b / (2 phi)
__global__ void __launch_bounds__(256) k_lkhd_genes(int N, int ldN, int P, const double* __restrict__ W,
                                                    const double* __restrict__ Nu, const double* __restrict__ Omega,
                                                    const double* __restrict__ Psi, const double* __restrict__ LD,
                                                    const double* __restrict__ bvec, const double* __restrict__ sol,
                                                    const double* __restrict__ phi, double* __restrict__ lkhds) {
  __shared__ double sh[32];
  const int j = blockIdx.x;
  const double* Wj = W + (size_t)j * ldN;
  const double* nj = Nu + (size_t)j * ldN;
  const double phij = phi[j];
  double a = 0.0, q = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const double om = Omega[i], w = Wj[i];
    a += log(om / w);
    q += nj[i] * nj[i] * (w / om);
  }
  const double* L = Psi + (size_t)j * P * P;
  double ld = 0.0, bx = 0.0;
  for (int k = threadIdx.x; k < P; k += blockDim.x) {
    ld += log(LD[k + (size_t)k * P]) - log(L[k + (size_t)k * P]);
    bx += bvec[(size_t)j * P + k] * sol[(size_t)j * P + k];
  }
  const double sa = block_sum(a, sh);
  const double sq = block_sum(q, sh);
  const double sld = block_sum(ld, sh);
  const double sbx = block_sum(bx, sh);
  if (threadIdx.x == 0)
    lkhds[j] = -((double)N) / 2.0 * log(phij) - sa / 2.0 + sld - sq / 2.0 / phij + sbx / 2.0 / phij;
}

// y_j = bx_j + DeltaInv v_j (DeltaInv as its factor L once cholDeltaInv has run: L (L^T v)), one
// CTA per gene: the FP64 operator Psi_j applied to the probe v_j, with bx = Z^T diag(W/Omega) Z v.
__global__ void __launch_bounds__(256) k_probe_apply(int P, const double* __restrict__ bx,
                                                     const double* __restrict__ Dinv, int factored,
                                                     const double* __restrict__ v, double* __restrict__ y) {
  extern __shared__ double vs[];  // v_j, then L^T v_j
  const int j = blockIdx.x;
  const double* vj = v + (size_t)j * P;
  double* ts = vs + P;
  for (int k = threadIdx.x; k < P; k += blockDim.x) vs[k] = vj[k];
  __syncthreads();
  if (factored) {
    for (int k = threadIdx.x; k < P; k += blockDim.x) {
      double t = 0.0;
      for (int l = k; l < P; l++) t = fma(Dinv[l + (size_t)k * P], vs[l], t);
      ts[k] = t;
    }
    __syncthreads();
  }
  for (int k = threadIdx.x; k < P; k += blockDim.x) {
    double s = 0.0;
    if (factored)
      for (int l = 0; l <= k; l++) s = fma(Dinv[k + (size_t)l * P], ts[l], s);
    else
      for (int l = 0; l < P; l++) s = fma(Dinv[k <= l ? k + (size_t)l * P : l + (size_t)k * P], vs[l], s);
    const size_t e = (size_t)j * P + k;
    y[e] = bx[e] + s;
  }
}

// lkhds_j -= (v_j . z_j - P) / 2 with z_j = Psi~_j^{-1} Psi_j v_j: the log-determinant correction.
__global__ void __launch_bounds__(256) k_probe_logdet(int P, const double* __restrict__ v,
                                                      const double* __restrict__ z, double* __restrict__ lkhds) {
  __shared__ double sh[32];
  const int j = blockIdx.x;
  double s = 0.0;
  for (int k = threadIdx.x; k < P; k += blockDim.x) s += v[(size_t)j * P + k] * z[(size_t)j * P + k];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) lkhds[j] -= 0.5 * (s - (double)P);
}

// The precision form's log det Psi_j as a smooth function of the parameters. The tensor-core Gram
// is a staircase in them (its BF16 hi/lo operands hold 16 significant bits, so a parameter change
// below about 2^-16 relative leaves it unchanged), and so is log det Psi~_j: an L-BFGS step too short
// to move it sees an objective whose log-determinant part is frozen while its gradient is not. With
// a fixed Rademacher probe v_j (v_j . v_j = P),
//     log det Psi~_j + v_j^T Psi~_j^{-1} Psi_j v_j - P
// equals log det Psi_j up to second order in Psi_j - Psi~_j (the expression is stationary at
// Psi~_j = Psi_j) and moves with Psi_j, which the FP64 operator applies exactly (the refinement's
// Z x and Z^T diag(W/Omega) E passes); the probe's own error is of the size of
// |Psi~_j^{-1} (Psi_j - Psi~_j)|_F.
static int probe_logdet(Ctx* c) {
  TcState& t = c->tc;
  if (!t.probe) {
    c->err = "the log-determinant probe is allocated with the tensor-core buffers";
    return GPL_ERR_STATE;
  }
  ProfScope ps(c, "logdet_probe");
  const int64_t PP = (int64_t)c->P * c->P;
  int rc;
  if ((rc = launch_zbeta(c, t.probe, c->scratch))) return rc;            // Z v
  if ((rc = launch_zt_u_ex(c, 0, c->scratch, c->bx))) return rc;        // Z^T diag(W/Omega) Z v
  k_probe_apply<<<c->J, 256, 2 * sizeof(double) * c->P, c->stream>>>(c->P, c->bx, c->DeltaInv, 1, t.probe, c->rres);
  GPL_LAUNCHED(c, "k_probe_apply");
  if ((rc = launch_solve_batched(c, c->Psi, c->P, PP, c->rres, c->P, c->bx, c->P, c->J))) return rc;
  k_probe_logdet<<<c->J, 256, 0, c->stream>>>(c->P, t.probe, c->bx, c->lkhds);
  GPL_LAUNCHED(c, "k_probe_logdet");
  return GPL_OK;
}

int launch_lkhd_genes(Ctx* c) {
  // b^T Psi^{-1} b enters as the difference q - b^T x of two large sums: in the precision form
  // x is refined against the FP64 operator (a 1e-6 error in x would survive the cancellation)
  int rc = solve_refined(c, c->bvec, c->sol, true);  // cholDeltaInv has run (ggplvm.cu:1206,1266)
  if (rc) return rc;
  {
    ProfScope ps(c, "lkhd_genes");
    k_lkhd_genes<<<c->J, 256, 0, c->stream>>>(c->N, c->ldN, c->P, c->W, c->Nu, c->Omega, c->Psi, c->DeltaInv,
                                              c->bvec, c->sol, c->phi, c->lkhds);
    GPL_LAUNCHED(c, "k_lkhd_genes");
  }
  if (c->precision == GPL_PREC_BF16X3 && c->logdet_probe) return probe_logdet(c);
  return GPL_OK;
}

// sum_j l_j - Q-prior - wt delta_GP sum_i Oinvt_i titsias_i - sum_i (igb/Omega_i + iga log Omega_i);
// Q-prior: N(0, 1) on X and T in dimensions 1..qp-1 (qp = 0 for none). The fit driver:
// wt = 0.1, igb = iga = 100, qp = 0 (ggplvm.cu:788-815); the variance-component driver: wt = 0,
// 30, 30 and qp = Q (ggplvm_delta.cu:677-704).
__global__ void __launch_bounds__(1024) k_collect(int J, int n, int ldN, int pvars, double wt, double igb, double iga,
                                                  int qp, int M, const double* __restrict__ X,
                                                  const double* __restrict__ T, const double* __restrict__ lkhds,
                                                  const double* __restrict__ W, const double* __restrict__ titsias,
                                                  const double* __restrict__ Omega, const double* __restrict__ delta,
                                                  double* __restrict__ out) {
  __shared__ double sh[32];
  double s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
  for (int k = threadIdx.x; k < J; k += blockDim.x) s1 += lkhds[k];
  const double* Oinvt = W + (size_t)J * ldN;
  const double dgp = delta[pvars - 1];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    s2 += wt * dgp * Oinvt[i] * titsias[i];
    s3 += igb / Omega[i] + iga * log(Omega[i]);
    for (int k = 1; k < qp; k++) s4 += X[i + (size_t)k * n] * X[i + (size_t)k * n] / 2.0;
  }
  for (int i = threadIdx.x; i < M && qp > 1; i += blockDim.x)
    for (int k = 1; k < qp; k++) s4 += T[i + (size_t)k * M] * T[i + (size_t)k * M] / 2.0;
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  s3 = block_sum(s3, sh);
  s4 = block_sum(s4, sh);
  if (threadIdx.x == 0) out[0] = s1 - s4 - s2 - s3;
}

int launch_collect_lkhd(Ctx* c, int n_cells, int slot) {
  ProfScope ps(c, "collect");
  const int qp = (c->vcomp && n_cells > 0) ? c->Q : 0;
  k_collect<<<1, 1024, 0, c->stream>>>(c->J, n_cells, c->ldN, c->p, c->vcomp ? 0.0 : kWt, c->vcomp ? 30.0 : kIgb,
                                       c->vcomp ? 30.0 : kIgap1, qp, c->M, c->X, c->T, c->lkhds, c->W, c->titsias,
                                       c->Omega, c->delta, c->lkhd_dev + slot);
  GPL_LAUNCHED(c, "k_collect");
  return GPL_OK;
}

int launch_init_beta_solve(Ctx* c) {
  // one factor (Psi slot 0) for every gene's right-hand side
  return launch_solve_batched(c, c->Psi, c->P, 0, c->bvec, c->P, c->Beta, c->P, c->J);
}

}  // namespace gpl
