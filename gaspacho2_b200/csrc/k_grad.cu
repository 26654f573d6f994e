// Gradient of the objective (replaces getGradLogDelta/collectGradLogDelta ggplvm.cu:210-281,
// getGradLogOmega :301-376, getC2 :57-100, getGradTau :103-145, getGradLogRho/collect
// :148-205).
//
// The reference solves Psi_j z_i for every (cell, gene) pair (N*J solves of size P). Here
// the explicit inverses S_j = Psi_j^{-1} are formed once per gene and the per-cell sums
// over genes become one contraction over the dense columns d_i of z_i,
//     A[i, a] = sum_j O_ij (S_j[DD] d_i)_a = sum_{j,b} (O_ij d_ib) S_j[b, a],   O = W / Omega
// plus per-group terms for the categorical levels (k_groups.cu). k_uq runs A as an FP64
// GEMM over the flattened (gene, dense column) index with the left operand O_ij d_ib formed
// while loading. Bound: FP64 FMA, N*J*n_d^2.
#include "gpl_internal.cuh"

namespace gpl {

namespace {
constexpr int TM = 64, TN = 64, TK = 16;
}

// ---- d/d log delta ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_grad_delta(int P, int M, int g0, const int* __restrict__ mk,
                                                    const double* __restrict__ delta, const double* __restrict__ K,
                                                    const double* __restrict__ S, const double* __restrict__ tBeta,
                                                    const double* __restrict__ phi, double* __restrict__ gdtmp) {
  __shared__ double sh[32];
  __shared__ double sq;
  const int j = blockIdx.x;
  const double* Sj = S + (size_t)j * P * P;
  const double* tb = tBeta + (size_t)j * P;
  // tb_GP^T Kmm tb_GP (quadform, util_cuda.cu:442-451)
  double part = 0.0;
  for (int a = threadIdx.x; a < M; a += blockDim.x) {
    double t = K[a + a * M] * tb[g0 + a];
    for (int b = a + 1; b < M; b++) t += 2.0 * K[a + b * M] * tb[g0 + b];
    part += tb[g0 + a] * t;
  }
  const double q = block_sum(part, sh);
  if (threadIdx.x == 0) sq = q;
  __syncthreads();
  const double phij = phi[j];
  for (int k = threadIdx.x; k < P; k += blockDim.x) {
    const double dk = delta[mk[k]];
    double psikk;
    if (k < g0) {
      psikk = Sj[k + (size_t)k * P];
    } else {  // (S_j Kmm[:, kk])_k over the GP block
      const int kk = k - g0;
      psikk = 0.0;
      for (int l = 0; l < M; l++) {
        const double kv = l < kk ? K[l + kk * M] : K[kk + l * M];
        psikk += Sj[k + (size_t)(g0 + l) * P] * kv;
      }
    }
    double sum = -(dk - psikk) / dk / dk / 2.0;
    if (k < g0) sum += tb[k] * tb[k] / dk / dk / phij / 2.0;
    else if (k == g0) sum += sq / dk / dk / phij / 2.0;
    gdtmp[k + (size_t)j * P] = sum * dk;
  }
}

__global__ void __launch_bounds__(256) k_collect_delta(int J, int P, int N, int ldN, int pvars,
                                                       const int* __restrict__ nh, const double* __restrict__ gdtmp,
                                                       const double* __restrict__ W, const double* __restrict__ titsias,
                                                       const double* __restrict__ delta, double* __restrict__ grad) {
  __shared__ double sh[32];
  const int l = blockIdx.x;
  const int k0 = nh[l], nk = nh[l + 1] - nh[l];
  double s = 0.0;
  for (int64_t e = threadIdx.x; e < (int64_t)J * nk; e += blockDim.x) {
    const int j = (int)(e / nk), k = k0 + (int)(e % nk);
    s += gdtmp[k + (size_t)j * P];
  }
  double t = 0.0;
  if (l == pvars - 1) {
    const double* Oinvt = W + (size_t)J * ldN;
    const double d = delta[pvars - 1];
    for (int i = threadIdx.x; i < N; i += blockDim.x) t += kWt * Oinvt[i] * titsias[i] * d;
  }
  s = block_sum(s, sh);
  t = block_sum(t, sh);
  if (threadIdx.x == 0) grad[N + l] = s - t;
}

int launch_grad_delta(Ctx* c) {
  ProfScope ps(c, "grad_delta");
  const int g0 = c->nh[c->p - 1];
  k_grad_delta<<<c->J, 256, 0, c->stream>>>(c->P, c->M, g0, c->mk_d, c->delta, c->Kmm, c->PsiInv, c->tBeta, c->phi,
                                            c->gdtmp);
  GPL_LAUNCHED(c, "k_grad_delta");
  k_collect_delta<<<c->p, 256, 0, c->stream>>>(c->J, c->P, c->N, c->ldN, c->p, c->nh_d, c->gdtmp, c->W, c->titsias,
                                               c->delta, c->grad);
  GPL_LAUNCHED(c, "k_collect_delta");
  return GPL_OK;
}

// ---- A = sum_j O_ij S_j[DD] d_i --------------------------------------------------------------
__global__ void __launch_bounds__(256) k_uq(int N, int ldN, int n_d, int n_dp, int P, int J,
                                            const double* __restrict__ D, const int* __restrict__ dcol,
                                            const double* __restrict__ W, const double* __restrict__ Omega,
                                            const double* __restrict__ S, double* __restrict__ U) {
  __shared__ double As[TK][TM + 1];
  __shared__ double Bs[TK][TN + 1];
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[4][4];
#pragma unroll
  for (int x = 0; x < 4; x++)
#pragma unroll
    for (int y = 0; y < 4; y++) acc[x][y] = 0.0;
  for (int j = 0; j < J; j++) {
    const double* Sj = S + (size_t)j * P * P;
    for (int b0 = 0; b0 < n_dp; b0 += TK) {
#pragma unroll
      for (int t = 0; t < (TM * TK) / 256; t++) {
        const int e = tid + t * 256;
        const int r = e % TM, k = e / TM;
        const int i = m0 + r, b = b0 + k;
        double v = 0.0;
        if (i < N && b < n_d) v = W[(size_t)j * ldN + i] / Omega[i] * D[(size_t)b * ldN + i];
        As[k][r] = v;
      }
#pragma unroll
      for (int t = 0; t < (TN * TK) / 256; t++) {
        const int e = tid + t * 256;
        const int k = e % TK, cc = e / TK;
        const int b = b0 + k, a = n0 + cc;
        Bs[k][cc] = (b < n_d && a < n_d) ? Sj[dcol[b] + (size_t)dcol[a] * P] : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < TK; k++) {
        double av[4], bv[4];
#pragma unroll
        for (int x = 0; x < 4; x++) av[x] = As[k][tx + 16 * x];
#pragma unroll
        for (int y = 0; y < 4; y++) bv[y] = Bs[k][ty + 16 * y];
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
          for (int y = 0; y < 4; y++) acc[x][y] = fma(av[x], bv[y], acc[x][y]);
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int x = 0; x < 4; x++) {
    const int i = m0 + tx + 16 * x;
    if (i >= N) continue;
#pragma unroll
    for (int y = 0; y < 4; y++) {
      const int a = n0 + ty + 16 * y;
      if (a < n_d) U[i + (size_t)a * ldN] = acc[x][y];
    }
  }
}

// per cell: sum_j tn_ij^2 / W_ij / phi_j with tn = O (nu - E), E = z_i . tBeta_j (in scratch)
__global__ void k_recip(int n, const double* __restrict__ x, double* __restrict__ r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = 1.0 / x[i];
}

__global__ void k_tn_sum(int N, int ldN, int J, const double* __restrict__ W, const double* __restrict__ Nu,
                         const double* __restrict__ E, const double* __restrict__ Omega,
                         const double* __restrict__ rphi, double* __restrict__ out) {
  // tn^2 / W / phi / 2 with tn = (W/Omega)(nu - E) is W (nu - E)^2 / (2 phi Omega^2): no division
  // per entry; four independent partial sums (genes 4q + r) keep loads in flight.
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  int j = 0;
  for (; j + 4 <= J; j += 4) {
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const size_t e = (size_t)(j + r) * ldN + i;
      const double d = Nu[e] - E[e];
      s[r] += W[e] * d * d * rphi[j + r];
    }
  }
  for (; j < J; j++) {
    const size_t e = (size_t)j * ldN + i;
    const double d = Nu[e] - E[e];
    s[0] += W[e] * d * d * rphi[j];
  }
  const double om = Omega[i];
  out[i] = ((s[0] + s[1]) + (s[2] + s[3])) / (2.0 * om * om);
}

// per-cell epilogue of getGradLogOmega (ggplvm.cu:352-374). With A = U (dense rows of
// sum_j O_ij S_j z_i without the level terms) and HK = [sum_j O_ij h_{j,g(i)} | sum_j O_ij
// kappa_{j,g(i)}] (absent when no variable is grouped):
//   sum_j O_ij z_i^T S_j z_i = d_i . (A_i + 2 H_i) + K_i,   sum_j O_ij (S_j z_i)_GP = A_i[GP] + H_i[GP]
__global__ void k_grad_omega_cell(int N, int ldN, int n_d, int dg0, int J, int M, int Q, int pvars,
                                  const double* __restrict__ D, const double* __restrict__ U,
                                  const double* __restrict__ HK, const double* __restrict__ tnsum,
                                  const double* __restrict__ W, const double* __restrict__ Omega,
                                  const double* __restrict__ delta, const double* __restrict__ titsias,
                                  const double* __restrict__ KinvKmn, const double* __restrict__ X,
                                  const double* __restrict__ T, const double* __restrict__ rho,
                                  double* __restrict__ C1, double* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double om = Omega[i];
  const double Oii = W[(size_t)J * ldN + i];
  double q = 0.0;
  for (int a = 0; a < n_d; a++) {
    double u = U[i + (size_t)a * ldN];
    if (HK) u += 2.0 * HK[i + (size_t)a * ldN];
    q += D[(size_t)a * ldN + i] * u;
  }
  if (HK) q += HK[i + (size_t)n_d * ldN];
  const double dgp = delta[pvars - 1];
  double sum = -((double)J) / om / 2.0 + q / om / 2.0 + tnsum[i];
  sum += kWt * dgp * Oii / om * titsias[i];
  grad[i] = sum * om + kIgb / om - kIgap1;
  double* gX = grad + N + pvars;
  double ci1 = 0.0, g0x = 0.0;
  for (int k = 0; k < M; k++) {
    double v = U[i + (size_t)(dg0 + k) * ldN];
    if (HK) v += HK[i + (size_t)(dg0 + k) * ldN];
    double cik = C1[i + (size_t)k * ldN] - v;
    cik += kWt * dgp * Oii * KinvKmn[i + (size_t)k * ldN];
    cik *= D[(size_t)(dg0 + k) * ldN + i];
    C1[i + (size_t)k * ldN] = cik;
    ci1 += cik;
    const double t = (X[i] - T[k]) / 2.0;
    g0x -= cik * sin(t) * cos(t) / rho[0];
  }
  gX[i] = g0x;
  for (int qd = 1; qd < Q; qd++) {
    double d = 0.0;
    for (int k = 0; k < M; k++) d += C1[i + (size_t)k * ldN] * T[k + qd * M];
    gX[i + (size_t)qd * N] = (d - ci1 * X[i + (size_t)qd * N]) / rho[qd];
  }
}

int launch_grad_omega(Ctx* c) {
  int rc = launch_zbeta(c, c->tBeta, c->scratch);  // E = Z tBeta
  if (rc) return rc;
  {
    ProfScope ps(c, "tn_sum");
    k_recip<<<div_up(c->J, 256), 256, 0, c->stream>>>(c->J, c->phi, c->rphi);
    GPL_LAUNCHED(c, "k_recip");
    k_tn_sum<<<div_up(c->N, 128), 128, 0, c->stream>>>(c->N, c->ldN, c->J, c->W, c->Nu, c->scratch, c->Omega,
                                                       c->rphi, c->red);
    GPL_LAUNCHED(c, "k_tn_sum");
  }
  rc = launch_c1_tn(c);  // C1 = sum_j tn/phi tBeta_GP
  if (rc) return rc;
  if (c->precision == GPL_PREC_BF16X3 && c->tc_grad) {
    rc = launch_tc_grad(c);
    if (rc) return rc;
  } else if ((rc = launch_pair_uq(c)) != GPL_ERR_ARG) {
    if (rc) return rc;
  } else {  // more dense columns than the staged pair contraction holds
    ProfScope ps(c, "uq");
    const int n_dp = div_up(c->n_d, TK) * TK;
    dim3 g(div_up(c->N, TM), div_up(c->n_d, TN));
    k_uq<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->n_d, n_dp, c->P, c->J, c->Dm, c->dcol_d, c->W, c->Omega,
                                   c->PsiInv, c->U);
    GPL_LAUNCHED(c, "k_uq");
  }
  rc = launch_group_tables(c);
  if (rc) return rc;
  rc = launch_hk(c);
  if (rc) return rc;
  ProfScope ps(c, "grad_omega_cell");
  k_grad_omega_cell<<<div_up(c->N, 128), 128, 0, c->stream>>>(
      c->N, c->ldN, c->n_d, c->dg0, c->J, c->M, c->Q, c->p, c->Dm, c->U, c->n_grp ? c->HK : nullptr, c->red, c->W,
      c->Omega, c->delta, c->titsias, c->KinvKmn, c->X, c->T, c->rho, c->C1, c->grad);
  GPL_LAUNCHED(c, "k_grad_omega_cell");
  return GPL_OK;
}

// ---- C2 (M x M adjoint of Kmm) --------------------------------------------------------------
__global__ void __launch_bounds__(256) k_c2(int N, int ldN, int J, int P, int M, int g0, int pvars,
                                            const double* __restrict__ KinvKmn, const double* __restrict__ W,
                                            const double* __restrict__ tBeta, const double* __restrict__ phi,
                                            const double* __restrict__ S, const double* __restrict__ KmmInv,
                                            const double* __restrict__ K, const double* __restrict__ delta,
                                            double* __restrict__ C2) {
  __shared__ double sh[32];
  // blockIdx.x enumerates pairs j <= k
  int k = (int)((sqrt(8.0 * blockIdx.x + 1.0) - 1.0) * 0.5);
  while ((k + 1) * (k + 2) / 2 <= (int)blockIdx.x) k++;
  while (k * (k + 1) / 2 > (int)blockIdx.x) k--;
  const int j = (int)blockIdx.x - k * (k + 1) / 2;
  const double* Oinvt = W + (size_t)J * ldN;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x)
    s1 += KinvKmn[i + (size_t)j * ldN] * KinvKmn[i + (size_t)k * ldN] * Oinvt[i];
  for (int g = threadIdx.x; g < J; g += blockDim.x) {
    s2 += tBeta[j + g0 + (size_t)g * P] * tBeta[k + g0 + (size_t)g * P] / phi[g];
    s3 += S[(size_t)g * P * P + (size_t)(k + g0) * P + (j + g0)];
  }
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  s3 = block_sum(s3, sh);
  if (threadIdx.x == 0) {
    const double d = delta[pvars - 1];
    double v = -kWt * d * s1 / 2.0;
    v -= s2 / d / 2.0;
    v -= s3 / d / 2.0;
    v += ((double)J) * KmmInv[j + k * M] / 2.0;
    v *= K[j + k * M];
    C2[j + k * M] = v;
    if (j < k) C2[k + j * M] = v;
  }
}

int launch_c2(Ctx* c) {
  ProfScope ps(c, "c2");
  // Kmm^{-1} from the factor in Kinv's lower triangle (column k = cholsl(Kinv, e_k))
  int rc = launch_cholinv_exact(c, c->Kinv, c->M, c->KmmInv);
  if (rc) return rc;
  const int np = c->M * (c->M + 1) / 2;
  k_c2<<<np, 256, 0, c->stream>>>(c->N, c->ldN, c->J, c->P, c->M, c->nh[c->p - 1], c->p, c->KinvKmn, c->W, c->tBeta,
                                  c->phi, c->PsiInv, c->KmmInv, c->Kmm, c->delta, c->C2);
  GPL_LAUNCHED(c, "k_c2");
  return GPL_OK;
}

// ---- d/dT and d/dlog rho -------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_grad_tau_rho(int N, int ldN, int M, int Q, int pvars,
                                                      const double* __restrict__ X, const double* __restrict__ T,
                                                      const double* __restrict__ rho, const double* __restrict__ C1,
                                                      const double* __restrict__ C2, double* __restrict__ grad,
                                                      double* __restrict__ grtmp) {
  __shared__ double sh[32];
  const int m = blockIdx.x, q = blockIdx.y;
  const double rq = rho[q];
  const double* c1 = C1 + (size_t)m * ldN;
  double a1 = 0.0, a2 = 0.0, r1 = 0.0;  // tau sums over cells, rho sum over cells
  double b1 = 0.0, b2 = 0.0, r2 = 0.0;  // the same over inducing points
  if (q == 0) {
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      const double t = (X[i] - T[m]) / 2.0;
      const double st = sin(t);
      a1 += c1[i] * st * cos(t);
      r1 += c1[i] * st * st / rq / rq;
    }
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
      const double t = (T[i] - T[m]) / 2.0;
      const double st = sin(t);
      b1 += C2[m + i * M] * st * cos(t);
      r2 += C2[i + m * M] * st * st / rq / rq;
    }
  } else {
    const double tm = T[m + q * M];
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      const double xi = X[i + (size_t)q * N];
      a1 += c1[i] * xi;
      a2 += c1[i];
      const double d = xi - tm;
      r1 += c1[i] * d * d / rq / rq / 2.0;
    }
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
      b1 += C2[m + i * M] * T[i + q * M];
      b2 += C2[m + i * M];
      const double d = T[i + q * M] - tm;
      r2 += C2[i + m * M] * d * d / rq / rq / 2.0;
    }
  }
  a1 = block_sum(a1, sh);
  a2 = block_sum(a2, sh);
  b1 = block_sum(b1, sh);
  b2 = block_sum(b2, sh);
  r1 = block_sum(r1, sh);
  r2 = block_sum(r2, sh);
  if (threadIdx.x == 0) {
    double* gT = grad + N + pvars + (size_t)N * Q;
    if (q == 0) {
      gT[m] = a1 / rho[0] + 2.0 * b1 / rho[0];
    } else {
      const double tm = T[m + q * M];
      gT[m + q * M] = (a1 - a2 * tm) / rq + 2.0 * (b1 - b2 * tm) / rq;
    }
    grtmp[q + m * Q] = (r1 + r2) * rq;
  }
}

__global__ void k_collect_rho(int N, int M, int Q, int pvars, const double* __restrict__ grtmp,
                              double* __restrict__ grad) {
  const int q = threadIdx.x;
  if (q >= Q) return;
  double s = 0.0;
  for (int k = 0; k < M; k++) s += grtmp[q + k * Q];
  grad[N + pvars + (size_t)N * Q + (size_t)M * Q + q] = s;
}

int launch_grad_tau_rho(Ctx* c) {
  ProfScope ps(c, "grad_tau_rho");
  dim3 g(c->M, c->Q);
  k_grad_tau_rho<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->M, c->Q, c->p, c->X, c->T, c->rho, c->C1, c->C2,
                                           c->grad, c->grtmp);
  GPL_LAUNCHED(c, "k_grad_tau_rho");
  k_collect_rho<<<1, 32 * div_up(c->Q, 32), 0, c->stream>>>(c->N, c->M, c->Q, c->p, c->grtmp, c->grad);
  GPL_LAUNCHED(c, "k_collect_rho");
  return GPL_OK;
}

}  // namespace gpl
