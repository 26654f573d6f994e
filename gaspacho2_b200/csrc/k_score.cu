// Genotype score statistics against the fitted model (getScoreStats, ggplvm_de.cu:489-535;
// launched after the fit over a J x L grid, :1205-1209). For gene j and genotype column g_l:
//   t = Z^T diag(W_j/Omega) g_l,  v = sum_i g_il^2 W_ij / Omega_i - t^T Psi_j^{-1} t,
//   s = sum_i g_il / Omega_i (y_ij - W_ij)  (matched counts; -g W / Omega elsewhere),
//   S[j, l] = s / sqrt(phi_j v).
// Here t is the Z^T u GEMM with a per-cell u (k_dgen), Psi_j^{-1} t the batched solve with the
// factor of the last objective, the two sums over all cells one split-K DMMA GEMM of W against
// [g^2/Omega | g/Omega], and the count sum a walk over each gene's matched prefix.
#include "gpl_internal.cuh"

namespace gpl {

// G2[c][i] = g_il^2 / Omega_i (c = l < L) and g_il / Omega_i (c = L + l)
__global__ void k_score_cols(int N, int L, const double* __restrict__ G, const double* __restrict__ Omega,
                             double* __restrict__ G2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y;
  if (i >= N) return;
  const double g = G[(size_t)l * N + i];
  G2[(size_t)l * N + i] = g * g / Omega[i];
  G2[(size_t)(L + l) * N + i] = g / Omega[i];
}

// td[j + l*J] = t_j . (Psi_j^{-1} t_j), one warp per gene
__global__ void k_score_dot(int J, int P, int l, const double* __restrict__ t, const double* __restrict__ t2,
                            double* __restrict__ td) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (j >= J) return;
  double s = 0.0;
  for (int k = lane; k < P; k += 32) s += t[(size_t)j * P + k] * t2[(size_t)j * P + k];
  s = warp_sum(s);
  if (lane == 0) td[j + (size_t)l * J] = s;
}

// sp[j + l*J] = sum over gene j's matched counts of g_il y / Omega_i, one CTA per gene
__global__ void __launch_bounds__(128) k_score_counts(int N, int J, int L, const int32_t* __restrict__ cell,
                                                      const int64_t* __restrict__ gptr,
                                                      const int32_t* __restrict__ gvalid,
                                                      const double* __restrict__ cnt, const double* __restrict__ G,
                                                      const double* __restrict__ Omega, double* __restrict__ sp) {
  __shared__ double sh[32];
  const int j = blockIdx.x;
  const int64_t b = gptr[j], e = gptr[j] + gvalid[j];
  for (int l = 0; l < L; l++) {
    double part = 0.0;
    for (int64_t q = b + threadIdx.x; q < e; q += blockDim.x) {
      const int i = cell[q];
      part += G[(size_t)l * N + i] * cnt[q] / Omega[i];
    }
    const double s = block_sum(part, sh);
    if (threadIdx.x == 0) sp[j + (size_t)l * J] = s;
    __syncthreads();
  }
}

// S = (sp - sum W g/Omega) / sqrt(phi (sum W g^2/Omega - td))
__global__ void k_score_final(int J, int L, const double* __restrict__ sp, const double* __restrict__ C,
                              const double* __restrict__ td, const double* __restrict__ phi,
                              double* __restrict__ S) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y;
  if (j >= J) return;
  const size_t e = j + (size_t)l * J;
  const double v = C[e] - td[e];
  S[e] = (sp[e] - C[j + (size_t)(L + l) * J]) / sqrt(phi[j] * v);
}

int launch_score_stats(Ctx* c, int L, const double* G, double* S, double* scratch) {
  // scratch: G2 (2L x N), C (J x 2L), td (J x L), sp (J x L)
  double* G2 = scratch;
  double* C = G2 + (size_t)2 * L * c->N;
  double* td = C + (size_t)2 * L * c->J;
  double* sp = td + (size_t)L * c->J;
  int rc;
  for (int l = 0; l < L; l++) {
    if ((rc = launch_zt_u_ex(c, 2, G + (size_t)l * c->N, c->bx))) return rc;
    if ((rc = launch_solve_batched(c, c->Psi, c->P, (int64_t)c->P * c->P, c->bx, c->P, c->rres, c->P, c->J)))
      return rc;
    k_score_dot<<<div_up(c->J, 8), 256, 0, c->stream>>>(c->J, c->P, l, c->bx, c->rres, td);
    GPL_LAUNCHED(c, "k_score_dot");
  }
  k_score_cols<<<dim3(div_up(c->N, 256), L), 256, 0, c->stream>>>(c->N, L, G, c->Omega, G2);
  GPL_LAUNCHED(c, "k_score_cols");
  if ((rc = dgen_weighted_colsums(c, G2, 2 * L, C))) return rc;
  k_score_counts<<<c->J, 128, 0, c->stream>>>(c->N, c->J, L, c->cell, c->gptr, c->gvalid, c->cnt, G, c->Omega, sp);
  GPL_LAUNCHED(c, "k_score_counts");
  k_score_final<<<dim3(div_up(c->J, 256), L), 256, 0, c->stream>>>(c->J, L, sp, C, td, c->phi, S);
  GPL_LAUNCHED(c, "k_score_final");
  return GPL_OK;
}

}  // namespace gpl
