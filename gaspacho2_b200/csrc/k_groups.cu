// Categorical covariates through cell groups.
//
// A categorical variable contributes one-hot columns to the model matrix (getModelMatrix,
// DataFrame.cu:72-82), and the reference's Gram treats them case by case
// (ggplvm.cu:628-674): level x numeric sums, level x level co-occurrence sums. Here every
// cell belongs to the group of its combination of levels (400 groups for batch x donor at
// config 2), and everything categorical reduces to per-(gene, group) sums over the cells of
// a group:
//
//   S[j][g][a] = sum_{i in g} w_ij D[i, a]       (dense column a; a = intercept gives sum w)
//   T[j][g]    = sum_{i in g} w_ij u_ij          (u = nu for Z^T diag(w) nu, y0 for initBeta)
//
// from which the categorical rows of Psi_j and of Z^T diag(w) nu are assembled exactly as the
// reference's case analysis defines them. In the gradient the same layout holds the
// categorical blocks of Psi_j^{-1} seen by each group:
//
//   h[j][g][a] = sum_{c in cats(g)} S_j[dcol[a], c],  kappa[j][g] = sum_{c,c' in cats(g)} S_j[c, c']
//
// so that z_i^T S_j z_i = d_i^T S_DD d_i + 2 d_i . h + kappa for a cell of group g.
// The group sums and HK are FP64 GEMMs over the gathered cells of one group (the shared
// register-tiled tile of k_gemm.cu's scheme), N*J*n_d multiply-adds each.
#include <algorithm>

#include "gpl_internal.cuh"

namespace gpl {

namespace {
constexpr int TM = 64, TN = 64, TK = 16;
}

// C[r, c] over K = gathered cells of group g: A(r = gene, k) = w(cell_k, gene), B(k, c = a) = D[a, cell_k]
template <int MODE>
__global__ void __launch_bounds__(256) k_group_sums(int N, int ldN, int J, int n_d, int n_grp,
                                                    const int* __restrict__ gcells, const int* __restrict__ gstart,
                                                    const double* __restrict__ W, const double* __restrict__ Omega,
                                                    const double* __restrict__ D, double* __restrict__ S) {
  __shared__ double As[TK][TM + 1];
  __shared__ double Bs[TK][TN + 1];
  const int g = blockIdx.z;
  const int j0 = blockIdx.x * TM, a0 = blockIdx.y * TN;
  const int c0 = gstart[g], nc = gstart[g + 1] - c0;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[4][4];
#pragma unroll
  for (int x = 0; x < 4; x++)
#pragma unroll
    for (int y = 0; y < 4; y++) acc[x][y] = 0.0;
  for (int k0 = 0; k0 < nc; k0 += TK) {
#pragma unroll
    for (int t = 0; t < (TM * TK) / 256; t++) {  // A: k fastest over cells
      const int e = tid + t * 256;
      const int k = e % TK, r = e / TK;
      const int j = j0 + r;
      double v = 0.0;
      if (k0 + k < nc && j < J) {
        const int i = gcells[c0 + k0 + k];
        v = MODE == 0 ? W[(size_t)j * ldN + i] / Omega[i] : 1.0;
      }
      As[k][r] = v;
    }
#pragma unroll
    for (int t = 0; t < (TN * TK) / 256; t++) {  // B: k fastest (cells of one dense column)
      const int e = tid + t * 256;
      const int k = e % TK, cc = e / TK;
      const int a = a0 + cc;
      double v = 0.0;
      if (k0 + k < nc && a < n_d) v = D[(size_t)a * ldN + gcells[c0 + k0 + k]];
      Bs[k][cc] = v;
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
  const int ld = n_d + 1;
#pragma unroll
  for (int x = 0; x < 4; x++) {
    const int j = j0 + tx + 16 * x;
    if (j >= J) continue;
#pragma unroll
    for (int y = 0; y < 4; y++) {
      const int a = a0 + ty + 16 * y;
      if (a < n_d) S[((size_t)j * n_grp + g) * ld + a] = acc[x][y];
    }
  }
}

// T[j][g] = sum_{i in g} w_ij u_ij, one warp per (gene, group); mode 0: w = W/Omega, u = nu;
// mode 2: w = 1, u = y0 (scratch).
template <int MODE>
__global__ void k_group_t(int ldN, int J, int n_grp, const int* __restrict__ gcells, const int* __restrict__ gstart,
                          const double* __restrict__ Wg, const double* __restrict__ Omega,
                          const double* __restrict__ U, double* __restrict__ T) {
  const int g = blockIdx.x;
  const int j = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= J) return;
  const int c0 = gstart[g], c1 = gstart[g + 1];
  double s = 0.0;
  for (int k = c0 + lane; k < c1; k += 32) {
    const int i = gcells[k];
    const size_t e = (size_t)j * ldN + i;
    if (MODE == 2) {
      s += U[e];
    } else {
      const double w = Wg[(size_t)j * ldN + k];  // W of cell i, read in group order
      s += MODE == 0 ? w / Omega[i] * U[e] : w / Omega[i] * U[i];
    }
  }
  s = warp_sum(s);
  if (lane == 0) T[(size_t)j * n_grp + g] = s;
}

// mode 0: S with w = W/Omega (Gram of the objective and the IRLS); 1: S of gene 0 with w = 1
// (GLM initialisation Gram); 2: T with w = 1, u = y0 (GLM initialisation right-hand side);
// 3: T with w = W/Omega, u = nu (Z^T diag(W/Omega) nu).
int launch_group_sums(Ctx* c, int mode) {
  if (c->n_grp == 0) return GPL_OK;
  if (mode == 0 || mode == 1) {
    ProfScope ps(c, "group_sums");
    {
      const int rc = dgen_group_sums(c, mode);
      if (rc != GPL_ERR_ARG) return rc;
    }
    const int J = mode == 1 ? 1 : c->J;
    dim3 g(div_up(J, TM), div_up(c->n_d, TN), c->n_grp);
    if (mode == 0)
      k_group_sums<0><<<g, 256, 0, c->stream>>>(c->N, c->ldN, J, c->n_d, c->n_grp, c->gcells_d, c->gstart_d, c->W,
                                                c->Omega, c->Dm, c->gsum);
    else
      k_group_sums<1><<<g, 256, 0, c->stream>>>(c->N, c->ldN, J, c->n_d, c->n_grp, c->gcells_d, c->gstart_d, c->W,
                                                c->Omega, c->Dm, c->gsum);
    GPL_LAUNCHED(c, "k_group_sums");
    return GPL_OK;
  }
  ProfScope pt(c, "group_t");
  dim3 g(c->n_grp, div_up(c->J, 8));
  if (mode == 2)
    k_group_t<2><<<g, 256, 0, c->stream>>>(c->ldN, c->J, c->n_grp, c->gcells_d, c->gstart_d, c->Wg, c->Omega,
                                           c->scratch, c->gT);
  else if (mode == 4)  // u per cell, the same for every gene
    k_group_t<4><<<g, 256, 0, c->stream>>>(c->ldN, c->J, c->n_grp, c->gcells_d, c->gstart_d, c->Wg, c->Omega,
                                           c->zt_u_src, c->gT);
  else
    k_group_t<0><<<g, 256, 0, c->stream>>>(c->ldN, c->J, c->n_grp, c->gcells_d, c->gstart_d, c->Wg, c->Omega,
                                           c->zt_u_src ? c->zt_u_src : c->Nu, c->gT);
  GPL_LAUNCHED(c, "k_group_t");
  return GPL_OK;
}

// Categorical rows and columns of Psi_j (both triangles) from the group sums, plus the
// prior's diagonal on them; the dense x dense entries are written by the Gram kernel. Every
// categorical entry is written once, as a sum over the groups at its level(s) taken in group
// order (the order of getPsi's case analysis, ggplvm.cu:628-674, over the cells of each group):
//   (level l, dense column a)   sum_{g at l} S[g][a]
//   (level l, level l)          sum_{g at l} S[g][0] + DeltaInv (S[.][0]: the intercept = sum w)
//   (level l, other level of the same variable)   0
//   (level l of v, level l2 of v2 != v)           sum_{g at l and l2} S[g][0]
__global__ void __launch_bounds__(256) k_assemble_psi(int P, int n_d, int NL, int n_cv, int n_grp,
                                                      const int* __restrict__ dcol, const int* __restrict__ lvl_cc,
                                                      const int* __restrict__ lvl_v, const int* __restrict__ lvl_ptr,
                                                      const int* __restrict__ lvl_grp, const int* __restrict__ cv_nh,
                                                      const int* __restrict__ glev, const double* __restrict__ S,
                                                      const double* __restrict__ Dinv, double* __restrict__ Psi) {
  const int j = blockIdx.x;
  double* Pj = Psi + (size_t)j * P * P;
  const double* Sj = S + (size_t)j * n_grp * (n_d + 1);
  const int ld = n_d + 1;
  for (int e = threadIdx.x; e < NL * n_d; e += blockDim.x) {
    const int l = e / n_d, a = e - l * n_d;
    double s = 0.0;
    for (int q = lvl_ptr[l]; q < lvl_ptr[l + 1]; q++) s += Sj[(size_t)lvl_grp[q] * ld + a];
    const size_t cc = lvl_cc[l], dc = dcol[a];
    Pj[cc + dc * P] = s;
    Pj[dc + cc * P] = s;
  }
  for (int e = threadIdx.x; e < NL * NL; e += blockDim.x) {
    const int l1 = e / NL, l2 = e - l1 * NL;
    const int v1 = lvl_v[l1], v2 = lvl_v[l2];
    const size_t c1 = lvl_cc[l1], c2 = lvl_cc[l2];
    double s = 0.0;
    if (v1 == v2) {
      if (l1 == l2) {
        for (int q = lvl_ptr[l1]; q < lvl_ptr[l1 + 1]; q++) s += Sj[(size_t)lvl_grp[q] * ld];
        s += Dinv[c1 + c1 * P];
      }
    } else {
      const int L2 = (int)c2 - cv_nh[v2];
      for (int q = lvl_ptr[l1]; q < lvl_ptr[l1 + 1]; q++) {
        const int g = lvl_grp[q];
        if (glev[(size_t)g * n_cv + v2] == L2) s += Sj[(size_t)g * ld];
      }
    }
    Pj[c1 + c2 * P] = s;
  }
}

// dst[col * ldN + pos] = src[col * ldN + cell(pos)]: the cells in group order (gcells)
__global__ void k_group_order(int N, int ldN, int ncols, const int* __restrict__ gcells, const double* __restrict__ src,
                              double* __restrict__ dst) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= N) return;
  const int i = gcells[pos];
  for (int col = blockIdx.y; col < ncols; col += gridDim.y) dst[(size_t)col * ldN + pos] = src[(size_t)col * ldN + i];
}

int launch_group_order(Ctx* c, const double* src, int ncols, double* dst) {
  dim3 g(div_up(c->N, 256), std::min(ncols, 65535));
  k_group_order<<<g, 256, 0, c->stream>>>(c->N, c->ldN, ncols, c->gcells_d, src, dst);
  GPL_LAUNCHED(c, "k_group_order");
  return GPL_OK;
}

int launch_assemble_psi(Ctx* c, int J) {
  if (c->n_grp == 0) return GPL_OK;
  ProfScope ps(c, "assemble_psi");
  k_assemble_psi<<<J, 256, 0, c->stream>>>(c->P, c->n_d, c->n_lvl, c->n_cv, c->n_grp, c->dcol_d, c->lvl_cc_d,
                                           c->lvl_v_d, c->lvl_ptr_d, c->lvl_grp_d, c->cv_nh_d, c->glev_d, c->gsum,
                                           c->DeltaInv, c->Psi);
  GPL_LAUNCHED(c, "k_assemble_psi");
  return GPL_OK;
}

// Categorical entries of bvec (P x J): sum over the groups at each level of T[j][g].
__global__ void k_assemble_b(int P, int J, int n_cv, int n_grp, const int* __restrict__ cv_nh,
                             const int* __restrict__ cv_nlev, const int* __restrict__ glev,
                             const double* __restrict__ T, double* __restrict__ b) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= J) return;
  double* bj = b + (size_t)j * P;
  for (int v = 0; v < n_cv; v++)
    for (int L = 0; L < cv_nlev[v]; L++) bj[cv_nh[v] + L] = 0.0;
  for (int g = 0; g < n_grp; g++) {
    const double t = T[(size_t)j * n_grp + g];
    for (int v = 0; v < n_cv; v++) bj[cv_nh[v] + glev[g * n_cv + v]] += t;
  }
}

int launch_assemble_b(Ctx* c, double* out) {
  if (c->n_grp == 0) return GPL_OK;
  ProfScope ps(c, "assemble_b");
  k_assemble_b<<<div_up(c->J, 128), 128, 0, c->stream>>>(c->P, c->J, c->n_cv, c->n_grp, c->cv_nh_d, c->cv_nlev_d,
                                                         c->glev_d, c->gT, out);
  GPL_LAUNCHED(c, "k_assemble_b");
  return GPL_OK;
}

// h and kappa per (gene, group) from Psi_j^{-1}
__global__ void k_group_tables(int P, int n_d, int n_cv, int n_grp, const int* __restrict__ dcol,
                               const int* __restrict__ cv_nh, const int* __restrict__ glev,
                               const double* __restrict__ S, double* __restrict__ tab) {
  const int j = blockIdx.x;
  const double* Sj = S + (size_t)j * P * P;
  const int ld = n_d + 1;
  double* tj = tab + (size_t)j * n_grp * ld;
  for (int e = threadIdx.x; e < n_grp * ld; e += blockDim.x) {
    const int g = e / ld, a = e % ld;
    const int* lv = glev + g * n_cv;
    double s = 0.0;
    if (a < n_d) {
      const size_t r = dcol[a];
      for (int v = 0; v < n_cv; v++) s += Sj[r + (size_t)(cv_nh[v] + lv[v]) * P];
    } else {
      for (int v = 0; v < n_cv; v++)
        for (int v2 = 0; v2 < n_cv; v2++) s += Sj[(cv_nh[v] + lv[v]) + (size_t)(cv_nh[v2] + lv[v2]) * P];
    }
    tj[e] = s;
  }
}

int launch_group_tables(Ctx* c) {
  if (c->n_grp == 0) return GPL_OK;
  ProfScope ps(c, "group_tables");
  k_group_tables<<<c->J, 256, 0, c->stream>>>(c->P, c->n_d, c->n_cv, c->n_grp, c->dcol_d, c->cv_nh_d, c->glev_d,
                                              c->PsiInv, c->gsum);
  GPL_LAUNCHED(c, "k_group_tables");
  return GPL_OK;
}

// HK[i, a] = sum_j O_ij tab[j][g(i)][a] over the gathered cells of each group (a <= n_d)
__global__ void __launch_bounds__(256) k_hk(int ldN, int J, int n_d, int n_grp, const int2* __restrict__ tiles,
                                            const int* __restrict__ gcells, const int* __restrict__ gstart,
                                            const double* __restrict__ W, const double* __restrict__ Omega,
                                            const double* __restrict__ tab, double* __restrict__ HK) {
  __shared__ double As[TK][TM + 1];
  __shared__ double Bs[TK][TN + 1];
  __shared__ int cells[TM];
  const int2 t2 = tiles[blockIdx.x];
  const int g = t2.x, r0 = t2.y;
  const int a0 = blockIdx.y * TN;
  const int c0 = gstart[g], nc = gstart[g + 1] - c0;
  const int ld = n_d + 1;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  if (tid < TM) cells[tid] = (r0 + tid < nc) ? gcells[c0 + r0 + tid] : -1;
  __syncthreads();
  double acc[4][4];
#pragma unroll
  for (int x = 0; x < 4; x++)
#pragma unroll
    for (int y = 0; y < 4; y++) acc[x][y] = 0.0;
  for (int k0 = 0; k0 < J; k0 += TK) {
#pragma unroll
    for (int t = 0; t < (TM * TK) / 256; t++) {
      const int e = tid + t * 256;
      const int r = e % TM, k = e / TM;
      const int i = cells[r], j = k0 + k;
      As[k][r] = (i >= 0 && j < J) ? W[(size_t)j * ldN + i] / Omega[i] : 0.0;
    }
#pragma unroll
    for (int t = 0; t < (TN * TK) / 256; t++) {
      const int e = tid + t * 256;
      const int cc = e % TN, k = e / TN;
      const int a = a0 + cc, j = k0 + k;
      Bs[k][cc] = (a < ld && j < J) ? tab[((size_t)j * n_grp + g) * ld + a] : 0.0;
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
#pragma unroll
  for (int x = 0; x < 4; x++) {
    const int i = cells[tx + 16 * x];
    if (i < 0) continue;
#pragma unroll
    for (int y = 0; y < 4; y++) {
      const int a = a0 + ty + 16 * y;
      if (a < ld) HK[i + (size_t)a * ldN] = acc[x][y];
    }
  }
}

int launch_hk(Ctx* c) {
  if (c->n_grp == 0) return GPL_OK;
  ProfScope ps(c, "hk");
  {
    const int rc = dgen_hk(c);
    if (rc != GPL_ERR_ARG) return rc;
  }
  dim3 g(c->n_hk_tiles, div_up(c->n_d + 1, TN));
  k_hk<<<g, 256, 0, c->stream>>>(c->ldN, c->J, c->n_d, c->n_grp, c->hk_tiles_d, c->gcells_d, c->gstart_d, c->W,
                                 c->Omega, c->gsum, c->HK);
  GPL_LAUNCHED(c, "k_hk");
  return GPL_OK;
}

}  // namespace gpl
