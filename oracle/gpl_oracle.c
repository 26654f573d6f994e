/*
 * gpl_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle; see gpl_oracle.h).
 *
 * Double-precision CPU restatement of the reference fit, function by function, in the
 * reference's buffer layouts and arithmetic order, parallelised over genes or cells
 * with OpenMP (every parallel loop writes disjoint outputs, so results do not depend
 * on the thread count). Citations are to the reference sources (src/ of GASPACHO2).
 *
 * Constants of the reference driver (ggplvm.cu:20-22): wt = 0.1 (Titsias weight),
 * igap1 = igb = 100 (inverse-gamma prior on Omega).
 */
#include "gpl_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const double WT = 0.1, IGAP1 = 100.0, IGB = 100.0;

struct orc_ctx {
  int N, J, M, Q, P, p;
  int gpv; /* 1 when the design carries the GP variable (M > 0); 0 for the DE null model */
  long L;
  int *ci, *gp;
  double *cx;
  int *vc, *vv, *nh, *mc, *mv, *mk;
  double **numcol; /* per model column: numeric data (intercept -> ones, GP -> Knm column) */
  int **catcol;    /* per model column: categorical level codes */
  double *varnum;  /* per variable: base pointer of numeric data (NULL for categorical) */
  double **varbase;
  int **varcat;
  double *ones, *numbody;
  int *catbody;
  double *Knm;
  double *Omega, *delta, *X, *T, *rho, *phi, *ls, *zeta;
  double *Kmm, *Kinv, *KinvKmn, *titsias, *DeltaInv;
  double *W, *Nu, *Psi, *PsiInv, *Beta, *tBeta, *lkhds, *lkhd;
  double *grad, *grad0, *SS, *XX, *ss, *gdtmp, *C1, *C2, *grtmp;
  long tot_max;
};

static void* xcalloc(size_t n, size_t s) { return calloc(n ? n : 1, s); }

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ---- dense helpers: chol.cu:7-97 -------------------------------------------------- */

/* getRb (chol.cu:7-17): b <- L^T b with L the lower factor stored in a (n x n, col-major). */
static void rb(const double* a, double* b, int n) {
  for (int j = 0; j < n; j++) {
    double t = 0.0;
    for (int i = j; i < n; i++) t += a[i + j * n] * b[i];
    b[j] = t;
  }
}

/* choldc (chol.cu:19-43): in-place Cholesky; reads the upper triangle, writes the lower
 * factor (diagonal included). A non-positive pivot zero-fills the whole matrix. */
static void choldc(double* a, int n) {
  for (int i = 0; i < n; i++) {
    for (int j = i; j < n; j++) {
      double sum = a[i + j * n];
      for (int k = i - 1; k >= 0; k--) sum -= a[i + k * n] * a[j + k * n];
      if (i == j) {
        if (sum <= 0.0) {
          memset(a, 0, sizeof(double) * (size_t)n * n);
          return;
        }
        a[j + i * n] = sqrt(sum);
      } else {
        a[j + i * n] = sum / a[i + i * n];
      }
    }
  }
}

/* cholslg (chol.cu:86-97): x = (L L^T)^{-1} b with strided b and x. */
static void cholslg(const double* a, int n, const double* b, int ldb, double* x, int ldx) {
  for (int i = 0; i < n; i++) {
    double sum = b[i * ldb];
    for (int k = i - 1; k >= 0; k--) sum -= a[i + k * n] * x[k * ldx];
    x[i * ldx] = sum / a[i + i * n];
  }
  for (int i = n - 1; i >= 0; i--) {
    double sum = x[i * ldx];
    for (int k = i + 1; k < n; k++) sum -= a[k + i * n] * x[k * ldx];
    x[i * ldx] = sum / a[i + i * n];
  }
}

static void cholsl(const double* a, int n, const double* b, double* x) { cholslg(a, n, b, 1, x, 1); }

/* quadform (util_cuda.cu:442-451): b^T A b with A upper-stored symmetric. */
static double quadform(const double* A, const double* b, int n) {
  double s = 0.0;
  for (int i = 0; i < n; i++) {
    s += A[i + i * n] * b[i] * b[i];
    for (int j = i + 1; j < n; j++) s += 2.0 * A[i + j * n] * b[i] * b[j];
  }
  return s;
}

/* mscale_d (util_cuda.cu:546-555) */
static void mscale(int Q, double* r, double m) {
  double mh = 0.0;
  for (int i = 0; i < Q; i++) mh += r[i];
  mh /= (double)Q;
  for (int i = 0; i < Q; i++) r[i] *= m / mh;
}

/* getModelMatrix (DataFrame.cu:72-82) */
static inline double zval(const orc_ctx* o, int i, int k) {
  if (o->mc[k] == 1) return o->numcol[k][i];
  return o->catcol[k][i] == o->mv[k] ? 1.0 : 0.0;
}

/* ---- construction: SparseMat.cu:37-52, DataFrame.cu:88-149, init.cu:27-48 --------- */

orc_ctx* orc_create(int N, int J, long nnz, const int* cell_idx, const int* gene_ptr, const double* counts,
                    int n_var, const int* c, const int* v, const void* body, long body_bytes, int M, int Q,
                    const double* ls, const double* X0) {
  if (N <= 0 || J <= 0 || M < 0 || Q <= 0 || n_var < 0 || nnz < 0) return NULL;
  orc_ctx* o = (orc_ctx*)xcalloc(1, sizeof(orc_ctx));
  o->N = N; o->J = J; o->M = M; o->Q = Q; o->L = nnz;
  o->ci = (int*)xcalloc(nnz, sizeof(int));
  o->gp = (int*)xcalloc(J + 1, sizeof(int));
  o->cx = (double*)xcalloc(nnz, sizeof(double));
  memcpy(o->ci, cell_idx, sizeof(int) * nnz);
  memcpy(o->gp, gene_ptr, sizeof(int) * (J + 1));
  memcpy(o->cx, counts, sizeof(double) * nnz);

  /* loadDataFrame (DataFrame.cu:56-75): intercept, the file's variables, then Knm when M > 0 */
  o->gpv = M > 0 ? 1 : 0;
  const int p = n_var + 1 + o->gpv;
  o->p = p;
  o->vc = (int*)xcalloc(p, sizeof(int));
  o->vv = (int*)xcalloc(p, sizeof(int));
  o->nh = (int*)xcalloc(p + 1, sizeof(int));
  o->vc[0] = 1; o->vv[0] = 1;
  for (int k = 0; k < n_var; k++) { o->vc[k + 1] = c[k]; o->vv[k + 1] = v[k]; }
  if (o->gpv) { o->vc[p - 1] = 1; o->vv[p - 1] = M; }
  long need = 0;
  for (int j = 0; j < p; j++) o->nh[j + 1] = o->nh[j] + o->vv[j] * o->vc[j];
  for (int k = 0; k < n_var; k++) need += (long)N * v[k] * (c[k] == 1 ? 8 : 4);
  if (need != body_bytes) { orc_destroy(o); return NULL; }
  const int P = o->nh[p];
  o->P = P;
  o->mc = (int*)xcalloc(P, sizeof(int));
  o->mv = (int*)xcalloc(P, sizeof(int));
  o->mk = (int*)xcalloc(P, sizeof(int));
  o->numcol = (double**)xcalloc(P, sizeof(double*));
  o->catcol = (int**)xcalloc(P, sizeof(int*));
  o->varbase = (double**)xcalloc(p, sizeof(double*));
  o->varcat = (int**)xcalloc(p, sizeof(int*));
  o->ones = (double*)xcalloc(N, sizeof(double));
  for (int i = 0; i < N; i++) o->ones[i] = 1.0;
  o->Knm = (double*)xcalloc((size_t)N * M, sizeof(double));
  /* copy the body (unaligned in the file: numeric blocks may follow int blocks) */
  const char* bp = (const char*)body;
  long off = 0;
  o->varbase[0] = o->ones;
  for (int j = 1; j <= n_var; j++) {
    long bytes = (long)N * o->vv[j] * (o->vc[j] == 1 ? 8 : 4);
    if (o->vc[j] == 1) {
      double* d = (double*)xcalloc((size_t)N * o->vv[j], sizeof(double));
      memcpy(d, bp + off, bytes);
      o->varbase[j] = d;
    } else {
      int* d = (int*)xcalloc((size_t)N * o->vv[j], sizeof(int));
      memcpy(d, bp + off, bytes);
      o->varcat[j] = d;
    }
    off += bytes;
  }
  if (o->gpv) o->varbase[p - 1] = o->Knm;
  for (int j = 0; j < p; j++) {
    for (int k = o->nh[j]; k < o->nh[j + 1]; k++) {
      o->mc[k] = o->vc[j];
      o->mv[k] = k - o->nh[j];
      o->mk[k] = j;
      if (o->vc[j] == 1) o->numcol[k] = o->varbase[j] + (size_t)N * o->mv[k];
      else o->catcol[k] = o->varcat[j];
    }
  }
  /* loadDataFrame stores 99.0, and newDataFrameOnDevice 199.0, at the start of the last
   * variable's block (DataFrame.cu:112-113, 131): that is Knm's first entry when M > 0
   * (rewritten by getKernelMats) and the first cell of the last design variable when M = 0
   * (the DE driver's null model), kept here for a numeric variable. For a categorical one the
   * double's bytes replace two level codes, which the reference then reads out of range; the
   * codes are left as loaded. */
  if (!o->gpv && o->vc[p - 1] == 1) o->varbase[p - 1][0] = 199.0;
  /* level codes must index an existing column (the reference does not check) */
  for (int j = 1; j <= n_var; j++)
    if (o->vc[j] != 1)
      for (int i = 0; i < N; i++)
        if (o->varcat[j][i] < 0 || o->varcat[j][i] >= o->vc[j] * o->vv[j]) { orc_destroy(o); return NULL; }

  o->Omega = (double*)xcalloc(2 * (size_t)N, sizeof(double));
  o->delta = (double*)xcalloc(2 * (size_t)p, sizeof(double));
  o->X = (double*)xcalloc(2 * (size_t)N * Q, sizeof(double));
  o->T = (double*)xcalloc(2 * (size_t)M * Q, sizeof(double));
  o->rho = (double*)xcalloc(2 * (size_t)Q, sizeof(double));
  o->phi = (double*)xcalloc(J, sizeof(double));
  o->ls = (double*)xcalloc(N, sizeof(double));
  o->zeta = (double*)xcalloc(P, sizeof(double));
  memcpy(o->ls, ls, sizeof(double) * N);
  memcpy(o->X, X0, sizeof(double) * (size_t)N * Q);
  for (int i = 0; i < M; i++) o->T[i] = ((double)(i + 1) / (double)(M + 1)) * 2.0 * 3.14159265358979;
  o->Kmm = (double*)xcalloc((size_t)M * M, sizeof(double));
  o->Kinv = (double*)xcalloc((size_t)M * M, sizeof(double));
  o->KinvKmn = (double*)xcalloc((size_t)M * N, sizeof(double));
  o->titsias = (double*)xcalloc(N, sizeof(double));
  o->DeltaInv = (double*)xcalloc((size_t)P * P, sizeof(double));
  o->W = (double*)xcalloc((size_t)N * (J + 1), sizeof(double));
  o->Nu = (double*)xcalloc((size_t)N * J, sizeof(double));
  o->Psi = (double*)xcalloc((size_t)J * P * P, sizeof(double));
  o->PsiInv = (double*)xcalloc((size_t)J * P * P, sizeof(double));
  o->Beta = (double*)xcalloc((size_t)P * J, sizeof(double));
  o->tBeta = (double*)xcalloc((size_t)P * J, sizeof(double));
  o->lkhds = (double*)xcalloc(J, sizeof(double));
  o->lkhd = (double*)xcalloc(50000, sizeof(double));
  o->tot_max = (long)N + p + (long)N * Q + (long)M * Q + Q;
  o->grad = (double*)xcalloc(o->tot_max, sizeof(double));
  o->grad0 = (double*)xcalloc(o->tot_max, sizeof(double));
  o->ss = (double*)xcalloc(o->tot_max, sizeof(double));
  o->SS = (double*)xcalloc(o->tot_max * 10, sizeof(double));
  o->XX = (double*)xcalloc(o->tot_max * 10, sizeof(double));
  o->gdtmp = (double*)xcalloc((size_t)P * J, sizeof(double));
  o->C1 = (double*)xcalloc((size_t)N * M, sizeof(double));
  o->C2 = (double*)xcalloc((size_t)M * M, sizeof(double));
  o->grtmp = (double*)xcalloc((size_t)M * Q, sizeof(double));
  orc_init_params(o);
  return o;
}

void orc_destroy(orc_ctx* o) {
  if (!o) return;
  const int nv_end = o->p - o->gpv; /* the file's variables are 1 .. nv_end - 1 */
  if (o->varbase)
    for (int j = 1; j < nv_end; j++) free(o->varbase[j]);
  if (o->varcat)
    for (int j = 1; j < nv_end; j++) free(o->varcat[j]);
  void* bufs[] = {o->ci, o->gp, o->cx, o->vc, o->vv, o->nh, o->mc, o->mv, o->mk, o->numcol, o->catcol,
                  o->varbase, o->varcat, o->ones, o->Knm, o->Omega, o->delta, o->X, o->T, o->rho, o->phi,
                  o->ls, o->zeta, o->Kmm, o->Kinv, o->KinvKmn, o->titsias, o->DeltaInv, o->W, o->Nu, o->Psi,
                  o->PsiInv, o->Beta, o->tBeta, o->lkhds, o->lkhd, o->grad, o->grad0, o->ss, o->SS, o->XX,
                  o->gdtmp, o->C1, o->C2, o->grtmp};
  for (size_t k = 0; k < sizeof(bufs) / sizeof(bufs[0]); k++) free(bufs[k]);
  free(o);
}

void orc_dims(const orc_ctx* o, int* d) {
  d[0] = o->N; d[1] = o->J; d[2] = o->M; d[3] = o->P; d[4] = o->p; d[5] = o->Q;
}

/* initParams (init.cu:27-48) */
void orc_init_params(orc_ctx* o) {
  const int p = o->p;
  o->delta[0] = 1.5;
  for (int i = 1; i < p - 1; i++) o->delta[i] = 0.01;
  o->delta[p - 1] = o->gpv ? 0.3 : 0.01;
  for (int i = 0; i < o->N; i++) o->Omega[i] = 1.0;
  for (int j = 0; j < o->J; j++) o->phi[j] = 1.0;
  o->rho[0] = 5.0;
  for (int k = 1; k < o->Q; k++) o->rho[k] = 10.0;
}

/* readParams (util_cuda.cu:520-544), from memory; NULL keeps a block. */
void orc_set_params(orc_ctx* o, const double* Omega, const double* delta, const double* X, const double* T,
                    const double* rho, const double* phi) {
  if (Omega) memcpy(o->Omega, Omega, sizeof(double) * o->N);
  if (delta) memcpy(o->delta, delta, sizeof(double) * o->p);
  if (X) memcpy(o->X, X, sizeof(double) * (size_t)o->N * o->Q);
  if (T) memcpy(o->T, T, sizeof(double) * (size_t)o->M * o->Q);
  if (rho) memcpy(o->rho, rho, sizeof(double) * o->Q);
  if (phi) memcpy(o->phi, phi, sizeof(double) * o->J);
}

void orc_set_beta(orc_ctx* o, const double* beta) { memcpy(o->Beta, beta, sizeof(double) * (size_t)o->P * o->J); }

/* ---- kernel matrices: kernel_funcs.cu:61-97, 101-135, 139-162 ---------------------- */

/* Squared distance term of one cell/inducing pair (or inducing/inducing pair): all latent
 * dimensions (getKernelMatsWithPer, kernel_funcs.cu:61-97: periodic dim 0, ARD dims >= 1)
 * when lv < 0, dimension lv alone otherwise (getKernelMatsWithPerSpecificLV,
 * kernel_funcs.cu:101-135). a and b index the two point sets with leading sizes na, nb. */
static double kern_sum(const double* A, int na, int a, const double* B, int nb, int b, const double* rho, int Q,
                       int lv) {
  double sum = 0.0, t;
  if (lv <= 0) {
    t = sin((A[a] - B[b]) / 2.0);
    sum += t * t / rho[0];
  }
  for (int k = 1; k < Q; k++) {
    if (lv >= 0 && k != lv) continue;
    t = A[a + (size_t)k * na] - B[b + (size_t)k * nb];
    sum += t * t / 2.0 / rho[k];
  }
  return sum;
}

static void kernel_mats_lv(orc_ctx* o, int lv) {
  const int N = o->N, M = o->M, Q = o->Q;
  const double *X = o->X, *T = o->T, *rho = o->rho;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < M; j++)
    for (int i = 0; i < N; i++) o->Knm[i + (size_t)j * N] = exp(-kern_sum(X, N, i, T, M, j, rho, Q, lv));
  for (int j = 0; j < M; j++) {
    for (int ii = 0; ii < M; ii++) {
      double val;
      if (ii == j) val = 1.0;
      else if (ii > j) val = 0.0;
      else val = exp(-kern_sum(T, M, ii, T, M, j, rho, Q, lv));
      o->Kmm[ii + j * M] = val;
      o->Kinv[ii + j * M] = val;
    }
  }
  /* cholKmm (kernel_funcs.cu:139-143) */
  choldc(o->Kinv, M);
  /* getKinvKmn (kernel_funcs.cu:154-162): Kmm^{-1} k_n and the Titsias residual */
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    double* x = o->KinvKmn + (size_t)i * M;
    cholslg(o->Kinv, M, o->Knm + i, N, x, 1);
    double d = 0.0;
    for (int k = 0; k < M; k++) d += o->Knm[i + (size_t)k * N] * x[k];
    o->titsias[i] = (1.0 - d) / 2.0;
  }
}

void orc_kernel_mats(orc_ctx* o) { kernel_mats_lv(o, -1); }

/* getKernelMats(..., q, ...) (kernel_funcs.cu:17-19): the GP over latent dimension q alone,
 * then cholKmm and getKinvKmn as for the full kernel (ggplvm_de.cu:1129-1133). */
void orc_kernel_mats_lv(orc_ctx* o, int q) { kernel_mats_lv(o, q < 0 ? -1 : q); }

/* expandDelta_k (util_cuda.cu:249-269): prior precision blockdiag(1/delta_k I, Kmm/delta_GP), upper. */
void orc_expand_delta(orc_ctx* o) {
  const int p = o->p, P = o->P, M = o->M;
  memset(o->DeltaInv, 0, sizeof(double) * (size_t)P * P);
  if (!o->gpv) { /* expandDeltaWOK_k (util_cuda.cu:235-246): no GP block */
    for (int i = 0; i < p; i++)
      for (int j = o->nh[i]; j < o->nh[i + 1]; j++) o->DeltaInv[j + j * P] = 1.0 / o->delta[i];
    return;
  }
  for (int i = 0; i < p - 1; i++)
    for (int j = o->nh[i]; j < o->nh[i + 1]; j++) o->DeltaInv[j + j * P] = 1.0 / o->delta[i];
  for (int j = 0; j < M; j++) {
    int jj = j + o->nh[p - 1];
    for (int k = j; k < M; k++) {
      int kk = k + o->nh[p - 1];
      o->DeltaInv[jj + kk * P] = o->Kmm[j + k * M] / o->delta[p - 1];
    }
  }
}

/* ---- GLM initialisation: init.cu:125-221, ggplvm.cu:1134-1137 --------------------- */

/* Upper-triangle sum over cells of z_k z_l w_i (getPsi's case analysis, ggplvm.cu:628-674;
 * initPsi, init.cu:130-176, is the same with w == 1). */
static double gram_entry(const orc_ctx* o, int k, int l, const double* w, const double* Omega) {
  const int N = o->N;
  double sum = 0.0;
#define WEIGHT(i) (Omega ? w[i] / Omega[i] : 1.0)
  if (o->mc[k] == 1) {
    const double* pd1 = o->numcol[k];
    if (o->mc[l] == 1) {
      const double* pd2 = o->numcol[l];
      if (Omega) for (int i = 0; i < N; i++) sum += pd1[i] * pd2[i] * w[i] / Omega[i];
      else for (int i = 0; i < N; i++) sum += pd1[i] * pd2[i];
    } else {
      const int* pi2 = o->catcol[l];
      int mvl = o->mv[l];
      if (Omega) { for (int i = 0; i < N; i++) if (pi2[i] == mvl) sum += pd1[i] * w[i] / Omega[i]; }
      else { for (int i = 0; i < N; i++) if (pi2[i] == mvl) sum += pd1[i]; }
    }
  } else {
    const int* pi1 = o->catcol[k];
    int mvk = o->mv[k];
    if (o->mc[l] == 1) {
      const double* pd2 = o->numcol[l];
      if (Omega) { for (int i = 0; i < N; i++) if (pi1[i] == mvk) sum += pd2[i] * w[i] / Omega[i]; }
      else { for (int i = 0; i < N; i++) if (pi1[i] == mvk) sum += pd2[i]; }
    } else {
      const int* pi2 = o->catcol[l];
      int mvl = o->mv[l];
      if (o->mk[k] == o->mk[l]) {
        if (k == l)
          for (int i = 0; i < N; i++)
            if (pi1[i] == mvk) sum += WEIGHT(i);
      } else {
        for (int i = 0; i < N; i++)
          if (pi1[i] == mvk && pi2[i] == mvl) sum += WEIGHT(i);
      }
    }
  }
#undef WEIGHT
  return sum;
}

void orc_glm_init(orc_ctx* o) {
  const int N = o->N, J = o->J, P = o->P;
  orc_expand_delta(o);
  double* Psi0 = o->Psi; /* initPsi writes the first P x P slot (init.cu:125-181) */
#pragma omp parallel for schedule(dynamic, 1)
  for (int l = 0; l < P; l++)
    for (int k = 0; k < P; k++)
      Psi0[k + l * P] = (k <= l) ? gram_entry(o, k, l, NULL, NULL) + o->DeltaInv[k + l * P] : 0.0;
  choldc(Psi0, P); /* initPsi2 (init.cu:185-191) */
  /* initBeta (init.cu:193-221): least squares on log((y + 0.05) / s) */
#pragma omp parallel
  {
    double* tmp = (double*)xcalloc(P, sizeof(double));
#pragma omp for schedule(dynamic, 4)
    for (int j = 0; j < J; j++) {
      memset(tmp, 0, sizeof(double) * P);
      int l = o->gp[j], lmax = o->gp[j + 1];
      for (int i = 0; i < N; i++) {
        double yi;
        if (l < lmax && o->ci[l] == i) { yi = log((o->cx[l] + 0.05) / o->ls[i]); l++; }
        else yi = log(0.05 / o->ls[i]);
        for (int m = 0; m < P; m++) tmp[m] += zval(o, i, m) * yi;
      }
      cholsl(Psi0, P, tmp, o->Beta + (size_t)j * P);
    }
    free(tmp);
  }
}

/* ---- IRLS: ggplvm.cu:418-514, 621-724, util_cuda.cu:462-487 ------------------------ */

/* getWForBeta (ggplvm.cu:468-514): W, working response nu; counts matched by the sorted
 * merge walk over the gene's CSR entries. */
static void w_nu(orc_ctx* o) {
  const int N = o->N, J = o->J, p = o->p, P = o->P;
#pragma omp parallel for schedule(dynamic, 4)
  for (int j = 0; j < J; j++) {
    const double* bj = o->Beta + (size_t)j * P;
    double* Wj = o->W + (size_t)j * N;
    double* nj = o->Nu + (size_t)j * N;
    int l = o->gp[j], lmax = o->gp[j + 1];
    for (int i = 0; i < N; i++) {
      double sum = 0.0, sum2 = 0.0;
      for (int k = 0; k < p; k++) {
        if (o->vc[k] == 1) {
          const double* pd = o->varbase[k];
          for (int m = 0; m < o->vv[k]; m++) {
            sum += pd[i + (size_t)m * N] * bj[o->nh[k] + m];
            sum2 += pd[i + (size_t)m * N] * (bj[o->nh[k] + m] - o->zeta[o->nh[k] + m]);
          }
        } else {
          int lev = o->varcat[k][i];
          sum += bj[o->nh[k] + lev];
          sum2 += (bj[o->nh[k] + lev] - o->zeta[o->nh[k] + lev]);
        }
      }
      double logW = sum + log(o->ls[i]) + o->delta[p - 1] * o->titsias[i] * WT;
      Wj[i] = exp(sum) * o->ls[i] * exp(o->delta[p - 1] * o->titsias[i] * WT);
      if (l < lmax && o->ci[l] == i) {
        nj[i] = sum2 + exp(log(o->cx[l]) - logW) - 1.0;
        l++;
      } else {
        nj[i] = sum2 - 1.0;
      }
    }
  }
}

/* getPsi (ggplvm.cu:621-680) + cholPsi (ggplvm.cu:683-692): per-gene Gram, then Cholesky. */
static void gram_chol(orc_ctx* o) {
  const int N = o->N, J = o->J, P = o->P;
#pragma omp parallel for schedule(dynamic, 1)
  for (int j = 0; j < J; j++) {
    double* Pj = o->Psi + (size_t)j * P * P;
    const double* w = o->W + (size_t)j * N;
    for (int l = 0; l < P; l++)
      for (int k = 0; k < P; k++)
        Pj[k + l * P] = (k <= l) ? gram_entry(o, k, l, w, o->Omega) + o->DeltaInv[k + l * P] : 0.0;
    choldc(Pj, P);
  }
}

/* getZtOinvjnj (util_cuda.cu:462-487): Z^T diag(W_j / Omega) nu_j */
static void zt_oinv_nu(const orc_ctx* o, const double* Wj, const double* nj, double* b) {
  const int N = o->N, p = o->p;
  memset(b, 0, sizeof(double) * o->P);
  for (int k = 0; k < p; k++) {
    if (o->vc[k] == 1) {
      const double* pd = o->varbase[k];
      for (int m = 0; m < o->vv[k]; m++) {
        double sum = 0.0;
        for (int i = 0; i < N; i++) sum += pd[i + (size_t)m * N] * Wj[i] / o->Omega[i] * nj[i];
        b[o->nh[k] + m] = sum;
      }
    } else {
      const int* pi = o->varcat[k];
      for (int i = 0; i < N; i++) b[o->nh[k] + pi[i]] += Wj[i] / o->Omega[i] * nj[i];
    }
  }
}

/* getBetaPhi (ggplvm.cu:418-464): damped beta update and dispersion with its clamps. */
static void beta_phi(orc_ctx* o, int jtr) {
  const int N = o->N, J = o->J, P = o->P;
  double r = (double)(jtr + 1) / 100.0;
  if (jtr > 100) r = 1.0;
#pragma omp parallel
  {
    double* b = (double*)xcalloc(P, sizeof(double));
    double* tmp = (double*)xcalloc(P, sizeof(double));
#pragma omp for schedule(dynamic, 4)
    for (int j = 0; j < J; j++) {
      const double* Wj = o->W + (size_t)j * N;
      const double* nj = o->Nu + (size_t)j * N;
      const double* Pj = o->Psi + (size_t)j * P * P;
      double* bj = o->Beta + (size_t)j * P;
      double phij = 0.0;
      zt_oinv_nu(o, Wj, nj, b);
      for (int i = 0; i < N; i++) phij += nj[i] * nj[i] * Wj[i] / o->Omega[i];
      cholsl(Pj, P, b, tmp);
      for (int k = 0; k < P; k++) {
        bj[k] = bj[k] * (1 - r) + tmp[k] * r;
        tmp[k] = bj[k];
        bj[k] += o->zeta[k];
      }
      rb(Pj, tmp, P);
      for (int k = 0; k < P; k++) phij -= tmp[k] * tmp[k];
      double ph = phij / (double)N;
      if (isnan(ph)) ph = 1.0;
      if (ph < 0.0) ph = 1.0;
      if (ph < 0.01) ph = 0.01;
      if (ph > 1000.0) ph = 1000.0;
      o->phi[j] = ph;
    }
    free(b);
    free(tmp);
  }
}

/* getLkhdPois (ggplvm.cu:703-724) */
static void lkhd_pois(orc_ctx* o) {
  const int N = o->N, J = o->J, p = o->p;
#pragma omp parallel for schedule(dynamic, 4)
  for (int j = 0; j < J; j++) {
    const double* Wj = o->W + (size_t)j * N;
    int l = o->gp[j], lmax = o->gp[j + 1];
    double sum = 0.0;
    for (int i = 0; i < N; i++) {
      if (l < lmax && o->ci[l] == i) {
        sum += (log(Wj[i]) - o->delta[p - 1] * o->titsias[i] * WT) * o->cx[l] - Wj[i];
        l++;
      } else {
        sum -= Wj[i];
      }
    }
    o->lkhds[j] = sum;
  }
}

/* collectLkhd (ggplvm.cu:788-815) with the cell count argument n (0 during IRLS). */
static double collect_lkhd(orc_ctx* o, int n, int slot) {
  const int J = o->J, p = o->p;
  const double* Oinvt = o->W + (size_t)n * J;
  double sum = 0.0;
  for (int k = 0; k < J; k++) sum += o->lkhds[k];
  for (int i = 0; i < n; i++) sum -= WT * o->delta[p - 1] * Oinvt[i] * o->titsias[i];
  for (int i = 0; i < n; i++) sum = sum - IGB / o->Omega[i] - IGAP1 * log(o->Omega[i]);
  o->lkhd[slot] = sum;
  return sum;
}

double orc_irls_sweep(orc_ctx* o, int jtr) {
  w_nu(o);
  gram_chol(o);
  beta_phi(o, jtr);
  lkhd_pois(o);
  return collect_lkhd(o, 0, jtr);
}

/* IRLS loop with the driver's stopping rule (ggplvm.cu:1152-1189); -1 on a NaN likelihood. */
int orc_irls(orc_ctx* o, int jtr_max) {
  int jtr;
  for (jtr = 0; jtr < jtr_max; jtr++) {
    orc_irls_sweep(o, jtr);
    if (jtr > 0) {
      if (isnan(o->lkhd[jtr])) return -1;
      if (jtr == jtr_max - 1 || fabs(o->lkhd[jtr - 1] - o->lkhd[jtr]) / fabs(o->lkhd[jtr]) < 1e-7) {
        jtr++;
        break;
      }
    }
  }
  return jtr;
}

/* ---- objective: ggplvm.cu:284-294, 695-700, 744-784 ------------------------------- */

static void oinvt(orc_ctx* o) {
  const int N = o->N, J = o->J;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    double s = 0.0;
    for (int j = 0; j < J; j++) s += o->W[i + (size_t)j * N] / o->Omega[i];
    o->W[(size_t)N * J + i] = s;
  }
}

/* getLkhd / getLkhdj (ggplvm.cu:744-784): per-gene Laplace/PQL marginal. */
static void lkhd_genes(orc_ctx* o) {
  const int N = o->N, J = o->J, P = o->P;
#pragma omp parallel
  {
    double* tmp = (double*)xcalloc(P, sizeof(double));
    double* tmp2 = (double*)xcalloc(P, sizeof(double));
#pragma omp for schedule(dynamic, 4)
    for (int j = 0; j < J; j++) {
      const double* Wj = o->W + (size_t)j * N;
      const double* nj = o->Nu + (size_t)j * N;
      const double* Pj = o->Psi + (size_t)j * P * P;
      double phij = o->phi[j];
      double l = -((double)N) / 2.0 * log(phij);
      for (int i = 0; i < N; i++) l -= log(o->Omega[i] / Wj[i]) / 2.0;
      for (int k = 0; k < P; k++) {
        l -= log(Pj[k + k * P]);
        l += log(o->DeltaInv[k + k * P]);
      }
      zt_oinv_nu(o, Wj, nj, tmp);
      for (int i = 0; i < N; i++) {
        double oij = Wj[i] / o->Omega[i];
        l -= nj[i] * nj[i] * oij / 2.0 / phij;
      }
      cholsl(Pj, P, tmp, tmp2);
      for (int k = 0; k < P; k++) {
        l += tmp[k] * tmp2[k] / 2.0 / phij;
        if (isnan(l)) break;
      }
      o->lkhds[j] = l;
    }
    free(tmp);
    free(tmp2);
  }
}

/* ggplvm.cu:1205-1211 */
double orc_objective_after_irls(orc_ctx* o) {
  oinvt(o);
  choldc(o->DeltaInv, o->P);
  lkhd_genes(o);
  return collect_lkhd(o, o->N, 0);
}

/* One line-search evaluation (ggplvm.cu:1258-1277). */
double orc_objective(orc_ctx* o, int slot) {
  oinvt(o);
  orc_kernel_mats(o);
  orc_expand_delta(o);
  gram_chol(o);
  choldc(o->DeltaInv, o->P);
  lkhd_genes(o);
  return collect_lkhd(o, o->N, slot);
}

/* ---- gradient: ggplvm.cu:46-281, 301-376, 406-414 --------------------------------- */

/* getTildeBeta (ggplvm.cu:406-414), getGradLogDelta (ggplvm.cu:210-253) and
 * collectGradLogDelta (ggplvm.cu:256-281) with Titsias weight wt: d/dlog delta into out[0..p). */
static void grad_log_delta(orc_ctx* o, double wt, double* out) {
  const int N = o->N, J = o->J, M = o->M, P = o->P, p = o->p;
  const int g0 = o->nh[p - 1];
  /* getTildeBeta (ggplvm.cu:406-414) */
#pragma omp parallel
  {
    double* b = (double*)xcalloc(P, sizeof(double));
#pragma omp for schedule(dynamic, 4)
    for (int j = 0; j < J; j++) {
      zt_oinv_nu(o, o->W + (size_t)j * N, o->Nu + (size_t)j * N, b);
      cholsl(o->Psi + (size_t)j * P * P, P, b, o->tBeta + (size_t)j * P);
    }
    free(b);
  }
  /* getGradLogDelta (ggplvm.cu:210-253) */
#pragma omp parallel
  {
    double* ek = (double*)xcalloc(P, sizeof(double));
    double* psijk = (double*)xcalloc(P, sizeof(double));
#pragma omp for schedule(dynamic, 1)
    for (int j = 0; j < J; j++) {
      const double* tbj = o->tBeta + (size_t)j * P;
      for (int k = 0; k < P; k++) {
        double dk = 0.0, sum = 0.0;
        for (int l = 0; l < p; l++)
          if (o->nh[l] <= k && k < o->nh[l + 1]) { dk = o->delta[l]; break; }
        memset(ek, 0, sizeof(double) * P);
        if (k < g0) ek[k] = 1.0;
        else {
          int kk = k - g0;
          for (int l = 0; l < kk; l++) ek[l + g0] = o->Kmm[l + kk * M];
          for (int l = kk; l < M; l++) ek[l + g0] = o->Kmm[kk + l * M];
        }
        memset(psijk, 0, sizeof(double) * P);
        cholsl(o->Psi + (size_t)j * P * P, P, ek, psijk);
        sum -= (dk - psijk[k]) / dk / dk / 2.0;
        if (k < g0) sum += tbj[k] * tbj[k] / dk / dk / o->phi[j] / 2.0;
        else if (k == g0) sum += quadform(o->Kmm, tbj + g0, M) / dk / dk / o->phi[j] / 2.0;
        o->gdtmp[k + (size_t)j * P] = sum * dk;
      }
    }
    free(ek);
    free(psijk);
  }
  /* collectGradLogDelta (ggplvm.cu:256-281) */
  {
    const double* Oinvt = o->W + (size_t)N * J;
    for (int l = 0; l < p; l++) {
      double sum = 0.0;
      for (int j = 0; j < J; j++)
        for (int k = o->nh[l]; k < o->nh[l + 1]; k++) sum += o->gdtmp[k + (size_t)j * P];
      if (l == p - 1)
        for (int i = 0; i < N; i++) sum -= wt * Oinvt[i] * o->titsias[i] * o->delta[p - 1];
      out[l] = sum;
    }
  }
}

void orc_gradient(orc_ctx* o, double* grad_out) {
  const int N = o->N, J = o->J, M = o->M, Q = o->Q, P = o->P, p = o->p;
  const int g0 = o->nh[p - 1];
  double* grad = o->grad;
  orc_expand_delta(o);
  oinvt(o);
  grad_log_delta(o, WT, grad + N);
  /* getGradLogOmega (ggplvm.cu:301-376): d/dlog Omega, adjoint C1, d/dX */
  {
    double* gO = grad;
    double* gX = grad + N + p;
#pragma omp parallel
    {
      double* zi = (double*)xcalloc(P, sizeof(double));
      double* pz = (double*)xcalloc(P, sizeof(double));
#pragma omp for schedule(dynamic, 8)
      for (int i = 0; i < N; i++) {
        double sum = 0.0, Oii = 0.0;
        for (int k = 0; k < P; k++) zi[k] = zval(o, i, k);
        double* ci = o->C1 + i;
        for (int k = 0; k < M; k++) ci[(size_t)k * N] = 0.0;
        for (int j = 0; j < J; j++) {
          const double* tbj = o->tBeta + (size_t)j * P;
          double Wij = o->W[i + (size_t)j * N];
          double Oij = Wij / o->Omega[i];
          Oii += Oij;
          cholsl(o->Psi + (size_t)j * P * P, P, zi, pz);
          double zt = 0.0, zp = 0.0;
          for (int k = 0; k < P; k++) zt += zi[k] * tbj[k];
          for (int k = 0; k < P; k++) zp += zi[k] * pz[k];
          double tn = Oij * o->Nu[i + (size_t)j * N] - Oij * zt;
          sum -= (1.0 / o->Omega[i] - zp / o->Omega[i] * Oij) / 2.0;
          sum += tn * tn / Wij / o->phi[j] / 2.0;
          for (int k = 0; k < M; k++) ci[(size_t)k * N] += (-pz[k + g0] * Oij + tn * tbj[k + g0] / o->phi[j]);
        }
        sum += WT * o->delta[p - 1] * Oii / o->Omega[i] * o->titsias[i];
        gO[i] = sum * o->Omega[i] + IGB / o->Omega[i] - IGAP1;
        o->W[(size_t)N * J + i] = Oii;
        for (int k = 0; k < M; k++) {
          ci[(size_t)k * N] += WT * o->delta[p - 1] * Oii * o->KinvKmn[k + (size_t)i * M];
          ci[(size_t)k * N] *= o->Knm[i + (size_t)k * N];
        }
        double ci1 = 0.0;
        gX[i] = 0.0;
        for (int k = 0; k < M; k++) {
          ci1 += ci[(size_t)k * N];
          double t = (o->X[i] - o->T[k]) / 2.0;
          gX[i] -= ci[(size_t)k * N] * sin(t) * cos(t) / o->rho[0];
        }
        for (int q = 1; q < Q; q++) {
          double d = 0.0;
          for (int k = 0; k < M; k++) d += ci[(size_t)k * N] * o->T[k + q * M];
          gX[i + (size_t)q * N] = (d - ci1 * o->X[i + (size_t)q * N]) / o->rho[q];
        }
      }
      free(zi);
      free(pz);
    }
  }
  /* solvePsi (ggplvm.cu:46-53): explicit Psi_j^{-1} */
#pragma omp parallel
  {
    double* e = (double*)xcalloc(P, sizeof(double));
#pragma omp for schedule(dynamic, 1)
    for (int j = 0; j < J; j++)
      for (int k = 0; k < P; k++) {
        memset(e, 0, sizeof(double) * P);
        e[k] = 1.0;
        cholsl(o->Psi + (size_t)j * P * P, P, e, o->PsiInv + (size_t)j * P * P + (size_t)k * P);
      }
    free(e);
  }
  /* getC2 (ggplvm.cu:57-100): M x M adjoint of Kmm */
  {
    const double* Oinvt = o->W + (size_t)N * J;
#pragma omp parallel
    {
      double* ev = (double*)xcalloc(M, sizeof(double));
      double* ev2 = (double*)xcalloc(M, sizeof(double));
#pragma omp for schedule(dynamic, 1)
      for (int k = 0; k < M; k++)
        for (int j = 0; j <= k; j++) {
          double sum = 0.0, c2;
          for (int i = 0; i < N; i++)
            sum += o->KinvKmn[j + (size_t)i * M] * o->KinvKmn[k + (size_t)i * M] * Oinvt[i];
          c2 = -WT * o->delta[p - 1] * sum / 2.0;
          sum = 0.0;
          for (int i = 0; i < J; i++)
            sum += o->tBeta[j + g0 + (size_t)i * P] * o->tBeta[k + g0 + (size_t)i * P] / o->phi[i];
          c2 -= sum / o->delta[p - 1] / 2.0;
          sum = 0.0;
          for (int i = 0; i < J; i++) sum += o->PsiInv[(size_t)i * P * P + (size_t)(k + g0) * P + (j + g0)];
          c2 -= sum / o->delta[p - 1] / 2.0;
          memset(ev, 0, sizeof(double) * M);
          ev[k] = 1.0;
          cholsl(o->Kinv, M, ev, ev2);
          c2 += ((double)J) * ev2[j] / 2.0;
          c2 *= o->Kmm[j + k * M];
          o->C2[j + k * M] = c2;
          if (j < k) o->C2[k + j * M] = c2;
        }
      free(ev);
      free(ev2);
    }
  }
  /* getGradTau (ggplvm.cu:103-145) */
  {
    double* gT = grad + N + p + (size_t)N * Q;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int m = 0; m < M; m++)
      for (int q = 0; q < Q; q++) {
        double sum = 0.0, cm1 = 0.0;
        if (q == 0) {
          for (int i = 0; i < N; i++) {
            double t = (o->X[i] - o->T[m]) / 2.0;
            sum += o->C1[i + (size_t)m * N] * sin(t) * cos(t);
          }
          gT[m] = sum / o->rho[0];
          sum = 0.0;
          for (int i = 0; i < M; i++) {
            double t = (o->T[i] - o->T[m]) / 2.0;
            sum += o->C2[m + i * M] * sin(t) * cos(t);
          }
          gT[m] += 2.0 * sum / o->rho[0];
        } else {
          for (int i = 0; i < N; i++) {
            sum += o->C1[i + (size_t)m * N] * o->X[i + (size_t)q * N];
            cm1 += o->C1[i + (size_t)m * N];
          }
          gT[m + q * M] = (sum - cm1 * o->T[m + q * M]) / o->rho[q];
          sum = 0.0;
          cm1 = 0.0;
          for (int i = 0; i < M; i++) {
            sum += o->C2[m + i * M] * o->T[i + q * M];
            cm1 += o->C2[m + i * M];
          }
          gT[m + q * M] += 2.0 * (sum - cm1 * o->T[m + q * M]) / o->rho[q];
        }
      }
  }
  /* getGradLogRho + collectGradLogRho (ggplvm.cu:148-205) */
  {
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int j = 0; j < M; j++)
      for (int q = 0; q < Q; q++) {
        double sum = 0.0, rq = o->rho[q];
        if (q == 0) {
          for (int i = 0; i < N; i++) {
            double t = sin((o->X[i + (size_t)q * N] - o->T[j + q * M]) / 2.0);
            sum += o->C1[i + (size_t)j * N] * t * t / rq / rq;
          }
          for (int i = 0; i < M; i++) {
            double t = sin((o->T[i + q * M] - o->T[j + q * M]) / 2.0);
            sum += o->C2[i + j * M] * t * t / rq / rq;
          }
        } else {
          for (int i = 0; i < N; i++) {
            double t = o->X[i + (size_t)q * N] - o->T[j + q * M];
            sum += o->C1[i + (size_t)j * N] * t * t / rq / rq / 2.0;
          }
          for (int i = 0; i < M; i++) {
            double t = o->T[i + q * M] - o->T[j + q * M];
            sum += o->C2[i + j * M] * t * t / rq / rq / 2.0;
          }
        }
        o->grtmp[q + j * Q] = sum * rq;
      }
    double* gr = grad + N + p + (size_t)N * Q + (size_t)M * Q;
    for (int q = 0; q < Q; q++) {
      double sum = 0.0;
      for (int k = 0; k < M; k++) sum += o->grtmp[q + k * Q];
      gr[q] = sum;
    }
  }
  if (grad_out) memcpy(grad_out, grad, sizeof(double) * o->tot_max);
}

/* ---- L-BFGS: ggplvm.cu:818-934, util_cuda.cu:187-232 ------------------------------ */

/* lbfgs (util_cuda.cu:187-232): two-loop recursion over the last min(itr, 10) pairs,
 * gamma = s^T y / y^T y, direction clipped to [-1, 1] and negated. */
static void lbfgs_dir(const double* S, const double* Y, const double* g, long n, int m, int itr, double* z) {
  int pt = (itr - 1) % m;
  double* q = (double*)xcalloc(n, sizeof(double));
  double a[64];
  memcpy(q, g, sizeof(double) * n);
  int lo = itr > m ? pt - m + 1 : 0;
  for (int i = pt; i >= lo; i--) {
    int ii = (i + m) % m;
    double num = 0.0, den = 0.0;
    for (long k = 0; k < n; k++) {
      num += S[k + ii * n] * q[k];
      den += S[k + ii * n] * Y[k + ii * n];
    }
    a[ii] = num / den;
    for (long k = 0; k < n; k++) q[k] -= a[ii] * Y[k + ii * n];
  }
  double num = 0.0, den = 0.0;
  for (long k = 0; k < n; k++) {
    num += S[k + pt * n] * Y[k + pt * n];
    den += Y[k + pt * n] * Y[k + pt * n];
  }
  for (long k = 0; k < n; k++) z[k] = num / den * q[k];
  for (int i = lo; i <= pt; i++) {
    int ii = (i + m) % m;
    num = 0.0;
    den = 0.0;
    for (long k = 0; k < n; k++) {
      num += Y[k + ii * n] * z[k];
      den += S[k + ii * n] * Y[k + ii * n];
    }
    for (long k = 0; k < n; k++) z[k] += S[k + ii * n] * (a[ii] - num / den);
  }
  for (long k = 0; k < n; k++) {
    if (z[k] > 1.0) z[k] = 1.0;
    if (z[k] < (-1.0)) z[k] = -1.0;
    z[k] = -z[k];
  }
  free(q);
}

/* LBFGS (ggplvm.cu:865-934): direction, backup, log-space step of Omega/delta/rho0. */
void orc_lbfgs_update(orc_ctx* o, int itr, int rhoflag) {
  const int N = o->N, M = o->M, Q = o->Q, p = o->p;
  const long tot = (long)N + p + (long)N * Q + (long)M * Q + rhoflag;
  const int pt = (itr - 1) % 10, ptp1 = itr % 10;
  double* ss = o->ss;
  if (itr == 0) {
    for (long k = 0; k < tot; k++) {
      ss[k] = -o->grad[k] / 100000.0;
      if (ss[k] > 1.0) ss[k] = 1.0;
      if (ss[k] < (-1.0)) ss[k] = -1.0;
      o->grad0[k] = o->grad[k];
    }
  } else {
    for (long k = 0; k < tot; k++) {
      o->XX[k + pt * tot] = o->grad[k] - o->grad0[k];
      o->grad0[k] = o->grad[k];
    }
    lbfgs_dir(o->SS, o->XX, o->grad, tot, 10, itr, ss);
  }
  for (int k = 0; k < N; k++) {
    o->Omega[k + N] = o->Omega[k];
    o->Omega[k] = exp(log(o->Omega[k]) - ss[k]);
    if (o->Omega[k] > 1000.) o->Omega[k] = 1000.;
    if (o->Omega[k] < .001) o->Omega[k] = .001;
  }
  for (int k = 0; k < p; k++) {
    o->delta[k + p] = o->delta[k];
    o->delta[k] = exp(log(o->delta[k]) - ss[N + k]);
  }
  for (long k = 0; k < (long)N * Q; k++) {
    o->X[k + (long)N * Q] = o->X[k];
    o->X[k] = o->X[k] - ss[N + p + k];
  }
  for (long k = 0; k < (long)M * Q; k++) {
    o->T[k + (long)M * Q] = o->T[k];
    o->T[k] = o->T[k] - ss[N + p + (long)N * Q + k];
  }
  o->rho[Q] = o->rho[0];
  o->rho[0] = exp(log(o->rho[0]) - ss[N + p + (long)N * Q + (long)M * Q] * ((double)rhoflag));
  mscale(Q - 1, o->rho + 1, 10.0);
  for (long k = 0; k < tot; k++) o->SS[k + ptp1 * tot] = ss[k];
}

/* Downdate (ggplvm.cu:818-859): restore the backup and take r times the step. */
void orc_downdate(orc_ctx* o, int itr, double r, int rhoflag) {
  const int N = o->N, M = o->M, Q = o->Q, p = o->p;
  const long tot = (long)N + p + (long)N * Q + (long)M * Q + rhoflag;
  const int ptp1 = itr % 10;
  const double* ss = o->ss;
  for (int k = 0; k < N; k++) {
    o->Omega[k] = exp(log(o->Omega[k + N]) - r * ss[k]);
    if (o->Omega[k] > 1000.) o->Omega[k] = 1000.;
    if (o->Omega[k] < .001) o->Omega[k] = .001;
  }
  for (int k = 0; k < p; k++) o->delta[k] = exp(log(o->delta[k + p]) - r * ss[N + k]);
  for (long k = 0; k < (long)N * Q; k++) o->X[k] = o->X[k + (long)N * Q] - r * ss[N + p + k];
  for (long k = 0; k < (long)M * Q; k++) o->T[k] = o->T[k + (long)M * Q] - r * ss[N + p + (long)N * Q + k];
  o->rho[0] = exp(log(o->rho[Q]) - r * ss[N + p + (long)N * Q + (long)M * Q] * ((double)rhoflag));
  mscale(Q - 1, o->rho + 1, 10.0);
  for (long k = 0; k < tot; k++) o->SS[k + ptp1 * tot] = r * ss[k];
}

/* getBetaFromTildeBeta (ggplvm.cu:394-402) */
void orc_beta_from_tilde(orc_ctx* o) {
  for (long k = 0; k < (long)o->P * o->J; k++) o->Beta[k] = o->tBeta[k] + o->zeta[k % o->P];
}

/* The driver's outer loop (ggplvm.cu:1146-1330) under explicit budgets. */
int orc_fit(orc_ctx* o, int itr_max, int lbfgs_budget, int* stats, double* trace, int trace_cap) {
  int itr, jtr, JTRMAX, rhoflag = 0, total_lbfgs = 0, total_irls = 0, total_evals = 0, ntrace = 0, rc = 0;
  int budget_hit = 0;
  for (itr = 0; itr < itr_max && !budget_hit; itr++) {
    JTRMAX = (itr == 0) ? 200 : 100;
    int n = orc_irls(o, JTRMAX);
    if (n < 0) { rc = 1; itr++; break; }
    total_irls += n;
    double l0 = orc_objective_after_irls(o);
    total_evals++;
    if (trace && ntrace < trace_cap) trace[ntrace++] = l0;
    if (itr > 20) rhoflag = 1;
    if (itr == 30) JTRMAX = 10000;
    for (jtr = 0; jtr < JTRMAX; jtr++) {
      orc_gradient(o, NULL);
      orc_lbfgs_update(o, jtr, rhoflag);
      double sr = 1.0;
      double* l = o->lkhd;
      for (int ktr = 1; ktr < 8; ktr++) {
        orc_objective(o, jtr + 1);
        total_evals++;
        if (l[jtr + 1] > l[jtr] || ktr == 7) break;
        else if (isnan(l[jtr + 1]) || isinf(l[jtr + 1])) sr *= 0.01;
        else if (l[jtr + 1] < l[jtr]) sr *= 0.1;
        orc_downdate(o, jtr, sr, rhoflag);
      }
      total_lbfgs++;
      if (trace && ntrace < trace_cap) trace[ntrace++] = l[jtr + 1];
      if (jtr > 0 && fabs(l[jtr + 1] - l[jtr]) < fabs(l[jtr + 1]) * 1e-8) break;
      if (lbfgs_budget > 0 && total_lbfgs >= lbfgs_budget) { budget_hit = 1; break; }
    }
    orc_expand_delta(o);
    orc_beta_from_tilde(o);
  }
  if (stats) { stats[0] = itr; stats[1] = total_irls; stats[2] = total_lbfgs; stats[3] = total_evals; }
  return rc;
}

/* getScoreStats (ggplvm_de.cu:489-535): for gene j and genotype column l of G (N x L,
 * column-major), t = Z^T diag(W_j / Omega) g (getZtOinvjnj), v = g^T diag(W_j/Omega) g -
 * t^T Psi_j^{-1} t (cholsl with the factored Psi_j), and the score
 * sum_i g_i / Omega_i (y_ij - W_ij) over the merge walk of gene j's counts (unmatched cells
 * contribute -g_i W_ij / Omega_i), divided by sqrt(phi_j v). S is J x L (S[j + l*J]). */
void orc_score_stats(orc_ctx* o, int L, const double* G, double* S) {
  const int N = o->N, J = o->J, P = o->P;
#pragma omp parallel
  {
    double* tmp = (double*)xcalloc(P, sizeof(double));
    double* tmp2 = (double*)xcalloc(P, sizeof(double));
#pragma omp for collapse(2) schedule(dynamic, 4)
    for (int lg = 0; lg < L; lg++)
      for (int j = 0; j < J; j++) {
        const double* Wj = o->W + (size_t)j * N;
        const double* gl = G + (size_t)lg * N;
        const double* Psij = o->Psi + (size_t)j * P * P;
        memset(tmp2, 0, sizeof(double) * P);
        zt_oinv_nu(o, Wj, gl, tmp);
        cholsl(Psij, P, tmp, tmp2);
        double v = 0.0;
        for (int i = 0; i < N; i++) v += gl[i] * gl[i] * Wj[i] / o->Omega[i];
        for (int i = 0; i < P; i++) v -= tmp[i] * tmp2[i];
        int l = o->gp[j];
        const int lmax = o->gp[j + 1];
        double ss = 0.0;
        for (int i = 0; i < N; i++) {
          if (l < lmax && i == o->ci[l]) {
            ss += gl[i] / o->Omega[i] * (o->cx[l] - Wj[i]);
            l++;
          } else {
            ss += gl[i] * Wj[i] / o->Omega[i] * (-1.0);
          }
        }
        S[j + (size_t)lg * J] = ss / sqrt(o->phi[j] * v);
      }
    free(tmp);
    free(tmp2);
  }
}

/* ---- the differential-expression driver's model comparison: ggplvm_de.cu ----------- */
/* The DE driver (ggplvm_de.cu:886-1237) refits the GLM part by IRLS, at the fitted Omega,
 * delta, X and rho, for a null model without the GP (Z0), one reduced model per latent
 * dimension (GP over that dimension alone, Mredc equispaced inducing points) and the full
 * model (Mfull inducing points, the fitted T), and keeps every model's per-gene
 * log-likelihood ("BFs", ggplvm_de.cu:1107,1200,1203-1207). Its kernels differ from the fit
 * driver's in the places restated below. */

/* getZeta (ggplvm_de.cu:34-47): the 1/phi-weighted mean coefficient over genes. */
static void de_zeta(orc_ctx* o) {
  const int J = o->J, P = o->P;
  for (int k = 0; k < P; k++) {
    double sum = 0.0, den = 0.0;
    for (int j = 0; j < J; j++) {
      sum += o->Beta[k + (size_t)j * P] / o->phi[j];
      den += 1.0 / o->phi[j];
    }
    o->zeta[k] = sum / den;
  }
}

/* getWForBeta of the DE driver (ggplvm_de.cu:442-486): the Titsias factor enters W with
 * weight 1, and nu = z.(beta - zeta) + (y - W)/W at a count, z.(beta - zeta) - 1 elsewhere. */
static void de_w_nu(orc_ctx* o) {
  const int N = o->N, J = o->J, p = o->p, P = o->P;
#pragma omp parallel for schedule(dynamic, 4)
  for (int j = 0; j < J; j++) {
    const double* bj = o->Beta + (size_t)j * P;
    double* Wj = o->W + (size_t)j * N;
    double* nj = o->Nu + (size_t)j * N;
    int l = o->gp[j], lmax = o->gp[j + 1];
    for (int i = 0; i < N; i++) {
      double sum = 0.0, sum2 = 0.0;
      for (int k = 0; k < p; k++) {
        if (o->vc[k] == 1) {
          const double* pd = o->varbase[k];
          for (int m = 0; m < o->vv[k]; m++) {
            sum += pd[i + (size_t)m * N] * bj[o->nh[k] + m];
            sum2 += pd[i + (size_t)m * N] * (bj[o->nh[k] + m] - o->zeta[o->nh[k] + m]);
          }
        } else {
          int lev = o->varcat[k][i];
          sum += bj[o->nh[k] + lev];
          sum2 += (bj[o->nh[k] + lev] - o->zeta[o->nh[k] + lev]);
        }
      }
      Wj[i] = exp(sum) * o->ls[i] * exp(o->delta[p - 1] * o->titsias[i]);
      if (l < lmax && o->ci[l] == i) {
        nj[i] = sum2 + (o->cx[l] - Wj[i]) / Wj[i];
        l++;
      } else {
        nj[i] = sum2 - 1.0;
      }
    }
  }
}

/* getBetaPhi of the DE driver (ggplvm_de.cu:413-438): undamped, beta = Psi^{-1} b + zeta,
 * phi = (sum nu^2 W/Omega - b . Psi^{-1} b) / N with clamps NaN -> 1, < 0 -> 100,
 * < 0.01 -> 0.01, > 100 -> 100. */
static void de_beta_phi(orc_ctx* o) {
  const int N = o->N, J = o->J, P = o->P;
#pragma omp parallel
  {
    double* b = (double*)xcalloc(P, sizeof(double));
#pragma omp for schedule(dynamic, 4)
    for (int j = 0; j < J; j++) {
      const double* Wj = o->W + (size_t)j * N;
      const double* nj = o->Nu + (size_t)j * N;
      double* bj = o->Beta + (size_t)j * P;
      double phij = 0.0;
      zt_oinv_nu(o, Wj, nj, b);
      for (int i = 0; i < N; i++) phij += nj[i] * nj[i] * Wj[i] / o->Omega[i];
      cholsl(o->Psi + (size_t)j * P * P, P, b, bj);
      for (int k = 0; k < P; k++) {
        phij -= bj[k] * b[k];
        bj[k] += o->zeta[k];
      }
      double ph = phij / (double)N;
      if (isnan(ph)) ph = 1.0;
      if (ph < 0.0) ph = 100.0;
      if (ph < 0.01) ph = 0.01;
      if (ph > 100.0) ph = 100.0;
      o->phi[j] = ph;
    }
    free(b);
  }
}

/* getLkhdPois of the DE driver (ggplvm_de.cu:667-693): per gene
 * (sum_i [(log W - delta_{p-1} titsias) y - W] / Omega - sum_k log L_kk) / phi + P log(2 pi') / 2
 * with the reference's pi' = 3.1415926535. */
static void de_lkhd(orc_ctx* o) {
  const int N = o->N, J = o->J, p = o->p, P = o->P;
#pragma omp parallel for schedule(dynamic, 4)
  for (int j = 0; j < J; j++) {
    const double* Wj = o->W + (size_t)j * N;
    const double* Pj = o->Psi + (size_t)j * P * P;
    int l = o->gp[j], lmax = o->gp[j + 1];
    double sum = 0.0;
    for (int i = 0; i < N; i++) {
      if (l < lmax && o->ci[l] == i) {
        sum += ((log(Wj[i]) - o->delta[p - 1] * o->titsias[i]) * o->cx[l] - Wj[i]) / o->Omega[i];
        l++;
      } else {
        sum -= Wj[i] / o->Omega[i];
      }
    }
    for (int k = 0; k < P; k++) sum -= log(Pj[k + k * P]);
    o->lkhds[j] = sum / o->phi[j] + log(2 * 3.1415926535) * ((double)P) / 2.0;
  }
}

/* One model of the DE driver: the GLM initialisation (initPsi, initPsi2, initBeta) and
 * getZeta (ggplvm_de.cu:1071-1077, 1135-1140), then IRLS sweeps of getWForBeta, getPsi,
 * cholPsi, getBetaPhi, getZeta, getLkhdPois and collectLkhd(N = 0, Q = 0), which sums the
 * per-gene values (ggplvm_de.cu:1079-1104, 1142-1177), stopping at a NaN/inf sum, at
 * jtr_max sweeps or when the relative change falls below tol (1e-5 for the null model,
 * 1e-8 for the others). Kernel matrices are set beforehand (orc_kernel_mats[_lv]); with
 * M = 0 there are none and titsias is 0 (initTitsias). Returns the number of sweeps; the
 * per-gene values are left in "lkhds", the sums in "lkhd". */
int orc_de_irls(orc_ctx* o, int jtr_max, double tol) {
  orc_glm_init(o);
  de_zeta(o);
  int jtr;
  for (jtr = 0; jtr < jtr_max; jtr++) {
    de_w_nu(o);
    gram_chol(o);
    de_beta_phi(o);
    de_zeta(o);
    de_lkhd(o);
    double sum = 0.0;
    for (int k = 0; k < o->J; k++) sum += o->lkhds[k];
    o->lkhd[jtr] = sum;
    if (jtr > 0) {
      if (isinf(sum) || isnan(sum)) { jtr++; break; }
      if (jtr == jtr_max - 1 || fabs(o->lkhd[jtr - 1] - sum) / fabs(sum) < tol) { jtr++; break; }
    }
  }
  return jtr;
}

/* initTaEquispaced (util.c:57-71): dim 0 on (0, 2 pi), dims >= 1 on (-3, 3). */
void orc_ta_equispaced(int M, int Q, double* T) {
  for (int i = 0; i < M; i++) T[i] = ((double)(i + 1) / (double)(M + 1)) * 2.0 * 3.14159265358979;
  for (int k = 1; k < Q; k++)
    for (int i = 0; i < M; i++) T[i + (size_t)k * M] = ((double)(i + 1) / (double)(M + 1) - 0.5) * 6.0;
}

/* ---- the variance-component driver: ggplvm_delta.cu --------------------------------- */
/* ggplvm_delta.cu re-optimises one prior variance, delta[p-2] (that of the last design
 * variable: the genotype when Z.bin ends with it), by L-BFGS on its log, at a fit's Omega, X,
 * T and rho, alternating with IRLS. Its IRLS uses the DE driver's forms (de_w_nu,
 * de_beta_phi, de_zeta); the rest differs from the fit driver as restated here. */

/* getLkhdPois of ggplvm_delta.cu (:610-631): the Titsias factor at weight 1. */
static void vc_lkhd_pois(orc_ctx* o) {
  const int N = o->N, J = o->J, p = o->p;
#pragma omp parallel for schedule(dynamic, 4)
  for (int j = 0; j < J; j++) {
    const double* Wj = o->W + (size_t)j * N;
    int l = o->gp[j], lmax = o->gp[j + 1];
    double sum = 0.0;
    for (int i = 0; i < N; i++) {
      if (l < lmax && o->ci[l] == i) {
        sum += (log(Wj[i]) - o->delta[p - 1] * o->titsias[i]) * o->cx[l] - Wj[i];
        l++;
      } else {
        sum -= Wj[i];
      }
    }
    o->lkhds[j] = sum;
  }
}

/* collectLkhd of ggplvm_delta.cu (:677-704): the genes' sum, N(0, 1) priors on X and T in
 * dimensions >= 1, the Titsias term at weight 0 and an inverse-gamma(30, 30) prior on Omega,
 * over n cells and Q dimensions (0 and 0 in the IRLS). */
static double vc_collect(orc_ctx* o, int n, int Q, int slot) {
  const int J = o->J, p = o->p, M = o->M;
  const double* Oinvt = o->W + (size_t)n * J;
  double sum = 0.0;
  for (int k = 0; k < J; k++) sum += o->lkhds[k];
  for (int i = 0; i < n; i++)
    for (int k = 1; k < Q; k++) sum -= o->X[i + (size_t)k * n] * o->X[i + (size_t)k * n] / 2.0;
  for (int i = 0; i < M; i++)
    for (int k = 1; k < Q; k++) sum -= o->T[i + (size_t)k * M] * o->T[i + (size_t)k * M] / 2.0;
  for (int i = 0; i < n; i++) sum -= 0.0 * o->delta[p - 1] * Oinvt[i] * o->titsias[i];
  for (int i = 0; i < n; i++) sum = sum - 30.0 / o->Omega[i] - 30.0 * log(o->Omega[i]);
  o->lkhd[slot] = sum;
  return sum;
}

/* The objective after an IRLS phase (ggplvm_delta.cu:1012-1020) and at a line-search point
 * (:1047-1070: kernel matrices, DeltaInv, Gram and both factorisations again). */
static double vc_objective(orc_ctx* o, int slot, int full) {
  oinvt(o);
  if (full) {
    orc_kernel_mats(o);
    orc_expand_delta(o);
    gram_chol(o);
  }
  choldc(o->DeltaInv, o->P);
  lkhd_genes(o);
  return vc_collect(o, o->N, o->Q, slot);
}

/* LBFGS of ggplvm_delta.cu (:734-782) on the single variable log delta[p-2]: the first step is
 * -g/10000 (clamped to +-0.01 beyond +-1); later ones run lbfgs (util_cuda.cu:187-232) with a
 * one-element history of that variable's steps and gradient changes but with grad[0], the
 * gradient of log delta[0], as the current gradient, as the reference does. */
static void vc_lbfgs(orc_ctx* o, int itr) {
  const int p = o->p, pt = (itr - 1) % 10, ptp1 = itr % 10;
  double *grad = o->grad, *ss = o->ss;
  if (itr == 0) {
    ss[0] = -grad[p - 2] / 10000.0;
    if (ss[0] > 1.0) ss[0] = 0.01;
    if (ss[0] < (-1.0)) ss[0] = -0.01;
    o->grad0[p - 2] = grad[p - 2];
  } else {
    o->XX[pt] = grad[p - 2] - o->grad0[p - 2];
    o->grad0[p - 2] = grad[p - 2];
    lbfgs_dir(o->SS, o->XX, grad, 1, 10, itr, ss);
  }
  o->delta[p - 2 + p] = o->delta[p - 2];
  o->delta[p - 2] = exp(log(o->delta[p - 2]) - ss[0]);
  o->SS[ptp1] = ss[0];
}

/* Downdate of ggplvm_delta.cu (:707-731): back along the step by the factor r. */
static void vc_downdate(orc_ctx* o, int itr, double r) {
  const int p = o->p, ptp1 = itr % 10;
  o->delta[p - 2] = exp(log(o->delta[p - 2 + p]) - r * o->ss[0]);
  o->SS[ptp1] = r * o->ss[0];
}

/* The driver (ggplvm_delta.cu:962-1097) from the parameters set (delta[p-2] the initial
 * variance), under budgets: itr_max outer iterations (the reference: 100), each an IRLS phase
 * of at most 30 sweeps (stopping at a relative change below 1e-5), the objective, and at most
 * lbfgs_max L-BFGS steps (the reference: 100) with the backtracking line search, stopping at a
 * relative change below 1e-8; then tilde-beta + zeta becomes beta and zeta is recomputed.
 * dg[itr] receives delta[p-2] after each outer iteration and obj[itr] the objective after its
 * last accepted step (up to cap). Returns the outer iterations run. */
int orc_vc_fit(orc_ctx* o, int itr_max, int lbfgs_max, double* dg, double* obj, int cap) {
  const int N = o->N, J = o->J, P = o->P, p = o->p;
  orc_kernel_mats(o);
  orc_glm_init(o);
  de_zeta(o);
  int itr;
  for (itr = 0; itr < itr_max; itr++) {
    const int JT = 30;
    for (int jtr = 0; jtr < JT; jtr++) {
      de_w_nu(o);
      gram_chol(o);
      de_beta_phi(o);
      de_zeta(o);
      vc_lkhd_pois(o);
      vc_collect(o, 0, 0, jtr);
      if (jtr > 0 && (jtr == JT - 1 || fabs(o->lkhd[jtr - 1] - o->lkhd[jtr]) / fabs(o->lkhd[jtr]) < 1e-5)) break;
    }
    vc_objective(o, 0, 0);
    double* l = o->lkhd;
    int jtr;
    for (jtr = 0; jtr < lbfgs_max; jtr++) {
      orc_expand_delta(o);
      oinvt(o);
      grad_log_delta(o, 0.0, o->grad);
      vc_lbfgs(o, jtr);
      double sr = 1.0;
      for (int ktr = 1; ktr < 8; ktr++) {
        vc_objective(o, jtr + 1, 1);
        if (l[jtr + 1] > l[jtr] || ktr == 7) break;
        else if (isnan(l[jtr + 1]) || isinf(l[jtr + 1])) sr *= 0.01;
        else if (l[jtr + 1] < l[jtr]) sr *= 0.1;
        vc_downdate(o, jtr, sr);
      }
      if (jtr > 0 && fabs(l[jtr + 1] - l[jtr]) < fabs(l[jtr + 1]) * 1e-8) { jtr++; break; }
    }
    if (obj && itr < cap) obj[itr] = l[jtr < lbfgs_max ? jtr : lbfgs_max];
    orc_expand_delta(o);
    for (int j = 0; j < J; j++) /* getBetaFromTildeBeta (ggplvm_delta.cu:380-389) */
      for (int k = 0; k < P; k++) o->Beta[k + (size_t)j * P] = o->tBeta[k + (size_t)j * P] + o->zeta[k];
    de_zeta(o);
    if (dg && itr < cap) dg[itr] = o->delta[p - 2];
  }
  (void)N;
  return itr;
}

long orc_get(orc_ctx* o, const char* name, double* out) {
  const size_t N = o->N, J = o->J, M = o->M, Q = o->Q, P = o->P, p = o->p;
  struct { const char* n; const double* ptr; size_t len; } items[] = {
      {"Omega", o->Omega, N},        {"delta", o->delta, p},       {"X", o->X, N * Q},
      {"T", o->T, M * Q},            {"rho", o->rho, Q},           {"phi", o->phi, J},
      {"Beta", o->Beta, P * J},      {"tBeta", o->tBeta, P * J},   {"Knm", o->Knm, N * M},
      {"Kmm", o->Kmm, M * M},        {"Kinv", o->Kinv, M * M},     {"KinvKmn", o->KinvKmn, N * M},
      {"titsias", o->titsias, N},    {"W", o->W, N * (J + 1)},     {"Nu", o->Nu, N * J},
      {"Psi", o->Psi, J * P * P},    {"PsiInv", o->PsiInv, J * P * P},
      {"DeltaInv", o->DeltaInv, P * P}, {"lkhds", o->lkhds, J},   {"C1", o->C1, N * M},
      {"C2", o->C2, M * M},          {"grad", o->grad, N + p + N * Q + M * Q + Q},
      {"ss", o->ss, N + p + N * Q + M * Q + Q},
      {"lkhd", o->lkhd, 50000},      {"zeta", o->zeta, P},
  };
  for (size_t k = 0; k < sizeof(items) / sizeof(items[0]); k++)
    if (strcmp(items[k].n, name) == 0) {
      if (out) memcpy(out, items[k].ptr, sizeof(double) * items[k].len);
      return (long)items[k].len;
    }
  return -1;
}
