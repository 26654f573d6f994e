/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY: drives the reference's own kernels,
 * compiled for the host through ref_shim.h, in the order the reference driver calls
 * them (ggplvm.cu:951-1354, `main`). Built by oracle/Makefile into oracle/_ref/.
 *
 * Nothing here computes model arithmetic: every number comes from the reference
 * kernels (kernel_funcs.cu, chol.cu, util_cuda.cu, init.cu, ggplvm.cu:1-935). The
 * harness only allocates the buffers main allocates (ggplvm.cu:1024-1060), launches
 * the kernels with main's grid/block shapes (ggplvm.cu:1068-1095), and exposes the
 * phases as C functions so tests can compare the product path with the reference
 * step by step. ITRMAX/JTRMAX are hard-coded in main; ref_fit takes them as budgets.
 *
 * Deviations from main, all forced by running without GSL or a GPU:
 *   - initTaWithPer (util.c:73-87, GSL MT19937) is not available: dim 0 of T gets
 *     main's equispaced grid and dims >= 1 start at zero; callers always pass T
 *     through ref_set_params (the --init-params path, ggplvm.cu:1103-1106).
 *   - device memory is calloc'd, so zeta and the unused tail of ss read as zero.
 *   - the per-iteration text dumps (X9.gz, phi.gz, Params9.bin; ggplvm.cu:1302-1315)
 *     are not written.
 */
#include <vector>
#include <string>
#include <cstring>

#include "SparseMat.cuh"
#include "util_cuda.cuh"
#include "init.cuh"
#include "kernel_funcs.cuh"

extern "C" int ref_verbose = 0;

/* kernels defined in ggplvm.cu (no header in the reference) */
extern double wt, igap1, igb;
void solvePsi(int J, int P, double* IdenP, double* Psi);
void getC2(int J, DataFrame* Z, double* Psi, double* W, double* delta, double* tBeta, double* phi, double* K,
           double* Kinv, double* KinvKmn, double wt, double* Work, double* C2);
void getGradTau(int Q, DataFrame* Z, double* Xi, double* Ta, double* rho, double* C1, double* C2, double* grad);
void collectGradLogRho(int Q, DataFrame* Z, double* gradLogRhoTmp, double* grad);
void getGradLogRho(int Q, DataFrame* Z, double* Xi, double* Ta, double* rho, double* C1, double* C2,
                   double* gradLogRhoTmp);
void getGradLogDelta(int J, DataFrame* Z, double* DeltaInv, double* delta, double* K, double* Psi, double* tBeta,
                     double* phi, double* Work, double* gradDeltaTmp);
void collectGradLogDelta(int J, DataFrame* Z, double* delta, double* gradDeltaTmp, double* W, double* titsias,
                         double wt, double* grad);
void getOinvt(int N, int J, double* Omega, double* W);
void getGradLogOmega(int J, int Q, DataFrame* Z, double* Omega, double* delta, double* phi, double* Nu, double* Psi,
                     double* W, double* tBeta, double* Xi, double* Ta, double* rho, double* KinvKmn,
                     double* titsias, double wt, double igap1, double igb, double* Work, double* C1, double* grad);
void getBetaFromTildeBeta(int J, DataFrame* Z, double* tBeta, double* zeta, double* Beta);
void getTildeBeta(int J, DataFrame* Z, double* ls, double* Psi, double* Omega, double* Nu, double* W, double* Work,
                  double* tBeta);
void getBetaPhi(int J, DataFrame* Z, double* ls, double* Psi, double* Omega, double* zeta, double* Nu, double* W,
                double* Work, int jtr, double* Beta, double* phi);
void getWForBeta(SparseMat* Y, DataFrame* Z, double* ls, double* Beta, double* zeta, double* delta, double* titsias,
                 double wt, double* W, double* Nu);
void getPsi(int J, DataFrame* Z, double* Omega, double* DeltaInv, double* W, double* Psi, int jtr);
void cholPsi(int J, int P, double* Psi);
void cholDeltaInv(int P, double* DeltaInv);
void getLkhdPois(SparseMat* Y, DataFrame* Z, double* W, double* delta, double* titsias, double wt, double* lkhds);
void getLkhd(int J, DataFrame* Z, double* Omega, double* DeltaInv, double* phi, double* Nu, double* Psi, double* W,
             double* Work, double* lkhds);
void collectLkhd(int N, int J, int Q, double* Omega, double* lkhds, int itr, int jtr, DataFrame* Z, double* delta,
                 double* Xi, double* Ta, double* W, double* titsias, double wt, double igap1, double igb,
                 double* lkhd_d);
void Downdate(int itr, int Q, DataFrame* Z, double* Omega, double* delta, double* K, double* Xi, double* Ta,
              double* rho, double* grad, double* grad0, double* SS, double* XX, double* ss, double r, int rhoflag);
void LBFGS(int itr, int Q, DataFrame* Z, double* Omega, double* delta, double* K, double* Xi, double* Ta, double* rho,
           double* grad, double* grad0, double* SS, double* XX, double* ss, double* Work, int rhoflag);

void getScoreStats(int L, SparseMat* Y, DataFrame* Z, double* G, double* Psi, double* W, double* Omega,
                   double* phi, double* Work, double* S);

/* the DE driver's own versions of six kernels (ggplvm_de.cu), built into namespace de */
namespace de {
void getZeta(int J, int P, double* Beta, double* phi, double* zeta);
void getBetaPhi(int J, DataFrame* Z, double* ls, double* Psi, double* Omega, double* zeta, double* Nu, double* W,
                double* Work, double* Beta, double* phi);
void getWForBeta(SparseMat* Y, DataFrame* Z, double* ls, double* Beta, double* zeta, double* delta, double* titsias,
                 double* W, double* Nu);
void getPsi(int J, DataFrame* Z, double* Omega, double* DeltaInv, double* W, double* Psi);
void getLkhdPois(SparseMat* Y, DataFrame* Z, double* W, double* delta, double* titsias, double* Psi, double* Omega,
                 double* phi, double* lkhds);
void collectLkhd(int N, int J, int Q, double* Omega, double* lkhds, int itr, int jtr, DataFrame* Z, double* delta,
                 double* Xi, double* Ta, double* W, double* titsias, double wt, double* lkhd_d);
}  // namespace de

/* the variance-component driver's kernels (ggplvm_delta.cu), built into namespace vc */
namespace vc {
void getZeta(int J, int P, double* Beta, double* phi, double* zeta);
void getBetaPhi(int J, DataFrame* Z, double* ls, double* Psi, double* Omega, double* zeta, double* Nu, double* W,
                double* Work, double* Beta, double* phi);
void getWForBeta(SparseMat* Y, DataFrame* Z, double* ls, double* Beta, double* zeta, double* delta, double* titsias,
                 double* W, double* Nu);
void getPsi(int J, DataFrame* Z, double* Omega, double* DeltaInv, double* W, double* Psi);
void cholPsi(int J, int P, double* Psi);
void cholDeltaInv(int P, double* DeltaInv);
void getLkhdPois(SparseMat* Y, DataFrame* Z, double* W, double* delta, double* titsias, double* lkhds);
void getLkhd(int J, DataFrame* Z, double* Omega, double* DeltaInv, double* phi, double* Nu, double* Psi, double* W,
             double* Work, double* lkhds);
void collectLkhd(int N, int J, int Q, double* Omega, double* lkhds, int itr, int jtr, DataFrame* Z, double* delta,
                 double* Xi, double* Ta, double* W, double* titsias, double wt, double* lkhd_d);
void getOinvt(int N, int J, double* Omega, double* W);
void getTildeBeta(int J, DataFrame* Z, double* ls, double* Psi, double* Omega, double* Nu, double* W, double* Work,
                  double* tBeta);
void getGradLogDelta(int J, DataFrame* Z, double* DeltaInv, double* delta, double* K, double* Psi, double* tBeta,
                     double* phi, double* Work, double* gradDeltaTmp);
void collectGradLogDelta(int J, DataFrame* Z, double* delta, double* gradDeltaTmp, double* W, double* titsias,
                         double wt, double* grad);
void getBetaFromTildeBeta(int J, DataFrame* Z, double* tBeta, double* zeta, double* Beta);
void LBFGS(int itr, int Q, DataFrame* Z, double* Omega, double* delta, double* K, double* Xi, double* Ta, double* rho,
           double* grad, double* grad0, double* SS, double* XX, double* ss, double* Work, int rhoflag);
void Downdate(int itr, int Q, DataFrame* Z, double* Omega, double* delta, double* K, double* Xi, double* Ta,
              double* rho, double* grad, double* grad0, double* SS, double* XX, double* ss, double r, int rhoflag);
}  // namespace vc

namespace {

struct RefCtx {
  int N, J, M, Q, P, p;
  SparseMat *Y_h, *Y;
  DataFrame *Z_h, *Z;
  double *Omega, *DeltaInv, *delta, *zeta, *ls, *phi, *Psi, *W, *Nu, *Beta, *tBeta, *lkhds, *lkhd_d;
  double *grad, *grad0, *SS, *XX, *ss, *gradDeltaTmp, *gradLogRhoTmp, *Work;
  double *rho, *Xi, *Ta, *K, *Kinv, *KinvKmn, *C1, *C2, *IdenP, *titsias;
  dim3 gridJ, gridJP, gridPsi, blockPsi, gridPP, gridN, blockN, gridDel, block1, gridNpMM, gridMM, gridMQ, gridQ;
  int rhoflag;
  std::vector<double> lkhd_h;
};

double* dalloc(size_t n) {
  void* p = nullptr;
  cudaMalloc(&p, sizeof(double) * (n ? n : 1));
  return (double*)p;
}

bool read_doubles(const char* path, double* dst, size_t n) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  size_t got = fread(dst, sizeof(double), n, f);
  fclose(f);
  return got == n;
}

}  // namespace

extern "C" {

/* Mirrors main up to the device boundary (ggplvm.cu:965-1101): reference loaders,
 * main's allocations and grid shapes, then initParams. Returns NULL on a file error. */
void* ref_open(const char* y_path, const char* z_path, const char* ls_path, const char* xi_path, int M, int Q) {
  FILE* probe;
  for (const char* pth : {y_path, z_path, ls_path, xi_path}) {
    if (!(probe = fopen(pth, "rb"))) return nullptr;
    fclose(probe);
  }
  RefCtx* c = new RefCtx();
  std::string yp(y_path), zp(z_path);
  c->Y_h = loadSparseMat(&yp[0]);
  c->N = c->Y_h->N;
  c->J = c->Y_h->J;
  c->Y = newSparseMatOnDevice(c->Y_h);
  c->M = M;
  c->Q = Q;
  c->Z_h = loadDataFrame(&zp[0], M);
  c->Z = newDataFrameOnDevice(c->Z_h);
  c->P = c->Z_h->P;
  c->p = c->Z_h->p;
  const int N = c->N, J = c->J, P = c->P, p = c->p;

  c->Psi = dalloc((size_t)J * P * P * 2);
  c->W = dalloc((size_t)N * (J + 1));
  c->Nu = dalloc((size_t)N * J);
  c->grad = dalloc(N + p + (size_t)(N + M + 1) * Q);
  c->grad0 = dalloc(N + p + (size_t)(N + M + 1) * Q);
  c->SS = dalloc((N + p + (size_t)(N + M + 1) * Q) * 10);
  c->XX = dalloc((N + p + (size_t)(N + M + 1) * Q) * 10);
  c->ss = dalloc(N + p + (size_t)(N + M + 1) * Q);
  size_t lwork = (size_t)(N < M * M ? M * M : N);
  if (lwork < (size_t)J * P) lwork = (size_t)J * P;
  lwork *= (2 * P);
  c->Work = dalloc(lwork);
  c->C1 = dalloc((size_t)N * M);
  c->C2 = dalloc((size_t)M * M);
  c->IdenP = dalloc((size_t)P * P);
  c->ls = dalloc(N);
  c->Omega = dalloc((size_t)N * 2);
  c->DeltaInv = dalloc((size_t)P * P);
  c->delta = dalloc((size_t)p * 2);
  c->phi = dalloc(J);
  c->gradDeltaTmp = dalloc((size_t)P * J);
  c->gradLogRhoTmp = dalloc((size_t)M * Q);
  c->zeta = dalloc(P);
  c->Beta = dalloc((size_t)P * J);
  c->tBeta = dalloc((size_t)P * J);
  c->lkhds = dalloc(J);
  c->lkhd_d = dalloc(50000);
  c->rho = dalloc((size_t)Q * 2);
  c->Xi = dalloc((size_t)N * Q * 2);
  c->Ta = dalloc((size_t)M * Q * 2);
  c->K = dalloc((size_t)M * M);
  c->Kinv = dalloc((size_t)M * M);
  c->KinvKmn = dalloc((size_t)N * M);
  c->titsias = dalloc(N);
  c->lkhd_h.assign(50000, 0.0);

  if (!read_doubles(xi_path, c->Xi, (size_t)N * Q) || !read_doubles(ls_path, c->ls, N)) {
    delete c;
    return nullptr;
  }
  for (int i = 0; i < M; i++) c->Ta[i] = ((double)(i + 1) / (double)(M + 1)) * 2.0 * 3.14159265358979;

  int sN = (int)(sqrt((double)N) / 4) + 1;
  c->gridJ = dim3(J, 1);
  c->gridJP = dim3(J, P);
  c->gridPsi = dim3(J, P);
  c->blockPsi = dim3(1, P);
  c->gridPP = dim3(P, P);
  c->gridN = dim3(sN, sN);
  c->blockN = dim3(4, 4);
  c->gridDel = dim3(p, 1);
  c->block1 = dim3(1, 1);
  c->gridNpMM = dim3(N + M, M);
  c->gridMM = dim3(M, M);
  c->gridMQ = dim3(M, Q);
  c->gridQ = dim3(Q, 1);
  c->rhoflag = 0;

  ref_launch(dim3(1), dim3(1), [&] { initParams(N, J, P, p, Q, c->delta, c->Omega, c->phi, c->rho, c->IdenP); });
  return c;
}

void ref_close(void* h) {
  /* buffers are left to process exit: the reference never frees most of them either */
  delete (RefCtx*)h;
}

void ref_dims(void* h, int* out) {
  RefCtx* c = (RefCtx*)h;
  out[0] = c->N; out[1] = c->J; out[2] = c->M; out[3] = c->P; out[4] = c->p; out[5] = c->Q;
}

/* readParams (util_cuda.cu:520-544) without the file: any NULL argument keeps the current value. */
void ref_set_params(void* h, const double* Omega, const double* delta, const double* X, const double* T,
                    const double* rho, const double* phi) {
  RefCtx* c = (RefCtx*)h;
  if (Omega) memcpy(c->Omega, Omega, sizeof(double) * c->N);
  if (delta) memcpy(c->delta, delta, sizeof(double) * c->p);
  if (X) memcpy(c->Xi, X, sizeof(double) * c->N * c->Q);
  if (T) memcpy(c->Ta, T, sizeof(double) * c->M * c->Q);
  if (rho) memcpy(c->rho, rho, sizeof(double) * c->Q);
  if (phi) memcpy(c->phi, phi, sizeof(double) * c->J);
}

void ref_set_beta(void* h, const double* beta) {
  RefCtx* c = (RefCtx*)h;
  memcpy(c->Beta, beta, sizeof(double) * (size_t)c->P * c->J);
}

/* ggplvm.cu:1111-1113 */
void ref_kernel_mats(void* h) {
  RefCtx* c = (RefCtx*)h;
  ref_launch(c->gridNpMM, c->block1, [&] { getKernelMats(c->Q, c->Xi, c->Ta, c->rho, c->Z, c->K, c->Kinv, c->KinvKmn); });
  ref_launch(dim3(1), dim3(1), [&] { cholKmm(c->M, c->Kinv); });
  ref_launch(c->gridN, c->blockN, [&] { getKinvKmn(c->Kinv, c->Z, c->KinvKmn, c->titsias); });
}

/* ggplvm.cu:1134-1137 (GLM initialisation) */
void ref_glm_init(void* h) {
  RefCtx* c = (RefCtx*)h;
  ref_launch(dim3(1), dim3(1), [&] { expandDelta_k(c->Z, c->delta, c->K, c->DeltaInv); });
  ref_launch(c->gridPP, c->block1, [&] { initPsi(c->Z, c->DeltaInv, c->Psi); });
  ref_launch(dim3(1), dim3(1), [&] { initPsi2(c->P, c->Psi); });
  ref_launch(c->gridJ, c->block1, [&] { initBeta(c->Y, c->ls, c->Z, c->Psi, c->Work, c->Beta); });
}

void ref_expand_delta(void* h) {
  RefCtx* c = (RefCtx*)h;
  ref_launch(dim3(1), dim3(1), [&] { expandDelta_k(c->Z, c->delta, c->K, c->DeltaInv); });
}

/* One IRLS sweep, ggplvm.cu:1156-1181; returns lkhd_d[jtr] (the Poisson log-likelihood sum). */
double ref_irls_sweep(void* h, int itr, int jtr) {
  RefCtx* c = (RefCtx*)h;
  ref_launch(c->gridJ, c->block1,
             [&] { getWForBeta(c->Y, c->Z, c->ls, c->Beta, c->zeta, c->delta, c->titsias, wt, c->W, c->Nu); });
  ref_launch(c->gridPsi, c->blockPsi, [&] { getPsi(c->J, c->Z, c->Omega, c->DeltaInv, c->W, c->Psi, jtr + 1); });
  ref_launch(c->gridJ, c->block1, [&] { cholPsi(c->J, c->P, c->Psi); });
  ref_launch(c->gridJ, c->block1, [&] {
    getBetaPhi(c->J, c->Z, c->ls, c->Psi, c->Omega, c->zeta, c->Nu, c->W, c->Work, jtr, c->Beta, c->phi);
  });
  ref_launch(c->gridJ, c->block1, [&] { getLkhdPois(c->Y, c->Z, c->W, c->delta, c->titsias, wt, c->lkhds); });
  ref_launch(dim3(1), dim3(1), [&] {
    collectLkhd(0, c->J, 0, c->Omega, c->lkhds, itr, jtr, c->Z, c->delta, c->Xi, c->Ta, c->W, c->titsias, wt, igap1,
                igb, c->lkhd_d);
  });
  c->lkhd_h[jtr] = c->lkhd_d[jtr];
  return c->lkhd_d[jtr];
}

/* The IRLS loop with main's stopping rule (ggplvm.cu:1152-1189). Returns the number of
 * sweeps run, or -1 when main would exit on a NaN likelihood (ggplvm.cu:1182). */
int ref_irls(void* h, int itr, int jtr_max) {
  RefCtx* c = (RefCtx*)h;
  int jtr;
  for (jtr = 0; jtr < jtr_max; jtr++) {
    ref_irls_sweep(h, itr, jtr);
    double* l = c->lkhd_h.data();
    if (jtr > 0) {
      if (std::isnan(l[jtr])) return -1;
      if (jtr == (jtr_max - 1) || fabs(l[jtr - 1] - l[jtr]) / fabs(l[jtr]) < 1e-7) { jtr++; break; }
    }
  }
  return jtr;
}

/* ggplvm.cu:1205-1211: objective at the IRLS solution, stored in lkhd_d[0]. */
double ref_objective_after_irls(void* h, int itr) {
  RefCtx* c = (RefCtx*)h;
  ref_launch(c->gridN, c->blockN, [&] { getOinvt(c->N, c->J, c->Omega, c->W); });
  ref_launch(dim3(1), dim3(1), [&] { cholDeltaInv(c->P, c->DeltaInv); });
  ref_launch(c->gridJ, c->block1, [&] {
    getLkhd(c->J, c->Z, c->Omega, c->DeltaInv, c->phi, c->Nu, c->Psi, c->W, c->Work, c->lkhds);
  });
  ref_launch(dim3(1), dim3(1), [&] {
    collectLkhd(c->N, c->J, c->Q, c->Omega, c->lkhds, itr, 0, c->Z, c->delta, c->Xi, c->Ta, c->W, c->titsias, wt,
                igap1, igb, c->lkhd_d);
  });
  c->lkhd_h[0] = c->lkhd_d[0];
  return c->lkhd_d[0];
}

/* One gradient evaluation, ggplvm.cu:1215-1240. Writes the N+p+N*Q+M*Q+Q vector. */
void ref_gradient(void* h, double* grad_out) {
  RefCtx* c = (RefCtx*)h;
  const int N = c->N, J = c->J, M = c->M, Q = c->Q, P = c->P, p = c->p;
  ref_launch(dim3(1), dim3(1), [&] { expandDelta_k(c->Z, c->delta, c->K, c->DeltaInv); });
  ref_launch(c->gridN, c->blockN, [&] { getOinvt(N, J, c->Omega, c->W); });
  ref_launch(c->gridJ, c->block1,
             [&] { getTildeBeta(J, c->Z, c->ls, c->Psi, c->Omega, c->Nu, c->W, c->Work, c->tBeta); });
  ref_launch(c->gridJP, c->block1, [&] {
    getGradLogDelta(J, c->Z, c->DeltaInv, c->delta, c->K, c->Psi, c->tBeta, c->phi, c->Work, c->gradDeltaTmp);
  });
  ref_launch(c->gridDel, c->block1,
             [&] { collectGradLogDelta(J, c->Z, c->delta, c->gradDeltaTmp, c->W, c->titsias, wt, c->grad); });
  ref_launch(c->gridN, c->blockN, [&] {
    getGradLogOmega(J, Q, c->Z, c->Omega, c->delta, c->phi, c->Nu, c->Psi, c->W, c->tBeta, c->Xi, c->Ta, c->rho,
                    c->KinvKmn, c->titsias, wt, igap1, igb, c->Work, c->C1, c->grad);
  });
  ref_launch(c->gridJP, c->block1, [&] { solvePsi(J, P, c->IdenP, c->Psi); });
  ref_launch(c->gridMM, c->block1, [&] {
    getC2(J, c->Z, c->Psi, c->W, c->delta, c->tBeta, c->phi, c->K, c->Kinv, c->KinvKmn, wt, c->Work, c->C2);
  });
  ref_launch(c->gridMQ, c->block1, [&] { getGradTau(Q, c->Z, c->Xi, c->Ta, c->rho, c->C1, c->C2, c->grad); });
  ref_launch(c->gridMQ, c->block1,
             [&] { getGradLogRho(Q, c->Z, c->Xi, c->Ta, c->rho, c->C1, c->C2, c->gradLogRhoTmp); });
  ref_launch(c->gridQ, c->block1, [&] { collectGradLogRho(Q, c->Z, c->gradLogRhoTmp, c->grad); });
  if (grad_out) memcpy(grad_out, c->grad, sizeof(double) * ((size_t)N + p + (size_t)N * Q + (size_t)M * Q + Q));
}

/* One line-search evaluation of the objective, ggplvm.cu:1258-1277; stores lkhd_d[slot]. */
double ref_objective(void* h, int itr, int slot) {
  RefCtx* c = (RefCtx*)h;
  ref_launch(c->gridN, c->blockN, [&] { getOinvt(c->N, c->J, c->Omega, c->W); });
  ref_launch(c->gridNpMM, c->block1,
             [&] { getKernelMats(c->Q, c->Xi, c->Ta, c->rho, c->Z, c->K, c->Kinv, c->KinvKmn); });
  ref_launch(dim3(1), dim3(1), [&] { expandDelta_k(c->Z, c->delta, c->K, c->DeltaInv); });
  ref_launch(dim3(1), dim3(1), [&] { cholKmm(c->M, c->Kinv); });
  ref_launch(c->gridN, c->blockN, [&] { getKinvKmn(c->Kinv, c->Z, c->KinvKmn, c->titsias); });
  ref_launch(c->gridPsi, c->blockPsi,
             [&] { getPsi(c->J, c->Z, c->Omega, c->DeltaInv, c->W, c->Psi, slot); });
  ref_launch(c->gridJ, c->block1, [&] { cholPsi(c->J, c->P, c->Psi); });
  ref_launch(dim3(1), dim3(1), [&] { cholDeltaInv(c->P, c->DeltaInv); });
  ref_launch(c->gridJ, c->block1, [&] {
    getLkhd(c->J, c->Z, c->Omega, c->DeltaInv, c->phi, c->Nu, c->Psi, c->W, c->Work, c->lkhds);
  });
  ref_launch(dim3(1), dim3(1), [&] {
    collectLkhd(c->N, c->J, c->Q, c->Omega, c->lkhds, itr, slot, c->Z, c->delta, c->Xi, c->Ta, c->W, c->titsias, wt,
                igap1, igb, c->lkhd_d);
  });
  c->lkhd_h[slot] = c->lkhd_d[slot];
  return c->lkhd_d[slot];
}

/* ggplvm.cu:1251 */
void ref_lbfgs_update(void* h, int jtr, int rhoflag) {
  RefCtx* c = (RefCtx*)h;
  ref_launch(dim3(1), dim3(1), [&] {
    LBFGS(jtr, c->Q, c->Z, c->Omega, c->delta, c->K, c->Xi, c->Ta, c->rho, c->grad, c->grad0, c->SS, c->XX, c->ss,
          c->Work, rhoflag);
  });
}

/* ggplvm.cu:1289 */
void ref_downdate(void* h, int jtr, double sr, int rhoflag) {
  RefCtx* c = (RefCtx*)h;
  ref_launch(dim3(1), dim3(1), [&] {
    Downdate(jtr, c->Q, c->Z, c->Omega, c->delta, c->K, c->Xi, c->Ta, c->rho, c->grad, c->grad0, c->SS, c->XX, c->ss,
             sr, rhoflag);
  });
}

/* ggplvm.cu:1324 */
void ref_beta_from_tilde(void* h) {
  RefCtx* c = (RefCtx*)h;
  ref_launch(c->gridJ, dim3(1), [&] { getBetaFromTildeBeta(c->J, c->Z, c->tBeta, c->zeta, c->Beta); });
}

/* The outer fit loop of main (ggplvm.cu:1146-1330) with its schedule, stopping rules and
 * line search, under explicit budgets: at most itr_max outer iterations and at most
 * lbfgs_budget L-BFGS steps in total (<= 0: no budget). stats[0..3] receive outer
 * iterations, total IRLS sweeps, total L-BFGS steps, total objective evaluations.
 * Returns 0, or 1 where main would exit on a NaN IRLS likelihood. */
int ref_fit(void* h, int itr_max, int lbfgs_budget, int* stats, double* lkhd_trace, int trace_cap) {
  RefCtx* c = (RefCtx*)h;
  int JTRMAX = 1000, itr, jtr, total_lbfgs = 0, total_irls = 0, total_evals = 0, ntrace = 0;
  int rhoflag = 0;
  int rc = 0;
  bool budget_hit = false;
  for (itr = 0; itr < itr_max && !budget_hit; itr++) {
    JTRMAX = (itr == 0) ? 200 : 100;
    int n = ref_irls(h, itr, JTRMAX);
    if (n < 0) { rc = 1; itr++; break; }
    total_irls += n;
    double l0 = ref_objective_after_irls(h, itr);
    total_evals++;
    if (lkhd_trace && ntrace < trace_cap) lkhd_trace[ntrace++] = l0;
    if (itr > 20) rhoflag = 1;
    if (itr == 30) JTRMAX = 10000;
    for (jtr = 0; jtr < JTRMAX; jtr++) {
      ref_gradient(h, nullptr);
      ref_lbfgs_update(h, jtr, rhoflag);
      double sr = 1.0;
      double* l = c->lkhd_h.data();
      for (int ktr = 1; ktr < 8; ktr++) {
        ref_objective(h, itr, jtr + 1);
        total_evals++;
        if (l[jtr + 1] > l[jtr] || ktr == 7) break;
        else if (std::isnan(l[jtr + 1]) || std::isinf(l[jtr + 1])) sr *= 0.01;
        else if (l[jtr + 1] < l[jtr]) sr *= 0.1;
        ref_downdate(h, jtr, sr, rhoflag);
      }
      total_lbfgs++;
      if (lkhd_trace && ntrace < trace_cap) lkhd_trace[ntrace++] = l[jtr + 1];
      if (jtr > 0 && fabs(l[jtr + 1] - l[jtr]) < fabs(l[jtr + 1]) * 1e-8) break;
      if (lbfgs_budget > 0 && total_lbfgs >= lbfgs_budget) { budget_hit = true; break; }
    }
    ref_expand_delta(h);
    ref_beta_from_tilde(h);
  }
  c->rhoflag = rhoflag;
  if (stats) { stats[0] = itr; stats[1] = total_irls; stats[2] = total_lbfgs; stats[3] = total_evals; }
  return rc;
}

/* Copies a named buffer out (element counts follow main's allocations). Returns the
 * number of doubles written, or -1 for an unknown name. */
long ref_get(void* h, const char* name, double* out) {
  RefCtx* c = (RefCtx*)h;
  const size_t N = c->N, J = c->J, M = c->M, Q = c->Q, P = c->P, p = c->p;
  struct Item { const char* n; const double* ptr; size_t len; };
  DataFrame* Zd = c->Z;
  const Item items[] = {
      {"Omega", c->Omega, N},        {"delta", c->delta, p},         {"X", c->Xi, N * Q},
      {"T", c->Ta, M * Q},           {"rho", c->rho, Q},             {"phi", c->phi, J},
      {"Beta", c->Beta, P * J},      {"tBeta", c->tBeta, P * J},     {"Knm", Zd->Knm, N * M},
      {"Kmm", c->K, M * M},          {"Kinv", c->Kinv, M * M},       {"KinvKmn", c->KinvKmn, N * M},
      {"titsias", c->titsias, N},    {"W", c->W, N * (J + 1)},       {"Nu", c->Nu, N * J},
      {"Psi", c->Psi, J * P * P},    {"PsiInv", c->Psi + J * P * P, J * P * P},
      {"DeltaInv", c->DeltaInv, P * P}, {"lkhds", c->lkhds, J},     {"C1", c->C1, N * M},
      {"C2", c->C2, M * M},          {"grad", c->grad, N + p + N * Q + M * Q + Q},
      {"ss", c->ss, N + p + N * Q + M * Q + Q},
      {"lkhd", c->lkhd_d, 50000},    {"zeta", c->zeta, P},
  };
  for (const Item& it : items) {
    if (strcmp(it.n, name) == 0) {
      if (out) memcpy(out, it.ptr, sizeof(double) * it.len);
      return (long)it.len;
    }
  }
  return -1;
}

/* Model-matrix column metadata from the reference loader (DataFrame.cu:88-149). */
void ref_model_meta(void* h, int* nh_out, int* mc_out, int* mv_out, int* mk_out) {
  RefCtx* c = (RefCtx*)h;
  if (nh_out) memcpy(nh_out, c->Z_h->nh, sizeof(int) * (c->p + 1));
  if (mc_out) memcpy(mc_out, c->Z_h->mc, sizeof(int) * c->P);
  if (mv_out) memcpy(mv_out, c->Z_h->mv, sizeof(int) * c->P);
  if (mk_out) memcpy(mk_out, c->Z_h->mk, sizeof(int) * c->P);
}

void ref_set_verbose(int v) { ref_verbose = v; }

/* The genotype score statistics of ggplvm_de.cu (getScoreStats :489-535, launched over a
 * J x L grid at :1205-1209) at the current W, Psi factor, Omega and phi. G is N x L
 * (column-major), S is J x L. */
void ref_score_stats(void* h, int L, const double* G, double* S) {
  RefCtx* c = (RefCtx*)h;
  std::vector<double> g(G, G + (size_t)c->N * L), work((size_t)2 * c->J * L * c->P), s((size_t)c->J * L);
  ref_launch(dim3(c->J, L), dim3(1), [&] {
    getScoreStats(L, c->Y, c->Z, g.data(), c->Psi, c->W, c->Omega, c->phi, work.data(), s.data());
  });
  std::memcpy(S, s.data(), sizeof(double) * s.size());
}

/* The model comparison of the differential-expression driver (ggplvm_de.cu:886-1207),
 * from its loaders to the per-gene log-likelihood table "BFs" (J x (Q + 2), gene fastest:
 * column 0 the null model Z0, column q + 1 the GP over latent dimension q alone with Mredc
 * inducing points, column Q + 1 the full model with Mfull), with main's allocations, grid
 * shapes and stopping rules, under a budget of jtr_max IRLS sweeps per model (main: 1000).
 * The fitted Omega, delta, X, T (Mfull x Q) and rho arrive as readParams would read them
 * (ggplvm_de.cu:1040-1043); phi restarts at 1 (initPhi) and titsias at 0 (initTitsias).
 * initTaEquispaced (util.c:57-71, in the GSL-dependent util.c) is restated for the reduced
 * models' inducing points. sweeps[Q + 2] receives each model's IRLS count; beta_full (P1 x J)
 * and phi_out (J) the last model's coefficients and dispersions (either may be NULL).
 * Returns P1, or -1 on a file error. */
int ref_de_bfs(const char* y_path, const char* z_path, const char* ls_path, int Q, int Mredc, int Mfull,
               const double* Omega_in, const double* delta_in, const double* X_in, const double* Tfull_in,
               const double* rho_in, int jtr_max, double* BFs_out, int* sweeps, double* beta_full, double* phi_out) {
  FILE* probe;
  for (const char* pth : {y_path, z_path, ls_path}) {
    if (!(probe = fopen(pth, "rb"))) return -1;
    fclose(probe);
  }
  std::string yp(y_path), zp(z_path);
  SparseMat* Y_h = loadSparseMat(&yp[0]);
  const int N = Y_h->N, J = Y_h->J;
  SparseMat* Y = newSparseMatOnDevice(Y_h);
  DataFrame* Z_h = loadDataFrame(&zp[0], Mredc);
  DataFrame* Z0_h = loadDataFrame(&zp[0]);
  DataFrame* Z1_h = loadDataFrame(&zp[0], Mfull);
  DataFrame* Z = newDataFrameOnDevice(Z_h);
  DataFrame* Z0 = newDataFrameOnDevice(Z0_h);
  DataFrame* Z1 = newDataFrameOnDevice(Z1_h);
  const int P0 = Z0_h->P, P1 = Z1_h->P, p = Z_h->p;
  int P = P1, M = Mfull;
  const int JTRMAX = jtr_max;
  const double wt = 0.0; /* ggplvm_de.cu:20 */

  double* Psi = dalloc((size_t)J * P * P * 2);
  double* W = dalloc((size_t)N * (J + 1));
  double* Nu = dalloc((size_t)N * J);
  size_t lwork = (size_t)(N < M * M ? M * M : N);
  lwork *= (2 * P);
  double* Work = dalloc(lwork);
  double* ls = dalloc(N);
  double* Omega = dalloc((size_t)N * 2);
  double* DeltaInv = dalloc((size_t)P * P);
  double* delta = dalloc((size_t)p * 2);
  double* phi = dalloc(J);
  double* zeta = dalloc(P);
  double* Beta = dalloc((size_t)P * J);
  double* lkhds = dalloc(J);
  double* BFs = dalloc((size_t)J * (Q + 2));
  double* lkhd_d = dalloc(JTRMAX);
  double* rho = dalloc((size_t)Q * 2);
  double* Xi = dalloc((size_t)N * Q * 2);
  double* Ta1 = dalloc((size_t)Mfull * Q * 2);
  double* Ta = dalloc((size_t)Mredc * Q * 2);
  double* K = dalloc((size_t)M * M);
  double* Kinv = dalloc((size_t)M * M);
  double* KinvKmn = dalloc((size_t)N * M);
  double* titsias = dalloc(N);
  std::vector<double> lkhd_h(JTRMAX);

  for (int i = 0; i < Mredc; i++) Ta[i] = ((double)(i + 1) / (double)(Mredc + 1)) * 2.0 * 3.14159265358979;
  for (int k = 1; k < Q; k++)
    for (int i = 0; i < Mredc; i++) Ta[i + k * Mredc] = ((double)(i + 1) / (double)(Mredc + 1) - 0.5) * 6.0;
  if (!read_doubles(ls_path, ls, N)) return -1;
  memcpy(Omega, Omega_in, sizeof(double) * N);
  memcpy(delta, delta_in, sizeof(double) * p);
  memcpy(Xi, X_in, sizeof(double) * (size_t)N * Q);
  memcpy(Ta1, Tfull_in, sizeof(double) * (size_t)Mfull * Q);
  memcpy(rho, rho_in, sizeof(double) * Q);

  const dim3 gridJ(J, 1), block1(1, 1), gridPsi0(J, P0), blockPsi0(1, P0), gridPP0(P0, P0);
  const int sN = (int)(sqrt((double)N) / 4) + 1;
  const dim3 gridN(sN, sN), blockN(4, 4);
  int q = 0, jtr = 0;

  /* null model (ggplvm_de.cu:1067-1107) */
  ref_launch(dim3(1), block1, [&] { initPhi(J, phi); });
  ref_launch(dim3(1), block1, [&] { initTitsias(N, titsias); });
  ref_launch(dim3(1), block1, [&] { expandDeltaWOK_k(Z0, delta, DeltaInv); });
  ref_launch(gridPP0, block1, [&] { initPsi(Z0, DeltaInv, Psi); });
  ref_launch(dim3(1), block1, [&] { initPsi2(P0, Psi); });
  ref_launch(gridJ, block1, [&] { initBeta(Y, ls, Z0, Psi, Work, Beta); });
  ref_launch(dim3(P0), block1, [&] { de::getZeta(J, P0, Beta, phi, zeta); });
  for (jtr = 0; jtr < JTRMAX; jtr++) {
    ref_launch(gridJ, block1, [&] { de::getWForBeta(Y, Z0, ls, Beta, zeta, delta, titsias, W, Nu); });
    ref_launch(gridPsi0, blockPsi0, [&] { de::getPsi(J, Z0, Omega, DeltaInv, W, Psi); });
    ref_launch(gridJ, block1, [&] { cholPsi(J, P0, Psi); });
    ref_launch(gridJ, block1, [&] { de::getBetaPhi(J, Z0, ls, Psi, Omega, zeta, Nu, W, Work, Beta, phi); });
    ref_launch(dim3(P0), block1, [&] { de::getZeta(J, P0, Beta, phi, zeta); });
    ref_launch(gridJ, block1, [&] { de::getLkhdPois(Y, Z0, W, delta, titsias, Psi, Omega, phi, lkhds); });
    ref_launch(dim3(1), block1, [&] {
      de::collectLkhd(0, J, 0, Omega, lkhds, q, jtr, Z0, delta, Xi, Ta, W, titsias, wt, lkhd_d);
    });
    lkhd_h[jtr] = lkhd_d[jtr];
    if (jtr > 0) {
      if (std::isinf(lkhd_h[jtr]) || std::isnan(lkhd_h[jtr])) break;
      if (jtr == (JTRMAX - 1) || fabs(lkhd_h[jtr - 1] - lkhd_h[jtr]) / fabs(lkhd_h[jtr]) < 1e-5) break;
    }
  }
  if (sweeps) sweeps[0] = jtr < JTRMAX ? jtr + 1 : JTRMAX;
  memcpy(BFs, lkhds, sizeof(double) * J);

  /* reduced models q = 0..Q-1 and the full model q = Q (ggplvm_de.cu:1110-1207) */
  for (q = 0; q < Q + 1; q++) {
    DataFrame *pZ, *pZ_h;
    double* pT;
    if (q == Q) {
      pZ = Z1; pZ_h = Z1_h; pT = Ta1; P = P1; M = Mfull;
      ref_launch(dim3(N + Mfull, Mfull), block1, [&] { getKernelMats(Q, Xi, pT, rho, pZ, K, Kinv, KinvKmn); });
    } else {
      M = Mredc; P = Z_h->P; pZ = Z; pZ_h = Z_h; pT = Ta;
      ref_launch(dim3(N + Mredc, Mredc), block1, [&] { getKernelMats(Q, Xi, pT, rho, pZ, q, K, Kinv, KinvKmn); });
    }
    ref_launch(dim3(1), block1, [&] { cholKmm(M, Kinv); });
    ref_launch(gridN, blockN, [&] { getKinvKmn(Kinv, pZ, KinvKmn, titsias); });
    ref_launch(dim3(1), block1, [&] { expandDelta_k(pZ, delta, K, DeltaInv); });
    ref_launch(dim3(pZ_h->P, pZ_h->P), block1, [&] { initPsi(pZ, DeltaInv, Psi); });
    ref_launch(dim3(1), block1, [&] { initPsi2(P, Psi); });
    ref_launch(gridJ, block1, [&] { initBeta(Y, ls, pZ, Psi, Work, Beta); });
    ref_launch(dim3(pZ_h->P), block1, [&] { de::getZeta(J, P, Beta, phi, zeta); });
    for (jtr = 0; jtr < JTRMAX; jtr++) {
      ref_launch(gridJ, block1, [&] { de::getWForBeta(Y, pZ, ls, Beta, zeta, delta, titsias, W, Nu); });
      ref_launch(dim3(J, P), dim3(1, P), [&] { de::getPsi(J, pZ, Omega, DeltaInv, W, Psi); });
      ref_launch(gridJ, block1, [&] { cholPsi(J, P, Psi); });
      ref_launch(gridJ, block1, [&] { de::getBetaPhi(J, pZ, ls, Psi, Omega, zeta, Nu, W, Work, Beta, phi); });
      ref_launch(dim3(pZ_h->P), block1, [&] { de::getZeta(J, P, Beta, phi, zeta); });
      ref_launch(gridJ, block1, [&] { de::getLkhdPois(Y, pZ, W, delta, titsias, Psi, Omega, phi, lkhds); });
      ref_launch(dim3(1), block1, [&] {
        de::collectLkhd(0, J, 0, Omega, lkhds, q, jtr, pZ, delta, Xi, pT, W, titsias, wt, lkhd_d);
      });
      lkhd_h[jtr] = lkhd_d[jtr];
      if (jtr > 0) {
        if (std::isinf(lkhd_h[jtr]) || std::isnan(lkhd_h[jtr])) break;
        if (jtr == (JTRMAX - 1) || fabs(lkhd_h[jtr - 1] - lkhd_h[jtr]) / fabs(lkhd_h[jtr]) < 1e-8) break;
      }
    }
    if (sweeps) sweeps[q + 1] = jtr < JTRMAX ? jtr + 1 : JTRMAX;
    memcpy(BFs + (size_t)J * (q + 1), lkhds, sizeof(double) * J);
  }
  memcpy(BFs_out, BFs, sizeof(double) * J * (Q + 2));
  if (beta_full) memcpy(beta_full, Beta, sizeof(double) * (size_t)P1 * J);
  if (phi_out) memcpy(phi_out, phi, sizeof(double) * J);
  return P1;
}

/* The variance-component driver (ggplvm_delta.cu:784-1097; its main does not compile in the
 * reference because it calls a __global__ printMetaDataFrame from the host at :823): main's
 * allocations, initialisation and loops, with the parameters given as arrays instead of the
 * params.bin its main reads from the working directory (ggplvm_delta.cu:944-956): Omega (N),
 * delta_file (the p - 1 values main reads), X (N x Q), T (M x Q), rho (Q). As main, delta[p-2]
 * becomes init_dg and delta[p-1] keeps initParams' value (main copies p - 1 values to the
 * device). Budgets: itr_max outer iterations (main: 100) and lbfgs_max L-BFGS steps per outer
 * iteration (main: 100). dg[itr] receives delta[p-2] after each outer iteration and obj[itr]
 * the objective after its last accepted step (up to cap). Returns the outer iterations run, or
 * -1 on a file error. */
int ref_vc_fit(const char* y_path, const char* z_path, const char* ls_path, int M, int Q, const double* Omega_in,
               const double* delta_file, const double* X_in, const double* T_in, const double* rho_in, double init_dg,
               int itr_max, int lbfgs_max, double* dg, double* obj, int cap) {
  FILE* probe;
  for (const char* pth : {y_path, z_path, ls_path}) {
    if (!(probe = fopen(pth, "rb"))) return -1;
    fclose(probe);
  }
  std::string yp(y_path), zp(z_path);
  SparseMat* Y_h = loadSparseMat(&yp[0]);
  const int N = Y_h->N, J = Y_h->J;
  SparseMat* Y = newSparseMatOnDevice(Y_h);
  DataFrame* Z_h = loadDataFrame(&zp[0], M);
  DataFrame* Z = newDataFrameOnDevice(Z_h);
  const int P = Z_h->P, p = Z_h->p;
  const double wt = 0.0; /* ggplvm_delta.cu:20 */
  const int JTRMAX = 1000;
  const size_t tot = (size_t)N + p + (size_t)(N + M + 1) * Q;
  double* Psi = dalloc((size_t)J * P * P * 2);
  double* W = dalloc((size_t)N * (J + 1));
  double* Nu = dalloc((size_t)N * J);
  double* grad = dalloc(tot);
  double* grad0 = dalloc(tot);
  double* SS = dalloc(tot * 10);
  double* XX = dalloc(tot * 10);
  double* ss = dalloc(tot);
  size_t lwork = (size_t)(N < M * M ? M * M : N) * (2 * P);
  if ((size_t)N < (size_t)J * P) lwork = (size_t)((size_t)J * P < (size_t)M * M ? (size_t)M * M : (size_t)J * P) * (2 * P);
  double* Work = dalloc(lwork);
  double* IdenP = dalloc((size_t)P * P);
  double* ls = dalloc(N);
  double* Omega = dalloc((size_t)N * 2);
  double* DeltaInv = dalloc((size_t)P * P);
  double* delta = dalloc((size_t)p * 2);
  double* phi = dalloc(J);
  double* gradDeltaTmp = dalloc((size_t)P * J);
  double* zeta = dalloc(P);
  double* Beta = dalloc((size_t)P * J);
  double* tBeta = dalloc((size_t)P * J);
  double* lkhds = dalloc(J);
  double* lkhd_d = dalloc(JTRMAX);
  double* rho = dalloc((size_t)Q * 2);
  double* Xi = dalloc((size_t)N * Q * 2);
  double* Ta = dalloc((size_t)M * Q * 2);
  double* K = dalloc((size_t)M * M);
  double* Kinv = dalloc((size_t)M * M);
  double* KinvKmn = dalloc((size_t)N * M);
  double* titsias = dalloc(N);
  std::vector<double> lkhd_h(JTRMAX);
  if (!read_doubles(ls_path, ls, N)) return -1;

  const dim3 gridJ(J, 1), gridJP(J, P), gridPsi(J, P), blockPsi(1, P), gridPP(P, P), gridP(P, 1), gridDel(p, 1),
      block1(1, 1), gridNpMM(N + M, M);
  const int sN = (int)(sqrt((double)N) / 4) + 1;
  const dim3 gridN(sN, sN), blockN(4, 4);

  ref_launch(dim3(1), block1, [&] { initParams(N, J, P, p, Q, delta, Omega, phi, rho, IdenP); });
  /* params.bin (ggplvm_delta.cu:944-956): p - 1 deltas, delta[p-2] <- init_dg, p - 1 copied */
  std::vector<double> delta_h(p);
  for (int k = 0; k < p - 1; k++) delta_h[k] = delta_file[k];
  delta_h[p - 1] = delta_h[p - 2];
  delta_h[p - 2] = init_dg;
  memcpy(Omega, Omega_in, sizeof(double) * N);
  memcpy(delta, delta_h.data(), sizeof(double) * (p - 1));
  memcpy(Xi, X_in, sizeof(double) * (size_t)N * Q);
  memcpy(Ta, T_in, sizeof(double) * (size_t)M * Q);
  memcpy(rho, rho_in, sizeof(double) * Q);

  ref_launch(gridNpMM, block1, [&] { getKernelMats(Q, Xi, Ta, rho, Z, K, Kinv, KinvKmn); });
  ref_launch(dim3(1), block1, [&] { cholKmm(M, Kinv); });
  ref_launch(gridN, blockN, [&] { getKinvKmn(Kinv, Z, KinvKmn, titsias); });
  ref_launch(dim3(1), block1, [&] { expandDelta_k(Z, delta, K, DeltaInv); });
  ref_launch(gridPP, block1, [&] { initPsi(Z, DeltaInv, Psi); });
  ref_launch(dim3(1), block1, [&] { initPsi2(P, Psi); });
  ref_launch(gridJ, block1, [&] { initBeta(Y, ls, Z, Psi, Work, Beta); });
  ref_launch(gridP, block1, [&] { vc::getZeta(J, P, Beta, phi, zeta); });

  int rhoflag = 0, itr, jtr;
  for (itr = 0; itr < itr_max; itr++) {
    const int JT = 30;
    for (jtr = 0; jtr < JT; jtr++) {
      ref_launch(gridJ, block1, [&] { vc::getWForBeta(Y, Z, ls, Beta, zeta, delta, titsias, W, Nu); });
      ref_launch(gridPsi, blockPsi, [&] { vc::getPsi(J, Z, Omega, DeltaInv, W, Psi); });
      ref_launch(gridJ, block1, [&] { vc::cholPsi(J, P, Psi); });
      ref_launch(gridJ, block1, [&] { vc::getBetaPhi(J, Z, ls, Psi, Omega, zeta, Nu, W, Work, Beta, phi); });
      ref_launch(gridP, block1, [&] { vc::getZeta(J, P, Beta, phi, zeta); });
      ref_launch(gridJ, block1, [&] { vc::getLkhdPois(Y, Z, W, delta, titsias, lkhds); });
      ref_launch(dim3(1), block1, [&] {
        vc::collectLkhd(0, J, 0, Omega, lkhds, itr, jtr, Z, delta, Xi, Ta, W, titsias, wt, lkhd_d);
      });
      lkhd_h[jtr] = lkhd_d[jtr];
      if (jtr > 0 && (jtr == (JT - 1) || fabs(lkhd_h[jtr - 1] - lkhd_h[jtr]) / fabs(lkhd_h[jtr]) < 1e-5)) break;
    }
    ref_launch(gridN, blockN, [&] { vc::getOinvt(N, J, Omega, W); });
    ref_launch(dim3(1), block1, [&] { vc::cholDeltaInv(P, DeltaInv); });
    ref_launch(gridJ, block1, [&] { vc::getLkhd(J, Z, Omega, DeltaInv, phi, Nu, Psi, W, Work, lkhds); });
    ref_launch(dim3(1), block1, [&] {
      vc::collectLkhd(N, J, Q, Omega, lkhds, itr, 0, Z, delta, Xi, Ta, W, titsias, wt, lkhd_d);
    });
    lkhd_h[0] = lkhd_d[0];
    if (itr > 10) rhoflag = 1;
    for (jtr = 0; jtr < lbfgs_max; jtr++) {
      ref_launch(dim3(1), block1, [&] { expandDelta_k(Z, delta, K, DeltaInv); });
      ref_launch(gridN, blockN, [&] { vc::getOinvt(N, J, Omega, W); });
      ref_launch(gridJ, block1, [&] { vc::getTildeBeta(J, Z, ls, Psi, Omega, Nu, W, Work, tBeta); });
      ref_launch(gridJP, block1, [&] {
        vc::getGradLogDelta(J, Z, DeltaInv, delta, K, Psi, tBeta, phi, Work, gradDeltaTmp);
      });
      ref_launch(gridDel, block1, [&] { vc::collectGradLogDelta(J, Z, delta, gradDeltaTmp, W, titsias, wt, grad); });
      ref_launch(dim3(1), block1, [&] {
        vc::LBFGS(jtr, Q, Z, Omega, delta, K, Xi, Ta, rho, grad, grad0, SS, XX, ss, Work, rhoflag);
      });
      double sr = 1.0;
      for (int ktr = 1; ktr < 8; ktr++) {
        ref_launch(gridN, blockN, [&] { vc::getOinvt(N, J, Omega, W); });
        ref_launch(gridNpMM, block1, [&] { getKernelMats(Q, Xi, Ta, rho, Z, K, Kinv, KinvKmn); });
        ref_launch(dim3(1), block1, [&] { expandDelta_k(Z, delta, K, DeltaInv); });
        ref_launch(dim3(1), block1, [&] { cholKmm(M, Kinv); });
        ref_launch(gridN, blockN, [&] { getKinvKmn(Kinv, Z, KinvKmn, titsias); });
        ref_launch(gridPsi, blockPsi, [&] { vc::getPsi(J, Z, Omega, DeltaInv, W, Psi); });
        ref_launch(gridJ, block1, [&] { vc::cholPsi(J, P, Psi); });
        ref_launch(dim3(1), block1, [&] { vc::cholDeltaInv(P, DeltaInv); });
        ref_launch(gridJ, block1, [&] { vc::getLkhd(J, Z, Omega, DeltaInv, phi, Nu, Psi, W, Work, lkhds); });
        ref_launch(dim3(1), block1, [&] {
          vc::collectLkhd(N, J, Q, Omega, lkhds, itr, jtr + 1, Z, delta, Xi, Ta, W, titsias, wt, lkhd_d);
        });
        for (int k = 0; k < jtr + 2; k++) lkhd_h[k] = lkhd_d[k];
        if (lkhd_h[jtr + 1] > lkhd_h[jtr] || ktr == 7) break;
        else if (std::isnan(lkhd_h[jtr + 1]) || std::isinf(lkhd_h[jtr + 1])) sr *= 0.01;
        else if (lkhd_h[jtr + 1] < lkhd_h[jtr]) sr *= 0.1;
        ref_launch(dim3(1), block1, [&] {
          vc::Downdate(jtr, Q, Z, Omega, delta, K, Xi, Ta, rho, grad, grad0, SS, XX, ss, sr, rhoflag);
        });
      }
      if (jtr > 0 && fabs(lkhd_h[jtr + 1] - lkhd_h[jtr]) < fabs(lkhd_h[jtr + 1]) * 1e-8) { jtr++; break; }
    }
    if (obj && itr < cap) obj[itr] = lkhd_h[jtr];
    ref_launch(dim3(1), block1, [&] { expandDelta_k(Z, delta, K, DeltaInv); });
    ref_launch(gridJ, dim3(1), [&] { vc::getBetaFromTildeBeta(J, Z, tBeta, zeta, Beta); });
    ref_launch(gridP, block1, [&] { vc::getZeta(J, P, Beta, phi, zeta); });
    if (dg && itr < cap) dg[itr] = delta[p - 2];
  }
  return itr;
}

}  // extern "C"
