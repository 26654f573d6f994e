// Per-cell placement at a fitted model: the plain method for a new cell's latent coordinates,
// the judge and the fallback of the amortised encoder (k_mlp.cu). It is the per-cell slice of the
// reference's L-BFGS phase (ggplvm.cu:1214-1301): with every gene's coefficients, the inducing
// points, the length-scales and the prior variances fixed at the fit, each cell's X_i is moved by
// its own L-BFGS with the reference's step rules (lbfgs, util_cuda.cu:187-232: memory 10, the
// first step -g/1e5, the two-loop recursion with scaling s.y / y.y, every coordinate clipped to
// [-1, 1]; the backtracking of ggplvm.cu:1278-1289: accept a rise or the 7th try, else shrink by
// 0.1, by 0.01 after a non-finite value; a non-finite 7th try is not accepted here).
//
// Per-cell objective: the Poisson log-probability of the cell's counts over all genes, with the
// mean of the IRLS's getLkhdPois (ggplvm.cu:703-724) and getWForBeta (ggplvm.cu:468-514), plus the
// N(0, 1) prior on the latent dimensions >= 1 that the reference's variance-component driver puts
// on X (ggplvm_delta.cu) and that keeps a single cell's problem bounded:
//     l_i(x) = sum_j [y_ij (eta_ij + log s_i) - W_ij - log(y_ij!)] - sum_{q >= 1} x_q^2 / 2,
//     eta_ij = z_i(x) . beta_j,  W_ij = s_i exp(eta_ij + wt delta_GP titsias_i(x)),
// where z_i(x) holds the cell's covariates and its kernel row k(x, T), and titsias_i =
// (1 - k^T Kmm^-1 k) / 2. Its gradient in x: d l / d Knm_ik = sum_j (y_ij - W_ij) beta_j[GP k]
// + wt delta_GP (sum_j W_ij) (Kmm^-1 k_i)_k, then through the periodic (dimension 0) and ARD
// kernels, minus x_q for q >= 1. All cells of a context are placed together; every cell keeps its
// own history, step and line search.
//
//   k_place_counts  the dense counts Y (cell x gene, cell fastest) from the CSR's matched prefix
//   k_place_resid   per cell over all genes: R = y - W (for the gradient GEMM), l_i and sum_j W
//   k_place_grad    per cell: d l / d x from G = R beta_GP^T (FFMA GEMM) and the kernel rows
//   k_place_dir     per cell: the L-BFGS step (on f = -l) and the trial point
//   k_place_accept  per cell: the line-search decision
#include <math.h>

#include <algorithm>
#include <vector>

#include "gpl_internal.cuh"

namespace gpl {

int launch_resid_gp(Ctx* c, const double* R, const double* B, double* G);  // k_gemm.cu

#define PLACE_RUN(expr)            \
  do {                             \
    const int rc_ = (expr);        \
    if (rc_ != GPL_OK) return rc_; \
  } while (0)

namespace {
constexpr int kMem = 10;  // L-BFGS memory (ggplvm.cu:872)

__global__ void k_place_counts(int ldN, const int32_t* __restrict__ cell, const int64_t* __restrict__ gptr,
                               const int32_t* __restrict__ gvalid, const double* __restrict__ cnt,
                               double* __restrict__ Y) {
  const int j = blockIdx.x;
  const int64_t b = gptr[j], e = gptr[j] + gvalid[j];
  for (int64_t l = b + threadIdx.x; l < e; l += blockDim.x) Y[(size_t)j * ldN + cell[l]] = cnt[l];
}

__global__ void k_place_resid(int N, int ldN, int J, int Q, int pvars, const double* __restrict__ E,
                              const double* __restrict__ Y, const double* __restrict__ ls,
                              const double* __restrict__ delta, const double* __restrict__ titsias,
                              const double* __restrict__ X, double* __restrict__ R, double* __restrict__ obj,
                              double* __restrict__ wsum) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double lsi = ls[i], lls = log(lsi), tt = delta[pvars - 1] * titsias[i] * kWt;
  double l = 0.0, ws = 0.0;
  for (int j = 0; j < J; j++) {
    const size_t e = (size_t)j * ldN + i;
    const double eta = E[e], y = Y[e];
    const double w = exp(eta) * lsi * exp(tt);
    if (R) R[e] = y - w;
    l += y * (eta + lls) - w;
    if (y > 0.0) l -= lgamma(y + 1.0);  // the full Poisson log-probability (constant in x)
    ws += w;
  }
  for (int q = 1; q < Q; q++) {  // N(0, 1) prior on the ARD dimensions
    const double x = X[i + (size_t)q * N];
    l -= 0.5 * x * x;
  }
  obj[i] = l;
  wsum[i] = ws;
}

// d l_i / d x_iq (stored as g[i + q N], the ascent direction of l)
__global__ void k_place_grad(int N, int ldN, int M, int Q, int pvars, const double* __restrict__ X,
                             const double* __restrict__ T, const double* __restrict__ rho,
                             const double* __restrict__ Knm, const double* __restrict__ KinvKmn,
                             const double* __restrict__ G, const double* __restrict__ wsum,
                             const double* __restrict__ delta, double* __restrict__ g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double tw = kWt * delta[pvars - 1] * wsum[i];
  double acc[16];
  for (int q = 0; q < Q; q++) acc[q] = 0.0;
  for (int k = 0; k < M; k++) {
    const double K = Knm[(size_t)k * ldN + i];
    const double C = (G[(size_t)k * ldN + i] + tw * KinvKmn[(size_t)k * ldN + i]) * K;
    acc[0] -= C * sin(X[i] - T[k]) / (2.0 * rho[0]);
    for (int q = 1; q < Q; q++) acc[q] -= C * (X[i + (size_t)q * N] - T[k + (size_t)q * M]) / rho[q];
  }
  for (int q = 1; q < Q; q++) acc[q] -= X[i + (size_t)q * N];  // the prior's gradient
  for (int q = 0; q < Q; q++) g[i + (size_t)q * N] = acc[q];
}

// The step of cell i on f = -l (gradient gf = -g): the first iteration -gf/1e5, then the two-loop
// recursion over the cell's history; every coordinate clipped to [-1, 1]. Backs up X_i and moves
// it to the trial point X_i + d.
__global__ void k_place_dir(int N, int Q, int it, double* __restrict__ X, const double* __restrict__ g,
                            const double* __restrict__ S, const double* __restrict__ Yh, double* __restrict__ X0,
                            double* __restrict__ d, double* __restrict__ sr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double q[16], z[16], a[kMem];
  for (int c = 0; c < Q; c++) q[c] = -g[i + (size_t)c * N];  // gradient of f
  const int nh = min(it, kMem);
  if (nh == 0) {
    for (int c = 0; c < Q; c++) z[c] = q[c] / 1e5;
  } else {
    for (int h = it - 1; h >= it - nh; h--) {
      const int s = h % kMem;
      double sq = 0.0, sy = 0.0;
      for (int c = 0; c < Q; c++) {
        const size_t e = ((size_t)s * Q + c) * N + i;
        sq += S[e] * q[c];
        sy += S[e] * Yh[e];
      }
      a[s] = sq / sy;
      for (int c = 0; c < Q; c++) q[c] -= a[s] * Yh[((size_t)s * Q + c) * N + i];
    }
    const int s0 = (it - 1) % kMem;
    double sy = 0.0, yy = 0.0;
    for (int c = 0; c < Q; c++) {
      const size_t e = ((size_t)s0 * Q + c) * N + i;
      sy += S[e] * Yh[e];
      yy += Yh[e] * Yh[e];
    }
    const double gam = sy / yy;
    for (int c = 0; c < Q; c++) z[c] = gam * q[c];
    for (int h = it - nh; h < it; h++) {
      const int s = h % kMem;
      double yz = 0.0, sy2 = 0.0;
      for (int c = 0; c < Q; c++) {
        const size_t e = ((size_t)s * Q + c) * N + i;
        yz += Yh[e] * z[c];
        sy2 += S[e] * Yh[e];
      }
      const double b = yz / sy2;
      for (int c = 0; c < Q; c++) z[c] += S[((size_t)s * Q + c) * N + i] * (a[s] - b);
    }
  }
  for (int c = 0; c < Q; c++) {
    double v = z[c];
    if (!(v == v)) v = 0.0;  // a degenerate history (s.y = 0) gives no step
    v = fmin(1.0, fmax(-1.0, v));
    const size_t e = i + (size_t)c * N;
    d[e] = -v;
    X0[e] = X[e];
    X[e] = X[e] - v;
  }
  sr[i] = 1.0;
}

// Line-search decision for cells still searching: accept a rise of l (or the 7th try); else
// shrink the step (x0.1, x0.01 after a non-finite value) and move to the new trial point. One
// departure from the reference's rule, for this per-cell use only: a 7th try whose value is not
// finite is not accepted; the cell goes back to the step's start, where the zero step that
// follows (a degenerate history gives no step) keeps it.
__global__ void k_place_accept(int N, int Q, int ktr, const double* __restrict__ f_new, const double* __restrict__ f_old,
                               double* __restrict__ X, const double* __restrict__ X0, const double* __restrict__ d,
                               double* __restrict__ sr, int* __restrict__ searching, int* __restrict__ n_open) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || !searching[i]) return;
  const double fn = f_new[i];
  if (fn > f_old[i] || ktr == 7) {
    if (!(fn > f_old[i]) && (isnan(fn) || isinf(fn)))
      for (int c = 0; c < Q; c++) X[i + (size_t)c * N] = X0[i + (size_t)c * N];
    searching[i] = 0;
    return;
  }
  sr[i] *= (isnan(fn) || isinf(fn)) ? 0.01 : 0.1;
  for (int c = 0; c < Q; c++) {
    const size_t e = i + (size_t)c * N;
    X[e] = X0[e] + sr[i] * d[e];
  }
  atomicAdd(n_open, 1);
}

// History after an accepted step: s = X - X0, y = gf_new - gf_old = -(g_new - g_old).
__global__ void k_place_hist(int N, int Q, int it, const double* __restrict__ X, const double* __restrict__ X0,
                             const double* __restrict__ g_new, const double* __restrict__ g_old,
                             double* __restrict__ S, double* __restrict__ Yh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int s = it % kMem;
  for (int c = 0; c < Q; c++) {
    const size_t e = i + (size_t)c * N, h = ((size_t)s * Q + c) * N + i;
    S[h] = X[e] - X0[e];
    Yh[h] = -(g_new[e] - g_old[e]);
  }
}

__global__ void k_fill_int(int n, int v, int* __restrict__ a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

struct PlaceBufs {
  double *X0 = nullptr, *d = nullptr, *g = nullptr, *g_old = nullptr, *S = nullptr, *Yh = nullptr;
  double *f = nullptr, *f_old = nullptr, *sr = nullptr, *wsum = nullptr;
  int *searching = nullptr, *n_open = nullptr;
  void release() {
    void* b[] = {X0, d, g, g_old, S, Yh, f, f_old, sr, wsum, searching, n_open};
    for (void* p : b)
      if (p) cudaFree(p);
  }
};

}  // namespace

// The objective of every cell at the X on the device (and, with `grad`, its gradient into pb.g).
static int place_eval(Ctx* c, PlaceBufs& pb, double* f, bool grad) {
  int rc = launch_kernel_mats(c);
  if (rc) return rc;
  if ((rc = launch_zbeta(c, c->Beta, c->scratch))) return rc;  // eta
  k_place_resid<<<div_up(c->N, 128), 128, 0, c->stream>>>(c->N, c->ldN, c->J, c->Q, c->p, c->scratch, c->Nu, c->ls,
                                                          c->delta, c->titsias, c->X, grad ? c->W : nullptr, f,
                                                          pb.wsum);
  GPL_LAUNCHED(c, "k_place_resid");
  if (!grad) return GPL_OK;
  if ((rc = launch_resid_gp(c, c->W, c->Beta, c->C1))) return rc;
  const double* Knm = c->Dm + (size_t)c->dg0 * c->ldN;
  k_place_grad<<<div_up(c->N, 128), 128, 0, c->stream>>>(c->N, c->ldN, c->M, c->Q, c->p, c->X, c->T, c->rho, Knm,
                                                         c->KinvKmn, c->C1, pb.wsum, c->delta, pb.g);
  GPL_LAUNCHED(c, "k_place_grad");
  return GPL_OK;
}

int place_cells(Ctx* c, int iters, double* X_host, double* obj_host, int32_t* stats) {
  const int N = c->N, Q = c->Q;
  if (Q > 16 || c->kernel_lv != kLvAll || c->de) {
    c->err = "placement needs Q <= 16 and the full GP model";
    return GPL_ERR_ARG;
  }
  PlaceBufs pb;
  const size_t nq = (size_t)N * Q;
  auto al = [&](auto** p, size_t n) {
    return cudaMalloc((void**)p, sizeof(**p) * (n ? n : 1)) == cudaSuccess;
  };
  if (!al(&pb.X0, nq) || !al(&pb.d, nq) || !al(&pb.g, nq) || !al(&pb.g_old, nq) || !al(&pb.S, nq * kMem) ||
      !al(&pb.Yh, nq * kMem) || !al(&pb.f, N) || !al(&pb.f_old, N) || !al(&pb.sr, N) || !al(&pb.wsum, N) ||
      !al(&pb.searching, N) || !al(&pb.n_open, 1)) {
    cudaGetLastError();
    pb.release();
    c->err = "device allocation failed: placement buffers";
    return GPL_ERR_ALLOC;
  }
  int rc = GPL_OK;
  int evals = 0, tries = 0;
  auto run = [&]() -> int {
    GPL_TRY(c, cudaMemcpyAsync(c->X, X_host, sizeof(double) * nq, cudaMemcpyHostToDevice, c->stream));
    // dense counts (Nu is not used by the placement otherwise)
    GPL_TRY(c, cudaMemsetAsync(c->Nu, 0, sizeof(double) * (size_t)c->ldN * c->J, c->stream));
    k_place_counts<<<c->J, 256, 0, c->stream>>>(c->ldN, c->cell, c->gptr, c->gvalid, c->cnt, c->Nu);
    GPL_LAUNCHED(c, "k_place_counts");
    PLACE_RUN(place_eval(c, pb, pb.f_old, true));
    evals++;
    const int nb = div_up(N, 128);
    for (int it = 0; it < iters; it++) {
      k_place_dir<<<nb, 128, 0, c->stream>>>(N, Q, it, c->X, pb.g, pb.S, pb.Yh, pb.X0, pb.d, pb.sr);
      GPL_LAUNCHED(c, "k_place_dir");
      k_fill_int<<<nb, 128, 0, c->stream>>>(N, 1, pb.searching);
      GPL_LAUNCHED(c, "k_fill_int");
      for (int ktr = 1; ktr < 8; ktr++) {
        PLACE_RUN(place_eval(c, pb, pb.f, false));
        evals++;
        tries++;
        GPL_TRY(c, cudaMemsetAsync(pb.n_open, 0, sizeof(int), c->stream));
        k_place_accept<<<nb, 128, 0, c->stream>>>(N, Q, ktr, pb.f, pb.f_old, c->X, pb.X0, pb.d, pb.sr, pb.searching,
                                                  pb.n_open);
        GPL_LAUNCHED(c, "k_place_accept");
        int open = 0;
        GPL_TRY(c, cudaMemcpyAsync(&open, pb.n_open, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        GPL_TRY(c, cudaStreamSynchronize(c->stream));
        if (open == 0) break;
      }
      GPL_TRY(c, cudaMemcpyAsync(pb.g_old, pb.g, sizeof(double) * nq, cudaMemcpyDeviceToDevice, c->stream));
      PLACE_RUN(place_eval(c, pb, pb.f_old, true));
      evals++;
      k_place_hist<<<nb, 128, 0, c->stream>>>(N, Q, it, c->X, pb.X0, pb.g, pb.g_old, pb.S, pb.Yh);
      GPL_LAUNCHED(c, "k_place_hist");
    }
    GPL_TRY(c, cudaMemcpyAsync(X_host, c->X, sizeof(double) * nq, cudaMemcpyDeviceToHost, c->stream));
    if (obj_host) GPL_TRY(c, cudaMemcpyAsync(obj_host, pb.f_old, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    GPL_TRY(c, cudaStreamSynchronize(c->stream));
    return GPL_OK;
  };
  rc = run();
  pb.release();
  if (stats) {
    stats[0] = iters;
    stats[1] = evals;
    stats[2] = tries;
  }
  return rc;
}

int cell_objective(Ctx* c, const double* X_host, double* obj_host, double* grad_host) {
  const int N = c->N;
  const size_t nq = (size_t)N * c->Q;
  if (c->Q > 16 || c->kernel_lv != kLvAll || c->de) {
    c->err = "placement needs Q <= 16 and the full GP model";
    return GPL_ERR_ARG;
  }
  PlaceBufs pb;
  if (cudaMalloc((void**)&pb.f, sizeof(double) * N) != cudaSuccess ||
      cudaMalloc((void**)&pb.wsum, sizeof(double) * N) != cudaSuccess ||
      (grad_host && cudaMalloc((void**)&pb.g, sizeof(double) * nq) != cudaSuccess)) {
    cudaGetLastError();
    pb.release();
    c->err = "device allocation failed: placement buffers";
    return GPL_ERR_ALLOC;
  }
  auto run = [&]() -> int {
    GPL_TRY(c, cudaMemcpyAsync(c->X, X_host, sizeof(double) * nq, cudaMemcpyHostToDevice, c->stream));
    GPL_TRY(c, cudaMemsetAsync(c->Nu, 0, sizeof(double) * (size_t)c->ldN * c->J, c->stream));
    k_place_counts<<<c->J, 256, 0, c->stream>>>(c->ldN, c->cell, c->gptr, c->gvalid, c->cnt, c->Nu);
    GPL_LAUNCHED(c, "k_place_counts");
    PLACE_RUN(place_eval(c, pb, pb.f, grad_host != nullptr));
    GPL_TRY(c, cudaMemcpyAsync(obj_host, pb.f, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    if (grad_host) GPL_TRY(c, cudaMemcpyAsync(grad_host, pb.g, sizeof(double) * nq, cudaMemcpyDeviceToHost, c->stream));
    GPL_TRY(c, cudaStreamSynchronize(c->stream));
    return GPL_OK;
  };
  const int rc = run();
  pb.release();
  return rc;
}

}  // namespace gpl
