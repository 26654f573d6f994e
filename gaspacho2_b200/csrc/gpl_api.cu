// C ABI of libgpl_b200: context management, data loading and the phase drivers that follow
// the reference driver's call order (ggplvm.cu:951-1354). See include/gpl.h.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "gpl_internal.cuh"

namespace gpl {

bool check(Ctx* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

ProfScope::ProfScope(Ctx* c_, const char* n) : c(c_), name(n) {
  if (!c->prof) return;
  if (c->event_pool.size() < 2) {
    for (int k = 0; k < 64; k++) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) == cudaSuccess) c->event_pool.push_back(e);
    }
  }
  if (c->event_pool.size() < 2) return;
  a = c->event_pool.back();
  c->event_pool.pop_back();
  b = c->event_pool.back();
  c->event_pool.pop_back();
  cudaEventRecord(a, c->stream);
}

ProfScope::~ProfScope() {
  if (!a) return;
  cudaEventRecord(b, c->stream);
  c->prof_pending.push_back({name, a, b});
  if (c->prof_pending.size() > 4096) {  // drain to bound the number of live events
    cudaEventSynchronize(b);
    for (auto& r : c->prof_pending) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, r.a, r.b);
      bool found = false;
      for (auto& t : c->prof_total)
        if (t.first == r.name) { t.second.first += ms; t.second.second++; found = true; break; }
      if (!found) c->prof_total.push_back({r.name, {ms, 1}});
      c->event_pool.push_back(r.a);
      c->event_pool.push_back(r.b);
    }
    c->prof_pending.clear();
  }
}

static void drain_profile(Ctx* c) {
  if (c->prof_pending.empty()) return;
  cudaEventSynchronize(c->prof_pending.back().b);
  for (auto& r : c->prof_pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    bool found = false;
    for (auto& t : c->prof_total)
      if (t.first == r.name) { t.second.first += ms; t.second.second++; found = true; break; }
    if (!found) c->prof_total.push_back({r.name, {ms, 1}});
    c->event_pool.push_back(r.a);
    c->event_pool.push_back(r.b);
  }
  c->prof_pending.clear();
}

template <class T>
static int dalloc(Ctx* c, T** p, size_t n, const char* what) {
  if (cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
    cudaGetLastError();
    c->err = std::string("device allocation failed: ") + what + " (" + std::to_string(sizeof(T) * n) + " bytes)";
    return GPL_ERR_ALLOC;
  }
  return GPL_OK;
}

static void free_state(Ctx* c) {
  tc_release(c);
  pair_release(c);
  void* extra[] = {c->cellfac, c->lvt, c->Dm, c->gsum, c->gT, c->HK, c->dcol_d, c->cv_nh_d, c->cv_nlev_d, c->gid_d, c->glev_d,
                   c->gcells_d, c->gstart_d, c->codes_d, c->hk_tiles_d, c->hk_tiles128_d, c->part, c->hk_cells_d,
                   c->lvl_cc_d, c->lvl_v_d, c->lvl_ptr_d, c->lvl_grp_d, c->hk_pos_d, c->Wg, c->Dg, c->rOmg,
                   c->gpos_d};
  for (void* q : extra)
    if (q) cudaFree(q);
  c->hk_tiles128_d = nullptr;
  c->hk_cells_d = nullptr;
  c->n_hk_tiles128 = 0;
  c->part = nullptr;
  c->part_n = 0;
  c->cellfac = c->lvt = c->Dm = c->gsum = c->gT = c->HK = nullptr;
  c->dcol_d = c->cv_nh_d = c->cv_nlev_d = c->gid_d = c->glev_d = c->gcells_d = c->gstart_d = c->codes_d = nullptr;
  c->lvl_cc_d = c->lvl_v_d = c->lvl_ptr_d = c->lvl_grp_d = c->hk_pos_d = nullptr;
  c->Wg = c->Dg = c->rOmg = nullptr;
  c->gpos_d = nullptr;
  c->n_lvl = 0;
  c->hk_tiles_d = nullptr;
  c->n_grp = c->n_cv = 0;
  void* bufs[] = {c->Z,      c->W,      c->Nu,      c->Psi,     c->PsiInv, c->Beta,   c->tBeta,  c->scratch,
                  c->U,      c->Kmm,    c->Kinv,    c->KinvKmn, c->titsias, c->DeltaInv, c->Omega, c->delta,
                  c->X,      c->T,      c->rho,     c->phi,     c->ls,     c->lkhds,  c->lkhd_dev, c->grad,
                  c->grad0,  c->ss,     c->SS,      c->XX,      c->gdtmp,  c->C1,     c->C2,     c->grtmp,
                  c->KmmInv, c->bvec,   c->sol,     c->red,     c->lb_work, c->mc_d,  c->mv_d,   c->mk_d,
                  c->nh_d,   c->rres,   c->bx,      c->rphi,    c->e0,      c->zeta};
  for (void* p : bufs)
    if (p) cudaFree(p);
  c->Z = c->W = c->Nu = c->Psi = c->PsiInv = c->Beta = c->tBeta = c->scratch = c->U = nullptr;
  c->Kmm = c->Kinv = c->KinvKmn = c->titsias = c->DeltaInv = c->Omega = c->delta = c->X = c->T = nullptr;
  c->rho = c->phi = c->ls = c->lkhds = c->lkhd_dev = c->grad = c->grad0 = c->ss = c->SS = c->XX = nullptr;
  c->gdtmp = c->C1 = c->C2 = c->grtmp = c->KmmInv = c->bvec = c->sol = c->red = c->lb_work = nullptr;
  c->mc_d = c->mv_d = c->mk_d = c->nh_d = nullptr;
  c->rres = c->bx = c->rphi = c->e0 = c->zeta = nullptr;
  c->have_design = false;
}

static void free_counts(Ctx* c) {
  if (c->gene_order_d) cudaFree(c->gene_order_d);
  if (c->queue_head_d) cudaFree(c->queue_head_d);
  c->gene_order_d = c->queue_head_d = nullptr;
  if (c->cell) cudaFree(c->cell);
  if (c->gptr) cudaFree(c->gptr);
  if (c->gvalid) cudaFree(c->gvalid);
  if (c->cnt) cudaFree(c->cnt);
  c->cell = nullptr;
  c->gptr = nullptr;
  c->gvalid = nullptr;
  c->cnt = nullptr;
  c->have_counts = false;
}

static int need_state(Ctx* c) {
  if (!c->have_counts || !c->have_design) {
    c->err = "counts and design must be loaded first";
    return GPL_ERR_STATE;
  }
  return GPL_OK;
}

#define GPL_RUN(expr)          \
  do {                         \
    int rc_ = (expr);          \
    if (rc_ != GPL_OK) return rc_; \
  } while (0)

static int read_slot(Ctx* c, int slot, double* out) {
  double v = 0.0;
  GPL_TRY(c, cudaMemcpyAsync(&v, c->lkhd_dev + slot, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  GPL_RUN(tc_error_flag(c));
  tune_harvest(c);
  c->lkhd[slot] = v;
  if (out) *out = v;
  return GPL_OK;
}

// ---- phases -------------------------------------------------------------------------------
// With the fused tail (FP64, the main driver's forms), Z^T diag(W/Omega) nu comes first (it does
// not read the factor) and one persistent launch does every gene's Cholesky, solve, coefficient
// update and Poisson likelihood; the results are the same bits as the separate kernels'.
static int irls_sweep(Ctx* c, int jtr, double* lk) {
  GPL_RUN(launch_w_nu(c));
  GPL_RUN(launch_gram(c, false));
  bool fused = false;
  if (c->fused_tail && c->precision == GPL_PREC_FP64 && !c->de) {
    GPL_RUN(launch_zt_u(c, 0));
    const int rc = launch_irls_tail(c, jtr, c->tail_ctas_per_sm);
    if (rc != GPL_OK && rc != GPL_ERR_ARG) return rc;
    fused = rc == GPL_OK;
    if (!fused) GPL_RUN(launch_chol_batched(c, c->Psi, c->P, c->J, (int64_t)c->P * c->P));
  } else {
    GPL_RUN(launch_chol_batched(c, c->Psi, c->P, c->J, (int64_t)c->P * c->P));
    GPL_RUN(launch_zt_u(c, 0));
  }
  if (!fused) {
    GPL_RUN(launch_beta_phi(c, jtr));
    GPL_RUN(launch_lkhd_pois(c));
  }
  GPL_RUN(launch_collect_lkhd(c, 0, jtr));
  return read_slot(c, jtr, lk);
}

static int irls(Ctx* c, int jtr_max, int* n_sweeps) {
  int jtr;
  for (jtr = 0; jtr < jtr_max; jtr++) {
    GPL_RUN(irls_sweep(c, jtr, nullptr));
    if (jtr > 0) {
      const double a = c->lkhd[jtr - 1], b = c->lkhd[jtr];
      if (isnan(b)) {
        if (n_sweeps) *n_sweeps = jtr + 1;
        c->err = "IRLS likelihood is NaN";
        return GPL_ERR_NAN;
      }
      if (jtr == jtr_max - 1 || fabs(a - b) / fabs(b) < 1e-7) {
        jtr++;
        break;
      }
    }
  }
  if (n_sweeps) *n_sweeps = jtr;
  return GPL_OK;
}

static int objective_after_irls(Ctx* c, double* lk) {
  GPL_RUN(launch_oinvt(c));
  GPL_RUN(launch_chol_single(c, c->DeltaInv, c->P));
  GPL_RUN(launch_zt_u(c, 0));
  GPL_RUN(launch_lkhd_genes(c));
  GPL_RUN(launch_collect_lkhd(c, c->N, 0));
  return read_slot(c, 0, lk);
}

static int objective_launch(Ctx* c, int slot) {
  GPL_RUN(launch_oinvt(c));
  GPL_RUN(launch_kernel_mats(c));
  GPL_RUN(launch_expand_delta(c));
  GPL_RUN(launch_gram(c, false));
  GPL_RUN(launch_chol_batched(c, c->Psi, c->P, c->J, (int64_t)c->P * c->P));
  GPL_RUN(launch_chol_single(c, c->DeltaInv, c->P));
  GPL_RUN(launch_zt_u(c, 0));
  GPL_RUN(launch_lkhd_genes(c));
  GPL_RUN(launch_collect_lkhd(c, c->N, slot));
  return GPL_OK;
}

// after_objective: the objective was just evaluated at this state (objective_launch or
// objective_after_irls), so Oinvt is current and getTildeBeta's solve Psi_j x = Z^T diag(W/Omega)
// nu_j (ggplvm.cu:406-414) is the one getLkhd already made with the same factor and right-hand
// side (ggplvm.cu:744-784): tilde-beta is that solution, copied instead of solved again.
static int gradient_launch(Ctx* c, bool after_objective = false) {
  GPL_RUN(launch_expand_delta(c));
  if (after_objective) {
    GPL_TRY(c, cudaMemcpyAsync(c->tBeta, c->sol, sizeof(double) * (size_t)c->P * c->J, cudaMemcpyDeviceToDevice,
                               c->stream));
  } else {
    GPL_RUN(launch_oinvt(c));
    GPL_RUN(launch_zt_u(c, 0));
    GPL_RUN(solve_refined(c, c->bvec, c->tBeta));
  }
  GPL_RUN(launch_inverse_batched(c));
  GPL_RUN(launch_grad_delta(c));
  GPL_RUN(launch_grad_omega(c));
  GPL_RUN(launch_c2(c));
  GPL_RUN(launch_grad_tau_rho(c));
  return GPL_OK;
}

// ---- evaluations as CUDA graphs ----------------------------------------------------------------
// The objective (about 40 launches) and the gradient after it (about 100) are captured once into
// graphs and replayed: one launch each instead of one per kernel, and no host work per kernel in
// the L-BFGS loop. The objective graph writes its value to a fixed slot, copied on the device to
// the slot the caller asked for. Capture needs every lazily sized buffer to exist already, so the
// first call runs eagerly and captures afterwards; if capture is refused (a call that a captured
// stream does not allow), the context stays eager and says why in graph_note.
constexpr int kGraphSlot = kLkhdSlots - 1;

void graph_reset(Ctx* c) {
  if (c->g_obj) cudaGraphExecDestroy(c->g_obj);
  if (c->g_grad) cudaGraphExecDestroy(c->g_grad);
  c->g_obj = c->g_grad = nullptr;
}

static bool graph_ok(const Ctx* c) {
  return c->use_graph && !c->prof && !c->tc_check && (!c->autotune || tune_settled_for_graphs(c));
}

template <class F>
static int capture(Ctx* c, cudaGraphExec_t* out, int64_t* n_kernels, F body) {
  cudaGraph_t g = nullptr;
  const int64_t l0 = c->launches;
  GPL_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  c->capturing = true;
  const int rc = body();
  c->capturing = false;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  *n_kernels = c->launches - l0;
  c->launches = l0;  // captured, not run
  if (rc != GPL_OK || e != cudaSuccess || g == nullptr) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    if (rc != GPL_OK) return rc;
    c->use_graph = false;
    c->graph_note = std::string("stream capture refused: ") + cudaGetErrorString(e);
    return GPL_OK;
  }
  const cudaError_t ei = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    c->use_graph = false;
    c->graph_note = std::string("graph instantiation failed: ") + cudaGetErrorString(ei);
  }
  return GPL_OK;
}

// objective_launch(c, slot), through the objective graph when graphs are on.
static int objective_run(Ctx* c, int slot) {
  if (!graph_ok(c)) return objective_launch(c, slot);
  if (!c->g_obj) {
    GPL_RUN(objective_launch(c, slot));
    return capture(c, &c->g_obj, &c->g_obj_kernels, [&] { return objective_launch(c, kGraphSlot); });
  }
  GPL_TRY(c, cudaGraphLaunch(c->g_obj, c->stream));
  c->launches += c->g_obj_kernels;
  c->graph_replays++;
  if (slot != kGraphSlot)
    GPL_TRY(c, cudaMemcpyAsync(c->lkhd_dev + slot, c->lkhd_dev + kGraphSlot, sizeof(double),
                               cudaMemcpyDeviceToDevice, c->stream));
  return GPL_OK;
}

// gradient_launch(c, true) (the gradient at the point of the last objective), through the
// gradient graph when graphs are on.
static int gradient_run(Ctx* c) {
  if (!graph_ok(c)) return gradient_launch(c, true);
  if (!c->g_grad) {
    GPL_RUN(gradient_launch(c, true));
    return capture(c, &c->g_grad, &c->g_grad_kernels, [&] { return gradient_launch(c, true); });
  }
  GPL_TRY(c, cudaGraphLaunch(c->g_grad, c->stream));
  c->launches += c->g_grad_kernels;
  c->graph_replays++;
  return GPL_OK;
}

// One outer iteration `itr` of the driver (ggplvm.cu:1146-1330): IRLS to convergence
// (JTRMAX 200 on the first iteration, 100 after), the objective, then L-BFGS steps with the
// backtracking line search (rhoflag once itr > 20; a 10000-step limit on itr 30), and the
// beta revival. lbfgs_budget > 0 caps the L-BFGS steps of this call. st = IRLS sweeps,
// L-BFGS steps, objective evaluations, trace entries written.
// The FP64 repeat of a precision-form line search that failed (option ls_fp64): back to the step's
// start, the FP64 objective there, the same backtracking rules against it, then the precision
// form's objective at the accepted point into slot jtr + 1 (the next step's comparison and the
// gradient's state). When the FP64 search finds no rise either, the parameters go back to the
// step's start. *evals = the objective evaluations made, negative in that case.
static int ls_fp64_retry(Ctx* c, int jtr, int rhoflag, int* evals) {
  std::vector<double>& l = c->lkhd;
  int n = 0;
  c->precision = GPL_PREC_FP64;
  graph_reset(c);
  GPL_RUN(launch_downdate(c, jtr, 0.0, rhoflag));  // the step's start
  GPL_RUN(objective_run(c, jtr + 1));
  GPL_RUN(read_slot(c, jtr + 1, nullptr));
  n++;
  const double l0 = l[jtr + 1];
  double sr = 1.0;
  bool rose = false;
  for (int ktr = 1; ktr < 8; ktr++) {
    GPL_RUN(launch_downdate(c, jtr, sr, rhoflag));
    GPL_RUN(objective_run(c, jtr + 1));
    GPL_RUN(read_slot(c, jtr + 1, nullptr));
    n++;
    if (l[jtr + 1] > l0) {
      rose = true;
      break;
    }
    if (ktr == 7) break;
    if (isnan(l[jtr + 1]) || isinf(l[jtr + 1])) sr *= 0.01;
    else sr *= 0.1;
  }
  if (!rose) GPL_RUN(launch_downdate(c, jtr, 0.0, rhoflag));  // no rise either: back to the start
  c->precision = GPL_PREC_BF16X3;
  graph_reset(c);
  GPL_RUN(objective_run(c, jtr + 1));
  GPL_RUN(read_slot(c, jtr + 1, nullptr));
  n++;
  c->ls_fp64_steps++;
  *evals = rose ? n : -n;
  return GPL_OK;
}

static int fit_outer(Ctx* c, int itr, int lbfgs_budget, int32_t* st, double* trace, int trace_cap) {
  int JTRMAX = (itr == 0) ? 200 : 100;
  int n = 0, ntrace = 0;
  int rc = irls(c, JTRMAX, &n);
  st[0] = n;
  if (rc) return rc;
  double l0 = 0.0;
  GPL_RUN(objective_after_irls(c, &l0));
  st[2]++;
  if (trace && ntrace < trace_cap) trace[ntrace++] = l0;
  const int rhoflag = itr > 20 ? 1 : 0;
  if (itr == 30) JTRMAX = 10000;
  // option ls_fp64 (precision form only): a line search whose seven tries all fail is repeated
  // with the FP64 objective (the tensor-core Gram resolves parameter changes only to about 2^-16
  // relative, so a short step's gain can be invisible to it); the fit then goes on in the
  // precision form from the point the FP64 search accepted
  const bool fp64_retry = c->ls_fp64 && c->precision == GPL_PREC_BF16X3;
  for (int jtr = 0; jtr < JTRMAX && jtr + 1 < kLkhdSlots; jtr++) {
    GPL_RUN(gradient_run(c));  // the last objective (after the IRLS or the accepted step) is here
    GPL_RUN(launch_lbfgs_update(c, jtr, rhoflag));
    double sr = 1.0;
    std::vector<double>& l = c->lkhd;
    for (int ktr = 1; ktr < 8; ktr++) {
      GPL_RUN(objective_run(c, jtr + 1));
      GPL_RUN(read_slot(c, jtr + 1, nullptr));
      st[2]++;
      if (l[jtr + 1] > l[jtr] || ktr == 7) break;
      else if (isnan(l[jtr + 1]) || isinf(l[jtr + 1])) sr *= 0.01;
      else if (l[jtr + 1] < l[jtr]) sr *= 0.1;
      GPL_RUN(launch_downdate(c, jtr, sr, rhoflag));
    }
    st[1]++;
    bool retried = false;
    if (fp64_retry && !(l[jtr + 1] > l[jtr])) {
      int rs = 0;
      GPL_RUN(ls_fp64_retry(c, jtr, rhoflag, &rs));
      st[2] += rs > 0 ? rs : -rs;
      retried = rs > 0;  // the FP64 search found a rise
      if (!retried) {    // it did not either: the reference's stop
        if (trace && ntrace < trace_cap) trace[ntrace++] = l[jtr + 1];
        break;
      }
    }
    if (trace && ntrace < trace_cap) trace[ntrace++] = l[jtr + 1];
    if (!retried && jtr > 0 && fabs(l[jtr + 1] - l[jtr]) < fabs(l[jtr + 1]) * 1e-8) break;
    if (lbfgs_budget > 0 && st[1] >= lbfgs_budget) break;
  }
  GPL_RUN(launch_expand_delta(c));
  GPL_RUN(launch_beta_from_tilde(c));
  st[3] = ntrace;
  return GPL_OK;
}

static int glm_init(Ctx* c) {
  GPL_RUN(launch_expand_delta(c));
  GPL_RUN(launch_gram(c, true));
  GPL_RUN(launch_chol_single(c, c->Psi, c->P));
  GPL_RUN(launch_init_response(c));
  GPL_RUN(launch_zt_u(c, 1));
  GPL_RUN(launch_init_beta_solve(c));
  return GPL_OK;
}

// One model of the DE driver (ggplvm_de.cu:1071-1104 for the null model, 1135-1177 for the
// others): GLM initialisation, zeta, then IRLS sweeps in the DE forms with its stopping rule.
// The summed likelihood is read back after every sweep, as the reference does.
static int de_irls(Ctx* c, int jtr_max, double tol, int* n_sweeps, double* trace, int trace_cap) {
  GPL_RUN(glm_init(c));
  GPL_RUN(launch_de_zeta(c));
  const int64_t PP = (int64_t)c->P * c->P;
  double prev = 0.0;
  int jtr;
  for (jtr = 0; jtr < jtr_max; jtr++) {
    GPL_RUN(launch_w_nu(c));
    GPL_RUN(launch_gram(c, false));
    GPL_RUN(launch_chol_batched(c, c->Psi, c->P, c->J, PP));
    GPL_RUN(launch_zt_u(c, 0));
    GPL_RUN(launch_de_beta_phi(c));
    GPL_RUN(launch_de_zeta(c));
    GPL_RUN(launch_de_lkhd(c, 0));
    double cur = 0.0;
    GPL_RUN(read_slot(c, 0, &cur));
    if (trace && jtr < trace_cap) trace[jtr] = cur;
    if (jtr > 0) {
      if (isinf(cur) || isnan(cur) || jtr == jtr_max - 1 || fabs(prev - cur) / fabs(cur) < tol) {
        jtr++;
        break;
      }
    }
    prev = cur;
  }
  *n_sweeps = jtr;
  return GPL_OK;
}

// ---- the variance-component driver (ggplvm_delta.cu) ------------------------------------------
// Host state of its one-variable L-BFGS (LBFGS, Downdate: ggplvm_delta.cu:707-782): the step
// history S, the gradient-change history Y (10 slots), the current step and the backup of
// delta[p-2].
struct VcLbfgs {
  double S[10] = {0}, Y[10] = {0}, ss = 0.0, g0 = 0.0, backup = 0.0;
};

// lbfgs (util_cuda.cu:187-232) for one variable: the two-loop recursion over the history, the
// initial scaling s.y / y.y, the clamp to [-1, 1] and the sign flip.
static double lbfgs_scalar(const VcLbfgs& h, double g, int itr) {
  const int m = 10, pt = (itr - 1) % m, lo = itr > m ? pt - m + 1 : 0;
  double a[10], q = g;
  for (int i = pt; i >= lo; i--) {
    const int ii = (i + m) % m;
    a[ii] = (0.0 + h.S[ii] * q) / (0.0 + h.S[ii] * h.Y[ii]);
    q -= a[ii] * h.Y[ii];
  }
  double z = (0.0 + h.S[pt] * h.Y[pt]) / (0.0 + h.Y[pt] * h.Y[pt]) * q;
  for (int i = lo; i <= pt; i++) {
    const int ii = (i + m) % m;
    z += h.S[ii] * (a[ii] - (0.0 + h.Y[ii] * z) / (0.0 + h.S[ii] * h.Y[ii]));
  }
  if (z > 1.0) z = 1.0;
  if (z < (-1.0)) z = -1.0;
  return -z;
}

static int set_delta_dg(Ctx* c, double v) {
  GPL_TRY(c, cudaMemcpyAsync(c->delta + (c->p - 2), &v, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  return GPL_OK;
}

// The driver's loop (ggplvm_delta.cu:962-1097) from the parameters set: per outer iteration an
// IRLS phase in the DE driver's forms (at most 30 sweeps, relative change 1e-5), the Laplace
// objective, then L-BFGS on log delta[p-2] with the backtracking line search (at most
// lbfgs_max steps, relative change 1e-8), and beta = tilde-beta + zeta. The gradient is only
// the delta block (getTildeBeta, getGradLogDelta, collectGradLogDelta); the reference's
// one-variable lbfgs reads grad[0], the gradient of log delta[0], as its current gradient
// while its history holds delta[p-2]'s steps and gradient changes, and so does this one.
static int vc_fit(Ctx* c, int itr_max, int lbfgs_max, double* dg, double* obj, int cap, int* n_itr) {
  const int p = c->p, N = c->N;
  const int64_t PP = (int64_t)c->P * c->P;
  GPL_RUN(launch_kernel_mats(c));
  GPL_RUN(glm_init(c));
  GPL_RUN(launch_de_zeta(c));
  VcLbfgs h;
  double dgv = 0.0;
  GPL_TRY(c, cudaMemcpy(&dgv, c->delta + (p - 2), sizeof(double), cudaMemcpyDeviceToHost));
  std::vector<double> l((size_t)lbfgs_max + 2, 0.0);
  int itr;
  for (itr = 0; itr < itr_max; itr++) {
    double prev = 0.0;
    for (int jtr = 0; jtr < 30; jtr++) {
      GPL_RUN(launch_w_nu(c));
      GPL_RUN(launch_gram(c, false));
      GPL_RUN(launch_chol_batched(c, c->Psi, c->P, c->J, PP));
      GPL_RUN(launch_zt_u(c, 0));
      GPL_RUN(launch_de_beta_phi(c));
      GPL_RUN(launch_de_zeta(c));
      GPL_RUN(launch_lkhd_pois(c));
      GPL_RUN(launch_collect_lkhd(c, 0, 0));
      double cur = 0.0;
      GPL_RUN(read_slot(c, 0, &cur));
      if (jtr > 0 && (jtr == 29 || fabs(prev - cur) / fabs(cur) < 1e-5)) break;
      prev = cur;
    }
    GPL_RUN(objective_after_irls(c, &l[0]));
    int jtr;
    for (jtr = 0; jtr < lbfgs_max; jtr++) {
      GPL_RUN(launch_expand_delta(c));
      GPL_RUN(launch_oinvt(c));
      GPL_RUN(launch_zt_u(c, 0));
      GPL_RUN(solve_refined(c, c->bvec, c->tBeta));
      GPL_RUN(launch_inverse_batched(c));
      GPL_RUN(launch_grad_delta(c));
      double g[2];  // d/dlog delta[0] and d/dlog delta[p-2]
      GPL_TRY(c, cudaMemcpyAsync(&g[0], c->grad + N, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      GPL_TRY(c, cudaMemcpyAsync(&g[1], c->grad + N + (p - 2), sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      GPL_TRY(c, cudaStreamSynchronize(c->stream));
      // LBFGS (ggplvm_delta.cu:734-782)
      const int pt = (jtr - 1) % 10, ptp1 = jtr % 10;
      if (jtr == 0) {
        h.ss = -g[1] / 10000.0;
        if (h.ss > 1.0) h.ss = 0.01;
        if (h.ss < (-1.0)) h.ss = -0.01;
      } else {
        h.Y[pt] = g[1] - h.g0;
        h.ss = lbfgs_scalar(h, g[0], jtr);
      }
      h.g0 = g[1];
      h.backup = dgv;
      dgv = exp(log(dgv) - h.ss);
      h.S[ptp1] = h.ss;
      GPL_RUN(set_delta_dg(c, dgv));
      double sr = 1.0;
      for (int ktr = 1; ktr < 8; ktr++) {
        GPL_RUN(objective_launch(c, 1));
        GPL_RUN(read_slot(c, 1, &l[jtr + 1]));
        if (l[jtr + 1] > l[jtr] || ktr == 7) break;
        else if (isnan(l[jtr + 1]) || isinf(l[jtr + 1])) sr *= 0.01;
        else if (l[jtr + 1] < l[jtr]) sr *= 0.1;
        // Downdate (ggplvm_delta.cu:707-731)
        dgv = exp(log(h.backup) - sr * h.ss);
        h.S[ptp1] = sr * h.ss;
        GPL_RUN(set_delta_dg(c, dgv));
      }
      if (jtr > 0 && fabs(l[jtr + 1] - l[jtr]) < fabs(l[jtr + 1]) * 1e-8) {
        jtr++;
        break;
      }
    }
    if (obj && itr < cap) obj[itr] = l[jtr];
    GPL_RUN(launch_expand_delta(c));
    GPL_RUN(launch_beta_from_tilde(c));
    GPL_RUN(launch_de_zeta(c));
    if (dg && itr < cap) dg[itr] = dgv;
  }
  *n_itr = itr;
  return GPL_OK;
}

// The reference's loader leaves 199.0 in the first cell of the last design variable of a
// design without GP (DataFrame.cu:112-113, 131): the null model sees it, the GP models do not.
static int de_loader_value(Ctx* c, bool on) {
  if (on && c->de_quirk_col < 0) {
    const int v = c->p - 2;  // last design variable (the intercept when there is none)
    if (c->vc[v] != 1) return GPL_OK;  // categorical: the reference reads out of range
    const int col = c->nh[v];
    int d = -1;
    for (int a = 0; a < c->n_d; a++)
      if (c->dcol[a] == col) d = a;
    if (d < 0) return GPL_OK;
    double* cell0 = c->Dm + (size_t)d * c->ldN;
    GPL_TRY(c, cudaMemcpyAsync(&c->de_quirk_orig, cell0, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GPL_TRY(c, cudaStreamSynchronize(c->stream));
    const double v199 = 199.0;
    GPL_TRY(c, cudaMemcpyAsync(cell0, &v199, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    GPL_TRY(c, cudaStreamSynchronize(c->stream));
    c->de_quirk_col = d;
  } else if (!on && c->de_quirk_col >= 0) {
    double* cell0 = c->Dm + (size_t)c->de_quirk_col * c->ldN;
    GPL_TRY(c, cudaMemcpyAsync(cell0, &c->de_quirk_orig, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    GPL_TRY(c, cudaStreamSynchronize(c->stream));
    c->de_quirk_col = -1;
  }
  return GPL_OK;
}

}  // namespace gpl

using namespace gpl;

static Ctx* C(gpl_ctx* h) { return &h->c; }

extern "C" {

int gpl_create(gpl_ctx** out, int device, void* stream) {
  if (!out) return GPL_ERR_ARG;
  *out = nullptr;
  gpl_ctx* h = new (std::nothrow) gpl_ctx();
  if (!h) return GPL_ERR_ALLOC;
  Ctx* c = C(h);
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return GPL_ERR_CUDA;
  }
  if (stream) {
    c->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete h;
      return GPL_ERR_CUDA;
    }
    c->own_stream = true;
  }
  c->lkhd.assign(kLkhdSlots, 0.0);
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && nsm > 0)
    c->sm_count = nsm;
  *out = h;
  return GPL_OK;
}

int gpl_destroy(gpl_ctx* h) {
  if (!h) return GPL_OK;
  Ctx* c = C(h);
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  graph_reset(c);
  tune_release(c);
  drain_profile(c);
  for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
  free_state(c);
  free_counts(c);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete h;
  return GPL_OK;
}

const char* gpl_last_error(const gpl_ctx* h) { return h ? h->c.err.c_str() : "null context"; }

int gpl_set_precision(gpl_ctx* h, int precision) {
  Ctx* c = C(h);
  if (precision != GPL_PREC_FP64 && precision != GPL_PREC_BF16X3) {
    c->err = "unknown precision";
    return GPL_ERR_ARG;
  }
  if (precision != c->precision) graph_reset(c);
  c->precision = precision;
  return GPL_OK;
}

int gpl_set_option(gpl_ctx* h, const char* name, int64_t value) {
  if (!h || !name) return GPL_ERR_ARG;
  Ctx* c = C(h);
  const std::string s(name);
  graph_reset(c);  // the captured graphs hold the old option's launches
  if (s == "tc_grad") {
    c->tc_grad = value != 0;
  } else if (s == "refine_steps") {
    if (value < 0 || value > 16) { c->err = "refine_steps must be in 0..16"; return GPL_ERR_ARG; }
    c->refine_steps = (int)value;
  } else if (s == "tc_run") {
    if (value < 1 || value > 64) { c->err = "tc_run must be in 1..64"; return GPL_ERR_ARG; }
    c->tc_run = (int)value;
    c->tc.run = (int)value;
  } else if (s == "tc_check") {
    c->tc_check = value != 0;
  } else if (s == "tc_pair") {
    c->tc_pair = value != 0;
  } else if (s == "ls_fp64") {
    c->ls_fp64 = value != 0;
  } else if (s == "logdet_probe") {
    c->logdet_probe = value != 0;
  } else if (s == "autotune") {
    c->autotune = value != 0;
  } else if (s == "fused_tail") {
    c->fused_tail = value != 0;
  } else if (s == "eta_tc") {
    c->eta_tc = value != 0;
  } else if (s == "tail_ctas_per_sm") {
    if (value < 1 || value > 2) { c->err = "tail_ctas_per_sm must be 1 or 2"; return GPL_ERR_ARG; }
    c->tail_ctas_per_sm = (int)value;
  } else if (s == "graph") {
    c->use_graph = value != 0;
    c->graph_note.clear();
  } else if (s == "pair_range_cells") {
    if (value < 0) { c->err = "pair_range_cells must be >= 0"; return GPL_ERR_ARG; }
    if (value != c->pair_range_cells) {
      GPL_TRY(c, cudaStreamSynchronize(c->stream));
      pair_release(c);  // the range size fixes the buffers: sized again on next use
    }
    c->pair_range_cells = value;
  } else {
    c->err = "unknown option: " + s;
    return GPL_ERR_ARG;
  }
  return GPL_OK;
}

int gpl_get_option(const gpl_ctx* h, const char* name, int64_t* value) {
  if (!h || !name || !value) return GPL_ERR_ARG;
  const Ctx* c = &h->c;
  const std::string s(name);
  if (s == "tc_grad") *value = c->tc_grad ? 1 : 0;
  else if (s == "refine_steps") *value = c->refine_steps;
  else if (s == "tc_run") *value = c->tc_run;
  else if (s == "tc_check") *value = c->tc_check ? 1 : 0;
  else if (s == "tc_pair") *value = c->tc_pair ? 1 : 0;
  else if (s == "ls_fp64") *value = c->ls_fp64 ? 1 : 0;
  else if (s == "ls_fp64_steps") *value = c->ls_fp64_steps;
  else if (s == "logdet_probe") *value = c->logdet_probe ? 1 : 0;
  else if (s == "pair_range_cells") *value = c->pair_range_cells;
  else if (s == "graph") *value = c->use_graph ? 1 : 0;
  else if (s == "fused_tail") *value = c->fused_tail ? 1 : 0;
  else if (s == "eta_tc") *value = c->eta_tc ? 1 : 0;
  else if (s == "autotune") *value = c->autotune ? 1 : 0;
  else if (s == "tail_ctas_per_sm") *value = c->tail_ctas_per_sm;
  else if (s == "graph_replays") *value = c->graph_replays;
  else return GPL_ERR_ARG;
  return GPL_OK;
}

int gpl_load_counts(gpl_ctx* h, int N, int J, int64_t nnz, const int32_t* cell_idx, const int32_t* gene_ptr,
                    const double* counts) {
  Ctx* c = C(h);
  cudaSetDevice(c->device);
  if (N <= 0 || J <= 0 || nnz < 0 || !gene_ptr || (nnz > 0 && (!cell_idx || !counts))) {
    c->err = "bad counts arguments";
    return GPL_ERR_ARG;
  }
  if (c->have_design && (N != c->N || J != c->J)) {
    c->err = "counts sizes differ from the loaded design";
    return GPL_ERR_ARG;
  }
  std::vector<int64_t> gp(J + 1);
  std::vector<int32_t> gv(J);
  for (int j = 0; j <= J; j++) gp[j] = gene_ptr[j];
  for (int j = 0; j < J; j++) {
    if (gp[j] < 0 || gp[j] > gp[j + 1] || gp[j + 1] > nnz) {
      c->err = "gene offsets are not monotone within [0, nnz]";
      return GPL_ERR_FORMAT;
    }
    // entries the reference's merge walk consumes (ggplvm.cu:505-511)
    int last = -1;
    int64_t l = gp[j];
    for (; l < gp[j + 1]; l++) {
      const int i = cell_idx[l];
      if (i <= last || i >= N) break;
      last = i;
    }
    gv[j] = (int32_t)(l - gp[j]);
  }
  free_counts(c);
  GPL_RUN(dalloc(c, &c->cell, (size_t)nnz, "cells"));
  GPL_RUN(dalloc(c, &c->gptr, (size_t)J + 1, "gene offsets"));
  GPL_RUN(dalloc(c, &c->gvalid, (size_t)J, "gene valid lengths"));
  GPL_RUN(dalloc(c, &c->cnt, (size_t)nnz, "counts"));
  if (nnz) {
    GPL_TRY(c, cudaMemcpy(c->cell, cell_idx, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->cnt, counts, sizeof(double) * nnz, cudaMemcpyHostToDevice));
  }
  GPL_TRY(c, cudaMemcpy(c->gptr, gp.data(), sizeof(int64_t) * (J + 1), cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->gvalid, gv.data(), sizeof(int32_t) * J, cudaMemcpyHostToDevice));
  // the persistent IRLS tail's gene queue: decreasing matched count (ties by gene index)
  std::vector<int32_t> order(J);
  for (int j = 0; j < J; j++) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return gv[a] > gv[b]; });
  GPL_RUN(dalloc(c, &c->gene_order_d, (size_t)J, "gene queue"));
  GPL_RUN(dalloc(c, &c->queue_head_d, 1, "gene queue head"));
  GPL_TRY(c, cudaMemcpy(c->gene_order_d, order.data(), sizeof(int32_t) * J, cudaMemcpyHostToDevice));
  c->N = N;
  c->J = J;
  c->nnz = nnz;
  c->have_counts = true;
  return GPL_OK;
}

int gpl_load_design(gpl_ctx* h, int N, int n_var, const int32_t* cv, const int32_t* vv, const void* body,
                    int64_t body_bytes, int M, int Q) {
  Ctx* c = C(h);
  cudaSetDevice(c->device);
  if (!c->have_counts) {
    c->err = "load the counts first";
    return GPL_ERR_STATE;
  }
  if (N != c->N || n_var < 0 || M <= 0 || Q <= 0 || (n_var > 0 && (!cv || !vv))) {
    c->err = "bad design arguments";
    return GPL_ERR_ARG;
  }
  const int p = n_var + 2;
  std::vector<int> vc(p), vvv(p), nh(p + 1, 0);
  vc[0] = 1;
  vvv[0] = 1;
  for (int k = 0; k < n_var; k++) {
    if (cv[k] < 1 || vv[k] < 1) {
      c->err = "level counts and widths must be >= 1";
      return GPL_ERR_FORMAT;
    }
    vc[k + 1] = cv[k];
    vvv[k + 1] = vv[k];
  }
  vc[p - 1] = 1;
  vvv[p - 1] = M;
  int64_t need = 0;
  for (int k = 0; k < n_var; k++) need += (int64_t)N * vv[k] * (cv[k] == 1 ? 8 : 4);
  if (need != body_bytes || (need > 0 && !body)) {
    c->err = "design body size does not match N, c and v";
    return GPL_ERR_FORMAT;
  }
  for (int j = 0; j < p; j++) nh[j + 1] = nh[j] + vvv[j] * vc[j];
  const int P = nh[p];
  std::vector<int> mc(P), mv(P), mk(P);
  for (int j = 0; j < p; j++)
    for (int k = nh[j]; k < nh[j + 1]; k++) {
      mc[k] = vc[j];
      mv[k] = k - nh[j];
      mk[k] = j;
    }
  const int J = c->J;
  const size_t ldN = (size_t)((N + 31) / 32 * 32);
  // variable data from the body (numeric: N x v doubles; categorical: N level codes)
  const char* bp = (const char*)body;
  std::vector<int64_t> voff(p, -1);
  {
    int64_t off = 0;
    for (int j = 1; j < p - 1; j++) {
      voff[j] = off;
      off += (int64_t)N * vvv[j] * (vc[j] == 1 ? 8 : 4);
    }
  }
  std::vector<int> catv;  // categorical variables (model variable index)
  std::vector<std::vector<int32_t>> codes;
  for (int j = 1; j < p - 1; j++) {
    if (vc[j] == 1) continue;
    std::vector<int32_t> cd(N);
    memcpy(cd.data(), bp + voff[j], sizeof(int32_t) * N);
    const int ncol = vc[j] * vvv[j];
    for (int i = 0; i < N; i++)
      if (cd[i] < 0 || cd[i] >= ncol) {
        c->err = "categorical level code out of range in variable " + std::to_string(j);
        return GPL_ERR_FORMAT;
      }
    catv.push_back(j);
    codes.push_back(std::move(cd));
  }
  // cell groups: cells sorted (stably) by their tuple of levels; runs of equal tuples
  std::vector<int32_t> order(N);
  for (int i = 0; i < N; i++) order[i] = i;
  const int ncat = (int)catv.size();
  std::vector<int32_t> gstart, glev;
  int n_grp = 0;
  if (ncat > 0) {
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
      for (int v = 0; v < ncat; v++)
        if (codes[v][a] != codes[v][b]) return codes[v][a] < codes[v][b];
      return false;
    });
    for (int k = 0; k < N; k++) {
      bool fresh = k == 0;
      for (int v = 0; v < ncat && !fresh; v++) fresh = codes[v][order[k]] != codes[v][order[k - 1]];
      if (fresh) {
        gstart.push_back(k);
        for (int v = 0; v < ncat; v++) glev.push_back(codes[v][order[k]]);
      }
    }
    gstart.push_back(N);
    n_grp = (int)gstart.size() - 1;
  }
  // dense columns: every numeric column; categorical one-hots too when grouping does not pay
  int n_dense_est = 1 + M;
  for (int j = 1; j < p - 1; j++)
    if (vc[j] == 1) n_dense_est += vvv[j];
  const double gsum_bytes = (double)J * n_grp * (n_dense_est + 1) * 8.0;
  const bool grouped = ncat > 0 && n_grp <= 8192 && n_grp <= N / 4 + 1 && gsum_bytes <= 24e9;
  std::vector<int> dcol;
  for (int k = 0; k < P; k++)
    if (mc[k] == 1 || !grouped) dcol.push_back(k);
  const int n_d = (int)dcol.size();
  std::vector<double> Dh(ldN * n_d, 0.0);
  for (int a = 0; a < n_d; a++) {
    const int k = dcol[a], j = mk[k];
    double* dst = &Dh[(size_t)a * ldN];
    if (j == 0) {
      for (int i = 0; i < N; i++) dst[i] = 1.0;
    } else if (j == p - 1) {
      // Knm: written by the kernel-matrix step
    } else if (vc[j] == 1) {
      memcpy(dst, bp + voff[j] + (int64_t)mv[k] * N * 8, sizeof(double) * N);
    } else {
      const int v = (int)(std::find(catv.begin(), catv.end(), j) - catv.begin());
      for (int i = 0; i < N; i++) dst[i] = codes[v][i] == mv[k] ? 1.0 : 0.0;
    }
  }
  free_state(c);
  c->M = M;
  c->Q = Q;
  c->p = p;
  c->P = P;
  c->n_var = n_var;
  c->vc = vc;
  c->vv = vvv;
  c->nh = nh;
  c->mc = mc;
  c->mv = mv;
  c->mk = mk;
  c->ldN = (int)ldN;
  c->dcol = dcol;
  c->n_d = n_d;
  c->dg0 = n_d - M;
  c->n_cv = grouped ? ncat : 0;
  c->n_grp = grouped ? n_grp : 0;
  c->cv_nh.clear();
  c->cv_nlev.clear();
  if (grouped)
    for (int v = 0; v < ncat; v++) {
      c->cv_nh.push_back(nh[catv[v]]);
      c->cv_nlev.push_back(vc[catv[v]] * vvv[catv[v]]);
    }
  std::vector<int2> tiles;
  if (grouped)
    for (int g = 0; g < n_grp; g++)
      for (int r0 = 0; r0 < gstart[g + 1] - gstart[g]; r0 += 64) tiles.push_back(make_int2(g, r0));
  c->n_hk_tiles = (int)tiles.size();
  std::vector<int2> tiles128;
  std::vector<int32_t> tile_cells;  // the cell of each of the 128 slots of every tile, -1 past the group
  std::vector<int32_t> tile_pos;    // the same slots as positions in group order
  if (grouped)
    for (int g = 0; g < n_grp; g++)
      for (int r0 = 0; r0 < gstart[g + 1] - gstart[g]; r0 += 128) {
        tiles128.push_back(make_int2(g, r0));
        for (int q = 0; q < 128; q++) {
          const bool in = r0 + q < gstart[g + 1] - gstart[g];
          tile_cells.push_back(in ? order[gstart[g] + r0 + q] : -1);
          tile_pos.push_back(in ? gstart[g] + r0 + q : -1);
        }
      }
  c->n_hk_tiles128 = (int)tiles128.size();
  c->tot_max = tot_len(c, 1);
  const size_t scratch_n = std::max({ldN * (size_t)J, (size_t)J * P * P, (size_t)c->tot_max, (size_t)M * M});
  GPL_RUN(dalloc(c, &c->Dm, ldN * n_d, "dense model columns"));
  GPL_RUN(dalloc(c, &c->dcol_d, (size_t)n_d, "dense column map"));
  GPL_RUN(dalloc(c, &c->W, ldN * (J + 1), "W"));
  GPL_RUN(dalloc(c, &c->Nu, ldN * J, "Nu"));
  GPL_RUN(dalloc(c, &c->Psi, (size_t)J * P * P, "Psi"));
  GPL_RUN(dalloc(c, &c->PsiInv, (size_t)J * P * P, "PsiInv"));
  GPL_RUN(dalloc(c, &c->Beta, (size_t)P * J, "Beta"));
  GPL_RUN(dalloc(c, &c->tBeta, (size_t)P * J, "tBeta"));
  GPL_RUN(dalloc(c, &c->bvec, (size_t)P * J, "bvec"));
  GPL_RUN(dalloc(c, &c->sol, (size_t)P * J, "sol"));
  GPL_RUN(dalloc(c, &c->rres, (size_t)P * J, "refinement residual"));
  GPL_RUN(dalloc(c, &c->bx, (size_t)P * J, "refinement product"));
  GPL_RUN(dalloc(c, &c->rphi, (size_t)J, "1/phi"));
  GPL_RUN(dalloc(c, &c->e0, ldN, "z.zeta"));
  GPL_RUN(dalloc(c, &c->zeta, (size_t)P, "zeta"));
  GPL_RUN(dalloc(c, &c->scratch, scratch_n, "scratch"));
  GPL_RUN(dalloc(c, &c->U, ldN * n_d, "U"));
  GPL_RUN(dalloc(c, &c->Kmm, (size_t)M * M, "Kmm"));
  GPL_RUN(dalloc(c, &c->Kinv, (size_t)M * M, "Kinv"));
  GPL_RUN(dalloc(c, &c->KmmInv, (size_t)M * M, "KmmInv"));
  GPL_RUN(dalloc(c, &c->KinvKmn, ldN * M, "KinvKmn"));
  GPL_RUN(dalloc(c, &c->titsias, ldN, "titsias"));
  GPL_RUN(dalloc(c, &c->DeltaInv, (size_t)P * P, "DeltaInv"));
  GPL_RUN(dalloc(c, &c->Omega, 2 * (size_t)N, "Omega"));
  GPL_RUN(dalloc(c, &c->delta, 2 * (size_t)p, "delta"));
  GPL_RUN(dalloc(c, &c->X, 2 * (size_t)N * Q, "X"));
  GPL_RUN(dalloc(c, &c->T, 2 * (size_t)M * Q, "T"));
  GPL_RUN(dalloc(c, &c->rho, 2 * (size_t)Q, "rho"));
  GPL_RUN(dalloc(c, &c->phi, (size_t)J, "phi"));
  GPL_RUN(dalloc(c, &c->ls, (size_t)N, "ls"));
  GPL_RUN(dalloc(c, &c->lkhds, (size_t)J, "lkhds"));
  GPL_RUN(dalloc(c, &c->lkhd_dev, (size_t)kLkhdSlots, "lkhd"));
  GPL_RUN(dalloc(c, &c->grad, (size_t)c->tot_max + Q, "grad"));
  GPL_RUN(dalloc(c, &c->grad0, (size_t)c->tot_max + Q, "grad0"));
  GPL_RUN(dalloc(c, &c->ss, (size_t)c->tot_max + Q, "ss"));
  GPL_RUN(dalloc(c, &c->SS, (size_t)c->tot_max * kHist, "SS"));
  GPL_RUN(dalloc(c, &c->XX, (size_t)c->tot_max * kHist, "XX"));
  GPL_RUN(dalloc(c, &c->gdtmp, (size_t)P * J, "gdtmp"));
  GPL_RUN(dalloc(c, &c->C1, ldN * M, "C1"));
  GPL_RUN(dalloc(c, &c->cellfac, 3 * ldN, "per-cell factors of W"));
  GPL_RUN(dalloc(c, &c->C2, (size_t)M * M, "C2"));
  GPL_RUN(dalloc(c, &c->grtmp, (size_t)M * Q, "grtmp"));
  GPL_RUN(dalloc(c, &c->red, std::max((size_t)ldN, (size_t)4096), "reduction"));
  GPL_RUN(dalloc(c, &c->lb_work, 64, "lbfgs scalars"));
  GPL_RUN(dalloc(c, &c->mc_d, (size_t)P, "mc"));
  GPL_RUN(dalloc(c, &c->mv_d, (size_t)P, "mv"));
  GPL_RUN(dalloc(c, &c->mk_d, (size_t)P, "mk"));
  GPL_RUN(dalloc(c, &c->nh_d, (size_t)p + 1, "nh"));
  if (c->n_grp) {
    std::vector<int32_t> codes_h((size_t)ncat * ldN, 0);
    for (int v = 0; v < ncat; v++) memcpy(&codes_h[(size_t)v * ldN], codes[v].data(), sizeof(int32_t) * N);
    GPL_RUN(dalloc(c, &c->codes_d, codes_h.size(), "level codes"));
    GPL_RUN(dalloc(c, &c->cv_nh_d, (size_t)ncat, "grouped variable columns"));
    GPL_RUN(dalloc(c, &c->cv_nlev_d, (size_t)ncat, "grouped variable levels"));
    GPL_RUN(dalloc(c, &c->glev_d, glev.size(), "group levels"));
    GPL_RUN(dalloc(c, &c->gcells_d, (size_t)N, "group cells"));
    GPL_RUN(dalloc(c, &c->gpos_d, (size_t)N, "group positions"));
    GPL_RUN(dalloc(c, &c->gid_d, (size_t)N, "cell groups"));
    GPL_RUN(dalloc(c, &c->lvt, (size_t)lvt_ld(J) * n_grp, "level sums per group"));
    GPL_RUN(dalloc(c, &c->gstart_d, gstart.size(), "group offsets"));
    GPL_RUN(dalloc(c, &c->hk_tiles_d, tiles.size(), "group tiles"));
    GPL_RUN(dalloc(c, &c->hk_tiles128_d, tiles128.size(), "group tiles"));
    GPL_RUN(dalloc(c, &c->hk_cells_d, tile_cells.size(), "group tile cells"));
    GPL_RUN(dalloc(c, &c->hk_pos_d, tile_pos.size(), "group tile positions"));
    GPL_RUN(dalloc(c, &c->Wg, ldN * (size_t)J, "W in group order"));
    GPL_RUN(dalloc(c, &c->Dg, ldN * (size_t)n_d, "dense columns in group order"));
    GPL_RUN(dalloc(c, &c->rOmg, ldN, "1/Omega in group order"));
    GPL_TRY(c, cudaMemset(c->Wg, 0, sizeof(double) * ldN * (size_t)J));
    GPL_RUN(dalloc(c, &c->gsum, (size_t)J * n_grp * (n_d + 1), "group sums"));
    GPL_RUN(dalloc(c, &c->gT, (size_t)J * n_grp, "group response sums"));
    GPL_RUN(dalloc(c, &c->HK, ldN * (n_d + 1), "HK"));
    GPL_TRY(c, cudaMemcpy(c->codes_d, codes_h.data(), sizeof(int32_t) * codes_h.size(), cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->cv_nh_d, c->cv_nh.data(), sizeof(int) * ncat, cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->cv_nlev_d, c->cv_nlev.data(), sizeof(int) * ncat, cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->glev_d, glev.data(), sizeof(int32_t) * glev.size(), cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->gcells_d, order.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
    {
      std::vector<int32_t> gid(N), gpos(N);
      for (int g = 0; g < n_grp; g++)
        for (int k = gstart[g]; k < gstart[g + 1]; k++) gid[order[k]] = g;
      for (int k = 0; k < N; k++) gpos[order[k]] = k;
      GPL_TRY(c, cudaMemcpy(c->gid_d, gid.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
      GPL_TRY(c, cudaMemcpy(c->gpos_d, gpos.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
    }
    GPL_TRY(c, cudaMemcpy(c->gstart_d, gstart.data(), sizeof(int32_t) * gstart.size(), cudaMemcpyHostToDevice));
    // per level of each grouped variable: its model column, its variable, its groups in order
    std::vector<int32_t> lvl_cc, lvl_v, lvl_ptr(1, 0), lvl_grp;
    for (int v = 0; v < ncat; v++)
      for (int L = 0; L < c->cv_nlev[v]; L++) {
        lvl_cc.push_back(c->cv_nh[v] + L);
        lvl_v.push_back(v);
        for (int g = 0; g < n_grp; g++)
          if (glev[(size_t)g * ncat + v] == L) lvl_grp.push_back(g);
        lvl_ptr.push_back((int32_t)lvl_grp.size());
      }
    c->n_lvl = (int)lvl_cc.size();
    GPL_RUN(dalloc(c, &c->lvl_cc_d, lvl_cc.size(), "level columns"));
    GPL_RUN(dalloc(c, &c->lvl_v_d, lvl_v.size(), "level variables"));
    GPL_RUN(dalloc(c, &c->lvl_ptr_d, lvl_ptr.size(), "level offsets"));
    GPL_RUN(dalloc(c, &c->lvl_grp_d, std::max<size_t>(1, lvl_grp.size()), "level groups"));
    GPL_TRY(c, cudaMemcpy(c->lvl_cc_d, lvl_cc.data(), sizeof(int32_t) * lvl_cc.size(), cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->lvl_v_d, lvl_v.data(), sizeof(int32_t) * lvl_v.size(), cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->lvl_ptr_d, lvl_ptr.data(), sizeof(int32_t) * lvl_ptr.size(), cudaMemcpyHostToDevice));
    if (!lvl_grp.empty())
      GPL_TRY(c, cudaMemcpy(c->lvl_grp_d, lvl_grp.data(), sizeof(int32_t) * lvl_grp.size(), cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->hk_tiles_d, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->hk_tiles128_d, tiles128.data(), sizeof(int2) * tiles128.size(), cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->hk_pos_d, tile_pos.data(), sizeof(int32_t) * tile_pos.size(), cudaMemcpyHostToDevice));
    GPL_TRY(c, cudaMemcpy(c->hk_cells_d, tile_cells.data(), sizeof(int32_t) * tile_cells.size(),
                          cudaMemcpyHostToDevice));
  }
  GPL_TRY(c, cudaMemcpy(c->Dm, Dh.data(), sizeof(double) * ldN * n_d, cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->dcol_d, dcol.data(), sizeof(int) * n_d, cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->mc_d, mc.data(), sizeof(int) * P, cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->mv_d, mv.data(), sizeof(int) * P, cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->mk_d, mk.data(), sizeof(int) * P, cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->nh_d, nh.data(), sizeof(int) * (p + 1), cudaMemcpyHostToDevice));
  // freshly allocated reference buffers read as zero (the harness' calloc convention)
  GPL_TRY(c, cudaMemset(c->W, 0, sizeof(double) * ldN * (J + 1)));
  GPL_TRY(c, cudaMemset(c->Nu, 0, sizeof(double) * ldN * J));
  GPL_TRY(c, cudaMemset(c->Psi, 0, sizeof(double) * (size_t)J * P * P));
  GPL_TRY(c, cudaMemset(c->PsiInv, 0, sizeof(double) * (size_t)J * P * P));
  GPL_TRY(c, cudaMemset(c->Beta, 0, sizeof(double) * (size_t)P * J));
  GPL_TRY(c, cudaMemset(c->tBeta, 0, sizeof(double) * (size_t)P * J));
  GPL_TRY(c, cudaMemset(c->bvec, 0, sizeof(double) * (size_t)P * J));
  GPL_TRY(c, cudaMemset(c->ss, 0, sizeof(double) * ((size_t)c->tot_max + Q)));
  GPL_TRY(c, cudaMemset(c->grad, 0, sizeof(double) * ((size_t)c->tot_max + Q)));
  GPL_TRY(c, cudaMemset(c->grad0, 0, sizeof(double) * ((size_t)c->tot_max + Q)));
  GPL_TRY(c, cudaMemset(c->SS, 0, sizeof(double) * (size_t)c->tot_max * kHist));
  GPL_TRY(c, cudaMemset(c->XX, 0, sizeof(double) * (size_t)c->tot_max * kHist));
  GPL_TRY(c, cudaMemset(c->titsias, 0, sizeof(double) * ldN));
  GPL_TRY(c, cudaMemset(c->X, 0, sizeof(double) * 2 * (size_t)N * Q));
  GPL_TRY(c, cudaMemset(c->T, 0, sizeof(double) * 2 * (size_t)M * Q));
  GPL_TRY(c, cudaMemset(c->lkhd_dev, 0, sizeof(double) * kLkhdSlots));
  c->have_design = true;
  std::vector<double> ones(N, 1.0);
  GPL_TRY(c, cudaMemcpy(c->ls, ones.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  return gpl_init_params(h);
}

int gpl_set_size_factors(gpl_ctx* h, const double* ls) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (!ls) return GPL_ERR_ARG;
  GPL_TRY(c, cudaMemcpy(c->ls, ls, sizeof(double) * c->N, cudaMemcpyHostToDevice));
  return GPL_OK;
}

int gpl_dims(const gpl_ctx* h, int32_t* d) {
  const Ctx* c = &h->c;
  if (!d) return GPL_ERR_ARG;
  d[0] = c->N; d[1] = c->J; d[2] = c->M; d[3] = c->P; d[4] = c->p; d[5] = c->Q;
  return GPL_OK;
}

int gpl_init_params(gpl_ctx* h) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  std::vector<double> delta(c->p, 0.01), rho(c->Q, 10.0), Om(c->N, 1.0), phi(c->J, 1.0), T0(c->M);
  delta[0] = 1.5;
  delta[c->p - 1] = 0.3;
  rho[0] = 5.0;
  for (int i = 0; i < c->M; i++) T0[i] = ((double)(i + 1) / (double)(c->M + 1)) * 2.0 * 3.14159265358979;
  GPL_TRY(c, cudaMemcpy(c->delta, delta.data(), sizeof(double) * c->p, cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->rho, rho.data(), sizeof(double) * c->Q, cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->Omega, Om.data(), sizeof(double) * c->N, cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->phi, phi.data(), sizeof(double) * c->J, cudaMemcpyHostToDevice));
  GPL_TRY(c, cudaMemcpy(c->T, T0.data(), sizeof(double) * c->M, cudaMemcpyHostToDevice));
  return GPL_OK;
}

int gpl_set_params(gpl_ctx* h, const double* Omega, const double* delta, const double* X, const double* T,
                   const double* rho, const double* phi) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  cudaSetDevice(c->device);
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  if (Omega) GPL_TRY(c, cudaMemcpy(c->Omega, Omega, sizeof(double) * c->N, cudaMemcpyHostToDevice));
  if (delta) GPL_TRY(c, cudaMemcpy(c->delta, delta, sizeof(double) * c->p, cudaMemcpyHostToDevice));
  if (X) GPL_TRY(c, cudaMemcpy(c->X, X, sizeof(double) * (size_t)c->N * c->Q, cudaMemcpyHostToDevice));
  if (T) GPL_TRY(c, cudaMemcpy(c->T, T, sizeof(double) * (size_t)c->M * c->Q, cudaMemcpyHostToDevice));
  if (rho) GPL_TRY(c, cudaMemcpy(c->rho, rho, sizeof(double) * c->Q, cudaMemcpyHostToDevice));
  if (phi) GPL_TRY(c, cudaMemcpy(c->phi, phi, sizeof(double) * c->J, cudaMemcpyHostToDevice));
  return GPL_OK;
}

int gpl_get_params(gpl_ctx* h, double* Omega, double* delta, double* X, double* T, double* rho, double* phi) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  if (Omega) GPL_TRY(c, cudaMemcpy(Omega, c->Omega, sizeof(double) * c->N, cudaMemcpyDeviceToHost));
  if (delta) GPL_TRY(c, cudaMemcpy(delta, c->delta, sizeof(double) * c->p, cudaMemcpyDeviceToHost));
  if (X) GPL_TRY(c, cudaMemcpy(X, c->X, sizeof(double) * (size_t)c->N * c->Q, cudaMemcpyDeviceToHost));
  if (T) GPL_TRY(c, cudaMemcpy(T, c->T, sizeof(double) * (size_t)c->M * c->Q, cudaMemcpyDeviceToHost));
  if (rho) GPL_TRY(c, cudaMemcpy(rho, c->rho, sizeof(double) * c->Q, cudaMemcpyDeviceToHost));
  if (phi) GPL_TRY(c, cudaMemcpy(phi, c->phi, sizeof(double) * c->J, cudaMemcpyDeviceToHost));
  return GPL_OK;
}

int gpl_set_beta(gpl_ctx* h, const double* beta) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  GPL_TRY(c, cudaMemcpy(c->Beta, beta, sizeof(double) * (size_t)c->P * c->J, cudaMemcpyHostToDevice));
  return GPL_OK;
}

int gpl_get_beta(gpl_ctx* h, double* beta) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  GPL_TRY(c, cudaMemcpy(beta, c->Beta, sizeof(double) * (size_t)c->P * c->J, cudaMemcpyDeviceToHost));
  return GPL_OK;
}

int gpl_kernel_mats(gpl_ctx* h) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  GPL_RUN(launch_kernel_mats(c));
  return GPL_OK;
}

int gpl_glm_init(gpl_ctx* h) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  GPL_RUN(glm_init(c));
  return GPL_OK;
}

int gpl_gram(gpl_ctx* h) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  GPL_RUN(launch_gram(c, false));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  return tc_error_flag(c);
}

int gpl_expand_delta(gpl_ctx* h) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  return launch_expand_delta(c);
}

int gpl_irls_sweep(gpl_ctx* h, int jtr, double* lkhd) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (jtr < 0 || jtr >= kLkhdSlots) return GPL_ERR_ARG;
  return irls_sweep(c, jtr, lkhd);
}

int gpl_irls(gpl_ctx* h, int jtr_max, int* n_sweeps) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (jtr_max < 1 || jtr_max >= kLkhdSlots) return GPL_ERR_ARG;
  return irls(c, jtr_max, n_sweeps);
}

int gpl_objective_after_irls(gpl_ctx* h, double* lkhd) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  return objective_after_irls(c, lkhd);
}

int gpl_objective(gpl_ctx* h, int slot, double* lkhd) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (slot < 0 || slot >= kGraphSlot) return GPL_ERR_ARG;
  GPL_RUN(objective_run(c, slot));
  return read_slot(c, slot, lkhd);
}

int gpl_gradient(gpl_ctx* h, double* grad) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  GPL_RUN(gradient_launch(c));
  if (grad) {
    const int64_t n = tot_len(c, 0) + c->Q;
    GPL_TRY(c, cudaMemcpyAsync(grad, c->grad, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    GPL_TRY(c, cudaStreamSynchronize(c->stream));
  }
  return tc_error_flag(c);
}

int gpl_lbfgs_update(gpl_ctx* h, int jtr, int rhoflag) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  return launch_lbfgs_update(c, jtr, rhoflag ? 1 : 0);
}

int gpl_downdate(gpl_ctx* h, int jtr, double sr, int rhoflag) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  return launch_downdate(c, jtr, sr, rhoflag ? 1 : 0);
}

int gpl_beta_from_tilde(gpl_ctx* h) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  return launch_beta_from_tilde(c);
}

int gpl_fit(gpl_ctx* h, int itr_max, int lbfgs_budget, int32_t* stats, double* trace, int trace_cap) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  int itr, total_lbfgs = 0, total_irls = 0, total_evals = 0, ntrace = 0, rc = GPL_OK;
  for (itr = 0; itr < itr_max; itr++) {
    int32_t st[4] = {0, 0, 0, 0};
    const int left = lbfgs_budget > 0 ? lbfgs_budget - total_lbfgs : 0;
    rc = fit_outer(c, itr, left, st, trace ? trace + ntrace : nullptr, trace ? trace_cap - ntrace : 0);
    total_irls += st[0];
    total_lbfgs += st[1];
    total_evals += st[2];
    ntrace += st[3];
    if (rc == GPL_ERR_NAN) {
      itr++;
      break;
    }
    if (rc) return rc;
    if (lbfgs_budget > 0 && total_lbfgs >= lbfgs_budget) {
      itr++;
      break;
    }
  }
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  if (stats) {
    stats[0] = itr;
    stats[1] = total_irls;
    stats[2] = total_lbfgs;
    stats[3] = total_evals;
  }
  return rc == GPL_ERR_NAN ? GPL_ERR_NAN : GPL_OK;
}

int gpl_fit_outer(gpl_ctx* h, int itr, int lbfgs_budget, int32_t* stats, double* trace, int trace_cap) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (itr < 0) {
    c->err = "itr must be >= 0";
    return GPL_ERR_ARG;
  }
  int32_t st[4] = {0, 0, 0, 0};
  const int rc = fit_outer(c, itr, lbfgs_budget, st, trace, trace ? trace_cap : 0);
  if (stats)
    for (int k = 0; k < 4; k++) stats[k] = st[k];
  if (rc == GPL_OK) GPL_TRY(c, cudaStreamSynchronize(c->stream));
  return rc;
}

int gpl_score_stats(gpl_ctx* h, int L, const double* G, double* S) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (L <= 0 || !G || !S) {
    c->err = "score statistics need L >= 1 genotype columns and non-NULL G and S";
    return GPL_ERR_ARG;
  }
  const size_t N = c->N, J = c->J;
  const int LB = 64;  // genotype columns per pass (two per column in the GEMM tile of 128)
  double *dG = nullptr, *dW = nullptr, *dS = nullptr;
  const size_t work = (size_t)2 * LB * N + (size_t)4 * LB * J;
  if (cudaMalloc((void**)&dG, sizeof(double) * N * LB) != cudaSuccess ||
      cudaMalloc((void**)&dW, sizeof(double) * work) != cudaSuccess ||
      cudaMalloc((void**)&dS, sizeof(double) * J * LB) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dG);
    cudaFree(dW);
    cudaFree(dS);
    c->err = "device allocation failed: score statistics";
    return GPL_ERR_ALLOC;
  }
  int rc = GPL_OK;
  for (int l0 = 0; l0 < L && rc == GPL_OK; l0 += LB) {
    const int nl = std::min(LB, L - l0);
    if (cudaMemcpyAsync(dG, G + (size_t)l0 * N, sizeof(double) * N * nl, cudaMemcpyHostToDevice, c->stream) !=
        cudaSuccess) {
      rc = GPL_ERR_CUDA;
      break;
    }
    rc = launch_score_stats(c, nl, dG, dS, dW);
    if (rc == GPL_OK &&
        cudaMemcpyAsync(S + (size_t)l0 * J, dS, sizeof(double) * J * nl, cudaMemcpyDeviceToHost, c->stream) !=
            cudaSuccess)
      rc = GPL_ERR_CUDA;
    if (rc == GPL_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = GPL_ERR_CUDA;
  }
  if (rc == GPL_ERR_CUDA && c->err.empty()) c->err = cudaGetErrorString(cudaGetLastError());
  cudaFree(dG);
  cudaFree(dW);
  cudaFree(dS);
  return rc;
}

int gpl_de_model(gpl_ctx* h, int model) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (model < GPL_DE_NULL || model >= c->Q) {
    c->err = "model must be GPL_DE_NULL, GPL_DE_FULL or a latent dimension in [0, Q)";
    return GPL_ERR_ARG;
  }
  graph_reset(c);  // the model changes the kernels an evaluation launches
  GPL_RUN(de_loader_value(c, model == GPL_DE_NULL));
  c->de = true;
  c->kernel_lv = model == GPL_DE_NULL ? kLvNone : (model == GPL_DE_FULL ? kLvAll : model);
  GPL_RUN(launch_kernel_mats(c));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  return GPL_OK;
}

int gpl_de_irls(gpl_ctx* h, int jtr_max, double tol, double* lkhds, int32_t* sweeps, double* trace, int trace_cap) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (!c->de) {
    c->err = "select a model with gpl_de_model first";
    return GPL_ERR_STATE;
  }
  if (jtr_max < 1 || !(tol >= 0.0) || (trace && trace_cap < 0)) {
    c->err = "jtr_max must be >= 1 and tol >= 0";
    return GPL_ERR_ARG;
  }
  const int prec = c->precision;
  c->precision = GPL_PREC_FP64;
  int n = 0;
  const int rc = de_irls(c, jtr_max, tol, &n, trace, trace ? trace_cap : 0);
  c->precision = prec;
  if (rc) return rc;
  if (lkhds) GPL_TRY(c, cudaMemcpy(lkhds, c->lkhds, sizeof(double) * c->J, cudaMemcpyDeviceToHost));
  if (sweeps) *sweeps = n;
  return GPL_OK;
}

int gpl_vc_fit(gpl_ctx* h, int itr_max, int lbfgs_max, double* dg, double* obj, int cap, int32_t* n_itr) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (itr_max < 1 || lbfgs_max < 1 || lbfgs_max + 2 >= kLkhdSlots || c->p < 3 || ((dg || obj) && cap < 0)) {
    c->err = "itr_max and lbfgs_max must be >= 1 and the design needs a variable besides intercept and GP";
    return GPL_ERR_ARG;
  }
  graph_reset(c);  // the driver's constants change the objective's launches
  const int prec = c->precision;
  const bool de = c->de, vcf = c->vcomp;
  const int lv = c->kernel_lv;
  GPL_RUN(de_loader_value(c, false));
  c->precision = GPL_PREC_FP64;
  c->de = true;
  c->vcomp = true;
  c->kernel_lv = kLvAll;
  int n = 0;
  const int rc = vc_fit(c, itr_max, lbfgs_max, dg, obj, (dg || obj) ? cap : 0, &n);
  c->precision = prec;
  c->de = de;
  c->vcomp = vcf;
  c->kernel_lv = lv;
  if (rc) return rc;
  if (n_itr) *n_itr = n;
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  return GPL_OK;
}

void gpl_ta_equispaced(int M, int Q, double* T) {
  if (!T || M <= 0 || Q <= 0) return;
  for (int i = 0; i < M; i++) T[i] = ((double)(i + 1) / (double)(M + 1)) * 2.0 * 3.14159265358979;
  for (int k = 1; k < Q; k++)
    for (int i = 0; i < M; i++) T[i + (size_t)k * M] = ((double)(i + 1) / (double)(M + 1) - 0.5) * 6.0;
}

int gpl_evaluate(gpl_ctx* h, const double* params, int64_t n_params, double* lkhd, double* grad) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  const int64_t n = tot_len(c, 0) + c->Q;
  if (!params || n_params != n) {
    c->err = "params must hold N + p + N*Q + M*Q + Q values";
    return GPL_ERR_ARG;
  }
  const double* p = params;
  GPL_TRY(c, cudaMemcpyAsync(c->Omega, p, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
  p += c->N;
  GPL_TRY(c, cudaMemcpyAsync(c->delta, p, sizeof(double) * c->p, cudaMemcpyHostToDevice, c->stream));
  p += c->p;
  GPL_TRY(c, cudaMemcpyAsync(c->X, p, sizeof(double) * (size_t)c->N * c->Q, cudaMemcpyHostToDevice, c->stream));
  p += (size_t)c->N * c->Q;
  GPL_TRY(c, cudaMemcpyAsync(c->T, p, sizeof(double) * (size_t)c->M * c->Q, cudaMemcpyHostToDevice, c->stream));
  p += (size_t)c->M * c->Q;
  GPL_TRY(c, cudaMemcpyAsync(c->rho, p, sizeof(double) * c->Q, cudaMemcpyHostToDevice, c->stream));
  GPL_RUN(objective_run(c, 1));
  GPL_RUN(gradient_run(c));
  if (grad) GPL_TRY(c, cudaMemcpyAsync(grad, c->grad, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  double v = 0.0;
  GPL_TRY(c, cudaMemcpyAsync(&v, c->lkhd_dev + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  c->lkhd[1] = v;
  if (lkhd) *lkhd = v;
  return tc_error_flag(c);
}

int gpl_evaluate_device(gpl_ctx* h) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  GPL_RUN(objective_run(c, 1));
  GPL_RUN(gradient_run(c));
  return GPL_OK;
}

int gpl_get(gpl_ctx* h, const char* name, double* out, int64_t cap, int64_t* len) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (!name) return GPL_ERR_ARG;
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  const size_t N = c->N, J = c->J, M = c->M, Q = c->Q, P = c->P, p = c->p, ldN = c->ldN;
  const int g0 = c->nh[c->p - 1];
  std::string s(name);
  auto plain = [&](const double* src, size_t n) -> int {
    if (len) *len = (int64_t)n;
    if (!out) return GPL_OK;
    if ((int64_t)n > cap) { c->err = "output buffer too small"; return GPL_ERR_ARG; }
    GPL_TRY(c, cudaMemcpy(out, src, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return GPL_OK;
  };
  // cell-fastest matrices with a padded leading dimension: copy column by column
  auto cols = [&](const double* src, size_t ncol) -> int {
    const size_t n = N * ncol;
    if (len) *len = (int64_t)n;
    if (!out) return GPL_OK;
    if ((int64_t)n > cap) { c->err = "output buffer too small"; return GPL_ERR_ARG; }
    GPL_TRY(c, cudaMemcpy2D(out, N * sizeof(double), src, ldN * sizeof(double), N * sizeof(double), ncol,
                            cudaMemcpyDeviceToHost));
    return GPL_OK;
  };
  if (s == "Omega") return plain(c->Omega, N);
  if (s == "delta") return plain(c->delta, p);
  if (s == "X") return plain(c->X, N * Q);
  if (s == "T") return plain(c->T, M * Q);
  if (s == "rho") return plain(c->rho, Q);
  if (s == "phi") return plain(c->phi, J);
  if (s == "Beta") return plain(c->Beta, P * J);
  if (s == "tBeta") return plain(c->tBeta, P * J);
  if (s == "Kmm") return plain(c->Kmm, M * M);
  if (s == "Kinv") return plain(c->Kinv, M * M);
  if (s == "titsias") return plain(c->titsias, N);
  if (s == "Psi") return plain(c->Psi, J * P * P);
  if (s == "PsiInv") return plain(c->PsiInv, J * P * P);
  if (s == "DeltaInv") return plain(c->DeltaInv, P * P);
  if (s == "lkhds") return plain(c->lkhds, J);
  if (s == "C2") return plain(c->C2, M * M);
  if (s == "grad") return plain(c->grad, N + p + N * Q + M * Q + Q);
  if (s == "ss") return plain(c->ss, N + p + N * Q + M * Q + Q);
  if (s == "zeta") {
    if (len) *len = (int64_t)P;
    if (out) memset(out, 0, sizeof(double) * P);
    return GPL_OK;
  }
  if (s == "lkhd_dev") return plain(c->lkhd_dev, 2);
  if (s == "lkhd") {
    if (len) *len = kLkhdSlots;
    if (out) {
      if (cap < kLkhdSlots) return GPL_ERR_ARG;
      memcpy(out, c->lkhd.data(), sizeof(double) * kLkhdSlots);
    }
    return GPL_OK;
  }
  if (s == "Knm") return cols(c->Dm + (size_t)c->dg0 * ldN, M);
  if (s == "W") return cols(c->W, J + 1);
  if (s == "Nu") return cols(c->Nu, J);
  if (s == "C1") return cols(c->C1, M);
  if (s == "Dm") return cols(c->Dm, (size_t)c->n_d);
  if (s == "KinvKmn") {  // reference layout M x N (k + i*M)
    if (len) *len = (int64_t)(M * N);
    if (!out) return GPL_OK;
    if ((int64_t)(M * N) > cap) return GPL_ERR_ARG;
    std::vector<double> tmp(N * M);
    GPL_TRY(c, cudaMemcpy2D(tmp.data(), N * sizeof(double), c->KinvKmn, ldN * sizeof(double), N * sizeof(double), M,
                            cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < N; i++)
      for (size_t k = 0; k < M; k++) out[k + i * M] = tmp[i + k * N];
    return GPL_OK;
  }
  c->err = "unknown buffer name: " + s;
  return GPL_ERR_ARG;
}

int gpl_profile_enable(gpl_ctx* h, int on) {
  C(h)->prof = on != 0;
  return GPL_OK;
}

int gpl_profile_reset(gpl_ctx* h) {
  Ctx* c = C(h);
  drain_profile(c);
  c->prof_total.clear();
  return GPL_OK;
}

int gpl_profile_read(gpl_ctx* h, const char* name, double* total_ms, int64_t* launches) {
  Ctx* c = C(h);
  drain_profile(c);
  for (auto& t : c->prof_total)
    if (t.first == name) {
      if (total_ms) *total_ms = t.second.first;
      if (launches) *launches = t.second.second;
      return GPL_OK;
    }
  if (total_ms) *total_ms = 0.0;
  if (launches) *launches = 0;
  return GPL_OK;
}

int gpl_launch_count(const gpl_ctx* h, int64_t* launches) {
  if (!h || !launches) return GPL_ERR_ARG;
  *launches = h->c.launches;
  return GPL_OK;
}

int gpl_sync(gpl_ctx* h) {
  Ctx* c = C(h);
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  tune_harvest(c);
  return tc_error_flag(c);
}

int gpl_wait_probe(gpl_ctx* h, int64_t limit_ns) {
  if (!h || limit_ns <= 0) return GPL_ERR_ARG;
  Ctx* c = C(h);
  return wait_probe(c, limit_ns);
}

int gpl_tuning(gpl_ctx* h, const char* name, int32_t* chosen, int32_t* cands, double* best_ms, int cap,
               int32_t* n_cands) {
  if (!h || !name) return GPL_ERR_ARG;
  Ctx* c = C(h);
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  tune_harvest(c);
  Tunable* t = tune_find(c, name);
  if (!t) {
    if (n_cands) *n_cands = 0;
    if (chosen) *chosen = -1;
    return GPL_OK;
  }
  const int n = (int)t->cands.size();
  if (n_cands) *n_cands = n;
  if (chosen) *chosen = t->best >= 0 ? t->cands[t->best] : -1;
  for (int k = 0; k < n && k < cap; k++) {
    if (cands) cands[k] = t->cands[k];
    if (best_ms) best_ms[k] = t->n[k] > 0 ? t->best_ms[k] : (t->from_cache ? -2.0 : -1.0);
  }
  return GPL_OK;
}

}  // extern "C"

extern "C" {

int gpl_place_cells(gpl_ctx* h, int iters, double* X, double* obj, int32_t* stats) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (iters < 0 || !X) return GPL_ERR_ARG;
  cudaSetDevice(c->device);
  return place_cells(c, iters, X, obj, stats);
}

int gpl_cell_objective(gpl_ctx* h, const double* X, double* obj, double* grad) {
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  if (!X || !obj) return GPL_ERR_ARG;
  cudaSetDevice(c->device);
  return cell_objective(c, X, obj, grad);
}

}  // extern "C"

extern "C" int gpl_init_latent(gpl_ctx* h, int pca_iters, int kmeans_iters, uint64_t seed, double* X, double* T) {
  if (!h || !X || !T || pca_iters < 1 || kmeans_iters < 0) return GPL_ERR_ARG;
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  cudaSetDevice(c->device);
  return init_latent(c, pca_iters, kmeans_iters, seed, X, T);
}

extern "C" int gpl_cis_stats(gpl_ctx* h, int donor_var, int n_donors, int V, const int8_t* dosages, double* S,
                             double* LR) {
  if (!h || !dosages || !S || V < 1 || n_donors < 1) return GPL_ERR_ARG;
  Ctx* c = C(h);
  GPL_RUN(need_state(c));
  cudaSetDevice(c->device);
  return cis_stats(c, donor_var, n_donors, V, dosages, S, LR);
}
