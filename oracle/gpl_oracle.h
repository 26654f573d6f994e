/*
 * gpl_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, double-precision restatement of the GASPACHO2 sparse GP-LVM fit
 * (the reference's ggplvm.cu, kernel_funcs.cu, chol.cu, util_cuda.cu, init.cu) used as
 * the checker for the CUDA path and as the host-core CPU baseline ("port"). Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU legs load it. Every function
 * cites the reference lines it restates; buffers use the reference's layouts.
 * Parity of this restatement is pinned against the reference's own kernels built for
 * the host (oracle/_ref) and against the golden vectors in tests/golden/.
 */
#ifndef GPL_ORACLE_H
#define GPL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* N cells, J genes, counts in gene-major CSR (SparseMat.cuh:3-10); the design as the file
 * part of a DataFrame (DataFrame.cu:88-149): n_var variables, c[] levels, v[] widths, and
 * the raw body bytes; M inducing points (0: no GP variable, the DE driver's null model),
 * Q latent dimensions. Returns NULL on bad input. */
orc_ctx* orc_create(int N, int J, long nnz, const int* cell_idx, const int* gene_ptr, const double* counts,
                    int n_var, const int* c, const int* v, const void* body, long body_bytes, int M, int Q,
                    const double* ls, const double* X0);
void orc_destroy(orc_ctx* o);
void orc_dims(const orc_ctx* o, int* out6); /* N, J, M, P, p, Q */

void orc_init_params(orc_ctx* o);
void orc_set_params(orc_ctx* o, const double* Omega, const double* delta, const double* X, const double* T,
                    const double* rho, const double* phi);
void orc_set_beta(orc_ctx* o, const double* beta);

void orc_kernel_mats(orc_ctx* o);
void orc_glm_init(orc_ctx* o);
void orc_expand_delta(orc_ctx* o);
double orc_irls_sweep(orc_ctx* o, int jtr);
int orc_irls(orc_ctx* o, int jtr_max);
double orc_objective_after_irls(orc_ctx* o);
void orc_gradient(orc_ctx* o, double* grad_out);
double orc_objective(orc_ctx* o, int slot);
void orc_lbfgs_update(orc_ctx* o, int jtr, int rhoflag);
void orc_downdate(orc_ctx* o, int jtr, double sr, int rhoflag);
void orc_beta_from_tilde(orc_ctx* o);
int orc_fit(orc_ctx* o, int itr_max, int lbfgs_budget, int* stats, double* trace, int trace_cap);
long orc_get(orc_ctx* o, const char* name, double* out);
void orc_score_stats(orc_ctx* o, int L, const double* G, double* S); /* getScoreStats */
/* the DE driver's model comparison (ggplvm_de.cu): kernel over one latent dimension
 * (q < 0: all), one model's IRLS with its stopping rule, initTaEquispaced */
void orc_kernel_mats_lv(orc_ctx* o, int q);
int orc_de_irls(orc_ctx* o, int jtr_max, double tol);
void orc_ta_equispaced(int M, int Q, double* T);
/* the variance-component driver (ggplvm_delta.cu): L-BFGS on log delta[p-2] with IRLS phases */
int orc_vc_fit(orc_ctx* o, int itr_max, int lbfgs_max, double* dg, double* obj, int cap);
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
