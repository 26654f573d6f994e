/*
 * gpl.h -- C ABI of the B200 GASPACHO2 sparse GP-LVM fit (libgpl_b200.so).
 *
 * The reference (GASPACHO2, src/) has no library boundary: its driver `main`
 * (ggplvm.cu:951-1354) reads four binary files, launches its kernels directly and
 * writes params.bin. This header exposes the same path as plain C entry points so a
 * C/C++ driver (the bundled `ggplvm` CLI), Python (ctypes) or any FFI can call it. Each
 * function names the reference code it replaces.
 *
 * Conventions
 *   - All arrays are HOST memory, in the reference's layouts (column-major, cell index
 *     fastest, exactly as the reference files and kernels use them). The context owns
 *     its device memory; nothing in the signatures is a device pointer or a torch type.
 *   - Every function returns GPL_OK (0) or a negative GPL_ERR_* code; gpl_last_error()
 *     gives the message. A context is used from one host thread at a time and runs its
 *     kernels in order on one CUDA stream (its own, or one given at creation).
 *   - Sizes: N cells, J genes, M inducing points, Q latent dimensions, p model variables
 *     (intercept + file variables + the GP block), P model-matrix columns.
 *   - The parameter vector of the optimiser ("grad" layout, ggplvm.cu:109,154,265,311)
 *     is [log Omega (N) | log delta (p) | X (N*Q) | T (M*Q) | log rho (Q)].
 */
#ifndef GPL_H
#define GPL_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GPL_API __attribute__((visibility("default")))
#else
#define GPL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GPL_OK 0
#define GPL_ERR_ARG (-1)      /* bad argument or inconsistent sizes */
#define GPL_ERR_CUDA (-2)     /* CUDA runtime error */
#define GPL_ERR_ALLOC (-3)    /* device or host allocation failed */
#define GPL_ERR_STATE (-4)    /* call out of order (e.g. counts not loaded) */
#define GPL_ERR_NAN (-5)      /* NaN likelihood where the reference driver exits (ggplvm.cu:1182) */
#define GPL_ERR_FORMAT (-6)   /* malformed input data (level code out of range, bad CSR offsets) */
#define GPL_ERR_IO (-7)       /* file could not be read or written */
#define GPL_ERR_LIMIT (-8)    /* size beyond a fixed limit of the allocation-free entry point */
#define GPL_ERR_TIMEOUT (-9)  /* a bounded device wait ran out; the kernel gave up and the context stays usable */

#define GPL_PREC_FP64 0       /* plain double precision: the drop-in path */
/* The precision form (no reference counterpart): the Gram and the gradient contraction on
 * tensor cores (BF16 hi/lo products, FP32 runs folded into FP64) over the dense columns
 * whitened by the prior's Cholesky factor, everything else FP64, and one FP64-residual
 * refinement step on every per-gene solve. Objective within ~1e-7 of GPL_PREC_FP64 per
 * evaluation. */
#define GPL_PREC_BF16X3 1

typedef struct gpl_ctx gpl_ctx;

/* Creates a context on CUDA device `device`. `stream` is a cudaStream_t to run on, or NULL
 * for a context-owned stream. No reference counterpart (main's cudaMalloc block,
 * ggplvm.cu:1024-1060, happens in gpl_load_design once sizes are known). */
GPL_API int gpl_create(gpl_ctx** out, int device, void* stream);
GPL_API int gpl_destroy(gpl_ctx* ctx);
GPL_API const char* gpl_last_error(const gpl_ctx* ctx);
/* Selects GPL_PREC_FP64 (default) or GPL_PREC_BF16X3 for the following calls. */
GPL_API int gpl_set_precision(gpl_ctx* ctx, int precision);

/* Named integer options of a context (no reference counterpart; the reference hard-codes its
 * schedule). Unknown names and out-of-range values give GPL_ERR_ARG.
 *   "tc_grad"           precision form: the gradient contraction on tensor cores (1, default)
 *                       or in FP64 (0)
 *   "refine_steps"      precision form: FP64-residual refinement steps per solve (0..16, default 1)
 *   "tc_run"            precision form: K chunks an FP32 accumulator collects before its fold
 *                       into the FP64 sum (1..64, default 4)
 *   "tc_check"          read the tensor-core kernels' error flag after each of their launches
 *                       (1) or only when a result is read back (0, default)
 *   "tc_pair"           precision form: the two tensor-core contractions on CTA pairs (one
 *                       M = 256 MMA over two CTAs, each loading half of B) (1) or one CTA per
 *                       tile (0, default); the same sums in the same order
 *   "logdet_probe"      precision form: log det Psi_j corrected with a fixed probe vector per gene
 *                       and one application of the FP64 operator (1, default), so that the objective
 *                       moves with parameter changes too small to change the BF16 hi/lo operands of
 *                       the tensor-core Gram; 0: the tensor-core factor's log-determinant alone
 *   "ls_fp64"           precision form, in gpl_fit / gpl_fit_outer: a line search whose seven
 *                       tries all fail is repeated with the FP64 objective from the step's start
 *                       (the tensor-core Gram does not resolve parameter changes below about 2^-16
 *                       relative), and the fit goes on in the precision form from the point it
 *                       accepted (1); or the reference's rule, the last try and its stop test
 *                       (0, default). "ls_fp64_steps" (read only) counts the steps so repeated.
 *   "eta_tc"            the linear predictor z_i . beta_j of every cell and gene (W / nu, the
 *                       gradient's predictions, the refinement) on the FP64 tensor cores (1,
 *                       default) or as an FFMA tile GEMM (0); the two differ by rounding
 *   "pair_range_cells"  cells per range of the FP64 pair GEMMs (0, default: as many as 8 GiB
 *                       of pair products holds; smaller values exercise the multi-range path)
 *   "graph"             1: each objective evaluation and each gradient after it (in gpl_fit,
 *                       gpl_fit_outer, gpl_objective, gpl_evaluate, gpl_evaluate_device) runs as
 *                       a CUDA graph, captured on its first use and replayed after (one launch
 *                       per evaluation instead of one per kernel; the same kernels and results).
 *                       Not while profiling or tc_check is on. Reads back as 0 if the capture
 *                       was refused; the context then runs eagerly. Default 0.
 *   "graph_replays"     (read only) graph launches so far
 *   "fused_tail"        1: each IRLS sweep's per-gene tail (cholPsi, the solve and coefficient
 *                       update of getBetaPhi, getLkhdPois: ggplvm.cu:683-692, 418-464, 703-724)
 *                       runs as one persistent launch whose CTAs take genes from a queue ordered
 *                       by decreasing count (FP64 path, P <= 288; else the separate kernels).
 *                       Same results bit for bit. Default 0.
 *   "tail_ctas_per_sm"  CTAs per SM of that launch (1 or 2, default 2)
 *   "autotune"          1: the tile orders of the FP64 pair GEMMs and of the tensor-core
 *                       contractions and the CTAs per SM of the fused tail are chosen by timing
 *                       each candidate on the context's own
 *                       launches (every candidate gives the same bits); the choices are kept for
 *                       the process per problem shape. Graphs are captured once all are chosen.
 *                       Default 0. */
GPL_API int gpl_set_option(gpl_ctx* ctx, const char* name, int64_t value);
GPL_API int gpl_get_option(const gpl_ctx* ctx, const char* name, int64_t* value);

/* The autotuner's record of one choice ("pair_gram", "pair_v", "irls_tail", "tc_gram",
 * "tc_grad", "eta_tile"): *chosen = the chosen candidate value (-1 while open), cands[k] the candidate
 * values and best_ms[k] each one's best measured launch time (-1 untimed, -2 chosen from the
 * process-wide record without timing), up to cap entries; *n_cands the number of candidates
 * (0 if the choice never came up). No reference counterpart. */
GPL_API int gpl_tuning(gpl_ctx* ctx, const char* name, int32_t* chosen, int32_t* cands, double* best_ms, int cap,
                       int32_t* n_cands);

/* Gene-major CSR counts: replaces loadSparseMat + newSparseMatOnDevice
 * (SparseMat.cu:37-52,127-142). Gene j owns entries gene_ptr[j]..gene_ptr[j+1]-1.
 * Count matching keeps the reference's merge-walk rule (ggplvm.cu:505-511): within a
 * gene, entries are used in order while the cell index increases and stays below N; the
 * first out-of-order, duplicated or out-of-range index ends that gene's counts. */
GPL_API int gpl_load_counts(gpl_ctx* ctx, int N, int J, int64_t nnz, const int32_t* cell_idx, const int32_t* gene_ptr,
                    const double* counts);

/* Covariate DataFrame: replaces loadDataFrame(fname, M) + newDataFrameOnDevice
 * (DataFrame.cu:88-191). `n_var` file variables with level counts c[] (1 = numeric) and
 * widths v[], and the file body (numeric: double[N*v] column-major; categorical:
 * int32[N] level codes). The intercept and the M-column Knm block are added as in the
 * reference. Allocates the device state for N, J (counts must be loaded first), M, Q.
 * Level codes outside 0..c*v-1 are rejected (GPL_ERR_FORMAT); the reference reads
 * beyond the column block for them. */
GPL_API int gpl_load_design(gpl_ctx* ctx, int N, int n_var, const int32_t* c, const int32_t* v, const void* body,
                    int64_t body_bytes, int M, int Q);

/* Size factors ls[N] (ggplvm.cu:1019-1022,1062). */
GPL_API int gpl_set_size_factors(gpl_ctx* ctx, const double* ls);

/* dims[6] = N, J, M, P, p, Q (ggplvm.cu:966-984). */
GPL_API int gpl_dims(const gpl_ctx* ctx, int32_t* dims);

/* initParams (init.cu:27-48): delta = (1.5, 0.01.., 0.3), Omega = 1, phi = 1, rho = (5, 10..);
 * T dimension 0 equispaced on (0, 2 pi) as initTaWithPer (util.c:73-87), others 0. */
GPL_API int gpl_init_params(gpl_ctx* ctx);

/* readParams / writeParams without the file (util_cuda.cu:520-580): Omega[N], delta[p],
 * X[N*Q], T[M*Q], rho[Q], phi[J]. A NULL pointer keeps (set) or skips (get) that block. */
GPL_API int gpl_set_params(gpl_ctx* ctx, const double* Omega, const double* delta, const double* X, const double* T,
                   const double* rho, const double* phi);
GPL_API int gpl_get_params(gpl_ctx* ctx, double* Omega, double* delta, double* X, double* T, double* rho, double* phi);

/* GLM coefficients beta[P*J] (column j = gene j). The reference never writes beta out
 * (it is only printed, ggplvm.cu:1325); this is the added output. */
GPL_API int gpl_set_beta(gpl_ctx* ctx, const double* beta);
GPL_API int gpl_get_beta(gpl_ctx* ctx, double* beta);

/* getKernelMats + cholKmm + getKinvKmn (ggplvm.cu:1111-1113, kernel_funcs.cu:61-162). */
GPL_API int gpl_kernel_mats(gpl_ctx* ctx);

/* expandDelta_k + initPsi + initPsi2 + initBeta (ggplvm.cu:1134-1137, init.cu:125-221). */
GPL_API int gpl_glm_init(gpl_ctx* ctx);

/* getPsi alone (ggplvm.cu:621-680): every gene's Gram Z^T diag(W_j/Omega) Z + DeltaInv at the
 * current W, Omega and DeltaInv, both triangles, before any factorization. */
GPL_API int gpl_gram(gpl_ctx* ctx);

/* expandDelta_k alone (util_cuda.cu:249-269). */
GPL_API int gpl_expand_delta(gpl_ctx* ctx);

/* One IRLS sweep: getWForBeta, getPsi, cholPsi, getBetaPhi, getLkhdPois, collectLkhd
 * (ggplvm.cu:1156-1180) with damping index jtr; *lkhd receives the Poisson sum. */
GPL_API int gpl_irls_sweep(gpl_ctx* ctx, int jtr, double* lkhd);

/* The IRLS loop with the driver's stopping rule (ggplvm.cu:1152-1189): up to jtr_max
 * sweeps, stop at relative change < 1e-7. *n_sweeps gets the count. GPL_ERR_NAN where the
 * reference exits on a NaN likelihood. */
GPL_API int gpl_irls(gpl_ctx* ctx, int jtr_max, int* n_sweeps);

/* getOinvt, cholDeltaInv, getLkhd, collectLkhd (ggplvm.cu:1205-1211). */
GPL_API int gpl_objective_after_irls(gpl_ctx* ctx, double* lkhd);

/* One line-search evaluation of the objective (ggplvm.cu:1258-1277) into slot `slot`. */
GPL_API int gpl_objective(gpl_ctx* ctx, int slot, double* lkhd);

/* One gradient evaluation (ggplvm.cu:1215-1240); grad may be NULL (kept on the device). */
GPL_API int gpl_gradient(gpl_ctx* ctx, double* grad);

/* LBFGS (ggplvm.cu:865-934, util_cuda.cu:187-232) and Downdate (ggplvm.cu:818-859). */
GPL_API int gpl_lbfgs_update(gpl_ctx* ctx, int jtr, int rhoflag);
GPL_API int gpl_downdate(gpl_ctx* ctx, int jtr, double sr, int rhoflag);

/* getBetaFromTildeBeta (ggplvm.cu:394-402), with zeta = 0 (the driver never sets it). */
GPL_API int gpl_beta_from_tilde(gpl_ctx* ctx);

/* The driver's outer loop (ggplvm.cu:1146-1330): IRLS, objective, L-BFGS with backtracking
 * line search, under budgets itr_max (outer iterations) and lbfgs_budget (total L-BFGS
 * steps, <= 0 for none). stats[4] = outer iterations, IRLS sweeps, L-BFGS steps,
 * objective evaluations; trace gets the accepted objective values (<= trace_cap). */
GPL_API int gpl_fit(gpl_ctx* ctx, int itr_max, int lbfgs_budget, int32_t* stats, double* trace, int trace_cap);

/* One outer iteration of that loop, numbered itr (0-based; it selects JTRMAX 200 or 100,
 * rhoflag for itr > 20 and the long L-BFGS run at itr 30), ending with the beta revival
 * (ggplvm.cu:1317-1319). The CLI calls it to write X9.gz, phi.gz and Params9.bin after every
 * outer iteration as the reference driver does (ggplvm.cu:1301-1315). lbfgs_budget > 0 caps
 * this call's L-BFGS steps. stats[4] = IRLS sweeps, L-BFGS steps, objective evaluations,
 * trace entries written. GPL_ERR_NAN when the IRLS likelihood is NaN (the reference exits 1). */
GPL_API int gpl_fit_outer(gpl_ctx* ctx, int itr, int lbfgs_budget, int32_t* stats, double* trace, int trace_cap);

/* One objective+gradient evaluation at host parameters (the unit of the throughput
 * metric): params = [Omega (N) | delta (p) | X (N*Q) | T (M*Q) | rho (Q)] in natural
 * scale (n_params = N + p + N*Q + M*Q + Q); the objective goes to *lkhd and the gradient
 * (optimiser layout above, N + p + N*Q + M*Q + Q values) to grad. W, nu, phi and beta stay
 * as the last IRLS phase left them, as inside the reference's L-BFGS loop. This is the
 * line-search evaluation followed by the gradient (ggplvm.cu:1258-1277 then 1215-1240). */
GPL_API int gpl_evaluate(gpl_ctx* ctx, const double* params, int64_t n_params, double* lkhd, double* grad);

/* Genotype score statistics against the fitted model: getScoreStats of the reference's
 * differential-expression driver (ggplvm_de.cu:489-535, run after its fit at :1205-1209).
 * G[N*L] holds L genotype columns (column-major, e.g. dosages 0/1/2); S[J*L] receives
 * S[j + l*J] = s / sqrt(phi_j v) with s = sum_i g_il/Omega_i (y_ij - W_ij) and
 * v = g^T diag(W_j/Omega) g - t^T Psi_j^{-1} t, t = Z^T diag(W_j/Omega) g, at the current W,
 * phi and factored Psi_j (call after gpl_fit, an IRLS phase or an objective). */
GPL_API int gpl_score_stats(gpl_ctx* ctx, int L, const double* G, double* S);

/* Cis genotype statistics per (gene, variant): getScoreStats' efficient score (ggplvm_de.cu:489-535)
 * for a separate set of V variants per gene whose dosages are per donor (every cell carries its
 * donor's). dosages[(d * J + j) * V + v] (int8, 0/1/2) is donor d's dosage of gene j's variant v;
 * the donor is design variable donor_var (0-based among the file variables; categorical, with
 * n_donors levels, handled through cell groups). S[j + v*J] = s / sqrt(phi_j v) as gpl_score_stats
 * defines s and v for the column g_i = dosage of cell i's donor, and LR[j + v*J] (may be NULL)
 * = S^2, the likelihood ratio of the IRLS working model for adding that column with every other
 * coefficient re-estimated. At the current W, nu, phi and factored Psi (after gpl_fit, an IRLS
 * sweep or an objective). Every sum over cells runs over the cell groups. */
GPL_API int gpl_cis_stats(gpl_ctx* ctx, int donor_var, int n_donors, int V, const int8_t* dosages, double* S,
                          double* LR);

/* The model comparison of the differential-expression driver (ggplvm_de.cu:1067-1207), which
 * refits the GLM part by IRLS at the fitted Omega, delta, X, T and rho for several GPs and
 * keeps each model's per-gene log-likelihood ("BFs", J x (Q+2), written to BFs_de.gz). One
 * context holds one model family: load the design with the model's M (Mfull, Mredc, or any M
 * >= 1 for the null model), set the parameters, then select the model and run its IRLS.
 *
 * gpl_de_model selects the GP (getKernelMats at ggplvm_de.cu:1118-1128 and the kernel
 * matrices after it) and switches the context's IRLS to the DE driver's kernels (getWForBeta,
 * getBetaPhi, getZeta, getLkhdPois of ggplvm_de.cu):
 *   GPL_DE_NULL  no GP, the null model Z0 (the GP block is held inert: Knm = 0, Kmm = I,
 *                titsias = 0, its coefficients stay 0 and it is left out of the likelihood).
 *                As the reference's loader (DataFrame.cu:112-113, 131), the first cell of the
 *                last design variable reads 199.0 while this model is selected, when that
 *                variable is numeric (for a categorical one the reference reads level codes
 *                out of range; the loaded codes are kept).
 *   GPL_DE_FULL  the GP over all latent dimensions (T as set: the fitted Mfull points)
 *   q in [0, Q)  the GP over latent dimension q alone (getKernelMatsWithPerSpecificLV,
 *                kernel_funcs.cu:101-135; T as set: the equispaced Mredc points, see
 *                gpl_ta_equispaced)
 *
 * gpl_de_irls runs that model's GLM initialisation (initPsi, initPsi2, initBeta, getZeta)
 * and IRLS sweeps until the relative change of the summed likelihood is below tol (the
 * reference: 1e-5 for the null model, 1e-8 for the others), a NaN/inf sum, or jtr_max sweeps
 * (the reference: 1000). phi carries in from the context (the reference starts at 1 and
 * keeps each model's final phi for the next model's zeta). lkhds[J] receives the per-gene
 * log-likelihoods, *sweeps the number of sweeps, trace the summed likelihood of every sweep
 * (up to trace_cap). Always FP64. */
#define GPL_DE_NULL (-2)
#define GPL_DE_FULL (-1)
GPL_API int gpl_de_model(gpl_ctx* ctx, int model);
GPL_API int gpl_de_irls(gpl_ctx* ctx, int jtr_max, double tol, double* lkhds, int32_t* sweeps, double* trace,
                        int trace_cap);

/* The variance-component driver (ggplvm_delta.cu:784-1097; the reference's main does not
 * compile): refits the prior variance delta[p-2] of the design's last variable (the genotype,
 * when Z.bin ends with it) at the parameters set, alternating IRLS phases in the DE driver's
 * forms (at most 30 sweeps, relative change 1e-5) with L-BFGS on log delta[p-2] under the
 * Laplace objective with N(0, 1) priors on X and T (dimensions >= 1) and an inverse-gamma
 * (30, 30) prior on Omega, at most lbfgs_max steps per outer iteration (the reference: 100),
 * itr_max outer iterations (the reference: 100). The reference's main reads params.bin with
 * p - 1 deltas, sets delta[p-2] to its --init-deltaG (default 0.01) and leaves delta[p-1] at
 * initParams' 0.3; callers that must match it set delta so. dg[itr] receives delta[p-2] and
 * obj[itr] the objective after each outer iteration (up to cap), *n_itr the iterations run.
 * Always FP64; the context's IRLS forms are restored afterwards. */
GPL_API int gpl_vc_fit(gpl_ctx* ctx, int itr_max, int lbfgs_max, double* dg, double* obj, int cap, int32_t* n_itr);

/* initTaEquispaced (util.c:57-71): M x Q inducing points (column-major), dim 0 equispaced on
 * (0, 2 pi), dims >= 1 on (-3, 3): the DE driver's points for the per-dimension models. */
GPL_API void gpl_ta_equispaced(int M, int Q, double* T);

/* The same evaluation at the parameters already on the device, enqueued on the context's
 * stream without host copies or synchronisation (device-resident throughput). The objective
 * lands in slot 1 of the trace; read it with gpl_get("lkhd_dev") or the next evaluate. */
GPL_API int gpl_evaluate_device(gpl_ctx* ctx);

/* Copies a named state buffer out in the reference layout (names as the reference's
 * variables: "Knm", "Kmm", "Kinv", "KinvKmn", "titsias", "W", "Nu", "Psi", "PsiInv",
 * "DeltaInv", "Beta", "tBeta", "phi", "lkhds", "lkhd", "C1", "C2", "grad", "ss",
 * "Omega", "delta", "X", "T", "rho"). *len gets the element count; out may be NULL. */
GPL_API int gpl_get(gpl_ctx* ctx, const char* name, double* out, int64_t cap, int64_t* len);

/* Per-kernel device time since the last reset: names[i] with total milliseconds and
 * launch counts, recorded with CUDA events on the context's stream when enabled. */
GPL_API int gpl_profile_enable(gpl_ctx* ctx, int on);
GPL_API int gpl_profile_reset(gpl_ctx* ctx);
GPL_API int gpl_profile_read(gpl_ctx* ctx, const char* name, double* total_ms, int64_t* launches);
GPL_API int gpl_launch_count(const gpl_ctx* ctx, int64_t* launches);

/* Kernel matrices without any device allocation. This entry point has no counterpart in the
 * reference; it serves callers that cannot allocate device memory: code enqueueing work while
 * a stream is captured into a CUDA graph, real-time loops that forbid allocation after
 * start-up, and plugins whose host framework owns all device memory. Every pointer is DEVICE
 * memory owned by the caller: X (N x Q), T (M x Q), rho (Q) in, Knm (N x M, cell fastest),
 * KinvKmn (N x M, cell fastest: the transpose of the reference's M x N buffer) and titsias (N)
 * out, computed as gpl_kernel_mats computes them. The M x M work matrix lives in a fixed
 * 512 KiB array inside the library (M <= GPL_NOALLOC_MAX_M, else GPL_ERR_LIMIT), shared by all
 * calls on a device: calls that overlap on the GPU race, so serialise them. Each call outside
 * stream capture looks the array's device address up (with the caller's device current) and
 * remembers it; a call under capture uses the remembered one, so make one call on the device
 * before any capture (GPL_ERR_STATE otherwise). stream: a cudaStream_t or NULL for the default
 * stream; the call only enqueues work and reports its own launches' status (GPL_ERR_CUDA), not
 * errors of earlier work. A Kmm that is not positive definite zero-fills its factor as the
 * reference's choldc does: KinvKmn and titsias are then inf/NaN and the call returns GPL_OK. */
#define GPL_NOALLOC_MAX_M 256
GPL_API int gpl_kernel_mats_noalloc(int N, int M, int Q, const double* X, const double* T, const double* rho,
                                    double* Knm, double* KinvKmn, double* titsias, void* stream);

/* Failure detection of the device waits: runs the bounded wait that the tensor-core kernels use
 * on every barrier, against a barrier whose phase nothing completes, with a limit of limit_ns
 * (> 0). The wait gives up, the kernel records it and returns, and this call reports
 * GPL_ERR_TIMEOUT, exactly as a tensor-core kernel whose wait ran out would; the context stays
 * usable. No reference counterpart (the reference's kernels never wait). */
GPL_API int gpl_wait_probe(gpl_ctx* ctx, int64_t limit_ns);

/* Per-cell placement at a fitted model: the per-cell slice of the reference's L-BFGS phase
 * (ggplvm.cu:1214-1301) for cells whose counts and covariates this context holds, with every
 * gene's coefficients (gpl_set_beta: the fit's beta), T, rho and delta (gpl_set_params) fixed.
 * Each cell's X_i maximises its Poisson log-probability over all genes (getLkhdPois,
 * ggplvm.cu:703-724, with getWForBeta's mean W = s exp(z(X_i).beta + wt delta_GP titsias_i),
 * ggplvm.cu:468-514, and the log(y!) terms) plus the N(0, 1) prior on latent dimensions >= 1 of
 * the reference's variance-component driver (ggplvm_delta.cu), by its own L-BFGS under the
 * reference's step rules (lbfgs,
 * util_cuda.cu:187-232; the backtracking of ggplvm.cu:1278-1289), `iters` steps. X (N x Q,
 * column-major) is the start in and the result out; obj[N] (may be NULL) the final per-cell
 * objectives; stats[3] (may be NULL) = steps, objective evaluations, line-search tries. Uses the
 * context's W, Nu and scratch buffers (an IRLS state there is overwritten). */
GPL_API int gpl_place_cells(gpl_ctx* ctx, int iters, double* X, double* obj, int32_t* stats);

/* The start of a fit from the loaded counts and size factors, computed on the device: X (N x Q,
 * column-major) = the leading Q principal component scores of log1p(y / s) (every gene, centred;
 * subspace iteration with pca_iters products by the gene covariance), each scaled to unit
 * variance; T (M x Q) = k-means centres of X after kmeans_iters Lloyd steps from M distinct
 * seeded cells. The reference reads both from files (X: argv[4], ggplvm.cu:1019-1022; T:
 * initTaWithPer or --init-params, ggplvm.cu:1011,1103-1106) and ships unused PCA kernels
 * (init.cu:329-357). Uses the context's scratch buffer. */
GPL_API int gpl_init_latent(gpl_ctx* ctx, int pca_iters, int kmeans_iters, uint64_t seed, double* X, double* T);
/* The per-cell objective above at X (N x Q) into obj[N] and, if grad is not NULL, its gradient
 * d obj_i / d X_iq into grad (N x Q, column-major). */
GPL_API int gpl_cell_objective(gpl_ctx* ctx, const double* X, double* obj, double* grad);

/* ---- The amortised encoder (no reference counterpart) -----------------------------------------
 * The reference places every cell by L-BFGS on its latent coordinates (ggplvm.cu:1214-1301). The
 * encoder learns that placement: an MLP n_in -> hidden -> hidden -> 2q (GELU; mean and
 * log-variance of the q latent coordinates) over log1p(y / s) of n_in selected genes, trained on
 * (cell profile, fitted X) pairs of a plain fit, with FP32 master weights, Adam, and BF16
 * products on the tensor cores. Its predictions start (or replace) the per-cell refinement
 * (gpl_place_cells). One encoder runs on one device and stream; hidden is a multiple of 128,
 * 2q <= 64, batch a multiple of 128. Host arrays throughout; X is N x q column-major. */
typedef struct gpl_enc gpl_enc;
GPL_API int gpl_enc_create(gpl_enc** out, int device, void* stream, int n_in, int hidden, int q, int batch,
                           uint64_t seed);
GPL_API int gpl_enc_destroy(gpl_enc* enc);
GPL_API const char* gpl_enc_last_error(const gpl_enc* enc);
/* A cell set's features (which = 0: training, 1: evaluation) from gene-major CSR counts (the
 * matched prefix of each gene, as gpl_load_counts reads them), size factors ls[N] and the n_in
 * feature genes; cell_of_row (a permutation of 0..N-1, or NULL) orders the rows (training
 * batches are runs of rows). */
GPL_API int gpl_enc_set_cells(gpl_enc* enc, int which, int N, int J, int64_t nnz, const int32_t* cell_idx,
                              const int32_t* gene_ptr, const double* counts, const double* ls, const int32_t* genes,
                              const int32_t* cell_of_row);
GPL_API int gpl_enc_set_targets(gpl_enc* enc, const double* X);  /* training targets, N x q */
/* Parameters as one float array: W1 [hidden][n_in], b1, W2 [hidden][hidden], b2, W3 [2q][hidden],
 * b3 (row-major); gpl_enc_n_params gives its length. */
GPL_API int gpl_enc_n_params(const gpl_enc* enc, int64_t* n);
GPL_API int gpl_enc_get_params(gpl_enc* enc, float* params);
GPL_API int gpl_enc_set_params(gpl_enc* enc, const float* params);
/* The mean loss of training batch `batch_index` (rows batch_index * batch ..) and every
 * parameter's gradient (same layout as the parameters), without updating anything. */
GPL_API int gpl_enc_grads(gpl_enc* enc, int batch_index, double* loss, float* grads);
/* `epochs` passes over the whole training batches in a seeded random order, one Adam step (lr)
 * per batch; loss_per_epoch[e] (may be NULL) = the epoch's mean loss. */
GPL_API int gpl_enc_train(gpl_enc* enc, int epochs, double lr, uint64_t seed, double* loss_per_epoch);
/* Predicted mean and log-variance (N x q column-major, either may be NULL) of a cell set. */
GPL_API int gpl_enc_predict(gpl_enc* enc, int which, double* mean, double* logvar);
GPL_API int gpl_enc_launch_count(const gpl_enc* enc, int64_t* launches);

/* Synchronises the context's stream. */
GPL_API int gpl_sync(gpl_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
