// Internal state and helpers of libgpl_b200 (not part of the C ABI).
//
// Device data layout (HBM), all double precision unless noted; ldN = N rounded up to a
// multiple of 32 so every column starts on a 256-byte boundary:
//   Dm       ldN x n_d the dense model-matrix columns, in model order: intercept, numeric
//                      covariates, any categorical one-hots kept dense, and last the M Knm
//                      columns (getKernelMats writes them in place, as the reference does);
//                      dcol[a] is the model column of dense column a
//   groups   categorical variables handled by groups: every cell belongs to the group of
//            its combination of levels; gid (cell -> group), glev (group -> levels), the
//            cells of each group (gcells, gstart) and per-variable level codes
//   gsum     J x n_grp x (n_d + 1): per (gene, group) weighted sums of the dense columns
//            (Gram) or, in the gradient, the categorical blocks of Psi^{-1}
//   W        ldN x (J+1) gene-major weights; column J holds Oinvt (ggplvm.cu:292)
//   Nu       ldN x J   working responses
//   Psi      J x (P x P) per-gene Gram, full symmetric, then Cholesky factor in the lower
//                      triangle (the reference's in-place layout)
//   PsiInv   J x (P x P) explicit inverses
//   Beta, tBeta  P x J
//   KinvKmn  M x N     (reference layout)
//   scratch  ldN x J   per-(cell, gene) intermediates
//   counts   CSR (int32 cells, int64 offsets, double values) + per-gene valid prefix length
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <deque>
#include <string>
#include <vector>

#include "gpl.h"

namespace gpl {

constexpr double kWt = 0.1;     // Titsias weight (ggplvm.cu:20)
constexpr double kIgap1 = 100;  // inverse-gamma prior shape+1 on Omega (ggplvm.cu:21)
constexpr double kIgb = 100;    // inverse-gamma prior scale on Omega (ggplvm.cu:22)
constexpr int kHist = 10;       // L-BFGS memory (ggplvm.cu:872)
constexpr int kLkhdSlots = 50000;

struct Ctx;

// Sum of a per-block partial array in a fixed order (deterministic reductions).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Operands, partial sums and TMA descriptors of the tensor-core contractions (k_tc.cu).
// Column-pair FP64 GEMM state (k_dgemm.cu): the pair list (a <= b over the dense columns),
// 1/Omega, the gathered Psi^{-1} pairs per gene and a range of V rows.
struct PairState {
  bool ready = false, wide = false;  // wide: a cell's V row exceeds k_v_to_u's shared memory
  int n_pairs = 0, pairs_pad = 0, cpad = 0, v_cells = 0;
  int smem_gram = 0, smem_v = 0, smem_vu = 0;
  int2* pairs = nullptr;
  double *rOm = nullptr, *Sp = nullptr, *V = nullptr;
  double* Gacc = nullptr;  // pairs x genes Gram accumulator when the cells need several ranges
};

struct TcState {
  bool ready = false;
  int cpad = 0, chunks_cells = 0, gram_tiles_n = 0, Jpad = 0;
  int n_pairs = 0, pair_tiles = 0;
  int smem_gram = 0, smem_gram2 = 0, smem_whiten = 0, run = 4;  // run: K chunks per FP32 accumulator run
  __nv_bfloat16 *whi = nullptr, *wlo = nullptr;   // w = W/Omega, gene rows x cpad
  __nv_bfloat16 *ahi = nullptr, *alo = nullptr;   // whitened pair products, pair rows x cpad
  __nv_bfloat16 *shi = nullptr, *slo = nullptr;   // whitened inverse pairs, pair rows x Jpad
  __nv_bfloat16 *ohi = nullptr, *olo = nullptr;   // (W/Omega)^T, cpad x Jpad
  float* DtC = nullptr;                           // whitened dense columns (cell fastest), FP32
  double* DwC = nullptr;                          // the same in FP64, ld ldN
  double *Lw = nullptr, *Gt = nullptr, *Tt = nullptr;  // prior factor, whitened Gram / inverse, product
  int2* pairs = nullptr;
  int* err = nullptr;
  CUtensorMap map_whi, map_wlo, map_ahi, map_alo, map_shi, map_slo, map_ohi, map_olo;
  CUtensorMap map_whi64, map_wlo64, map_ohi64, map_olo64;  // 64-row boxes: the CTA-pair kernel's B halves
  double* probe = nullptr;  // P x J fixed Rademacher probes of the log-determinant correction
};

// One open or settled choice of the autotuner (tune.cu): candidate values, each one's best
// time so far and number of timings, the launches whose events are not read yet.
struct Tunable {
  struct Pending {
    int cand;
    cudaEvent_t a, b;
  };
  std::string name;
  std::vector<int> cands;
  std::vector<double> best_ms;
  std::vector<int> n;
  std::vector<Pending> pending;
  int best = -1, cur = 0;
  bool from_cache = false;
};

constexpr int kLvAll = -1;   // kernel over every latent dimension
constexpr int kLvNone = -2;  // no GP (inert GP block): the DE driver's null model

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int precision = GPL_PREC_FP64;
  bool tc_grad = true;     // precision form: the gradient contraction on tcgen05 too (else FP64 DMMA)
  int refine_steps = 1;              // precision form: FP64-residual refinement steps per solve
  const double* zt_u_src = nullptr;  // u of Z^T diag(W/Omega) u when not nu (set during a refinement)
  double *rres = nullptr, *bx = nullptr;  // refinement residual and product, P x J
  double* rphi = nullptr;                 // 1/phi, refreshed before each gradient
  // the differential-expression driver's model comparison (ggplvm_de.cu)
  int kernel_lv = kLvAll;  // GP over all latent dimensions, one dimension (>= 0), or none (kLvNone)
  bool de = false;         // IRLS in the DE driver's forms (W/nu, beta/phi, zeta, per-gene likelihood)
  bool vcomp = false;      // the variance-component driver's likelihood constants (ggplvm_delta.cu)
  double* e0 = nullptr;    // z_i . zeta per cell (DE working response)
  double* zeta = nullptr;  // the DE driver's zeta (P)
  int de_quirk_col = -1;   // dense column whose first cell holds the null model's loader value
  double de_quirk_orig = 0.0;
  // options (gpl_set_option)
  bool tc_check = false;      // read the tensor-core error flag after every tensor-core launch
  int tc_run = 4;             // precision form: K chunks per FP32 accumulator run before the FP64 fold
  bool tc_pair = false;       // precision form: the tensor-core contractions on CTA pairs (k_tc_gram2)
  bool ls_fp64 = false;       // precision form: repeat a failed line search with the FP64 objective
  int64_t ls_fp64_steps = 0;  // steps so repeated
  bool logdet_probe = true;   // precision form: the probe correction of log det Psi (k_lkhd.cu)
  int64_t pair_range_cells = 0;  // cells per range of the pair GEMMs (0: as many as 8 GiB holds)
  // CUDA graphs of one objective evaluation and of the gradient that follows it (option
  // "graph"): captured on first use, replayed after; dropped whenever a buffer they captured
  // is reallocated or an option or the precision changes (graph_reset)
  bool use_graph = false;
  // the IRLS sweep's per-gene tail (Cholesky, solve, coefficient update, Poisson likelihood) as
  // one persistent launch over a gene queue (option "fused_tail"), with this many CTAs per SM
  bool fused_tail = false;
  // the linear predictor on the FP64 tensor cores (option "eta_tc", k_eta_dmma; the default)
  bool eta_tc = true;
  int tail_ctas_per_sm = 2;
  int sm_count = 148;
  int* gene_order_d = nullptr;   // genes by decreasing matched count (the queue's order)
  int* queue_head_d = nullptr;   // the queue's head, reset before each launch
  // the autotuner (option "autotune"): open and settled choices (tune.cu)
  bool autotune = false;
  bool capturing = false;  // a stream capture is in progress (no timing, no lazy allocation)
  std::deque<Tunable> tun;
  cudaGraphExec_t g_obj = nullptr, g_grad = nullptr;
  int64_t g_obj_kernels = 0, g_grad_kernels = 0, graph_replays = 0;
  std::string graph_note;  // why capture was given up, when it was
  std::string err;

  // sizes
  int N = 0, J = 0, M = 0, Q = 0, P = 0, p = 0, n_var = 0;
  int ldN = 0;
  int64_t nnz = 0;
  bool have_counts = false, have_design = false;

  // host copies of the model-matrix metadata (DataFrame.cu:96-134)
  std::vector<int> vc, vv, nh, mc, mv, mk;

  // dense columns and categorical groups
  int n_d = 0, dg0 = 0;             // dense columns; dense index of the first Knm column
  std::vector<int> dcol;            // model column of each dense column (ascending)
  int n_cv = 0, n_grp = 0;          // grouped categorical variables; groups
  std::vector<int> cv_nh, cv_nlev;  // first model column and level count of each grouped variable
  int *dcol_d = nullptr, *cv_nh_d = nullptr, *cv_nlev_d = nullptr, *gid_d = nullptr, *glev_d = nullptr;
  int *gcells_d = nullptr, *gstart_d = nullptr, *codes_d = nullptr;
  int* gpos_d = nullptr;  // position of each cell in the group order (the inverse of gcells_d)
  double* lvt = nullptr;  // J x n_grp: per gene and cell group, the sum of its levels' coefficients
  double* cellfac = nullptr;  // 3 x ldN: exp(dgp t_i wt), dgp t_i wt and log s_i of the W / Nu pass
  // levels of the grouped variables: model column, variable, and the groups at that level
  // (ascending) as offsets into a list
  int n_lvl = 0;
  int *lvl_cc_d = nullptr, *lvl_v_d = nullptr, *lvl_ptr_d = nullptr, *lvl_grp_d = nullptr;
  int2* hk_tiles_d = nullptr;       // (group, first row) of every 64-cell tile of the group lists
  int n_hk_tiles = 0;
  int2* hk_tiles128_d = nullptr;    // the same for 128-cell tiles
  int* hk_cells_d = nullptr;        // the cell of each slot of those tiles (-1 past the group)
  int* hk_pos_d = nullptr;          // the same slots as positions in group order (-1 past the group)
  // cells in group order (the cells of each group contiguous): W (refreshed with W), the dense
  // columns and 1/Omega (refreshed per use), so that the group-sum GEMMs read contiguous rows
  double *Wg = nullptr, *Dg = nullptr, *rOmg = nullptr;
  int n_hk_tiles128 = 0;
  double* part = nullptr;           // split-K partial sums
  size_t part_n = 0;
  double *Dm = nullptr, *gsum = nullptr, *gT = nullptr, *HK = nullptr;

  // device buffers
  double *Z = nullptr, *W = nullptr, *Nu = nullptr, *Psi = nullptr, *PsiInv = nullptr;
  double *Beta = nullptr, *tBeta = nullptr, *scratch = nullptr, *U = nullptr;
  double *Kmm = nullptr, *Kinv = nullptr, *KinvKmn = nullptr, *titsias = nullptr, *DeltaInv = nullptr;
  double *Omega = nullptr, *delta = nullptr, *X = nullptr, *T = nullptr, *rho = nullptr, *phi = nullptr;
  double *ls = nullptr, *lkhds = nullptr, *lkhd_dev = nullptr;
  double *grad = nullptr, *grad0 = nullptr, *ss = nullptr, *SS = nullptr, *XX = nullptr;
  double *gdtmp = nullptr, *C1 = nullptr, *C2 = nullptr, *grtmp = nullptr, *KmmInv = nullptr;
  double *bvec = nullptr;     // P x J right-hand sides Z^T diag(W/Omega) nu
  double *sol = nullptr;      // P x J solutions Psi^{-1} bvec
  double *red = nullptr;      // reduction partials
  double *lb_work = nullptr;  // L-BFGS scalars
  int *mc_d = nullptr, *mv_d = nullptr, *mk_d = nullptr, *nh_d = nullptr;
  int32_t* cell = nullptr;    // CSR cell indices
  int64_t* gptr = nullptr;    // CSR offsets (J+1)
  int32_t* gvalid = nullptr;  // per gene: entries matched by the reference's merge walk
  double* cnt = nullptr;      // CSR values
  int64_t tot_max = 0;

  // host mirror of the objective trace (lkhd_d in the reference, ggplvm.cu:1052)
  std::vector<double> lkhd;

  TcState tc;
  PairState pr;

  // profiling
  bool prof = false;
  struct ProfRec {
    std::string name;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> prof_pending;
  std::vector<std::pair<std::string, std::pair<double, int64_t>>> prof_total;
  std::vector<cudaEvent_t> event_pool;
  int64_t launches = 0;
};

// Throws-free error plumbing: every CUDA call goes through check().
bool check(Ctx* c, cudaError_t e, const char* what);
#define GPL_TRY(c, expr)                                    \
  do {                                                      \
    if (!::gpl::check((c), (expr), #expr)) return GPL_ERR_CUDA; \
  } while (0)
#define GPL_LAUNCHED(c, name)                                                          \
  do {                                                                                 \
    (c)->launches++;                                                                   \
    if (!::gpl::check((c), cudaGetLastError(), name)) return GPL_ERR_CUDA;            \
  } while (0)

// Scoped profiling range on the context stream.
struct ProfScope {
  Ctx* c;
  const char* name;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(Ctx* c_, const char* n);
  ~ProfScope();
};

// Drops the captured evaluation graphs (before any buffer they reference is freed or resized).
void graph_reset(Ctx* c);

// The autotuner (tune.cu). tune_pick returns the candidate value for this launch (`fallback`
// when tuning is off) and, while the choice is open, the Tunable to time the launch with a
// TuneScope around it; tune_harvest reads finished timings (after a host synchronisation);
// tune_settled: no choice of the context is open.
int tune_pick(Ctx* c, const char* name, const std::vector<int>& cands, int fallback, Tunable** slot);
Tunable* tune_find(Ctx* c, const char* name);
void tune_harvest(Ctx* c);
bool tune_settled(const Ctx* c);
bool tune_settled_for_graphs(const Ctx* c);  // the choices inside a captured evaluation are made
void tune_release(Ctx* c);
struct TuneScope {
  Ctx* c;
  Tunable* t;
  cudaEvent_t a = nullptr, b = nullptr;
  TuneScope(Ctx* c_, Tunable* t_);
  ~TuneScope();
};

inline int64_t tot_len(const Ctx* c, int rhoflag) {
  return (int64_t)c->N + c->p + (int64_t)c->N * c->Q + (int64_t)c->M * c->Q + rhoflag;
}
inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// ---- launchers (one per kernel family; each returns GPL_OK or an error code) ----------
// k_kmats.cu
int launch_kernel_mats(Ctx* c);          // Knm into Z, Kmm, Kinv copy, chol(Kinv), KinvKmn, titsias
int launch_kernel_mats_lv(Ctx* c, int lv);  // the same over latent dimension lv alone, all (kLvAll), none (kLvNone)
int launch_expand_delta(Ctx* c);         // DeltaInv (upper + diag)
int launch_chol_single(Ctx* c, double* A, int n);  // choldc on one n x n matrix
// k_groups.cu
int launch_group_sums(Ctx* c, int mode);  // 0: S (W/Omega); 1: S unweighted (gene 0); 2: T of y0; 3: T of nu;
                                          // 4: T of a per-cell u (zt_u_src)
int launch_assemble_psi(Ctx* c, int J);   // categorical rows/columns of Psi from the group sums
int launch_assemble_b(Ctx* c, double* out);  // categorical entries of Z^T u (P x J) from the group sums
int launch_group_tables(Ctx* c);          // per (gene, group) categorical blocks of Psi^{-1}
int launch_hk(Ctx* c);                    // HK[i] = sum_j O_ij [h_{j,g(i)} | kappa_{j,g(i)}]
int launch_group_order(Ctx* c, const double* src, int ncols, double* dst);  // dst[col][pos] = src[col][cell(pos)]
// k_gemm.cu
int launch_w_nu(Ctx* c);                 // W, Nu from Beta (getWForBeta)
// out = z_i . B_j (ldN x J, cell fastest) on the FP64 tensor cores (k_dgemm.cu)
int launch_eta_dmma(Ctx* c, const double* B, double* out);
// row stride of the per-group level sums (groups x genes): J rounded up to even
inline int lvt_ld(int J) { return J + (J & 1); }
int launch_zt_u(Ctx* c, int mode);       // bvec = Z^T u; mode 0: u = W/Omega*Nu; 1: init response
int launch_zt_u_ex(Ctx* c, int mode, const double* u, double* out);  // the same for another u / output;
                                                                      // mode 2: u is one value per cell
int solve_refined(Ctx* c, const double* b, double* x, bool dinv_factored = false);  // Psi_j x = b; FP64-residual
                                                        // refinement in the precision form
int launch_init_response(Ctx* c);        // scratch = log((y+0.05)/ls) or log(0.05/ls)
int launch_zbeta(Ctx* c, const double* B, double* out);  // out[ldN x J] = Z * B
int launch_eta_one(Ctx* c, const double* b, double* out);  // out[N] = Z * b for one coefficient vector
int launch_c1_tn(Ctx* c);                // C1 partial from tn/phi and tBeta GP block
// k_gram.cu
int launch_gram(Ctx* c, bool unweighted);  // Psi (full symmetric) = Z^T diag(W/Omega) Z + DeltaInv
int launch_chol_batched(Ctx* c, double* A, int n, int batch, int64_t stride);
int launch_solve_batched(Ctx* c, const double* L, int n, int64_t lstride, const double* B, int64_t bstride,
                         double* X, int64_t xstride, int batch);
int launch_inverse_batched(Ctx* c);      // PsiInv from Psi's factor
int launch_potrf_panels(Ctx* c, double* A, int n, int batch, int64_t stride);  // 32-column panels, DMMA
int launch_inverse_panels(Ctx* c);       // the same in 32-column panels with DMMA block products
int launch_irls_tail(Ctx* c, int jtr, int ctas_per_sm);  // persistent per-gene IRLS tail; GPL_ERR_ARG:
                                                          // P beyond the panel Cholesky's range
int launch_inverse_single(Ctx* c, const double* L, int n, double* tmp, double* out);
int launch_cholinv_exact(Ctx* c, const double* L, int n, double* out);  // cholsl order, no FMA
cudaError_t launch_chol_exact_raw(cudaStream_t st, double* A, int n);  // the launch's own status
int launch_kernel_mats_raw(cudaStream_t st, int N, int M, int Q, const double* X, const double* T,
                           const double* rho, double* Knm, double* KinvKmn, double* titsias, double* Lwork);
// k_tc.cu (precision form)
int launch_pair_gram(Ctx* c);             // dense block of every Psi_j, FP64 DMMA over column pairs
int launch_pair_uq(Ctx* c);               // U = sum_j O_ij S_j[DD] d_i, FP64 DMMA over column pairs
void pair_release(Ctx* c);
int pair_prepare(Ctx* c);                 // column-pair list, 1/Omega, gathered S pairs, V rows
int recip_omega(Ctx* c, const double** rOm);  // 1/Omega (0 past N), refreshed on every call
int dgen_zt_u(Ctx* c, int mode, const double* u, double* out);          // DMMA forms of the cell x gene GEMMs (k_dgen.cu);
int dgen_c1_tn(Ctx* c);                   // GPL_ERR_ARG when the dense columns exceed one tile
int dgen_group_sums(Ctx* c, int mode);
int dgen_hk(Ctx* c);
int dgen_weighted_colsums(Ctx* c, const double* G2, int n2, double* out);  // out[j + c*J] = sum_i W_ij G2[c][i]
int launch_score_stats(Ctx* c, int L, const double* G, double* S, double* scratch);  // device G (N x L) -> S (J x L)
int dgen_unwhiten(Ctx* c, const double* Gt, double* Tt, const double* Lw);  // Psi_DD = L G L^T + DeltaInv
int dgen_whiten_inverse(Ctx* c, const double* Lw, double* Tt, double* St);  // S~ = L^T S_DD L per gene
int launch_v_to_u_cells(Ctx* c, int c0, int c1, const double* D);  // U from the V rows of cells [c0, c1)
int launch_tc_gram(Ctx* c);               // dense block of every Psi_j on tensor cores
int launch_tc_grad(Ctx* c);               // U = sum_j O_ij S_j[DD] d_i on tensor cores
int tc_error_flag(Ctx* c);                // GPL_ERR_TIMEOUT if a tensor-core kernel gave up waiting
int wait_probe(Ctx* c, int64_t limit_ns); // the bounded wait against a barrier nothing completes
// k_cis.cu (per-gene cis genotype statistics through donor-level group sums)
int cis_stats(Ctx* c, int donor_var, int n_donors, int V, const int8_t* dos_host, double* S_host, double* LR_host);
// k_init.cu (the start: PCA of log1p(y / s) and k-means inducing points)
int init_latent(Ctx* c, int pca_iters, int kmeans_iters, uint64_t seed, double* X_host, double* T_host);
// k_place.cu (per-cell placement at a fitted model)
int place_cells(Ctx* c, int iters, double* X_host, double* obj_host, int32_t* stats);
int cell_objective(Ctx* c, const double* X_host, double* obj_host, double* grad_host);
void tc_release(Ctx* c);
// k_lkhd.cu
int launch_oinvt(Ctx* c);
int launch_beta_phi(Ctx* c, int jtr);
int launch_lkhd_pois(Ctx* c);
int launch_lkhd_genes(Ctx* c);
int launch_collect_lkhd(Ctx* c, int n_cells, int slot);
int launch_init_beta_solve(Ctx* c);
// k_de.cu (the DE driver's IRLS forms)
int launch_de_zeta(Ctx* c);               // zeta from Beta and phi (getZeta), then e0 = Z zeta
int launch_de_beta_phi(Ctx* c);           // beta = Psi^{-1} b + zeta, phi with the DE clamps
int launch_de_lkhd(Ctx* c, int slot);     // per-gene DE log-likelihood, their sum into lkhd slot
// k_grad.cu
int launch_grad_delta(Ctx* c);
int launch_grad_omega(Ctx* c);
int launch_c2(Ctx* c);
int launch_grad_tau_rho(Ctx* c);
// k_lbfgs.cu
int launch_lbfgs_update(Ctx* c, int itr, int rhoflag);
int launch_downdate(Ctx* c, int itr, double r, int rhoflag);
int launch_beta_from_tilde(Ctx* c);

}  // namespace gpl

struct gpl_ctx {
  gpl::Ctx c;
};

// ---- device helpers --------------------------------------------------------------------
namespace gpl {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum (fixed shuffle tree, then fixed order over warps); all threads
// of the block must call it; the result is valid in every thread. `sh` needs 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (wid == 0) {
    t = lane < nw ? sh[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) sh[0] = t;
  }
  __syncthreads();
  return sh[0];
}

}  // namespace gpl
