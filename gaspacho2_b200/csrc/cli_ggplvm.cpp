// ggplvm: the process-level drop-in for the reference driver (ggplvm.cu:951-1347), calling
// the CUDA library only through the C ABI of include/gpl.h.
//
//   ggplvm Y.bin Z.bin ls.bin Xi.bin [-M m] [-Q q] [--init-params params.bin]
//          [--max-outer n] [--max-lbfgs-iters n] [--precision fp64|bf16x3] [--device d]
//          [--out-dir dir] [--phi-gz omega|phi] [--seed s] [--genotypes G.bin -L l] [--quiet]
//
// Inputs (same formats as the reference): Y.bin gene-major compressed counts
// (int N, J, L; int i[L]; int p[J+1]; double x[L], SparseMat.cu:37-52), Z.bin covariate
// DataFrame (int N, p'; int c[p']; int v[p']; per variable double[N*v] or int[N*v],
// DataFrame.cu:56-117), ls.bin double[N] size factors, Xi.bin double[N*Q] (column-major)
// initial latent coordinates, and optionally params.bin (headerless double Omega[N],
// delta[p], X[N*Q], T[M*Q], rho[Q], phi[J], util_cuda.cu:520-535). -M and -Q default to 100
// and 51 as in the reference (ggplvm.cu:974-978).
//
// Outputs, in --out-dir (default: the working directory, as the reference):
//   Tau.bin      double[M*Q]  the initial inducing points (ggplvm.cu:1009)
//   X9.gz        after every outer iteration: N rows of X, M rows of T, one row of rho, each
//                value "%lf," (ggplvm.cu:1301-1314)
//   phi.gz       after every outer iteration, J lines "%lf". The reference copies the first
//                J values of the Omega buffer here (ggplvm.cu:1304), not phi; that is kept
//                (values past N, which the reference never writes, are written as 0) unless
//                --phi-gz phi asks for the fitted dispersions.
//   Params9.bin  after every outer iteration: int N, J, M, P, p, Q then the parameter
//                blocks (util_cuda.cu:566-577)
//   params.bin   at the end: the headerless parameter blocks (ggplvm.cu:1333-1346)
//   beta.bin     at the end: double[P*J], gene j's coefficients at j*P (the reference
//                never writes beta)
//   ScoreStats.gz with --genotypes: after the fit, J rows of the L genotype columns' score
//                statistics, "%lf," each (the output of the reference's differential-expression
//                driver, ggplvm_de.cu:1205-1214; G.bin holds double[N*L], column-major, already
//                transformed as that driver does with its dox and scaling)
// Exit status 0 on success, 1 on an input, allocation or CUDA error or a NaN IRLS
// likelihood (the reference returns 1 there, ggplvm.cu:1182), 2 on bad usage.
//
// --max-outer (default 5000, the reference's ITRMAX) and --max-lbfgs-iters (total L-BFGS
// steps, default unlimited) bound the run; the reference loop has no other exit.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

#include <string>
#include <vector>

#include "cli_io.h"
#include "gpl.h"

namespace {

using namespace cli;

struct Options {
  std::string y, z, ls, xi, init_params, out_dir = ".", precision = "fp64", phi_gz = "omega", genotypes;
  int M = 100, Q = 51, max_outer = 5000, max_lbfgs = 0, device = 0, L = 0;
  uint64_t seed = 0;
  bool quiet = false;
  bool init_latent = false;  // compute X (written to Xi.bin) and T from the counts
};

void usage() {
  fprintf(stderr,
          "usage: ggplvm Y.bin Z.bin ls.bin Xi.bin [-M m] [-Q q] [--init-params params.bin]\n"
          "              [--max-outer n] [--max-lbfgs-iters n] [--precision fp64|bf16x3] [--device d]\n"
          "              [--out-dir dir] [--phi-gz omega|phi] [--seed s] [--genotypes G.bin -L l] [--quiet]\n"
          "              [--init-latent]   (Xi.bin is then written: PCA of log1p(y/s); T by k-means)\n");
}

bool parse_int(const char* s, long lo, long hi, long* out) {
  char* end = nullptr;
  const long v = strtol(s, &end, 10);
  if (!s[0] || *end || v < lo || v > hi) return false;
  *out = v;
  return true;
}

// Returns 0 on success, 2 on bad usage.
int parse(int argc, char** argv, Options* o) {
  std::vector<std::string> pos;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto need = [&](const char* what) -> const char* {
      if (i + 1 >= argc) {
        fprintf(stderr, "ggplvm: %s needs a value\n", what);
        return nullptr;
      }
      return argv[++i];
    };
    long v;
    if (a == "-M" || a == "-Q" || a == "-L" || a == "--max-outer" || a == "--max-lbfgs-iters" || a == "--device") {
      const char* s = need(a.c_str());
      if (!s) return 2;
      const long lo = (a == "--max-lbfgs-iters" || a == "--device") ? 0 : 1;
      if (!parse_int(s, lo, 1L << 30, &v)) {
        fprintf(stderr, "ggplvm: bad value for %s: %s\n", a.c_str(), s);
        return 2;
      }
      if (a == "-M") o->M = (int)v;
      else if (a == "-Q") o->Q = (int)v;
      else if (a == "-L") o->L = (int)v;
      else if (a == "--max-outer") o->max_outer = (int)v;
      else if (a == "--max-lbfgs-iters") o->max_lbfgs = (int)v;
      else o->device = (int)v;
    } else if (a == "--seed") {
      const char* s = need("--seed");
      if (!s || !parse_int(s, 0, 1L << 62, &v)) return 2;
      o->seed = (uint64_t)v;
    } else if (a == "--init-params" || a == "--precision" || a == "--out-dir" || a == "--phi-gz" ||
               a == "--genotypes") {
      const char* s = need(a.c_str());
      if (!s) return 2;
      if (a == "--genotypes") o->genotypes = s;
      else if (a == "--init-params") o->init_params = s;
      else if (a == "--precision") o->precision = s;
      else if (a == "--out-dir") o->out_dir = s;
      else o->phi_gz = s;
    } else if (a == "--quiet") {
      o->quiet = true;
    } else if (a == "--init-latent") {
      o->init_latent = true;
    } else if (a == "-h" || a == "--help") {
      usage();
      return 2;
    } else if (!a.empty() && a[0] == '-') {
      fprintf(stderr, "ggplvm: unknown option %s\n", a.c_str());
      return 2;
    } else {
      pos.push_back(a);
    }
  }
  if (pos.size() != 4) {
    usage();
    return 2;
  }
  if (!o->genotypes.empty() && o->L < 1) {
    fprintf(stderr, "ggplvm: --genotypes needs -L with the number of genotype columns\n");
    return 2;
  }
  if (o->precision != "fp64" && o->precision != "bf16x3") {
    fprintf(stderr, "ggplvm: --precision must be fp64 or bf16x3\n");
    return 2;
  }
  if (o->phi_gz != "omega" && o->phi_gz != "phi") {
    fprintf(stderr, "ggplvm: --phi-gz must be omega or phi\n");
    return 2;
  }
  o->y = pos[0];
  o->z = pos[1];
  o->ls = pos[2];
  o->xi = pos[3];
  return 0;
}

// Seeded standard normals for T's dimensions 1..Q-1 (splitmix64 + Box-Muller). The
// reference draws them from GSL's MT19937 (util.c:73-87), which is not reproduced: pass T
// through --init-params for runs that must match the reference.
struct Normal {
  uint64_t s;
  explicit Normal(uint64_t seed) : s(seed ^ 0x9E3779B97F4A7C15ull) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
  double operator()() {
    const double u1 = uniform(), u2 = uniform();
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  }
};

bool write_x9(const std::string& path, const Params& q, int N, int M, int Q) {
  gzFile f = gzopen(path.c_str(), "w6h");
  if (!f) {
    fprintf(stderr, "ggplvm: cannot write %s\n", path.c_str());
    return false;
  }
  for (int i = 0; i < N; i++) {
    for (int k = 0; k < Q; k++) gzprintf(f, "%lf,", q.X[i + (size_t)k * N]);
    gzprintf(f, "\n");
  }
  for (int i = 0; i < M; i++) {
    for (int k = 0; k < Q; k++) gzprintf(f, "%lf,", q.T[i + (size_t)k * M]);
    gzprintf(f, "\n");
  }
  for (int k = 0; k < Q; k++) gzprintf(f, "%lf,", q.rho[k]);
  gzprintf(f, "\n");
  return gzclose(f) == Z_OK;
}

bool write_phi(const std::string& path, const Params& q, int N, int J, bool omega) {
  gzFile f = gzopen(path.c_str(), "w6h");
  if (!f) {
    fprintf(stderr, "ggplvm: cannot write %s\n", path.c_str());
    return false;
  }
  for (int k = 0; k < J; k++) {
    const double v = omega ? (k < N ? q.Omega[k] : 0.0) : q.phi[k];
    gzprintf(f, "%lf\n", v);
  }
  return gzclose(f) == Z_OK;
}

int fail(gpl_ctx* ctx, const char* what, int rc) {
  fprintf(stderr, "ggplvm: %s failed (status %d): %s\n", what, rc, ctx ? gpl_last_error(ctx) : "");
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  const int prc = parse(argc, argv, &o);
  if (prc) return prc;

  Counts y;
  Design z;
  if (!load_counts(o.y, &y) || !load_design(o.z, &z)) return 1;
  if (z.N != y.N) {
    fprintf(stderr, "ggplvm: %s has N=%d but %s has N=%d\n", o.z.c_str(), z.N, o.y.c_str(), y.N);
    return 1;
  }
  const int N = y.N, J = y.J, M = o.M, Q = o.Q;
  std::vector<double> ls(N), Xi((size_t)N * Q);
  if (!load_doubles(o.ls, ls.data(), N) || (!o.init_latent && !load_doubles(o.xi, Xi.data(), (size_t)N * Q)))
    return 1;

  gpl_ctx* ctx = nullptr;
  int rc = gpl_create(&ctx, o.device, nullptr);
  if (rc) return fail(nullptr, "gpl_create", rc);
  struct Guard {
    gpl_ctx* c;
    ~Guard() { gpl_destroy(c); }
  } guard{ctx};
  if ((rc = gpl_set_precision(ctx, o.precision == "bf16x3" ? GPL_PREC_BF16X3 : GPL_PREC_FP64)))
    return fail(ctx, "gpl_set_precision", rc);
  if ((rc = gpl_load_counts(ctx, N, J, y.L, y.i.data(), y.p.data(), y.x.data())))
    return fail(ctx, "gpl_load_counts", rc);
  if ((rc = gpl_load_design(ctx, N, z.n_var, z.c.data(), z.v.data(), z.body.data(), (int64_t)z.body.size(), M, Q)))
    return fail(ctx, "gpl_load_design", rc);
  if ((rc = gpl_set_size_factors(ctx, ls.data()))) return fail(ctx, "gpl_set_size_factors", rc);
  int32_t dims[6];
  if ((rc = gpl_dims(ctx, dims))) return fail(ctx, "gpl_dims", rc);
  const int P = dims[3], p = dims[4];
  if (!o.quiet) printf("N=%d, J=%d, P=%d, p=%d, M=%d, Q=%d\n", N, J, P, p, M, Q);

  // initParams (init.cu:27-48), then T as initTaWithPer: dimension 0 equispaced on
  // (0, 2 pi), the others standard normal; written to Tau.bin before any --init-params.
  if ((rc = gpl_init_params(ctx))) return fail(ctx, "gpl_init_params", rc);
  Params q(N, J, M, p, Q);
  if ((rc = gpl_get_params(ctx, q.Omega.data(), q.delta.data(), nullptr, q.T.data(), q.rho.data(), q.phi.data())))
    return fail(ctx, "gpl_get_params", rc);
  Normal rng(o.seed);
  for (int k = 1; k < Q; k++)
    for (int i = 0; i < M; i++) q.T[i + (size_t)k * M] = rng();
  if (o.init_latent) {
    // X from the principal components of log1p(y / s), T from k-means on X (gpl_init_latent)
    if ((rc = gpl_init_latent(ctx, 60, 25, o.seed, Xi.data(), q.T.data()))) return fail(ctx, "gpl_init_latent", rc);
    if (!write_file(o.xi, {{Xi.data(), Xi.size() * 8}})) return 1;
    if (!o.quiet) printf("Xi written to %s (PCA of log1p counts), T by k-means\n", o.xi.c_str());
  }
  if (!write_file(join(o.out_dir, "Tau.bin"), {{q.T.data(), q.T.size() * 8}})) return 1;
  q.X = Xi;
  if (!o.init_params.empty()) {
    Reader r(o.init_params);
    if (!r.read(q.Omega.data(), 8, N) || !r.read(q.delta.data(), 8, p) || !r.read(q.X.data(), 8, (size_t)N * Q) ||
        !r.read(q.T.data(), 8, (size_t)M * Q) || !r.read(q.rho.data(), 8, Q) || !r.read(q.phi.data(), 8, J))
      return 1;
    if (!o.quiet) printf("Init param=%s\n", o.init_params.c_str());
  }
  if ((rc = gpl_set_params(ctx, q.Omega.data(), q.delta.data(), q.X.data(), q.T.data(), q.rho.data(), q.phi.data())))
    return fail(ctx, "gpl_set_params", rc);

  // getKernelMats, cholKmm, getKinvKmn, expandDelta, initPsi, initBeta (ggplvm.cu:1111-1137)
  if ((rc = gpl_kernel_mats(ctx))) return fail(ctx, "gpl_kernel_mats", rc);
  if ((rc = gpl_glm_init(ctx))) return fail(ctx, "gpl_glm_init", rc);

  std::vector<double> trace(16384);
  int lbfgs_total = 0;
  for (int itr = 0; itr < o.max_outer; itr++) {
    int32_t st[4] = {0, 0, 0, 0};
    const int left = o.max_lbfgs > 0 ? o.max_lbfgs - lbfgs_total : 0;
    rc = gpl_fit_outer(ctx, itr, left, st, trace.data(), (int)trace.size());
    if (rc == GPL_ERR_NAN) {
      fprintf(stderr, "ggplvm: IRLS likelihood is NaN at outer iteration %d\n", itr);
      return 1;
    }
    if (rc) return fail(ctx, "gpl_fit_outer", rc);
    lbfgs_total += st[1];
    if ((rc = gpl_get_params(ctx, q.Omega.data(), q.delta.data(), q.X.data(), q.T.data(), q.rho.data(),
                             q.phi.data())))
      return fail(ctx, "gpl_get_params", rc);
    if (!o.quiet)
      printf("itr=%d irls=%d lbfgs=%d evals=%d lkhd=%.12g\n", itr, st[0], st[1], st[2],
             st[3] > 0 ? trace[st[3] - 1] : NAN);
    std::vector<int32_t> hdr = {N, J, M, P, p, Q};
    auto blocks = q.blocks();
    blocks.insert(blocks.begin(), {hdr.data(), hdr.size() * 4});
    if (!write_x9(join(o.out_dir, "X9.gz"), q, N, M, Q) ||
        !write_phi(join(o.out_dir, "phi.gz"), q, N, J, o.phi_gz == "omega") ||
        !write_file(join(o.out_dir, "Params9.bin"), blocks))
      return 1;
    if (o.max_lbfgs > 0 && lbfgs_total >= o.max_lbfgs) break;
  }
  if (!o.quiet) printf("Iteration end...\n");
  std::vector<double> beta((size_t)P * J);
  if ((rc = gpl_get_beta(ctx, beta.data()))) return fail(ctx, "gpl_get_beta", rc);
  if (!o.genotypes.empty()) {
    std::vector<double> G((size_t)N * o.L), S((size_t)J * o.L);
    if (!load_doubles(o.genotypes, G.data(), G.size())) return 1;
    if ((rc = gpl_score_stats(ctx, o.L, G.data(), S.data()))) return fail(ctx, "gpl_score_stats", rc);
    const std::string path = join(o.out_dir, "ScoreStats.gz");
    gzFile f = gzopen(path.c_str(), "w6h");
    if (!f) {
      fprintf(stderr, "ggplvm: cannot write %s\n", path.c_str());
      return 1;
    }
    for (int j = 0; j < J; j++) {
      for (int l = 0; l < o.L; l++) gzprintf(f, "%lf,", S[j + (size_t)l * J]);
      gzprintf(f, "\n");
    }
    if (gzclose(f) != Z_OK) return 1;
  }
  if (!write_file(join(o.out_dir, "params.bin"), q.blocks()) ||
      !write_file(join(o.out_dir, "beta.bin"), {{beta.data(), beta.size() * 8}}))
    return 1;
  return 0;
}
