// ggplvm_de: the process-level drop-in for the reference's differential-expression driver
// (ggplvm_de.cu:886-1237), calling the CUDA library only through the C ABI of include/gpl.h.
//
//   ggplvm_de Y.bin Z.bin ls.bin [G.bin dox.bin] --init-params params.bin [-Mf m] [-Mr m]
//             [-Q q] [-L l] [--max-sweeps n] [--device d] [--out-dir dir] [--no-knm] [--quiet]
//
// Inputs: Y.bin, Z.bin and ls.bin as for ggplvm; params.bin holds the fit's parameters
// (headerless double Omega[N], delta[p], X[N*Q], T[Mf*Q], rho[Q], phi[J]; the reference reads
// it with M = Mf, ggplvm_de.cu:1040-1043, and runs on uninitialised memory without it, so it
// is required here). With -L l > 0, G.bin (double[N*l], column-major genotypes) and dox.bin
// (double[N]) follow ls.bin: every genotype column is multiplied by dox and centred
// (ggplvm_de.cu:986-999). -Mf, -Mr and -Q default to 50, 5 and 51 as in the reference
// (ggplvm_de.cu:905-916).
//
// The driver refits the GLM part by IRLS at the fitted Omega, delta, X and rho for the null
// model (no GP), one model per latent dimension q (the GP over dimension q alone, Mr
// equispaced inducing points) and the full model (Mf inducing points, the fitted T), each to
// the reference's tolerance (1e-5 for the null model, 1e-8 otherwise) or --max-sweeps sweeps
// (the reference's JTRMAX, 1000). Outputs, in --out-dir:
//   BFs_de.gz        J rows of Q + 2 per-gene log-likelihoods "%lf,": null, q = 0..Q-1, full
//                    (ggplvm_de.cu:1220-1225)
//   Beta_de.gz       appended per GP model: J rows of P coefficients (ggplvm_de.cu:1181-1185)
//   Knm_de.gz        appended per GP model: N rows of Knm, M rows of Kmm (ggplvm_de.cu:1186-1199);
//                    --no-knm skips this file
//   ScoreStats.gz    with -L: J rows of the l score statistics at the full model's state
//                    (ggplvm_de.cu:1229-1236)
//   DesignMatrix.gz  with -L: N rows of the full model's P columns, then W[i + N] (the second
//                    gene's W, as the reference prints) and Omega_i (ggplvm_de.cu:1238-1247)
// The two appended files keep the reference's append mode ("a6h"): remove them between runs.
// Exit status 0 on success, 1 on an input, allocation or CUDA error, 2 on bad usage.
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
  std::string y, z, ls, g, dox, init_params, out_dir = ".";
  int Mf = 50, Mr = 5, Q = 51, L = 0, max_sweeps = 1000, device = 0;
  bool quiet = false, knm = true;
};

void usage() {
  fprintf(stderr,
          "usage: ggplvm_de Y.bin Z.bin ls.bin [G.bin dox.bin] --init-params params.bin [-Mf m] [-Mr m]\n"
          "                 [-Q q] [-L l] [--max-sweeps n] [--device d] [--out-dir dir] [--no-knm] [--quiet]\n");
}

bool parse_int(const char* s, long lo, long hi, long* out) {
  char* end = nullptr;
  const long v = strtol(s, &end, 10);
  if (!s[0] || *end || v < lo || v > hi) return false;
  *out = v;
  return true;
}

int parse(int argc, char** argv, Options* o) {
  std::vector<std::string> pos;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto need = [&](const char* what) -> const char* {
      if (i + 1 >= argc) {
        fprintf(stderr, "ggplvm_de: %s needs a value\n", what);
        return nullptr;
      }
      return argv[++i];
    };
    long v;
    if (a == "-Mf" || a == "-Mr" || a == "-Q" || a == "-L" || a == "--max-sweeps" || a == "--device") {
      const char* s = need(a.c_str());
      if (!s) return 2;
      const long lo = (a == "-L" || a == "--device") ? 0 : 1;
      if (!parse_int(s, lo, 1L << 30, &v)) {
        fprintf(stderr, "ggplvm_de: bad value for %s: %s\n", a.c_str(), s);
        return 2;
      }
      if (a == "-Mf") o->Mf = (int)v;
      else if (a == "-Mr") o->Mr = (int)v;
      else if (a == "-Q") o->Q = (int)v;
      else if (a == "-L") o->L = (int)v;
      else if (a == "--max-sweeps") o->max_sweeps = (int)v;
      else o->device = (int)v;
    } else if (a == "--init-params" || a == "--out-dir") {
      const char* s = need(a.c_str());
      if (!s) return 2;
      if (a == "--init-params") o->init_params = s;
      else o->out_dir = s;
    } else if (a == "--quiet") {
      o->quiet = true;
    } else if (a == "--no-knm") {
      o->knm = false;
    } else if (a == "-h" || a == "--help") {
      usage();
      return 2;
    } else if (!a.empty() && a[0] == '-') {
      fprintf(stderr, "ggplvm_de: unknown option %s\n", a.c_str());
      return 2;
    } else {
      pos.push_back(a);
    }
  }
  if (pos.size() != (o->L > 0 ? 5u : 3u)) {
    usage();
    return 2;
  }
  if (o->init_params.empty()) {
    fprintf(stderr, "ggplvm_de: --init-params is required (the fit's parameters)\n");
    return 2;
  }
  o->y = pos[0];
  o->z = pos[1];
  o->ls = pos[2];
  if (o->L > 0) {
    o->g = pos[3];
    o->dox = pos[4];
  }
  return 0;
}

int fail(gpl_ctx* ctx, const char* what, int rc) {
  fprintf(stderr, "ggplvm_de: %s failed (status %d): %s\n", what, rc, ctx ? gpl_last_error(ctx) : "");
  return 1;
}

struct Ctx {
  gpl_ctx* h = nullptr;
  ~Ctx() { gpl_destroy(h); }
};

// One context with the counts, the design (with M inducing points) and size factors.
int open_ctx(const Options& o, const Counts& y, const Design& z, const std::vector<double>& ls, int M, Ctx* c) {
  int rc = gpl_create(&c->h, o.device, nullptr);
  if (rc) return fail(nullptr, "gpl_create", rc);
  if ((rc = gpl_load_counts(c->h, y.N, y.J, y.L, y.i.data(), y.p.data(), y.x.data())))
    return fail(c->h, "gpl_load_counts", rc);
  if ((rc = gpl_load_design(c->h, y.N, z.n_var, z.c.data(), z.v.data(), z.body.data(), (int64_t)z.body.size(), M,
                            o.Q)))
    return fail(c->h, "gpl_load_design", rc);
  if ((rc = gpl_set_size_factors(c->h, ls.data()))) return fail(c->h, "gpl_set_size_factors", rc);
  return 0;
}

bool gz_rows(gzFile f, const double* a, int rows, int cols, size_t ld_row, size_t ld_col) {
  for (int i = 0; i < rows; i++) {
    for (int k = 0; k < cols; k++) gzprintf(f, "%lf,", a[i * ld_row + k * ld_col]);
    gzprintf(f, "\n");
  }
  return true;
}

gzFile gz_open(const std::string& path, const char* mode) {
  gzFile f = gzopen(path.c_str(), mode);
  if (!f) fprintf(stderr, "ggplvm_de: cannot write %s\n", path.c_str());
  return f;
}

int64_t get_len(gpl_ctx* h, const char* name) {
  int64_t n = 0;
  return gpl_get(h, name, nullptr, 0, &n) == GPL_OK ? n : -1;
}

}  // namespace

int main(int argc, char** argv) {
  prog() = "ggplvm_de";
  Options o;
  const int prc = parse(argc, argv, &o);
  if (prc) return prc;

  Counts y;
  Design z;
  if (!load_counts(o.y, &y) || !load_design(o.z, &z)) return 1;
  if (z.N != y.N) {
    fprintf(stderr, "ggplvm_de: %s has N=%d but %s has N=%d\n", o.z.c_str(), z.N, o.y.c_str(), y.N);
    return 1;
  }
  const int N = y.N, J = y.J, Q = o.Q;
  std::vector<double> ls(N);
  if (!load_doubles(o.ls, ls.data(), N)) return 1;
  const int p = z.n_var + 2;  // intercept, the design's variables, the GP

  // the fit's parameters, read as readParams with M = Mf (ggplvm_de.cu:1040-1043)
  std::vector<double> Omega(N), delta(p), X((size_t)N * Q), Tf((size_t)o.Mf * Q), rho(Q), phi_in(J);
  {
    Reader r(o.init_params);
    if (!r.read(Omega.data(), 8, N) || !r.read(delta.data(), 8, p) || !r.read(X.data(), 8, X.size()) ||
        !r.read(Tf.data(), 8, Tf.size()) || !r.read(rho.data(), 8, Q) || !r.read(phi_in.data(), 8, J))
      return 1;
  }
  std::vector<double> Tr((size_t)o.Mr * Q), T1((size_t)Q, 0.0), phi(J, 1.0);  // initPhi
  gpl_ta_equispaced(o.Mr, Q, Tr.data());

  std::vector<double> BFs((size_t)J * (Q + 2)), lk(J);
  const std::string beta_path = join(o.out_dir, "Beta_de.gz"), knm_path = join(o.out_dir, "Knm_de.gz");

  // one model: parameters (phi carried from the previous model), selection, IRLS, outputs
  auto run = [&](gpl_ctx* h, int model, const double* T, double tol, int col, bool write) -> int {
    int rc;
    if ((rc = gpl_set_params(h, Omega.data(), delta.data(), X.data(), T, rho.data(), phi.data())))
      return fail(h, "gpl_set_params", rc);
    if ((rc = gpl_de_model(h, model))) return fail(h, "gpl_de_model", rc);
    int32_t sweeps = 0;
    if ((rc = gpl_de_irls(h, o.max_sweeps, tol, lk.data(), &sweeps, nullptr, 0))) return fail(h, "gpl_de_irls", rc);
    memcpy(BFs.data() + (size_t)J * col, lk.data(), sizeof(double) * J);
    if ((rc = gpl_get_params(h, nullptr, nullptr, nullptr, nullptr, nullptr, phi.data())))
      return fail(h, "gpl_get_params", rc);
    double sum = 0.0;
    for (int j = 0; j < J; j++) sum += lk[j];
    if (!o.quiet) printf("model %d: %d sweeps, lkhd=%.12g\n", col, sweeps, sum);
    if (!write) return 0;
    int32_t dims[6];
    if ((rc = gpl_dims(h, dims))) return fail(h, "gpl_dims", rc);
    const int P = dims[3], M = dims[2];
    std::vector<double> beta((size_t)P * J);
    if ((rc = gpl_get_beta(h, beta.data()))) return fail(h, "gpl_get_beta", rc);
    gzFile f = gz_open(beta_path, "a6h");
    if (!f) return 1;
    gz_rows(f, beta.data(), J, P, (size_t)P, 1);
    if (gzclose(f) != Z_OK) return 1;
    if (o.knm) {
      std::vector<double> knm((size_t)N * M), kmm((size_t)M * M);
      int64_t n = 0;
      if ((rc = gpl_get(h, "Knm", knm.data(), (int64_t)knm.size(), &n)) ||
          (rc = gpl_get(h, "Kmm", kmm.data(), (int64_t)kmm.size(), &n)))
        return fail(h, "gpl_get", rc);
      gzFile g = gz_open(knm_path, "a6h");
      if (!g) return 1;
      gz_rows(g, knm.data(), N, M, 1, (size_t)N);
      gz_rows(g, kmm.data(), M, M, 1, (size_t)M);
      if (gzclose(g) != Z_OK) return 1;
    }
    return 0;
  };

  int rc;
  {  // null model (ggplvm_de.cu:1067-1107): a one-column GP block held inert
    Ctx c0;
    if ((rc = open_ctx(o, y, z, ls, 1, &c0))) return rc;
    if ((rc = run(c0.h, GPL_DE_NULL, T1.data(), 1e-5, 0, false))) return rc;
  }
  {  // one model per latent dimension (ggplvm_de.cu:1120-1126)
    Ctx cr;
    if ((rc = open_ctx(o, y, z, ls, o.Mr, &cr))) return rc;
    for (int q = 0; q < Q; q++)
      if ((rc = run(cr.h, q, Tr.data(), 1e-8, q + 1, true))) return rc;
  }
  Ctx cf;  // the full model (ggplvm_de.cu:1112-1119), kept for the score statistics
  if ((rc = open_ctx(o, y, z, ls, o.Mf, &cf))) return rc;
  if ((rc = run(cf.h, GPL_DE_FULL, Tf.data(), 1e-8, Q + 1, true))) return rc;

  {
    gzFile f = gz_open(join(o.out_dir, "BFs_de.gz"), "w6h");
    if (!f) return 1;
    gz_rows(f, BFs.data(), J, Q + 2, 1, (size_t)J);
    if (gzclose(f) != Z_OK) return 1;
  }
  if (o.L > 0) {
    std::vector<double> G((size_t)N * o.L), dox(N), S((size_t)J * o.L);
    if (!load_doubles(o.g, G.data(), G.size()) || !load_doubles(o.dox, dox.data(), N)) return 1;
    for (int l = 0; l < o.L; l++) {  // dox * genotype, then centred (scale, util.c:100-110)
      double* g = G.data() + (size_t)l * N;
      for (int i = 0; i < N; i++) g[i] *= dox[i];
      double m = 0.0;
      for (int i = 0; i < N; i++) m += g[i];
      m /= (double)N;
      for (int i = 0; i < N; i++) g[i] -= m;
    }
    if ((rc = gpl_score_stats(cf.h, o.L, G.data(), S.data()))) return fail(cf.h, "gpl_score_stats", rc);
    gzFile f = gz_open(join(o.out_dir, "ScoreStats.gz"), "w6h");
    if (!f) return 1;
    gz_rows(f, S.data(), J, o.L, 1, (size_t)J);
    if (gzclose(f) != Z_OK) return 1;

    // the full model's design matrix (getDesignMatrix, ggplvm_de.cu:24-31), W[i + N], Omega
    int32_t dims[6];
    if ((rc = gpl_dims(cf.h, dims))) return fail(cf.h, "gpl_dims", rc);
    const int P = dims[3], M = o.Mf;
    std::vector<double> knm((size_t)N * M), W;
    int64_t n = 0;
    const int64_t nw = get_len(cf.h, "W");
    if (nw < 0) return fail(cf.h, "gpl_get(W)", GPL_ERR_ARG);
    W.resize((size_t)nw);
    if ((rc = gpl_get(cf.h, "Knm", knm.data(), (int64_t)knm.size(), &n)) ||
        (rc = gpl_get(cf.h, "W", W.data(), nw, &n)))
      return fail(cf.h, "gpl_get", rc);
    gzFile d = gz_open(join(o.out_dir, "DesignMatrix.gz"), "w6h");
    if (!d) return 1;
    std::vector<double> row(P);
    for (int i = 0; i < N; i++) {
      int col = 0;
      row[col++] = 1.0;
      size_t off = 0;
      for (int k = 0; k < z.n_var; k++) {
        const int cv = z.c[k], vv = z.v[k];
        if (cv == 1) {
          const double* x = reinterpret_cast<const double*>(z.body.data() + off);
          for (int m = 0; m < vv; m++) row[col++] = x[i + (size_t)m * N];
          off += (size_t)N * vv * sizeof(double);
        } else {
          int32_t code;
          memcpy(&code, z.body.data() + off + (size_t)i * sizeof(int32_t), sizeof(int32_t));
          for (int m = 0; m < cv * vv; m++) row[col++] = (code == m) ? 1.0 : 0.0;
          off += (size_t)N * vv * sizeof(int32_t);
        }
      }
      for (int m = 0; m < M; m++) row[col++] = knm[i + (size_t)m * N];
      for (int k = 0; k < P; k++) gzprintf(d, "%lf,", row[k]);
      gzprintf(d, "%lf,%lf\n", W[(size_t)i + N], Omega[i]);
    }
    if (gzclose(d) != Z_OK) return 1;
  }
  if (!o.quiet) printf("Done.\n");
  return 0;
}
