// ggplvm_delta: the process-level drop-in for the reference's variance-component driver
// (ggplvm_delta.cu:784-1097, whose main does not compile as shipped: it calls a __global__
// printMetaDataFrame from the host at :823), calling the CUDA library only through the C ABI.
//
//   ggplvm_delta Y.bin Z.bin ls.bin Xi.bin [-M m] [-Q q] [--init-deltaG d]
//                [--init-params params.bin] [--max-outer n] [--max-lbfgs-iters n] [--device d] [--quiet]
//
// Inputs as for ggplvm; Z.bin ends with the variable whose prior variance is refitted (the
// genotype). The fit's parameters come from params.bin in the working directory, as the
// reference reads them (ggplvm_delta.cu:944-956; --init-params names another file): Omega[N],
// the p - 1 deltas of the design without that variable, X[N*Q], T[M*Q], rho[Q]. delta[p-2]
// starts at --init-deltaG (default 0.01) and delta[p-1] keeps initParams' 0.3, as in the
// reference; Xi.bin is read and then replaced by params.bin's X, as there. -M and -Q default
// to 100 and 51. --max-outer (default 100, the reference's ITRMAX) and --max-lbfgs-iters
// (default 100 per outer iteration, its inner limit) bound the run.
//
// Output: one line per outer iteration, "itr=<i> delta_G=<value> lkhd=<objective>", on
// standard output (the reference prints its progress and writes no file: its params.bin
// dump is commented out, ggplvm_delta.cu:1106-1113). Exit status 0 on success, 1 on an input,
// allocation or CUDA error, 2 on bad usage.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "cli_io.h"
#include "gpl.h"

namespace {

using namespace cli;

struct Options {
  std::string y, z, ls, xi, init_params = "params.bin";
  int M = 100, Q = 51, max_outer = 100, max_lbfgs = 100, device = 0;
  double init_dg = 0.01;
  bool quiet = false;
};

void usage() {
  fprintf(stderr,
          "usage: ggplvm_delta Y.bin Z.bin ls.bin Xi.bin [-M m] [-Q q] [--init-deltaG d]\n"
          "                    [--init-params params.bin] [--max-outer n] [--max-lbfgs-iters n] [--device d]"
          " [--quiet]\n");
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
        fprintf(stderr, "ggplvm_delta: %s needs a value\n", what);
        return nullptr;
      }
      return argv[++i];
    };
    long v;
    if (a == "-M" || a == "-Q" || a == "--max-outer" || a == "--max-lbfgs-iters" || a == "--device") {
      const char* s = need(a.c_str());
      if (!s) return 2;
      if (!parse_int(s, a == "--device" ? 0 : 1, 1L << 30, &v)) {
        fprintf(stderr, "ggplvm_delta: bad value for %s: %s\n", a.c_str(), s);
        return 2;
      }
      if (a == "-M") o->M = (int)v;
      else if (a == "-Q") o->Q = (int)v;
      else if (a == "--max-outer") o->max_outer = (int)v;
      else if (a == "--max-lbfgs-iters") o->max_lbfgs = (int)v;
      else o->device = (int)v;
    } else if (a == "--init-deltaG") {
      const char* s = need("--init-deltaG");
      if (!s) return 2;
      char* end = nullptr;
      o->init_dg = strtod(s, &end);
      if (!s[0] || *end || !(o->init_dg > 0.0)) {
        fprintf(stderr, "ggplvm_delta: --init-deltaG must be a positive number\n");
        return 2;
      }
    } else if (a == "--init-params") {
      const char* s = need("--init-params");
      if (!s) return 2;
      o->init_params = s;
    } else if (a == "--quiet") {
      o->quiet = true;
    } else if (a == "-h" || a == "--help") {
      usage();
      return 2;
    } else if (!a.empty() && a[0] == '-') {
      fprintf(stderr, "ggplvm_delta: unknown option %s\n", a.c_str());
      return 2;
    } else {
      pos.push_back(a);
    }
  }
  if (pos.size() != 4) {
    usage();
    return 2;
  }
  o->y = pos[0];
  o->z = pos[1];
  o->ls = pos[2];
  o->xi = pos[3];
  return 0;
}

int fail(gpl_ctx* ctx, const char* what, int rc) {
  fprintf(stderr, "ggplvm_delta: %s failed (status %d): %s\n", what, rc, ctx ? gpl_last_error(ctx) : "");
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  prog() = "ggplvm_delta";
  Options o;
  const int prc = parse(argc, argv, &o);
  if (prc) return prc;
  Counts y;
  Design z;
  if (!load_counts(o.y, &y) || !load_design(o.z, &z)) return 1;
  if (z.N != y.N) {
    fprintf(stderr, "ggplvm_delta: %s has N=%d but %s has N=%d\n", o.z.c_str(), z.N, o.y.c_str(), y.N);
    return 1;
  }
  if (z.n_var < 1) {
    fprintf(stderr, "ggplvm_delta: %s has no variable whose variance could be refitted\n", o.z.c_str());
    return 1;
  }
  const int N = y.N, J = y.J, M = o.M, Q = o.Q, p = z.n_var + 2;
  std::vector<double> ls(N), Xi((size_t)N * Q);
  if (!load_doubles(o.ls, ls.data(), N) || !load_doubles(o.xi, Xi.data(), Xi.size())) return 1;
  // params.bin (ggplvm_delta.cu:944-956): p - 1 deltas; delta[p-2] <- init, delta[p-1] <- 0.3
  std::vector<double> Omega(N), delta(p), X((size_t)N * Q), T((size_t)M * Q), rho(Q), phi(J, 1.0);
  {
    Reader r(o.init_params);
    if (!r.read(Omega.data(), 8, N) || !r.read(delta.data(), 8, p - 1) || !r.read(X.data(), 8, X.size()) ||
        !r.read(T.data(), 8, T.size()) || !r.read(rho.data(), 8, Q))
      return 1;
  }
  delta[p - 2] = o.init_dg;
  delta[p - 1] = 0.3;  // initParams (init.cu:27-48): the reference copies only p - 1 values

  gpl_ctx* ctx = nullptr;
  int rc = gpl_create(&ctx, o.device, nullptr);
  if (rc) return fail(nullptr, "gpl_create", rc);
  struct Guard {
    gpl_ctx* c;
    ~Guard() { gpl_destroy(c); }
  } guard{ctx};
  if ((rc = gpl_load_counts(ctx, N, J, y.L, y.i.data(), y.p.data(), y.x.data())))
    return fail(ctx, "gpl_load_counts", rc);
  if ((rc = gpl_load_design(ctx, N, z.n_var, z.c.data(), z.v.data(), z.body.data(), (int64_t)z.body.size(), M, Q)))
    return fail(ctx, "gpl_load_design", rc);
  if ((rc = gpl_set_size_factors(ctx, ls.data()))) return fail(ctx, "gpl_set_size_factors", rc);
  if ((rc = gpl_set_params(ctx, Omega.data(), delta.data(), X.data(), T.data(), rho.data(), phi.data())))
    return fail(ctx, "gpl_set_params", rc);
  std::vector<double> dg(o.max_outer), obj(o.max_outer);
  int32_t n = 0;
  if ((rc = gpl_vc_fit(ctx, o.max_outer, o.max_lbfgs, dg.data(), obj.data(), o.max_outer, &n)))
    return fail(ctx, "gpl_vc_fit", rc);
  for (int i = 0; i < n; i++) printf("itr=%d delta_G=%.12g lkhd=%.12g\n", i, dg[i], obj[i]);
  if (!o.quiet) printf("Iteration end...\n");
  return 0;
}
