// Input/output helpers shared by the command-line drop-ins (bin/ggplvm, bin/ggplvm_de): the
// reference's binary formats read with exact-size checks (its freads are unchecked) and the
// headerless parameter blocks (util_cuda.cu:520-577). Messages carry the program's name.
#pragma once
#include <stdint.h>
#include <stdio.h>

#include <string>
#include <utility>
#include <vector>

namespace cli {

inline const char*& prog() {
  static const char* name = "ggplvm";
  return name;
}

// Whole-file reader with exact-size checks (the reference's freads are unchecked).
struct Reader {
  FILE* f = nullptr;
  std::string path;
  bool ok = true;
  explicit Reader(const std::string& p) : path(p) {
    f = fopen(p.c_str(), "rb");
    if (!f) {
      fprintf(stderr, "%s: cannot open %s\n", prog(), p.c_str());
      ok = false;
    }
  }
  ~Reader() {
    if (f) fclose(f);
  }
  bool read(void* dst, size_t size, size_t n) {
    if (!ok) return false;
    if (n && fread(dst, size, n, f) != n) {
      fprintf(stderr, "%s: %s is truncated\n", prog(), path.c_str());
      ok = false;
    }
    return ok;
  }
};

struct Counts {
  int N = 0, J = 0, L = 0;
  std::vector<int32_t> i, p;
  std::vector<double> x;
};

inline bool load_counts(const std::string& path, Counts* y) {
  Reader r(path);
  int32_t hdr[3];
  if (!r.read(hdr, sizeof(int32_t), 3)) return false;
  y->N = hdr[0];
  y->J = hdr[1];
  y->L = hdr[2];
  if (y->N <= 0 || y->J <= 0 || y->L < 0) {
    fprintf(stderr, "%s: %s: bad header N=%d J=%d L=%d\n", prog(), path.c_str(), y->N, y->J, y->L);
    return false;
  }
  y->i.resize(y->L);
  y->p.resize((size_t)y->J + 1);
  y->x.resize(y->L);
  return r.read(y->i.data(), sizeof(int32_t), y->L) && r.read(y->p.data(), sizeof(int32_t), (size_t)y->J + 1) &&
         r.read(y->x.data(), sizeof(double), y->L);
}

struct Design {
  int N = 0, n_var = 0;
  std::vector<int32_t> c, v;
  std::vector<unsigned char> body;
};

inline bool load_design(const std::string& path, Design* z) {
  Reader r(path);
  int32_t hdr[2];
  if (!r.read(hdr, sizeof(int32_t), 2)) return false;
  z->N = hdr[0];
  z->n_var = hdr[1];
  if (z->N <= 0 || z->n_var < 0) {
    fprintf(stderr, "%s: %s: bad header N=%d p=%d\n", prog(), path.c_str(), z->N, z->n_var);
    return false;
  }
  z->c.resize(z->n_var);
  z->v.resize(z->n_var);
  if (!r.read(z->c.data(), sizeof(int32_t), z->n_var) || !r.read(z->v.data(), sizeof(int32_t), z->n_var)) return false;
  size_t bytes = 0;
  for (int k = 0; k < z->n_var; k++) {
    if (z->c[k] < 1 || z->v[k] < 1) {
      fprintf(stderr, "%s: %s: variable %d has c=%d v=%d\n", prog(), path.c_str(), k, z->c[k], z->v[k]);
      return false;
    }
    bytes += (size_t)z->N * z->v[k] * (z->c[k] == 1 ? sizeof(double) : sizeof(int32_t));
  }
  z->body.resize(bytes);
  return r.read(z->body.data(), 1, bytes);
}

inline bool load_doubles(const std::string& path, double* dst, size_t n) {
  Reader r(path);
  return r.read(dst, sizeof(double), n);
}

inline std::string join(const std::string& dir, const char* name) { return dir.empty() ? name : dir + "/" + name; }

inline bool write_file(const std::string& path, const std::vector<std::pair<const void*, size_t>>& parts) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) {
    fprintf(stderr, "%s: cannot write %s\n", prog(), path.c_str());
    return false;
  }
  bool ok = true;
  for (auto& pr : parts) ok = ok && (pr.second == 0 || fwrite(pr.first, 1, pr.second, f) == pr.second);
  ok = (fclose(f) == 0) && ok;
  if (!ok) fprintf(stderr, "%s: short write to %s\n", prog(), path.c_str());
  return ok;
}

struct Params {
  std::vector<double> Omega, delta, X, T, rho, phi;
  Params(int N, int J, int M, int p, int Q) : Omega(N), delta(p), X((size_t)N * Q), T((size_t)M * Q), rho(Q), phi(J) {}
  std::vector<std::pair<const void*, size_t>> blocks() const {
    return {{Omega.data(), Omega.size() * 8}, {delta.data(), delta.size() * 8}, {X.data(), X.size() * 8},
            {T.data(), T.size() * 8},         {rho.data(), rho.size() * 8},     {phi.data(), phi.size() * 8}};
  }
};


}  // namespace cli
