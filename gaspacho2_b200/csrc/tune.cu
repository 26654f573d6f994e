// The autotuner of libgpl_b200 (no reference counterpart): picks launch shapes and tile orders
// of the hot kernels by timing them on the live workload.
//
// Every tunable choice here changes only WHICH CTA computes WHICH output tile or gene, or in
// what order the tiles are walked, never the arithmetic of an output: each candidate gives the
// same bits. So the tuner can use the real launches of a fit as its trials ("online" tuning):
// while a choice is open, each launch of that kernel takes the candidate with the fewest
// timings, its CUDA events (on the context's stream) are read at the next host synchronisation,
// and once every candidate has kReps timings the fastest (by its best time) is fixed. The
// result is remembered for the process per (choice, N, J, dense columns, P, precision), so later
// contexts of the same shape start settled. CUDA-graph capture waits until every open choice
// of the context has settled, so graphs hold the chosen launches.
#include <map>
#include <mutex>

#include "gpl_internal.cuh"

namespace gpl {

namespace {
constexpr int kReps = 2;
std::mutex g_cache_mu;
std::map<std::string, int> g_cache;  // key -> chosen candidate value

std::string cache_key(const Ctx* c, const char* name) {
  return std::string(name) + "|" + std::to_string(c->N) + "|" + std::to_string(c->J) + "|" +
         std::to_string(c->n_d) + "|" + std::to_string(c->P) + "|" + std::to_string(c->precision);
}
}  // namespace

Tunable* tune_find(Ctx* c, const char* name) {
  for (auto& t : c->tun)
    if (t.name == name) return &t;
  return nullptr;
}

int tune_pick(Ctx* c, const char* name, const std::vector<int>& cands, int fallback, Tunable** slot) {
  *slot = nullptr;
  if (!c->autotune || cands.empty()) return fallback;
  Tunable* t = tune_find(c, name);
  if (!t) {
    c->tun.push_back(Tunable());
    t = &c->tun.back();
    t->name = name;
    t->cands = cands;
    t->best_ms.assign(cands.size(), 1e300);
    t->n.assign(cands.size(), 0);
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_cache.find(cache_key(c, name));
    if (it != g_cache.end())
      for (size_t k = 0; k < cands.size(); k++)
        if (cands[k] == it->second) {
          t->best = (int)k;
          t->from_cache = true;
        }
  }
  if (t->best >= 0) return t->cands[t->best];
  if (c->capturing) return fallback;  // no timing inside a captured graph
  // the candidate with the fewest timings, counting launches whose events are not read yet
  std::vector<int> seen = t->n;
  for (auto& p : t->pending) seen[p.cand]++;
  int k = 0;
  for (size_t q = 1; q < seen.size(); q++)
    if (seen[q] < seen[k]) k = (int)q;
  *slot = t;
  t->cur = k;
  return t->cands[k];
}

TuneScope::TuneScope(Ctx* c_, Tunable* t_) : c(c_), t(t_) {
  if (!t) return;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    cudaGetLastError();
    t = nullptr;
    return;
  }
  cudaEventRecord(a, c->stream);
}

TuneScope::~TuneScope() {
  if (!t) return;
  cudaEventRecord(b, c->stream);
  t->pending.push_back({t->cur, a, b});
}

void tune_harvest(Ctx* c) {
  for (auto& t : c->tun) {
    if (t.pending.empty()) continue;
    std::vector<Tunable::Pending> keep;
    for (auto& p : t.pending) {
      if (cudaEventQuery(p.b) != cudaSuccess) {
        cudaGetLastError();
        keep.push_back(p);
        continue;
      }
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
        t.best_ms[p.cand] = std::min(t.best_ms[p.cand], (double)ms);
        t.n[p.cand]++;
      } else {
        cudaGetLastError();
      }
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    t.pending.swap(keep);
    if (t.best >= 0) continue;
    bool done = true;
    for (int n : t.n) done = done && n >= kReps;
    if (!done) continue;
    int k = 0;
    for (size_t q = 1; q < t.cands.size(); q++)
      if (t.best_ms[q] < t.best_ms[k]) k = (int)q;
    t.best = k;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_cache[cache_key(c, t.name.c_str())] = t.cands[k];
  }
}

bool tune_settled(const Ctx* c) {
  for (auto& t : c->tun)
    if (t.best < 0 || !t.pending.empty()) return false;
  return true;
}

// The choices made inside an evaluation (the objective's Gram, the gradient's pair contraction):
// capture waits for these only; the IRLS tail is never part of a captured evaluation.
bool tune_settled_for_graphs(const Ctx* c) {
  for (auto& t : c->tun) {
    const bool in_eval = t.name == "pair_gram" || t.name == "pair_v" || t.name == "tc_gram" || t.name == "tc_grad" ||
                         t.name == "eta_tile";
    if (in_eval && (t.best < 0 || !t.pending.empty())) return false;
  }
  return true;
}

void tune_release(Ctx* c) {
  for (auto& t : c->tun)
    for (auto& p : t.pending) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
  c->tun.clear();
}

}  // namespace gpl
