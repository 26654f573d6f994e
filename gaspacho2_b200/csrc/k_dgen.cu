// FP64 tensor-core (DMMA) forms of the cell x gene contractions around the Gram: one
// register-staged GEMM template whose operand loaders apply the element-wise prologues
// (W/Omega, products with nu, a cell group's slice) and whose epilogues scatter the results.
//
//   zt_u      bvec[dcol a, j] = sum_i D_ia u_ij (getZtOinvjnj util_cuda.cu:462-487 with
//             u = W nu / Omega; initBeta init.cu:193-221 with u = y0), split over the cells
//             into 8-32 ranges (chosen to fill the last wave) whose partial sums are added in
//             order; its own kernel (k_zt_u), whose raw operands arrive by cp.async.
//             2*N*J*n_d flops.
//   c1_tn     C1[i, a] = sum_j (tn_ij / phi_j) tBeta_j[GP a] (ggplvm.cu:344).  2*N*J*M flops.
//   group     S[j][g][a] = sum_{i in g} w_ij D_ia, K = the group's cells, read from copies of
//             W, D and 1/Omega in group order (each group a contiguous run of rows); its own
//             kernel (k_group_sums_dmma), whose raw operands arrive by cp.async.
//   hk        HK[i, a] = sum_j O_ij tab[j][g(i)][a] for 128-cell tiles of each group, O read
//             from the group-ordered copies and HK scattered back to the cells; its own kernel
//             (k_hk), whose raw operands arrive by cp.async.
//
// Tile: 8 warps as WARPS_M x WARPS_N, each warp WM x WN DMMA tiles of 16 x 8, K slices of 16
// staged through registers (the next slice's global loads are in flight during the current
// slice's MMAs; operands computed from several loads keep the raw values in registers and do
// their arithmetic only when the slice is stored) into double-buffered shared memory laid out
// [k][m] and [k][n] with rows padded to 4 mod 16 doubles (conflict-free fragment loads).
#include <algorithm>
#include <cmath>

#include "dmma_common.cuh"
#include "gpl_internal.cuh"

namespace gpl {

namespace {

template <int WARPS_M_, int WM_, int WN_>
struct DTile {
  static constexpr int WARPS_M = WARPS_M_, WARPS_N = 8 / WARPS_M_, WM = WM_, WN = WN_;
  static constexpr int BM = WARPS_M * WM * 16, BN = WARPS_N * WN * 8, BK = 16;
  static constexpr int SA = BM + 4, SB = BN + 4;
  static constexpr int NA = BM * BK / 256, NB = BN * BK / 256;
  static constexpr int smem() { return (int)sizeof(double) * 2 * BK * (SA + SB); }
};
using TileSq = DTile<2, 4, 4>;    // 128 x 128
using TileTall = DTile<1, 9, 2>;  // 144 x 128: the dense columns (n_d <= 144) in one tile
using TileWide = DTile<4, 2, 9>;  // 128 x 144: the dense columns (n_d <= 144) across one tile

constexpr int kSplitK = 8;

}  // namespace

// A loader whose element combines several loaded values (a product, a scaled value) declares
// `Raw`, `load()` returning the loaded values and `finish()` doing the arithmetic: the kernel
// keeps the raw values in registers until it stores the slice into shared memory, so the next
// slice's loads stay in flight while the current slice's MMAs run. Other loaders return the
// element itself. finish(Raw{}) is 0 (the padding outside the matrix).
template <class L, class = void>
struct Staged {
  using Raw = double;
  __device__ static Raw load(const L& l, int a, int b, int z) { return l(a, b, z); }
  __device__ static double finish(const L&, const Raw& v) { return v; }
};
template <class L>
struct Staged<L, decltype((void)sizeof(typename L::Raw))> {
  using Raw = typename L::Raw;
  __device__ static Raw load(const L& l, int a, int b, int z) { return l.load(a, b, z); }
  __device__ static double finish(const L& l, const Raw& v) { return l.finish(v); }
};

// KR(z) -> [kbeg, kend); A(r, k, z); B(k, c, z); E(r, c, z, v). kFastK: the loader's K index
// is the contiguous one in memory (threads sweep k first).
template <class T, class LA, class LB, class KR, class Epi>
__global__ void __launch_bounds__(256, 1) k_dgen(int m, int n, LA A, LB B, KR kr, Epi epi) {
  extern __shared__ __align__(16) double sm[];
  double* As = sm;
  double* Bs = sm + 2 * T::BK * T::SA;
  constexpr int BK = T::BK;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int wm = warp / T::WARPS_N, wn = warp % T::WARPS_N;
  const int m0 = blockIdx.x * T::BM, n0 = blockIdx.y * T::BN, z = blockIdx.z;
  const int2 kk = kr(z);
  const int nsl = kk.y > kk.x ? (kk.y - kk.x + BK - 1) / BK : 0;
  using SA_ = Staged<LA>;
  using SB_ = Staged<LB>;
  typename SA_::Raw ra[T::NA];
  typename SB_::Raw rb[T::NB];

  auto fetch = [&](int s) {
    const int k0 = kk.x + s * BK;
#pragma unroll
    for (int q = 0; q < T::NA; q++) {
      const int e = tid + q * 256;
      int r, k;
      if (LA::kFastK) { k = e % BK; r = e / BK; } else { r = e % T::BM; k = e / T::BM; }
      ra[q] = (m0 + r < m && k0 + k < kk.y) ? SA_::load(A, m0 + r, k0 + k, z) : typename SA_::Raw{};
    }
#pragma unroll
    for (int q = 0; q < T::NB; q++) {
      const int e = tid + q * 256;
      int c, k;
      if (LB::kFastK) { k = e % BK; c = e / BK; } else { c = e % T::BN; k = e / T::BN; }
      rb[q] = (n0 + c < n && k0 + k < kk.y) ? SB_::load(B, k0 + k, n0 + c, z) : typename SB_::Raw{};
    }
  };
  auto stash = [&](int buf) {
    double* as = As + buf * BK * T::SA;
    double* bs = Bs + buf * BK * T::SB;
#pragma unroll
    for (int q = 0; q < T::NA; q++) {
      const int e = tid + q * 256;
      int r, k;
      if (LA::kFastK) { k = e % BK; r = e / BK; } else { r = e % T::BM; k = e / T::BM; }
      as[k * T::SA + r] = SA_::finish(A, ra[q]);
    }
#pragma unroll
    for (int q = 0; q < T::NB; q++) {
      const int e = tid + q * 256;
      int c, k;
      if (LB::kFastK) { k = e % BK; c = e / BK; } else { c = e % T::BN; k = e / T::BN; }
      bs[k * T::SB + c] = SB_::finish(B, rb[q]);
    }
  };

  double acc[T::WM][T::WN][4];
#pragma unroll
  for (int x = 0; x < T::WM; x++)
#pragma unroll
    for (int y = 0; y < T::WN; y++)
#pragma unroll
      for (int w = 0; w < 4; w++) acc[x][y][w] = 0.0;

  // The stash into buffer s & 1 happens after the barrier of slice s - 1, which every thread
  // passes only once it finished the MMAs of slice s - 2 that read that buffer.
  if (nsl > 0) fetch(0);
  for (int s = 0; s < nsl; s++) {
    const int buf = s & 1;
    stash(buf);
    __syncthreads();
    if (s + 1 < nsl) fetch(s + 1);
    const double* as = As + buf * BK * T::SA + wm * T::WM * 16 + g;
    const double* bs = Bs + buf * BK * T::SB + wn * T::WN * 8 + g;
#pragma unroll
    for (int k4 = 0; k4 < BK / 4; k4++) {
      double a[T::WM][2], b[T::WN];
#pragma unroll
      for (int x = 0; x < T::WM; x++) {
        a[x][0] = as[(k4 * 4 + t) * T::SA + x * 16];
        a[x][1] = as[(k4 * 4 + t) * T::SA + x * 16 + 8];
      }
#pragma unroll
      for (int y = 0; y < T::WN; y++) b[y] = bs[(k4 * 4 + t) * T::SB + y * 8];
#pragma unroll
      for (int x = 0; x < T::WM; x++)
#pragma unroll
        for (int y = 0; y < T::WN; y++) dmma_16x8x4(acc[x][y], a[x][0], a[x][1], b[y]);
    }
  }
#pragma unroll
  for (int x = 0; x < T::WM; x++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = m0 + wm * T::WM * 16 + x * 16 + g + 8 * h;
      if (r >= m) continue;
#pragma unroll
      for (int y = 0; y < T::WN; y++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int c = n0 + wn * T::WN * 8 + y * 8 + 2 * t + e;
          if (c < n) epi(r, c, z, acc[x][y][2 * h + e]);
        }
    }
}

// ---- operand loaders ------------------------------------------------------------------------
namespace {

struct KSplit {  // z-th of the equal ranges of [0, K)
  int K, per;
  __device__ int2 operator()(int z) const { return make_int2(min(K, z * per), min(K, (z + 1) * per)); }
};
struct KAll {
  int K;
  __device__ int2 operator()(int) const { return make_int2(0, K); }
};

struct LdTn {  // A(r = cell, k = gene) = (O nu - O E) / phi, O = W / Omega (1/phi given)
  static constexpr bool kFastK = false;
  const double *W, *Nu, *E, *rOm, *rphi;
  int ldN;
  struct Raw {
    double w, r, u, e, f;
  };
  __device__ Raw load(int r, int k, int) const {
    const size_t e = (size_t)k * ldN + r;
    return Raw{W[e], rOm[r], Nu[e], E[e], rphi[k]};
  }
  __device__ double finish(const Raw& v) const {
    const double o = v.w * v.r;
    return (o * v.u - o * v.e) * v.f;
  }
};
struct LdTBetaGP {  // B(k = gene, c = a) = tBeta[g0 + c + k*P]
  static constexpr bool kFastK = false;
  const double* tB;
  int P, g0;
  __device__ double operator()(int k, int c, int) const { return tB[g0 + c + (size_t)k * P]; }
};

// ---- epilogues -------------------------------------------------------------------------------
struct EpPart {  // split-K partials part[z][r][c]
  double* part;
  int m, n;
  __device__ void operator()(int r, int c, int z, double v) const { part[((size_t)z * m + r) * n + c] = v; }
};
struct EpColMajor {  // out[r + c*ld]
  double* out;
  int64_t ld;
  __device__ void operator()(int r, int c, int, double v) const { out[r + (size_t)c * ld] = v; }
};

// Un-whitening of the precision form's Gram, one gene per z: T = G L^T, then L T.
struct LdGene {  // A(r, k, z) = G_z[r + k*n] (r contiguous)
  static constexpr bool kFastK = false;
  const double* G;
  int n;
  __device__ double operator()(int r, int k, int z) const { return G[(size_t)z * n * n + r + (size_t)k * n]; }
};
struct LdGeneT {  // B(k, c, z) = T_z[k + c*n] (k contiguous)
  static constexpr bool kFastK = true;
  const double* T;
  int n;
  __device__ double operator()(int k, int c, int z) const { return T[(size_t)z * n * n + k + (size_t)c * n]; }
};
// L is the lower triangle of a factor whose strict upper triangle still holds the input
struct LdLT {  // B(k, c) = L[c][k] = L[c + k*n] (c contiguous), 0 above the diagonal
  static constexpr bool kFastK = false;
  const double* L;
  int n;
  __device__ double operator()(int k, int c, int) const { return c >= k ? L[c + (size_t)k * n] : 0.0; }
};
struct LdL {  // A(r, k) = L[r][k] = L[r + k*n] (r contiguous), 0 above the diagonal
  static constexpr bool kFastK = false;
  const double* L;
  int n;
  __device__ double operator()(int r, int k, int) const { return r >= k ? L[r + (size_t)k * n] : 0.0; }
};
struct LdGeneS {  // A(r = a, k = b, z) = S_z[dcol a, dcol b] (the dense block of Psi_z^{-1})
  static constexpr bool kFastK = false;
  const double* S;
  const int* dcol;
  int P;
  __device__ double operator()(int r, int k, int z) const {
    return S[(size_t)z * P * P + dcol[r] + (size_t)dcol[k] * P];
  }
};
struct LdLk {  // B(k, c) = L[k][c] = L[k + c*n] (k contiguous), 0 above the diagonal
  static constexpr bool kFastK = true;
  const double* L;
  int n;
  __device__ double operator()(int k, int c, int) const { return k >= c ? L[k + (size_t)c * n] : 0.0; }
};
struct LdLTk {  // A(r, k) = L[k][r] = L[k + r*n] (k contiguous), 0 above the diagonal
  static constexpr bool kFastK = true;
  const double* L;
  int n;
  __device__ double operator()(int r, int k, int) const { return k >= r ? L[k + (size_t)r * n] : 0.0; }
};
struct EpGene {  // T_z[r + c*n]
  double* T;
  int n;
  __device__ void operator()(int r, int c, int z, double v) const { T[(size_t)z * n * n + r + (size_t)c * n] = v; }
};
// The per-gene n x n products of the whitening as two GEMMs each, over all genes at once: the
// genes' matrices stacked as rows (A(r = z n + a, k)) against one n x n factor, or the factor
// against the genes' matrices side by side as columns (B(k, col = z n + c)).
struct LdGeneRows {  // A(r = z n + a, k) = G_z[a + k*n] (a contiguous)
  static constexpr bool kFastK = false;
  const double* G;
  int n;
  __device__ double operator()(int r, int k, int) const {
    const int z = r / n, a = r - z * n;
    return G[(size_t)z * n * n + a + (size_t)k * n];
  }
};
struct LdGeneSRows {  // A(r = z n + a, k) = S_z[dcol a, dcol k] (the dense block of Psi_z^{-1})
  static constexpr bool kFastK = false;
  const double* S;
  const int* dcol;
  int n, P;
  __device__ double operator()(int r, int k, int) const {
    const int z = r / n, a = r - z * n;
    return S[(size_t)z * P * P + dcol[a] + (size_t)dcol[k] * P];
  }
};
struct EpGeneRows {  // T_z[a + c*n] for r = z n + a
  double* T;
  int n;
  __device__ void operator()(int r, int c, int, double v) const {
    const int z = r / n, a = r - z * n;
    T[(size_t)z * n * n + a + (size_t)c * n] = v;
  }
};
struct EpPsiDDCols {  // column col = z n + c: Psi_z at (dcol r, dcol c) and its mirror, plus DeltaInv; r <= c
  double* Psi;
  const double* Dinv;
  const int* dcol;
  int P, n;
  __device__ void operator()(int r, int col, int, double v) const {
    const int z = col / n, c = col - z * n;
    if (r > c) return;
    const size_t mk = dcol[r], ml = dcol[c];
    const double x = v + Dinv[mk + ml * P];
    double* Pz = Psi + (size_t)z * P * P;
    Pz[mk + ml * P] = x;
    Pz[ml + mk * P] = x;
  }
};
struct EpPsiDD {  // Psi_z at (dcol r, dcol c) and its mirror, plus DeltaInv; r <= c only
  double* Psi;
  const double* Dinv;
  const int* dcol;
  int P;
  __device__ void operator()(int r, int c, int z, double v) const {
    if (r > c) return;
    const size_t mk = dcol[r], ml = dcol[c];
    const double x = v + Dinv[mk + ml * P];
    double* Pz = Psi + (size_t)z * P * P;
    Pz[mk + ml * P] = x;
    Pz[ml + mk * P] = x;
  }
};

}  // namespace

// bvec[dcol[a] + j*P] = sum_z part[z][a][j]
__global__ void k_reduce_bvec(int n_d, int J, int P, int nz, const int* __restrict__ dcol,
                              const double* __restrict__ part, double* __restrict__ bvec) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y;
  if (j >= J) return;
  double s = 0.0;
  for (int z = 0; z < nz; z++) s += part[((size_t)z * n_d + a) * J + j];
  bvec[dcol[a] + (size_t)j * P] = s;
}

template <class T, class LA, class LB, class KR, class Epi>
static int launch_dgen(Ctx* c, dim3 grid, int m, int n, LA A, LB B, KR kr, Epi epi, const char* name) {
  auto* fn = k_dgen<T, LA, LB, KR, Epi>;
  const int smem = T::smem();
  GPL_TRY(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  fn<<<grid, 256, smem, c->stream>>>(m, n, A, B, kr, epi);
  GPL_LAUNCHED(c, name);
  return GPL_OK;
}

static int ensure_part(Ctx* c, size_t n) {
  if (c->part_n >= n) return GPL_OK;
  graph_reset(c);
  if (c->part) cudaFree(c->part);
  c->part = nullptr;
  c->part_n = 0;
  if (cudaMalloc((void**)&c->part, sizeof(double) * n) != cudaSuccess) {
    cudaGetLastError();
    c->err = "device allocation failed: split-K partials";
    return GPL_ERR_ALLOC;
  }
  c->part_n = n;
  return GPL_OK;
}

// The number of cell ranges of a split-K launch of `tiles` output tiles at one CTA per SM: the
// S in [8, 32] whose S x tiles CTAs fill their last wave best (the smallest such S). At config 2
// (79 gene tiles, 148 SMs) S = 28 puts 2,212 CTAs in 14.95 waves where S = 8 gave 4.27 waves.
static int split_count(int tiles, int sms) {
  int best = kSplitK;
  double best_fill = 0.0;
  for (int s = kSplitK; s <= 32; s++) {
    const double waves = (double)tiles * s / sms;
    const double fill = waves / std::ceil(waves);
    if (fill > best_fill + 1e-9) {
      best_fill = fill;
      best = s;
    }
  }
  return best;
}

// Z^T u with the operands' raw values copied by cp.async: a three-stage pipeline of 16-cell
// slices (the dense columns [a][cell], W and u [gene][cell], cells contiguous in rows of kZtS;
// 1/Omega and a per-cell u [cell]) with one barrier per slice, the B operand w * (1/Omega) * u
// formed as its fragments are read (the same product, in the same order, as the register-staged
// form, so the sums are those of TileTall's k_dgen over the same cell ranges). Tile: all dense
// columns (<= 144) x 128 genes, 8 warps along the genes, each 9 x 2 DMMA tiles of 16 x 8; CTA
// (gene tile, cell range z) writes its partial sums to part[z][a][j]. MODE 0: B = W u / Omega
// (u cells x genes); 1: B = u; 2: B = W g / Omega with g one value per cell. The cell ranges
// start at even cells, so every 16-byte copy is aligned (ldN is a multiple of 32).
namespace {
constexpr int kZtBK = 16, kZtS = kZtBK + 4;  // slice depth; row stride, 4 mod 16 doubles
constexpr int kZtBM = 144, kZtBN = 128, kZtStages = 3;
constexpr int kZtStage = kZtBM * kZtS + 2 * kZtBN * kZtS + 2 * kZtBK;  // doubles per stage
constexpr int kZtSmem = (int)sizeof(double) * kZtStages * kZtStage;
}  // namespace

template <int MODE>
__global__ void __launch_bounds__(256, 1)
    k_zt_u(int m, int n, int N, int ldN, int per, const double* __restrict__ D, const double* __restrict__ W,
           const double* __restrict__ U, const double* __restrict__ rOm, double* __restrict__ part) {
  extern __shared__ __align__(16) double zs[];
  const int tid = threadIdx.x, wn = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int n0 = blockIdx.y * kZtBN, z = blockIdx.z;
  const int kbeg = min(N, z * per), kend = min(N, (z + 1) * per);
  const int nsl = kend > kbeg ? (kend - kbeg + kZtBK - 1) / kZtBK : 0;

  // slice s into stage st; a pair of cells past the range is zero-filled (8 bytes of a pair
  // whose second cell is past it), its source clamped into the matrix
  auto load = [&](int s, int st) {
    double* As = zs + st * kZtStage;
    double* Ws = As + kZtBM * kZtS;
    double* Us = Ws + kZtBN * kZtS;
    double* Rs = Us + kZtBN * kZtS;
    double* Vs = Rs + kZtBK;
    const int k0 = kbeg + s * kZtBK;
    for (int ch = tid; ch < kZtBM * (kZtBK / 2); ch += 256) {
      const int r = ch >> 3, kc = (ch & 7) * 2, k = k0 + kc;
      const int nb = (r < m && k < kend) ? (k + 1 < kend ? 16 : 8) : 0;
      cp_async16(As + r * kZtS + kc, D + (size_t)min(r, m - 1) * ldN + min(k, ldN - 2), nb);
    }
#pragma unroll
    for (int q = 0; q < (kZtBN * (kZtBK / 2)) / 256; q++) {
      const int ch = tid + q * 256;
      const int cc = ch >> 3, kc = (ch & 7) * 2, k = k0 + kc;
      const int nb = (n0 + cc < n && k < kend) ? (k + 1 < kend ? 16 : 8) : 0;
      const size_t src = (size_t)min(n0 + cc, n - 1) * ldN + min(k, ldN - 2);
      if (MODE != 1) cp_async16(Ws + cc * kZtS + kc, W + src, nb);
      if (MODE != 2) cp_async16(Us + cc * kZtS + kc, U + src, nb);
    }
    if (tid < kZtBK) {
      const int k = k0 + tid, nb = k < kend ? 8 : 0;
      if (MODE != 1) cp_async8(Rs + tid, rOm + min(k, N - 1), nb);
      if (MODE == 2) cp_async8(Vs + tid, U + min(k, N - 1), nb);
    }
  };

  double acc[9][2][4];
#pragma unroll
  for (int x = 0; x < 9; x++)
#pragma unroll
    for (int y = 0; y < 2; y++)
#pragma unroll
      for (int w = 0; w < 4; w++) acc[x][y][w] = 0.0;
  if (nsl > 0) load(0, 0);
  cp_async_commit();
  if (nsl > 1) load(1, 1);
  cp_async_commit();
  for (int s = 0; s < nsl; s++) {
    cp_async_wait<1>();  // slice s landed
    __syncthreads();     // and every warp is done with slice s - 1, whose stage is refilled next
    if (s + 2 < nsl) load(s + 2, (s + 2) % kZtStages);
    cp_async_commit();
    const double* As = zs + (s % kZtStages) * kZtStage;
    const double* Ws = As + kZtBM * kZtS;
    const double* Us = Ws + kZtBN * kZtS;
    const double* Rs = Us + kZtBN * kZtS;
    const double* Vs = Rs + kZtBK;
#pragma unroll
    for (int k4 = 0; k4 < kZtBK / 4; k4++) {
      const int kk = k4 * 4 + t;
      double a[9][2], b[2];
#pragma unroll
      for (int x = 0; x < 9; x++) {
        a[x][0] = As[(x * 16 + g) * kZtS + kk];
        a[x][1] = As[(x * 16 + g + 8) * kZtS + kk];
      }
#pragma unroll
      for (int y = 0; y < 2; y++) {
        const int e = (wn * 16 + y * 8 + g) * kZtS + kk;
        b[y] = MODE == 1 ? Us[e] : MODE == 0 ? Ws[e] * Rs[kk] * Us[e] : Ws[e] * Rs[kk] * Vs[kk];
      }
#pragma unroll
      for (int x = 0; x < 9; x++)
#pragma unroll
        for (int y = 0; y < 2; y++) dmma_16x8x4(acc[x][y], a[x][0], a[x][1], b[y]);
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int x = 0; x < 9; x++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = x * 16 + g + 8 * h;
      if (r >= m) continue;
#pragma unroll
      for (int y = 0; y < 2; y++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int cc = n0 + wn * 16 + y * 8 + 2 * t + e;
          if (cc < n) part[((size_t)z * m + r) * n + cc] = acc[x][y][2 * h + e];
        }
    }
}

int dgen_zt_u(Ctx* c, int mode, const double* u, double* out) {
  if (c->n_d > kZtBM) return GPL_ERR_ARG;
  const double* rOm = nullptr;
  if (mode != 1) {
    int rc = recip_omega(c, &rOm);
    if (rc) return rc;
  }
  const int tiles = div_up(c->J, kZtBN);
  const int S = split_count(tiles, c->sm_count);
  int rc = ensure_part(c, (size_t)S * c->n_d * c->J);
  if (rc) return rc;
  int per = (c->N + S - 1) / S;
  per += per & 1;  // even range starts: aligned 16-byte copies
  dim3 g(1, tiles, S);
  auto* fn = mode == 0 ? k_zt_u<0> : mode == 1 ? k_zt_u<1> : k_zt_u<2>;
  GPL_TRY(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kZtSmem));
  fn<<<g, 256, kZtSmem, c->stream>>>(c->n_d, c->J, c->N, c->ldN, per, c->Dm, c->W, u, rOm, c->part);
  GPL_LAUNCHED(c, "k_zt_u");
  dim3 g2(div_up(c->J, 256), c->n_d);
  k_reduce_bvec<<<g2, 256, 0, c->stream>>>(c->n_d, c->J, c->P, S, c->dcol_d, c->part, out);
  GPL_LAUNCHED(c, "k_reduce_bvec");
  return GPL_OK;
}

// C1 over S gene ranges (S = 1..4, the count whose CTAs fill their last wave best: 3 at config
// 2, 2,346 CTAs in 15.85 waves against 782 in 5.28) whose partials are added in order.
__global__ void k_reduce_parts_ld(int m, int n, int nz, const double* __restrict__ part, double* __restrict__ out,
                                  int64_t ld) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, cc = blockIdx.y;
  if (r >= m) return;
  double s = 0.0;
  for (int z = 0; z < nz; z++) s += part[((size_t)z * m + r) * n + cc];
  out[r + (size_t)cc * ld] = s;
}

int dgen_c1_tn(Ctx* c) {
  using T = TileSq;
  const double* rOm = nullptr;
  int rc = recip_omega(c, &rOm);
  if (rc) return rc;
  const int g0 = c->nh[c->p - 1];
  const int tiles = div_up(c->N, T::BM) * div_up(c->M, T::BN);
  int S = 1;
  double best = 0.0;
  for (int z = 1; z <= 4; z++) {
    const double waves = (double)tiles * z / c->sm_count, fill = waves / std::ceil(waves);
    if (fill > best + 1e-9) {
      best = fill;
      S = z;
    }
  }
  LdTn A{c->W, c->Nu, c->scratch, rOm, c->rphi, c->ldN};
  LdTBetaGP B{c->tBeta, c->P, g0};
  if (S == 1) {
    dim3 g(div_up(c->N, T::BM), div_up(c->M, T::BN), 1);
    return launch_dgen<T>(c, g, c->N, c->M, A, B, KAll{c->J}, EpColMajor{c->C1, (int64_t)c->ldN}, "k_dgen(c1_tn)");
  }
  if ((rc = ensure_part(c, (size_t)S * c->N * c->M))) return rc;
  dim3 g(div_up(c->N, T::BM), div_up(c->M, T::BN), S);
  rc = launch_dgen<T>(c, g, c->N, c->M, A, B, KSplit{c->J, (c->J + S - 1) / S}, EpPart{c->part, c->N, c->M},
                      "k_dgen(c1_tn)");
  if (rc) return rc;
  dim3 g2(div_up(c->N, 256), c->M);
  k_reduce_parts_ld<<<g2, 256, 0, c->stream>>>(c->N, c->M, S, c->part, c->C1, (int64_t)c->ldN);
  GPL_LAUNCHED(c, "k_reduce_parts_ld");
  return GPL_OK;
}

// S[j][g][a] = sum over group g's cells of w_ij D_ia (w = W/Omega, MODE 0; 1, MODE 1): grid
// (gene tiles, groups), the group's cells (a contiguous run in group order) in 16-cell slices
// through a three-stage cp.async pipeline of the raw operands, 8-byte copies (a group starts at
// any cell): the dense columns [a][cell] from their group-ordered copy, W's group-ordered values
// [gene][cell] and 1/Omega [cell]; w formed at the fragment loads, the same product in the same
// order as the register-staged form, so the sums are TileTall's.
template <int MODE>
__global__ void __launch_bounds__(256, 1)
    k_group_sums_dmma(int m, int n, int n_grp, int ldN, const int* __restrict__ gstart, const double* __restrict__ Dg,
                      const double* __restrict__ Wg, const double* __restrict__ rOmg, double* __restrict__ S) {
  extern __shared__ __align__(16) double zs[];
  const int tid = threadIdx.x, wn = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int n0 = blockIdx.y * kZtBN, z = blockIdx.z;
  const int kbeg = gstart[z], kend = gstart[z + 1];
  const int nsl = kend > kbeg ? (kend - kbeg + kZtBK - 1) / kZtBK : 0;
  const int last = max(kend - 1, 0);  // a cell of the matrix, for the sources of zero-fill copies

  auto load = [&](int s, int st) {
    double* As = zs + st * kZtStage;
    double* Ws = As + kZtBM * kZtS;
    double* Rs = Ws + 2 * kZtBN * kZtS;
    const int k0 = kbeg + s * kZtBK;
    for (int e = tid; e < kZtBM * kZtBK; e += 256) {
      const int r = e >> 4, kc = e & 15, k = k0 + kc;
      const int nb = (r < m && k < kend) ? 8 : 0;
      cp_async8(As + r * kZtS + kc, Dg + (size_t)min(r, m - 1) * ldN + min(k, last), nb);
    }
    if (MODE == 0) {
#pragma unroll
      for (int q = 0; q < (kZtBN * kZtBK) / 256; q++) {
        const int e = tid + q * 256, cc = e >> 4, kc = e & 15, k = k0 + kc;
        const int nb = (n0 + cc < n && k < kend) ? 8 : 0;
        cp_async8(Ws + cc * kZtS + kc, Wg + (size_t)min(n0 + cc, n - 1) * ldN + min(k, last), nb);
      }
      if (tid < kZtBK) {
        const int k = k0 + tid;
        cp_async8(Rs + tid, rOmg + min(k, last), k < kend ? 8 : 0);
      }
    }
  };

  double acc[9][2][4];
#pragma unroll
  for (int x = 0; x < 9; x++)
#pragma unroll
    for (int y = 0; y < 2; y++)
#pragma unroll
      for (int w = 0; w < 4; w++) acc[x][y][w] = 0.0;
  if (nsl > 0) load(0, 0);
  cp_async_commit();
  if (nsl > 1) load(1, 1);
  cp_async_commit();
  for (int s = 0; s < nsl; s++) {
    cp_async_wait<1>();  // slice s landed
    __syncthreads();     // and every warp is done with slice s - 1, whose stage is refilled next
    if (s + 2 < nsl) load(s + 2, (s + 2) % kZtStages);
    cp_async_commit();
    const double* As = zs + (s % kZtStages) * kZtStage;
    const double* Ws = As + kZtBM * kZtS;
    const double* Rs = Ws + 2 * kZtBN * kZtS;
    const int live = kend - (kbeg + s * kZtBK);  // cells of this slice in the group
#pragma unroll
    for (int k4 = 0; k4 < kZtBK / 4; k4++) {
      const int kk = k4 * 4 + t;
      double a[9][2], b[2];
#pragma unroll
      for (int x = 0; x < 9; x++) {
        a[x][0] = As[(x * 16 + g) * kZtS + kk];
        a[x][1] = As[(x * 16 + g + 8) * kZtS + kk];
      }
#pragma unroll
      for (int y = 0; y < 2; y++) {
        const int e = (wn * 16 + y * 8 + g) * kZtS + kk;
        b[y] = MODE == 0 ? Ws[e] * Rs[kk] : (kk < live && n0 + wn * 16 + y * 8 + g < n ? 1.0 * 1.0 : 0.0);
      }
#pragma unroll
      for (int x = 0; x < 9; x++)
#pragma unroll
        for (int y = 0; y < 2; y++) dmma_16x8x4(acc[x][y], a[x][0], a[x][1], b[y]);
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int x = 0; x < 9; x++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = x * 16 + g + 8 * h;
      if (r >= m) continue;
#pragma unroll
      for (int y = 0; y < 2; y++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int j = n0 + wn * 16 + y * 8 + 2 * t + e;
          if (j < n) S[((size_t)j * n_grp + z) * (m + 1) + r] = acc[x][y][2 * h + e];
        }
    }
}

int dgen_group_sums(Ctx* c, int mode) {
  if (c->n_d > kZtBM) return GPL_ERR_ARG;
  int rc;
  if (mode == 0) {
    const double* rOm = nullptr;
    if ((rc = recip_omega(c, &rOm))) return rc;
    if ((rc = launch_group_order(c, rOm, 1, c->rOmg))) return rc;
  }
  if ((rc = launch_group_order(c, c->Dm, c->n_d, c->Dg))) return rc;
  const int J = mode == 1 ? 1 : c->J;
  dim3 g(1, div_up(J, kZtBN), c->n_grp);
  auto* fn = mode == 0 ? k_group_sums_dmma<0> : k_group_sums_dmma<1>;
  GPL_TRY(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kZtSmem));
  fn<<<g, 256, kZtSmem, c->stream>>>(c->n_d, J, c->n_grp, c->ldN, c->gstart_d, c->Dg, c->Wg, c->rOmg, c->gsum);
  GPL_LAUNCHED(c, "k_group_sums_dmma");
  return GPL_OK;
}

// HK[i, a] = sum_j O_ij tab[j][g(i)][a] for the 128 cell slots of each group tile (grid z =
// tile), the genes in 16-deep slices through a four-stage cp.async pipeline of the raw operands:
// the group's table rows tab[j][g][0..ld) ([gene][a]) and W's group-ordered values of the tile's
// slots ([gene][slot]), by 8-byte copies (neither row starts at an even offset in general);
// 1/Omega of the slots is read once. The B operand W (1/Omega) is formed at the fragment loads,
// the same product in the same order as the register-staged form, so the sums are TileTall's.
namespace {
constexpr int kHkBK = 16, kHkSA = 148, kHkSB = 132, kHkStages = 4;  // row strides 4 mod 16
constexpr int kHkStage = kHkBK * kHkSA + kHkBK * kHkSB;             // doubles per stage
constexpr int kHkSmem = (int)sizeof(double) * (kHkStages * kHkStage + 128);
}  // namespace

__global__ void __launch_bounds__(256, 1)
    k_hk(int ld, int J, int n_grp, int ldN, const double* __restrict__ tab, const int2* __restrict__ tiles,
         const double* __restrict__ Wg, const double* __restrict__ rOmg, const int* __restrict__ pos,
         const int* __restrict__ cells, double* __restrict__ HK) {
  extern __shared__ __align__(16) double hs[];
  double* Rs = hs + kHkStages * kHkStage;  // [128] 1/Omega of the slots, 0 past the group
  const int tid = threadIdx.x, wn = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int z = blockIdx.z, grp = tiles[z].x;
  const int myq = pos[(size_t)z * 128 + (tid & 127)];  // this thread's slot in every B copy
  if (tid < 128) Rs[tid] = myq < 0 ? 0.0 : rOmg[myq];
  const int nsl = (J + kHkBK - 1) / kHkBK;

  auto load = [&](int s, int st) {
    double* As = hs + st * kHkStage;
    double* Bs = As + kHkBK * kHkSA;
    const int k0 = s * kHkBK;
    for (int e = tid; e < kHkBK * 144; e += 256) {
      const int k = e / 144, r = e - k * 144, j = k0 + k;
      const int nb = (r < ld && j < J) ? 8 : 0;
      cp_async8(As + k * kHkSA + r, tab + ((size_t)min(j, J - 1) * n_grp + grp) * ld + min(r, ld - 1), nb);
    }
#pragma unroll
    for (int q = 0; q < (kHkBK * 128) / 256; q++) {
      const int k = (tid >> 7) + 2 * q, j = k0 + k;
      const int nb = (myq >= 0 && j < J) ? 8 : 0;
      cp_async8(Bs + k * kHkSB + (tid & 127), Wg + (size_t)min(j, J - 1) * ldN + max(myq, 0), nb);
    }
  };

  double acc[9][2][4];
#pragma unroll
  for (int x = 0; x < 9; x++)
#pragma unroll
    for (int y = 0; y < 2; y++)
#pragma unroll
      for (int w = 0; w < 4; w++) acc[x][y][w] = 0.0;
#pragma unroll
  for (int s = 0; s < kHkStages - 1; s++) {
    if (s < nsl) load(s, s);
    cp_async_commit();
  }
  for (int s = 0; s < nsl; s++) {
    cp_async_wait<kHkStages - 2>();  // slice s landed
    __syncthreads();                 // and every warp is done with slice s - 1, whose stage is refilled next
    if (s + kHkStages - 1 < nsl) load(s + kHkStages - 1, (s + kHkStages - 1) % kHkStages);
    cp_async_commit();
    const double* As = hs + (s % kHkStages) * kHkStage;
    const double* Bs = As + kHkBK * kHkSA;
#pragma unroll
    for (int k4 = 0; k4 < kHkBK / 4; k4++) {
      const int kk = k4 * 4 + t;
      double a[9][2], b[2];
#pragma unroll
      for (int x = 0; x < 9; x++) {
        a[x][0] = As[kk * kHkSA + x * 16 + g];
        a[x][1] = As[kk * kHkSA + x * 16 + g + 8];
      }
#pragma unroll
      for (int y = 0; y < 2; y++) {
        const int cs = wn * 16 + y * 8 + g;
        b[y] = Bs[kk * kHkSB + cs] * Rs[cs];
      }
#pragma unroll
      for (int x = 0; x < 9; x++)
#pragma unroll
        for (int y = 0; y < 2; y++) dmma_16x8x4(acc[x][y], a[x][0], a[x][1], b[y]);
    }
  }
  cp_async_wait<0>();
  const int* cz = cells + (size_t)z * 128;
#pragma unroll
  for (int x = 0; x < 9; x++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = x * 16 + g + 8 * h;
      if (r >= ld) continue;
#pragma unroll
      for (int y = 0; y < 2; y++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int i = cz[wn * 16 + y * 8 + 2 * t + e];
          if (i >= 0) HK[i + (size_t)r * ldN] = acc[x][y][2 * h + e];
        }
    }
}

int dgen_hk(Ctx* c) {
  const int ld = c->n_d + 1;
  if (ld > 144) return GPL_ERR_ARG;
  const double* rOm = nullptr;
  int rc = recip_omega(c, &rOm);
  if (rc) return rc;
  if ((rc = launch_group_order(c, rOm, 1, c->rOmg))) return rc;
  if (c->n_hk_tiles128 == 0) return GPL_OK;
  GPL_TRY(c, cudaFuncSetAttribute(k_hk, cudaFuncAttributeMaxDynamicSharedMemorySize, kHkSmem));
  k_hk<<<dim3(1, 1, c->n_hk_tiles128), 256, kHkSmem, c->stream>>>(ld, c->J, c->n_grp, c->ldN, c->gsum,
                                                                   c->hk_tiles128_d, c->Wg, c->rOmg, c->hk_pos_d,
                                                                   c->hk_cells_d, c->HK);
  GPL_LAUNCHED(c, "k_hk");
  return GPL_OK;
}

// Psi_DD,j = L G~_j L^T + DeltaInv_DD for every gene: T_j = G~_j L^T as one GEMM over the stacked
// rows of all genes (J n x n against L^T), then L T_j as one GEMM over the genes' columns side by
// side (L against n x J n). Per gene (grid z = gene) where J n exceeds the grid's column limit.
int dgen_unwhiten(Ctx* c, const double* Gt, double* Tt, const double* Lw) {
  const int n = c->n_d;
  const int64_t Jn = (int64_t)c->J * n;
  if (n > TileWide::BN || n > TileTall::BM) return GPL_ERR_ARG;
  if (div_up(Jn, (int64_t)TileTall::BN) <= 65535) {
    int rc = launch_dgen<TileWide>(c, dim3((unsigned)div_up(Jn, (int64_t)TileWide::BM), 1, 1), (int)Jn, n,
                                   LdGeneRows{Gt, n}, LdLT{Lw, n}, KAll{n}, EpGeneRows{Tt, n},
                                   "k_dgen(unwhiten GL^T)");
    if (rc) return rc;
    return launch_dgen<TileTall>(c, dim3(1, (unsigned)div_up(Jn, (int64_t)TileTall::BN), 1), n, (int)Jn,
                                 LdL{Lw, n}, LdGeneT{Tt, n}, KAll{n},
                                 EpPsiDDCols{c->Psi, c->DeltaInv, c->dcol_d, c->P, n}, "k_dgen(unwhiten L(GL^T))");
  }
  using T = TileTall;
  if (c->J > 65535) return GPL_ERR_ARG;
  dim3 g(1, div_up(n, T::BN), c->J);
  int rc = launch_dgen<T>(c, g, n, n, LdGene{Gt, n}, LdLT{Lw, n}, KAll{n}, EpGene{Tt, n}, "k_dgen(unwhiten GL^T)");
  if (rc) return rc;
  return launch_dgen<T>(c, g, n, n, LdL{Lw, n}, LdGeneT{Tt, n}, KAll{n}, EpPsiDD{c->Psi, c->DeltaInv, c->dcol_d, c->P},
                        "k_dgen(unwhiten L(GL^T))");
}

// S~_j = L^T S_DD,j L for every gene, in the same two stacked GEMMs (S_DD,j L over the genes'
// rows, then L^T against the genes' columns).
int dgen_whiten_inverse(Ctx* c, const double* Lw, double* Tt, double* St) {
  const int n = c->n_d;
  const int64_t Jn = (int64_t)c->J * n;
  if (n > TileWide::BN || n > TileTall::BM) return GPL_ERR_ARG;
  if (div_up(Jn, (int64_t)TileTall::BN) <= 65535) {
    int rc = launch_dgen<TileWide>(c, dim3((unsigned)div_up(Jn, (int64_t)TileWide::BM), 1, 1), (int)Jn, n,
                                   LdGeneSRows{c->PsiInv, c->dcol_d, n, c->P}, LdLk{Lw, n}, KAll{n},
                                   EpGeneRows{Tt, n}, "k_dgen(S L)");
    if (rc) return rc;
    return launch_dgen<TileTall>(c, dim3(1, (unsigned)div_up(Jn, (int64_t)TileTall::BN), 1), n, (int)Jn,
                                 LdLTk{Lw, n}, LdGeneT{Tt, n}, KAll{n}, EpGene{St, n}, "k_dgen(L^T S L)");
  }
  using T = TileTall;
  if (c->J > 65535) return GPL_ERR_ARG;
  dim3 g(1, div_up(n, T::BN), c->J);
  int rc = launch_dgen<T>(c, g, n, n, LdGeneS{c->PsiInv, c->dcol_d, c->P}, LdLk{Lw, n}, KAll{n}, EpGene{Tt, n},
                          "k_dgen(S L)");
  if (rc) return rc;
  return launch_dgen<T>(c, g, n, n, LdLTk{Lw, n}, LdGeneT{Tt, n}, KAll{n}, EpGene{St, n}, "k_dgen(L^T S L)");
}

// Score statistics: C[j][c] = sum_i W_ij G2[c][i] over all cells, split over the cells into
// kSplitK ranges whose partials are added in order.
namespace {
struct LdWrow {  // A(r = gene, k = cell) = W[r*ldN + k]
  static constexpr bool kFastK = true;
  const double* W;
  int ldN;
  __device__ double operator()(int r, int k, int) const { return W[(size_t)r * ldN + k]; }
};
struct LdCols {  // B(k = cell, c) = G2[c*N + k]
  static constexpr bool kFastK = true;
  const double* G2;
  int N;
  __device__ double operator()(int k, int c, int) const { return G2[(size_t)c * N + k]; }
};
}  // namespace

__global__ void k_reduce_parts(int m, int n, int nz, const double* __restrict__ part, double* __restrict__ out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, cc = blockIdx.y;
  if (r >= m) return;
  double s = 0.0;
  for (int z = 0; z < nz; z++) s += part[((size_t)z * m + r) * n + cc];
  out[r + (size_t)cc * m] = s;
}

int dgen_weighted_colsums(Ctx* c, const double* G2, int n2, double* out) {
  using T = TileSq;
  if (n2 > T::BN) return GPL_ERR_ARG;
  int rc = ensure_part(c, (size_t)kSplitK * c->J * n2);
  if (rc) return rc;
  const int per = (c->N + kSplitK - 1) / kSplitK;
  dim3 g(div_up(c->J, T::BM), 1, kSplitK);
  rc = launch_dgen<T>(c, g, c->J, n2, LdWrow{c->W, c->ldN}, LdCols{G2, c->N}, KSplit{c->N, per},
                      EpPart{c->part, c->J, n2}, "k_dgen(score sums)");
  if (rc) return rc;
  dim3 g2(div_up(c->J, 256), n2);
  k_reduce_parts<<<g2, 256, 0, c->stream>>>(c->J, n2, kSplitK, c->part, out);
  GPL_LAUNCHED(c, "k_reduce_parts");
  return GPL_OK;
}

}  // namespace gpl
