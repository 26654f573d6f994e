// FP64 tensor-core (DMMA, mma.sync m16n8k4 .f64) forms of the two dominant contractions of
// the plain FP64 path. Both are written over the unique column pairs (a <= b) of the dense
// model columns, which turns the per-gene P x P products into two plain GEMMs and uses the
// symmetry of Psi_j and Psi_j^{-1} to halve the work.
//
//   k_pair_products  A[i, p] = D_ia D_ib / Omega_i for a range of cells, row-major with the
//                 pairs contiguous (the layout of V): the Gram's K-major A operand, written once
//                 per range (N * pairs doubles in all; a few ms of HBM writes per Gram).
//   k_pair_gram   G[p, j] = sum_i A[i, p] W_ij over a range of cells (M = pairs, N = genes,
//                 K = cells), both operands by cp.async (three stages, one barrier per slice),
//                 written straight into Psi_j (both triangles, plus DeltaInv) at model columns
//                 (dcol a, dcol b) when one range covers all cells: the dense block of getPsi
//                 (ggplvm.cu:621-680); otherwise added up range by range in a pairs x genes
//                 buffer that k_pair_scatter moves into Psi. Work: N*J*n_d*(n_d+1) flops.
//   k_pair_v      V[i, p] = (1/Omega_i) sum_j W_ij S_j[a, b] for a cell range, S_j = Psi_j^{-1}
//                 gathered per pair (k_gather_spair). M = cells, N = pairs, K = genes; both
//                 operands by cp.async. Work: N*J*n_d*(n_d+1) flops.
//   k_v_to_u      U[i, a] = sum_b D_ib V[i, pair(a, b)]: the gradient contraction
//                 sum_j O_ij S_j[DD] d_i of getGradLogOmega (ggplvm.cu:301-376) from V.
//
// CTA tile 128 x 128 x 16 (K), 8 warps as 2 (M) x 4 (N), warp tile 64 x 32 (4 x 4 DMMA tiles
// of 16 x 8), three-stage cp.async pipelines with one barrier per slice. m16n8k4 fragments (lane = 4*g + t):
// A 16x4 row-major a0 = A[g][t], a1 = A[g+8][t]; B 4x8 b0 = B[t][g]; C 16x8
// c0,c1 = C[g][2t, 2t+1], c2,c3 = C[g+8][2t, 2t+1]. Shared rows are padded so that the
// 16 lanes of each half-warp hit 16 distinct 8-byte bank pairs.
#include <algorithm>
#include <cstdlib>

#include "dmma_common.cuh"
#include "gpl_internal.cuh"

namespace gpl {

namespace {
constexpr int BM = 128, BN = 128, BK = 16;
constexpr int SA = BM + 4;   // As[k][m]
constexpr int SBT = BK + 4;  // Bs[n][k] (weights, k contiguous)
constexpr int SBN = BN + 4;  // Bs[k][n] (S pairs, n contiguous)
constexpr int kThreads = 256;
}  // namespace

// Grouped tile order: a 1-D grid of tm x tn output tiles in which consecutive blocks walk
// group_m tile rows down one tile column before moving to the next column, so that the ~148
// resident blocks cover a group_m x ~(148 / group_m) patch and share both operands' tiles
// through L2 (row-major order would re-read one operand from DRAM for nearly every block).
// group_m is the autotuner's choice (default 12); it changes only which block computes which
// tile, never a tile's sums.
constexpr int kGroupM = 12;
__device__ __forceinline__ int2 grouped_tile(int id, int tm, int tn, int group_m) {
  const int per = group_m * tn;
  const int grp = id / per, first = grp * group_m;
  const int gm = min(tm - first, group_m);
  const int r = id - grp * per;
  return make_int2(first + r % gm, r / gm);
}

// One 16-deep K slice of the warp tile. kNT: B stored [n][k] (true) or [k][n] (false).
template <bool kNT>
__device__ __forceinline__ void warp_slice(const double* __restrict__ As, const double* __restrict__ Bs, int wm,
                                           int wn, int g, int t, double (&acc)[4][4][4]) {
#pragma unroll
  for (int kk = 0; kk < BK / 4; kk++) {
    double a[4][2], b[4];
    const double* ar = As + (kk * 4 + t) * SA + wm * 64 + g;
#pragma unroll
    for (int mt = 0; mt < 4; mt++) {
      a[mt][0] = ar[mt * 16];
      a[mt][1] = ar[mt * 16 + 8];
    }
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
      const int n = wn * 32 + nt * 8 + g;
      b[nt] = kNT ? Bs[n * SBT + kk * 4 + t] : Bs[(kk * 4 + t) * SBN + n];
    }
#pragma unroll
    for (int mt = 0; mt < 4; mt++)
#pragma unroll
      for (int nt = 0; nt < 4; nt++) dmma_16x8x4(acc[mt][nt], a[mt][0], a[mt][1], b[nt]);
  }
}

// ---------------------------------------------------------------------------------------------
// Gram over the dense column pairs
// ---------------------------------------------------------------------------------------------
// A[(i - c0) * pairs_pad + p] for cells [c0, c1): 8 cells per block, their dense-column
// values and 1/Omega staged in shared memory, stores along the pairs (coalesced). Padding
// pairs and cells past N (1/Omega = 0 there) give 0.
constexpr int kProdCells = 8;

__global__ void __launch_bounds__(256) k_pair_products(int ldN, int n_d, int c0, int c1, int n_pairs, int pairs_pad,
                                                       const int2* __restrict__ pairs, const double* __restrict__ D,
                                                       const double* __restrict__ rOm, double* __restrict__ A) {
  extern __shared__ double dsh[];  // [n_d][kProdCells] then rOm[kProdCells]
  const int i0 = c0 + blockIdx.x * kProdCells;
  const int nc = min(kProdCells, c1 - i0);
  for (int e = threadIdx.x; e < n_d * kProdCells; e += blockDim.x) {
    const int a = e / kProdCells, r = e - a * kProdCells;
    dsh[e] = r < nc ? D[(size_t)a * ldN + i0 + r] : 0.0;
  }
  if (threadIdx.x < kProdCells) dsh[n_d * kProdCells + threadIdx.x] = threadIdx.x < nc ? rOm[i0 + threadIdx.x] : 0.0;
  __syncthreads();
  const double* ro = dsh + n_d * kProdCells;
  for (int p = threadIdx.x; p < pairs_pad; p += blockDim.x) {
    double v[kProdCells];
    if (p < n_pairs) {
      const int2 q = pairs[p];
      const double* da = dsh + q.x * kProdCells;
      const double* db = dsh + q.y * kProdCells;
#pragma unroll
      for (int r = 0; r < kProdCells; r++) v[r] = da[r] * db[r] * ro[r];
    } else {
#pragma unroll
      for (int r = 0; r < kProdCells; r++) v[r] = 0.0;
    }
    for (int r = 0; r < nc; r++) A[(size_t)(i0 - c0 + r) * pairs_pad + p] = v[r];
  }
}

// epilogue modes of k_pair_gram
constexpr int kGramPsi = 0;  // one range: Psi_j[mk, ml] = Psi_j[ml, mk] = G + DeltaInv
constexpr int kGramSet = 1;  // first of several ranges: Gacc[p * J + j] = G
constexpr int kGramAdd = 2;  // later ranges: Gacc[p * J + j] += G

__global__ void __launch_bounds__(kThreads, 1)
    k_pair_gram(int N, int ldN, int J, int P, int c0, int c1, int pairs_pad, int n_pairs, int mode,
                const double* __restrict__ A, const int2* __restrict__ pairs, const int* __restrict__ dcol,
                const double* __restrict__ W, const double* __restrict__ Dinv, double* __restrict__ Psi,
                double* __restrict__ Gacc, int group_m) {
  extern __shared__ __align__(16) double smem_d[];
  double* As = smem_d;              // [3][BK][SA]   pair products (pairs contiguous)
  double* Bs = As + 3 * BK * SA;    // [3][BN][SBT]  weights (cells contiguous)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3, wm = warp >> 2, wn = warp & 3;
  const int2 tile = grouped_tile(blockIdx.x, (n_pairs + BM - 1) / BM, (J + BN - 1) / BN, group_m);
  const int p0 = tile.x * BM, j0 = tile.y * BN;
  const int nsl = (c1 - c0 + BK - 1) / BK;

  // slice s: cells [c0 + 16 s, c0 + 16 s + 16) of both operands (16-byte copies; rows of A
  // past the range and weights past N arrive as zeros)
  auto load = [&](int s, int st) {
    const int kb = s * BK;
#pragma unroll
    for (int r = 0; r < (BM * BK / 2) / kThreads; r++) {
      const int ch = tid + r * kThreads;
      const int k = ch >> 6, part = ch & 63;
      const int row = kb + k;
      const int nb = (c0 + row < c1) ? 16 : 0;
      const double* src = A + (size_t)min(row, c1 - c0 - 1) * pairs_pad + p0 + part * 2;
      cp_async16(As + st * BK * SA + k * SA + part * 2, src, nb);
    }
#pragma unroll
    for (int r = 0; r < (BN * BK / 2) / kThreads; r++) {
      const int ch = tid + r * kThreads;
      const int n = ch >> 3, part = ch & 7;
      const int j = j0 + n, i = c0 + kb + part * 2;
      const int nb = (j < J) ? 8 * max(0, min(2, min(N, c1) - i)) : 0;
      const double* src = W + (size_t)min(j, J - 1) * ldN + min(i, ldN - 2);
      cp_async16(Bs + st * BN * SBT + n * SBT + part * 2, src, nb);
    }
  };

  double acc[4][4][4];
#pragma unroll
  for (int x = 0; x < 4; x++)
#pragma unroll
    for (int y = 0; y < 4; y++)
#pragma unroll
      for (int z = 0; z < 4; z++) acc[x][y][z] = 0.0;

  // three stages, one barrier per slice (as k_pair_v)
  load(0, 0);
  cp_async_commit();
  if (nsl > 1) load(1, 1);
  cp_async_commit();
  for (int s = 0; s < nsl; s++) {
    cp_async_wait<1>();  // slice s landed
    __syncthreads();
    if (s + 2 < nsl) load(s + 2, (s + 2) % 3);
    cp_async_commit();
    warp_slice<true>(As + (s % 3) * BK * SA, Bs + (s % 3) * BN * SBT, wm, wn, g, t, acc);
  }
  cp_async_wait<0>();

#pragma unroll
  for (int mt = 0; mt < 4; mt++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int p = p0 + wm * 64 + mt * 16 + g + h * 8;
      if (p >= n_pairs) continue;
      size_t mk = 0, ml = 0;
      double dv = 0.0;
      if (mode == kGramPsi) {
        const int2 q = pairs[p];
        mk = dcol[q.x];
        ml = dcol[q.y];
        dv = Dinv[mk + ml * P];
      }
#pragma unroll
      for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int j = j0 + wn * 32 + nt * 8 + 2 * t + e;
          if (j >= J) continue;
          const double v = acc[mt][nt][h * 2 + e];
          if (mode == kGramPsi) {
            double* Pj = Psi + (size_t)j * P * P;
            Pj[mk + ml * P] = v + dv;
            Pj[ml + mk * P] = v + dv;
          } else if (mode == kGramSet) {
            Gacc[(size_t)p * J + j] = v;
          } else {
            Gacc[(size_t)p * J + j] += v;
          }
        }
    }
}

// Psi_j[mk, ml] = Psi_j[ml, mk] = Gacc[p * J + j] + DeltaInv[mk, ml] after several ranges
__global__ void k_pair_scatter(int J, int P, int n_pairs, const int2* __restrict__ pairs,
                               const int* __restrict__ dcol, const double* __restrict__ Gacc,
                               const double* __restrict__ Dinv, double* __restrict__ Psi) {
  const int p = blockIdx.x;
  const int2 q = pairs[p];
  const size_t mk = dcol[q.x], ml = dcol[q.y];
  const double dv = Dinv[mk + ml * P];
  for (int j = threadIdx.x; j < J; j += blockDim.x) {
    const double v = Gacc[(size_t)p * J + j] + dv;
    double* Pj = Psi + (size_t)j * P * P;
    Pj[mk + ml * P] = v;
    Pj[ml + mk * P] = v;
  }
}

__global__ void k_recip_omega(int N, int cpad, const double* __restrict__ Omega, double* __restrict__ rOm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cpad) rOm[i] = i < N ? 1.0 / Omega[i] : 0.0;
}

// ---------------------------------------------------------------------------------------------
// Gradient contraction over the pairs
// ---------------------------------------------------------------------------------------------
// Spair[j][p] = S_j[dcol a_p, dcol b_p] (0 for the padding pairs)
__global__ void k_gather_spair(int J, int P, int n_pairs, int pairs_pad, const int2* __restrict__ pairs,
                               const int* __restrict__ dcol, const double* __restrict__ S,
                               double* __restrict__ Sp) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pairs_pad) return;
  int2 q = make_int2(0, 0);
  const bool live = p < n_pairs;
  if (live) q = pairs[p];
  const size_t off = live ? (size_t)dcol[q.x] + (size_t)dcol[q.y] * P : 0;
  for (int j = blockIdx.y; j < J; j += gridDim.y)
    Sp[(size_t)j * pairs_pad + p] = live ? S[(size_t)j * P * P + off] : 0.0;
}

__global__ void __launch_bounds__(kThreads, 1)
    k_pair_v(int N, int ldN, int J, int c0, int c1, int pairs_pad, const double* __restrict__ W,
             const double* __restrict__ Sp, const double* __restrict__ rOm, double* __restrict__ V, int group_m) {
  extern __shared__ __align__(16) double smem_d[];
  double* As = smem_d;                // [3][BK][SA]  W rows (cells contiguous)
  double* Bs = smem_d + 3 * BK * SA;  // [3][BK][SBN] S pairs (pairs contiguous)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3, wm = warp >> 2, wn = warp & 3;
  const int2 tile = grouped_tile(blockIdx.x, (c1 - c0 + BM - 1) / BM, pairs_pad / BN, group_m);
  const int i0 = c0 + tile.x * BM, n0 = tile.y * BN;
  const int nsl = (J + BK - 1) / BK;

  auto load = [&](int s, int buf) {
    const int jb = s * BK;
#pragma unroll
    for (int r = 0; r < (BM * BK / 2) / kThreads; r++) {
      const int ch = tid + r * kThreads;
      const int k = ch >> 6, part = ch & 63;
      const int j = jb + k, i = i0 + part * 2;
      const int nb = (j < J) ? 8 * max(0, min(2, min(N, c1) - i)) : 0;
      const double* src = W + (size_t)min(j, J - 1) * ldN + min(max(i, 0), ldN - 2);
      cp_async16(As + buf * BK * SA + k * SA + part * 2, src, nb);
    }
#pragma unroll
    for (int r = 0; r < (BN * BK / 2) / kThreads; r++) {
      const int ch = tid + r * kThreads;
      const int k = ch >> 6, part = ch & 63;
      const int j = jb + k;
      const int nb = (j < J) ? 16 : 0;
      const double* src = Sp + (size_t)min(j, J - 1) * pairs_pad + n0 + part * 2;
      cp_async16(Bs + buf * BK * SBN + k * SBN + part * 2, src, nb);
    }
  };

  double acc[4][4][4];
#pragma unroll
  for (int x = 0; x < 4; x++)
#pragma unroll
    for (int y = 0; y < 4; y++)
#pragma unroll
      for (int z = 0; z < 4; z++) acc[x][y][z] = 0.0;

  // three stages, one barrier per slice: after the barrier of iteration s every warp is done
  // with slice s - 1, whose stage (s + 2) % 3 is refilled while slice s is multiplied
  load(0, 0);
  cp_async_commit();
  if (nsl > 1) load(1, 1);
  cp_async_commit();
  for (int s = 0; s < nsl; s++) {
    cp_async_wait<1>();  // slice s landed
    __syncthreads();
    if (s + 2 < nsl) load(s + 2, (s + 2) % 3);
    cp_async_commit();
    warp_slice<false>(As + (s % 3) * BK * SA, Bs + (s % 3) * BK * SBN, wm, wn, g, t, acc);
  }
  cp_async_wait<0>();

#pragma unroll
  for (int mt = 0; mt < 4; mt++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int i = i0 + wm * 64 + mt * 16 + g + h * 8;
      if (i >= N || i >= c1) continue;
      const double r = rOm[i];
      double* vrow = V + (size_t)(i - c0) * pairs_pad + n0 + wn * 32 + 2 * t;
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        double2 v = make_double2(acc[mt][nt][h * 2] * r, acc[mt][nt][h * 2 + 1] * r);
        *reinterpret_cast<double2*>(vrow + nt * 8) = v;
      }
    }
}

// U[i, a] = sum_b D_ib V[i, pair(min(a,b), max(a,b))], one CTA per cell, the V row staged in
// shared memory; pair(a, b) = a*n_d - a*(a-1)/2 + (b - a) (row-major upper triangle).
__global__ void __launch_bounds__(256) k_v_to_u(int N, int ldN, int n_d, int n_pairs, int pairs_pad, int c0,
                                                int c1, const double* __restrict__ D,
                                                const double* __restrict__ V, double* __restrict__ U) {
  extern __shared__ __align__(16) double vs[];
  double* ds = vs + pairs_pad;  // D row of the cell
  for (int i = c0 + blockIdx.x; i < c1 && i < N; i += gridDim.x) {
    const double* vr = V + (size_t)(i - c0) * pairs_pad;
    for (int e = threadIdx.x; e < n_pairs; e += blockDim.x) vs[e] = vr[e];
    for (int e = threadIdx.x; e < n_d; e += blockDim.x) ds[e] = D[(size_t)e * ldN + i];
    __syncthreads();
    for (int a = threadIdx.x; a < n_d; a += blockDim.x) {
      double s = 0.0;
      // b < a: pair(b, a)
      for (int b = 0; b < a; b++) s = fma(ds[b], vs[b * n_d - b * (b - 1) / 2 + (a - b)], s);
      // b >= a: pair(a, b), contiguous
      const double* row = vs + a * n_d - a * (a - 1) / 2 - a;
      for (int b = a; b < n_d; b++) s = fma(ds[b], row[b], s);
      U[i + (size_t)a * ldN] = s;
    }
    __syncthreads();
  }
}

// The same sums when a cell's V row exceeds the shared-memory budget (more than about 220 dense
// columns): the row is read from global memory (L1 / L2) instead of staged, the dense row of
// the cell is staged; identical operations in identical order.
__global__ void __launch_bounds__(256) k_v_to_u_wide(int N, int ldN, int n_d, int pairs_pad, int c0, int c1,
                                                     const double* __restrict__ D, const double* __restrict__ V,
                                                     double* __restrict__ U) {
  extern __shared__ __align__(16) double ds[];  // D row of the cell
  for (int i = c0 + blockIdx.x; i < c1 && i < N; i += gridDim.x) {
    const double* vr = V + (size_t)(i - c0) * pairs_pad;
    for (int e = threadIdx.x; e < n_d; e += blockDim.x) ds[e] = D[(size_t)e * ldN + i];
    __syncthreads();
    for (int a = threadIdx.x; a < n_d; a += blockDim.x) {
      double s = 0.0;
      for (int b = 0; b < a; b++) s = fma(ds[b], __ldg(vr + b * n_d - b * (b - 1) / 2 + (a - b)), s);
      const double* row = vr + a * n_d - a * (a - 1) / 2 - a;
      for (int b = a; b < n_d; b++) s = fma(ds[b], __ldg(row + b), s);
      U[i + (size_t)a * ldN] = s;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
int pair_prepare(Ctx* c) {
  PairState& s = c->pr;
  if (s.ready) return GPL_OK;
  const int n_d = c->n_d;
  std::vector<int2> pairs;
  for (int a = 0; a < n_d; a++)
    for (int b = a; b < n_d; b++) pairs.push_back(make_int2(a, b));
  s.n_pairs = (int)pairs.size();
  s.pairs_pad = (s.n_pairs + BN - 1) / BN * BN;
  s.cpad = (c->N + BM - 1) / BM * BM;
  // V (the gradient's V rows, or the Gram's pair products) holds a range of cells at a time:
  // all cells when that fits in 8 GiB (one range: the Gram writes Psi directly), else ranges
  // of at most 8 GiB. The option pair_range_cells sets a smaller range (tests of the multi-range path).
  const size_t row = (size_t)s.pairs_pad * sizeof(double);
  size_t cap = std::max<size_t>(BM, ((size_t)8 << 30) / row / BM * BM);
  if (c->pair_range_cells >= BM) cap = std::min<size_t>(cap, (size_t)c->pair_range_cells / BM * BM);
  s.v_cells = (int)std::min<size_t>((size_t)s.cpad, cap);
  s.smem_gram = (int)sizeof(double) * 3 * (BK * SA + BN * SBT);
  s.smem_v = (int)sizeof(double) * 3 * (BK * SA + BK * SBN);
  s.smem_vu = (int)sizeof(double) * (s.pairs_pad + n_d);
  // more dense columns than k_v_to_u stages per cell: k_v_to_u_wide reads the V rows from
  // global memory instead
  s.wide = s.smem_vu > 200 * 1024;
  if (cudaMalloc((void**)&s.pairs, sizeof(int2) * pairs.size()) != cudaSuccess ||
      cudaMalloc((void**)&s.rOm, sizeof(double) * s.cpad) != cudaSuccess ||
      cudaMalloc((void**)&s.Sp, sizeof(double) * (size_t)c->J * s.pairs_pad) != cudaSuccess ||
      cudaMalloc((void**)&s.V, sizeof(double) * (size_t)s.v_cells * s.pairs_pad) != cudaSuccess) {
    cudaGetLastError();
    pair_release(c);
    c->err = "device allocation failed: pair GEMM buffers";
    return GPL_ERR_ALLOC;
  }
  GPL_TRY(c, cudaMemcpy(s.pairs, pairs.data(), sizeof(int2) * pairs.size(), cudaMemcpyHostToDevice));
  if (s.v_cells < c->N &&
      cudaMalloc((void**)&s.Gacc, sizeof(double) * (size_t)s.n_pairs * c->J) != cudaSuccess) {
    cudaGetLastError();
    pair_release(c);
    c->err = "device allocation failed: pair Gram accumulator";
    return GPL_ERR_ALLOC;
  }
  GPL_TRY(c, cudaFuncSetAttribute(k_pair_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, s.smem_gram));
  GPL_TRY(c, cudaFuncSetAttribute(k_pair_v, cudaFuncAttributeMaxDynamicSharedMemorySize, s.smem_v));
  if (!s.wide) GPL_TRY(c, cudaFuncSetAttribute(k_v_to_u, cudaFuncAttributeMaxDynamicSharedMemorySize, s.smem_vu));
  s.ready = true;
  return GPL_OK;
}

void pair_release(Ctx* c) {
  graph_reset(c);
  PairState& s = c->pr;
  void* bufs[] = {s.pairs, s.rOm, s.Sp, s.V, s.Gacc};
  for (void* p : bufs)
    if (p) cudaFree(p);
  s = PairState();
}

int recip_omega(Ctx* c, const double** rOm) {
  int rc = pair_prepare(c);
  if (rc) return rc;
  PairState& s = c->pr;
  k_recip_omega<<<div_up(s.cpad, 256), 256, 0, c->stream>>>(c->N, s.cpad, c->Omega, s.rOm);
  GPL_LAUNCHED(c, "k_recip_omega");
  *rOm = s.rOm;
  return GPL_OK;
}

static int launch_recip(Ctx* c) {
  PairState& s = c->pr;
  k_recip_omega<<<div_up(s.cpad, 256), 256, 0, c->stream>>>(c->N, s.cpad, c->Omega, s.rOm);
  GPL_LAUNCHED(c, "k_recip_omega");
  return GPL_OK;
}

int launch_pair_gram(Ctx* c) {
  int rc = pair_prepare(c);
  if (rc) return rc;
  PairState& s = c->pr;
  if ((rc = launch_recip(c))) return rc;
  ProfScope ps(c, "gram");
  const bool one = s.v_cells >= c->N;
  for (int c0 = 0; c0 < c->N; c0 += s.v_cells) {
    const int c1 = std::min(c->N, c0 + s.v_cells);
    const int smem_p = (int)sizeof(double) * (c->n_d + 1) * kProdCells;
    k_pair_products<<<div_up(c1 - c0, kProdCells), 256, smem_p, c->stream>>>(
        c->ldN, c->n_d, c0, c1, s.n_pairs, s.pairs_pad, s.pairs, c->Dm, s.rOm, s.V);
    GPL_LAUNCHED(c, "k_pair_products");
    const int mode = one ? kGramPsi : (c0 == 0 ? kGramSet : kGramAdd);
    const int g = div_up(s.n_pairs, BM) * div_up(c->J, BN);
    Tunable* tu = nullptr;
    const int gm = tune_pick(c, "pair_gram", {8, 12, 16}, kGroupM, &tu);
    TuneScope ts(c, one ? tu : nullptr);
    k_pair_gram<<<g, kThreads, s.smem_gram, c->stream>>>(c->N, c->ldN, c->J, c->P, c0, c1, s.pairs_pad, s.n_pairs,
                                                        mode, s.V, s.pairs, c->dcol_d, c->W, c->DeltaInv, c->Psi,
                                                        s.Gacc, gm);
    GPL_LAUNCHED(c, "k_pair_gram");
  }
  if (!one) {
    k_pair_scatter<<<s.n_pairs, 256, 0, c->stream>>>(c->J, c->P, s.n_pairs, s.pairs, c->dcol_d, s.Gacc,
                                                    c->DeltaInv, c->Psi);
    GPL_LAUNCHED(c, "k_pair_scatter");
  }
  return GPL_OK;
}

int launch_pair_uq(Ctx* c) {
  int rc = pair_prepare(c);
  if (rc) return rc;
  PairState& s = c->pr;
  if ((rc = launch_recip(c))) return rc;
  {
    ProfScope ps(c, "spair");
    dim3 g(div_up(s.pairs_pad, 256), std::min(c->J, 65535));
    k_gather_spair<<<g, 256, 0, c->stream>>>(c->J, c->P, s.n_pairs, s.pairs_pad, s.pairs, c->dcol_d, c->PsiInv,
                                             s.Sp);
    GPL_LAUNCHED(c, "k_gather_spair");
  }
  for (int c0 = 0; c0 < c->N; c0 += s.v_cells) {
    const int c1 = std::min(c->N, c0 + s.v_cells);
    {
      ProfScope ps(c, "uq");
      const int g = div_up(c1 - c0, BM) * (s.pairs_pad / BN);
      Tunable* tu = nullptr;
      const int gm = tune_pick(c, "pair_v", {8, 12, 16}, kGroupM, &tu);
      TuneScope ts(c, c1 - c0 == c->N ? tu : nullptr);
      k_pair_v<<<g, kThreads, s.smem_v, c->stream>>>(c->N, c->ldN, c->J, c0, c1, s.pairs_pad, c->W, s.Sp, s.rOm,
                                                     s.V, gm);
      GPL_LAUNCHED(c, "k_pair_v");
    }
    if ((rc = launch_v_to_u_cells(c, c0, c1, c->Dm))) return rc;
  }
  return GPL_OK;
}

int launch_v_to_u_cells(Ctx* c, int c0, int c1, const double* D) {
  PairState& s = c->pr;
  ProfScope ps(c, "v_to_u");
  const int grid = std::min(c1 - c0, 148 * 8);
  if (s.wide) {
    k_v_to_u_wide<<<grid, 256, sizeof(double) * c->n_d, c->stream>>>(c->N, c->ldN, c->n_d, s.pairs_pad, c0, c1, D,
                                                                    s.V, c->U);
    GPL_LAUNCHED(c, "k_v_to_u_wide");
    return GPL_OK;
  }
  k_v_to_u<<<grid, 256, s.smem_vu, c->stream>>>(c->N, c->ldN, c->n_d, s.n_pairs, s.pairs_pad, c0, c1, D, s.V, c->U);
  GPL_LAUNCHED(c, "k_v_to_u");
  return GPL_OK;
}

// ---------------------------------------------------------------------------------------------
// Linear predictor over the dense columns (option eta_tc)
// ---------------------------------------------------------------------------------------------
// out[j * ldN + i] = D_i . B_j[dcol] + Lv[group(i), j] for 128-cell x 128-gene tiles, where
// Lv[g, j] is the sum of gene j's coefficients of the levels of cell group g (k_level_sums, per
// launch; genes contiguous in rows of ldJ, even, so that a lane reads its two genes' sums as one
// 16-byte load and the eight cells of a quad row touch at most eight lines): K = the dense columns in 16-deep slices (DMMA steps past n_d skipped), A = D by
// 16-byte cp.async (cells contiguous), B = the genes' dense coefficients gathered through dcol by
// 8-byte cp.async (k contiguous in shared memory). Persistent: one CTA per SM walks the tiles
// cell-tile-major with a stride of the grid, so the CTAs resident at any time share a few cell
// tiles of D and all of B through L2; the next tile's first two slices are in flight while the
// current tile's epilogue stores (evict-first) run. The weights that follow (W, Nu) are an
// element-wise pass of their own: inside this kernel's epilogue, at one CTA per SM, the
// dependent FP64 operations of exp() left the tensor pipe idle for most of the launch.
struct EtaArgs {
  int N, ldN, P, J, ldJ, n_d, n_grp;
  const double *D, *B, *lvt;
  const int *dcol, *gid;
  double* out;
};

// Lv[g * ldJ + j] = sum over the grouped variables v (in order) of B[cv_nh[v] + level + j * P]
__global__ void k_level_sums(int J, int ldJ, int n_grp, int n_cv, int P, const int* __restrict__ cv_nh,
                             const int* __restrict__ glev, const double* __restrict__ B, double* __restrict__ Lv) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)J * n_grp) return;
  const int g = (int)(e / J), j = (int)(e - (int64_t)g * J);
  double s = 0.0;
  for (int v = 0; v < n_cv; v++) s += B[cv_nh[v] + glev[(size_t)g * n_cv + v] + (size_t)j * P];
  Lv[(size_t)g * ldJ + j] = s;
}

// One 16-deep K slice of a warp tile of MT x 16 cells x 32 genes (A rows of stride sa), with only
// the first nkk of its four k4 steps live when kLive.
template <int MT, bool kLive>
__device__ __forceinline__ void warp_slice_eta(const double* __restrict__ As, const double* __restrict__ Bs, int sa,
                                               int wm, int wn, int g, int t, int nkk, double (&acc)[MT][4][4]) {
#pragma unroll
  for (int kk = 0; kk < BK / 4; kk++) {
    if (kLive && kk >= nkk) break;
    double av[MT][2], b[4];
    const double* ar = As + (kk * 4 + t) * sa + wm * (MT * 16) + g;
#pragma unroll
    for (int mt = 0; mt < MT; mt++) {
      av[mt][0] = ar[mt * 16];
      av[mt][1] = ar[mt * 16 + 8];
    }
#pragma unroll
    for (int nt = 0; nt < 4; nt++) b[nt] = Bs[(wn * 32 + nt * 8 + g) * SBT + kk * 4 + t];
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
      for (int nt = 0; nt < 4; nt++) dmma_16x8x4(acc[mt][nt], av[mt][0], av[mt][1], b[nt]);
  }
}

// Tiles of MT x 32 cells x 128 genes: MT = 4 (128 cells, one CTA per SM) or MT = 2 (64 cells, two
// CTAs per SM, so that one CTA's epilogue overlaps the other's MMAs). Every output is the same
// sum in the same order in both, so the autotuner may pick either.
template <int MT>
size_t eta_smem_bytes(int n_d) {
  const int KP = (n_d + BK - 1) / BK * BK;
  return sizeof(double) * (3 * BK * (MT * 32 + 4) + 3 * BN * SBT) + sizeof(int) * (size_t)KP;
}

template <int MT>
__global__ void __launch_bounds__(kThreads, MT == 2 ? 2 : 1) k_eta_dmma(const EtaArgs a) {
  constexpr int BMt = MT * 32, SAt = BMt + 4;
  extern __shared__ __align__(16) double smem_d[];
  double* As = smem_d;             // [3][BK][SAt] D rows (cells contiguous)
  double* Bs = As + 3 * BK * SAt;  // [3][BN][SBT] dense coefficients (k contiguous)
  const int KP = (a.n_d + BK - 1) / BK * BK;
  int* dcs = reinterpret_cast<int*>(Bs + 3 * BN * SBT);  // [KP] dcol, 0 past n_d
  const double* __restrict__ D = a.D;
  const double* __restrict__ B = a.B;
  const double* __restrict__ lvt = a.lvt;
  const int* __restrict__ gid = a.gid;
  double* __restrict__ out = a.out;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3, wm = warp >> 2, wn = warp & 3;
  const int tm = (a.N + BMt - 1) / BMt, tn = (a.J + BN - 1) / BN;
  const int tiles = tm * tn, nsl = KP / BK;
  for (int k = tid; k < KP; k += kThreads) dcs[k] = k < a.n_d ? a.dcol[k] : 0;
  __syncthreads();

  // slice s of the tile at (m0, j0) into stage st
  auto load = [&](int m0, int j0, int s, int st) {
    const int kb = s * BK;
#pragma unroll
    for (int r = 0; r < (BMt * BK / 2) / kThreads; r++) {
      const int ch = tid + r * kThreads;
      const int k = ch / (BMt / 2), part = ch % (BMt / 2);
      const int col = kb + k, i = m0 + part * 2;
      const int nb = (col < a.n_d && i < a.ldN) ? 16 : 0;  // ldN is even: a chunk is in or out whole
      const double* src = D + (size_t)min(col, a.n_d - 1) * a.ldN + min(i, a.ldN - 2);
      cp_async16(As + st * BK * SAt + k * SAt + part * 2, src, nb);
    }
#pragma unroll
    for (int r = 0; r < (BN * BK) / kThreads; r++) {
      const int ch = tid + r * kThreads;
      const int n = ch >> 4, k = ch & 15;
      const int col = kb + k, j = j0 + n;
      const int nb = (col < a.n_d && j < a.J) ? 8 : 0;
      const double* src = B + dcs[col] + (size_t)min(j, a.J - 1) * a.P;
      cp_async8(Bs + st * BN * SBT + n * SBT + k, src, nb);
    }
  };

  int base = 0;  // slices issued before this tile (stage of slice s = (base + s) % 3)
  int w = blockIdx.x;
  if (w < tiles) {
    const int m0 = (w / tn) * BMt, j0 = (w % tn) * BN;
    load(m0, j0, 0, 0);
    cp_async_commit();
    if (nsl > 1) load(m0, j0, 1, 1);
    cp_async_commit();
  }
  for (; w < tiles; w += gridDim.x) {
    const int m0 = (w / tn) * BMt, j0 = (w % tn) * BN;
    double acc[MT][4][4];
#pragma unroll
    for (int x = 0; x < MT; x++)
#pragma unroll
      for (int y = 0; y < 4; y++)
#pragma unroll
        for (int z = 0; z < 4; z++) acc[x][y][z] = 0.0;
    for (int s = 0; s < nsl; s++) {
      cp_async_wait<1>();  // slice s landed
      __syncthreads();
      if (s + 2 < nsl) load(m0, j0, s + 2, (base + s + 2) % 3);
      cp_async_commit();
      const int st = (base + s) % 3;
      if (s + 1 < nsl) {
        warp_slice_eta<MT, false>(As + st * BK * SAt, Bs + st * BN * SBT, SAt, wm, wn, g, t, 4, acc);
      } else {  // the last slice: only the k4 steps that reach a dense column
        const int nkk = min(BK / 4, (a.n_d - s * BK + 3) / 4);
        warp_slice_eta<MT, true>(As + st * BK * SAt, Bs + st * BN * SBT, SAt, wm, wn, g, t, nkk, acc);
      }
    }
    // the next tile's first two slices go to the two stages that no warp reads any more
    base += nsl;
    const int wn2 = w + gridDim.x;
    if (wn2 < tiles) {
      const int m1 = (wn2 / tn) * BMt, j1 = (wn2 % tn) * BN;
      load(m1, j1, 0, base % 3);
      cp_async_commit();
      if (nsl > 1) load(m1, j1, 1, (base + 1) % 3);
      cp_async_commit();
    }
    // the cells' level sums, then the stores
    if (a.n_grp > 0) {
#pragma unroll
      for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int i = min(m0 + wm * (MT * 16) + mt * 16 + g + h * 8, a.N - 1);
          const double* lg = lvt + (size_t)gid[i] * a.ldJ;
#pragma unroll
          for (int nt = 0; nt < 4; nt++) {
            // genes j, j + 1 (j even); past J only columns that are never stored
            const int j = min(j0 + wn * 32 + nt * 8 + 2 * t, a.ldJ - 2);
            const double2 v = *reinterpret_cast<const double2*>(lg + j);
            acc[mt][nt][h * 2] += v.x;
            acc[mt][nt][h * 2 + 1] += v.y;
          }
        }
    }
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int i = m0 + wm * (MT * 16) + mt * 16 + g + h * 8;
        if (i >= a.N) continue;
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int j = j0 + wn * 32 + nt * 8 + 2 * t + e;
            if (j < a.J) __stcs(out + (size_t)j * a.ldN + i, acc[mt][nt][h * 2 + e]);
          }
      }
  }
  cp_async_wait<0>();
}

int launch_eta_dmma(Ctx* c, const double* B, double* out) {
  if (eta_smem_bytes<4>(c->n_d) > 227 * 1024) {
    c->err = "too many dense columns for the linear-predictor kernel";
    return GPL_ERR_LIMIT;
  }
  if (c->n_grp > 0) {
    const int64_t n = (int64_t)c->J * c->n_grp;
    k_level_sums<<<(unsigned)div_up(n, 256), 256, 0, c->stream>>>(c->J, lvt_ld(c->J), c->n_grp, c->n_cv, c->P,
                                                                 c->cv_nh_d, c->glev_d, B, c->lvt);
    GPL_LAUNCHED(c, "k_level_sums");
  }
  EtaArgs a{};
  a.N = c->N;
  a.ldN = c->ldN;
  a.P = c->P;
  a.J = c->J;
  a.ldJ = lvt_ld(c->J);
  a.n_d = c->n_d;
  a.n_grp = c->n_grp;
  a.D = c->Dm;
  a.B = B;
  a.lvt = c->lvt;
  a.dcol = c->dcol_d;
  a.gid = c->gid_d;
  a.out = out;
  // tile height: 128 cells (one CTA per SM) or 64 (two), the autotuner's choice (same sums)
  Tunable* tu = nullptr;
  const int cells = tune_pick(c, "eta_tile", {128, 64}, 128, &tu);
  TuneScope ts(c, tu);
  if (cells == 64) {
    const size_t smem = eta_smem_bytes<2>(c->n_d);
    GPL_TRY(c, cudaFuncSetAttribute(k_eta_dmma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int tiles = div_up(c->N, 64) * div_up(c->J, BN);
    k_eta_dmma<2><<<std::min(tiles, 2 * c->sm_count), kThreads, smem, c->stream>>>(a);
  } else {
    const size_t smem = eta_smem_bytes<4>(c->n_d);
    GPL_TRY(c, cudaFuncSetAttribute(k_eta_dmma<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int tiles = div_up(c->N, 128) * div_up(c->J, BN);
    k_eta_dmma<4><<<std::min(tiles, c->sm_count), kThreads, smem, c->stream>>>(a);
  }
  GPL_LAUNCHED(c, "k_eta_dmma");
  return GPL_OK;
}

}  // namespace gpl
