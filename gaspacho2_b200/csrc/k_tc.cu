// Tensor-core (tcgen05) forms of the two dominant contractions (the precision form,
// GPL_PREC_BF16X3): BF16 hi/lo split products, FP32 MMA accumulation in TMEM, and FP64
// accumulation of short FP32 runs, also in TMEM.
//
// Precision. x ~= hi + lo (hi = bf16(x), lo = bf16(x - hi)) keeps 16 significant bits per
// operand; each product is hi*hi + hi*lo + lo*hi (three MMAs), the dropped lo*lo term is below
// 2^-16 relative. The tensor core adds every MMA result into its FP32 accumulator with a small
// downward bias (measured on B200: about 2^-25 relative per accumulating instruction), which
// over a 100K-cell reduction would reach 3e-5. So an FP32 accumulator only ever collects a few
// 64-wide K chunks; drain warps then add it into an FP64 running sum kept in TMEM (two 32-bit
// columns per value) and the MMAs continue in the other FP32 buffer. The bias is then that of
// a few chunks (~1e-6) and the long reduction is FP64.
//
// k_tc_gram   C[p, n] = sum_k A[p, k] B[n, k] for 128 column pairs p and 128 columns n per CTA,
//             A and B both BF16 hi/lo, K-major, 128-byte swizzled, by TMA (64-wide K chunks,
//             three stages). TMEM: two FP32 128 x 128 accumulators (columns 0-255) and the FP64
//             sum (columns 256-511). Two uses:
//             * the Gram: A = products of the whitened dense columns per pair, B = w = W/Omega
//               per gene, K = cells; the FP64 tile goes to the whitened Gram of every gene
//               (un-whitened in FP64 afterwards) or straight into Psi_j;
//             * the gradient pairs: A = S~_j[pair] (the whitened inverse, per gene), B = O^T
//               (W/Omega per cell), K = genes; the FP64 tile goes to V[cell][pair].
//             Work per use: N*J*n_d*(n_d+1) useful flops (3x on the tensor pipe).
//
// Whitening. The reference adds no jitter to Kmm, so cond(Psi_j) reaches ~1e14 and a 1e-6
// relative Gram error fails the Cholesky. The dense columns are therefore first mapped to
// L^{-1} d_i with DeltaInv_DD = L L^T (k_whiten_rows): the Gram of those, G~, enters Psi as
// L G~ L^T + DeltaInv, so its errors are relative to a matrix bounded below by the identity.
// The gradient contraction runs on the same coordinates: U_i = S_DD d_i = L^{-T} S~ d~_i with
// S~ = L^T S_DD L (k_unwhiten_u maps U~ back).
//
// Warp roles (192 threads): warp 0 allocates TMEM and issues the TMA loads, warp 1 issues the
// MMAs (one thread), warps 2-5 drain the accumulators and write the results (warp w reads TMEM
// lanes 32*(w % 4) .. +31). Full barriers count the TMA bytes; empty barriers and the
// accumulator barriers are armed by tcgen05.commit; drained barriers count the 128 drain
// threads. Every wait is bounded: one that runs out records an error code, and every role
// drains what it started before TMEM is freed.
#include <cuda.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "gpl_internal.cuh"
#include "tc_common.cuh"

namespace gpl {

using namespace tc;

namespace {
constexpr int kThreadsGram = 192;       // TMA, MMA and 4 drain warps
constexpr int kStagesGram = 3;          // pipeline depth (192 KB of operand tiles)
constexpr int kMaxStages = 4;          // barriers held (the CTA-pair kernel's stages)
constexpr int kGramN = 128;             // genes per Gram tile
constexpr int kSBGram = 4;              // chunks per FP32 run (default; the option tc_run overrides)
constexpr int kTileA = 128 * 128;       // 128 rows x 64 BF16
constexpr int kTileBG = kGramN * 128;   // 128 gene rows x 64 BF16
constexpr int kMaxWhiten = 160;         // dense columns the whitened rows kernel holds per cell
constexpr uint32_t kIdescGram = idesc_bf16_f32(128, kGramN);
}  // namespace

struct TcShared {
  uint64_t full[kMaxStages];
  uint64_t empty[kMaxStages];
  uint64_t accb[2];
  uint64_t drained[2];
  uint64_t fin;
  uint32_t tmem;
  int abort;
};

__device__ __forceinline__ void tc_fail(int* err, TcShared* sh, int code) {
  atomicExch(&sh->abort, 1);
  atomicCAS(err, 0, code);
}

__device__ __forceinline__ void tc_init(TcShared* sh, const int* err, int full_count) {
  for (int s = 0; s < kMaxStages; s++) {
    mbar_init(&sh->full[s], full_count);
    mbar_init(&sh->empty[s], 1);
  }
  for (int b = 0; b < 2; b++) {
    mbar_init(&sh->accb[b], 1);
    mbar_init(&sh->drained[b], 128);
  }
  mbar_init(&sh->fin, 1);
  sh->abort = *(const volatile int*)err != 0;
  fence_barrier_init();
}

// True in every lane when `v` holds in every lane of the warp: the warp-wide TMEM loads and
// stores after it then run converged.
__device__ __forceinline__ bool warp_all(bool v) { return __all_sync(0xffffffffu, v); }

__device__ __forceinline__ bool aborted(const TcShared* sh) { return *(const volatile int*)&sh->abort != 0; }

// The MMA thread's last act: wait (bounded) until every MMA it issued has completed, so that
// TMEM is never freed under a running MMA, also on the error path.
__device__ __forceinline__ void mma_finish(TcShared* sh, int* err, int code) {
  mma_commit(&sh->fin);
  if (!mbar_wait(&sh->fin, 0, nullptr)) atomicCAS(err, 0, code);
}

// Adds the FP32 accumulator columns [src, src + ncol) of this thread's lane into the FP64 sum
// at columns [dst, dst + 2*ncol) (first: overwrite). ncol is a multiple of 32.
__device__ __forceinline__ void drain_f32_to_f64(uint32_t lane_addr, uint32_t src, uint32_t dst, int ncol,
                                                 bool first) {
  for (int cb = 0; cb < ncol; cb += 32) {
    float f[32];
    tmem_ld32(lane_addr + src + cb, f);
#pragma unroll
    for (int h = 0; h < 2; h++) {
      double d[16];
      const uint32_t fa = lane_addr + dst + 2 * (cb + 16 * h);
      if (first) {
#pragma unroll
        for (int k = 0; k < 16; k++) d[k] = (double)f[16 * h + k];
      } else {
        tmem_ld_f64x16(fa, d);
#pragma unroll
        for (int k = 0; k < 16; k++) d[k] += (double)f[16 * h + k];
      }
      tmem_st_f64x16(fa, d);
    }
  }
  tmem_wait_st();
}

// ---------------------------------------------------------------------------------------------
// Gram
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreadsGram, 1)
    k_tc_gram(const __grid_constant__ CUtensorMap map_ahi, const __grid_constant__ CUtensorMap map_alo,
              const __grid_constant__ CUtensorMap map_whi, const __grid_constant__ CUtensorMap map_wlo,
              const int2* __restrict__ pairs, int n_pairs,
              int chunks_total, const int* __restrict__ dcol, int P, int J, const double* __restrict__ Dinv,
              double* __restrict__ Psi, double* __restrict__ Gt, int n_d, int n_base, double* __restrict__ V,
              int v_ld, int run, int* __restrict__ err, int group) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* A_hi = base;
  unsigned char* A_lo = A_hi + kStagesGram * kTileA;
  unsigned char* B_hi = A_lo + kStagesGram * kTileA;
  unsigned char* B_lo = B_hi + kStagesGram * kTileBG;
  TcShared* sh = (TcShared*)(B_lo + kStagesGram * kTileBG);
  int2* spairs = (int2*)(sh + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // tile order: group == 0 takes the launch order (pair tile fastest: the ~148 resident CTAs share
  // one or two column tiles and every pair tile); group > 0 walks `group` pair tiles down each
  // column tile before the next, so that the resident CTAs share both operands' tiles through L2.
  // Either order computes every tile with the same sums.
  int ptile = blockIdx.x, ntile = blockIdx.y;
  if (group > 0) {
    const int id = blockIdx.y * gridDim.x + blockIdx.x, tm = gridDim.x;
    const int per = group * gridDim.y, grp = id / per, first = grp * group;
    const int gm = min(tm - first, group), r = id - grp * per;
    ptile = first + r % gm;
    ntile = r / gm;
  }
  const int n0 = ntile * kGramN;
  const int nch = chunks_total;
  const int nsb = (nch + run - 1) / run;

  if (threadIdx.x == 0) tc_init(sh, err, 1);
  __syncthreads();
  if (sh->abort) return;
  for (int r = threadIdx.x; r < 128; r += kThreadsGram) {
    const int p = ptile * 128 + r;
    spairs[r] = p < n_pairs ? pairs[p] : make_int2(-1, -1);
  }
  if (warp == 0) {
    tmem_alloc(&sh->tmem, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem;

  if (warp == 0) {
    if (lane == 0) {  // TMA: pair products (128 pairs) and weights (128 genes) of 64 cells per stage
      int issued = 0;
      for (int it = 0; it < nch; it++) {
        const int s = it % kStagesGram;
        if (it >= kStagesGram && !mbar_wait(&sh->empty[s], ((it / kStagesGram) - 1) & 1, err)) { tc_fail(err, sh, 11); break; }
        if (sh->abort) break;
        mbar_arrive_expect_tx(&sh->full[s], 2u * kTileA + 2u * kTileBG);
        const int x = it * 64;
        tma_load_2d(A_hi + s * kTileA, &map_ahi, &sh->full[s], x, ptile * 128);
        tma_load_2d(A_lo + s * kTileA, &map_alo, &sh->full[s], x, ptile * 128);
        tma_load_2d(B_hi + s * kTileBG, &map_whi, &sh->full[s], x, n_base + n0);
        tma_load_2d(B_lo + s * kTileBG, &map_wlo, &sh->full[s], x, n_base + n0);
        issued = it + 1;
      }
      for (int it = max(0, issued - kStagesGram); it < issued; it++)
        if (!mbar_wait(&sh->full[it % kStagesGram], (it / kStagesGram) & 1, nullptr)) atomicCAS(err, 0, 12);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      for (int it = 0; it < nch; it++) {
        const int s = it % kStagesGram, sb = it / run, pos = it % run, buf = sb & 1;
        if (pos == 0 && sb >= 2 && !mbar_wait(&sh->drained[buf], ((sb >> 1) - 1) & 1, err)) {
          tc_fail(err, sh, 16);
          break;
        }
        if (!mbar_wait(&sh->full[s], (it / kStagesGram) & 1, err)) { tc_fail(err, sh, 13); break; }
        if (sh->abort) break;
        tc_fence_after();
        const uint32_t acc = tmem + buf * kGramN;
        const uint32_t ah = smem_u32(A_hi + s * kTileA), al = smem_u32(A_lo + s * kTileA);
        const uint32_t bh = smem_u32(B_hi + s * kTileBG), bl = smem_u32(B_lo + s * kTileBG);
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint32_t off = k * 32;
          mma_bf16(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bh + off), kIdescGram, (pos | k) ? 1u : 0u);
          mma_bf16(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bl + off), kIdescGram, 1u);
          mma_bf16(acc, umma_desc_sw128(al + off), umma_desc_sw128(bh + off), kIdescGram, 1u);
        }
        mma_commit(&sh->empty[s]);
        if (pos == run - 1 || it == nch - 1) mma_commit(&sh->accb[buf]);
      }
      mma_finish(sh, err, 17);
    }
  } else {
    // drain warps: FP32 runs -> FP64 sum, then the results into Psi
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const uint32_t lane_addr = tmem + ((uint32_t)(q * 32) << 16);
    bool ok = true;
    for (int sb = 0; sb < nsb; sb++) {
      const int buf = sb & 1;
      const bool w = mbar_wait(&sh->accb[buf], (sb >> 1) & 1, err);
      if (!warp_all(w)) {
        if (!w) tc_fail(err, sh, 15);
        ok = false;
        break;
      }
      tc_fence_after();
      drain_f32_to_f64(lane_addr, buf * kGramN, 256, kGramN, sb == 0);
      tc_fence_before();
      mbar_arrive(&sh->drained[buf]);
    }
    if (warp_all(ok && !aborted(sh))) {
      tc_fence_after();
      const int2 ab = spairs[row];
      const bool live = ab.x >= 0;
      const size_t mk = live ? dcol[ab.x] : 0, ml = live ? dcol[ab.y] : 0;
      const double dv = live ? Dinv[mk + ml * P] : 0.0;
      for (int cb = 0; cb < kGramN; cb += 16) {
        double v[16];
        tmem_ld_f64x16(lane_addr + 256 + 2 * cb, v);  // warp-wide: every lane loads
#pragma unroll
        for (int k = 0; k < 16; k++) {
          const int j = n0 + cb + k;
          if (live && n_base + j < J) {
            if (V) {  // gradient pairs: V[cell][pair] for the cells of this launch
              V[(size_t)j * v_ld + ptile * 128 + row] = v[k];
            } else if (Gt) {  // whitened Gram of the dense columns, both triangles, un-whitened later
              double* Gj = Gt + (size_t)j * n_d * n_d;
              Gj[ab.x + (size_t)ab.y * n_d] = v[k];
              Gj[ab.y + (size_t)ab.x * n_d] = v[k];
            } else {
              double* Pj = Psi + (size_t)j * P * P;
              Pj[ml + mk * P] = v[k] + dv;
              Pj[mk + ml * P] = v[k] + dv;
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------------------------------------
// The same contraction on CTA pairs (option tc_pair): a cluster of two CTAs computes 256 pairs x
// 128 columns with one tcgen05.mma.cta_group::2 (M = 256) per K step, issued by the even CTA.
// Each CTA loads its own 128 pair rows of A and half (64 rows) of B, so a CTA moves 48 KB per
// 64-wide K chunk instead of 64 KB and four stages fit in shared memory instead of three: more
// bytes in flight per MMA, against the single-CTA kernel's bound (bytes in flight against L2
// latency). Each CTA's TMEM holds its 128 rows of the accumulators; both CTAs drain their own
// rows into FP64 and write their own pairs' results, as in k_tc_gram (the same sums in the same
// order per output: the K steps and the FP32 runs are those of k_tc_gram).
//
// Barriers: full[s] of the even CTA counts both CTAs' TMA bytes (the odd CTA's loads signal it
// through its cluster address); empty[s] and accb[b] of both CTAs receive the MMA thread's
// multicast commits; drained[b] of the even CTA counts both CTAs' four drain warps. Every wait is
// bounded; both CTAs meet at the hardware cluster barrier after initialisation and before TMEM
// is freed, on every path.
namespace {
constexpr int kStagesPair = 4;
constexpr int kTileBPair = 64 * 128;  // 64 rows x 64 BF16
constexpr uint32_t kIdescPair = idesc_bf16_f32(256, kGramN);
}  // namespace

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreadsGram, 1)
    k_tc_gram2(const __grid_constant__ CUtensorMap map_ahi, const __grid_constant__ CUtensorMap map_alo,
               const __grid_constant__ CUtensorMap map_bhi, const __grid_constant__ CUtensorMap map_blo,
               const int2* __restrict__ pairs, int n_pairs, int chunks_total, const int* __restrict__ dcol, int P,
               int J, const double* __restrict__ Dinv, double* __restrict__ Psi, double* __restrict__ Gt, int n_d,
               int n_base, double* __restrict__ V, int v_ld, int run, int* __restrict__ err, int group) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* A_hi = base;
  unsigned char* A_lo = A_hi + kStagesPair * kTileA;
  unsigned char* B_hi = A_lo + kStagesPair * kTileA;
  unsigned char* B_lo = B_hi + kStagesPair * kTileBPair;
  TcShared* sh = (TcShared*)(B_lo + kStagesPair * kTileBPair);
  int2* spairs = (int2*)(sh + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  // tile order over super tiles (two pair tiles) x column tiles, as k_tc_gram's
  const int tm2 = gridDim.x >> 1;
  int stile = blockIdx.x >> 1, ntile = blockIdx.y;
  if (group > 0) {
    const int id = blockIdx.y * tm2 + stile;
    const int per = group * gridDim.y, grp = id / per, first = grp * group;
    const int gm = min(tm2 - first, group), r = id - grp * per;
    stile = first + r % gm;
    ntile = r / gm;
  }
  const int ptile = 2 * stile + (int)rank;
  const int n0 = ntile * kGramN;
  const int nb0 = n0 + 64 * (int)rank;  // this CTA's half of the B rows
  const int nch = chunks_total;
  const int nsb = (nch + run - 1) / run;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesPair; s++) {
      mbar_init(&sh->full[s], 1);
      mbar_init(&sh->empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&sh->accb[b], 1);
      mbar_init(&sh->drained[b], 8);  // one arrival per drain warp of both CTAs
    }
    mbar_init(&sh->fin, 1);
    sh->abort = *(const volatile int*)err != 0;
    fence_barrier_init();
  }
  for (int r = threadIdx.x; r < 128; r += kThreadsGram) {
    const int p = ptile * 128 + r;
    spairs[r] = p < n_pairs ? pairs[p] : make_int2(-1, -1);
  }
  if (warp == 0) {
    tmem_alloc_pair(&sh->tmem, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // the even CTA's barriers exist before any signal from the odd CTA
  tc_fence_after();
  const uint32_t tmem = sh->tmem;

  if (warp == 0) {
    if (lane == 0) {  // TMA: this CTA's pair products (128 pairs) and half of the weights (64 genes)
      int issued = 0;
      for (int it = 0; it < nch; it++) {
        const int s = it % kStagesPair;
        if (it >= kStagesPair && !mbar_wait(&sh->empty[s], ((it / kStagesPair) - 1) & 1, err)) {
          tc_fail(err, sh, 21);
          break;
        }
        if (sh->abort) break;
        const uint32_t fb = mapa_shared(smem_u32(&sh->full[s]), 0);
        if (rank == 0) mbar_arrive_expect_tx(&sh->full[s], 2u * (2u * kTileA + 2u * kTileBPair));
        const int x = it * 64;
        tma_load_2d_pair(A_hi + s * kTileA, &map_ahi, fb, x, ptile * 128);
        tma_load_2d_pair(A_lo + s * kTileA, &map_alo, fb, x, ptile * 128);
        tma_load_2d_pair(B_hi + s * kTileBPair, &map_bhi, fb, x, n_base + nb0);
        tma_load_2d_pair(B_lo + s * kTileBPair, &map_blo, fb, x, n_base + nb0);
        issued = it + 1;
      }
      // the even CTA sees both CTAs' last loads land before the final cluster barrier
      if (rank == 0)
        for (int it = max(0, issued - kStagesPair); it < issued; it++)
          if (!mbar_wait(&sh->full[it % kStagesPair], (it / kStagesPair) & 1, nullptr)) atomicCAS(err, 0, 22);
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {  // MMA issuer (even CTA)
      for (int it = 0; it < nch; it++) {
        const int s = it % kStagesPair, sb = it / run, pos = it % run, buf = sb & 1;
        if (pos == 0 && sb >= 2 && !mbar_wait(&sh->drained[buf], ((sb >> 1) - 1) & 1, err)) {
          tc_fail(err, sh, 26);
          break;
        }
        if (!mbar_wait(&sh->full[s], (it / kStagesPair) & 1, err)) {
          tc_fail(err, sh, 23);
          break;
        }
        if (sh->abort) break;
        tc_fence_after();
        const uint32_t acc = tmem + buf * kGramN;
        const uint32_t ah = smem_u32(A_hi + s * kTileA), al = smem_u32(A_lo + s * kTileA);
        const uint32_t bh = smem_u32(B_hi + s * kTileBPair), bl = smem_u32(B_lo + s * kTileBPair);
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint32_t off = k * 32;
          mma_bf16_pair(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bh + off), kIdescPair, (pos | k) ? 1u : 0u);
          mma_bf16_pair(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bl + off), kIdescPair, 1u);
          mma_bf16_pair(acc, umma_desc_sw128(al + off), umma_desc_sw128(bh + off), kIdescPair, 1u);
        }
        mma_commit_pair_mc(&sh->empty[s], 3);
        if (pos == run - 1 || it == nch - 1) mma_commit_pair_mc(&sh->accb[buf], 3);
      }
      mma_commit_pair(&sh->fin);
      if (!mbar_wait(&sh->fin, 0, nullptr)) atomicCAS(err, 0, 27);
    }
  } else {
    // drain warps (both CTAs): FP32 runs -> FP64 sum, then this CTA's results
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const uint32_t lane_addr = tmem + ((uint32_t)(q * 32) << 16);
    const uint32_t drained0 = mapa_shared(smem_u32(&sh->drained[0]), 0);
    const uint32_t drained1 = mapa_shared(smem_u32(&sh->drained[1]), 0);
    bool ok = true;
    for (int sb = 0; sb < nsb; sb++) {
      const int buf = sb & 1;
      const bool w = mbar_wait(&sh->accb[buf], (sb >> 1) & 1, err);
      if (!warp_all(w)) {
        if (!w) tc_fail(err, sh, 25);
        ok = false;
        break;
      }
      tc_fence_after();
      drain_f32_to_f64(lane_addr, buf * kGramN, 256, kGramN, sb == 0);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(buf ? drained1 : drained0);
    }
    if (warp_all(ok && !aborted(sh) && *(const volatile int*)err == 0)) {
      tc_fence_after();
      const int2 ab = spairs[row];
      const bool live = ab.x >= 0;
      const size_t mk = live ? dcol[ab.x] : 0, ml = live ? dcol[ab.y] : 0;
      const double dv = live ? Dinv[mk + ml * P] : 0.0;
      for (int cb = 0; cb < kGramN; cb += 16) {
        double v[16];
        tmem_ld_f64x16(lane_addr + 256 + 2 * cb, v);  // warp-wide: every lane loads
#pragma unroll
        for (int k = 0; k < 16; k++) {
          const int j = n0 + cb + k;
          if (live && n_base + j < J) {
            if (V) {
              V[(size_t)j * v_ld + ptile * 128 + row] = v[k];
            } else if (Gt) {
              double* Gj = Gt + (size_t)j * n_d * n_d;
              Gj[ab.x + (size_t)ab.y * n_d] = v[k];
              Gj[ab.y + (size_t)ab.x * n_d] = v[k];
            } else {
              double* Pj = Psi + (size_t)j * P * P;
              Pj[ml + mk * P] = v[k] + dv;
              Pj[mk + ml * P] = v[k] + dv;
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // both CTAs are done with TMEM and the even CTA saw every load land
  tc_fence_after();
  if (warp == 0) tmem_dealloc_pair(tmem, 512);
}

// w = W/Omega as BF16 hi/lo, gene-major with the cell dimension padded to cpad (zeros)
__global__ void k_split_weights(int N, int ldN, int J, int cpad, const double* __restrict__ W,
                                const double* __restrict__ Omega, __nv_bfloat16* __restrict__ whi,
                                __nv_bfloat16* __restrict__ wlo) {
  for (int j = blockIdx.y; j < J; j += gridDim.y)
    for (int i2 = (blockIdx.x * blockDim.x + threadIdx.x) * 2; i2 < cpad; i2 += gridDim.x * blockDim.x * 2) {
      const float a = i2 < N ? (float)(W[(size_t)j * ldN + i2] / Omega[i2]) : 0.f;
      const float b = i2 + 1 < N ? (float)(W[(size_t)j * ldN + i2 + 1] / Omega[i2 + 1]) : 0.f;
      uint32_t h, l;
      split_bf16x2(a, b, h, l);
      *reinterpret_cast<uint32_t*>(whi + (size_t)j * cpad + i2) = h;
      *reinterpret_cast<uint32_t*>(wlo + (size_t)j * cpad + i2) = l;
    }
}

// The prior block of the dense columns, DeltaInv[dcol a, dcol b] (upper triangle, a <= b), for
// its Cholesky factor L (DeltaInv_DD = L L^T).
__global__ void k_gather_dinv(int n_d, int P, const int* __restrict__ dcol, const double* __restrict__ Dinv,
                              double* __restrict__ Lw) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
  if (a >= n_d) return;
  Lw[a + (size_t)b * n_d] = a <= b ? Dinv[dcol[a] + (size_t)dcol[b] * P] : 0.0;
}

// Whitened dense rows L^{-1} d_i in FP64 by forward substitution, stored column by column in
// FP32 (cpad per column, zero padding) and FP64 (ld ldN). The factor's lower triangle is staged
// in shared memory.
__global__ void __launch_bounds__(128) k_whiten_rows(int N, int ldN, int n_d, int rows,
                                                     const double* __restrict__ D, const double* __restrict__ Lw,
                                                     float* __restrict__ DtC, double* __restrict__ DwC) {
  extern __shared__ double ls[];  // lower triangle, row a at a*(a+1)/2
  for (int e = threadIdx.x; e < n_d * n_d; e += blockDim.x) {
    const int a = e % n_d, b = e / n_d;
    if (b <= a) ls[a * (a + 1) / 2 + b] = Lw[a + (size_t)b * n_d];
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows) return;
  if (i >= N) {
    for (int a = 0; a < n_d; a++) DtC[(size_t)a * rows + i] = 0.f;
    return;
  }
  double y[kMaxWhiten];
  for (int a = 0; a < n_d; a++) {
    const double* la = ls + a * (a + 1) / 2;
    double s = D[(size_t)a * ldN + i];
    for (int b = 0; b < a; b++) s = fma(-la[b], y[b], s);
    y[a] = s / la[a];
    DtC[(size_t)a * rows + i] = (float)y[a];
    DwC[(size_t)a * ldN + i] = y[a];
  }
}

// Pair products of the whitened columns as BF16 hi/lo, one row of cells per column pair
// (rows past the pairs are zero): the A operand of the tensor-core Gram, read by TMA.
__global__ void k_pair_split(int cpad, int n_pairs, const int2* __restrict__ pairs, const float* __restrict__ DtC,
                             __nv_bfloat16* __restrict__ ahi, __nv_bfloat16* __restrict__ alo) {
  const int p = blockIdx.y;
  const int2 ab = p < n_pairs ? pairs[p] : make_int2(-1, -1);
  for (int i2 = (blockIdx.x * blockDim.x + threadIdx.x) * 2; i2 < cpad; i2 += gridDim.x * blockDim.x * 2) {
    float x0 = 0.f, x1 = 0.f;
    if (ab.x >= 0) {
      const float2 da = *reinterpret_cast<const float2*>(DtC + (size_t)ab.x * cpad + i2);
      const float2 db = *reinterpret_cast<const float2*>(DtC + (size_t)ab.y * cpad + i2);
      x0 = da.x * db.x;
      x1 = da.y * db.y;
    }
    uint32_t h, l;
    split_bf16x2(x0, x1, h, l);
    *reinterpret_cast<uint32_t*>(ahi + (size_t)p * cpad + i2) = h;
    *reinterpret_cast<uint32_t*>(alo + (size_t)p * cpad + i2) = l;
  }
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// The whitened inverse's pairs S~_j[a, b] (a <= b) as BF16 hi/lo, pair rows x gene columns
// (Jpad, zero padding): the A operand of the tensor-core gradient contraction.
__global__ void k_split_spairs(int J, int Jpad, int n_d, int n_pairs, const int2* __restrict__ pairs,
                               const double* __restrict__ St, __nv_bfloat16* __restrict__ shi,
                               __nv_bfloat16* __restrict__ slo) {
  const int p = blockIdx.y;
  const int2 ab = p < n_pairs ? pairs[p] : make_int2(-1, -1);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < Jpad; j += gridDim.x * blockDim.x) {
    float x = 0.f;
    if (ab.x >= 0 && j < J) x = (float)St[(size_t)j * n_d * n_d + ab.x + (size_t)ab.y * n_d];
    split_bf16(x, shi[(size_t)p * Jpad + j], slo[(size_t)p * Jpad + j]);
  }
}

// O^T = (W/Omega)^T as BF16 hi/lo, cell rows x gene columns (cpad x Jpad, zero padding), by
// 32 x 32 tiles through shared memory (reads along cells, writes along genes).
__global__ void k_split_ot(int N, int ldN, int J, int Jpad, const double* __restrict__ W,
                           const double* __restrict__ Omega, __nv_bfloat16* __restrict__ ohi,
                           __nv_bfloat16* __restrict__ olo) {
  __shared__ float tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, i = i0 + threadIdx.x;
    tile[r][threadIdx.x] = (j < J && i < N) ? (float)(W[(size_t)j * ldN + i] / Omega[i]) : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, j = j0 + threadIdx.x;
    if (j < Jpad) split_bf16(tile[threadIdx.x][r], ohi[(size_t)i * Jpad + j], olo[(size_t)i * Jpad + j]);
  }
}

// U_i = L^{-T} U~_i per cell (in place), by back substitution with the prior factor.
__global__ void __launch_bounds__(128) k_unwhiten_u(int N, int ldN, int n_d, const double* __restrict__ Lw,
                                                    double* __restrict__ U) {
  extern __shared__ double ls[];  // lower triangle, row a at a*(a+1)/2
  for (int e = threadIdx.x; e < n_d * n_d; e += blockDim.x) {
    const int a = e % n_d, b = e / n_d;
    if (b <= a) ls[a * (a + 1) / 2 + b] = Lw[a + (size_t)b * n_d];
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double u[kMaxWhiten];
  for (int a = n_d - 1; a >= 0; a--) {
    double s = U[i + (size_t)a * ldN];
    for (int b = a + 1; b < n_d; b++) s = fma(-ls[b * (b + 1) / 2 + a], u[b], s);
    u[a] = s / ls[a * (a + 1) / 2 + a];
    U[i + (size_t)a * ldN] = u[a];
  }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// 2-D BF16 map over a row-major [rows][cols] array, box (64 cols, box_rows), 128-byte swizzle
static bool make_map(CUtensorMap* m, void* ptr, uint64_t cols, uint64_t rows, uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {cols * 2};
  const cuuint32_t box[2] = {64, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <class T>
static int tc_alloc(Ctx* c, T** p, size_t n, const char* what) {
  if (cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
    cudaGetLastError();
    c->err = std::string("device allocation failed: ") + what;
    return GPL_ERR_ALLOC;
  }
  return GPL_OK;
}

int tc_prepare(Ctx* c) {
  if (c->tc.ready) return GPL_OK;
  TcState& t = c->tc;
  const int J = c->J, n_d = c->n_d;
  if (n_d > kMaxWhiten || J > 65535) {
    c->err = "the tensor-core form supports at most 160 dense model columns and 65535 genes";
    return GPL_ERR_ARG;
  }
  t.cpad = (c->N + 127) / 128 * 128;  // cells: a multiple of 64 for K and of 128 for the V tiles
  t.chunks_cells = t.cpad / 64;
  t.gram_tiles_n = (J + kGramN - 1) / kGramN;
  t.Jpad = (J + 63) / 64 * 64;
  std::vector<int2> pairs;
  for (int a = 0; a < n_d; a++)
    for (int b = a; b < n_d; b++) pairs.push_back(make_int2(a, b));
  t.n_pairs = (int)pairs.size();
  t.pair_tiles = (t.n_pairs + 127) / 128;
  const size_t prow = (size_t)t.pair_tiles * 128;
  int rc;
  if ((rc = tc_alloc(c, &t.whi, (size_t)J * t.cpad, "w hi"))) return rc;
  if ((rc = tc_alloc(c, &t.wlo, (size_t)J * t.cpad, "w lo"))) return rc;
  if ((rc = tc_alloc(c, &t.DtC, (size_t)t.cpad * n_d, "whitened dense columns"))) return rc;
  if ((rc = tc_alloc(c, &t.DwC, (size_t)c->ldN * n_d, "whitened dense columns (FP64)"))) return rc;
  if ((rc = tc_alloc(c, &t.ahi, prow * t.cpad, "pair products hi"))) return rc;
  if ((rc = tc_alloc(c, &t.alo, prow * t.cpad, "pair products lo"))) return rc;
  if ((rc = tc_alloc(c, &t.shi, prow * t.Jpad, "inverse pairs hi"))) return rc;
  if ((rc = tc_alloc(c, &t.slo, prow * t.Jpad, "inverse pairs lo"))) return rc;
  if ((rc = tc_alloc(c, &t.ohi, (size_t)t.cpad * t.Jpad, "O^T hi"))) return rc;
  if ((rc = tc_alloc(c, &t.olo, (size_t)t.cpad * t.Jpad, "O^T lo"))) return rc;
  if ((rc = tc_alloc(c, &t.pairs, (size_t)t.n_pairs, "pairs"))) return rc;
  if ((rc = tc_alloc(c, &t.err, 1, "tc error flag"))) return rc;
  if ((rc = tc_alloc(c, &t.Lw, (size_t)n_d * n_d, "prior factor"))) return rc;
  if ((rc = tc_alloc(c, &t.Gt, (size_t)J * n_d * n_d, "whitened Gram"))) return rc;
  if ((rc = tc_alloc(c, &t.Tt, (size_t)J * n_d * n_d, "un-whitening product"))) return rc;
  {
    // fixed Rademacher probes (+-1) of the log-determinant correction, one P-vector per gene
    if ((rc = tc_alloc(c, &t.probe, (size_t)c->P * J, "log-determinant probes"))) return rc;
    std::vector<double> v((size_t)c->P * J);
    uint64_t state = 0x9E3779B97F4A7C15ull;
    for (size_t e = 0; e < v.size(); e++) {
      state ^= state << 13;
      state ^= state >> 7;
      state ^= state << 17;
      v[e] = (state >> 63) ? 1.0 : -1.0;
    }
    GPL_TRY(c, cudaMemcpy(t.probe, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice));
  }
  t.smem_whiten = (int)sizeof(double) * n_d * (n_d + 1) / 2;
  GPL_TRY(c, cudaFuncSetAttribute(k_whiten_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, t.smem_whiten));
  GPL_TRY(c, cudaFuncSetAttribute(k_unwhiten_u, cudaFuncAttributeMaxDynamicSharedMemorySize, t.smem_whiten));
  GPL_TRY(c, cudaMemset(t.err, 0, sizeof(int)));
  GPL_TRY(c, cudaMemcpy(t.pairs, pairs.data(), sizeof(int2) * pairs.size(), cudaMemcpyHostToDevice));
  if (!make_map(&t.map_shi, t.shi, t.Jpad, prow, 128) || !make_map(&t.map_slo, t.slo, t.Jpad, prow, 128) ||
      !make_map(&t.map_ohi, t.ohi, t.Jpad, t.cpad, 128) || !make_map(&t.map_olo, t.olo, t.Jpad, t.cpad, 128) ||
      !make_map(&t.map_ahi, t.ahi, t.cpad, prow, 128) || !make_map(&t.map_alo, t.alo, t.cpad, prow, 128) ||
      !make_map(&t.map_whi, t.whi, t.cpad, J, kGramN) || !make_map(&t.map_wlo, t.wlo, t.cpad, J, kGramN) ||
      !make_map(&t.map_whi64, t.whi, t.cpad, J, 64) || !make_map(&t.map_wlo64, t.wlo, t.cpad, J, 64) ||
      !make_map(&t.map_ohi64, t.ohi, t.Jpad, t.cpad, 64) || !make_map(&t.map_olo64, t.olo, t.Jpad, t.cpad, 64)) {
    c->err = "cuTensorMapEncodeTiled failed";
    return GPL_ERR_CUDA;
  }
  t.run = c->tc_run > 0 ? c->tc_run : kSBGram;
  t.smem_gram = 1024 + kStagesGram * (2 * kTileA + 2 * kTileBG) + (int)sizeof(TcShared) + 128 * (int)sizeof(int2);
  GPL_TRY(c, cudaFuncSetAttribute(k_tc_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, t.smem_gram));
  t.smem_gram2 = 1024 + kStagesPair * (2 * kTileA + 2 * kTileBPair) + (int)sizeof(TcShared) + 128 * (int)sizeof(int2);
  GPL_TRY(c, cudaFuncSetAttribute(k_tc_gram2, cudaFuncAttributeMaxDynamicSharedMemorySize, t.smem_gram2));
  t.ready = true;
  return GPL_OK;
}

void tc_release(Ctx* c) {
  graph_reset(c);
  TcState& t = c->tc;
  void* bufs[] = {t.whi, t.wlo, t.pairs, t.err, t.Lw, t.Gt, t.Tt, t.DtC, t.DwC, t.ahi, t.alo, t.shi, t.slo,
                  t.ohi, t.olo, t.probe};
  for (void* p : bufs)
    if (p) cudaFree(p);
  t = TcState();
}

static int tc_check_flag(Ctx* c) {
  int flag = 0;
  GPL_TRY(c, cudaMemcpyAsync(&flag, c->tc.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  if (flag) {
    c->err = "tensor-core kernel gave up waiting (code " + std::to_string(flag) + ")";
    return GPL_ERR_TIMEOUT;
  }
  return GPL_OK;
}

// The bounded wait of the tensor-core kernels (mbar_wait) against a barrier whose phase nothing
// completes: the wait runs out after limit_ns and the CTA records code 99 in the flag and
// returns. No copy, MMA or TMEM allocation is in flight, so giving up leaves nothing behind.
__global__ void k_wait_probe(uint64_t limit_ns, int* __restrict__ flag) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0, nullptr, limit_ns)) atomicCAS(flag, 0, 99);
}

int wait_probe(Ctx* c, int64_t limit_ns) {
  int* flag = nullptr;
  if (cudaMalloc((void**)&flag, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    c->err = "device allocation failed: probe flag";
    return GPL_ERR_ALLOC;
  }
  int v = 0;
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), c->stream);
  if (e == cudaSuccess) {
    k_wait_probe<<<1, 32, 0, c->stream>>>((uint64_t)limit_ns, flag);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&v, flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(flag);
  GPL_TRY(c, e);
  c->launches++;
  if (v) {
    c->err = "device wait gave up after " + std::to_string(limit_ns) + " ns (code " + std::to_string(v) + ")";
    return GPL_ERR_TIMEOUT;
  }
  return GPL_OK;
}

int launch_tc_gram(Ctx* c) {
  int rc = tc_prepare(c);
  if (rc) return rc;
  TcState& t = c->tc;
  {
    // Whitening by the prior's factor: the tensor-core Gram of L^{-1} d_i, whose errors are then
    // relative to a matrix bounded below by the identity, is mapped back as L G L^T + DeltaInv in
    // FP64. Without it, cond(Psi_j) ~ 1e14 (no jitter on Kmm) turns 1e-6 Gram errors into failed
    // Cholesky factorizations.
    ProfScope ps(c, "whiten");
    dim3 g(div_up(c->n_d, 128), c->n_d);
    k_gather_dinv<<<g, 128, 0, c->stream>>>(c->n_d, c->P, c->dcol_d, c->DeltaInv, t.Lw);
    GPL_LAUNCHED(c, "k_gather_dinv");
    launch_chol_exact_raw(c->stream, t.Lw, c->n_d);
    GPL_LAUNCHED(c, "k_chol_exact");
    k_whiten_rows<<<t.cpad / 128, 128, t.smem_whiten, c->stream>>>(c->N, c->ldN, c->n_d, t.cpad, c->Dm, t.Lw,
                                                                    t.DtC, t.DwC);
    GPL_LAUNCHED(c, "k_whiten_rows");
    dim3 gp(std::min(16, div_up(t.cpad, 512)), t.pair_tiles * 128);
    k_pair_split<<<gp, 256, 0, c->stream>>>(t.cpad, t.n_pairs, t.pairs, t.DtC, t.ahi, t.alo);
    GPL_LAUNCHED(c, "k_pair_split");
  }
  {
    ProfScope ps(c, "split_weights");
    dim3 g(std::min(64, div_up(t.cpad, 512)), std::min(c->J, 65535));
    k_split_weights<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->J, t.cpad, c->W, c->Omega, t.whi, t.wlo);
    GPL_LAUNCHED(c, "k_split_weights");
  }
  {
    ProfScope ps(c, "gram");
    dim3 g(t.pair_tiles, t.gram_tiles_n);
    Tunable* tu = nullptr;
    const int grp = tune_pick(c, "tc_gram", {0, 8, 16}, 8, &tu);
    TuneScope ts(c, tu);
    if (c->tc_pair) {
      dim3 g2(2 * div_up(t.pair_tiles, 2), t.gram_tiles_n);
      k_tc_gram2<<<g2, kThreadsGram, t.smem_gram2, c->stream>>>(t.map_ahi, t.map_alo, t.map_whi64, t.map_wlo64,
                                                                t.pairs, t.n_pairs, t.chunks_cells, c->dcol_d, c->P,
                                                                c->J, c->DeltaInv, c->Psi, t.Gt, c->n_d, 0, nullptr,
                                                                0, t.run, t.err, grp);
      GPL_LAUNCHED(c, "k_tc_gram2");
    } else {
      k_tc_gram<<<g, kThreadsGram, t.smem_gram, c->stream>>>(t.map_ahi, t.map_alo, t.map_whi, t.map_wlo, t.pairs,
                                                             t.n_pairs, t.chunks_cells, c->dcol_d, c->P, c->J,
                                                             c->DeltaInv, c->Psi, t.Gt, c->n_d, 0, nullptr, 0, t.run,
                                                             t.err, grp);
      GPL_LAUNCHED(c, "k_tc_gram");
    }
  }
  {
    ProfScope ps(c, "unwhiten");
    if ((rc = dgen_unwhiten(c, t.Gt, t.Tt, t.Lw))) return rc;
  }
  return c->tc_check ? tc_check_flag(c) : GPL_OK;
}

// The gradient contraction on tensor cores, over the column pairs of the whitened columns:
// S~_j = L^T S_DD,j L (FP64), V[i, pair] = sum_j O_ij S~_j[pair] (tcgen05, FP64-accumulated),
// U~_i = sum_b D~_ib V[i, pair(a, b)], and U_i = L^{-T} U~_i (FP64). Needs the factor and the
// whitened columns of the preceding tensor-core Gram.
int launch_tc_grad(Ctx* c) {
  int rc = tc_prepare(c);
  if (rc) return rc;
  if ((rc = pair_prepare(c))) return rc;
  TcState& t = c->tc;
  PairState& s = c->pr;
  {
    ProfScope ps(c, "spair");
    if ((rc = dgen_whiten_inverse(c, t.Lw, t.Tt, t.Gt))) return rc;
    dim3 g(std::min(64, div_up(t.Jpad, 256)), t.pair_tiles * 128);
    k_split_spairs<<<g, 256, 0, c->stream>>>(c->J, t.Jpad, c->n_d, t.n_pairs, t.pairs, t.Gt, t.shi, t.slo);
    GPL_LAUNCHED(c, "k_split_spairs");
    dim3 g2(t.cpad / 32, t.Jpad / 32);
    k_split_ot<<<g2, dim3(32, 8), 0, c->stream>>>(c->N, c->ldN, c->J, t.Jpad, c->W, c->Omega, t.ohi, t.olo);
    GPL_LAUNCHED(c, "k_split_ot");
  }
  for (int c0 = 0; c0 < c->N; c0 += s.v_cells) {
    const int c1 = std::min(c->N, c0 + s.v_cells);
    {
      ProfScope ps(c, "uq");
      dim3 g(t.pair_tiles, div_up(c1 - c0, kGramN));
      Tunable* tu = nullptr;
      const int grp = tune_pick(c, "tc_grad", {0, 8, 16}, 8, &tu);
      TuneScope ts(c, c1 - c0 == c->N ? tu : nullptr);
      if (c->tc_pair) {
        dim3 g2(2 * div_up(t.pair_tiles, 2), div_up(c1 - c0, kGramN));
        k_tc_gram2<<<g2, kThreadsGram, t.smem_gram2, c->stream>>>(t.map_shi, t.map_slo, t.map_ohi64, t.map_olo64,
                                                                  t.pairs, t.n_pairs, t.Jpad / 64, c->dcol_d, c->P, c1,
                                                                  c->DeltaInv, nullptr, nullptr, c->n_d, c0, s.V,
                                                                  s.pairs_pad, t.run, t.err, grp);
        GPL_LAUNCHED(c, "k_tc_gram2(gradient pairs)");
      } else {
        k_tc_gram<<<g, kThreadsGram, t.smem_gram, c->stream>>>(t.map_shi, t.map_slo, t.map_ohi, t.map_olo, t.pairs,
                                                               t.n_pairs, t.Jpad / 64, c->dcol_d, c->P, c1,
                                                               c->DeltaInv, nullptr, nullptr, c->n_d, c0, s.V,
                                                               s.pairs_pad, t.run, t.err, grp);
        GPL_LAUNCHED(c, "k_tc_gram(gradient pairs)");
      }
    }
    if ((rc = launch_v_to_u_cells(c, c0, c1, t.DwC))) return rc;
  }
  {
    ProfScope ps(c, "unwhiten_u");
    k_unwhiten_u<<<div_up(c->N, 128), 128, t.smem_whiten, c->stream>>>(c->N, c->ldN, c->n_d, t.Lw, c->U);
    GPL_LAUNCHED(c, "k_unwhiten_u");
  }
  return c->tc_check ? tc_check_flag(c) : GPL_OK;
}

int tc_error_flag(Ctx* c) { return c->tc.ready ? tc_check_flag(c) : GPL_OK; }

}  // namespace gpl
