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
// k_tc_gram   G[p, j] = sum_i (D_ia D_ib) w_ij for the dense column pairs p = (a <= b) and
//             128 genes per CTA over every cell, written straight into Psi_j (both triangles,
//             plus DeltaInv). M = 128 pairs, N = 128 genes, K = 64 cells per stage. The pair
//             products are generated by four producer warps straight into the 128-byte-swizzled
//             A tiles; w = W/Omega (BF16 hi/lo, gene x cell) arrives by TMA. TMEM: two FP32
//             128 x 128 accumulators (columns 0-255) and the FP64 sum (columns 256-511).
//             Algorithmic work: N*J*n_d*(n_d+1) flops.
// k_tc_grad   U[i, a] = sum_{j,b} (O_ij D_ib) S_j[b, a] over dense columns a, b: M = 128 cells,
//             N = n_d rounded to 16 (<= 160), K = (gene, b) flattened, 64 per stage, split over
//             4 K ranges whose FP64 partials are summed in order. One FP32 accumulator drained
//             every 8 chunks into the FP64 sum. Algorithmic work: 2*N*J*n_d^2 flops.
//
// Warp roles (320 threads): warp 0 allocates TMEM and issues the TMA loads, warp 1 issues the
// MMAs (one thread), warps 2-5 produce the A tiles, warps 6-9 drain the accumulators and write
// the results (warp w reads TMEM lanes 32*(w % 4) .. +31). Full barriers count the TMA bytes
// plus 128 producer arrivals; empty barriers and the accumulator barriers are armed by
// tcgen05.commit; drained barriers count the 128 drain threads. Every wait is bounded: one that
// runs out records an error code, and every role drains what it started before TMEM is freed.
#include <cuda.h>
#include <stdlib.h>

#include <algorithm>

#include "gpl_internal.cuh"
#include "tc_common.cuh"

namespace gpl {

using namespace tc;

namespace {
constexpr int kThreads = 320;           // gradient: TMA, MMA, 4 producer and 4 drain warps
constexpr int kThreadsGram = 192;       // Gram: TMA, MMA and 4 drain warps
constexpr int kStagesGram = 3;          // pipeline depth, Gram (192 KB of operand tiles)
constexpr int kStagesGrad = 2;          // pipeline depth, gradient (B tiles up to 20 KB, plus D rows)
constexpr int kMaxStages = 3;
constexpr int kGramN = 128;             // genes per Gram tile
constexpr int kSBGram = 4;              // chunks per FP32 run (Gram)
constexpr int kSBGrad = 8;              // chunks per FP32 run (gradient)
constexpr int kTileA = 128 * 128;       // 128 rows x 64 BF16
constexpr int kTileBG = kGramN * 128;   // 128 gene rows x 64 BF16
constexpr int kGradSplits = 4;
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
              double* __restrict__ Psi, double* __restrict__ Gt, int n_d, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* A_hi = base;
  unsigned char* A_lo = A_hi + kStagesGram * kTileA;
  unsigned char* B_hi = A_lo + kStagesGram * kTileA;
  unsigned char* B_lo = B_hi + kStagesGram * kTileBG;
  TcShared* sh = (TcShared*)(B_lo + kStagesGram * kTileBG);
  int2* spairs = (int2*)(sh + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ptile = blockIdx.x, n0 = blockIdx.y * kGramN;
  const int nch = chunks_total;
  const int nsb = (nch + kSBGram - 1) / kSBGram;

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
        tma_load_2d(B_hi + s * kTileBG, &map_whi, &sh->full[s], x, n0);
        tma_load_2d(B_lo + s * kTileBG, &map_wlo, &sh->full[s], x, n0);
        issued = it + 1;
      }
      for (int it = max(0, issued - kStagesGram); it < issued; it++)
        if (!mbar_wait(&sh->full[it % kStagesGram], (it / kStagesGram) & 1, nullptr)) atomicCAS(err, 0, 12);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      for (int it = 0; it < nch; it++) {
        const int s = it % kStagesGram, sb = it / kSBGram, pos = it % kSBGram, buf = sb & 1;
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
        if (pos == kSBGram - 1 || it == nch - 1) mma_commit(&sh->accb[buf]);
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
          if (live && j < J) {
            if (Gt) {  // whitened Gram of the dense columns, both triangles, un-whitened later
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

// Dense model columns as FP32, cell-major rows of n_dp (zero padding)
__global__ void k_dense_rows(int N, int ldN, int n_d, int n_dp, int rows, const double* __restrict__ D,
                             float* __restrict__ Dt) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)rows * n_dp) return;
  const int i = (int)(e / n_dp), a = (int)(e % n_dp);
  Dt[e] = (i < N && a < n_d) ? (float)D[(size_t)a * ldN + i] : 0.f;
}

// The prior block of the dense columns, DeltaInv[dcol a, dcol b] (upper triangle, a <= b), for
// its Cholesky factor L (DeltaInv_DD = L L^T).
__global__ void k_gather_dinv(int n_d, int P, const int* __restrict__ dcol, const double* __restrict__ Dinv,
                              double* __restrict__ Lw) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
  if (a >= n_d) return;
  Lw[a + (size_t)b * n_d] = a <= b ? Dinv[dcol[a] + (size_t)dcol[b] * P] : 0.0;
}

// Whitened dense rows L^{-1} d_i in FP64 by forward substitution, stored as FP32 rows of n_dp
// (zero padding). The factor's lower triangle is staged in shared memory.
__global__ void __launch_bounds__(128) k_whiten_rows(int N, int ldN, int n_d, int n_dp, int rows,
                                                     const double* __restrict__ D, const double* __restrict__ Lw,
                                                     float* __restrict__ Dt, float* __restrict__ DtC) {
  extern __shared__ double ls[];  // lower triangle, row a at a*(a+1)/2
  for (int e = threadIdx.x; e < n_d * n_d; e += blockDim.x) {
    const int a = e % n_d, b = e / n_d;
    if (b <= a) ls[a * (a + 1) / 2 + b] = Lw[a + (size_t)b * n_d];
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows) return;
  float* out = Dt + (size_t)i * n_dp;
  if (i >= N) {
    for (int a = 0; a < n_dp; a++) out[a] = 0.f;
    for (int a = 0; a < n_d; a++) DtC[(size_t)a * rows + i] = 0.f;
    return;
  }
  double y[kMaxWhiten];
  for (int a = 0; a < n_d; a++) {
    const double* la = ls + a * (a + 1) / 2;
    double s = D[(size_t)a * ldN + i];
    for (int b = 0; b < a; b++) s = fma(-la[b], y[b], s);
    y[a] = s / la[a];
    out[a] = (float)y[a];
    DtC[(size_t)a * rows + i] = (float)y[a];
  }
  for (int a = n_d; a < n_dp; a++) out[a] = 0.f;
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

// ---------------------------------------------------------------------------------------------
// Gradient contraction
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_grad(const __grid_constant__ CUtensorMap map_bhi, const __grid_constant__ CUtensorMap map_blo, int N,
              int ldN, int n_d, int n_b, const float* __restrict__ Dt, int n_dp, const double* __restrict__ W,
              const double* __restrict__ Omega, int64_t K_total, int chunks_total, int chunks_per_split,
              int cpad, double* __restrict__ Up, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tileB = n_b * 128;  // n_b rows x 128 bytes
  const int tileBa = (tileB + 1023) & ~1023;
  unsigned char* A_hi = base;
  unsigned char* A_lo = A_hi + kStagesGrad * kTileA;
  unsigned char* B_hi = A_lo + kStagesGrad * kTileA;
  unsigned char* B_lo = B_hi + kStagesGrad * tileBa;
  float* Ds = (float*)(B_lo + kStagesGrad * tileBa);  // 128 x (n_d + 1)
  TcShared* sh = (TcShared*)(Ds + 128 * (n_d + 1));
  const int ldD = n_d + 1;
  const int nb32 = (n_b + 31) / 32 * 32;          // FP32 columns drained (multiple of 32)
  const uint32_t f64col = (uint32_t)nb32;         // FP64 sum at columns [nb32, 3*nb32)
  uint32_t tcols = 32;                            // TMEM columns allocated: a power of two >= 3*nb32
  while (tcols < 3u * nb32) tcols <<= 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i0 = blockIdx.x * 128, split = blockIdx.y;
  const int kc0 = split * chunks_per_split;
  const int kc1 = min(chunks_total, kc0 + chunks_per_split);
  const int nch = kc1 - kc0;
  const int nsb = (nch + kSBGrad - 1) / kSBGrad;
  const uint32_t idesc = idesc_bf16_f32(128, n_b);

  if (threadIdx.x == 0) tc_init(sh, err, 1 + 128);
  __syncthreads();
  if (sh->abort) return;
  for (int e = threadIdx.x; e < 128 * n_d; e += kThreads) {
    const int r = e / n_d, a = e % n_d;
    Ds[r * ldD + a] = Dt[(size_t)(i0 + r) * n_dp + a];
  }
  if (warp == 0) {
    tmem_alloc(&sh->tmem, tcols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem;

  if (warp == 0) {
    if (lane == 0) {
      int issued = 0;
      for (int it = 0; it < nch; it++) {
        const int s = it % kStagesGrad;
        if (it >= kStagesGrad && !mbar_wait(&sh->empty[s], ((it / kStagesGrad) - 1) & 1, err)) { tc_fail(err, sh, 21); break; }
        if (sh->abort) break;
        mbar_arrive_expect_tx(&sh->full[s], 2u * (uint32_t)tileB);
        const int x = (kc0 + it) * 64;
        tma_load_2d(B_hi + s * tileBa, &map_bhi, &sh->full[s], x, 0);
        tma_load_2d(B_lo + s * tileBa, &map_blo, &sh->full[s], x, 0);
        issued = it + 1;
      }
      for (int it = max(0, issued - kStagesGrad); it < issued; it++)
        if (!mbar_wait(&sh->full[it % kStagesGrad], (it / kStagesGrad) & 1, nullptr)) atomicCAS(err, 0, 22);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      for (int it = 0; it < nch; it++) {
        const int s = it % kStagesGrad, sb = it / kSBGrad, pos = it % kSBGrad;
        if (pos == 0 && sb >= 1 && !mbar_wait(&sh->drained[0], (sb - 1) & 1, err)) { tc_fail(err, sh, 26); break; }
        if (!mbar_wait(&sh->full[s], (it / kStagesGrad) & 1, err)) { tc_fail(err, sh, 23); break; }
        if (sh->abort) break;
        tc_fence_after();
        const uint32_t ah = smem_u32(A_hi + s * kTileA), al = smem_u32(A_lo + s * kTileA);
        const uint32_t bh = smem_u32(B_hi + s * tileBa), bl = smem_u32(B_lo + s * tileBa);
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint32_t off = k * 32;
          mma_bf16(tmem, umma_desc_sw128(ah + off), umma_desc_sw128(bh + off), idesc, (pos | k) ? 1u : 0u);
          mma_bf16(tmem, umma_desc_sw128(ah + off), umma_desc_sw128(bl + off), idesc, 1u);
          mma_bf16(tmem, umma_desc_sw128(al + off), umma_desc_sw128(bh + off), idesc, 1u);
        }
        mma_commit(&sh->empty[s]);
        if (pos == kSBGrad - 1 || it == nch - 1) mma_commit(&sh->accb[0]);
      }
      mma_finish(sh, err, 27);
    }
  } else if (warp < 6) {
    const int r = threadIdx.x - 64;
    const int i = i0 + r;
    const bool live = i < N;
    const double om = live ? Omega[i] : 1.0;
    const float* drow = Ds + r * ldD;
    int jcur = -1;
    float ocur = 0.f;
    for (int it = 0; it < nch; it++) {
      const int s = it % kStagesGrad;
      if (it >= kStagesGrad && !mbar_wait(&sh->empty[s], ((it / kStagesGrad) - 1) & 1, err)) { tc_fail(err, sh, 24); break; }
      if (sh->abort) break;
      const int64_t k0 = (int64_t)(kc0 + it) * 64;
      int j = (int)(k0 / n_d), b = (int)(k0 - (int64_t)j * n_d);
      const uint32_t ah = smem_u32(A_hi + s * kTileA), al = smem_u32(A_lo + s * kTileA);
#pragma unroll 1
      for (int c16 = 0; c16 < 8; c16++) {
        float x[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
          const int64_t kk = k0 + c16 * 8 + e;
          float v = 0.f;
          if (live && kk < K_total) {
            if (j != jcur) {
              jcur = j;
              ocur = (float)(W[(size_t)j * ldN + i] / om);
            }
            v = ocur * drow[b];
          }
          x[e] = v;
          if (++b == n_d) { b = 0; j++; }
        }
        uint32_t h[4], l[4];
#pragma unroll
        for (int q = 0; q < 4; q++) split_bf16x2(x[2 * q], x[2 * q + 1], h[q], l[q]);
        const uint32_t o = sw128_offset(r, c16);
        st_shared_v4(ah + o, h[0], h[1], h[2], h[3]);
        st_shared_v4(al + o, l[0], l[1], l[2], l[3]);
      }
      fence_proxy_async();
      mbar_arrive(&sh->full[s]);
    }
  } else {
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const uint32_t lane_addr = tmem + ((uint32_t)(q * 32) << 16);
    bool ok = true;
    for (int sb = 0; sb < nsb; sb++) {
      const bool w = mbar_wait(&sh->accb[0], sb & 1, err);
      if (!warp_all(w)) {
        if (!w) tc_fail(err, sh, 25);
        ok = false;
        break;
      }
      tc_fence_after();
      drain_f32_to_f64(lane_addr, 0, f64col, nb32, sb == 0);
      tc_fence_before();
      mbar_arrive(&sh->drained[0]);
    }
    if (warp_all(ok && !aborted(sh)) && nsb > 0) {
      tc_fence_after();
      const int i = i0 + row;
      for (int cb = 0; cb < nb32; cb += 16) {
        double v[16];
        tmem_ld_f64x16(lane_addr + f64col + 2 * cb, v);
#pragma unroll
        for (int k = 0; k < 16; k++) {
          const int a = cb + k;
          if (a < n_d) Up[((size_t)split * n_b + a) * cpad + i] = v[k];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, tcols);
}

// S_j[DD] as the B operand: Bt[a][j*n_d + b] = S_j[dcol[b], dcol[a]] in BF16 hi/lo (rows n_b)
__global__ void k_split_sdd(int J, int P, int n_d, int64_t Kpad, const int* __restrict__ dcol,
                            const double* __restrict__ S, __nv_bfloat16* __restrict__ bhi,
                            __nv_bfloat16* __restrict__ blo) {
  const int a = blockIdx.y;
  const int64_t K = (int64_t)J * n_d;
  for (int64_t k2 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 2; k2 < Kpad;
       k2 += (int64_t)gridDim.x * blockDim.x * 2) {
    float v[2];
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int64_t kk = k2 + e;
      float x = 0.f;
      if (a < n_d && kk < K) {
        const int j = (int)(kk / n_d), b = (int)(kk - (int64_t)j * n_d);
        x = (float)S[(size_t)j * P * P + dcol[b] + (size_t)dcol[a] * P];
      }
      v[e] = x;
    }
    uint32_t h, l;
    split_bf16x2(v[0], v[1], h, l);
    *reinterpret_cast<uint32_t*>(bhi + (size_t)a * Kpad + k2) = h;
    *reinterpret_cast<uint32_t*>(blo + (size_t)a * Kpad + k2) = l;
  }
}

__global__ void k_tc_grad_reduce(int N, int ldN, int n_d, int n_b, int cpad, int nsplit,
                                 const double* __restrict__ Up, double* __restrict__ U) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y;
  if (i >= N || a >= n_d) return;
  double s = 0.0;
  for (int k = 0; k < nsplit; k++) s += Up[((size_t)k * n_b + a) * cpad + i];
  U[i + (size_t)a * ldN] = s;
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
  t.n_dp = (n_d + 3) / 4 * 4;
  t.cpad = (c->N + 127) / 128 * 128;  // cells: a multiple of 64 for K and of 128 for the gradient tiles
  t.chunks_cells = t.cpad / 64;
  t.gram_tiles_n = (J + kGramN - 1) / kGramN;
  std::vector<int2> pairs;
  for (int a = 0; a < n_d; a++)
    for (int b = a; b < n_d; b++) pairs.push_back(make_int2(a, b));
  t.n_pairs = (int)pairs.size();
  t.pair_tiles = (t.n_pairs + 127) / 128;
  t.n_b = (n_d + 15) / 16 * 16;
  const int64_t K = (int64_t)J * n_d;
  t.Kpad = (K + 63) / 64 * 64;
  t.grad_chunks = (int)(t.Kpad / 64);
  t.grad_chunks_per_split = (t.grad_chunks + kGradSplits - 1) / kGradSplits;
  t.grad_splits = (t.grad_chunks + t.grad_chunks_per_split - 1) / t.grad_chunks_per_split;  // none empty
  if (3 * ((t.n_b + 31) / 32 * 32) > 512) {
    c->err = "the tensor-core form supports at most 160 dense model columns";
    return GPL_ERR_ARG;
  }
  int rc;
  if ((rc = tc_alloc(c, &t.whi, (size_t)J * t.cpad, "w hi"))) return rc;
  if ((rc = tc_alloc(c, &t.wlo, (size_t)J * t.cpad, "w lo"))) return rc;
  if ((rc = tc_alloc(c, &t.Dt, (size_t)t.cpad * t.n_dp, "dense rows"))) return rc;
  if ((rc = tc_alloc(c, &t.DtC, (size_t)t.cpad * n_d, "whitened dense columns"))) return rc;
  if ((rc = tc_alloc(c, &t.ahi, (size_t)t.pair_tiles * 128 * t.cpad, "pair products hi"))) return rc;
  if ((rc = tc_alloc(c, &t.alo, (size_t)t.pair_tiles * 128 * t.cpad, "pair products lo"))) return rc;
  if ((rc = tc_alloc(c, &t.pairs, (size_t)t.n_pairs, "pairs"))) return rc;
  if ((rc = tc_alloc(c, &t.bhi, (size_t)t.n_b * t.Kpad, "S hi"))) return rc;
  if ((rc = tc_alloc(c, &t.blo, (size_t)t.n_b * t.Kpad, "S lo"))) return rc;
  if ((rc = tc_alloc(c, &t.Up, (size_t)t.grad_splits * t.n_b * t.cpad, "grad partials"))) return rc;
  if ((rc = tc_alloc(c, &t.err, 1, "tc error flag"))) return rc;
  if ((rc = tc_alloc(c, &t.Lw, (size_t)n_d * n_d, "prior factor"))) return rc;
  if ((rc = tc_alloc(c, &t.Gt, (size_t)J * n_d * n_d, "whitened Gram"))) return rc;
  if ((rc = tc_alloc(c, &t.Tt, (size_t)J * n_d * n_d, "un-whitening product"))) return rc;
  if (n_d > kMaxWhiten || J > 65535) {
    c->err = "the tensor-core form supports at most 160 dense model columns and 65535 genes";
    return GPL_ERR_ARG;
  }
  t.smem_whiten = (int)sizeof(double) * n_d * (n_d + 1) / 2;
  GPL_TRY(c, cudaFuncSetAttribute(k_whiten_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, t.smem_whiten));
  GPL_TRY(c, cudaMemset(t.err, 0, sizeof(int)));
  GPL_TRY(c, cudaMemcpy(t.pairs, pairs.data(), sizeof(int2) * pairs.size(), cudaMemcpyHostToDevice));
  if (!make_map(&t.map_ahi, t.ahi, t.cpad, (uint64_t)t.pair_tiles * 128, 128) ||
      !make_map(&t.map_alo, t.alo, t.cpad, (uint64_t)t.pair_tiles * 128, 128) ||
      !make_map(&t.map_whi, t.whi, t.cpad, J, kGramN) || !make_map(&t.map_wlo, t.wlo, t.cpad, J, kGramN) ||
      !make_map(&t.map_bhi, t.bhi, t.Kpad, t.n_b, t.n_b) || !make_map(&t.map_blo, t.blo, t.Kpad, t.n_b, t.n_b)) {
    c->err = "cuTensorMapEncodeTiled failed";
    return GPL_ERR_CUDA;
  }
  t.smem_gram = 1024 + kStagesGram * (2 * kTileA + 2 * kTileBG) + (int)sizeof(TcShared) + 128 * (int)sizeof(int2);
  const int tileBa = (t.n_b * 128 + 1023) & ~1023;
  t.smem_grad = 1024 + kStagesGrad * (2 * kTileA + 2 * tileBa) + 128 * (n_d + 1) * 4 + (int)sizeof(TcShared);
  if (t.smem_grad > 227 * 1024) {
    c->err = "the tensor-core gradient needs more shared memory than a CTA has";
    return GPL_ERR_ARG;
  }
  GPL_TRY(c, cudaFuncSetAttribute(k_tc_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, t.smem_gram));
  GPL_TRY(c, cudaFuncSetAttribute(k_tc_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, t.smem_grad));
  t.ready = true;
  return GPL_OK;
}

void tc_release(Ctx* c) {
  TcState& t = c->tc;
  void* bufs[] = {t.whi, t.wlo, t.Dt, t.pairs, t.bhi, t.blo, t.Up, t.err, t.Lw, t.Gt, t.Tt, t.DtC, t.ahi, t.alo};
  for (void* p : bufs)
    if (p) cudaFree(p);
  const bool keep = t.check_each;
  t = TcState();
  t.check_each = keep;
}

static int tc_check_flag(Ctx* c) {
  int flag = 0;
  GPL_TRY(c, cudaMemcpyAsync(&flag, c->tc.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  GPL_TRY(c, cudaStreamSynchronize(c->stream));
  if (flag) {
    c->err = "tensor-core kernel gave up waiting (code " + std::to_string(flag) + ")";
    return GPL_ERR_CUDA;
  }
  return GPL_OK;
}

int launch_dense_rows(Ctx* c) {
  TcState& t = c->tc;
  const size_t n = (size_t)t.cpad * t.n_dp;
  k_dense_rows<<<div_up((int64_t)n, 256), 256, 0, c->stream>>>(c->N, c->ldN, c->n_d, t.n_dp, t.cpad, c->Dm, t.Dt);
  GPL_LAUNCHED(c, "k_dense_rows");
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
    k_whiten_rows<<<t.cpad / 128, 128, t.smem_whiten, c->stream>>>(c->N, c->ldN, c->n_d, t.n_dp, t.cpad, c->Dm,
                                                                    t.Lw, t.Dt, t.DtC);
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
    k_tc_gram<<<g, kThreadsGram, t.smem_gram, c->stream>>>(t.map_ahi, t.map_alo, t.map_whi, t.map_wlo, t.pairs,
                                                           t.n_pairs,
                                                       t.chunks_cells, c->dcol_d, c->P, c->J, c->DeltaInv, c->Psi,
                                                       t.Gt, c->n_d, t.err);
    GPL_LAUNCHED(c, "k_tc_gram");
  }
  {
    ProfScope ps(c, "unwhiten");
    if ((rc = dgen_unwhiten(c, t.Gt, t.Tt, t.Lw))) return rc;
  }
  return c->tc.check_each ? tc_check_flag(c) : GPL_OK;
}

int launch_tc_grad(Ctx* c) {
  int rc = tc_prepare(c);
  if (rc) return rc;
  TcState& t = c->tc;
  if ((rc = launch_dense_rows(c))) return rc;
  {
    ProfScope ps(c, "split_sdd");
    dim3 g(std::min<int64_t>(1024, div_up(t.Kpad, 512)), t.n_b);
    k_split_sdd<<<g, 256, 0, c->stream>>>(c->J, c->P, c->n_d, t.Kpad, c->dcol_d, c->PsiInv, t.bhi, t.blo);
    GPL_LAUNCHED(c, "k_split_sdd");
  }
  {
    ProfScope ps(c, "uq");
    dim3 g(t.cpad / 128, t.grad_splits);
    k_tc_grad<<<g, kThreads, t.smem_grad, c->stream>>>(t.map_bhi, t.map_blo, c->N, c->ldN, c->n_d, t.n_b, t.Dt,
                                                       t.n_dp, c->W, c->Omega, (int64_t)c->J * c->n_d,
                                                       t.grad_chunks, t.grad_chunks_per_split, t.cpad, t.Up, t.err);
    GPL_LAUNCHED(c, "k_tc_grad");
  }
  {
    ProfScope ps(c, "grad_reduce");
    dim3 g(div_up(c->N, 256), c->n_d);
    k_tc_grad_reduce<<<g, 256, 0, c->stream>>>(c->N, c->ldN, c->n_d, t.n_b, t.cpad, t.grad_splits, t.Up, c->U);
    GPL_LAUNCHED(c, "k_tc_grad_reduce");
  }
  return c->tc.check_each ? tc_check_flag(c) : GPL_OK;
}

int tc_error_flag(Ctx* c) { return c->tc.ready ? tc_check_flag(c) : GPL_OK; }

}  // namespace gpl
