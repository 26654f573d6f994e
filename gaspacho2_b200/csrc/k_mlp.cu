// The amortised encoder (no reference counterpart: the reference places every cell by L-BFGS,
// ggplvm.cu:1214-1301): a 2-hidden-layer MLP from a cell's expression profile to the mean and
// log-variance of its latent coordinates, trained and run by this file's kernels.
//
// Network n_in -> H -> H -> 2Q, GELU (erf form). FP32 master weights and Adam state; every
// matrix product takes BF16 operands on the 5th-generation tensor cores (tcgen05.mma kind::f16,
// FP32 accumulation in TMEM), operands staged by TMA in 128-byte-swizzled K-major tiles.
//
//   k_mlp_gemm     C[m, n] = sum_k A[m, k] B[n, k], A and B BF16 K-major (row = output index,
//                  K contiguous), one 128 x 128 output tile per CTA, K in 64-wide chunks through
//                  a 4-stage TMA pipeline; warp 0 issues the TMA loads, warp 1 the MMAs (one
//                  thread), warps 2-5 read the accumulator and run the epilogue:
//                    kFwdGelu  v = acc + b[n]; pre = v (FP32); act = bf16(gelu(v)) in both the
//                              K-major layout (next layer's A) and transposed (the weight
//                              gradient's B)
//                    kFwdOut   out = acc + b[n] (FP32)
//                    kBwdGelu  d = acc * gelu'(pre); dpre = d (FP32, bias gradient); bf16(d) in
//                              both layouts
//                    kStore    out = acc (FP32: weight gradients)
//                  Every mbarrier wait is bounded; a wait that runs out records an error code,
//                  the MMA thread waits (bounded) for its MMAs before TMEM is freed.
//   k_enc_features log1p(y / s) of the selected genes' counts, written as BF16 into the
//                  cell-major feature matrix F and its transpose FT (rows = features).
//   k_enc_loss     the Gaussian negative log-likelihood of the targets per cell and the
//                  output gradient, FP32 and BF16 (both layouts).
//   k_colsum       bias gradients: column sums over the batch, one thread per column, rows in
//                  order (deterministic).
//   k_adam         Adam on the FP32 masters, then the BF16 copies the GEMMs read (and the
//                  transposed copies of W2 and W3 for the backward products).
//
// Layout (device, all row-major): F [Npad][Kin] and FT [Kin][Npad] (Kin = n_in rounded up to 128,
// Npad = cells rounded up to the batch), per-batch activations [B][H] and transposes [H][B],
// outputs [B][128], W1 [H][Kin], W2 [H][H], W3 [128][H] (rows past 2Q zero), W2T [H][H],
// W3T [H][64] (columns past 2Q zero).
#include <cuda.h>
#include <math.h>

#include <algorithm>
#include <random>
#include <string>
#include <vector>

#include "gpl_internal.cuh"
#include "tc_common.cuh"

using namespace gpl;
using namespace gpl::tc;

namespace {

constexpr int kThreads = 192;
constexpr int kStages = 4;
constexpr int kTile = 128 * 128;  // bytes of a 128-row x 64-column BF16 tile
constexpr uint32_t kIdesc = idesc_bf16_f32(128, 128);

enum Epi { kFwdGelu = 0, kFwdOut = 1, kBwdGelu = 2, kStore = 3 };

struct EpiArgs {
  int mode, m_valid, n_valid;
  const float* bias;       // kFwdGelu, kFwdOut
  const float* pre_in;     // kBwdGelu: the forward pre-activations [m][ld32]
  float* out32;            // pre (kFwdGelu), out (kFwdOut, kStore), dpre (kBwdGelu): [m][ld32]
  int ld32;
  __nv_bfloat16* act;      // [m][ldb] (kFwdGelu, kBwdGelu)
  int ldb;
  __nv_bfloat16* actT;     // [n][ldt] (kFwdGelu, kBwdGelu)
  int ldt;
};

struct MlpShared {
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t accb;
  uint64_t fin;
  uint32_t tmem;
  int abort;
};

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * expf(-0.5f * x * x) * 0.39894228040143268f;
}

__device__ __forceinline__ void mlp_fail(int* err, MlpShared* sh, int code) {
  atomicExch(&sh->abort, 1);
  atomicCAS(err, 0, code);
}

__global__ void __launch_bounds__(kThreads, 1)
    k_mlp_gemm(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b, int nch,
               int a_x0, int a_y0, int b_x0, int b_y0, EpiArgs ep, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* As = base;
  unsigned char* Bs = As + kStages * kTile;
  MlpShared* sh = (MlpShared*)(Bs + kStages * kTile);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * 128;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&sh->full[s], 1);
      mbar_init(&sh->empty[s], 1);
    }
    mbar_init(&sh->accb, 1);
    mbar_init(&sh->fin, 1);
    sh->abort = *(const volatile int*)err != 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (sh->abort) return;
  if (warp == 0) {
    tmem_alloc(&sh->tmem, 128);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      int issued = 0;
      for (int it = 0; it < nch; it++) {
        const int s = it % kStages;
        if (it >= kStages && !mbar_wait(&sh->empty[s], ((it / kStages) - 1) & 1, err)) {
          mlp_fail(err, sh, 31);
          break;
        }
        if (*(volatile int*)&sh->abort) break;
        mbar_arrive_expect_tx(&sh->full[s], 2u * kTile);
        tma_load_2d(As + s * kTile, &map_a, &sh->full[s], a_x0 + it * 64, a_y0 + m0);
        tma_load_2d(Bs + s * kTile, &map_b, &sh->full[s], b_x0 + it * 64, b_y0 + n0);
        issued = it + 1;
      }
      // copies still in flight land before the CTA may exit
      for (int it = max(0, issued - kStages); it < issued; it++)
        if (!mbar_wait(&sh->full[it % kStages], (it / kStages) & 1, nullptr)) atomicCAS(err, 0, 32);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      for (int it = 0; it < nch; it++) {
        const int s = it % kStages;
        if (!mbar_wait(&sh->full[s], (it / kStages) & 1, err)) {
          mlp_fail(err, sh, 33);
          break;
        }
        if (*(volatile int*)&sh->abort) break;
        tc_fence_after();
        const uint32_t a = smem_u32(As + s * kTile), b = smem_u32(Bs + s * kTile);
#pragma unroll
        for (int k = 0; k < 4; k++)
          mma_bf16(tmem, umma_desc_sw128(a + k * 32), umma_desc_sw128(b + k * 32), kIdesc, (it | k) ? 1u : 0u);
        mma_commit(&sh->empty[s]);
      }
      mma_commit(&sh->accb);
      mma_commit(&sh->fin);
      if (!mbar_wait(&sh->fin, 0, nullptr)) atomicCAS(err, 0, 34);
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 = output rows
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const int m = m0 + row;
    const uint32_t lane_addr = tmem + ((uint32_t)(q * 32) << 16);
    const bool w = mbar_wait(&sh->accb, 0, err);
    if (!__all_sync(0xffffffffu, w)) {
      if (!w) mlp_fail(err, sh, 35);
    } else if (!__any_sync(0xffffffffu, *(volatile int*)&sh->abort != 0)) {
      tc_fence_after();
      const bool live_m = m < ep.m_valid;
      for (int cb = 0; cb < 128; cb += 32) {
        float v[32];
        tmem_ld32(lane_addr + cb, v);  // warp-wide: every lane loads
        if (!live_m) continue;
#pragma unroll 4
        for (int k = 0; k < 32; k++) {
          const int n = n0 + cb + k;
          if (n >= ep.n_valid) break;
          const float a = v[k];
          if (ep.mode == kStore) {
            ep.out32[(size_t)m * ep.ld32 + n] = a;
          } else if (ep.mode == kFwdOut) {
            ep.out32[(size_t)m * ep.ld32 + n] = a + ep.bias[n];
          } else if (ep.mode == kFwdGelu) {
            const float pre = a + ep.bias[n];
            ep.out32[(size_t)m * ep.ld32 + n] = pre;
            const __nv_bfloat16 h = __float2bfloat16_rn(gelu_f(pre));
            ep.act[(size_t)m * ep.ldb + n] = h;
            ep.actT[(size_t)n * ep.ldt + m] = h;
          } else {  // kBwdGelu
            const float d = a * gelu_grad_f(ep.pre_in[(size_t)m * ep.ld32 + n]);
            ep.out32[(size_t)m * ep.ld32 + n] = d;
            const __nv_bfloat16 h = __float2bfloat16_rn(d);
            ep.act[(size_t)m * ep.ldb + n] = h;
            ep.actT[(size_t)n * ep.ldt + m] = h;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, 128);
}

// log1p(y / s) of feature f's gene for the cells of its matched counts; rows in `row_of` order.
__global__ void k_enc_features(int n_feat, const int32_t* __restrict__ genes, const int64_t* __restrict__ gptr,
                               const int32_t* __restrict__ gvalid, const int32_t* __restrict__ cell,
                               const double* __restrict__ cnt, const double* __restrict__ ls,
                               const int32_t* __restrict__ row_of, __nv_bfloat16* __restrict__ F, int ldf,
                               __nv_bfloat16* __restrict__ FT, int ldt) {
  const int f = blockIdx.y;
  if (f >= n_feat) return;
  const int g = genes[f];
  const int64_t b = gptr[g], e = gptr[g] + gvalid[g];
  for (int64_t l = b + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < e; l += (int64_t)gridDim.x * blockDim.x) {
    const int i = cell[l];
    const int r = row_of[i];
    const __nv_bfloat16 v = __float2bfloat16_rn((float)log1p(cnt[l] / ls[i]));
    F[(size_t)r * ldf + f] = v;
    FT[(size_t)f * ldt + r] = v;
  }
}

// Per row r < rows of the batch: out[r][0..Q) = mean, [Q..2Q) = log-variance, X[r][q] target.
// loss_rows[r] = 0.5 sum_q (lv + (x - mu)^2 e^-lv); the output gradient (scaled by 1/rows) as
// FP32 d32[r][0..2Q), BF16 dq[r][0..64) (K-major, zero past 2Q) and dqT[0..128)[r].
__global__ void k_enc_loss(int rows, int Q, const float* __restrict__ out, int ldo, const float* __restrict__ X,
                           float* __restrict__ loss_rows, float* __restrict__ d32, __nv_bfloat16* __restrict__ dq,
                           __nv_bfloat16* __restrict__ dqT, int ldt) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const float inv = 1.0f / (float)rows;
  float l = 0.f;
  for (int q = 0; q < Q; q++) {
    const float mu = out[(size_t)r * ldo + q], lv = out[(size_t)r * ldo + Q + q];
    const float d = X[(size_t)r * Q + q] - mu, e = expf(-lv);
    l += lv + d * d * e;
    const float gm = -d * e * inv, gl = 0.5f * (1.0f - d * d * e) * inv;
    d32[(size_t)r * ldo + q] = gm;
    d32[(size_t)r * ldo + Q + q] = gl;
    dq[(size_t)r * 64 + q] = __float2bfloat16_rn(gm);
    dq[(size_t)r * 64 + Q + q] = __float2bfloat16_rn(gl);
    dqT[(size_t)q * ldt + r] = __float2bfloat16_rn(gm);
    dqT[(size_t)(Q + q) * ldt + r] = __float2bfloat16_rn(gl);
  }
  loss_rows[r] = 0.5f * l;
}

// out[n] = sum_{r < rows} d[r][n] for n < cols (rows in order)
__global__ void k_colsum(int rows, int cols, const float* __restrict__ d, int ld, float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; r++) s += d[(size_t)r * ld + n];
  out[n] = s;
}

// sum of a small array in order (one thread): the batch loss
__global__ void k_sum_ordered(int n, const float* __restrict__ a, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < n; i++) s += a[i];
  *out = s;
}

// Adam on one parameter block of rows x cols (FP32 master w, gradient g, moments m, v), then
// the BF16 copy wb[r][c] (row-major ld ldw) and, if given, the transposed copy wt[c][r] (ld ldwt).
__global__ void k_adam(int rows, int cols, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ wb, int ldw, __nv_bfloat16* __restrict__ wt, int ldwt) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= rows * cols) return;
  const int r = e / cols, c = e - r * cols;
  const float gr = g[e];
  const float mm = b1 * m[e] + (1.f - b1) * gr;
  const float vv = b2 * v[e] + (1.f - b2) * gr * gr;
  m[e] = mm;
  v[e] = vv;
  const float nw = w[e] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  w[e] = nw;
  if (wb) wb[(size_t)r * ldw + c] = __float2bfloat16_rn(nw);
  if (wt) wt[(size_t)c * ldwt + r] = __float2bfloat16_rn(nw);
}

// BF16 copies of an FP32 block (after the weights are set from the host)
__global__ void k_to_bf16(int rows, int cols, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int ldw,
                          __nv_bfloat16* __restrict__ wt, int ldwt) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= rows * cols) return;
  const int r = e / cols, c = e - r * cols;
  const __nv_bfloat16 h = __float2bfloat16_rn(w[e]);
  if (wb) wb[(size_t)r * ldw + c] = h;
  if (wt) wt[(size_t)c * ldwt + r] = h;
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn2)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

namespace {

EncodeTiledFn2 encode_fn2() {
  static EncodeTiledFn2 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn2)p;
  }
  return fn;
}

// BF16 row-major [rows][cols] (cols a multiple of 64, rows a multiple of 128), box 64 x 128
bool bf16_map(CUtensorMap* m, const void* ptr, uint64_t cols, uint64_t rows) {
  EncodeTiledFn2 fn = encode_fn2();
  if (!fn) return false;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {cols * 2};
  const cuuint32_t box[2] = {64, 128};
  const cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int rup(int a, int b) { return (a + b - 1) / b * b; }

}  // namespace

struct gpl_enc {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  int n_in = 0, H = 0, Q = 0, B = 0, Kin = 0;
  int64_t launches = 0;
  // parameters: FP32 masters, gradients, Adam moments (flat blocks W1 b1 W2 b2 W3 b3, padded)
  float *W1 = nullptr, *b1 = nullptr, *W2 = nullptr, *b2 = nullptr, *W3 = nullptr, *b3 = nullptr;
  float *gW1 = nullptr, *gb1 = nullptr, *gW2 = nullptr, *gb2 = nullptr, *gW3 = nullptr, *gb3 = nullptr;
  float* adam = nullptr;  // m then v for every block, same layout as the masters
  size_t n_par = 0;       // padded parameter count (W1 [H][Kin] b1 [H] W2 [H][H] b2 [H] W3 [128][H] b3 [128])
  int64_t step = 0;
  __nv_bfloat16 *W1b = nullptr, *W2b = nullptr, *W2T = nullptr, *W3b = nullptr, *W3T = nullptr;
  // per-batch activations
  float *pre1 = nullptr, *pre2 = nullptr, *out = nullptr, *d32 = nullptr, *dpre1 = nullptr, *dpre2 = nullptr;
  float *loss_rows = nullptr, *Xb = nullptr;
  double* loss_sum = nullptr;
  __nv_bfloat16 *H1 = nullptr, *H1T = nullptr, *H2 = nullptr, *H2T = nullptr, *dq = nullptr, *dqT = nullptr;
  __nv_bfloat16 *dP2 = nullptr, *dP2T = nullptr, *dP1 = nullptr, *dP1T = nullptr;
  int* err_d = nullptr;
  // cell sets: 0 training, 1 evaluation
  struct Set {
    int N = 0, Npad = 0;
    __nv_bfloat16 *F = nullptr, *FT = nullptr;
    float* X = nullptr;  // targets [Npad][Q] in row order (training set)
    std::vector<int32_t> cell_of_row;
    CUtensorMap mapF, mapFT;
  } set[2];
  CUtensorMap mW1, mW2, mW2T, mW3, mW3T, mH1, mH1T, mH2, mH2T, mdq, mdqT, mdP2, mdP2T, mdP1T;
};

#define ENC_TRY(e, expr)                                                 \
  do {                                                                   \
    cudaError_t err_ = (expr);                                           \
    if (err_ != cudaSuccess) {                                           \
      (e)->err = std::string(#expr) + ": " + cudaGetErrorString(err_);   \
      return GPL_ERR_CUDA;                                               \
    }                                                                    \
  } while (0)
#define ENC_LAUNCHED(e, name)                                                     \
  do {                                                                            \
    (e)->launches++;                                                              \
    cudaError_t err_ = cudaGetLastError();                                        \
    if (err_ != cudaSuccess) {                                                    \
      (e)->err = std::string(name) + ": " + cudaGetErrorString(err_);             \
      return GPL_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

namespace {

template <class T>
int ealloc(gpl_enc* e, T** p, size_t n) {
  if (cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
    cudaGetLastError();
    e->err = "device allocation failed (" + std::to_string(sizeof(T) * n) + " bytes)";
    return GPL_ERR_ALLOC;
  }
  return cudaMemsetAsync(*p, 0, sizeof(T) * (n ? n : 1), e->stream) == cudaSuccess ? GPL_OK : GPL_ERR_CUDA;
}

constexpr int kSmem = 1024 + kStages * 2 * kTile + (int)sizeof(MlpShared);

int gemm(gpl_enc* e, const CUtensorMap& A, const CUtensorMap& Bm, int M, int N, int K, int a_x0, int a_y0, int b_x0,
         int b_y0, const EpiArgs& ep) {
  static bool attr = false;
  if (!attr) {
    ENC_TRY(e, cudaFuncSetAttribute(k_mlp_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem));
    attr = true;
  }
  dim3 g(M / 128, N / 128);
  k_mlp_gemm<<<g, kThreads, kSmem, e->stream>>>(A, Bm, K / 64, a_x0, a_y0, b_x0, b_y0, ep, e->err_d);
  ENC_LAUNCHED(e, "k_mlp_gemm");
  return GPL_OK;
}

int check_err(gpl_enc* e) {
  int v = 0;
  ENC_TRY(e, cudaMemcpyAsync(&v, e->err_d, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  ENC_TRY(e, cudaStreamSynchronize(e->stream));
  if (v) {
    e->err = "tensor-core GEMM gave up waiting (code " + std::to_string(v) + ")";
    return GPL_ERR_TIMEOUT;
  }
  return GPL_OK;
}

// Forward of rows [r0, r0 + B) of a cell set into the batch buffers (pre1/H1/H1T, pre2/H2/H2T,
// out). m_valid limits the rows written (the last, partial batch of a prediction).
int forward(gpl_enc* e, int s, int r0, int m_valid) {
  const int H = e->H, B = e->B;
  EpiArgs ep{};
  ep.mode = kFwdGelu;
  ep.m_valid = m_valid;
  ep.n_valid = H;
  ep.bias = e->b1;
  ep.out32 = e->pre1;
  ep.ld32 = H;
  ep.act = e->H1;
  ep.ldb = H;
  ep.actT = e->H1T;
  ep.ldt = B;
  int rc = gemm(e, e->set[s].mapF, e->mW1, B, H, e->Kin, 0, r0, 0, 0, ep);
  if (rc) return rc;
  ep.bias = e->b2;
  ep.out32 = e->pre2;
  ep.act = e->H2;
  ep.actT = e->H2T;
  if ((rc = gemm(e, e->mH1, e->mW2, B, H, H, 0, 0, 0, 0, ep))) return rc;
  EpiArgs eo{};
  eo.mode = kFwdOut;
  eo.m_valid = m_valid;
  eo.n_valid = 2 * e->Q;
  eo.bias = e->b3;
  eo.out32 = e->out;
  eo.ld32 = 128;
  return gemm(e, e->mH2, e->mW3, B, 128, H, 0, 0, 0, 0, eo);
}

// Loss and every gradient of one training batch (rows [r0, r0 + B) of set 0) into gW*, gb*.
int backward(gpl_enc* e, int r0) {
  const int H = e->H, B = e->B, Q = e->Q;
  gpl_enc::Set& S = e->set[0];
  k_enc_loss<<<(B + 127) / 128, 128, 0, e->stream>>>(B, Q, e->out, 128, S.X + (size_t)r0 * Q, e->loss_rows, e->d32,
                                                     e->dq, e->dqT, B);
  ENC_LAUNCHED(e, "k_enc_loss");
  EpiArgs st{};
  st.mode = kStore;
  st.m_valid = 2 * Q;
  st.n_valid = H;
  st.out32 = e->gW3;
  st.ld32 = H;
  int rc = gemm(e, e->mdqT, e->mH2T, 128, H, B, 0, 0, 0, 0, st);  // dW3 = dO^T H2
  if (rc) return rc;
  EpiArgs bg{};
  bg.mode = kBwdGelu;
  bg.m_valid = B;
  bg.n_valid = H;
  bg.pre_in = e->pre2;
  bg.out32 = e->dpre2;
  bg.ld32 = H;
  bg.act = e->dP2;
  bg.ldb = H;
  bg.actT = e->dP2T;
  bg.ldt = B;
  if ((rc = gemm(e, e->mdq, e->mW3T, B, H, 64, 0, 0, 0, 0, bg))) return rc;  // dA2 = (dO W3) * gelu'(a2)
  st.m_valid = H;
  st.out32 = e->gW2;
  if ((rc = gemm(e, e->mdP2T, e->mH1T, H, H, B, 0, 0, 0, 0, st))) return rc;  // dW2 = dA2^T H1
  bg.pre_in = e->pre1;
  bg.out32 = e->dpre1;
  bg.act = e->dP1;
  bg.actT = e->dP1T;
  if ((rc = gemm(e, e->mdP2, e->mW2T, B, H, H, 0, 0, 0, 0, bg))) return rc;  // dA1 = (dA2 W2) * gelu'(a1)
  st.out32 = e->gW1;
  st.ld32 = e->Kin;
  st.n_valid = e->n_in;
  if ((rc = gemm(e, e->mdP1T, S.mapFT, H, e->Kin, B, 0, 0, r0, 0, st))) return rc;  // dW1 = dA1^T F
  k_colsum<<<(H + 127) / 128, 128, 0, e->stream>>>(B, H, e->dpre1, H, e->gb1);
  ENC_LAUNCHED(e, "k_colsum");
  k_colsum<<<(H + 127) / 128, 128, 0, e->stream>>>(B, H, e->dpre2, H, e->gb2);
  ENC_LAUNCHED(e, "k_colsum");
  k_colsum<<<1, 128, 0, e->stream>>>(B, 2 * Q, e->d32, 128, e->gb3);
  ENC_LAUNCHED(e, "k_colsum");
  k_sum_ordered<<<1, 32, 0, e->stream>>>(B, e->loss_rows, e->loss_sum);
  ENC_LAUNCHED(e, "k_sum_ordered");
  return GPL_OK;
}

struct Block {
  float *w, *g;
  int rows, cols;
  __nv_bfloat16* wb;
  int ldw;
  __nv_bfloat16* wt;
  int ldwt;
};

std::vector<Block> blocks(gpl_enc* e) {
  const int H = e->H, Q = e->Q;
  return {{e->W1, e->gW1, H, e->Kin, e->W1b, e->Kin, nullptr, 0},
          {e->b1, e->gb1, 1, H, nullptr, 0, nullptr, 0},
          {e->W2, e->gW2, H, H, e->W2b, H, e->W2T, H},
          {e->b2, e->gb2, 1, H, nullptr, 0, nullptr, 0},
          {e->W3, e->gW3, 2 * Q, H, e->W3b, H, e->W3T, 64},
          {e->b3, e->gb3, 1, 2 * Q, nullptr, 0, nullptr, 0}};
}

int adam_step(gpl_enc* e, float lr) {
  e->step++;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, (float)e->step), c2 = 1.f - powf(b2, (float)e->step);
  size_t off = 0;
  for (const Block& b : blocks(e)) {
    const int n = b.rows * b.cols;
    float* m = e->adam + off;
    float* v = e->adam + e->n_par + off;
    k_adam<<<(n + 255) / 256, 256, 0, e->stream>>>(b.rows, b.cols, b.w, b.g, m, v, lr, b1, b2, eps, c1, c2, b.wb,
                                                   b.ldw, b.wt, b.ldwt);
    ENC_LAUNCHED(e, "k_adam");
    off += (size_t)n;
  }
  return GPL_OK;
}

int refresh_bf16(gpl_enc* e) {
  for (const Block& b : blocks(e)) {
    if (!b.wb && !b.wt) continue;
    const int n = b.rows * b.cols;
    k_to_bf16<<<(n + 255) / 256, 256, 0, e->stream>>>(b.rows, b.cols, b.w, b.wb, b.ldw, b.wt, b.ldwt);
    ENC_LAUNCHED(e, "k_to_bf16");
  }
  return GPL_OK;
}

}  // namespace

extern "C" {

int gpl_enc_create(gpl_enc** out, int device, void* stream, int n_in, int hidden, int q, int batch, uint64_t seed) {
  if (!out || n_in < 1 || hidden < 128 || hidden % 128 || q < 1 || 2 * q > 64 || batch < 128 || batch % 128)
    return GPL_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return GPL_ERR_CUDA;
  }
  gpl_enc* e = new gpl_enc();
  e->device = device;
  if (stream) {
    e->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete e;
      return GPL_ERR_CUDA;
    }
    e->own_stream = true;
  }
  e->n_in = n_in;
  e->H = hidden;
  e->Q = q;
  e->B = batch;
  e->Kin = rup(n_in, 128);
  const int H = hidden, B = batch, Kin = e->Kin;
  // parameter blocks, padded: W1 [H][Kin] b1 [H] W2 [H][H] b2 [H] W3 [2Q][H] b3 [2Q]
  e->n_par = (size_t)H * Kin + H + (size_t)H * H + H + (size_t)2 * q * H + 2 * q;
  int rc = GPL_OK;
  float* P = nullptr;
  float* G = nullptr;
  if ((rc = ealloc(e, &P, e->n_par)) || (rc = ealloc(e, &G, e->n_par)) || (rc = ealloc(e, &e->adam, 2 * e->n_par)) ||
      (rc = ealloc(e, &e->W1b, (size_t)H * Kin)) || (rc = ealloc(e, &e->W2b, (size_t)H * H)) ||
      (rc = ealloc(e, &e->W2T, (size_t)H * H)) || (rc = ealloc(e, &e->W3b, (size_t)128 * H)) ||
      (rc = ealloc(e, &e->W3T, (size_t)H * 64)) || (rc = ealloc(e, &e->pre1, (size_t)B * H)) ||
      (rc = ealloc(e, &e->pre2, (size_t)B * H)) || (rc = ealloc(e, &e->out, (size_t)B * 128)) ||
      (rc = ealloc(e, &e->d32, (size_t)B * 128)) || (rc = ealloc(e, &e->dpre1, (size_t)B * H)) ||
      (rc = ealloc(e, &e->dpre2, (size_t)B * H)) || (rc = ealloc(e, &e->loss_rows, (size_t)B)) ||
      (rc = ealloc(e, &e->loss_sum, 1)) || (rc = ealloc(e, &e->H1, (size_t)B * H)) ||
      (rc = ealloc(e, &e->H1T, (size_t)H * B)) || (rc = ealloc(e, &e->H2, (size_t)B * H)) ||
      (rc = ealloc(e, &e->H2T, (size_t)H * B)) || (rc = ealloc(e, &e->dq, (size_t)B * 64)) ||
      (rc = ealloc(e, &e->dqT, (size_t)128 * B)) || (rc = ealloc(e, &e->dP2, (size_t)B * H)) ||
      (rc = ealloc(e, &e->dP2T, (size_t)H * B)) || (rc = ealloc(e, &e->dP1, (size_t)B * H)) ||
      (rc = ealloc(e, &e->dP1T, (size_t)H * B)) || (rc = ealloc(e, &e->err_d, 1))) {
    gpl_enc_destroy(e);
    return rc;
  }
  size_t off = 0;
  float** mp[6] = {&e->W1, &e->b1, &e->W2, &e->b2, &e->W3, &e->b3};
  float** gp[6] = {&e->gW1, &e->gb1, &e->gW2, &e->gb2, &e->gW3, &e->gb3};
  const size_t sz[6] = {(size_t)H * Kin, (size_t)H, (size_t)H * H, (size_t)H, (size_t)2 * q * H, (size_t)2 * q};
  for (int k = 0; k < 6; k++) {
    *mp[k] = P + off;
    *gp[k] = G + off;
    off += sz[k];
  }
  if (!bf16_map(&e->mW1, e->W1b, Kin, H) || !bf16_map(&e->mW2, e->W2b, H, H) || !bf16_map(&e->mW2T, e->W2T, H, H) ||
      !bf16_map(&e->mW3, e->W3b, H, 128) || !bf16_map(&e->mW3T, e->W3T, 64, H) || !bf16_map(&e->mH1, e->H1, H, B) ||
      !bf16_map(&e->mH1T, e->H1T, B, H) || !bf16_map(&e->mH2, e->H2, H, B) || !bf16_map(&e->mH2T, e->H2T, B, H) ||
      !bf16_map(&e->mdq, e->dq, 64, B) || !bf16_map(&e->mdqT, e->dqT, B, 128) || !bf16_map(&e->mdP2, e->dP2, H, B) ||
      !bf16_map(&e->mdP2T, e->dP2T, B, H) || !bf16_map(&e->mdP1T, e->dP1T, B, H)) {
    e->err = "cuTensorMapEncodeTiled failed";
    gpl_enc_destroy(e);
    return GPL_ERR_CUDA;
  }
  // seeded initialisation: weights N(0, 1/fan_in), biases zero
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::vector<float> h(e->n_par, 0.f);
  for (int r = 0; r < H; r++)
    for (int c = 0; c < n_in; c++) h[(size_t)r * Kin + c] = nd(rng) / sqrtf((float)n_in);
  const size_t o2 = (size_t)H * Kin + H, o3 = o2 + (size_t)H * H + H;
  for (size_t k = 0; k < (size_t)H * H; k++) h[o2 + k] = nd(rng) / sqrtf((float)H);
  for (size_t k = 0; k < (size_t)2 * q * H; k++) h[o3 + k] = nd(rng) / sqrtf((float)H);
  if (cudaMemcpyAsync(P, h.data(), sizeof(float) * e->n_par, cudaMemcpyHostToDevice, e->stream) != cudaSuccess ||
      refresh_bf16(e) != GPL_OK || cudaStreamSynchronize(e->stream) != cudaSuccess) {
    gpl_enc_destroy(e);
    return GPL_ERR_CUDA;
  }
  *out = e;
  return GPL_OK;
}

int gpl_enc_destroy(gpl_enc* e) {
  if (!e) return GPL_OK;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  void* bufs[] = {e->W1,  e->gW1, e->adam, e->W1b, e->W2b,   e->W2T,  e->W3b, e->W3T,  e->pre1, e->pre2,
                  e->out, e->d32, e->dpre1, e->dpre2, e->loss_rows, e->loss_sum, e->H1, e->H1T, e->H2, e->H2T,
                  e->dq,  e->dqT, e->dP2,  e->dP2T, e->dP1,  e->dP1T, e->err_d};
  for (void* p : bufs)
    if (p) cudaFree(p);
  for (auto& s : e->set) {
    if (s.F) cudaFree(s.F);
    if (s.FT) cudaFree(s.FT);
    if (s.X) cudaFree(s.X);
  }
  if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return GPL_OK;
}

const char* gpl_enc_last_error(const gpl_enc* e) { return e ? e->err.c_str() : "null encoder"; }

int gpl_enc_set_cells(gpl_enc* e, int which, int N, int J, int64_t nnz, const int32_t* cell_idx,
                      const int32_t* gene_ptr, const double* counts, const double* ls, const int32_t* genes,
                      const int32_t* cell_of_row) {
  if (!e || which < 0 || which > 1 || N <= 0 || J <= 0 || nnz < 0 || !gene_ptr || !ls || !genes ||
      (nnz > 0 && (!cell_idx || !counts)))
    return GPL_ERR_ARG;
  cudaSetDevice(e->device);
  for (int f = 0; f < e->n_in; f++)
    if (genes[f] < 0 || genes[f] >= J) {
      e->err = "feature gene out of range";
      return GPL_ERR_ARG;
    }
  gpl_enc::Set& S = e->set[which];
  if (S.F) cudaFree(S.F);
  if (S.FT) cudaFree(S.FT);
  if (S.X) cudaFree(S.X);
  S = gpl_enc::Set();
  S.N = N;
  S.Npad = rup(N, e->B);
  S.cell_of_row.resize(N);
  std::vector<int32_t> row_of(N, -1);
  for (int r = 0; r < N; r++) {
    const int i = cell_of_row ? cell_of_row[r] : r;
    if (i < 0 || i >= N || row_of[i] >= 0) {
      e->err = "cell_of_row must be a permutation of 0..N-1";
      return GPL_ERR_ARG;
    }
    S.cell_of_row[r] = i;
    row_of[i] = r;
  }
  // the merge walk's matched prefix of each gene (as the fit reads its counts)
  std::vector<int64_t> gp(J + 1);
  std::vector<int32_t> gv(J);
  for (int j = 0; j <= J; j++) gp[j] = gene_ptr[j];
  for (int j = 0; j < J; j++) {
    if (gp[j] < 0 || gp[j] > gp[j + 1] || gp[j + 1] > nnz) {
      e->err = "gene offsets are not monotone within [0, nnz]";
      return GPL_ERR_FORMAT;
    }
    int last = -1;
    int64_t l = gp[j];
    for (; l < gp[j + 1]; l++) {
      const int i = cell_idx[l];
      if (i <= last || i >= N) break;
      last = i;
    }
    gv[j] = (int32_t)(l - gp[j]);
  }
  int rc;
  int32_t *cell_d = nullptr, *gv_d = nullptr, *genes_d = nullptr, *row_d = nullptr;
  int64_t* gp_d = nullptr;
  double *cnt_d = nullptr, *ls_d = nullptr;
  if ((rc = ealloc(e, &S.F, (size_t)S.Npad * e->Kin)) || (rc = ealloc(e, &S.FT, (size_t)e->Kin * S.Npad)) ||
      (rc = ealloc(e, &S.X, (size_t)S.Npad * e->Q)) || (rc = ealloc(e, &cell_d, (size_t)nnz)) ||
      (rc = ealloc(e, &gv_d, (size_t)J)) || (rc = ealloc(e, &genes_d, (size_t)e->n_in)) ||
      (rc = ealloc(e, &row_d, (size_t)N)) || (rc = ealloc(e, &gp_d, (size_t)J + 1)) ||
      (rc = ealloc(e, &cnt_d, (size_t)nnz)) || (rc = ealloc(e, &ls_d, (size_t)N)))
    return rc;
  ENC_TRY(e, cudaMemcpyAsync(cell_d, cell_idx, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, e->stream));
  ENC_TRY(e, cudaMemcpyAsync(cnt_d, counts, sizeof(double) * nnz, cudaMemcpyHostToDevice, e->stream));
  ENC_TRY(e, cudaMemcpyAsync(gp_d, gp.data(), sizeof(int64_t) * (J + 1), cudaMemcpyHostToDevice, e->stream));
  ENC_TRY(e, cudaMemcpyAsync(gv_d, gv.data(), sizeof(int32_t) * J, cudaMemcpyHostToDevice, e->stream));
  ENC_TRY(e, cudaMemcpyAsync(genes_d, genes, sizeof(int32_t) * e->n_in, cudaMemcpyHostToDevice, e->stream));
  ENC_TRY(e, cudaMemcpyAsync(row_d, row_of.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice, e->stream));
  ENC_TRY(e, cudaMemcpyAsync(ls_d, ls, sizeof(double) * N, cudaMemcpyHostToDevice, e->stream));
  dim3 g(8, e->n_in);
  k_enc_features<<<g, 256, 0, e->stream>>>(e->n_in, genes_d, gp_d, gv_d, cell_d, cnt_d, ls_d, row_d, S.F, e->Kin,
                                           S.FT, S.Npad);
  ENC_LAUNCHED(e, "k_enc_features");
  ENC_TRY(e, cudaStreamSynchronize(e->stream));
  void* tmp[] = {cell_d, gv_d, genes_d, row_d, gp_d, cnt_d, ls_d};
  for (void* p : tmp) cudaFree(p);
  if (!bf16_map(&S.mapF, S.F, e->Kin, S.Npad) || !bf16_map(&S.mapFT, S.FT, S.Npad, e->Kin)) {
    e->err = "cuTensorMapEncodeTiled failed";
    return GPL_ERR_CUDA;
  }
  return GPL_OK;
}

int gpl_enc_set_targets(gpl_enc* e, const double* X) {
  if (!e || !X || e->set[0].N == 0) return GPL_ERR_ARG;
  gpl_enc::Set& S = e->set[0];
  const int N = S.N, Q = e->Q;
  std::vector<float> h((size_t)S.Npad * Q, 0.f);
  for (int r = 0; r < N; r++)
    for (int q = 0; q < Q; q++) h[(size_t)r * Q + q] = (float)X[S.cell_of_row[r] + (size_t)q * N];
  ENC_TRY(e, cudaMemcpyAsync(S.X, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, e->stream));
  ENC_TRY(e, cudaStreamSynchronize(e->stream));
  return GPL_OK;
}

int gpl_enc_n_params(const gpl_enc* e, int64_t* n) {
  if (!e || !n) return GPL_ERR_ARG;
  *n = (int64_t)e->H * e->n_in + e->H + (int64_t)e->H * e->H + e->H + 2LL * e->Q * e->H + 2 * e->Q;
  return GPL_OK;
}

// flat host layout: W1 [H][n_in], b1, W2 [H][H], b2, W3 [2Q][H], b3 (row-major)
static int copy_params(gpl_enc* e, float* host, bool to_host, bool grads) {
  const int H = e->H, Q = e->Q, n_in = e->n_in, Kin = e->Kin;
  float* base = grads ? e->gW1 : e->W1;
  if (to_host) {
    std::vector<float> d(e->n_par);
    ENC_TRY(e, cudaMemcpyAsync(d.data(), base, sizeof(float) * e->n_par, cudaMemcpyDeviceToHost, e->stream));
    ENC_TRY(e, cudaStreamSynchronize(e->stream));
    size_t o = 0;
    for (int r = 0; r < H; r++)
      for (int c = 0; c < n_in; c++) host[o++] = d[(size_t)r * Kin + c];
    for (size_t k = (size_t)H * Kin; k < e->n_par; k++) host[o++] = d[k];
  } else {
    std::vector<float> d(e->n_par, 0.f);
    size_t o = 0;
    for (int r = 0; r < H; r++)
      for (int c = 0; c < n_in; c++) d[(size_t)r * Kin + c] = host[o++];
    for (size_t k = (size_t)H * Kin; k < e->n_par; k++) d[k] = host[o++];
    ENC_TRY(e, cudaMemcpyAsync(base, d.data(), sizeof(float) * e->n_par, cudaMemcpyHostToDevice, e->stream));
    int rc = refresh_bf16(e);
    if (rc) return rc;
    ENC_TRY(e, cudaStreamSynchronize(e->stream));
  }
  (void)Q;
  return GPL_OK;
}

int gpl_enc_get_params(gpl_enc* e, float* p) { return (e && p) ? copy_params(e, p, true, false) : GPL_ERR_ARG; }
int gpl_enc_set_params(gpl_enc* e, const float* p) {
  return (e && p) ? copy_params(e, const_cast<float*>(p), false, false) : GPL_ERR_ARG;
}

int gpl_enc_grads(gpl_enc* e, int batch_index, double* loss, float* grads) {
  if (!e || !loss || !grads || e->set[0].N == 0) return GPL_ERR_ARG;
  const int r0 = batch_index * e->B;
  if (batch_index < 0 || r0 + e->B > e->set[0].Npad) return GPL_ERR_ARG;
  int rc;
  if ((rc = forward(e, 0, r0, e->B)) || (rc = backward(e, r0))) return rc;
  double s = 0.0;
  ENC_TRY(e, cudaMemcpyAsync(&s, e->loss_sum, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
  if ((rc = check_err(e))) return rc;
  *loss = s / e->B;
  return copy_params(e, grads, true, true);
}

int gpl_enc_train(gpl_enc* e, int epochs, double lr, uint64_t seed, double* loss_per_epoch) {
  if (!e || epochs < 0 || e->set[0].N < e->B) return GPL_ERR_ARG;
  cudaSetDevice(e->device);
  const int nb = e->set[0].N / e->B;  // whole batches of the (shuffled) training rows
  std::mt19937_64 rng(seed);
  std::vector<int> order(nb);
  std::vector<double> bl(nb);
  for (int ep = 0; ep < epochs; ep++) {
    for (int b = 0; b < nb; b++) order[b] = b;
    std::shuffle(order.begin(), order.end(), rng);
    double tot = 0.0;
    for (int k = 0; k < nb; k++) {
      const int r0 = order[k] * e->B;
      int rc;
      if ((rc = forward(e, 0, r0, e->B)) || (rc = backward(e, r0)) || (rc = adam_step(e, (float)lr))) return rc;
      double s = 0.0;
      ENC_TRY(e, cudaMemcpyAsync(&s, e->loss_sum, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
      ENC_TRY(e, cudaStreamSynchronize(e->stream));
      tot += s;
    }
    if (loss_per_epoch) loss_per_epoch[ep] = tot / ((double)nb * e->B);
  }
  return check_err(e);
}

int gpl_enc_predict(gpl_enc* e, int which, double* mean, double* logvar) {
  if (!e || which < 0 || which > 1 || e->set[which].N == 0 || (!mean && !logvar)) return GPL_ERR_ARG;
  cudaSetDevice(e->device);
  gpl_enc::Set& S = e->set[which];
  const int N = S.N, Q = e->Q, B = e->B;
  std::vector<float> o((size_t)B * 128);
  for (int r0 = 0; r0 < N; r0 += B) {
    const int rows = std::min(B, N - r0);
    int rc = forward(e, which, r0, rows);
    if (rc) return rc;
    ENC_TRY(e, cudaMemcpyAsync(o.data(), e->out, sizeof(float) * (size_t)B * 128, cudaMemcpyDeviceToHost, e->stream));
    ENC_TRY(e, cudaStreamSynchronize(e->stream));
    for (int r = 0; r < rows; r++) {
      const int i = S.cell_of_row[r0 + r];
      for (int q = 0; q < Q; q++) {
        if (mean) mean[i + (size_t)q * N] = o[(size_t)r * 128 + q];
        if (logvar) logvar[i + (size_t)q * N] = o[(size_t)r * 128 + Q + q];
      }
    }
  }
  return check_err(e);
}

int gpl_enc_launch_count(const gpl_enc* e, int64_t* n) {
  if (!e || !n) return GPL_ERR_ARG;
  *n = e->launches;
  return GPL_OK;
}

}  // extern "C"
