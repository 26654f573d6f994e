// On-device L-BFGS (replaces LBFGS ggplvm.cu:865-934, lbfgs util_cuda.cu:187-232, Downdate
// ggplvm.cu:818-859, getBetaFromTildeBeta :394-402).
//
// The reference runs the two-loop recursion in a single GPU thread (~40 D-length passes,
// D = N + p + N*Q + M*Q + rhoflag). Here every pass is a grid-wide kernel: dot products are
// two-stage deterministic reductions (fixed grid, then one block summing the partials in
// order) whose scalars stay in device memory, so the whole update is a fixed kernel
// sequence with no host round trip. HBM-bound: ~4 * m * D * 8 bytes per step.
#include "gpl_internal.cuh"

namespace gpl {

namespace {
constexpr int kDotBlocks = 296;  // 2 x 148 SMs
constexpr int kDotThreads = 256;
// lb_work slots
constexpr int kA = 0;         // a[10]
constexpr int kNum = 16, kDen = 17;
}  // namespace

// partial sums of x1.y1 and x2.y2 (x2/y2 may be null)
__global__ void __launch_bounds__(kDotThreads) k_dot2_partial(int64_t n, const double* __restrict__ x1,
                                                              const double* __restrict__ y1,
                                                              const double* __restrict__ x2,
                                                              const double* __restrict__ y2, double* __restrict__ part) {
  __shared__ double sh[32];
  double s1 = 0.0, s2 = 0.0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    s1 += x1[k] * y1[k];
    if (x2) s2 += x2[k] * y2[k];
  }
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1;
    part[2 * blockIdx.x + 1] = s2;
  }
}

// sums the partials in block order into out[0], out[1]; if a_slot >= 0 also stores out0/out1 there
__global__ void k_dot2_final(int nblk, const double* __restrict__ part, double* __restrict__ w, int o0, int o1,
                             int a_slot) {
  __shared__ double sh[32];
  double s1 = 0.0, s2 = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    s1 += part[2 * b];
    s2 += part[2 * b + 1];
  }
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    w[o0] = s1;
    w[o1] = s2;
    if (a_slot >= 0) w[a_slot] = s1 / s2;
  }
}

// y += sign * (w[s] ) * x    (scalar read on device)
__global__ void k_axpy_dev(int64_t n, double* __restrict__ y, const double* __restrict__ x,
                           const double* __restrict__ w, int s, double sign) {
  const double a = w[s];
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    y[k] += sign * a * x[k];
}

// z = (num/den) q
__global__ void k_scale_ratio(int64_t n, double* __restrict__ z, const double* __restrict__ q,
                              const double* __restrict__ w) {
  const double g = w[kNum] / w[kDen];
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    z[k] = g * q[k];
}

// z += S_ii (a_ii - num/den)
__global__ void k_axpy_second(int64_t n, double* __restrict__ z, const double* __restrict__ S,
                              const double* __restrict__ w, int ii) {
  const double f = w[kA + ii] - w[kNum] / w[kDen];
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    z[k] += S[k] * f;
}

__global__ void k_first_step(int64_t n, const double* __restrict__ g, double* __restrict__ ss,
                             double* __restrict__ g0) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    double s = -g[k] / 100000.0;
    if (s > 1.0) s = 1.0;
    if (s < (-1.0)) s = -1.0;
    ss[k] = s;
    g0[k] = g[k];
  }
}

__global__ void k_ydiff(int64_t n, const double* __restrict__ g, double* __restrict__ g0, double* __restrict__ y,
                        double* __restrict__ q) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    y[k] = g[k] - g0[k];
    g0[k] = g[k];
    q[k] = g[k];
  }
}

__global__ void k_clip_neg(int64_t n, double* __restrict__ z) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    double v = z[k];
    if (v > 1.0) v = 1.0;
    if (v < (-1.0)) v = -1.0;
    z[k] = -v;
  }
}

// Applies scale * ss to the parameters from `base` (the backup when downdating, the current
// values otherwise, which are first copied to the backup), and records scale*ss in SS.
__global__ void k_apply_step(int N, int p, int Q, int M, int64_t tot, double scale, int backup,
                             const double* __restrict__ ss, double* __restrict__ Omega, double* __restrict__ delta,
                             double* __restrict__ X, double* __restrict__ T, double* __restrict__ SScol) {
  const int64_t nx = (int64_t)N * Q, nt = (int64_t)M * Q;
  const int64_t n = (int64_t)N + p + nx + nt;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double s = scale * ss[k];
    if (k < N) {
      double base;
      if (backup) { base = Omega[k]; Omega[k + N] = base; } else base = Omega[k + N];
      double o = exp(log(base) - s);
      if (o > 1000.) o = 1000.;
      if (o < .001) o = .001;
      Omega[k] = o;
    } else if (k < N + p) {
      const int d = (int)(k - N);
      double base;
      if (backup) { base = delta[d]; delta[d + p] = base; } else base = delta[d + p];
      delta[d] = exp(log(base) - s);
    } else if (k < N + p + nx) {
      const int64_t e = k - N - p;
      double base;
      if (backup) { base = X[e]; X[e + nx] = base; } else base = X[e + nx];
      X[e] = base - s;
    } else {
      const int64_t e = k - N - p - nx;
      double base;
      if (backup) { base = T[e]; T[e + nt] = base; } else base = T[e + nt];
      T[e] = base - s;
    }
  }
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < tot; k += (int64_t)gridDim.x * blockDim.x)
    SScol[k] = scale * ss[k];
}

// rho_0 step and the renormalisation of rho_1.. to mean 10 (mscale_d, util_cuda.cu:546-555)
__global__ void k_rho_step(int Q, int64_t irho, double scale, int backup, int rhoflag, const double* __restrict__ ss,
                           double* __restrict__ rho) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double base;
  if (backup) { base = rho[0]; rho[Q] = base; } else base = rho[Q];
  rho[0] = exp(log(base) - scale * ss[irho] * ((double)rhoflag));
  double mh = 0.0;
  for (int i = 1; i < Q; i++) mh += rho[i];
  mh /= (double)(Q - 1);
  for (int i = 1; i < Q; i++) rho[i] *= 10.0 / mh;
}

static int dot2(Ctx* c, int64_t n, const double* x1, const double* y1, const double* x2, const double* y2, int o0,
                int o1, int a_slot) {
  k_dot2_partial<<<kDotBlocks, kDotThreads, 0, c->stream>>>(n, x1, y1, x2, y2, c->red);
  GPL_LAUNCHED(c, "k_dot2_partial");
  k_dot2_final<<<1, 256, 0, c->stream>>>(kDotBlocks, c->red, c->lb_work, o0, o1, a_slot);
  GPL_LAUNCHED(c, "k_dot2_final");
  return GPL_OK;
}

static int apply(Ctx* c, int itr, double scale, int backup, int rhoflag) {
  const int64_t tot = tot_len(c, rhoflag);
  const int ptp1 = itr % kHist;
  k_apply_step<<<kDotBlocks * 2, 256, 0, c->stream>>>(c->N, c->p, c->Q, c->M, tot, scale, backup, c->ss, c->Omega,
                                                     c->delta, c->X, c->T, c->SS + (size_t)ptp1 * tot);
  GPL_LAUNCHED(c, "k_apply_step");
  k_rho_step<<<1, 32, 0, c->stream>>>(c->Q, tot_len(c, 0), scale, backup, rhoflag, c->ss, c->rho);
  GPL_LAUNCHED(c, "k_rho_step");
  return GPL_OK;
}

int launch_lbfgs_update(Ctx* c, int itr, int rhoflag) {
  ProfScope ps(c, "lbfgs");
  const int64_t tot = tot_len(c, rhoflag);
  const int m = kHist;
  const dim3 g(kDotBlocks * 2), b(256);
  if (itr == 0) {
    k_first_step<<<g, b, 0, c->stream>>>(tot, c->grad, c->ss, c->grad0);
    GPL_LAUNCHED(c, "k_first_step");
  } else {
    const int pt = (itr - 1) % m;
    double* q = c->scratch;  // tot doubles of work space
    k_ydiff<<<g, b, 0, c->stream>>>(tot, c->grad, c->grad0, c->XX + (size_t)pt * tot, q);
    GPL_LAUNCHED(c, "k_ydiff");
    const int lo = itr > m ? pt - m + 1 : 0;
    for (int i = pt; i >= lo; i--) {
      const int ii = (i + m) % m;
      const double* S = c->SS + (size_t)ii * tot;
      const double* Y = c->XX + (size_t)ii * tot;
      int rc = dot2(c, tot, S, q, S, Y, kNum, kDen, kA + ii);
      if (rc) return rc;
      k_axpy_dev<<<g, b, 0, c->stream>>>(tot, q, Y, c->lb_work, kA + ii, -1.0);
      GPL_LAUNCHED(c, "k_axpy_dev");
    }
    {
      const double* S = c->SS + (size_t)pt * tot;
      const double* Y = c->XX + (size_t)pt * tot;
      int rc = dot2(c, tot, S, Y, Y, Y, kNum, kDen, -1);
      if (rc) return rc;
      k_scale_ratio<<<g, b, 0, c->stream>>>(tot, c->ss, q, c->lb_work);
      GPL_LAUNCHED(c, "k_scale_ratio");
    }
    for (int i = lo; i <= pt; i++) {
      const int ii = (i + m) % m;
      const double* S = c->SS + (size_t)ii * tot;
      const double* Y = c->XX + (size_t)ii * tot;
      int rc = dot2(c, tot, Y, c->ss, S, Y, kNum, kDen, -1);
      if (rc) return rc;
      k_axpy_second<<<g, b, 0, c->stream>>>(tot, c->ss, S, c->lb_work, ii);
      GPL_LAUNCHED(c, "k_axpy_second");
    }
    k_clip_neg<<<g, b, 0, c->stream>>>(tot, c->ss);
    GPL_LAUNCHED(c, "k_clip_neg");
  }
  return apply(c, itr, 1.0, 1, rhoflag);
}

int launch_downdate(Ctx* c, int itr, double r, int rhoflag) {
  ProfScope ps(c, "downdate");
  return apply(c, itr, r, 0, rhoflag);
}

// Beta = tBeta + zeta (getBetaFromTildeBeta): zeta is 0 in the fit driver, the DE driver's
// zeta in the variance-component driver
__global__ void k_add_zeta(int P, int64_t n, const double* __restrict__ tB, const double* __restrict__ zeta,
                           double* __restrict__ B) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) B[e] = tB[e] + zeta[e % P];
}

int launch_beta_from_tilde(Ctx* c) {
  if (!c->de) {
    GPL_TRY(c, cudaMemcpyAsync(c->Beta, c->tBeta, sizeof(double) * (size_t)c->P * c->J, cudaMemcpyDeviceToDevice,
                               c->stream));
    return GPL_OK;
  }
  const int64_t n = (int64_t)c->P * c->J;
  k_add_zeta<<<div_up(n, 256), 256, 0, c->stream>>>(c->P, n, c->tBeta, c->zeta, c->Beta);
  GPL_LAUNCHED(c, "k_add_zeta");
  return GPL_OK;
}

}  // namespace gpl
