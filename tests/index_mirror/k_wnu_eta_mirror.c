/*
 * CPU mirror of the memory indexing of the linear predictor, the W / nu pass, Z^T u, HK and
 * the group sums: k_eta_dmma<MT> and k_level_sums (gaspacho2_b200/csrc/k_dgemm.cu), k_w_nu and
 * k_w_nu_counts (gaspacho2_b200/csrc/k_gemm.cu), k_zt_u<MODE>, k_hk and k_group_sums_dmma<MODE>
 * (gaspacho2_b200/csrc/k_dgen.cu).
 *
 * The kernels' own index expressions are replayed for every block and thread of a launch
 * (256 threads; lane = 4 g + t as in the DMMA fragments), over a sweep of sizes: cell counts
 * around the tile heights and the padded column length (ldN = N rounded up to 32), gene counts
 * around the tile width and odd ones, dense-column counts with ragged last slices, with and
 * without cell groups, and persistent grids smaller than the tile count. Each global index is
 * checked against its allocation (the sizes gaspacho2_b200/csrc/gpl_api.cu allocates), each
 * shared index against the launch's dynamic shared memory, including the source of a
 * zero-byte (zero-fill) cp.async; outputs are counted: every (cell, gene) of the predictor and
 * of W, nu and W's group-ordered copy is written exactly once, every persistent tile visited
 * once.
 *
 *   k_wnu_eta_mirror        prints "ok eta4 <sizes>", "ok eta2 <sizes>", "ok levels <sizes>",
 *                           "ok w_nu <sizes>", "ok counts <sizes>", "ok zt_u <sizes>",
 *                           "ok hk <sizes>", "ok group_sums <sizes>" and exits 0, or lists the
 *                           first faults and exits 1.
 *   k_wnu_eta_mirror plant  the same with the level sums' rows left unpadded (J instead of J
 *                           rounded up to even): must fail on an odd gene count.
 *   k_wnu_eta_mirror plant-odd  Z^T u alone with its cell ranges left at ceil(N / S) cells
 *                           (not rounded up to even): must fail on a misaligned 16-byte copy.
 *
 * Compiled and run by tests/test_index_mirror.py. Keep it in step with the two kernels.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define BN 128
#define BK 16
#define SBT (BK + 4)
#define NT 256
#define WNU_GENES 4

static long faults = 0;
static void fault(const char* what, const char* ctx, long idx, long lim) {
  if (faults < 20) fprintf(stderr, "%s: %s index %ld outside [0, %ld)\n", ctx, what, idx, lim);
  faults++;
}
#define CHK(what, i, lim) do { long i_ = (long)(i), l_ = (long)(lim); if (i_ < 0 || i_ >= l_) fault(what, ctx, i_, l_); } while (0)

static int imin(int a, int b) { return a < b ? a : b; }
static int div_up(int a, int b) { return (a + b - 1) / b; }
static int ld_cells(int N) { return (N + 31) / 32 * 32; }
static int plant_unpadded = 0; /* "plant": the level sums' rows left at J (unpadded) */
static int plant_odd = 0;      /* "plant-odd": Z^T u's cell ranges not rounded to even */
static int lvt_ld(int J) { return plant_unpadded ? J : J + (J & 1); }

/* k_eta_dmma<MT>: loads, fragment reads, level sums and stores of every tile a grid of
 * `grid` persistent CTAs walks. */
static void mirror_eta(int MT, int N, int J, int n_d, int n_grp, int grid) {
  char ctx[96];
  snprintf(ctx, sizeof ctx, "eta%d N=%d J=%d n_d=%d n_grp=%d grid=%d", MT, N, J, n_d, n_grp, grid);
  const int ldN = ld_cells(N), P = n_d + 3 + (n_grp ? 4 : 0), ldJ = lvt_ld(J);
  const int BMt = MT * 32, SAt = BMt + 4;
  const int KP = (n_d + BK - 1) / BK * BK, nsl = KP / BK;
  /* shared memory in doubles: As [3][BK][SAt], Bs [3][BN][SBT], then KP ints */
  const long as_n = 3L * BK * SAt, bs_n = 3L * BN * SBT;
  const long D_n = (long)n_d * ldN, B_n = (long)P * J, lvt_n = (long)n_grp * ldJ, out_n = (long)ldN * J;
  int* dcol = malloc(sizeof(int) * (n_d ? n_d : 1));
  for (int k = 0; k < n_d; k++) dcol[k] = 1 + (k * 7) % (P - 1); /* any column of the P model columns */
  int* gid = malloc(sizeof(int) * N);
  for (int i = 0; i < N; i++) gid[i] = n_grp ? (i * 5 + 1) % n_grp : 0;
  int* dcs = malloc(sizeof(int) * KP);
  for (int k = 0; k < KP; k++) dcs[k] = k < n_d ? dcol[k] : 0;
  unsigned char* written = calloc((size_t)out_n, 1);
  const int tm = (N + BMt - 1) / BMt, tn = (J + BN - 1) / BN, tiles = tm * tn;
  int* visits = calloc((size_t)tiles, sizeof(int));

  for (int b = 0; b < grid; b++) {
    /* the persistent walk and the next tile's prefetch */
    for (int w = b; w < tiles; w += grid) {
      visits[w]++;
      const int m0 = (w / tn) * BMt, j0 = (w % tn) * BN;
      for (int s = 0; s < nsl; s++) {
        const int kb = s * BK;
        for (int st = 0; st < 3; st += 2) { /* any stage: check stages 0 and 2 */
          for (int tid = 0; tid < NT; tid++) {
            for (int r = 0; r < (BMt * BK / 2) / NT; r++) {
              const int ch = tid + r * NT;
              const int k = ch / (BMt / 2), part = ch % (BMt / 2);
              const int col = kb + k, i = m0 + part * 2;
              const long src = (long)imin(col, n_d - 1) * ldN + imin(i, ldN - 2);
              CHK("A source", src, D_n);
              CHK("A source + 1", src + 1, D_n);
              const long dst = (long)st * BK * SAt + (long)k * SAt + part * 2;
              CHK("A stage", dst, as_n);
              CHK("A stage + 1", dst + 1, as_n);
            }
            for (int r = 0; r < (BN * BK) / NT; r++) {
              const int ch = tid + r * NT;
              const int n = ch >> 4, k = ch & 15;
              const int col = kb + k, j = j0 + n;
              CHK("dcol slot", col, KP);
              const long src = (long)dcs[col] + (long)imin(j, J - 1) * P;
              CHK("B source", src, B_n);
              CHK("B stage", (long)st * BN * SBT + (long)n * SBT + k, bs_n);
            }
          }
        }
      }
      /* fragment reads of one stage (warp_slice_eta), every k4 step */
      for (int tid = 0; tid < NT; tid++) {
        const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3, wm = warp >> 2, wn = warp & 3;
        for (int kk = 0; kk < BK / 4; kk++) {
          for (int mt = 0; mt < MT; mt++) {
            const long a = (long)(kk * 4 + t) * SAt + wm * (MT * 16) + g + mt * 16;
            CHK("A fragment", a, (long)BK * SAt);
            CHK("A fragment + 8", a + 8, (long)BK * SAt);
          }
          for (int nt = 0; nt < 4; nt++) CHK("B fragment", (long)(wn * 32 + nt * 8 + g) * SBT + kk * 4 + t, (long)BN * SBT);
        }
        /* level sums, then the stores */
        for (int mt = 0; mt < MT; mt++)
          for (int h = 0; h < 2; h++) {
            if (n_grp > 0) {
              const int ic = imin(m0 + wm * (MT * 16) + mt * 16 + g + h * 8, N - 1);
              CHK("gid", ic, N);
              const long lg = (long)gid[ic] * ldJ;
              for (int nt = 0; nt < 4; nt++) {
                const int j = imin(j0 + wn * 32 + nt * 8 + 2 * t, ldJ - 2);
                CHK("level sum", lg + j, lvt_n);
                CHK("level sum + 1", lg + j + 1, lvt_n);
                if ((lg + j) % 2) fault("level sum alignment", ctx, lg + j, 2);
              }
            }
            const int i = m0 + wm * (MT * 16) + mt * 16 + g + h * 8;
            if (i >= N) continue;
            for (int nt = 0; nt < 4; nt++)
              for (int e = 0; e < 2; e++) {
                const int j = j0 + wn * 32 + nt * 8 + 2 * t + e;
                if (j < J) {
                  const long o = (long)j * ldN + i;
                  CHK("out", o, out_n);
                  if (o >= 0 && o < out_n) written[o]++;
                }
              }
          }
      }
      const int w2 = w + grid;
      if (w2 < tiles) {
        const int m1 = (w2 / tn) * BMt, j1 = (w2 % tn) * BN;
        CHK("next tile row", m1, tm * BMt);
        CHK("next tile column", j1, tn * BN);
      }
    }
  }
  for (int w = 0; w < tiles; w++)
    if (visits[w] != 1) fault("tile visit count", ctx, visits[w], 1);
  for (int j = 0; j < J; j++)
    for (int i = 0; i < N; i++)
      if (written[(long)j * ldN + i] != 1) {
        fault("output write count", ctx, written[(long)j * ldN + i], 1);
        j = J;
        break;
      }
  free(dcol);
  free(gid);
  free(dcs);
  free(written);
  free(visits);
}

/* k_level_sums: one thread per (group, gene), Lv[g * ldJ + j]. */
static void mirror_levels(int J, int n_grp) {
  char ctx[64];
  snprintf(ctx, sizeof ctx, "levels J=%d n_grp=%d", J, n_grp);
  const int ldJ = lvt_ld(J);
  const long n = (long)J * n_grp, lvt_n = (long)n_grp * ldJ;
  unsigned char* written = calloc((size_t)(lvt_n ? lvt_n : 1), 1);
  const long blocks = (n + 255) / 256;
  for (long b = 0; b < blocks; b++)
    for (int tx = 0; tx < 256; tx++) {
      const long e = b * 256 + tx;
      if (e >= n) continue;
      const int g = (int)(e / J), j = (int)(e - (long)g * J);
      const long o = (long)g * ldJ + j;
      CHK("Lv", o, lvt_n);
      if (o >= 0 && o < lvt_n) written[o]++;
    }
  for (int g = 0; g < n_grp; g++)
    for (int j = 0; j < J; j++)
      if (written[(long)g * ldJ + j] != 1) fault("Lv write count", ctx, written[(long)g * ldJ + j], 1);
  free(written);
}

/* k_w_nu over the launcher's 2-D grid (cell pairs x gene quads, the y extent capped at
 * 65535 so that larger gene counts take a stride); gridy_cap lets a small case take it. */
static void mirror_w_nu(int N, int J, int groups, int gridy_cap) {
  char ctx[80];
  snprintf(ctx, sizeof ctx, "w_nu N=%d J=%d groups=%d ycap=%d", N, J, groups, gridy_cap);
  const int ldN = ld_cells(N);
  const long E_n = (long)ldN * J, W_n = (long)ldN * (J + 1), Nu_n = (long)ldN * J, Wg_n = (long)ldN * J;
  int* gpos = malloc(sizeof(int) * N);
  for (int k = 0; k < N; k++) gpos[k] = (int)(((long)k * 7919) % N); /* a permutation when N is not a multiple of 7919 */
  unsigned char* wr_w = calloc((size_t)W_n, 1);
  unsigned char* wr_nu = calloc((size_t)Nu_n, 1);
  unsigned char* wr_g = calloc((size_t)Wg_n, 1);
  const int gx = div_up(N, 512), gy = imin(div_up(J, WNU_GENES), gridy_cap);
  for (int by = 0; by < gy; by++)
    for (int bx = 0; bx < gx; bx++)
      for (int tx = 0; tx < 256; tx++) {
        const int i = 2 * (bx * 256 + tx);
        if (i >= N) continue;
        const int two = i + 1 < N;
        CHK("ls / e0 / gpos", i, N);
        CHK("cell factors", i, 3L * ldN);
        if (two) CHK("ls / e0 / gpos + 1", i + 1, N);
        const int p0 = groups ? gpos[i] : 0, p1 = groups && two ? gpos[i + 1] : 0;
        for (int jb = by * WNU_GENES; jb < J; jb += gy * WNU_GENES)
          for (int u = 0; u < WNU_GENES; u++) {
            const int j = jb + u;
            if (j >= J) break;
            const long o = (long)j * ldN + i;
            CHK("eta pair", o, E_n);
            CHK("eta pair + 1", o + 1, E_n);
            if (o % 2) fault("pair alignment", ctx, o, 2);
            if (two) {
              CHK("W pair", o + 1, W_n);
              CHK("Nu pair", o + 1, Nu_n);
              wr_w[o]++, wr_w[o + 1]++, wr_nu[o]++, wr_nu[o + 1]++;
            } else {
              CHK("W", o, W_n);
              CHK("Nu", o, Nu_n);
              wr_w[o]++, wr_nu[o]++;
            }
            if (groups) {
              const long q0 = (long)j * ldN + p0;
              CHK("Wg", q0, Wg_n);
              wr_g[q0]++;
              if (two) {
                const long q1 = (long)j * ldN + p1;
                CHK("Wg", q1, Wg_n);
                wr_g[q1]++;
              }
            }
          }
      }
  for (int j = 0; j < J; j++)
    for (int i = 0; i < N; i++) {
      const long o = (long)j * ldN + i;
      if (wr_w[o] != 1 || wr_nu[o] != 1 || (groups && wr_g[o] != 1)) {
        fault("W / nu / Wg write count", ctx, o, 1);
        j = J;
        break;
      }
    }
  free(gpos);
  free(wr_w);
  free(wr_nu);
  free(wr_g);
}

/* k_w_nu_counts: one block of 256 threads per gene, kCountsIlp entries per thread per round. */
static void mirror_counts(int N, int J, int dens) {
  char ctx[64];
  snprintf(ctx, sizeof ctx, "counts N=%d J=%d dens=%d", N, J, dens);
  const int ldN = ld_cells(N), ILP = 4;
  /* CSR with a matched prefix of increasing cells per gene: every dens-th cell */
  long* gptr = malloc(sizeof(long) * (J + 1));
  int* gvalid = malloc(sizeof(int) * J);
  gptr[0] = 0;
  for (int j = 0; j < J; j++) {
    const int cnt = (N + dens - 1 - (j % dens)) / dens;
    gvalid[j] = cnt > 0 ? cnt : 0;
    gptr[j + 1] = gptr[j] + gvalid[j] + (j % 3); /* unmatched tail entries after the prefix */
  }
  const long L = gptr[J];
  int* cell = malloc(sizeof(int) * (L ? L : 1));
  for (int j = 0; j < J; j++) {
    long l = gptr[j];
    for (int i = j % dens; i < N; i += dens) cell[l++] = i;
    for (; l < gptr[j + 1]; l++) cell[l] = 0; /* past the prefix: never read */
  }
  unsigned char* wr = calloc((size_t)ldN * J, 1);
  for (int j = 0; j < J; j++)
    for (int tx = 0; tx < 256; tx++) {
      const long b = gptr[j], e = gptr[j] + gvalid[j];
      for (long l0 = b + tx; l0 < e; l0 += (long)ILP * 256)
        for (int u = 0; u < ILP; u++) {
          const long l = l0 + (long)u * 256;
          if (l >= e) continue;
          CHK("CSR entry", l, L);
          const int i = cell[l];
          CHK("cell", i, N);
          CHK("eta / nu", (long)j * ldN + i, (long)ldN * J);
          CHK("cell factors", 2L * ldN + i, 3L * ldN);
          wr[(long)j * ldN + i]++;
        }
    }
  for (int j = 0; j < J; j++)
    for (long l = gptr[j]; l < gptr[j] + gvalid[j]; l++)
      if (wr[(long)j * ldN + cell[l]] != 1) {
        fault("matched count write count", ctx, wr[(long)j * ldN + cell[l]], 1);
        break;
      }
  free(gptr);
  free(gvalid);
  free(cell);
  free(wr);
}

/* k_zt_u<MODE>: grid (1, gene tiles, S cell ranges); three stages of 16-cell slices. */
#define ZT_BK 16
#define ZT_S (ZT_BK + 4)
#define ZT_BM 144
#define ZT_BN 128
#define ZT_STAGE (ZT_BM * ZT_S + 2 * ZT_BN * ZT_S + 2 * ZT_BK)
static void mirror_zt_u(int mode, int N, int J, int m, int S) {
  char ctx[80];
  snprintf(ctx, sizeof ctx, "zt_u mode=%d N=%d J=%d n_d=%d S=%d", mode, N, J, m, S);
  const int ldN = ld_cells(N), n = J;
  int per = (N + S - 1) / S;
  if (!plant_odd) per += per & 1;
  const long D_n = (long)m * ldN, U_n = mode == 2 ? (long)N : (long)ldN * J, W_n = (long)ldN * (J + 1);
  const long R_n = N, part_n = (long)S * m * n, sm_n = 3L * ZT_STAGE;
  const int tiles = (J + ZT_BN - 1) / ZT_BN;
  unsigned char* wr = calloc((size_t)part_n, 1);
  unsigned char* cellhit = calloc((size_t)N, 1);
  for (int z = 0; z < S; z++) {
    const int kbeg = imin(N, z * per), kend = imin(N, (z + 1) * per);
    const int nsl = kend > kbeg ? (kend - kbeg + ZT_BK - 1) / ZT_BK : 0;
    if (kbeg < kend && kbeg % 2) fault("odd range start", ctx, kbeg, 2); /* an empty range loads nothing */
    for (int by = 0; by < tiles; by++) {
      const int n0 = by * ZT_BN;
      for (int s = 0; s < nsl; s++) {
        const int st = s % 3, k0 = kbeg + s * ZT_BK;
        const long As = (long)st * ZT_STAGE, Ws = As + ZT_BM * ZT_S, Us = Ws + ZT_BN * ZT_S, Rs = Us + ZT_BN * ZT_S,
                   Vs = Rs + ZT_BK;
        for (int tid = 0; tid < 256; tid++) {
          for (int ch = tid; ch < ZT_BM * (ZT_BK / 2); ch += 256) {
            const int r = ch >> 3, kc = (ch & 7) * 2, k = k0 + kc;
            const int nb = (r < m && k < kend) ? (k + 1 < kend ? 16 : 8) : 0;
            const long src = (long)imin(r, m - 1) * ldN + imin(k, ldN - 2);
            CHK("D", src, D_n);
            CHK("D + 1", src + 1, D_n);
            if (src % 2) fault("D alignment", ctx, src, 2);
            CHK("A stage", As + r * ZT_S + kc + 1, Ws);
            if ((As + r * ZT_S + kc) % 2) fault("A stage alignment", ctx, As + r * ZT_S + kc, 2);
            if (nb && by == 0 && r == 0) {
              cellhit[k]++;
              if (nb == 16) cellhit[k + 1]++;
            }
          }
          for (int q = 0; q < (ZT_BN * (ZT_BK / 2)) / 256; q++) {
            const int ch = tid + q * 256;
            const int cc = ch >> 3, kc = (ch & 7) * 2, k = k0 + kc;
            const long src = (long)imin(n0 + cc, n - 1) * ldN + imin(k, ldN - 2);
            if (src % 2) fault("W / u alignment", ctx, src, 2);
            if (mode != 1) CHK("W", src + 1, W_n);
            if (mode != 2) CHK("u", src + 1, U_n);
            CHK("W stage", Ws + cc * ZT_S + kc + 1, Us);
            CHK("u stage", Us + cc * ZT_S + kc + 1, Rs);
          }
          if (tid < ZT_BK) {
            const int k = k0 + tid;
            if (mode != 1) CHK("1/Omega", imin(k, N - 1), R_n);
            if (mode == 2) CHK("per-cell u", imin(k, N - 1), U_n);
            CHK("1/Omega stage", Rs + tid, Vs);
            CHK("per-cell u stage", Vs + tid, (long)(st + 1) * ZT_STAGE);
          }
          /* fragment reads of this stage */
          const int wn = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
          for (int k4 = 0; k4 < ZT_BK / 4; k4++) {
            const int kk = k4 * 4 + t;
            for (int x = 0; x < 9; x++) {
              CHK("A fragment", As + (x * 16 + g) * ZT_S + kk, Ws);
              CHK("A fragment + 8", As + (x * 16 + g + 8) * ZT_S + kk, Ws);
            }
            for (int y = 0; y < 2; y++) {
              const long e = (long)(wn * 16 + y * 8 + g) * ZT_S + kk;
              CHK("W fragment", Ws + e, Us);
              CHK("u fragment", Us + e, Rs);
            }
            CHK("1/Omega fragment", Rs + kk, Vs);
            CHK("stage end", Vs + kk, sm_n);
          }
        }
      }
      /* the partial sums */
      for (int tid = 0; tid < 256; tid++) {
        const int wn = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
        for (int x = 0; x < 9; x++)
          for (int h = 0; h < 2; h++) {
            const int r = x * 16 + g + 8 * h;
            if (r >= m) continue;
            for (int y = 0; y < 2; y++)
              for (int e = 0; e < 2; e++) {
                const int cc = n0 + wn * 16 + y * 8 + 2 * t + e;
                if (cc >= n) continue;
                const long o = ((long)z * m + r) * n + cc;
                CHK("part", o, part_n);
                if (o >= 0 && o < part_n) wr[o]++;
              }
          }
      }
    }
  }
  for (long o = 0; o < part_n; o++)
    if (wr[o] != 1) {
      fault("partial write count", ctx, wr[o], 1);
      break;
    }
  for (int k = 0; k < N; k++)
    if (cellhit[k] != 1) {
      fault("cell load count", ctx, cellhit[k], 1);
      break;
    }
  free(wr);
  free(cellhit);
}

/* k_hk: grid z = the 128-slot tiles of every group (gpl_api.cu's tile list), four stages of
 * 16-gene slices; groups of the given sizes, the cells in group order a permutation. */
#define HK_BK 16
#define HK_SA 148
#define HK_SB 132
#define HK_STAGE (HK_BK * HK_SA + HK_BK * HK_SB)
static void mirror_hk(int n_d, int J, const int* sizes, int n_grp) {
  char ctx[80];
  int N = 0;
  for (int q = 0; q < n_grp; q++) N += sizes[q];
  snprintf(ctx, sizeof ctx, "hk n_d=%d J=%d n_grp=%d N=%d", n_d, J, n_grp, N);
  if (N == 0) return;
  const int ld = n_d + 1, ldN = ld_cells(N);
  const long tab_n = (long)J * n_grp * ld, Wg_n = (long)ldN * J, HK_n = (long)ldN * ld;
  const long sm_n = 4L * HK_STAGE + 128;
  int* gstart = malloc(sizeof(int) * (n_grp + 1));
  gstart[0] = 0;
  for (int q = 0; q < n_grp; q++) gstart[q + 1] = gstart[q] + sizes[q];
  int* order = malloc(sizeof(int) * N);
  for (int k = 0; k < N; k++) order[k] = (int)(((long)k * 7919) % N);
  int ntiles = 0;
  for (int q = 0; q < n_grp; q++) ntiles += (sizes[q] + 127) / 128;
  int* tg = malloc(sizeof(int) * (ntiles ? ntiles : 1));
  int* tcell = malloc(sizeof(int) * 128 * (ntiles ? ntiles : 1));
  int* tpos = malloc(sizeof(int) * 128 * (ntiles ? ntiles : 1));
  int nt = 0;
  for (int q = 0; q < n_grp; q++)
    for (int r0 = 0; r0 < sizes[q]; r0 += 128, nt++) {
      tg[nt] = q;
      for (int c = 0; c < 128; c++) {
        const int in = r0 + c < sizes[q];
        tcell[nt * 128 + c] = in ? order[gstart[q] + r0 + c] : -1;
        tpos[nt * 128 + c] = in ? gstart[q] + r0 + c : -1;
      }
    }
  unsigned char* wr = calloc((size_t)HK_n, 1);
  const int nsl = (J + HK_BK - 1) / HK_BK;
  for (int z = 0; z < ntiles; z++) {
    const int grp = tg[z];
    CHK("group", grp, n_grp);
    for (int tid = 0; tid < 256; tid++) {
      const int myq = tpos[z * 128 + (tid & 127)];
      if (myq >= 0) CHK("1/Omega slot", myq, N);
      if (tid < 128) CHK("1/Omega stage", 4L * HK_STAGE + tid, sm_n);
      for (int s = 0; s < nsl; s++) {
        const int st = s % 4, k0 = s * HK_BK;
        const long As = (long)st * HK_STAGE, Bs = As + HK_BK * HK_SA;
        for (int e = tid; e < HK_BK * 144; e += 256) {
          const int k = e / 144, r = e - k * 144, j = k0 + k;
          CHK("table", ((long)imin(j, J - 1) * n_grp + grp) * ld + imin(r, ld - 1), tab_n);
          CHK("table stage", As + (long)k * HK_SA + r, Bs);
        }
        for (int q = 0; q < (HK_BK * 128) / 256; q++) {
          const int k = (tid >> 7) + 2 * q, j = k0 + k;
          CHK("W group order", (long)imin(j, J - 1) * ldN + (myq > 0 ? myq : 0), Wg_n);
          CHK("W stage", Bs + (long)k * HK_SB + (tid & 127), (long)(st + 1) * HK_STAGE);
        }
        const int wn = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
        for (int k4 = 0; k4 < HK_BK / 4; k4++) {
          const int kk = k4 * 4 + t;
          for (int x = 0; x < 9; x++) CHK("table fragment", As + (long)kk * HK_SA + x * 16 + g + 8, Bs);
          for (int y = 0; y < 2; y++) {
            const int cs = wn * 16 + y * 8 + g;
            CHK("W fragment", Bs + (long)kk * HK_SB + cs, (long)(st + 1) * HK_STAGE);
            CHK("slot", cs, 128);
          }
        }
      }
      const int wn = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
      for (int x = 0; x < 9; x++)
        for (int h = 0; h < 2; h++) {
          const int r = x * 16 + g + 8 * h;
          if (r >= ld) continue;
          for (int y = 0; y < 2; y++)
            for (int e = 0; e < 2; e++) {
              const int i = tcell[z * 128 + wn * 16 + y * 8 + 2 * t + e];
              if (i < 0) continue;
              CHK("HK", i + (long)r * ldN, HK_n);
              wr[i + (long)r * ldN]++;
            }
        }
    }
  }
  for (int r = 0; r < ld; r++)
    for (int i = 0; i < N; i++)
      if (wr[i + (long)r * ldN] != 1) {
        fault("HK write count", ctx, wr[i + (long)r * ldN], 1);
        r = ld;
        break;
      }
  free(gstart);
  free(order);
  free(tg);
  free(tcell);
  free(tpos);
  free(wr);
}

/* k_group_sums_dmma<MODE>: grid (gene tiles, groups); three stages of 16-cell slices of the
 * group's run of cells in group order, the stage layout of k_zt_u. */
static void mirror_group_sums(int mode, int m, int J, const int* sizes, int n_grp) {
  char ctx[80];
  int N = 0;
  for (int q = 0; q < n_grp; q++) N += sizes[q];
  snprintf(ctx, sizeof ctx, "group_sums mode=%d n_d=%d J=%d n_grp=%d N=%d", mode, m, J, n_grp, N);
  if (N == 0) return;
  const int ldN = ld_cells(N), n = mode == 1 ? 1 : J;
  const long Dg_n = (long)m * ldN, Wg_n = (long)ldN * J, R_n = ldN, S_n = (long)J * n_grp * (m + 1);
  int* gstart = malloc(sizeof(int) * (n_grp + 1));
  gstart[0] = 0;
  for (int q = 0; q < n_grp; q++) gstart[q + 1] = gstart[q] + sizes[q];
  unsigned char* wr = calloc((size_t)S_n, 1);
  const int tiles = (n + ZT_BN - 1) / ZT_BN;
  for (int z = 0; z < n_grp; z++) {
    const int kbeg = gstart[z], kend = gstart[z + 1];
    const int nsl = kend > kbeg ? (kend - kbeg + ZT_BK - 1) / ZT_BK : 0;
    const int last = kend - 1 > 0 ? kend - 1 : 0;
    unsigned char* hit = calloc((size_t)(kend - kbeg + 1), 1);
    for (int by = 0; by < tiles; by++) {
      const int n0 = by * ZT_BN;
      for (int s = 0; s < nsl; s++) {
        const int st = s % 3, k0 = kbeg + s * ZT_BK;
        const long As = (long)st * ZT_STAGE, Ws = As + ZT_BM * ZT_S, Rs = Ws + 2L * ZT_BN * ZT_S;
        for (int tid = 0; tid < 256; tid++) {
          for (int e = tid; e < ZT_BM * ZT_BK; e += 256) {
            const int r = e >> 4, kc = e & 15, k = k0 + kc;
            CHK("Dg", (long)imin(r, m - 1) * ldN + imin(k, last), Dg_n);
            CHK("A stage", As + r * ZT_S + kc, Ws);
            if (r < m && k < kend && by == 0 && r == 0) hit[k - kbeg]++;
          }
          if (mode == 0) {
            for (int q = 0; q < (ZT_BN * ZT_BK) / 256; q++) {
              const int e = tid + q * 256, cc = e >> 4, kc = e & 15, k = k0 + kc;
              CHK("Wg", (long)imin(n0 + cc, n - 1) * ldN + imin(k, last), Wg_n);
              CHK("W stage", Ws + cc * ZT_S + kc, Ws + ZT_BN * ZT_S);
            }
            if (tid < ZT_BK) {
              CHK("1/Omega", imin(k0 + tid, last), R_n);
              CHK("1/Omega stage", Rs + tid, (long)(st + 1) * ZT_STAGE);
            }
          }
          const int wn = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
          for (int k4 = 0; k4 < ZT_BK / 4; k4++) {
            const int kk = k4 * 4 + t;
            for (int x = 0; x < 9; x++) CHK("A fragment", As + (x * 16 + g + 8) * ZT_S + kk, Ws);
            for (int y = 0; y < 2; y++) CHK("W fragment", Ws + (long)(wn * 16 + y * 8 + g) * ZT_S + kk, Ws + ZT_BN * ZT_S);
            CHK("1/Omega fragment", Rs + kk, (long)(st + 1) * ZT_STAGE);
          }
        }
      }
      for (int tid = 0; tid < 256; tid++) {
        const int wn = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
        for (int x = 0; x < 9; x++)
          for (int h = 0; h < 2; h++) {
            const int r = x * 16 + g + 8 * h;
            if (r >= m) continue;
            for (int y = 0; y < 2; y++)
              for (int e = 0; e < 2; e++) {
                const int j = n0 + wn * 16 + y * 8 + 2 * t + e;
                if (j >= n) continue;
                const long o = ((long)j * n_grp + z) * (m + 1) + r;
                CHK("S", o, S_n);
                if (o >= 0 && o < S_n) wr[o]++;
              }
          }
      }
    }
    for (int k = 0; k < kend - kbeg; k++)
      if (hit[k] != 1) {
        fault("group cell load count", ctx, hit[k], 1);
        break;
      }
    free(hit);
  }
  for (int j = 0; j < n; j++)
    for (int z = 0; z < n_grp; z++)
      for (int r = 0; r < m; r++)
        if (wr[((long)j * n_grp + z) * (m + 1) + r] != 1) {
          fault("S write count", ctx, wr[((long)j * n_grp + z) * (m + 1) + r], 1);
          j = n, z = n_grp;
          break;
        }
  free(gstart);
  free(wr);
}

int main(int argc, char** argv) {
  plant_unpadded = argc > 1 && strcmp(argv[1], "plant") == 0;
  plant_odd = argc > 1 && strcmp(argv[1], "plant-odd") == 0;
  static const int Ns[] = {1, 2, 3, 31, 32, 33, 63, 64, 65, 127, 128, 129, 130, 255, 257, 511, 512, 513, 1001};
  static const int Js[] = {1, 2, 3, 5, 127, 128, 129, 131, 256, 257};
  static const int nds[] = {1, 2, 4, 15, 16, 17, 33, 132, 144, 260};
  static const int grps[] = {0, 1, 3};
  const int nN = sizeof Ns / sizeof *Ns, nJ = sizeof Js / sizeof *Js, nD = sizeof nds / sizeof *nds;
  for (int MT = 4; MT >= 2 && !plant_odd; MT -= 2) {
    long sizes = 0;
    for (int a = 0; a < nN; a++)
      for (int b = 0; b < nJ; b++)
        for (int d = 0; d < nD; d++)
          for (int q = 0; q < 3; q++) {
            const int N = Ns[a], J = Js[b], tiles = ((N + MT * 32 - 1) / (MT * 32)) * ((J + BN - 1) / BN);
            /* the launcher's grid (148 SMs, one or two CTAs each) and a small one that strides */
            const int full = imin(tiles, (MT == 2 ? 2 : 1) * 148);
            mirror_eta(MT, N, J, nds[d], grps[q], full);
            if (tiles > 3) mirror_eta(MT, N, J, nds[d], grps[q], 3);
            sizes++;
          }
    if (faults) return 1;
    printf("ok eta%d %ld\n", MT, sizes);
  }
  long sizes = 0;
  for (int b = 0; b < nJ && !plant_odd; b++)
    for (int q = 0; q < 3; q++, sizes++) mirror_levels(Js[b], grps[q]);
  if (faults) return 1;
  printf("ok levels %ld\n", sizes);
  sizes = 0;
  for (int a = 0; a < nN && !plant_odd; a++)
    for (int b = 0; b < nJ; b++)
      for (int grp = 0; grp < 2; grp++, sizes++) {
        mirror_w_nu(Ns[a], Js[b], grp, 65535);
        mirror_w_nu(Ns[a], Js[b], grp, 2); /* the y stride */
      }
  if (faults) return 1;
  printf("ok w_nu %ld\n", sizes);
  sizes = 0;
  for (int a = 0; a < nN && !plant_odd; a++)
    for (int b = 0; b < nJ; b++)
      for (int dens = 1; dens <= 7; dens += 3, sizes++) mirror_counts(Ns[a], Js[b], dens);
  if (faults) return 1;
  printf("ok counts %ld\n", sizes);
  static const int zN[] = {1, 2, 3, 17, 31, 33, 100, 255, 1001, 3001};
  static const int zJ[] = {1, 3, 128, 129, 257};
  static const int zM[] = {1, 2, 17, 132, 144};
  static const int zS[] = {1, 2, 8, 28, 32};
  sizes = 0;
  for (int mode = 0; mode < 3; mode++)
    for (int a = 0; a < 10; a++)
      for (int b = 0; b < 5; b++)
        for (int d = 0; d < 5; d++)
          for (int q = 0; q < 5; q++, sizes++) mirror_zt_u(mode, zN[a], zJ[b], zM[d], zS[q]);
  if (faults) return 1;
  printf("ok zt_u %ld\n", sizes);
  if (plant_odd) return 0;
  static const int g1[] = {1};
  static const int g2[] = {127, 128, 129, 0, 255, 3};
  static const int g3[] = {300, 1, 1, 2, 513, 64, 0, 77};
  static const int hd[] = {1, 2, 17, 100, 132, 143};
  static const int hJ[] = {1, 3, 16, 17, 100};
  sizes = 0;
  for (int d = 0; d < 6; d++)
    for (int b = 0; b < 5; b++, sizes += 3) {
      mirror_hk(hd[d], hJ[b], g1, 1);
      mirror_hk(hd[d], hJ[b], g2, 6);
      mirror_hk(hd[d], hJ[b], g3, 8);
    }
  if (faults) return 1;
  printf("ok hk %ld\n", sizes);
  sizes = 0;
  for (int mode = 0; mode < 2; mode++)
    for (int d = 0; d < 6; d++)
      for (int b = 0; b < 5; b++, sizes += 3) {
        mirror_group_sums(mode, hd[d] < 144 ? hd[d] : 144, hJ[b] * 3, g1, 1);
        mirror_group_sums(mode, hd[d], hJ[b] * 3, g2, 6);
        mirror_group_sums(mode, hd[d], hJ[b] * 3, g3, 8);
      }
  if (faults) return 1;
  printf("ok group_sums %ld\n", sizes);
  return 0;
}
