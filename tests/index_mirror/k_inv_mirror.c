/*
 * CPU mirror of the memory indexing of the batched Cholesky and inverse panel kernels
 * (gaspacho2_b200/csrc/k_inv.cu: k_potrf_panel, k_trtri_panel, k_lauum_panel).
 *
 * Every loop of the three kernels is replayed for every thread of a block (256 threads,
 * warps of 32, lane = 4 g + t as in the DMMA fragments) and every block of one matrix, with
 * the kernels' own index expressions. Each shared-memory index is checked against the
 * dynamic shared-memory size the launcher requests, each global index against the P x P
 * matrix, and the outputs are counted: every entry the kernel must produce is written, and
 * every row of a Cholesky panel receives the update of the finished columns exactly once.
 * A source address formed for a zero-byte (zero-fill) cp.async must lie inside the
 * allocation too.
 *
 *   k_inv_mirror <potrf|trtri|lauum> <P first> <P last>
 *
 * prints "ok <kernel> <first>..<last>" and exits 0, or lists the first faults and exits 1.
 * Compiled and run by tests/test_index_mirror.py. Keep it in step with k_inv.cu.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define IB 32
#define IS 36
#define LS 33
#define CW 8
#define NT 256

static long faults = 0;
static void fault(const char* what, int P, long idx, long lim) {
  if (faults < 20) fprintf(stderr, "P=%d %s index %ld outside [0, %ld)\n", P, what, idx, lim);
  faults++;
}
#define SH(i) do { long i_ = (long)(i); if (i_ < 0 || i_ >= sh_n) fault("shared", P, i_, sh_n); } while (0)
#define GL(i) do { long i_ = (long)(i); if (i_ < 0 || i_ >= gl_n) fault("global", P, i_, gl_n); } while (0)

static int imin(int a, int b) { return a < b ? a : b; }

static long potrf_smem_doubles(int P) {
  const int rows_pad = (P + 15) / 16 * 16;
  return (long)rows_pad * IS + 2L * CW * (rows_pad + 4) + IB;
}
static long inverse_smem_doubles(int P) {
  const int nb = (P + IB - 1) / IB;
  return (long)nb * IB * IS + 2L * IB * IS + 2L * IB * LS + IB;
}

static void mirror_potrf(int P) {
  const long sh_n = potrf_smem_doubles(P), gl_n = (long)P * P;
  const int rows_pad = (P + 15) / 16 * 16, SA = rows_pad + 4;
  const long Ap = 0, La = (long)rows_pad * IS, Rd = La + 2L * CW * SA;
  const int nb = (P + IB - 1) / IB;
  int* written = calloc((size_t)P * P, sizeof(int));
  int* covered = malloc(sizeof(int) * (rows_pad + 16));
  for (int kp = 0; kp < nb; kp++) {
    const int c0 = kp * IB, rows = P - c0, ncol = imin(IB, rows);
    const int rpad = (rows + 15) / 16 * 16;
    for (int tid = 0; tid < NT; tid++)
      for (int e = tid; e < rpad * IB; e += NT) {
        const int cc = e / rpad, r = e - cc * rpad;
        SH(Ap + r * IS + cc);
        if (r < rows && cc < ncol) GL((long)(c0 + r) + (long)(c0 + cc) * P);
      }
    if (kp > 0) {
      memset(covered, 0, sizeof(int) * (rows_pad + 16));
      const int nch = c0 / CW;
      for (int ch = 0; ch < nch; ch++) {
        const int buf = ch & 1;
        for (int tid = 0; tid < NT; tid++)
          for (int e = tid; e < CW * rpad; e += NT) {
            const int q = e / rpad, r = e - q * rpad;
            const int ok = r < rows;
            SH(La + (long)buf * CW * SA + q * SA + r);
            GL(ok ? (long)(c0 + r) + (long)(ch * CW + q) * P : 0);
          }
        for (int tid = 0; tid < NT; tid++) {
          const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
          for (int k4 = 0; k4 < CW / 4; k4++) {
            const long lr = La + (long)buf * CW * SA + (k4 * 4 + t) * SA;
            for (int y = 0; y < 4; y++) SH(lr + y * 8 + g);
            for (int x = 0; x < 2; x++) {
              const int mt = warp + 8 * x;
              if (mt * 16 < rpad) {
                SH(lr + mt * 16 + g);
                SH(lr + mt * 16 + g + 8);
              }
            }
          }
        }
      }
      for (int tid = 0; tid < NT; tid++) {
        const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
        for (int x = 0; x < 2; x++) {
          const int mt = warp + 8 * x;
          if (mt * 16 >= rpad) continue;
          for (int y = 0; y < 4; y++)
            for (int h = 0; h < 2; h++)
              for (int e = 0; e < 2; e++) {
                const int r = mt * 16 + g + 8 * h;
                SH(Ap + r * IS + y * 8 + 2 * t + e);
                if (y == 0 && t == 0 && e == 0) covered[r]++;
              }
        }
      }
      for (int r = 0; r < rows; r++)
        if (covered[r] != 1) {
          if (faults < 20) fprintf(stderr, "P=%d panel %d row %d updated %d times\n", P, kp, r, covered[r]);
          faults++;
        }
    }
    for (int lane = 0; lane < 32; lane++) {
      for (int q = 0; q < IB; q++)
        if (lane < ncol) SH(Ap + lane * IS + q);
      for (int cc = 0; cc < IB; cc++)
        if (cc < ncol && lane == cc) SH(Rd + cc);
    }
    for (int tid = 0; tid < NT; tid++)
      for (int r = IB + tid; r < rows; r += NT) {
        for (int q = 0; q < IB; q++) SH(Ap + r * IS + q);
        for (int cc = 0; cc < IB; cc++)
          if (cc < ncol) {
            SH(Rd + cc);
            for (int q = cc + 1; q < IB; q++) SH(Ap + q * IS + cc);
          }
      }
    for (int tid = 0; tid < NT; tid++)
      for (int e = tid; e < rows * IB; e += NT) {
        const int cc = e / rows, r = e - cc * rows;
        if (cc < ncol && r >= cc) {
          SH(Ap + r * IS + cc);
          const long gi = (long)(c0 + r) + (long)(c0 + cc) * P;
          GL(gi);
          if (gi >= 0 && gi < gl_n) written[gi]++;
        }
      }
  }
  for (int col = 0; col < P; col++)
    for (int row = col; row < P; row++)
      if (written[row + (long)col * P] != 1) {
        if (faults < 20) fprintf(stderr, "P=%d factor (%d, %d) written %d times\n", P, row, col,
                                 written[row + (long)col * P]);
        faults++;
      }
  free(written);
  free(covered);
}

static void mirror_trtri(int P) {
  const long sh_n = inverse_smem_doubles(P), gl_n = (long)P * P;
  const int nb = (P + IB - 1) / IB;
  const long Yp = 0, As = (long)nb * IB * IS, Ld = As + 2L * IB * IS, Rs = Ld + (long)IB * LS, Rd = Rs + (long)IB * LS;
  int* written = calloc((size_t)P * P, sizeof(int));
  for (int jb = 0; jb < nb; jb++) {
    const int r0 = jb * IB;
    for (int ib = jb; ib < nb; ib++) {
      const int rb = ib * IB, nch = ib - jb;
      for (int ch = 0; ch < nch; ch++) {
        const int buf = ch & 1;
        for (int tid = 0; tid < NT; tid++)
          for (int e = tid; e < IB * IB; e += NT) {
            const int k = e >> 5, m = e & 31, row = rb + m;
            SH(As + (long)buf * IB * IS + k * IS + m);
            GL((long)imin(row, P - 1) + (long)(r0 + ch * IB + k) * P);
          }
      }
      for (int tid = 0; tid < NT; tid++)
        for (int e = tid; e < IB * IB; e += NT) {
          const int q = e >> 5, m = e & 31, row = rb + m, col = rb + q;
          if (row < P && col < P && q <= m) GL(row + (long)col * P);
          SH(Ld + m * LS + q);
        }
      for (int ch = 0; ch < nch; ch++)
        for (int tid = 0; tid < NT; tid++) {
          const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
          const int m0 = (warp >> 2) * 16, n0 = (warp & 3) * 8;
          const long as = As + (long)(ch & 1) * IB * IS, yp = Yp + (long)ch * IB * IS;
          for (int kb = 0; kb < IB; kb += 8)
            for (int d = 0; d < 8; d += 4) {
              SH(as + (kb + d + t) * IS + m0 + g);
              SH(as + (kb + d + t) * IS + m0 + g + 8);
              SH(yp + (kb + d + t) * IS + n0 + g);
            }
        }
      const int K = nch * IB;
      for (int tid = 0; tid < NT; tid++) {
        const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
        const int m0 = (warp >> 2) * 16, n0 = (warp & 3) * 8;
        for (int h = 0; h < 2; h++)
          for (int e = 0; e < 2; e++) SH(Rs + (m0 + g + 8 * h) * LS + n0 + 2 * t + e);
        if (tid < IB) {
          SH(Rd + tid);
          SH(Ld + tid * LS + tid);
        }
        for (int c = 0; c < 4; c++) SH(Rs + lane * LS + 4 * warp + c);
        for (int q = 0; q < IB; q++) {
          SH(Rd + q);
          SH(Ld + lane * LS + q);
        }
        for (int c = 0; c < 4; c++) SH(Yp + (long)(K + lane) * IS + 4 * warp + c);
      }
    }
    const int ncol = imin(IB, P - r0), nrow = P - r0;
    for (int tid = 0; tid < NT; tid++)
      for (int e = tid; e < nrow * ncol; e += NT) {
        const int c = e / nrow, r = e - c * nrow;
        SH(Yp + r * IS + c);
        const long gi = (long)(r0 + r) + (long)(r0 + c) * P;
        GL(gi);
        if (gi >= 0 && gi < gl_n) written[gi]++;
      }
  }
  for (int col = 0; col < P; col++)
    for (int row = col; row < P; row++)
      if (written[row + (long)col * P] != 1) {
        if (faults < 20) fprintf(stderr, "P=%d inverse factor (%d, %d) written %d times\n", P, row, col,
                                 written[row + (long)col * P]);
        faults++;
      }
  free(written);
}

static void mirror_lauum(int P) {
  const long sh_n = inverse_smem_doubles(P), gl_n = (long)P * P;
  const int nb = (P + IB - 1) / IB;
  const long Vb = 0, Ak = (long)nb * IB * IS;
  int* written = calloc((size_t)P * P, sizeof(int));
  for (int b = 0; b < nb; b++) {
    const int c0 = b * IB, ncol = imin(IB, P - c0);
    const int kb_rows = (P - c0 + 3) / 4 * 4;
    for (int tid = 0; tid < NT; tid++)
      for (int e = tid; e < kb_rows * IB; e += NT) {
        const int n = e / kb_rows, k = e - n * kb_rows, row = c0 + k, col = c0 + n;
        const int ok = row < P && col < P;
        SH(Vb + k * IS + n);
        GL(ok ? (long)row + (long)col * P : 0);
      }
    for (int a = b; a < nb; a++) {
      const int a0 = a * IB, K = (P - a0 + 3) / 4 * 4, nch = (K + IB - 1) / IB, off = a0 - c0;
      for (int ch = 0; ch < nch; ch++) {
        const int buf = ch & 1, k0 = ch * IB, kn = imin(IB, K - k0);
        for (int tid = 0; tid < NT; tid++)
          for (int e = tid; e < kn * IB; e += NT) {
            const int m = e / kn, k = e - m * kn, row = a0 + k0 + k, col = a0 + m;
            const int ok = row < P && col < P;
            SH(Ak + (long)buf * IB * IS + k * IS + m);
            GL(ok ? (long)row + (long)col * P : 0);
          }
        for (int tid = 0; tid < NT; tid++) {
          const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
          const int m0 = (warp >> 2) * 16, n0 = (warp & 3) * 8;
          const long ak = Ak + (long)buf * IB * IS, vb = Vb + (long)(off + ch * IB) * IS;
          if (kn % 4) {
            if (faults < 20) fprintf(stderr, "P=%d lauum chunk of %d rows\n", P, kn);
            faults++;
          }
          for (int kb = 0; kb < kn; kb += 4) {
            SH(ak + (kb + t) * IS + m0 + g);
            SH(ak + (kb + t) * IS + m0 + g + 8);
            SH(vb + (kb + t) * IS + n0 + g);
            /* the rows of Vb read here must have been loaded (row index < kb_rows) */
            if (off + ch * IB + kb + t >= kb_rows) {
              if (faults < 20) fprintf(stderr, "P=%d lauum reads unloaded row %d\n", P, off + ch * IB + kb + t);
              faults++;
            }
          }
        }
      }
      for (int tid = 0; tid < NT; tid++) {
        const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
        const int m0 = (warp >> 2) * 16, n0 = (warp & 3) * 8;
        for (int h = 0; h < 2; h++)
          for (int e = 0; e < 2; e++) {
            const int m = m0 + g + 8 * h, n = n0 + 2 * t + e, row = a0 + m, col = c0 + n;
            if (row < P && n < ncol) {
              GL(row + (long)col * P);
              GL(col + (long)row * P);
              if (row + (long)col * P < gl_n) written[row + (long)col * P]++;
              if (col + (long)row * P < gl_n) written[col + (long)row * P]++;
            }
          }
      }
    }
  }
  for (long e = 0; e < gl_n; e++)
    if (written[e] < 1) {
      if (faults < 20) fprintf(stderr, "P=%d inverse entry %ld not written\n", P, e);
      faults++;
    }
  free(written);
}

int main(int argc, char** argv) {
  if (argc != 4) {
    fprintf(stderr, "usage: %s <potrf|trtri|lauum> <P first> <P last>\n", argv[0]);
    return 2;
  }
  const int a = atoi(argv[2]), b = atoi(argv[3]);
  void (*f)(int) = !strcmp(argv[1], "potrf") ? mirror_potrf
                   : !strcmp(argv[1], "trtri") ? mirror_trtri
                   : !strcmp(argv[1], "lauum") ? mirror_lauum
                                               : NULL;
  if (!f || a < 1 || b < a) return 2;
  for (int P = a; P <= b; P++) f(P);
  if (faults) {
    fprintf(stderr, "%ld faults\n", faults);
    return 1;
  }
  printf("ok %s %d..%d\n", argv[1], a, b);
  return 0;
}
