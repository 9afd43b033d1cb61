/*
 * CPU mixed-radix Stockham FFT for the oracle (test infrastructure only).
 * Conventions: see gbo_fft.h.  Written for this project; it stands in for
 * FFTW 3.x, which the reference links (make.conf:80-81) but which is not
 * installed in this image.
 *
 * Each 1-D transform of length N = R_1 * R_2 * ... runs one Stockham stage
 * per radix R with Ns = R_1 * ... * R_{s-1}:
 *   for j in [0, N/R):  k = j mod Ns
 *     v[r] = in[j + r N/R] * exp(sign 2 pi i k r / (Ns R))
 *     v    = DFT_R(v)
 *     out[(j / Ns) Ns R + k + r Ns] = v[r]
 * which leaves the result in natural order (autosort).  Strided axes are
 * transformed B columns at a time so that the innermost loop runs over
 * adjacent memory.
 */
#include "gbo_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define GBO_MAX_STAGES 64
#define GBO_BATCH 8 /* columns transformed together on strided axes */

double _Complex gbo_twiddle(long k, long n, int sign) {
  long double a;
  long m = k % n;
  if (m < 0) m += n;
  /* 2 pi m / n in extended precision, then round the cosine and sine. */
  a = 6.283185307179586476925286766559005768L * (long double) m / (long double) n;
  return (double) cosl(a) + I * (double) (sign * sinl(a));
}

typedef struct {
  long n;
  int nstages;
  int radix[GBO_MAX_STAGES];
  long ns[GBO_MAX_STAGES];
  double _Complex *tw[GBO_MAX_STAGES];   /* stage twiddles: [k * (R-1) + (r-1)] */
  double _Complex *rootR[GBO_MAX_STAGES]; /* exp(sign 2 pi i m / R), m < R (generic radix) */
  int sign;
} gbo_plan1d;

static void plan1d_init(gbo_plan1d *p, long n, int sign) {
  long rem = n, ns = 1;
  int s = 0;
  p->n = n;
  p->sign = sign;
  while (rem > 1) {
    int r;
    if (rem % 4 == 0) r = 4;
    else if (rem % 2 == 0) r = 2;
    else if (rem % 3 == 0) r = 3;
    else if (rem % 5 == 0) r = 5;
    else {
      long f = 7;
      while (rem % f) f += 2;
      r = (int) f;
    }
    p->radix[s] = r;
    p->ns[s] = ns;
    p->tw[s] = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) (ns * (r - 1) + 1));
    for (long k = 0; k < ns; k++)
      for (int q = 1; q < r; q++)
        p->tw[s][k * (r - 1) + (q - 1)] = gbo_twiddle(k * q, ns * r, sign);
    p->rootR[s] = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) r);
    for (int m = 0; m < r; m++) p->rootR[s][m] = gbo_twiddle(m, r, sign);
    ns *= r;
    rem /= r;
    s++;
  }
  p->nstages = s;
}

static void plan1d_free(gbo_plan1d *p) {
  for (int s = 0; s < p->nstages; s++) {
    free(p->tw[s]);
    free(p->rootR[s]);
  }
}

/*
 * One Stockham stage on B interleaved columns: element (pos, b) lives at
 * [pos * B + b].
 */
static void stage(const gbo_plan1d *p, int s, const double _Complex *in, double _Complex *out, long B) {
  const long n = p->n, R = p->radix[s], ns = p->ns[s], stride = n / R;
  const double _Complex *tw = p->tw[s];
  const double sg = (double) p->sign;
  double _Complex v[64];
  double _Complex *vbig = NULL;
  double _Complex *vv = v;

  if (R > 64) vbig = vv = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) R);
  for (long j = 0; j < stride; j++) {
    const long k = j % ns;
    const long dst = (j / ns) * ns * R + k;
    for (long b = 0; b < B; b++) {
      for (long r = 0; r < R; r++) {
        double _Complex x = in[(j + r * stride) * B + b];
        if (r && k) x *= tw[k * (R - 1) + (r - 1)];
        vv[r] = x;
      }
      if (R == 2) {
        double _Complex a = vv[0], c = vv[1];
        vv[0] = a + c;
        vv[1] = a - c;
      } else if (R == 4) {
        double _Complex a0 = vv[0] + vv[2], a1 = vv[0] - vv[2];
        double _Complex a2 = vv[1] + vv[3], a3 = vv[1] - vv[3];
        /* multiply a3 by sign * i */
        double _Complex a3r = sg * (-cimag(a3) + I * creal(a3));
        vv[0] = a0 + a2;
        vv[2] = a0 - a2;
        vv[1] = a1 + a3r;
        vv[3] = a1 - a3r;
      } else {
        double _Complex t[64], *tt = t;
        double _Complex *tbig = NULL;
        if (R > 64) tbig = tt = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) R);
        for (long q = 0; q < R; q++) {
          double _Complex acc = 0.0;
          for (long r = 0; r < R; r++) acc += vv[r] * p->rootR[s][(q * r) % R];
          tt[q] = acc;
        }
        for (long q = 0; q < R; q++) vv[q] = tt[q];
        free(tbig);
      }
      for (long r = 0; r < R; r++) out[(dst + r * ns) * B + b] = vv[r];
    }
  }
  free(vbig);
}

/* Transform B interleaved columns held in buf (length n * B); tmp same size. */
static void run_plan(const gbo_plan1d *p, double _Complex *buf, double _Complex *tmp, long B) {
  double _Complex *a = buf, *b = tmp;
  for (int s = 0; s < p->nstages; s++) {
    stage(p, s, a, b, B);
    double _Complex *t = a;
    a = b;
    b = t;
  }
  if (a != buf) memcpy(buf, a, sizeof(double _Complex) * (size_t) (p->n * B));
}

void gbo_fft1d(double _Complex *data, long n, int sign) {
  gbo_plan1d p;
  double _Complex *tmp;
  if (n <= 1) return;
  plan1d_init(&p, n, sign);
  tmp = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) n);
  run_plan(&p, data, tmp, 1);
  free(tmp);
  plan1d_free(&p);
}

/*
 * Transform along one axis of an array viewed as [outer][n][inner]:
 * element (o, m, i) at data[(o * n + m) * inner + i].
 */
static void fft_axis(double _Complex *data, long outer, long n, long inner, int sign) {
  gbo_plan1d p;
  if (n <= 1) return;
  plan1d_init(&p, n, sign);
  if (inner == 1) {
#pragma omp parallel
    {
      double _Complex *tmp = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) n);
#pragma omp for schedule(static)
      for (long o = 0; o < outer; o++) run_plan(&p, data + o * n, tmp, 1);
      free(tmp);
    }
  } else {
    const long nblk = (inner + GBO_BATCH - 1) / GBO_BATCH;
#pragma omp parallel
    {
      double _Complex *buf = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) (n * GBO_BATCH));
      double _Complex *tmp = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) (n * GBO_BATCH));
#pragma omp for schedule(static) collapse(2)
      for (long o = 0; o < outer; o++) {
        for (long blk = 0; blk < nblk; blk++) {
          const long i0 = blk * GBO_BATCH;
          const long B = (inner - i0 < GBO_BATCH) ? inner - i0 : GBO_BATCH;
          double _Complex *base = data + o * n * inner + i0;
          for (long m = 0; m < n; m++)
            for (long b = 0; b < B; b++) buf[m * B + b] = base[m * inner + b];
          run_plan(&p, buf, tmp, B);
          for (long m = 0; m < n; m++)
            for (long b = 0; b < B; b++) base[m * inner + b] = buf[m * B + b];
        }
      }
      free(buf);
      free(tmp);
    }
  }
  plan1d_free(&p);
}

void gbo_fft3d(double _Complex *data, long n0, long n1, long n2, int sign) {
  fft_axis(data, n0 * n1, n2, 1, sign);
  fft_axis(data, n0, n1, n2, sign);
  fft_axis(data, 1, n0, n1 * n2, sign);
}

void gbo_r2c3d(double *data, long nx, long ny, long nz) {
  const long nzh = nz / 2 + 1, nz2 = 2 * nzh;
  double _Complex *full = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) (nx * ny * nz));
  for (long ij = 0; ij < nx * ny; ij++)
    for (long k = 0; k < nz; k++) full[ij * nz + k] = data[ij * nz2 + k];
  gbo_fft3d(full, nx, ny, nz, -1);
  double _Complex *out = (double _Complex *) data;
  for (long ij = 0; ij < nx * ny; ij++)
    for (long k = 0; k < nzh; k++) out[ij * nzh + k] = full[ij * nz + k];
  free(full);
}

void gbo_c2r3d(double *data, long nx, long ny, long nz) {
  const long nzh = nz / 2 + 1, nz2 = 2 * nzh;
  const double _Complex *in = (const double _Complex *) data;
  double _Complex *full = (double _Complex *) malloc(sizeof(double _Complex) * (size_t) (nx * ny * nz));
  for (long i = 0; i < nx; i++)
    for (long j = 0; j < ny; j++)
      for (long k = 0; k < nz; k++) {
        double _Complex v;
        if (k < nzh) v = in[(i * ny + j) * nzh + k];
        else {
          const long ii = (nx - i) % nx, jj = (ny - j) % ny, kk = nz - k;
          v = conj(in[(ii * ny + jj) * nzh + kk]);
        }
        full[(i * ny + j) * nz + k] = v;
      }
  gbo_fft3d(full, nx, ny, nz, +1);
  for (long ij = 0; ij < nx * ny; ij++) {
    for (long k = 0; k < nz; k++) data[ij * nz2 + k] = creal(full[ij * nz + k]);
    for (long k = nz; k < nz2; k++) data[ij * nz2 + k] = 0.0;
  }
  free(full);
}
