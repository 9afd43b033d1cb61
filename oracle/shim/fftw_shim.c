/*
 * FFTW 3.x API stand-in backed by the oracle's own transforms
 * (oracle/gbo_fft.c).  Test infrastructure only: it exists so the
 * reference's unchanged CPU sources can be compiled into oracle/_ref.
 *
 * Plans record their array and geometry; fftw_execute runs the transform
 * in place.  Planning flags (MEASURE/PATIENT/...) are accepted and ignored,
 * which also removes FFTW_MEASURE's run-to-run nondeterminism
 * (reference src/threads.c:10).
 */
#include <complex.h>
#include <stdlib.h>

#include "fftw3.h"
#include "../gbo_fft.h"

enum { GBO_C2C = 0, GBO_R2C = 1, GBO_C2R = 2 };

struct gbo_fftw_plan_s {
  int kind;
  int sign;
  long n0, n1, n2;
  void *in, *out;
};

void *fftw_malloc(size_t n) {
  void *p = NULL;
  if (posix_memalign(&p, 64, n ? n : 1)) return NULL;
  return p;
}

void fftw_free(void *p) { free(p); }

int fftw_init_threads(void) { return 1; }

void fftw_plan_with_nthreads(int nthreads) { (void) nthreads; }

static fftw_plan mk(int kind, int sign, int n0, int n1, int n2, void *in, void *out) {
  fftw_plan p = (fftw_plan) malloc(sizeof(*p));
  if (!p) return NULL;
  p->kind = kind;
  p->sign = sign;
  p->n0 = n0;
  p->n1 = n1;
  p->n2 = n2;
  p->in = in;
  p->out = out;
  return p;
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void) flags;
  return mk(GBO_C2C, sign, n0, n1, n2, in, out);
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags) {
  (void) flags;
  return mk(GBO_R2C, -1, n0, n1, n2, in, out);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags) {
  (void) flags;
  return mk(GBO_C2R, +1, n0, n1, n2, in, out);
}

void fftw_execute(const fftw_plan p) {
  /* The reference only plans in-place transforms (in == out). */
  switch (p->kind) {
    case GBO_C2C:
      gbo_fft3d((double _Complex *) p->in, p->n0, p->n1, p->n2, p->sign);
      break;
    case GBO_R2C:
      gbo_r2c3d((double *) p->in, p->n0, p->n1, p->n2);
      break;
    case GBO_C2R:
      gbo_c2r3d((double *) p->out, p->n0, p->n1, p->n2);
      break;
  }
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

int fftw_export_wisdom_to_filename(const char *filename) {
  (void) filename;
  return 1;
}

int fftw_import_wisdom_from_filename(const char *filename) {
  (void) filename;
  return 0;
}
