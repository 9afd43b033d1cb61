/*
 * Minimal FFTW 3.x API stand-in used only to compile the reference's CPU
 * sources into the oracle (oracle/_ref).  FFTW itself is not installed in
 * this image; this header declares exactly the symbols the reference calls
 * (src/cgrid_fft.c:22-146, src/rgrid_fft.c:25-129, src/grid_fft.c:35-69,
 * src/threads.c:9-157, src/cgrid.c:65,342, src/rgrid.c:53-59) with FFTW's
 * documented signatures and sign/normalisation conventions.  The transforms
 * behind it are the project's own (oracle/gbo_fft.c).
 *
 * Test infrastructure only: no shipped code includes this header.
 */
#ifndef GBO_FFTW3_SHIM_H
#define GBO_FFTW3_SHIM_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_Complex_I) && defined(complex) && defined(I)
typedef double _Complex fftw_complex;
typedef float _Complex fftwf_complex;
typedef long double _Complex fftwl_complex;
#else
typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef long double fftwl_complex[2];
#endif

typedef struct gbo_fftw_plan_s *fftw_plan;
typedef struct gbo_fftw_plan_s *fftwf_plan;
typedef struct gbo_fftw_plan_s *fftwl_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_WISDOM_ONLY (1U << 21)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_export_wisdom_to_filename(const char *filename);
int fftw_import_wisdom_from_filename(const char *filename);

#ifdef __cplusplus
}
#endif

#endif
