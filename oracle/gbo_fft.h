/*
 * CPU discrete Fourier transforms for the oracle (test infrastructure only;
 * nothing in the shipped library links this).
 *
 * Conventions follow FFTW 3.x, the library the reference links for its CPU
 * path (reference make.conf:80-81, src/cgrid_fft.c:48-52):
 *   sign -1 (forward):  X[k] = sum_n x[n] exp(-2 pi i n k / N)
 *   sign +1 (backward): X[k] = sum_n x[n] exp(+2 pi i n k / N)
 * Both are unnormalised.  Multi-dimensional transforms are row-major with the
 * last index fastest, the layout of the reference grids (src/cgrid.c:4).
 *
 * The 1-D engine is a mixed-radix Stockham autosort transform (radices 4, 2,
 * 3, 5 and a direct DFT for any remaining prime factor) with twiddles
 * computed by octant reduction so every twiddle is correctly rounded to
 * within libm's accuracy.
 */
#ifndef GBO_FFT_H
#define GBO_FFT_H

#include <complex.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* In-place complex transform of an n0 x n1 x n2 array (n2 fastest). */
void gbo_fft3d(double _Complex *data, long n0, long n1, long n2, int sign);

/* In-place complex transform of a single contiguous line of length n. */
void gbo_fft1d(double _Complex *data, long n, int sign);

/*
 * Real-to-complex 3-D transform in the in-place padded layout used by FFTW's
 * r2c plans on the reference rgrid (src/rgrid.c:46-47, src/rgrid_fft.c:50-55):
 * rows of nz2 = 2 (nz/2 + 1) reals hold nz/2 + 1 complex outputs.
 */
void gbo_r2c3d(double *data, long nx, long ny, long nz);

/* Complex-to-real inverse of gbo_r2c3d (unnormalised, sign +1). */
void gbo_c2r3d(double *data, long nx, long ny, long nz);

/* exp(sign * 2 pi i * k / n), accurate to libm's sin/cos. */
double _Complex gbo_twiddle(long k, long n, int sign);

#ifdef __cplusplus
}
#endif

#endif
