/*
 * ORACLE (test infrastructure only; never linked into the shipped library).
 *
 * Plain-C restatement of libgrid's wavefunction-propagation path on
 * double-complex arrays in the reference's layout (row-major, z fastest;
 * src/cgrid.c:4-7; real grids padded to nz2 = 2 (nz/2 + 1),
 * src/rgrid.c:46-47).  Each function names the reference lines it follows.
 * Transforms come from gbo_fft.c (FFTW conventions).
 *
 * Used by the tests and by the benchmark's CPU baseline leg to check and
 * time the GPU path; it is checked itself against the reference's own
 * sources compiled into oracle/_ref (see oracle/build_ref.sh).
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gbo_fft.h"

typedef double _Complex cplx;

#define GBO_HBAR 1.0 /* make.conf:45 */

static double step_factor(long nx, long ny, long nz, double step) {
  double f = 1.0;
  if (nx != 1) f *= step;
  if (ny != 1) f *= step;
  if (nz != 1) f *= step;
  return f;
}

/* src/grid_wf.c:185-203 */
double gbo_absorb(long i, long j, long k, const long *lh) {
  double t = 0.0;
  const long lx = lh[0], hx = lh[1], ly = lh[2], hy = lh[3], lz = lh[4], hz = lh[5];
  if (i < lx) t += ((double) (lx - i)) / (double) lx;
  else if (i > hx) t += ((double) (i - hx)) / (double) lx;
  if (j < ly) t += ((double) (ly - j)) / (double) ly;
  else if (j > hy) t += ((double) (j - hy)) / (double) ly;
  if (k < lz) t += ((double) (lz - k)) / (double) lz;
  else if (k > hz) t += ((double) (k - hz)) / (double) lz;
  t *= 2.0 / 3.0;
  if (t > 1.0) return 1.0;
  return t;
}

/*
 * src/grid_wf_fft.c:141-193 (cutoff == 0) and :206-262 (cutoff != 0):
 * psi_k *= cexp(time_mass |k - k0|^2), time_mass = -i time hbar / (2 m);
 * k = (i or i - n) 2 pi / (n step) - k0 with i <= n/2 non-negative.
 */
void gbo_kinetic_fft(cplx *psi, long nx, long ny, long nz, double step, double mass, cplx time, double kx0, double ky0,
                     double kz0, int cutoff, double kmax) {
  const cplx time_mass = -I * time * GBO_HBAR / (mass * 2.0);
  const double lx = 2.0 * M_PI / (step * (double) nx), ly = 2.0 * M_PI / (step * (double) ny),
               lz = 2.0 * M_PI / (step * (double) nz), kmax2 = kmax * kmax;
#pragma omp parallel for schedule(static)
  for (long ij = 0; ij < nx * ny; ij++) {
    const long i = ij / ny, j = ij % ny;
    const double kx = (i <= nx / 2 ? (double) i : (double) (i - nx)) * lx - kx0;
    const double ky = (j <= ny / 2 ? (double) j : (double) (j - ny)) * ly - ky0;
    for (long k = 0; k < nz; k++) {
      const double kz = (k <= nz / 2 ? (double) k : (double) (k - nz)) * lz - kz0;
      const double tot = kx * kx + ky * ky + kz * kz;
      if (cutoff && !(tot < kmax2)) psi[ij * nz + k] = 0.0;
      else psi[ij * nz + k] *= cexp(time_mass * tot);
    }
  }
}

/*
 * src/grid_wf.c:569-600: psi *= cexp(c (cons + V)), c = -i tstep / hbar, or
 * with the absorbing ramp a(r): c = -i ((1 - a) Re tstep - i Re tstep a)/hbar.
 * The potential is either complex (vc, rows of nz) or real padded
 * (vr, rows of nz2) plus g |psi|^2 (the nonlinear term built from psi as it
 * is when the factor is applied).  lh == NULL: no absorbing region.
 */
void gbo_potential(cplx *psi, long nx, long ny, long nz, cplx tstep, const cplx *vc, const double *vr, double g,
                   double cons, const long *lh) {
  const long nz2 = 2 * (nz / 2 + 1);
#pragma omp parallel for schedule(static)
  for (long ij = 0; ij < nx * ny; ij++) {
    const long i = ij / ny, j = ij % ny;
    for (long k = 0; k < nz; k++) {
      cplx c;
      if (lh) {
        const double t = gbo_absorb(i, j, k, lh);
        c = -I * ((1.0 - t) * creal(tstep) - I * creal(tstep) * t) / GBO_HBAR;
      } else c = -I * tstep / GBO_HBAR;
      cplx v = 0.0;
      if (vc) v = vc[ij * nz + k];
      if (vr) v = vr[ij * nz2 + k];
      if (g != 0.0) {
        const cplx p = psi[ij * nz + k];
        v += g * (creal(p) * creal(p) + cimag(p) * cimag(p));
      }
      psi[ij * nz + k] = psi[ij * nz + k] * cexp(c * (cons + v));
    }
  }
}

/* cgrid_inverse_fft_norm (src/cgrid.c:1857-1876): unnormalised inverse FFT,
 * then a separate multiplication by 1 / (nx ny nz). */
static void ifft_norm(cplx *psi, long nx, long ny, long nz) {
  const long n = nx * ny * nz;
  const double norm = 1.0 / (double) n;
  gbo_fft3d(psi, nx, ny, nz, +1);
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; q++) psi[q] *= norm;
}

/*
 * 2nd-order FFT split-operator step (src/grid_wf.c:424-430):
 * FFT, K(dt/2), IFFT/N, V(dt), FFT, K(dt/2), IFFT/N.  The potential step uses
 * vc or (vr, g); all NULL / 0 skips it as grid_wf_propagate_potential does
 * for a NULL potential (src/grid_wf.c:576).
 */
void gbo_fft_step(cplx *psi, long nx, long ny, long nz, double step, double mass, cplx time, double kx0, double ky0,
                  double kz0, const cplx *vc, const double *vr, double g, int cutoff, double kmax) {
  const cplx half = 0.5 * time;
  const double cons = -(GBO_HBAR * GBO_HBAR / (2.0 * mass)) * (kx0 * kx0 + ky0 * ky0 + kz0 * kz0);
  gbo_fft3d(psi, nx, ny, nz, -1);
  gbo_kinetic_fft(psi, nx, ny, nz, step, mass, half, kx0, ky0, kz0, cutoff, kmax);
  ifft_norm(psi, nx, ny, nz);
  if (vc || vr || g != 0.0) gbo_potential(psi, nx, ny, nz, time, vc, vr, g, cons, NULL);
  gbo_fft3d(psi, nx, ny, nz, -1);
  gbo_kinetic_fft(psi, nx, ny, nz, step, mass, half, kx0, ky0, kz0, cutoff, kmax);
  ifft_norm(psi, nx, ny, nz);
}

/* ---------------------------------------------------------------- CN */

/* src/linalg.c:62-92: Thomas with sub = 1 - c2 (2 in the last row) and
 * sup = 1 + c2 (2 in the first row); b and v are overwritten. */
static void tri_system2(long n, cplx *b, cplx *v, cplx *x, cplx c2, long str) {
  const cplx cc2p = 1.0 + c2, cc2m = 1.0 - c2;
  cplx m, a, c;
  for (long i = 1; i < n; i++) {
    a = (i == n - 1) ? 2.0 : cc2m;
    c = (i == 1) ? 2.0 : cc2p;
    m = a / b[i - 1];
    b[i] -= m * c;
    v[i] -= m * v[i - 1];
  }
  x[str * (n - 1)] = v[n - 1] / b[n - 1];
  for (long i = n - 2; i >= 0; --i) {
    c = (i == 0) ? 2.0 : cc2p;
    x[i * str] = (v[i] - c * x[(i + 1) * str]) / b[i];
  }
}

/* src/linalg.c:111-138: uniform sub = 1 - c2, sup = 1 + c2 */
static void tri_system3(long n, cplx *b, cplx *v, cplx *x, cplx c2, long str) {
  const cplx cc2p = 1.0 + c2, cc2m = 1.0 - c2;
  for (long i = 1; i < n; i++) {
    const cplx m = cc2m / b[i - 1];
    b[i] -= m * cc2p;
    v[i] -= m * v[i - 1];
  }
  x[str * (n - 1)] = v[n - 1] / b[n - 1];
  for (long i = n - 2; i >= 0; --i) x[i * str] = (v[i] - cc2p * x[(i + 1) * str]) / b[i];
}

/* src/linalg.c:206-230: periodic (Sherman-Morrison) solve; bb is workspace */
static void tri_cyclic2(long n, cplx *b, cplx *v, cplx *x, cplx c2, long str, cplx *bb) {
  const cplx alpha = 1.0 + c2, beta = 1.0 - c2, gamma = -b[0];
  b[0] = bb[0] = b[0] - gamma;
  b[n - 1] = bb[n - 1] = b[n - 1] - alpha * beta / gamma;
  for (long i = 1; i < n - 1; i++) bb[i] = b[i];
  tri_system3(n, bb, v, x, c2, str);
  v[0] = gamma;
  v[n - 1] = alpha;
  for (long i = 1; i < n - 1; i++) v[i] = 0.0;
  tri_system3(n, b, v, bb, c2, 1);
  const cplx fact = (x[0] + beta * x[str * (n - 1)] / gamma) / (1.0 + bb[0] + beta * bb[n - 1] / gamma);
  for (long i = 0; i < n; i++) x[str * i] -= fact * bb[i];
}

/*
 * One Crank-Nicolson line along an axis with element stride `str` starting
 * at psi0 (src/grid_wf_cn.c:129-209 for x; :260-340 for y; :390-468 for z):
 * builds the diagonal d and right-hand side b, including the boundary rows,
 * then solves with tri_system2 (Dirichlet/Neumann) or tri_cyclic2 (periodic).
 * bc: 1 Dirichlet, 2 Neumann, 3 periodic.  c3c = c3 * (perpendicular
 * coordinate) (zero for the z axis, which has no rotation term).  ts_a[i] is
 * the absorbing ramp of element i, or NULL.
 */
static void cn_line(cplx *psi0, long n, long str, int bc, cplx c, cplx tstep, cplx c2, cplx c3c, const double *ts_a,
                    cplx *d, cplx *b, cplx *w) {
  cplx tim, cp;
#define P(q) psi0[(q) * str]
  for (long i = 1; i < n - 1; i++) {
    tim = ts_a ? (1.0 - ts_a[i]) * creal(tstep) - I * creal(tstep) * ts_a[i] : tstep;
    cp = c / tim;
    d[i] = cp - 2.0;
    b[i] = cp * P(i) - (P(i + 1) - 2.0 * P(i) + P(i - 1)) - c2 * (P(i + 1) - P(i - 1)) - c3c * (P(i + 1) - P(i - 1));
  }
  tim = ts_a ? (1.0 - ts_a[0]) * creal(tstep) - I * creal(tstep) * ts_a[0] : tstep;
  cp = c / tim;
  switch (bc) {
    case 1: b[0] = cp * P(0) - (P(1) - 2.0 * P(0)) - c2 * P(1) - c3c * P(1); break;
    case 2: b[0] = cp * P(0) - (2.0 * P(1) - 2.0 * P(0)); break;
    default:
      b[0] = cp * P(0) - (P(1) - 2.0 * P(0) + P(n - 1)) - c2 * (P(1) - P(n - 1)) - c3c * (P(1) - P(n - 1));
      break;
  }
  d[0] = cp - 2.0;
  tim = ts_a ? (1.0 - ts_a[n - 1]) * creal(tstep) - I * creal(tstep) * ts_a[n - 1] : tstep;
  cp = c / tim;
  switch (bc) {
    case 1: b[n - 1] = cp * P(n - 1) - (P(n - 2) - 2.0 * P(n - 1)) + c2 * P(n - 2) + c3c * P(n - 2); break;
    case 2: b[n - 1] = cp * P(n - 1) - (2.0 * P(n - 2) - 2.0 * P(n - 1)); break;
    default:
      b[n - 1] = cp * P(n - 1) - (P(n - 2) - 2.0 * P(n - 1) + P(0)) - c2 * (P(0) - P(n - 2)) - c3c * (P(0) - P(n - 2));
      break;
  }
  d[n - 1] = cp - 2.0;
#undef P
  if (bc == 3) tri_cyclic2(n, d, b, psi0, c2 + c3c, str, w);
  else tri_system2(n, d, b, psi0, c2 + c3c, str);
}

/*
 * grid_wf_propagate_kinetic_cn (src/grid_wf_cn.c:65-79): x, y, z sweeps
 * (axes of length 1 skipped) with c = 4 i m h^2 / hbar, c2 = -i h k0,
 * c3 = +i m omega h / hbar (x) and -i m omega h / hbar (y); the rotation
 * coordinate is y = (j - ny/2) h - y0 for x lines and x = (i - nx/2) h - x0
 * for y lines.  lh != NULL enables the absorbing ramp.
 */
void gbo_cn_kinetic(cplx *psi, long nx, long ny, long nz, double step, double mass, cplx tstep, int bc, double kx0,
                    double ky0, double kz0, double omega, double x0, double y0, const long *lh) {
  const cplx c = 4.0 * I * mass * step * step / GBO_HBAR;
  const long nyz = ny * nz, nmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
  if (nx != 1) {
    const cplx c2 = -I * step * kx0, c3 = mass * omega * I * step / GBO_HBAR;
#pragma omp parallel
    {
      cplx *d = malloc(sizeof(cplx) * nmax), *b = malloc(sizeof(cplx) * nmax), *w = malloc(sizeof(cplx) * nmax);
      double *ta = lh ? malloc(sizeof(double) * nmax) : NULL;
#pragma omp for schedule(static)
      for (long jk = 0; jk < nyz; jk++) {
        const long j = jk / nz, k = jk % nz;
        const double y = ((double) (j - ny / 2)) * step - y0;
        if (ta)
          for (long i = 0; i < nx; i++) ta[i] = gbo_absorb(i, j, k, lh);
        cn_line(&psi[j * nz + k], nx, nyz, bc, c, tstep, c2, c3 * y, ta, d, b, w);
      }
      free(d);
      free(b);
      free(w);
      free(ta);
    }
  }
  if (ny != 1) {
    const cplx c2 = -I * step * ky0, c3 = -mass * omega * I * step / GBO_HBAR;
#pragma omp parallel
    {
      cplx *d = malloc(sizeof(cplx) * nmax), *b = malloc(sizeof(cplx) * nmax), *w = malloc(sizeof(cplx) * nmax);
      double *ta = lh ? malloc(sizeof(double) * nmax) : NULL;
#pragma omp for schedule(static)
      for (long ik = 0; ik < nx * nz; ik++) {
        const long i = ik / nz, k = ik % nz;
        const double x = ((double) (i - nx / 2)) * step - x0;
        if (ta)
          for (long j = 0; j < ny; j++) ta[j] = gbo_absorb(i, j, k, lh);
        cn_line(&psi[i * nyz + k], ny, nz, bc, c, tstep, c2, c3 * x, ta, d, b, w);
      }
      free(d);
      free(b);
      free(w);
      free(ta);
    }
  }
  if (nz != 1) {
    const cplx c2 = -I * step * kz0;
#pragma omp parallel
    {
      cplx *d = malloc(sizeof(cplx) * nmax), *b = malloc(sizeof(cplx) * nmax), *w = malloc(sizeof(cplx) * nmax);
      double *ta = lh ? malloc(sizeof(double) * nmax) : NULL;
#pragma omp for schedule(static)
      for (long ij = 0; ij < nx * ny; ij++) {
        const long i = ij / ny, j = ij % ny;
        if (ta)
          for (long k = 0; k < nz; k++) ta[k] = gbo_absorb(i, j, k, lh);
        cn_line(&psi[i * nyz + j * nz], nz, 1, bc, c, tstep, c2, 0.0, ta, d, b, w);
      }
      free(d);
      free(b);
      free(w);
      free(ta);
    }
  }
}

/*
 * 2nd-order CN step (src/grid_wf.c:526-530): V(dt/2), CN(dt), V(dt/2), with
 * cons = 0.  The potential is complex (vc) or real padded (vr) plus
 * g |psi|^2 taken from psi at each half-step.
 */
void gbo_cn_step(cplx *psi, long nx, long ny, long nz, double step, double mass, cplx time, int bc, double kx0,
                 double ky0, double kz0, double omega, double x0, double y0, const cplx *vc, const double *vr, double g,
                 const long *lh) {
  const cplx half = 0.5 * time;
  const int has_v = vc || vr || g != 0.0;
  if (has_v) gbo_potential(psi, nx, ny, nz, half, vc, vr, g, 0.0, lh);
  gbo_cn_kinetic(psi, nx, ny, nz, step, mass, time, bc, kx0, ky0, kz0, omega, x0, y0, lh);
  if (has_v) gbo_potential(psi, nx, ny, nz, half, vc, vr, g, 0.0, lh);
}

/* ----------------------------------------------------------- analysis */

/* src/cgrid.c:1610-1629 */
double gbo_norm(const cplx *psi, long nx, long ny, long nz, double step) {
  double s = 0.0;
  const long n = nx * ny * nz;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long q = 0; q < n; q++) s += creal(psi[q]) * creal(psi[q]) + cimag(psi[q]) * cimag(psi[q]);
  return s * step_factor(nx, ny, nz, step);
}

/* Boundary access of src/cgrid_bc.c:21-86 (bc 0 Dirichlet with value
 * `outside`, 1 Neumann, 2 periodic). */
static cplx bc_value(const cplx *a, long nx, long ny, long nz, long i, long j, long k, int bc, cplx outside) {
  if (i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz) return a[(i * ny + j) * nz + k];
  if (bc == 0) return outside;
  if (bc == 1) {
    if (i < 0) i = -i;
    if (i > nx - 1) i = 2 * nx - i - 2;
    if (j < 0) j = -j;
    if (j > ny - 1) j = 2 * ny - j - 2;
    if (k < 0) k = -k;
    if (k > nz - 1) k = 2 * nz - k - 2;
    if (i < 0 || i >= nx) i = 0;
    if (j < 0 || j >= ny) j = 0;
    if (k < 0 || k >= nz) k = 0;
    return a[(i * ny + j) * nz + k];
  }
  i %= nx;
  if (i < 0) i += nx;
  j %= ny;
  if (j < 0) j += ny;
  k %= nz;
  if (k < 0) k += nz;
  return a[(i * ny + j) * nz + k];
}

/* src/cgrid_diff.c:303-336 (7-point Laplacian, reference summation order) */
void gbo_fd_laplace(const cplx *a, cplx *out, long nx, long ny, long nz, double step, int bc, cplx outside) {
  const double inv = 1.0 / (step * step);
#pragma omp parallel for schedule(static)
  for (long ij = 0; ij < nx * ny; ij++) {
    const long i = ij / ny, j = ij % ny;
    for (long k = 0; k < nz; k++)
      out[ij * nz + k] =
          inv * (-6.0 * bc_value(a, nx, ny, nz, i, j, k, bc, outside) + bc_value(a, nx, ny, nz, i, j, k + 1, bc, outside) +
                 bc_value(a, nx, ny, nz, i, j, k - 1, bc, outside) + bc_value(a, nx, ny, nz, i, j + 1, k, bc, outside) +
                 bc_value(a, nx, ny, nz, i, j - 1, k, bc, outside) + bc_value(a, nx, ny, nz, i + 1, j, k, bc, outside) +
                 bc_value(a, nx, ny, nz, i - 1, j, k, bc, outside));
  }
}

/* grid_wf_kinetic_energy_cn (src/grid_wf_cn.c:37-49) */
double gbo_kinetic_energy_fd(const cplx *psi, long nx, long ny, long nz, double step, double mass, int bc, cplx outside) {
  const long n = nx * ny * nz;
  cplx *lap = malloc(sizeof(cplx) * n);
  double sr = 0.0;
  gbo_fd_laplace(psi, lap, nx, ny, nz, step, bc, outside);
  const double f = -GBO_HBAR * GBO_HBAR / (2.0 * mass);
#pragma omp parallel for reduction(+ : sr) schedule(static)
  for (long q = 0; q < n; q++) sr += creal(conj(psi[q]) * (lap[q] * f));
  free(lap);
  return sr * step_factor(nx, ny, nz, step);
}

/* grid_wf_kinetic_energy_fft (src/grid_wf_fft.c:119-129) with
 * cgrid_fft_laplace_expectation_value (src/cgrid_diff.c:817-879): no k0 */
double gbo_kinetic_energy_fft(const cplx *psi, long nx, long ny, long nz, double step, double mass) {
  const long n = nx * ny * nz;
  cplx *w = malloc(sizeof(cplx) * n);
  memcpy(w, psi, sizeof(cplx) * n);
  gbo_fft3d(w, nx, ny, nz, -1);
  const double lx = 2.0 * M_PI / (step * (double) nx), ly = 2.0 * M_PI / (step * (double) ny),
               lz = 2.0 * M_PI / (step * (double) nz);
  double sum = 0.0;
#pragma omp parallel for reduction(+ : sum) schedule(static)
  for (long ij = 0; ij < nx * ny; ij++) {
    const long i = ij / ny, j = ij % ny;
    const double kx = (i <= nx / 2 ? (double) i : (double) (i - nx)) * lx;
    const double ky = (j <= ny / 2 ? (double) j : (double) (j - ny)) * ly;
    double ssum = 0.0;
    for (long k = 0; k < nz; k++) {
      const double kz = (k <= nz / 2 ? (double) k : (double) (k - nz)) * lz;
      const cplx v = w[ij * nz + k];
      ssum -= (kx * kx + ky * ky + kz * kz) * (creal(v) * creal(v) + cimag(v) * cimag(v));
    }
    sum += ssum;
  }
  free(w);
  const double norm2 = step_factor(nx, ny, nz, step) / (double) n;
  return -GBO_HBAR * GBO_HBAR / (2.0 * mass) * (sum * norm2);
}

/* grid_grid_expectation_value (src/ngrid.c:355-378), real padded V */
double gbo_potential_energy(const cplx *psi, const double *vr, long nx, long ny, long nz, double step) {
  const long nz2 = 2 * (nz / 2 + 1);
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long ij = 0; ij < nx * ny; ij++)
    for (long k = 0; k < nz; k++) {
      const cplx p = psi[ij * nz + k];
      s += (creal(p) * creal(p) + cimag(p) * cimag(p)) * vr[ij * nz2 + k];
    }
  return s * step_factor(nx, ny, nz, step);
}
