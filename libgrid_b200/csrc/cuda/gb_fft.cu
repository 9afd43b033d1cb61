// C ABI for the FFT / split-operator path, kinetic-factor tables, the
// standalone pointwise kinetic and potential factors, and the deterministic
// partial-sum finisher.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gb_fft_impl.cuh"
#include "gb_internal_cuda.h"

using gbfft::PassArgs;

// ---------------------------------------------------------- kinetic tables

// Per-axis kinetic quantities, one thread per (axis, index):
//   k = (i <= n/2 ? i : i - n) * l - k0,   l = 2 pi / (n step)
//   ksq = k^2, fac = exp(tm * k^2)
// (reference src/grid_wf_fft.c:152-190).
template <typename T>
__global__ void k_kin_tables(C2<T> *fac, double *ksq, long nx, long ny, long nz, double lx, double ly, double lz,
                             double kx0, double ky0, double kz0, double tm_re, double tm_im) {
  const long tot = nx + ny + nz;
  for (long t = blockIdx.x * (long) blockDim.x + threadIdx.x; t < tot; t += (long) gridDim.x * blockDim.x) {
    long n, i;
    double l, k0;
    if (t < nx) {
      n = nx;
      i = t;
      l = lx;
      k0 = kx0;
    } else if (t < nx + ny) {
      n = ny;
      i = t - nx;
      l = ly;
      k0 = ky0;
    } else {
      n = nz;
      i = t - nx - ny;
      l = lz;
      k0 = kz0;
    }
    const double k = (i <= n / 2 ? (double) i : (double) (i - n)) * l - k0;
    const double k2 = k * k;
    ksq[t] = k2;
    double s, c;
    sincos(tm_im * k2, &s, &c);
    const double m = (tm_re != 0.0) ? exp(tm_re * k2) : 1.0;
    fac[t] = C2<T>{(T) (m * c), (T) (m * s)};
  }
}

struct KinKey {
  long nx, ny, nz;
  double step, tm_re, tm_im, kx0, ky0, kz0;
  int prec, unshifted;
};
static KinKey g_kin_key;
static bool g_kin_valid = false;

int gb__kin_tables(const gb_geom *g, const gb_kinetic *kin, int unshifted, GbKinTables *out) {
  const long tot = g->nx + g->ny + g->nz;
  const size_t facb = (size_t) tot * 16, sqb = (size_t) tot * 8;
  unsigned char *base = (unsigned char *) gb__scratch(GB_SCR_KIN, facb + sqb);
  if (!base) return gb_last_error();
  KinKey key;
  memset(&key, 0, sizeof(key));
  key.nx = g->nx;
  key.ny = g->ny;
  key.nz = g->nz;
  key.step = g->step;
  key.tm_re = unshifted ? 0.0 : kin->tm_re;
  key.tm_im = unshifted ? 0.0 : kin->tm_im;
  key.kx0 = unshifted ? 0.0 : kin->kx0;
  key.ky0 = unshifted ? 0.0 : kin->ky0;
  key.kz0 = unshifted ? 0.0 : kin->kz0;
  key.prec = g->prec;
  key.unshifted = unshifted;
  double *ksq = (double *) (base + facb);
  const size_t esz = (g->prec == GB_FP32) ? 8 : 16;
  if (!g_kin_valid || memcmp(&key, &g_kin_key, sizeof(key)) != 0) {
    const double lx = 2.0 * M_PI / (g->step * (double) g->nx);
    const double ly = 2.0 * M_PI / (g->step * (double) g->ny);
    const double lz = 2.0 * M_PI / (g->step * (double) g->nz);
    const unsigned nb = (unsigned) ((tot + 255) / 256);
    if (g->prec == GB_FP32)
      k_kin_tables<float><<<nb, 256, 0, gb__stream()>>>((float2 *) base, ksq, g->nx, g->ny, g->nz, lx, ly, lz,
                                                         key.kx0, key.ky0, key.kz0, key.tm_re, key.tm_im);
    else
      k_kin_tables<double><<<nb, 256, 0, gb__stream()>>>((double2 *) base, ksq, g->nx, g->ny, g->nz, lx, ly, lz,
                                                          key.kx0, key.ky0, key.kz0, key.tm_re, key.tm_im);
    GB_CHECK_LAUNCH("kinetic tables");
    g_kin_key = key;
    g_kin_valid = true;
  }
  out->kfac[0] = base;
  out->kfac[1] = base + esz * (size_t) g->nx;
  out->kfac[2] = base + esz * (size_t) (g->nx + g->ny);
  out->ksq[0] = ksq;
  out->ksq[1] = ksq + g->nx;
  out->ksq[2] = ksq + g->nx + g->ny;
  return 0;
}

// The same tables for one geometry into caller-owned buffers: fac holds
// nx + ny + nz factors in the storage precision, ksq as many k^2 values.
int gb__kin_tables_at(void *fac, double *ksq, const gb_geom *g, const gb_kinetic *kin) {
  const long tot = g->nx + g->ny + g->nz;
  const double lx = 2.0 * M_PI / (g->step * (double) g->nx);
  const double ly = 2.0 * M_PI / (g->step * (double) g->ny);
  const double lz = 2.0 * M_PI / (g->step * (double) g->nz);
  const unsigned nb = (unsigned) ((tot + 255) / 256);
  if (g->prec == GB_FP32)
    k_kin_tables<float><<<nb, 256, 0, gb__stream()>>>((float2 *) fac, ksq, g->nx, g->ny, g->nz, lx, ly, lz, kin->kx0,
                                                       kin->ky0, kin->kz0, kin->tm_re, kin->tm_im);
  else
    k_kin_tables<double><<<nb, 256, 0, gb__stream()>>>((double2 *) fac, ksq, g->nx, g->ny, g->nz, lx, ly, lz,
                                                        kin->kx0, kin->ky0, kin->kz0, kin->tm_re, kin->tm_im);
  GB_CHECK_LAUNCH("kinetic tables");
  return 0;
}

// ------------------------------------------------------ partial-sum finisher

__global__ void k_sum_partials(const double *__restrict__ p, long n, double *out) {
  __shared__ double sbuf[32];
  double s = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) s += p[i];
  double r = gbfft::block_sum<1024>(s, sbuf);
  if (threadIdx.x == 0) *out = r;
}

int gb__sum_partials(const double *partial, long n, double *out_host) {
  double *res = (double *) gb__result_slot();
  if (!res) return gb_last_error();
  k_sum_partials<<<1, 1024, 0, gb__stream()>>>(partial, n, res);
  GB_CHECK_LAUNCH("sum partials");
  return gb__read_result(out_host, sizeof(double));
}

// ------------------------------------------------- standalone pointwise ops

// psi_k *= exp(tm |k - k0|^2) (zero beyond the cutoff), evaluated per point
// as in src/grid_wf_fft.c:173-190 / :238-259.
template <typename T>
__global__ void k_kinetic_multiply(C2<T> *psi, long nx, long ny, long nz, double lx, double ly, double lz, gb_kinetic kin) {
  const long n = nx * ny * nz;
  for (long g = blockIdx.x * (long) blockDim.x + threadIdx.x; g < n; g += (long) gridDim.x * blockDim.x) {
    const long k = g % nz, ij = g / nz, j = ij % ny, i = ij / ny;
    const double kx = (i <= nx / 2 ? (double) i : (double) (i - nx)) * lx - kin.kx0;
    const double ky = (j <= ny / 2 ? (double) j : (double) (j - ny)) * ly - kin.ky0;
    const double kz = (k <= nz / 2 ? (double) k : (double) (k - nz)) * lz - kin.kz0;
    const double tot = kx * kx + ky * ky + kz * kz;
    C2<T> v = psi[g];
    if (kin.cutoff && !(tot < kin.kmax2)) {
      v = C2<T>{(T) 0, (T) 0};
    } else {
      C2<T> f = cexp_phase<T>(kin.tm_re * tot, kin.tm_im * tot, kin.tm_re != 0.0);
      v = cmul(v, f);
      if (kin.scale != 1.0) v = cscale(v, (T) kin.scale);
    }
    psi[g] = v;
  }
}

template <typename T> __global__ void k_potential_multiply(C2<T> *psi, PassArgs a) {
  const long n = a.nx * a.ny * a.nz;
  for (long g = blockIdx.x * (long) blockDim.x + threadIdx.x; g < n; g += (long) gridDim.x * blockDim.x) {
    const long k = g % a.nz, ij = g / a.nz, j = ij % a.ny, i = ij / a.ny;
    const long vidx = (i * a.ny + j) * a.pot.vrow + k;
    psi[g] = gbfft::pot_factor_apply<T>(psi[g], i, j, k, (unsigned) vidx, a);
  }
}

// dst = src * (-k^2) (src/cgrid_diff.c:601-665) or src * i k_axis
// (src/cgrid_diff.c:454-599), with the reference's own expressions for k.
template <typename T>
__global__ void k_kspace(int op, C2<T> *dst, const C2<T> *src, long nx, long ny, long nz, double step) {
  const long n = nx * ny * nz;
  const double lx = 2.0 * M_PI / (step * (double) nx);
  const double ly = 2.0 * M_PI / (step * (double) ny);
  const double lz = 2.0 * M_PI / (step * (double) nz);
  for (long g = blockIdx.x * (long) blockDim.x + threadIdx.x; g < n; g += (long) gridDim.x * blockDim.x) {
    const long k = g % nz, ij = g / nz, j = ij % ny, i = ij / ny;
    const C2<T> v = src[g];
    C2<T> r;
    if (op == GB_K_LAPLACE) {
      const double kx = (i <= nx / 2 ? (double) i : (double) (i - nx)) * lx;
      const double ky = (j <= ny / 2 ? (double) j : (double) (j - ny)) * ly;
      const double kz = (k <= nz / 2 ? (double) k : (double) (k - nz)) * lz;
      const T f = (T) (-(kx * kx + ky * ky + kz * kz));
      r = cscale(v, f);
    } else {
      double kk;
      if (op == GB_K_GRADIENT_X)
        kk = 2.0 * M_PI * (double) (i <= nx / 2 ? i : i - nx) / ((double) nx * step);
      else if (op == GB_K_GRADIENT_Y)
        kk = 2.0 * M_PI * (double) (j <= ny / 2 ? j : j - ny) / ((double) ny * step);
      else
        kk = (k <= nz / 2 ? (double) k : (double) (k - nz)) * lz;
      // v * (i kk)
      r = C2<T>{(T) (-(double) v.y * kk), (T) ((double) v.x * kk)};
    }
    dst[g] = r;
  }
}

static unsigned pw_blocks(long n) {
  long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned) (b < 1 ? 1 : b);
}

// ---------------------------------------------------------------- C ABI

// The line-pass FFT takes power-of-two lengths up to 4096 on every axis of
// length > 1 and grids below 2^31 points (32-bit in-tile offsets).
static int fft_geom_ok(const gb_geom *g) {
  const long n[3] = {g->nx, g->ny, g->nz};
  for (int d = 0; d < 3; d++)
    if (n[d] < 1 || (n[d] > 1 && ((n[d] & (n[d] - 1)) != 0 || n[d] > 4096)))
      return gb__set_error(1002, "FFT line length must be a power of two in [2, 4096]");
  if ((double) g->nx * (double) g->ny * (double) g->nz >= 2147483648.0)
    return gb__set_error(1006, "FFT grid must have fewer than 2^31 points");
  return 0;
}

extern "C" int gb_fft3d(void *data, const gb_geom *g, int sign, double scale) {
  if (fft_geom_ok(g)) return gb_last_error();
  if (g->prec == GB_FP32) return gb__fft3d_t<float>(data, g, sign, scale);
  return gb__fft3d_t<double>(data, g, sign, scale);
}

extern "C" int gb_split_step(void *psi, const gb_geom *g, const gb_kinetic *kin, const gb_potential *pot) {
  if (fft_geom_ok(g)) return gb_last_error();
  if (g->prec == GB_FP32) return gb__split_step_t<float>(psi, g, kin, pot);
  return gb__split_step_t<double>(psi, g, kin, pot);
}

extern "C" int gb_split_steps(void *psi, const gb_geom *g, const gb_kinetic *kin, const gb_potential *pot, int nsteps) {
  if (fft_geom_ok(g)) return gb_last_error();
  if (g->prec == GB_FP32) return gb__split_steps_t<float>(psi, g, kin, pot, nsteps);
  return gb__split_steps_t<double>(psi, g, kin, pot, nsteps);
}

extern "C" int gb_fft_ksq_sum(const void *psi, void *work, const gb_geom *g, double *out) {
  if (fft_geom_ok(g)) return gb_last_error();
  if (g->prec == GB_FP32) return gb__ksq_sum_t<float>(psi, work, g, out);
  return gb__ksq_sum_t<double>(psi, work, g, out);
}

// Self-test of the phase sine/cosine: gb_sincos against the CUDA library
// sincos, element by element.
__global__ void k_sincos_check(const double *x, long n, double *err) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s0, c0, s1, c1;
  sincos(x[i], &s0, &c0);
  gb_sincos(x[i], &s1, &c1);
  err[2 * i] = fabs(s1 - s0);
  err[2 * i + 1] = fabs(c1 - c0);
}

extern "C" int gb_sincos_selftest(const double *x_host, long n, double *max_err) {
  if (n <= 0) return gb__set_error(1020, "sincos self-test: empty input");
  double *d = nullptr;
  if (cudaMalloc(&d, (size_t) n * 3 * sizeof(double)) != cudaSuccess) return gb__set_error(2, "sincos self-test");
  cudaStream_t st = gb__stream();
  cudaMemcpyAsync(d, x_host, (size_t) n * sizeof(double), cudaMemcpyHostToDevice, st);
  k_sincos_check<<<(unsigned) ((n + 255) / 256), 256, 0, st>>>(d, n, d + n);
  double *h = (double *) malloc((size_t) n * 2 * sizeof(double));
  cudaMemcpyAsync(h, d + n, (size_t) n * 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(d);
  if (e != cudaSuccess) {
    free(h);
    return gb__set_error((int) e, "sincos self-test");
  }
  max_err[0] = max_err[1] = 0.0;
  for (long i = 0; i < n; i++) {
    if (h[2 * i] > max_err[0]) max_err[0] = h[2 * i];
    if (h[2 * i + 1] > max_err[1]) max_err[1] = h[2 * i + 1];
  }
  free(h);
  gb__count_launch();
  return 0;
}

extern "C" int gb_kspace_op(int op, void *dst, const void *src, const gb_geom *g) {
  const long n = g->nx * g->ny * g->nz;
  if (g->prec == GB_FP32)
    k_kspace<float><<<pw_blocks(n), 256, 0, gb__stream()>>>(op, (float2 *) dst, (const float2 *) src, g->nx, g->ny, g->nz, g->step);
  else
    k_kspace<double><<<pw_blocks(n), 256, 0, gb__stream()>>>(op, (double2 *) dst, (const double2 *) src, g->nx, g->ny, g->nz,
                                                             g->step);
  GB_CHECK_LAUNCH("kspace op");
  return 0;
}

extern "C" int gb_kinetic_multiply(void *psi, const gb_geom *g, const gb_kinetic *kin) {
  const double lx = 2.0 * M_PI / (g->step * (double) g->nx);
  const double ly = 2.0 * M_PI / (g->step * (double) g->ny);
  const double lz = 2.0 * M_PI / (g->step * (double) g->nz);
  const long n = g->nx * g->ny * g->nz;
  if (g->prec == GB_FP32)
    k_kinetic_multiply<float><<<pw_blocks(n), 256, 0, gb__stream()>>>((float2 *) psi, g->nx, g->ny, g->nz, lx, ly, lz, *kin);
  else
    k_kinetic_multiply<double><<<pw_blocks(n), 256, 0, gb__stream()>>>((double2 *) psi, g->nx, g->ny, g->nz, lx, ly, lz, *kin);
  GB_CHECK_LAUNCH("kinetic multiply");
  return 0;
}

extern "C" int gb_potential_multiply(void *psi, const gb_geom *g, const gb_potential *pot) {
  if ((double) g->nx * (double) g->ny * (double) (pot->vrow > g->nz ? pot->vrow : g->nz) >= 4294967296.0)
    return gb__set_error(1006, "potential grid must have fewer than 2^32 elements");
  PassArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = g->nx;
  a.ny = g->ny;
  a.nz = g->nz;
  a.pot = *pot;
  const long n = g->nx * g->ny * g->nz;
  if (g->prec == GB_FP32) k_potential_multiply<float><<<pw_blocks(n), 256, 0, gb__stream()>>>((float2 *) psi, a);
  else k_potential_multiply<double><<<pw_blocks(n), 256, 0, gb__stream()>>>((double2 *) psi, a);
  GB_CHECK_LAUNCH("potential multiply");
  return 0;
}
