// Pointwise grid algebra and deterministic FP64 reductions.
//
// Replaces the reference's per-operation SIMT kernels (src/cgrid-cuda2.cu,
// src/rgrid-cuda2.cu, src/ngrid-cuda2.cu, src/grid_wf-cuda2.cu:111-176) and
// its reductions, which sum each 512-thread block serially in thread 0 and
// finish on the host (src/cgrid-cuda2.cu:975-996).  Here each reduction is a
// grid-stride pass with a fixed per-thread order, a fixed shuffle tree per
// block and a fixed-order finish over the block partials, so the result does
// not depend on scheduling.
#include <stdio.h>
#include <string.h>

#include "gb_common.cuh"
#include "gb_internal_cuda.h"

namespace {

constexpr int kThreads = 256;

unsigned blocks_for(size_t n) {
  size_t b = (n + kThreads - 1) / kThreads;
  if (b > 148u * 16u) b = 148u * 16u;
  if (b < 1) b = 1;
  return (unsigned) b;
}

template <typename T>
__global__ void k_complex_op(int op, C2<T> *c, const C2<T> *a, const C2<T> *b, size_t n, double dre, double dim) {
  const C2<T> d{(T) dre, (T) dim};
  for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x) {
    switch (op) {
      case GB_OP_CONST: c[i] = d; break;
      case GB_OP_SCALE: c[i] = cmul(c[i], d); break;
      case GB_OP_ADD_CONST: c[i] = cadd(c[i], d); break;
      case GB_OP_SUM: c[i] = cadd(a[i], b[i]); break;
      case GB_OP_DIFF: c[i] = csub(a[i], b[i]); break;
      case GB_OP_PRODUCT: c[i] = cmul(a[i], b[i]); break;
      case GB_OP_CONJ_PRODUCT: c[i] = cconjmul(a[i], b[i]); break;
      case GB_OP_ADD_SCALED: c[i] = cadd(c[i], cmul(d, a[i])); break;
      case GB_OP_ADD_SCALED_PRODUCT: c[i] = cadd(c[i], cmul(cmul(d, a[i]), b[i])); break;
      case GB_OP_COPY: c[i] = a[i]; break;
    }
  }
}

template <typename T> __global__ void k_real_op(int op, T *c, const T *a, const T *b, size_t n, double dd) {
  const T d = (T) dd;
  for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x) {
    switch (op) {
      case GB_OP_CONST: c[i] = d; break;
      case GB_OP_SCALE: c[i] = c[i] * d; break;
      case GB_OP_ADD_CONST: c[i] = c[i] + d; break;
      case GB_OP_SUM: c[i] = a[i] + b[i]; break;
      case GB_OP_DIFF: c[i] = a[i] - b[i]; break;
      case GB_OP_PRODUCT: c[i] = a[i] * b[i]; break;
      case GB_OP_ADD_SCALED: c[i] = c[i] + d * a[i]; break;
      case GB_OP_ADD_SCALED_PRODUCT: c[i] = c[i] + d * a[i] * b[i]; break;
      case GB_OP_COPY: c[i] = a[i]; break;
    }
  }
}

// Mixed complex / padded-real ops over the logical (nx, ny, nz) points.
template <typename TC, typename TR>
__global__ void k_mixed(int op, C2<TC> *c, TR *r, const TR *r1, long nxy, long nz, long rrow) {
  const size_t n = (size_t) nxy * nz;
  for (size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x; g < n; g += (size_t) gridDim.x * blockDim.x) {
    const size_t ij = g / nz, k = g - ij * nz;
    const size_t ri = ij * rrow + k;
    switch (op) {
      case GB_MIX_REAL_TO_COMPLEX_RE: c[g] = C2<TC>{(TC) r[ri], (TC) 0}; break;
      case GB_MIX_PRODUCT_NORM: {
        const C2<TC> v = c[g];
        r[ri] = r1[ri] * (TR) (v.x * v.x + v.y * v.y);
      } break;
      case GB_MIX_PRODUCT_COMPLEX_REAL: c[g] = cscale(c[g], (TC) r[ri]); break;
      case GB_MIX_DENSITY: {
        const C2<TC> v = c[g];
        r[ri] = (TR) (v.x * v.x + v.y * v.y);
      } break;
    }
  }
}

// src/grid_wf.c:185-203 (ramp) and :745-754 (blend)
template <typename T>
__global__ void k_merge(C2<T> *dst, const C2<T> *wr, const C2<T> *wi, long nx, long ny, long nz, long lx, long hx,
                        long ly, long hy, long lz, long hz) {
  const size_t n = (size_t) nx * ny * nz;
  for (size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x; g < n; g += (size_t) gridDim.x * blockDim.x) {
    const long k = (long) (g % nz), ij = (long) (g / nz), j = ij % ny, i = ij / ny;
    double t = 0.0;
    if (i < lx) t += (double) (lx - i) / (double) lx;
    else if (i > hx) t += (double) (i - hx) / (double) lx;
    if (j < ly) t += (double) (ly - j) / (double) ly;
    else if (j > hy) t += (double) (j - hy) / (double) ly;
    if (k < lz) t += (double) (lz - k) / (double) lz;
    else if (k > hz) t += (double) (k - hz) / (double) lz;
    t *= 2.0 / 3.0;
    const double al = t > 1.0 ? 1.0 : t;
    const C2<T> a = wr[g], b = wi[g];
    dst[g] = C2<T>{(T) ((1.0 - al) * a.x + al * b.x), (T) ((1.0 - al) * a.y + al * b.y)};
  }
}

// FFT convolution in k-space (src/cgrid.c:1912-1944, src/rgrid.c:1848-1878):
// c = a * b with the sign (-1)^(i + j + k) that moves the result's origin to
// the grid centre.  nzc complex entries per (i, j) row: nz for a cgrid,
// nz2 / 2 for the half spectrum of a padded rgrid.
template <typename T>
__global__ void k_fft_convolute(C2<T> *c, const C2<T> *a, const C2<T> *b, long ny, long nzc, size_t n) {
  for (size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x; g < n; g += (size_t) gridDim.x * blockDim.x) {
    const long k = (long) (g % nzc), ij = (long) (g / nzc), j = ij % ny, i = ij / ny;
    const C2<T> p = cmul(a[g], b[g]);
    c[g] = ((i + j + k) & 1) ? C2<T>{-p.x, -p.y} : p;
  }
}

// Trilinear interpolation of a source grid at the destination's points
// (cgrid_extrapolate / rgrid_extrapolate, src/cgrid.c:2067-2151,
// src/rgrid.c:2208-2300): the same coordinate arithmetic, the same boundary
// values for the corners outside the source (Dirichlet constant, Neumann
// mirror, periodic wrap) and the same summation order as the reference's
// cgrid_value (nested) and rgrid_value (eight products, left to right), with
// every product and sum rounded separately.
struct InterpArgs {
  long dnx, dny, dnz, drow;
  double dstep, dx0, dy0, dz0;
  long snx, sny, snz, srow;
  double sstep, sx0, sy0, sz0;
  int bc;
  double out_re, out_im;
};

__device__ __forceinline__ bool interp_map(long &i, long n, int bc) {
  if (i >= 0 && i < n) return true;
  if (bc == GB_BC_DIRICHLET) return false;
  if (bc == GB_BC_PERIODIC) {
    i %= n;
    if (i < 0) i += n;
    return true;
  }
  if (i < 0) i = -i;
  if (i > n - 1) i = 2 * n - i - 2;
  if (i < 0 || i >= n) i = 0;
  return true;
}

// Value of the source at (i, j, k), with the boundary rule outside.
template <bool REAL>
__device__ __forceinline__ double2 interp_fetch(const void *src, long i, long j, long k, const InterpArgs &a) {
  if (i < 0 || i >= a.snx || j < 0 || j >= a.sny || k < 0 || k >= a.snz) {
    if (a.bc == GB_BC_DIRICHLET || !interp_map(i, a.snx, a.bc) || !interp_map(j, a.sny, a.bc) ||
        !interp_map(k, a.snz, a.bc))
      return make_double2(a.out_re, REAL ? 0.0 : a.out_im);
  }
  const size_t q = (size_t) (i * a.sny + j) * a.srow + k;
  if (REAL) return make_double2(((const double *) src)[q], 0.0);
  return ((const double2 *) src)[q];
}

// index and fraction along one axis (src/cgrid.c:2074-2078)
__device__ __forceinline__ long interp_axis(double c, double x0, double step, long n, double &f) {
  double x = __ddiv_rn(__dadd_rn(c, x0), step);
  long i = (long) x;
  if (x < 0) i--;
  f = __dsub_rn(x, (double) i);
  return i + n / 2;
}

template <bool REAL> __global__ void k_interp(void *dst, const void *src, InterpArgs a) {
  const size_t n = (size_t) a.dnx * a.dny * a.dnz;
  for (size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x; g < n; g += (size_t) gridDim.x * blockDim.x) {
    const long kd = (long) (g % a.dnz), ij = (long) (g / a.dnz), jd = ij % a.dny, id = ij / a.dny;
    const double xc = __dsub_rn(__dmul_rn((double) (id - a.dnx / 2), a.dstep), a.dx0);
    const double yc = __dsub_rn(__dmul_rn((double) (jd - a.dny / 2), a.dstep), a.dy0);
    const double zc = __dsub_rn(__dmul_rn((double) (kd - a.dnz / 2), a.dstep), a.dz0);
    double x, y, z;
    const long i = interp_axis(xc, a.sx0, a.sstep, a.snx, x);
    const long j = interp_axis(yc, a.sy0, a.sstep, a.sny, y);
    const long k = interp_axis(zc, a.sz0, a.sstep, a.snz, z);
    const double2 f000 = interp_fetch<REAL>(src, i, j, k, a), f100 = interp_fetch<REAL>(src, i + 1, j, k, a),
                  f010 = interp_fetch<REAL>(src, i, j + 1, k, a), f001 = interp_fetch<REAL>(src, i, j, k + 1, a),
                  f110 = interp_fetch<REAL>(src, i + 1, j + 1, k, a), f101 = interp_fetch<REAL>(src, i + 1, j, k + 1, a),
                  f011 = interp_fetch<REAL>(src, i, j + 1, k + 1, a),
                  f111 = interp_fetch<REAL>(src, i + 1, j + 1, k + 1, a);
    const double omx = __dsub_rn(1.0, x), omy = __dsub_rn(1.0, y), omz = __dsub_rn(1.0, z);
    const size_t q = (size_t) (id * a.dny + jd) * a.drow + kd;
    if (REAL) {
      // omx omy omz f000 + x omy omz f100 + omx y omz f010 + omx omy z f001
      //   + x y omz f110 + x omy z f101 + omx y z f011 + x y z f111
      auto t3 = [](double p, double q2, double r, double f) { return __dmul_rn(__dmul_rn(__dmul_rn(p, q2), r), f); };
      double s = t3(omx, omy, omz, f000.x);
      s = __dadd_rn(s, t3(x, omy, omz, f100.x));
      s = __dadd_rn(s, t3(omx, y, omz, f010.x));
      s = __dadd_rn(s, t3(omx, omy, z, f001.x));
      s = __dadd_rn(s, t3(x, y, omz, f110.x));
      s = __dadd_rn(s, t3(x, omy, z, f101.x));
      s = __dadd_rn(s, t3(omx, y, z, f011.x));
      s = __dadd_rn(s, t3(x, y, z, f111.x));
      ((double *) dst)[q] = s;
    } else {
      // omx (omy (omz f000 + z f001) + y (omz f010 + z f011))
      //   + x (omy (omz f100 + z f101) + y (omz f110 + z f111)), per component
      auto lin = [](double w0, double a0, double w1, double a1) { return __dadd_rn(__dmul_rn(w0, a0), __dmul_rn(w1, a1)); };
      double2 r;
      r.x = lin(omx, lin(omy, lin(omz, f000.x, z, f001.x), y, lin(omz, f010.x, z, f011.x)), x,
                lin(omy, lin(omz, f100.x, z, f101.x), y, lin(omz, f110.x, z, f111.x)));
      r.y = lin(omx, lin(omy, lin(omz, f000.y, z, f001.y), y, lin(omz, f010.y, z, f011.y)), x,
                lin(omy, lin(omz, f100.y, z, f101.y), y, lin(omz, f110.y, z, f111.y)));
      ((double2 *) dst)[q] = r;
    }
  }
}

// Padded real rows (nz2 scalars = nz/2 + 1 complex) <-> complex grids.
__global__ void k_r2c_pack(double2 *r, const double2 *c, long nx, long ny, long nz) {
  const long nh = nz / 2 + 1;
  const size_t n = (size_t) nx * ny * nh;
  for (size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x; g < n; g += (size_t) gridDim.x * blockDim.x) {
    const size_t ij = g / nh, k = g - ij * nh;
    r[ij * nh + k] = c[ij * nz + k];
  }
}

__global__ void k_c2r_unpack(double2 *c, const double2 *r, long nx, long ny, long nz) {
  const long nh = nz / 2 + 1;
  const size_t n = (size_t) nx * ny * nz;
  for (size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x; g < n; g += (size_t) gridDim.x * blockDim.x) {
    const long k = (long) (g % nz), ij = (long) (g / nz), j = ij % ny, i = ij / ny;
    double2 v;
    if (k < nh) {
      v = r[ij * nh + k];
    } else {
      const long ii = (nx - i) % nx, jj = (ny - j) % ny, kk = nz - k;
      const double2 w = r[(ii * ny + jj) * nh + kk];
      v = make_double2(w.x, -w.y);
    }
    c[g] = v;
  }
}

__global__ void k_real_part(double *r, const double2 *c, long nxy, long nz, long rrow) {
  const size_t n = (size_t) nxy * nz;
  for (size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x; g < n; g += (size_t) gridDim.x * blockDim.x) {
    const size_t ij = g / nz, k = g - ij * nz;
    r[ij * rrow + k] = c[g].x;
  }
}

// ------------------------------------------------------------- reductions

template <int THREADS> __device__ __forceinline__ void block_sum2(double &x, double &y, double *sb) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    x += __shfl_down_sync(0xffffffffu, x, off);
    y += __shfl_down_sync(0xffffffffu, y, off);
  }
  constexpr int NW = THREADS / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    sb[2 * w] = x;
    sb[2 * w + 1] = y;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sx = 0.0, sy = 0.0;
    for (int q = 0; q < NW; q++) {
      sx += sb[2 * q];
      sy += sb[2 * q + 1];
    }
    x = sx;
    y = sy;
  }
}

// Contribution of element g (row ij, column k) to a reduction op.
template <int OP, typename TA, typename TB> struct RedTerm {
  static __device__ __forceinline__ double2 at(size_t g, const void *av, const void *bv, long nz, long arow, long brow,
                                               long nx, long ny, double step) {
    if constexpr (OP == GB_RED_SUM) {
      const C2<TA> a = ((const C2<TA> *) av)[g];
      return double2{(double) a.x, (double) a.y};
    } else if constexpr (OP == GB_RED_NORM2) {
      const C2<TA> a = ((const C2<TA> *) av)[g];
      return double2{(double) a.x * (double) a.x + (double) a.y * (double) a.y, 0.0};
    } else if constexpr (OP == GB_RED_CONJ_PRODUCT) {
      const C2<TA> a = ((const C2<TA> *) av)[g];
      const C2<TB> b = ((const C2<TB> *) bv)[g];
      const double ar = a.x, ai = a.y, br = b.x, bi = b.y;
      return double2{ar * br + ai * bi, ar * bi - ai * br};
    } else if constexpr (OP == GB_RED_EXPECT_COMPLEX) {
      const C2<TA> a = ((const C2<TA> *) av)[g];
      const C2<TB> b = ((const C2<TB> *) bv)[g];
      const double w = (double) a.x * (double) a.x + (double) a.y * (double) a.y;
      return double2{w * (double) b.x, w * (double) b.y};
    } else if constexpr (OP == GB_RED_EXPECT_REAL) {
      const size_t ij = g / (size_t) nz, k = g - ij * (size_t) nz;
      const C2<TA> a = ((const C2<TA> *) av)[g];
      const double w = (double) a.x * (double) a.x + (double) a.y * (double) a.y;
      return double2{w * (double) ((const TB *) bv)[ij * brow + k], 0.0};
    } else if constexpr (OP == GB_RED_REAL_SUM) {
      const size_t ij = g / (size_t) nz, k = g - ij * (size_t) nz;
      return double2{(double) ((const TA *) av)[ij * arow + k], 0.0};
    } else {
      // GB_RED_KSQ_NORM2 (src/cgrid_diff.c:838-871)
      const size_t ij = g / (size_t) nz, k = g - ij * (size_t) nz;
      const long j = (long) (ij % (size_t) ny), i = (long) (ij / (size_t) ny);
      const double lx = 2.0 * M_PI / (step * (double) nx), ly = 2.0 * M_PI / (step * (double) ny),
                   lz = 2.0 * M_PI / (step * (double) nz);
      const double kx = (i <= nx / 2 ? (double) i : (double) (i - nx)) * lx;
      const double ky = (j <= ny / 2 ? (double) j : (double) (j - ny)) * ly;
      const double kz = ((long) k <= nz / 2 ? (double) k : (double) ((long) k - nz)) * lz;
      const C2<TA> a = ((const C2<TA> *) av)[g];
      return double2{(kx * kx + ky * ky + kz * kz) * ((double) a.x * (double) a.x + (double) a.y * (double) a.y), 0.0};
    }
  }
};

// Grid-stride sum with four independent terms per iteration (four loads in
// flight per thread); the block count, each thread's order of terms and the
// combination order are fixed, so the result is the same on every run.
template <typename TA, typename TB, int OP>
__global__ void __launch_bounds__(kThreads) k_reduce(const void *av, const void *bv, long nxy, long nz, long arow,
                                                   long brow, double2 *partial, long nx, long ny, double step) {
  __shared__ double sb[2 * kThreads / 32];
  using R = RedTerm<OP, TA, TB>;
  const size_t n = (size_t) nxy * nz;
  const size_t stride = (size_t) gridDim.x * blockDim.x;
  size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x;
  double sx[4] = {0.0, 0.0, 0.0, 0.0}, sy[4] = {0.0, 0.0, 0.0, 0.0};
  for (; g + 3 * stride < n; g += 4 * stride) {
    double2 e[4];
#pragma unroll
    for (int u = 0; u < 4; u++) e[u] = R::at(g + u * stride, av, bv, nz, arow, brow, nx, ny, step);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      sx[u] += e[u].x;
      sy[u] += e[u].y;
    }
  }
  for (; g < n; g += stride) {
    const double2 e = R::at(g, av, bv, nz, arow, brow, nx, ny, step);
    sx[0] += e.x;
    sy[0] += e.y;
  }
  double tx = (sx[0] + sx[1]) + (sx[2] + sx[3]);
  double ty = (sy[0] + sy[1]) + (sy[2] + sy[3]);
  block_sum2<kThreads>(tx, ty, sb);
  if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(tx, ty);
}

template <typename TA, typename TB>
static void launch_reduce(int op, int nb, cudaStream_t st, const void *a, const void *b, long nxy, long nz, long arow,
                          long brow, double2 *partial, long nx, long ny, double step) {
#define GB_RED_CASE(OPV)                                                                                       \
  case OPV:                                                                                                    \
    k_reduce<TA, TB, OPV><<<nb, kThreads, 0, st>>>(a, b, nxy, nz, arow, brow, partial, nx, ny, step); \
    break;
  switch (op) {
    GB_RED_CASE(GB_RED_SUM)
    GB_RED_CASE(GB_RED_NORM2)
    GB_RED_CASE(GB_RED_CONJ_PRODUCT)
    GB_RED_CASE(GB_RED_EXPECT_COMPLEX)
    GB_RED_CASE(GB_RED_EXPECT_REAL)
    GB_RED_CASE(GB_RED_REAL_SUM)
    GB_RED_CASE(GB_RED_KSQ_NORM2)
  }
#undef GB_RED_CASE
}

__global__ void k_finish2(const double2 *__restrict__ p, int n, double2 *out) {
  __shared__ double sb[2 * 1024 / 32];
  double sx = 0.0, sy = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    sx += p[i].x;
    sy += p[i].y;
  }
  block_sum2<1024>(sx, sy, sb);
  if (threadIdx.x == 0) *out = make_double2(sx, sy);
}

}  // namespace

extern "C" int gb_complex_op(int op, void *c, const void *a, const void *b, size_t n, double d_re, double d_im, int prec) {
  if (prec == GB_FP32)
    k_complex_op<float><<<blocks_for(n), kThreads, 0, gb__stream()>>>(op, (float2 *) c, (const float2 *) a,
                                                                       (const float2 *) b, n, d_re, d_im);
  else
    k_complex_op<double><<<blocks_for(n), kThreads, 0, gb__stream()>>>(op, (double2 *) c, (const double2 *) a,
                                                                        (const double2 *) b, n, d_re, d_im);
  GB_CHECK_LAUNCH("complex op");
  return 0;
}

extern "C" int gb_real_op(int op, void *c, const void *a, const void *b, size_t n, double d, int prec) {
  if (prec == GB_FP32)
    k_real_op<float><<<blocks_for(n), kThreads, 0, gb__stream()>>>(op, (float *) c, (const float *) a, (const float *) b, n, d);
  else
    k_real_op<double><<<blocks_for(n), kThreads, 0, gb__stream()>>>(op, (double *) c, (const double *) a, (const double *) b,
                                                                    n, d);
  GB_CHECK_LAUNCH("real op");
  return 0;
}

extern "C" int gb_mixed_op(int op, void *c, void *r, const void *r1, const gb_geom *g, long rrow, int cprec, int rprec) {
  const long nxy = g->nx * g->ny;
  const size_t n = (size_t) nxy * g->nz;
  if (cprec == GB_FP32 && rprec == GB_FP32)
    k_mixed<float, float><<<blocks_for(n), kThreads, 0, gb__stream()>>>(op, (float2 *) c, (float *) r, (const float *) r1,
                                                                         nxy, g->nz, rrow);
  else if (cprec == GB_FP32)
    k_mixed<float, double><<<blocks_for(n), kThreads, 0, gb__stream()>>>(op, (float2 *) c, (double *) r,
                                                                          (const double *) r1, nxy, g->nz, rrow);
  else if (rprec == GB_FP32)
    k_mixed<double, float><<<blocks_for(n), kThreads, 0, gb__stream()>>>(op, (double2 *) c, (float *) r,
                                                                          (const float *) r1, nxy, g->nz, rrow);
  else
    k_mixed<double, double><<<blocks_for(n), kThreads, 0, gb__stream()>>>(op, (double2 *) c, (double *) r,
                                                                           (const double *) r1, nxy, g->nz, rrow);
  GB_CHECK_LAUNCH("mixed op");
  return 0;
}

extern "C" int gb_wf_merge(void *dst, const void *wr, const void *wi, const gb_geom *g, long lx, long hx, long ly, long hy,
                           long lz, long hz) {
  const size_t n = (size_t) g->nx * g->ny * g->nz;
  if (g->prec == GB_FP32)
    k_merge<float><<<blocks_for(n), kThreads, 0, gb__stream()>>>((float2 *) dst, (const float2 *) wr, (const float2 *) wi,
                                                                  g->nx, g->ny, g->nz, lx, hx, ly, hy, lz, hz);
  else
    k_merge<double><<<blocks_for(n), kThreads, 0, gb__stream()>>>((double2 *) dst, (const double2 *) wr,
                                                                   (const double2 *) wi, g->nx, g->ny, g->nz, lx, hx, ly,
                                                                   hy, lz, hz);
  GB_CHECK_LAUNCH("merge");
  return 0;
}

extern "C" int gb_fft_convolute(void *c, const void *a, const void *b, long nx, long ny, long nzc, int prec) {
  const size_t n = (size_t) nx * ny * nzc;
  if (n == 0) return 0;
  if (prec == GB_FP32)
    k_fft_convolute<float><<<blocks_for(n), kThreads, 0, gb__stream()>>>((float2 *) c, (const float2 *) a,
                                                                          (const float2 *) b, ny, nzc, n);
  else
    k_fft_convolute<double><<<blocks_for(n), kThreads, 0, gb__stream()>>>((double2 *) c, (const double2 *) a,
                                                                           (const double2 *) b, ny, nzc, n);
  GB_CHECK_LAUNCH("fft convolute");
  return 0;
}

extern "C" int gb_interpolate(void *dst, const gb_grid_frame *d, const void *src, const gb_grid_frame *s, int bc,
                              double out_re, double out_im, int is_real) {
  InterpArgs a;
  a.dnx = d->nx;
  a.dny = d->ny;
  a.dnz = d->nz;
  a.drow = d->row;
  a.dstep = d->step;
  a.dx0 = d->x0;
  a.dy0 = d->y0;
  a.dz0 = d->z0;
  a.snx = s->nx;
  a.sny = s->ny;
  a.snz = s->nz;
  a.srow = s->row;
  a.sstep = s->step;
  a.sx0 = s->x0;
  a.sy0 = s->y0;
  a.sz0 = s->z0;
  a.bc = bc;
  a.out_re = out_re;
  a.out_im = out_im;
  const size_t n = (size_t) a.dnx * a.dny * a.dnz;
  if (n == 0) return 0;
  if (is_real) k_interp<true><<<blocks_for(n), kThreads, 0, gb__stream()>>>(dst, src, a);
  else k_interp<false><<<blocks_for(n), kThreads, 0, gb__stream()>>>(dst, src, a);
  GB_CHECK_LAUNCH("interpolate");
  return 0;
}

extern "C" int gb_r2c_pack(void *r, const void *c, const gb_geom *g) {
  const size_t n = (size_t) g->nx * g->ny * (g->nz / 2 + 1);
  k_r2c_pack<<<blocks_for(n), kThreads, 0, gb__stream()>>>((double2 *) r, (const double2 *) c, g->nx, g->ny, g->nz);
  GB_CHECK_LAUNCH("r2c pack");
  return 0;
}

extern "C" int gb_c2r_unpack(void *c, const void *r, const gb_geom *g) {
  const size_t n = (size_t) g->nx * g->ny * g->nz;
  k_c2r_unpack<<<blocks_for(n), kThreads, 0, gb__stream()>>>((double2 *) c, (const double2 *) r, g->nx, g->ny, g->nz);
  GB_CHECK_LAUNCH("c2r unpack");
  return 0;
}

extern "C" int gb_complex_real_part(void *r, const void *c, const gb_geom *g, long rrow) {
  const size_t n = (size_t) g->nx * g->ny * g->nz;
  k_real_part<<<blocks_for(n), kThreads, 0, gb__stream()>>>((double *) r, (const double2 *) c, g->nx * g->ny, g->nz, rrow);
  GB_CHECK_LAUNCH("real part");
  return 0;
}

// Fixed reduction geometry: the block count depends only on the grid size.
static int reduce_blocks(size_t n) {
  size_t b = (n + kThreads * 8 - 1) / (kThreads * 8);
  if (b > 148 * 8) b = 148 * 8;
  if (b < 1) b = 1;
  return (int) b;
}

static bool reduce_op_ok(int op) { return op >= GB_RED_SUM && op <= GB_RED_KSQ_NORM2; }

extern "C" int gb_reduce(int op, const void *a, const void *b, const gb_geom *g, long arow, long brow, int bprec, double *out) {
  if (!reduce_op_ok(op)) return gb__set_error(1023, "gb_reduce: unknown reduction op");
  const long nxy = g->nx * g->ny;
  const size_t n = (size_t) nxy * g->nz;
  const int nb = reduce_blocks(n);
  double2 *partial = (double2 *) gb__scratch(GB_SCR_PARTIAL, sizeof(double2) * (size_t) (nb + 1));
  double2 *res = (double2 *) gb__result_slot();
  if (!partial || !res) return gb_last_error();
  cudaStream_t st = gb__stream();
  const bool af = (g->prec == GB_FP32);
  const bool bf = (bprec == GB_FP32);
  if (af && bf) launch_reduce<float, float>(op, nb, st, a, b, nxy, g->nz, arow, brow, partial, g->nx, g->ny, g->step);
  else if (af) launch_reduce<float, double>(op, nb, st, a, b, nxy, g->nz, arow, brow, partial, g->nx, g->ny, g->step);
  else if (bf) launch_reduce<double, float>(op, nb, st, a, b, nxy, g->nz, arow, brow, partial, g->nx, g->ny, g->step);
  else launch_reduce<double, double>(op, nb, st, a, b, nxy, g->nz, arow, brow, partial, g->nx, g->ny, g->step);
  GB_CHECK_LAUNCH("reduce");
  k_finish2<<<1, 1024, 0, st>>>(partial, nb, res);
  GB_CHECK_LAUNCH("reduce finish");
  double2 h;
  int rc = gb__read_result(&h, sizeof(double2));
  out[0] = h.x;
  out[1] = h.y;
  return rc;
}

// ---------------------------------------------------------------------------
// Normalisation without a host round trip: the norm is reduced into a device
// scalar (fixed order, as gb_reduce) and the scale kernel reads it, so a loop
// of propagation steps and renormalisations never waits for the host.

template <typename T>
__global__ void k_scale_to_norm(C2<T> *__restrict__ psi, size_t n, const double2 *__restrict__ sum, double target,
                                double step_factor) {
  const double nrm = sum->x * step_factor;
  const T s = (T) (nrm > 0.0 ? sqrt(target / nrm) : 1.0);
  for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    psi[i] = cscale(psi[i], s);
}

extern "C" int gb_normalize_device(void *psi, const gb_geom *g, double target, double step_factor) {
  const long nxy = g->nx * g->ny;
  const size_t n = (size_t) nxy * g->nz;
  const int nb = reduce_blocks(n);
  double2 *partial = (double2 *) gb__scratch(GB_SCR_PARTIAL, sizeof(double2) * (size_t) (nb + 1));
  double2 *res = (double2 *) gb__scratch(GB_SCR_RESULT, 64);
  if (!partial || !res) return gb_last_error();
  cudaStream_t st = gb__stream();
  if (g->prec == GB_FP32) {
    launch_reduce<float, float>(GB_RED_NORM2, nb, st, psi, nullptr, nxy, g->nz, g->nz, 0, partial, g->nx, g->ny, g->step);
    GB_CHECK_LAUNCH("normalize: reduce");
    k_finish2<<<1, 1024, 0, st>>>(partial, nb, res);
    GB_CHECK_LAUNCH("normalize: finish");
    k_scale_to_norm<float><<<blocks_for(n), kThreads, 0, st>>>((float2 *) psi, n, res, target, step_factor);
  } else {
    launch_reduce<double, double>(GB_RED_NORM2, nb, st, psi, nullptr, nxy, g->nz, g->nz, 0, partial, g->nx, g->ny,
                                  g->step);
    GB_CHECK_LAUNCH("normalize: reduce");
    k_finish2<<<1, 1024, 0, st>>>(partial, nb, res);
    GB_CHECK_LAUNCH("normalize: finish");
    k_scale_to_norm<double><<<blocks_for(n), kThreads, 0, st>>>((double2 *) psi, n, res, target, step_factor);
  }
  GB_CHECK_LAUNCH("normalize: scale");
  return 0;
}

// ---------------------------------------------------------------------------
// Thomas-Fermi statistics of a padded real potential for a trial chemical
// potential mu: sum max(0, mu - V), the number of points with V < mu, and
// min V (the caller's Newton iteration on the piecewise-linear norm).

__global__ void __launch_bounds__(kThreads) k_tf_stats(const double *__restrict__ v, long nxy, long nz, long vrow,
                                                       double mu, double *__restrict__ part) {
  __shared__ double sb[2 * kThreads / 32];
  __shared__ double sm[kThreads / 32];
  const size_t n = (size_t) nxy * nz;
  double s = 0.0, c = 0.0, vmin = 1e300, vs = 0.0;
  for (size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x; g < n; g += (size_t) gridDim.x * blockDim.x) {
    const size_t ij = g / nz, k = g - ij * nz;
    const double x = v[ij * vrow + k];
    if (x < mu) {
      s += mu - x;
      c += 1.0;
    }
    vmin = fmin(vmin, x);
    vs += x;
  }
  block_sum2<kThreads>(s, c, sb);
  __syncthreads();
  double zero = 0.0;
  block_sum2<kThreads>(vs, zero, sb);
  for (int o = 16; o > 0; o >>= 1) vmin = fmin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = vmin;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / 32; w++) vmin = fmin(vmin, sm[w]);
    part[4 * blockIdx.x] = s;
    part[4 * blockIdx.x + 1] = c;
    part[4 * blockIdx.x + 2] = vmin;
    part[4 * blockIdx.x + 3] = vs;
  }
}

__global__ void k_tf_finish(const double *__restrict__ part, int nb, double *out) {
  if (threadIdx.x != 0) return;
  double s = 0.0, c = 0.0, vmin = 1e300, vs = 0.0;
  for (int b = 0; b < nb; b++) {
    s += part[4 * b];
    c += part[4 * b + 1];
    vmin = fmin(vmin, part[4 * b + 2]);
    vs += part[4 * b + 3];
  }
  out[0] = s;
  out[1] = c;
  out[2] = vmin;
  out[3] = vs;
}

extern "C" int gb_tf_stats(const void *v, const gb_geom *g, long vrow, double mu, double *out4) {
  const long nxy = g->nx * g->ny;
  const size_t n = (size_t) nxy * g->nz;
  const int nb = reduce_blocks(n);
  double *part = (double *) gb__scratch(GB_SCR_PARTIAL, sizeof(double) * 4 * (size_t) nb);
  double *res = (double *) gb__result_slot();
  if (!part || !res) return gb_last_error();
  cudaStream_t st = gb__stream();
  k_tf_stats<<<nb, kThreads, 0, st>>>((const double *) v, nxy, g->nz, vrow, mu, part);
  GB_CHECK_LAUNCH("tf stats");
  k_tf_finish<<<1, 32, 0, st>>>(part, nb, res);
  GB_CHECK_LAUNCH("tf stats finish");
  return gb__read_result(out4, 4 * sizeof(double));
}

// ---------------------------------------------------------------------------
// Allocation-free reduction (gb_reduce_noalloc).
//
// Some callers cannot let a library allocate device memory on their behalf:
// applications that hand out all device memory from their own pool or under
// a fixed budget, and latency-critical loops in which a cudaMalloc, or the
// device-wide synchronisation of cudaFree, is not acceptable.  For them this
// variant of gb_reduce keeps its block partial sums and its result in a
// file-scope __device__ array of fixed size instead of library scratch, so
// no call allocates anything.
//
// Limits and sharing:
//  * One block per 2048 grid points and at most 8192 blocks: grids of up to
//    16,777,216 points (256^3).  Larger grids are rejected with an error
//    before any work is launched.
//  * The array (8193 x 16 bytes) lives in every GPU that loads the library
//    until the process exits.  Every call uses the same array and leaves its
//    last contents behind; each call writes every slot it reads, so nothing
//    needs clearing, but two calls that overlap on the GPU (e.g. from
//    different streams or processes sharing the context) race on it.
//  * The host code needs the array's device address, which the first call on
//    a device obtains with cudaGetSymbolAddress while that device is current.
//    Make that first call before any stream capture.
//  * The library stream must exist (gb_init / cuda_enable called first).
namespace {

constexpr int kNoallocThreads = 256;
constexpr int kNoallocPerThread = 8;
constexpr long kNoallocBlockElems = (long) kNoallocThreads * kNoallocPerThread;
constexpr long kNoallocMaxBlocks = 8192;

__device__ __align__(256) double2 g_noalloc_scratch[kNoallocMaxBlocks + 1];

double2 *g_noalloc_dev_ptr = nullptr;
int g_noalloc_device = -1;

// One element's contribution to the reductions of gb_reduce.
template <typename TA, typename TB>
__device__ __forceinline__ void noalloc_term(int op, const void *av, const void *bv, size_t g, size_t ij, size_t k,
                                             long arow, long brow, long nx, long ny, long nz, double step, double &sx,
                                             double &sy) {
  switch (op) {
    case GB_RED_SUM: {
      const C2<TA> a = ((const C2<TA> *) av)[g];
      sx += (double) a.x;
      sy += (double) a.y;
    } break;
    case GB_RED_NORM2: {
      const C2<TA> a = ((const C2<TA> *) av)[g];
      sx += (double) a.x * (double) a.x + (double) a.y * (double) a.y;
    } break;
    case GB_RED_CONJ_PRODUCT: {
      const C2<TA> a = ((const C2<TA> *) av)[g];
      const C2<TB> b = ((const C2<TB> *) bv)[g];
      const double ar = a.x, ai = a.y, br = b.x, bi = b.y;
      sx += ar * br + ai * bi;
      sy += ar * bi - ai * br;
    } break;
    case GB_RED_EXPECT_COMPLEX: {
      const C2<TA> a = ((const C2<TA> *) av)[g];
      const C2<TB> b = ((const C2<TB> *) bv)[g];
      const double w = (double) a.x * (double) a.x + (double) a.y * (double) a.y;
      sx += w * (double) b.x;
      sy += w * (double) b.y;
    } break;
    case GB_RED_EXPECT_REAL: {
      const C2<TA> a = ((const C2<TA> *) av)[g];
      const double w = (double) a.x * (double) a.x + (double) a.y * (double) a.y;
      sx += w * (double) ((const TB *) bv)[ij * brow + k];
    } break;
    case GB_RED_REAL_SUM: sx += (double) ((const TA *) av)[ij * arow + k]; break;
    case GB_RED_KSQ_NORM2: {
      const long j = (long) (ij % ny), i = (long) (ij / ny);
      const double lx = 2.0 * M_PI / (step * (double) nx), ly = 2.0 * M_PI / (step * (double) ny),
                   lz = 2.0 * M_PI / (step * (double) nz);
      const double kx = (i <= nx / 2 ? (double) i : (double) (i - nx)) * lx;
      const double ky = (j <= ny / 2 ? (double) j : (double) (j - ny)) * ly;
      const double kz = ((long) k <= nz / 2 ? (double) k : (double) ((long) k - nz)) * lz;
      const C2<TA> a = ((const C2<TA> *) av)[g];
      sx += (kx * kx + ky * ky + kz * kz) * ((double) a.x * (double) a.x + (double) a.y * (double) a.y);
    } break;
  }
}

// Block b sums grid points [2048 b, 2048 (b + 1)) in a fixed order and
// writes one partial into scratch[b].
template <typename TA, typename TB>
__global__ void __launch_bounds__(kNoallocThreads)
    k_reduce_noalloc(int op, const void *av, const void *bv, long nxy, long nz, long arow, long brow, double2 *scratch,
                     long nx, long ny, double step) {
  __shared__ double sb[2 * kNoallocThreads / 32];
  const size_t n = (size_t) nxy * nz;
  const size_t base = (size_t) blockIdx.x * kNoallocBlockElems;
  double sx = 0.0, sy = 0.0;
#pragma unroll
  for (int r = 0; r < kNoallocPerThread; r++) {
    const size_t g = base + (size_t) r * kNoallocThreads + threadIdx.x;
    if (g < n) {
      const size_t ij = g / nz, k = g - ij * nz;
      noalloc_term<TA, TB>(op, av, bv, g, ij, k, arow, brow, nx, ny, nz, step, sx, sy);
    }
  }
  block_sum2<kNoallocThreads>(sx, sy, sb);
  if (threadIdx.x == 0) scratch[blockIdx.x] = make_double2(sx, sy);
}

// Fixed-order sum of the nb partials into scratch[kNoallocMaxBlocks].
__global__ void k_finish_noalloc(double2 *scratch, int nb) {
  __shared__ double sb[2 * 1024 / 32];
  double sx = 0.0, sy = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    sx += scratch[i].x;
    sy += scratch[i].y;
  }
  block_sum2<1024>(sx, sy, sb);
  if (threadIdx.x == 0) scratch[kNoallocMaxBlocks] = make_double2(sx, sy);
}

}  // namespace

extern "C" int gb_reduce_noalloc(int op, const void *a, const void *b, const gb_geom *g, long arow, long brow, int bprec,
                                 double *out) {
  if (!reduce_op_ok(op)) return gb__set_error(1023, "gb_reduce_noalloc: unknown reduction op");
  const long nxy = g->nx * g->ny;
  const double npts = (double) nxy * (double) g->nz;
  if (npts > (double) (kNoallocMaxBlocks * kNoallocBlockElems)) {
    char msg[160];
    snprintf(msg, sizeof(msg), "gb_reduce_noalloc: %.0f grid points exceed the %ld-point limit of its static scratch", npts,
             kNoallocMaxBlocks * kNoallocBlockElems);
    return gb__set_error(1020, msg);
  }
  cudaStream_t st = gb__stream();
  if (!st) return gb__set_error(1021, "gb_reduce_noalloc: library not initialised (call gb_init or cuda_enable first)");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return gb__set_error(1022, "gb_reduce_noalloc: cudaGetDevice failed");
  if (!g_noalloc_dev_ptr || dev != g_noalloc_device) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return gb__set_error((int) e, "gb_reduce_noalloc: cudaGetSymbolAddress failed");
    g_noalloc_dev_ptr = (double2 *) p;
    g_noalloc_device = dev;
  }
  const int nb = (int) ((nxy * g->nz + kNoallocBlockElems - 1) / kNoallocBlockElems);
  if (nb < 1) {
    out[0] = out[1] = 0.0;
    return 0;
  }
  const bool af = (g->prec == GB_FP32);
  const bool bf = (bprec == GB_FP32);
  double2 *sp = g_noalloc_dev_ptr;
  if (af && bf) k_reduce_noalloc<float, float><<<nb, kNoallocThreads, 0, st>>>(op, a, b, nxy, g->nz, arow, brow, sp, g->nx, g->ny, g->step);
  else if (af) k_reduce_noalloc<float, double><<<nb, kNoallocThreads, 0, st>>>(op, a, b, nxy, g->nz, arow, brow, sp, g->nx, g->ny, g->step);
  else if (bf) k_reduce_noalloc<double, float><<<nb, kNoallocThreads, 0, st>>>(op, a, b, nxy, g->nz, arow, brow, sp, g->nx, g->ny, g->step);
  else k_reduce_noalloc<double, double><<<nb, kNoallocThreads, 0, st>>>(op, a, b, nxy, g->nz, arow, brow, sp, g->nx, g->ny, g->step);
  GB_CHECK_LAUNCH("reduce noalloc");
  k_finish_noalloc<<<1, 1024, 0, st>>>(sp, nb);
  GB_CHECK_LAUNCH("reduce noalloc finish");
  double2 h;
  const cudaError_t e = cudaMemcpyAsync(&h, sp + kNoallocMaxBlocks, sizeof(double2), cudaMemcpyDeviceToHost, st);
  const cudaError_t s = (e == cudaSuccess) ? cudaStreamSynchronize(st) : e;
  if (s != cudaSuccess) return gb__set_error((int) s, "gb_reduce_noalloc: result copy");
  out[0] = h.x;
  out[1] = h.y;
  return 0;
}
