// Pointwise grid algebra and deterministic FP64 reductions.
//
// Replaces the reference's per-operation SIMT kernels (src/cgrid-cuda2.cu,
// src/rgrid-cuda2.cu, src/ngrid-cuda2.cu, src/grid_wf-cuda2.cu:111-176) and
// its reductions, which sum each 512-thread block serially in thread 0 and
// finish on the host (src/cgrid-cuda2.cu:975-996).  Here each reduction is a
// grid-stride pass with a fixed per-thread order, a fixed shuffle tree per
// block and a fixed-order finish over the block partials, so the result does
// not depend on scheduling.
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

template <typename TA, typename TB>
__global__ void __launch_bounds__(kThreads) k_reduce(int op, const void *av, const void *bv, long nxy, long nz, long arow,
                                                   long brow, double2 *partial, long nx, long ny, double step) {
  __shared__ double sb[2 * kThreads / 32];
  const size_t n = (size_t) nxy * nz;
  double sx = 0.0, sy = 0.0;
  for (size_t g = blockIdx.x * (size_t) blockDim.x + threadIdx.x; g < n; g += (size_t) gridDim.x * blockDim.x) {
    const size_t ij = g / nz, k = g - ij * nz;
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
        // src/cgrid_diff.c:838-871
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
  block_sum2<kThreads>(sx, sy, sb);
  if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(sx, sy);
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

extern "C" int gb_reduce(int op, const void *a, const void *b, const gb_geom *g, long arow, long brow, int bprec, double *out) {
  const long nxy = g->nx * g->ny;
  const size_t n = (size_t) nxy * g->nz;
  const int nb = reduce_blocks(n);
  double2 *partial = (double2 *) gb__scratch(GB_SCR_PARTIAL, sizeof(double2) * (size_t) (nb + 1));
  double2 *res = (double2 *) gb__scratch(GB_SCR_RESULT, 64);
  if (!partial || !res) return gb_last_error();
  cudaStream_t st = gb__stream();
  const bool af = (g->prec == GB_FP32);
  const bool bf = (bprec == GB_FP32);
  if (af && bf) k_reduce<float, float><<<nb, kThreads, 0, st>>>(op, a, b, nxy, g->nz, arow, brow, partial, g->nx, g->ny, g->step);
  else if (af) k_reduce<float, double><<<nb, kThreads, 0, st>>>(op, a, b, nxy, g->nz, arow, brow, partial, g->nx, g->ny, g->step);
  else if (bf) k_reduce<double, float><<<nb, kThreads, 0, st>>>(op, a, b, nxy, g->nz, arow, brow, partial, g->nx, g->ny, g->step);
  else k_reduce<double, double><<<nb, kThreads, 0, st>>>(op, a, b, nxy, g->nz, arow, brow, partial, g->nx, g->ny, g->step);
  GB_CHECK_LAUNCH("reduce");
  k_finish2<<<1, 1024, 0, st>>>(partial, nb, res);
  GB_CHECK_LAUNCH("reduce finish");
  double2 h;
  int rc = gb_d2h(&h, res, sizeof(double2));
  out[0] = h.x;
  out[1] = h.y;
  return rc;
}
