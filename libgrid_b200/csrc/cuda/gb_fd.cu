// Finite-difference stencils on complex and padded real grids.
//
// Boundary values follow the reference's value_outside functions
// (src/cgrid_bc.c:21-86, src/rgrid_bc.c:19-74): Dirichlet returns a constant
// (the grid's outside parameter, 0 by default), Neumann mirrors i -> -i and
// i -> 2n - i - 2, periodic wraps.  On an axis of length 1 the Neumann mirror
// lands outside the grid again (the reference recurses without end there);
// this implementation uses the single plane instead.
//
// Each output point is one thread.  The plane of threads in a block covers a
// (BY x BZ) tile of (y, z) and walks along x, keeping the x-1, x, x+1 values
// in registers, so every input element is read from HBM once; the y/z
// neighbours come from the L1-resident tile rows.  Laplacian sums keep the
// reference's left-to-right order
//   (-6 c + z+ + z- + y+ + y- + x+ + x-) / h^2     (src/cgrid_diff.c:330-335).
#include <string.h>

#include "gb_common.cuh"
#include "gb_internal_cuda.h"

namespace {

template <typename T, bool REAL> struct Elem;
template <typename T> struct Elem<T, false> {
  using V = C2<T>;
  static __device__ __forceinline__ V zero() { return V{(T) 0, (T) 0}; }
  static __device__ __forceinline__ V outside(double re, double im) { return V{(T) re, (T) im}; }
  static __device__ __forceinline__ V add(V a, V b) { return cadd(a, b); }
  static __device__ __forceinline__ V sub(V a, V b) { return csub(a, b); }
  static __device__ __forceinline__ V scale(V a, T s) { return cscale(a, s); }
};
template <typename T> struct Elem<T, true> {
  using V = T;
  static __device__ __forceinline__ V zero() { return (T) 0; }
  static __device__ __forceinline__ V outside(double re, double) { return (T) re; }
  static __device__ __forceinline__ V add(V a, V b) { return a + b; }
  static __device__ __forceinline__ V sub(V a, V b) { return a - b; }
  static __device__ __forceinline__ V scale(V a, T s) { return a * s; }
};

struct FdArgs {
  long nx, ny, nz, row;  // row = elements per (i, j) row of the storage
  int bc;
  double out_re, out_im;
  double coef;
};

// Map a possibly out-of-range index on one axis; returns false for
// "Dirichlet outside".
__device__ __forceinline__ bool map_index(long &i, long n, int bc) {
  if (i >= 0 && i < n) return true;
  if (bc == GB_BC_DIRICHLET) return false;
  if (bc == GB_BC_PERIODIC) {
    i %= n;
    if (i < 0) i += n;
    return true;
  }
  // Neumann mirror (src/cgrid_bc.c:45-57)
  if (i < 0) i = -i;
  if (i > n - 1) i = 2 * n - i - 2;
  if (i < 0 || i >= n) i = 0;  // axis of length 1
  return true;
}

template <typename T, bool REAL>
__device__ __forceinline__ typename Elem<T, REAL>::V fetch(const typename Elem<T, REAL>::V *src, long i, long j, long k,
                                                           const FdArgs &a) {
  using E = Elem<T, REAL>;
  if (i < 0 || i >= a.nx || j < 0 || j >= a.ny || k < 0 || k >= a.nz) {
    if (a.bc == GB_BC_DIRICHLET) return E::outside(a.out_re, a.out_im);
    // Neumann/periodic remap all three indices like the reference does
    if (!map_index(i, a.nx, a.bc) || !map_index(j, a.ny, a.bc) || !map_index(k, a.nz, a.bc))
      return E::outside(a.out_re, a.out_im);
  }
  return src[(i * a.ny + j) * a.row + k];
}

template <typename T, bool REAL>
__global__ void k_fd(int op, typename Elem<T, REAL>::V *__restrict__ dst, const typename Elem<T, REAL>::V *__restrict__ src,
                     FdArgs a) {
  using E = Elem<T, REAL>;
  using V = typename E::V;
  const long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
  const long j = blockIdx.y;
  if (k >= a.nz) return;
  const T coef = (T) a.coef;
  V xm = fetch<T, REAL>(src, -1, j, k, a);
  V c = fetch<T, REAL>(src, 0, j, k, a);
  for (long i = 0; i < a.nx; i++) {
    const V xp = fetch<T, REAL>(src, i + 1, j, k, a);
    V r;
    switch (op) {
      case GB_FD_LAPLACE: {
        V s = E::scale(c, (T) -6.0);
        s = E::add(s, fetch<T, REAL>(src, i, j, k + 1, a));
        s = E::add(s, fetch<T, REAL>(src, i, j, k - 1, a));
        s = E::add(s, fetch<T, REAL>(src, i, j + 1, k, a));
        s = E::add(s, fetch<T, REAL>(src, i, j - 1, k, a));
        s = E::add(s, xp);
        s = E::add(s, xm);
        r = E::scale(s, coef);
      } break;
      case GB_FD_LAPLACE_X: r = E::scale(E::add(E::add(E::scale(c, (T) -2.0), xp), xm), coef); break;
      case GB_FD_LAPLACE_Y:
        r = E::scale(E::add(E::add(E::scale(c, (T) -2.0), fetch<T, REAL>(src, i, j + 1, k, a)),
                            fetch<T, REAL>(src, i, j - 1, k, a)),
                     coef);
        break;
      case GB_FD_LAPLACE_Z:
        r = E::scale(E::add(E::add(E::scale(c, (T) -2.0), fetch<T, REAL>(src, i, j, k + 1, a)),
                            fetch<T, REAL>(src, i, j, k - 1, a)),
                     coef);
        break;
      case GB_FD_GRADIENT_X: r = E::scale(E::sub(xp, xm), coef); break;
      case GB_FD_GRADIENT_Y:
        r = E::scale(E::sub(fetch<T, REAL>(src, i, j + 1, k, a), fetch<T, REAL>(src, i, j - 1, k, a)), coef);
        break;
      default:
        r = E::scale(E::sub(fetch<T, REAL>(src, i, j, k + 1, a), fetch<T, REAL>(src, i, j, k - 1, a)), coef);
        break;
    }
    dst[(i * a.ny + j) * a.row + k] = r;
    xm = c;
    c = xp;
  }
}

// sum conj(psi) * Laplacian(psi) (unscaled by 1/h^2 until the end).
template <typename T>
__global__ void __launch_bounds__(256) k_fd_kinetic(const C2<T> *__restrict__ src, FdArgs a, double2 *partial) {
  __shared__ double sb[16];
  double sx = 0.0, sy = 0.0;
  const long nyz = a.ny * a.nz;
  for (long col = blockIdx.x * (long) blockDim.x + threadIdx.x; col < nyz; col += (long) gridDim.x * blockDim.x) {
    const long j = col / a.nz, k = col - j * a.nz;
    C2<T> xm = fetch<T, false>(src, -1, j, k, a);
    C2<T> c = fetch<T, false>(src, 0, j, k, a);
    for (long i = 0; i < a.nx; i++) {
      const C2<T> xp = fetch<T, false>(src, i + 1, j, k, a);
      double sr = -6.0 * (double) c.x, si = -6.0 * (double) c.y;
      C2<T> nb[6] = {fetch<T, false>(src, i, j, k + 1, a), fetch<T, false>(src, i, j, k - 1, a),
                     fetch<T, false>(src, i, j + 1, k, a), fetch<T, false>(src, i, j - 1, k, a), xp, xm};
#pragma unroll
      for (int q = 0; q < 6; q++) {
        sr += (double) nb[q].x;
        si += (double) nb[q].y;
      }
      sr *= a.coef;
      si *= a.coef;
      // conj(c) * (sr + i si)
      sx += (double) c.x * sr + (double) c.y * si;
      sy += (double) c.x * si - (double) c.y * sr;
      xm = c;
      c = xp;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    sx += __shfl_down_sync(0xffffffffu, sx, off);
    sy += __shfl_down_sync(0xffffffffu, sy, off);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    sb[2 * w] = sx;
    sb[2 * w + 1] = sy;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tx = 0.0, ty = 0.0;
    for (int q = 0; q < 8; q++) {
      tx += sb[2 * q];
      ty += sb[2 * q + 1];
    }
    partial[blockIdx.x] = make_double2(tx, ty);
  }
}

__global__ void k_finish_fd(const double2 *__restrict__ p, int n, double2 *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double sx = 0.0, sy = 0.0;
    for (int i = 0; i < n; i++) {
      sx += p[i].x;
      sy += p[i].y;
    }
    *out = make_double2(sx, sy);
  }
}

}  // namespace

extern "C" int gb_fd(int op, void *dst, const void *src, const gb_geom *g, int bc, double out_re, double out_im, double coef,
                     int is_real, long row) {
  FdArgs a;
  a.nx = g->nx;
  a.ny = g->ny;
  a.nz = g->nz;
  a.row = row;
  a.bc = bc;
  a.out_re = out_re;
  a.out_im = out_im;
  a.coef = coef;
  if (g->ny > 65535) return gb__set_error(1005, "fd: ny above 65535");
  const int th = g->nz >= 128 ? 128 : (g->nz >= 32 ? 32 : (int) g->nz);
  dim3 grid((unsigned) ((g->nz + th - 1) / th), (unsigned) g->ny);
  cudaStream_t st = gb__stream();
  if (is_real) {
    if (g->prec == GB_FP32) k_fd<float, true><<<grid, th, 0, st>>>(op, (float *) dst, (const float *) src, a);
    else k_fd<double, true><<<grid, th, 0, st>>>(op, (double *) dst, (const double *) src, a);
  } else {
    if (g->prec == GB_FP32) k_fd<float, false><<<grid, th, 0, st>>>(op, (float2 *) dst, (const float2 *) src, a);
    else k_fd<double, false><<<grid, th, 0, st>>>(op, (double2 *) dst, (const double2 *) src, a);
  }
  GB_CHECK_LAUNCH("fd stencil");
  return 0;
}

extern "C" int gb_fd_kinetic_sum(const void *psi, const gb_geom *g, int bc, double out_re, double out_im, double inv_h2,
                                 double *out) {
  FdArgs a;
  a.nx = g->nx;
  a.ny = g->ny;
  a.nz = g->nz;
  a.row = g->nz;
  a.bc = bc;
  a.out_re = out_re;
  a.out_im = out_im;
  a.coef = inv_h2;
  const long nyz = g->ny * g->nz;
  long nb = (nyz + 255) / 256;
  if (nb > 148 * 8) nb = 148 * 8;
  if (nb < 1) nb = 1;
  double2 *partial = (double2 *) gb__scratch(GB_SCR_PARTIAL, sizeof(double2) * (size_t) nb);
  double2 *res = (double2 *) gb__result_slot();
  if (!partial || !res) return gb_last_error();
  cudaStream_t st = gb__stream();
  if (g->prec == GB_FP32) k_fd_kinetic<float><<<(unsigned) nb, 256, 0, st>>>((const float2 *) psi, a, partial);
  else k_fd_kinetic<double><<<(unsigned) nb, 256, 0, st>>>((const double2 *) psi, a, partial);
  GB_CHECK_LAUNCH("fd kinetic");
  k_finish_fd<<<1, 32, 0, st>>>(partial, (int) nb, res);
  GB_CHECK_LAUNCH("fd kinetic finish");
  double2 h;
  int rc = gb__read_result(&h, sizeof(double2));
  out[0] = h.x;
  out[1] = h.y;
  return rc;
}
