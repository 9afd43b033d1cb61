// Finite-difference stencils on complex and padded real grids.
//
// Boundary values follow the reference's value_outside functions
// (src/cgrid_bc.c:21-86, src/rgrid_bc.c:19-74): Dirichlet returns a constant
// (the grid's outside parameter, 0 by default), Neumann mirrors i -> -i and
// i -> 2n - i - 2, periodic wraps.  On an axis of length 1 the Neumann mirror
// lands outside the grid again (the reference recurses without end there);
// this implementation uses the single plane instead.
//
// Each output column (j, k) is one thread of a CTA whose 8 x 32 (y, z) tile
// marches along a chunk of x planes (k_fd below): x neighbours in registers,
// y/z neighbours from a shared-memory plane with a one-point halo, so every
// input element is read from HBM about once.  Laplacian sums keep the
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

// Tiles: a CTA of 256 threads owns a (kFdTY x kFdTZ) = (8 x 32) tile of
// (y, z) over kFdXC consecutive x planes and marches along x.  Each thread
// keeps its own column's x-1, x and x+1 values in registers and loads the
// x+2 plane two steps ahead; the current plane's tile and its one-point y/z
// halo sit in a double-buffered shared-memory plane, so the y/z neighbours
// come from shared memory and every element is read from HBM about once
// ((kFdXC + 2) / kFdXC planes per chunk, plus the halo rows from L2).  The
// halo points are loaded two steps ahead as well: warp 0 the row y-1,
// warp 1 the row y+8, warp 2 the columns z-1 (lanes 0-7) and z+32 (lanes
// 8-15).  Measured at 256^3: two planes ahead at four CTAs per SM beat four
// planes ahead at three.
constexpr int kFdTY = 8, kFdTZ = 32, kFdXC = 16, kFdThreads = kFdTY * kFdTZ;

template <typename T, bool REAL> struct FdTile {
  using E = Elem<T, REAL>;
  using V = typename E::V;
  V xm, c, xp, xq;  // this thread's column, planes i-1, i, i+1, i+2
  V h, hn;          // its halo point (if it owns one), planes i and i+1
  long hj, hk;      // halo point (y, z); may lie outside the grid
  int hy, hz;       // its place in the shared plane
  bool has_h;       // whether this thread owns a halo point

  __device__ void init(const V *src, const FdArgs &a, long i0, long j, long k, int ty, int tz) {
    const long j0 = j - ty, k0 = k - tz;
    hj = hk = 0;
    hy = hz = 0;
    has_h = ty < 2 || (ty == 2 && tz < 2 * kFdTY);
    if (ty == 0) {
      hj = j0 - 1, hk = k, hy = 0, hz = tz + 1;
    } else if (ty == 1) {
      hj = j0 + kFdTY, hk = k, hy = kFdTY + 1, hz = tz + 1;
    } else if (ty == 2 && tz < 2 * kFdTY) {
      const int r = tz & (kFdTY - 1);
      hj = j0 + r, hk = tz < kFdTY ? k0 - 1 : k0 + kFdTZ, hy = r + 1, hz = tz < kFdTY ? 0 : kFdTZ + 1;
    }
    // every thread of the tile loads its column, also past the far edge of
    // the grid (a partial tile): there fetch returns the boundary value the
    // last row/column needs as its neighbour
    xm = fetch<T, REAL>(src, i0 - 1, j, k, a);
    c = fetch<T, REAL>(src, i0, j, k, a);
    xp = fetch<T, REAL>(src, i0 + 1, j, k, a);
    xq = E::zero();
    h = has_h ? fetch<T, REAL>(src, i0, hj, hk, a) : E::zero();
    hn = has_h ? fetch<T, REAL>(src, i0 + 1, hj, hk, a) : E::zero();
  }

  // loads of plane i + 2 (column and halo), issued at the top of step i;
  // returns the halo value for the shift
  __device__ __forceinline__ V prefetch(const V *src, const FdArgs &a, long i, long i1, long j, long k) {
    if (i + 2 <= i1) xq = fetch<T, REAL>(src, i + 2, j, k, a);
    return (has_h && i + 2 < i1) ? fetch<T, REAL>(src, i + 2, hj, hk, a) : E::zero();
  }

  __device__ __forceinline__ void shift(V hq) {
    xm = c;
    c = xp;
    xp = xq;
    h = hn;
    hn = hq;
  }
};

template <typename T, bool REAL>
__global__ void __launch_bounds__(kFdThreads, 4) k_fd(int op, typename Elem<T, REAL>::V *__restrict__ dst,
                                                   const typename Elem<T, REAL>::V *__restrict__ src, FdArgs a) {
  using E = Elem<T, REAL>;
  using V = typename E::V;
  __shared__ V sm[2][kFdTY + 2][kFdTZ + 2];
  const int tz = threadIdx.x % kFdTZ, ty = threadIdx.x / kFdTZ;
  const long k = blockIdx.x * (long) kFdTZ + tz, j = blockIdx.y * (long) kFdTY + ty;
  const long i0 = blockIdx.z * (long) kFdXC;
  const long i1 = i0 + kFdXC < a.nx ? i0 + kFdXC : a.nx;
  const bool in = k < a.nz && j < a.ny;
  const T coef = (T) a.coef;
  FdTile<T, REAL> t;
  t.init(src, a, i0, j, k, ty, tz);
  V *out = dst + (i0 * a.ny + j) * a.row + k;
  const long pstride = a.ny * a.row;
  for (long i = i0; i < i1; i++) {
    const V hq = t.prefetch(src, a, i, i1, j, k);
    const int b = (int) ((i - i0) & 1);
    const V c = t.c, xm = t.xm, xp = t.xp;
    sm[b][ty + 1][tz + 1] = c;
    if (t.has_h) sm[b][t.hy][t.hz] = t.h;
    __syncthreads();
    const V zp = sm[b][ty + 1][tz + 2], zm = sm[b][ty + 1][tz];
    const V yp = sm[b][ty + 2][tz + 1], ym = sm[b][ty][tz + 1];
    V r;
    switch (op) {
      case GB_FD_LAPLACE: {
        V s = E::scale(c, (T) -6.0);
        s = E::add(s, zp);
        s = E::add(s, zm);
        s = E::add(s, yp);
        s = E::add(s, ym);
        s = E::add(s, xp);
        s = E::add(s, xm);
        r = E::scale(s, coef);
      } break;
      case GB_FD_LAPLACE_X: r = E::scale(E::add(E::add(E::scale(c, (T) -2.0), xp), xm), coef); break;
      case GB_FD_LAPLACE_Y: r = E::scale(E::add(E::add(E::scale(c, (T) -2.0), yp), ym), coef); break;
      case GB_FD_LAPLACE_Z: r = E::scale(E::add(E::add(E::scale(c, (T) -2.0), zp), zm), coef); break;
      case GB_FD_GRADIENT_X: r = E::scale(E::sub(xp, xm), coef); break;
      case GB_FD_GRADIENT_Y: r = E::scale(E::sub(yp, ym), coef); break;
      default: r = E::scale(E::sub(zp, zm), coef); break;
    }
    if (in) out[(i - i0) * pstride] = r;
    t.shift(hq);
  }
}

// sum conj(psi) * Laplacian(psi) over the grid, the Laplacian summed in the
// stencil kernel's order and scaled by 1/h^2 (a.coef) before the product.
// Same tiles and march as k_fd; each CTA writes one partial (x, y) sum,
// reduced in a fixed order, so the result is the same from run to run.
template <typename T>
__global__ void __launch_bounds__(kFdThreads) k_fd_kinetic(const C2<T> *__restrict__ src, FdArgs a,
                                                           double2 *__restrict__ partial) {
  using E = Elem<T, false>;
  using V = C2<T>;
  __shared__ V sm[2][kFdTY + 2][kFdTZ + 2];
  __shared__ double sb[2 * kFdThreads / 32];
  const int tz = threadIdx.x % kFdTZ, ty = threadIdx.x / kFdTZ;
  const long k = blockIdx.x * (long) kFdTZ + tz, j = blockIdx.y * (long) kFdTY + ty;
  const long i0 = blockIdx.z * (long) kFdXC;
  const long i1 = i0 + kFdXC < a.nx ? i0 + kFdXC : a.nx;
  const bool in = k < a.nz && j < a.ny;
  FdTile<T, false> t;
  t.init(src, a, i0, j, k, ty, tz);
  double sx = 0.0, sy = 0.0;
  for (long i = i0; i < i1; i++) {
    const V hq = t.prefetch(src, a, i, i1, j, k);
    const int b = (int) ((i - i0) & 1);
    const V c = t.c;
    sm[b][ty + 1][tz + 1] = c;
    if (t.has_h) sm[b][t.hy][t.hz] = t.h;
    __syncthreads();
    if (in) {
      const V nb[6] = {sm[b][ty + 1][tz + 2], sm[b][ty + 1][tz], sm[b][ty + 2][tz + 1], sm[b][ty][tz + 1], t.xp, t.xm};
      double sr = -6.0 * (double) c.x, si = -6.0 * (double) c.y;
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
    }
    t.shift(hq);
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
    double tx = 0.0, tyy = 0.0;
    for (int q = 0; q < kFdThreads / 32; q++) {
      tx += sb[2 * q];
      tyy += sb[2 * q + 1];
    }
    partial[((long) blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = make_double2(tx, tyy);
  }
}

// Sum of n partials by one CTA of 256 threads: strided per-thread sums,
// then a fixed shuffle tree (deterministic).
__global__ void __launch_bounds__(256) k_finish_fd(const double2 *__restrict__ p, long n, double2 *out) {
  __shared__ double sb[16];
  double sx = 0.0, sy = 0.0;
  for (long i = threadIdx.x; i < n; i += 256) {
    sx += p[i].x;
    sy += p[i].y;
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
    *out = make_double2(tx, ty);
  }
}

// Launch grid of the tiled stencils: (z tiles, y tiles, x chunks).
int fd_grid(const gb_geom *g, dim3 *grid) {
  const long gz = (g->nz + kFdTZ - 1) / kFdTZ, gy = (g->ny + kFdTY - 1) / kFdTY, gx = (g->nx + kFdXC - 1) / kFdXC;
  if (gy > 65535 || gx > 65535) return gb__set_error(1005, "fd: grid too large for the stencil tiling");
  *grid = dim3((unsigned) gz, (unsigned) gy, (unsigned) gx);
  return 0;
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
  dim3 grid;
  if (fd_grid(g, &grid)) return gb_last_error();
  cudaStream_t st = gb__stream();
  if (is_real) {
    if (g->prec == GB_FP32) k_fd<float, true><<<grid, kFdThreads, 0, st>>>(op, (float *) dst, (const float *) src, a);
    else k_fd<double, true><<<grid, kFdThreads, 0, st>>>(op, (double *) dst, (const double *) src, a);
  } else {
    if (g->prec == GB_FP32) k_fd<float, false><<<grid, kFdThreads, 0, st>>>(op, (float2 *) dst, (const float2 *) src, a);
    else k_fd<double, false><<<grid, kFdThreads, 0, st>>>(op, (double2 *) dst, (const double2 *) src, a);
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
  dim3 grid;
  if (fd_grid(g, &grid)) return gb_last_error();
  const long nb = (long) grid.x * grid.y * grid.z;
  double2 *partial = (double2 *) gb__scratch(GB_SCR_PARTIAL, sizeof(double2) * (size_t) nb);
  double2 *res = (double2 *) gb__result_slot();
  if (!partial || !res) return gb_last_error();
  cudaStream_t st = gb__stream();
  if (g->prec == GB_FP32) k_fd_kinetic<float><<<grid, kFdThreads, 0, st>>>((const float2 *) psi, a, partial);
  else k_fd_kinetic<double><<<grid, kFdThreads, 0, st>>>((const double2 *) psi, a, partial);
  GB_CHECK_LAUNCH("fd kinetic");
  k_finish_fd<<<1, 256, 0, st>>>(partial, nb, res);
  GB_CHECK_LAUNCH("fd kinetic finish");
  double2 h;
  int rc = gb__read_result(&h, sizeof(double2));
  out[0] = h.x;
  out[1] = h.y;
  return rc;
}
