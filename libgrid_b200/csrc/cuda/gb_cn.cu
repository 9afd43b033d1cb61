// Dimension-split Crank-Nicolson kinetic propagation on the B200.
//
// Follows the reference's grid_wf_propagate_cn_{x,y,z} (src/grid_wf_cn.c:
// 93-469) line by line, including its boundary rows: the Dirichlet and
// Neumann cases use grid_solve_tridiagonal_system2 (src/linalg.c:62-92),
// whose first super-diagonal and last sub-diagonal are 2 (so Dirichlet lines
// pair a zero-ghost right-hand side with Neumann-style end coefficients), and
// the Neumann right-hand side drops the moving-frame/rotation terms at the
// ends; the periodic case uses the Sherman-Morrison form of
// grid_solve_tridiagonal_system_cyclic2 (src/linalg.c:206-230).
//
// Fast path (no rotation, no absorbing region): every line of an axis sees
// the same matrix, so the elimination multipliers m_i, the reciprocal pivots
// 1/b'_i and (periodic) the Sherman-Morrison vector z are computed once on
// the host and each line needs only the right-hand side, one forward and one
// backward sweep.  A CTA is one warp that owns up to 32 lines: the tile is
// brought into shared memory with bulk asynchronous copies (one mbarrier,
// bounded wait), the optional potential half-step is applied in place, each
// lane sweeps its line, the second potential half-step is applied and the
// tile is written back with bulk copies.  Contiguous (z) lines are padded by
// one element in shared memory so the lane-per-line accesses hit distinct
// banks; strided (x, y) tiles hold 32 adjacent columns per row.
//
// General path (rotation or absorbing boundary): one thread per line with
// per-element pivots in a global workspace laid out [i][line].
#include <complex>
#include <math.h>
#include <string.h>
#include <vector>

#include "gb_common.cuh"
#include "gb_internal_cuda.h"

namespace {

using cd = std::complex<double>;

struct CnAxis {
  long nx, ny, nz;
  int axis;    // 0 x, 1 y, 2 z
  long n;      // line length
  long inner;  // strided: inner extent; contiguous: 1
  long outer;  // strided: outer extent; contiguous: number of lines
  int lpc;     // lines per CTA (fast path)
  int boundary;
  double2 cp;     // c / tstep (fast path)
  double2 c;      // 4 i m h^2 / hbar
  double2 tstep;  // base time step
  double2 c2;     // -i h k0 (axis)
  double2 c3;     // rotation coefficient (axis)
  double coord_off;
  double step;
  const double2 *tab;  // fast path: m[n], rb[n], z[n]
  long klo, khi;       // fast path: rows klo..khi take m, rb, Q from mc, rbc, qc
  double2 mc, rbc, qc;
  double2 beta, gamma, den;
  gb_potential pre, post;
  int absorb;
  long lx, hx, ly, hy, lz, hz;
  int *err;
  double2 *work;  // general path: 4 arrays of n * nlines
  long nlines;
};

__device__ __forceinline__ double2 cm(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 ca(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cs(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 csc(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// (ix, iy, iz) of element i of a line.  Contiguous lines: lid = line index
// over the two other axes in memory order.  Strided: lid = outer index o,
// q = inner index.
__device__ __forceinline__ void cn_decode(const CnAxis &a, long lid, long i, long q, long &ix, long &iy, long &iz) {
  if (a.axis == 2) {
    ix = lid / a.ny;
    iy = lid - ix * a.ny;
    iz = i;
  } else if (a.axis == 1) {
    ix = lid;
    iy = i;
    iz = q;
  } else {
    ix = i;
    iy = q / a.nz;
    iz = q - iy * a.nz;
  }
}

__device__ __forceinline__ double cn_absorb(long i, long j, long k, const CnAxis &a) {
  double t = 0.0;
  if (i < a.lx) t += (double) (a.lx - i) / (double) a.lx;
  else if (i > a.hx) t += (double) (i - a.hx) / (double) a.lx;
  if (j < a.ly) t += (double) (a.ly - j) / (double) a.ly;
  else if (j > a.hy) t += (double) (j - a.hy) / (double) a.ly;
  if (k < a.lz) t += (double) (a.lz - k) / (double) a.lz;
  else if (k > a.hz) t += (double) (k - a.hz) / (double) a.lz;
  t *= 2.0 / 3.0;
  return t > 1.0 ? 1.0 : t;
}


// psi * exp(c (cons + V + g |psi|^2)) (src/grid_wf.c:586-598), V given
__device__ __forceinline__ double2 cn_pot_with(double2 x, double2 v, long ix, long iy, long iz,
                                               const gb_potential &pt) {
  double wr = pt.cons + v.x, wi = v.y;
  if (pt.g != 0.0) wr += pt.g * (x.x * x.x + x.y * x.y);
  double cr = pt.c_re, ci = pt.c_im;
  if (pt.absorb) {
    double t = 0.0;
    if (ix < pt.lx) t += (double) (pt.lx - ix) / (double) pt.lx;
    else if (ix > pt.hx) t += (double) (ix - pt.hx) / (double) pt.lx;
    if (iy < pt.ly) t += (double) (pt.ly - iy) / (double) pt.ly;
    else if (iy > pt.hy) t += (double) (iy - pt.hy) / (double) pt.ly;
    if (iz < pt.lz) t += (double) (pt.lz - iz) / (double) pt.lz;
    else if (iz > pt.hz) t += (double) (iz - pt.hz) / (double) pt.lz;
    t *= 2.0 / 3.0;
    const double am = t > 1.0 ? 1.0 : t;
    cr = -pt.treal * am;
    ci = -pt.treal * (1.0 - am);
  }
  const double ar = cr * wr - ci * wi, ai = cr * wi + ci * wr;
  double s, c;
  gb_sincos(ai, &s, &c);
  if (ar != 0.0) {
    const double m = exp(ar);
    s *= m;
    c *= m;
  }
  return cm(x, make_double2(c, s));
}

// Right-hand side row i of a line (src/grid_wf_cn.c:139-201 and the y/z
// twins).  pm, p0, pp = psi[i-1], psi[i], psi[i+1]; pfirst/plast = psi[0],
// psi[n-1] for the periodic wrap; c3y = c3 * (perpendicular coordinate).
__device__ __forceinline__ double2 cn_rhs(long i, long n, int bc, double2 cp, double2 c2, double2 c3y, double2 pm,
                                          double2 p0, double2 pp, double2 pfirst, double2 plast) {
  const double2 two_p0 = csc(p0, 2.0);
  if (i > 0 && i < n - 1) {
    const double2 lap = ca(cs(pp, two_p0), pm);
    const double2 dif = cs(pp, pm);
    return cs(cs(cs(cm(cp, p0), lap), cm(c2, dif)), cm(c3y, dif));
  }
  if (i == 0) {
    if (bc == 1) return cs(cs(cs(cm(cp, p0), cs(pp, two_p0)), cm(c2, pp)), cm(c3y, pp));
    if (bc == 2) return cs(cm(cp, p0), cs(csc(pp, 2.0), two_p0));
    const double2 dif = cs(pp, plast);
    return cs(cs(cs(cm(cp, p0), ca(cs(pp, two_p0), plast)), cm(c2, dif)), cm(c3y, dif));
  }
  // i == n - 1
  if (bc == 1) return ca(ca(cs(cm(cp, p0), cs(pm, two_p0)), cm(c2, pm)), cm(c3y, pm));
  if (bc == 2) return cs(cm(cp, p0), cs(csc(pm, 2.0), two_p0));
  const double2 dif = cs(pfirst, pm);
  return cs(cs(cs(cm(cp, p0), ca(cs(pm, two_p0), pfirst)), cm(c2, dif)), cm(c3y, dif));
}

// Potential factor on the elements i = i0, i0 + di, ... < n of one tile line
// or column whose element i sits at base[i * es]; V of element i at
// vbase + i * vstep, coordinates (ix, iy, iz) with the line's own axis
// running along i.  No division per element; V loads batched by B.
__device__ __forceinline__ void cn_pot_elems(double2 *base, int es, int i0, int di, int n, long vbase, long vstep,
                                             long ix, long iy, long iz, const CnAxis &a, const gb_potential &pt) {
  constexpr int B = 4;
  for (int ib = i0; ib < n; ib += di * B) {
    double2 v[B];
#pragma unroll
    for (int k = 0; k < B; k++) {
      const int i = ib + k * di;
      v[k] = make_double2(0.0, 0.0);
      if (i < n) {
        const long vi = vbase + i * vstep;
        // streaming loads: V is read once per sweep, and evict-first keeps
        // the solver's coefficient tables in the small L1 left beside the
        // shared-memory tiles
        if (pt.kind == GB_POT_COMPLEX) v[k] = __ldcs((const double2 *) pt.v + vi);
        else if (pt.kind == GB_POT_REAL) v[k].x = __ldcs((const double *) pt.v + vi);
      }
    }
#pragma unroll
    for (int k = 0; k < B; k++) {
      const int i = ib + k * di;
      if (i < n) {
        double2 &r = base[i * es];
        const long jx = a.axis == 0 ? i : ix, jy = a.axis == 1 ? i : iy, jz = a.axis == 2 ? i : iz;
        r = cn_pot_with(r, v[k], jx, jy, jz, pt);
      }
    }
  }
}

// Potential factor over a whole tile in shared memory.  Contiguous tiles
// (lines along z, element (l, i) at sm[l * pitch + i]): one line per warp
// at a time, lanes along the line.  Strided tiles (element (l, i) at
// sm[i * pitch + l], pitch >= cols): one column per thread, `cols` columns
// side by side, threads of equal column spaced along the rows.
template <bool CONTIG>
__device__ __forceinline__ void cn_tile_pot(double2 *sm, int pitch, int cols, int nl, long line0, long o, long col0,
                                            const CnAxis &a, const gb_potential &pt) {
  const int n = (int) a.n, nthr = (int) blockDim.x;
  const long vrow = pt.vrow;
  if constexpr (CONTIG) {
    for (int l = (int) (threadIdx.x >> 5); l < nl; l += nthr >> 5) {
      const long lid = line0 + l;
      const long ix = lid / a.ny, iy = lid - ix * a.ny;
      cn_pot_elems(sm + (long) l * pitch, 1, (int) (threadIdx.x & 31), 32, n, (ix * a.ny + iy) * vrow, 1, ix, iy, 0,
                   a, pt);
    }
  } else {
    const int l = (int) threadIdx.x % cols;
    if (l >= nl) return;
    const long q = col0 + l;
    long ix = 0, iy = 0, iz = 0, vbase, vstep;
    if (a.axis == 0) {
      iy = q / a.nz;
      iz = q - iy * a.nz;
      vbase = iy * vrow + iz;
      vstep = a.ny * vrow;
    } else {
      ix = o;
      iz = q;
      vbase = ix * a.ny * vrow + iz;
      vstep = vrow;
    }
    cn_pot_elems(sm + l, pitch, (int) threadIdx.x / cols, nthr / cols, n, vbase, vstep, ix, iy, iz, a, pt);
  }
}

// Segments per line in the fast kernel (= warps per CTA).
constexpr int kSeg = 16;

// Contiguous tile rows are padded to an odd number of 16-byte elements so a
// warp's lane-per-line accesses fall in distinct shared-memory banks.
__host__ __device__ inline long contig_row(long n) { return (n & 1) ? n : n + 1; }

// Shared-memory element (l, i) of a tile; row = padded line length
// (contiguous) or lines per tile (strided).
template <bool CONTIG> __device__ __forceinline__ double2 &tile_at(double2 *sm, int l, long i, long row) {
  if constexpr (CONTIG) return sm[(long) l * row + i];
  else return sm[i * row + l];
}

// Fast path.  A CTA of 16 warps owns up to 32 lines (lane = line); warp s
// owns segment s = [s S, (s+1) S) of every line, S = ceil(n / 16) (at most
// SMAX when SMAX > 0).  Both
// Thomas recurrences are linear with line-independent coefficients:
//   forward  v_i = b_i - m_i v_{i-1}
//   backward x_i = rb_i v_i + Q_i x_{i+1},   Q_i = -rb_i c_i
// so each warp runs the particular recurrence of its segment from a zero
// carry-in, one warp chains the 16 segment carries per line, and every
// element then adds (carry-in) x (homogeneous response), whose tables
// H_i = prod(-m_j) and G_i = prod(Q_j) over the segment are precomputed.
// Loop k = 0 .. cnt - 1 (seg_loop_rev: downwards) over a segment; SMAX > 0
// unrolls it for segments of at most SMAX points, so the table loads of
// all steps issue ahead of the recurrence.
template <int SMAX, class F> __device__ __forceinline__ void seg_loop(int cnt, F &&f) {
  if constexpr (SMAX > 0) {
#pragma unroll
    for (int k = 0; k < SMAX; k++)
      if (k < cnt) f(k);
  } else {
    for (int k = 0; k < cnt; k++) f(k);
  }
}

template <int SMAX, class F> __device__ __forceinline__ void seg_loop_rev(int cnt, F &&f) {
  if constexpr (SMAX > 0) {
#pragma unroll
    for (int k = SMAX - 1; k >= 0; k--)
      if (k < cnt) f(k);
  } else {
    for (int k = cnt - 1; k >= 0; k--) f(k);
  }
}

template <bool CONTIG, int SMAX>
__global__ void __launch_bounds__(32 * kSeg, 2) k_cn_fast(double2 *__restrict__ psi, CnAxis a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(8) uint64_t bar;
  // segment end values, replaced in place by the segments' carries
  __shared__ double2 s_car[kSeg][32];
  __shared__ double2 s_fact[32];
  double2 *sm = (double2 *) smraw;
  const int tid = threadIdx.x, lane = tid & 31, seg = tid >> 5;
  const long n = a.n;
  const int lpc = a.lpc;
  const long row = CONTIG ? contig_row(n) : (long) lpc;
  long line0 = 0, o = 0, col0 = 0;
  int nl;
  if constexpr (CONTIG) {
    line0 = (long) blockIdx.x * lpc;
    const long rem = a.outer - line0;
    nl = (int) (rem < lpc ? rem : lpc);
  } else {
    o = blockIdx.y;
    col0 = (long) blockIdx.x * lpc;
    nl = lpc;
  }
  const double2 zero = make_double2(0.0, 0.0);

  // ---- tile load (bulk copies, one mbarrier, bounded wait)
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(&bar, (unsigned) (nl * n * 16));
  }
  __syncthreads();
  if constexpr (CONTIG) {
    for (int l = tid; l < nl; l += 32 * kSeg) bulk_g2s(sm + (long) l * row, psi + (line0 + l) * n, (unsigned) (n * 16), &bar);
  } else {
    for (long i = tid; i < n; i += 32 * kSeg)
      bulk_g2s(sm + i * row, psi + o * n * a.inner + i * a.inner + col0, (unsigned) (nl * 16), &bar);
  }
  if (!mbar_wait_bounded(&bar, 0)) {
    if (tid == 0) atomicExch(a.err, 1);
    mbar_wait_bounded(&bar, 0);
    return;
  }

  // ---- optional first potential half-step (all threads, element-parallel)
  if (a.pre.kind != GB_POT_NONE || a.pre.g != 0.0)
    cn_tile_pot<CONTIG>(sm, (int) row, lpc, nl, line0, o, col0, a, a.pre);
  __syncthreads();

  const double2 *tm = a.tab, *trb = a.tab + n, *tz = a.tab + 2 * n, *tH = a.tab + 3 * n, *tQ = a.tab + 4 * n,
                *tG = a.tab + 5 * n;
  const long S = (n + kSeg - 1) / kSeg;
  const long a0 = seg * S, e0 = (a0 + S < n) ? a0 + S : n;
  const int cnt = a0 < e0 ? (int) (e0 - a0) : 0;
  const long klo = a.klo, khi = a.khi;
  const double2 mc = a.mc, rbc = a.rbc, qc = a.qc;
  const bool active = (lane < nl) && (cnt > 0);
  const int bc = a.boundary;

  // ---- neighbours of the segment, read before anything is overwritten
  double2 pfirst = zero, plast = zero, p_before = zero, p_after = zero;
  if (lane < nl) {
    pfirst = tile_at<CONTIG>(sm, lane, 0, row);
    plast = tile_at<CONTIG>(sm, lane, n - 1, row);
  }
  if (active) {
    p_before = (a0 > 0) ? tile_at<CONTIG>(sm, lane, a0 - 1, row) : plast;
    p_after = (e0 < n) ? tile_at<CONTIG>(sm, lane, e0, row) : pfirst;
  }
  __syncthreads();

  // ---- right-hand side + forward particular recurrence (zero carry-in)
  double2 u = zero;
  if (active) {
    double2 pm = p_before, p0 = tile_at<CONTIG>(sm, lane, a0, row);
    seg_loop<SMAX>(cnt, [&](int k) {
      const long i = a0 + k;
      const double2 pp = (k + 1 < cnt) ? tile_at<CONTIG>(sm, lane, i + 1, row) : p_after;
      const double2 b = cn_rhs(i, n, bc, a.cp, a.c2, zero, pm, p0, pp, pfirst, plast);
      const double2 mi = (i >= klo && i <= khi) ? mc : __ldg(tm + i);
      u = (k == 0) ? b : cs(b, cm(mi, u));
      tile_at<CONTIG>(sm, lane, i, row) = u;
      pm = p0;
      p0 = pp;
    });
  }
  if (lane < nl) s_car[seg][lane] = u;
  __syncthreads();
  if (seg == 0 && lane < nl) {
    double2 vin = zero;
#pragma unroll
    for (int s = 0; s < kSeg; s++) {
      const long as = s * S, es = (as + S < n) ? as + S : n;
      const double2 e = s_car[s][lane];
      s_car[s][lane] = vin;
      if (as < es) vin = ca(e, cm(__ldg(tH + es - 1), vin));
    }
  }
  __syncthreads();

  // ---- forward fix-up fused with the backward particular recurrence
  double2 y = zero;
  if (active) {
    const double2 vin = s_car[seg][lane];
    seg_loop_rev<SMAX>(cnt, [&](int k) {
      const long i = a0 + k;
      const double2 v = ca(tile_at<CONTIG>(sm, lane, i, row), cm(__ldg(tH + i), vin));
      const bool cst = i >= klo && i <= khi;
      const double2 rbi = cst ? rbc : __ldg(trb + i), qi = cst ? qc : __ldg(tQ + i);
      y = (k == cnt - 1) ? cm(rbi, v) : ca(cm(rbi, v), cm(qi, y));
      tile_at<CONTIG>(sm, lane, i, row) = y;
    });
  }
  if (lane < nl) s_car[seg][lane] = y;
  __syncthreads();
  if (seg == 0 && lane < nl) {
    double2 xin = zero;
#pragma unroll
    for (int s = kSeg - 1; s >= 0; s--) {
      const long as = s * S, es = (as + S < n) ? as + S : n;
      const double2 e = s_car[s][lane];
      s_car[s][lane] = xin;
      if (as < es) xin = ca(e, cm(__ldg(tG + as), xin));
    }
    if (bc == 3) {
      // Sherman-Morrison: fact = (x_0 + beta x_{n-1} / gamma) / den; the
      // segment holding n-1 has a zero carry-in, so x_{n-1} = y_{n-1}.
      const double2 xl = tile_at<CONTIG>(sm, lane, n - 1, row);
      s_fact[lane] = cm(ca(xin, cm(a.beta, cm(xl, a.gamma))), a.den);  // gamma, den hold reciprocals
    }
  }
  __syncthreads();

  // ---- backward fix-up and periodic correction
  if (active) {
    const double2 xin = s_car[seg][lane];
    const double2 fact = (bc == 3) ? s_fact[lane] : zero;
    seg_loop<SMAX>(cnt, [&](int k) {
      const long i = a0 + k;
      double2 x = ca(tile_at<CONTIG>(sm, lane, i, row), cm(__ldg(tG + i), xin));
      if (bc == 3) x = cs(x, cm(fact, __ldg(tz + i)));
      tile_at<CONTIG>(sm, lane, i, row) = x;
    });
  }
  // ---- optional second potential half-step (element-parallel)
  if (a.post.kind != GB_POT_NONE || a.post.g != 0.0) {
    __syncthreads();
    cn_tile_pot<CONTIG>(sm, (int) row, lpc, nl, line0, o, col0, a, a.post);
  }

  // ---- tile store
  fence_proxy_async_smem();
  __syncthreads();
  if constexpr (CONTIG) {
    for (int l = tid; l < nl; l += 32 * kSeg) bulk_s2g(psi + (line0 + l) * n, sm + (long) l * row, (unsigned) (n * 16));
  } else {
    for (long i = tid; i < n; i += 32 * kSeg)
      bulk_s2g(psi + o * n * a.inner + i * a.inner + col0, sm + i * row, (unsigned) (nl * 16));
  }
  bulk_commit();
  // the CTA may leave once the stores have read shared memory; their global
  // writes complete with the grid
  bulk_wait_read_all();
}

// ---------------------------------------------------------------------------
// Warp-cooperative fast path for lines of up to 32 * kLaneSegMax points.
//
// One warp solves one line.  Lane s owns the contiguous segment
// [s S, s S + S) of the line, S = ceil(n / 32) <= kLaneSegMax, held in
// registers.  Each lane runs the two Thomas recurrences of its segment from a
// zero carry (forward v_i = b_i - m_i v_{i-1}, backward
// x_i = rb_i v_i + q_i x_{i+1}); the true carries are then the prefix sums of
// the affine segment maps carry_out = u_end + A_s carry_in (backward:
// y_start + B_s carry_in), which a warp-shuffle scan (recursive doubling,
// 5 levels) resolves.  The matrix is the same for every line, so the
// segment responses A_s = prod(-m) and B_s = prod(q) and their window
// products for each scan level are host-precomputed tables, and the scan
// costs one complex multiply-add per level.  The fix-ups add carry x
// homogeneous response (tables H, G) to every element.  No CTA barrier sits
// inside the solve.
//
// CTAs are persistent and double-buffered: while the warps solve the lines
// of one tile (W lines, one per warp), warp 0 has the bulk copies of the
// next tile in flight.  Tiles: W consecutive lines (contiguous axis, rows
// padded to an odd length) or W adjacent columns x n rows (strided axes, row
// pitch W + 1), so the lanes' segment accesses hit at most two-way bank
// conflicts.
constexpr int kLaneSegMax = 8;
constexpr int kCnWarps = 8;  // warps per CTA
constexpr int kCnWarpThreads = 32 * kCnWarps;
// lines per tile: one per warp on the contiguous axis; two per warp on the
// strided axes, so each row of a strided tile is one 256-byte copy
template <bool CONTIG> __host__ __device__ constexpr int tile_lines() { return CONTIG ? kCnWarps : 2 * kCnWarps; }

__host__ __device__ inline long warp_pitch(bool contig, long n) {
  return contig ? contig_row(n) : (contig ? kCnWarps : 2 * kCnWarps) + 1;
}

// Offsets of the scan tables behind the six per-element tables.
__host__ __device__ inline long warp_scan_off(long n) { return 6 * n; }

__device__ __forceinline__ double2 shfl_up2(double2 v, int d) {
  return make_double2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ double2 shfl_down2(double2 v, int d) {
  return make_double2(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
}

// Solve line l of the tile in place (the whole warp); SMAX >= ceil(n / 32).
template <bool CONTIG, int SMAX>
__device__ __forceinline__ void cn_warp_line(double2 *sm, int pitch, int l, const CnAxis &a, int lane) {
  const int n = (int) a.n;
  const int S = (n + 31) >> 5;
  const int bc = a.boundary;
  const double2 zero = make_double2(0.0, 0.0);
  const double2 *tm = a.tab, *trb = a.tab + n, *tz = a.tab + 2 * n, *tH = a.tab + 3 * n, *tQ = a.tab + 4 * n,
                *tG = a.tab + 5 * n;
  const double2 *wf = a.tab + warp_scan_off(n), *wb = wf + 5 * 32;
  // element i of the line: contiguous tiles hold lines as rows, strided
  // tiles hold them as columns
  double2 *const base = CONTIG ? sm + l * pitch : sm + l;
  const int es = CONTIG ? 1 : pitch;
  auto at = [&](int i) -> double2 & { return base[i * es]; };
  const int a0 = lane * S;
  const int cnt = a0 >= n ? 0 : (n - a0 < S ? n - a0 : S);
  double2 p[SMAX];
#pragma unroll
  for (int j = 0; j < SMAX; j++) p[j] = (j < cnt) ? at(a0 + j) : zero;
  // the line's first and last elements and the segment neighbours, read
  // before any lane writes (selecting them from the register arrays by a
  // runtime index would move the arrays to local memory)
  const double2 pfirst = at(0), plast = at(n - 1);
  const double2 p_before = (a0 > 0 && a0 <= n) ? at(a0 - 1) : zero;
  const double2 p_after = (a0 + cnt < n) ? at(a0 + cnt) : zero;
  __syncwarp();

  // right-hand side and forward particular recurrence (zero carry-in)
  double2 u = zero, pm = p_before;
#pragma unroll
  for (int j = 0; j < SMAX; j++) {
    if (j < cnt) {
      const int i = a0 + j;
      const double2 p0 = p[j];
      const double2 pp = (j + 1 < cnt) ? p[j + 1] : p_after;
      const double2 b = cn_rhs(i, n, bc, a.cp, a.c2, zero, pm, p0, pp, pfirst, plast);
      u = (j == 0) ? b : cs(b, cm(__ldg(tm + i), u));
      pm = p0;
      p[j] = u;
    }
  }
  // forward carries: inclusive scan of carry_out = u_end + A_s carry_in
  double2 x = (cnt > 0) ? u : zero;
#pragma unroll
  for (int d = 0; d < 5; d++) {
    const double2 y = shfl_up2(x, 1 << d);
    if (lane >= (1 << d)) x = ca(x, cm(__ldg(wf + d * 32 + lane), y));
  }
  double2 vin = shfl_up2(x, 1);
  if (lane == 0) vin = zero;
  // forward fix-up fused with the backward particular recurrence
  double2 yv = zero, ystart = zero;
#pragma unroll
  for (int j = SMAX - 1; j >= 0; j--) {
    if (j < cnt) {
      const int i = a0 + j;
      const double2 v = ca(p[j], cm(__ldg(tH + i), vin));
      yv = (j == cnt - 1) ? cm(__ldg(trb + i), v) : ca(cm(__ldg(trb + i), v), cm(__ldg(tQ + i), yv));
      p[j] = yv;
      ystart = yv;
    }
  }
  // backward carries: suffix scan of carry_out = y_start + B_s carry_in
  x = ystart;
#pragma unroll
  for (int d = 0; d < 5; d++) {
    const double2 y = shfl_down2(x, 1 << d);
    if (lane + (1 << d) < 32) x = ca(x, cm(__ldg(wb + d * 32 + lane), y));
  }
  double2 xin = shfl_down2(x, 1);
  if (lane == 31) xin = zero;
#pragma unroll
  for (int j = 0; j < SMAX; j++)
    if (j < cnt) {
      p[j] = ca(p[j], cm(__ldg(tG + a0 + j), xin));
      at(a0 + j) = p[j];
    }
  if (bc == 3) {
    // Sherman-Morrison: fact = (x_0 + beta x_{n-1} / gamma) / den, with
    // x_0 and x_{n-1} read back from the line
    __syncwarp();
    const double2 x0 = at(0), xl = at(n - 1);
    const double2 fact = cm(ca(x0, cm(a.beta, cm(xl, a.gamma))), a.den);  // gamma, den hold reciprocals
    __syncwarp();
#pragma unroll
    for (int j = 0; j < SMAX; j++)
      if (j < cnt) at(a0 + j) = cs(p[j], cm(fact, __ldg(tz + a0 + j)));
  }
}

// Potential half-step on every element of a tile (all threads).  Each
// thread keeps one line (contiguous) or one column (strided) and walks its
// elements, so the grid coordinates of the line are decoded once; the V
// values of a batch of elements are loaded before any phase is applied.
struct CnTile {
  long line0, o, col0;
  int nl;
};

template <bool CONTIG> __device__ __forceinline__ CnTile cn_tile_of(const CnAxis &a, long t, long tpo) {
  CnTile c;
  constexpr int TL = tile_lines<CONTIG>();
  if constexpr (CONTIG) {
    c.line0 = t * TL;
    const long rem = a.outer - c.line0;
    c.nl = (int) (rem < TL ? rem : TL);
    c.o = c.col0 = 0;
  } else {
    c.o = t / tpo;
    c.col0 = (t - c.o * tpo) * TL;
    const long rem = a.inner - c.col0;
    c.nl = (int) (rem < TL ? rem : TL);
    c.line0 = 0;
  }
  return c;
}

// This thread's bulk copy of one tile between global memory and a shared
// buffer: contiguous tiles one line per thread, strided tiles one row per
// thread (n <= 256 rows; load completion on bar).
template <bool CONTIG, bool LOAD>
__device__ __forceinline__ void cn_tile_copy(double2 *psi, double2 *buf, int pitch, const CnTile &c, const CnAxis &a,
                                             uint64_t *bar, int tid) {
  const long n = a.n;
  if constexpr (CONTIG) {
    if (tid < c.nl) {
      double2 *g = psi + (c.line0 + tid) * n;
      if (LOAD) bulk_g2s(buf + tid * pitch, g, (unsigned) (n * 16), bar);
      else bulk_s2g(g, buf + tid * pitch, (unsigned) (n * 16));
    }
  } else {
    for (int i = tid; i < n; i += kCnWarpThreads) {
      double2 *g = psi + (c.o * n + i) * a.inner + c.col0;
      if (LOAD) bulk_g2s(buf + i * pitch, g, (unsigned) (c.nl * 16), bar);
      else bulk_s2g(g, buf + i * pitch, (unsigned) (c.nl * 16));
    }
  }
}

template <bool CONTIG, int SMAX>
__global__ void __launch_bounds__(kCnWarpThreads, 2) k_cn_warp(double2 *__restrict__ psi, CnAxis a, long ntiles, long tpo) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(8) uint64_t bars[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = (int) a.n;
  const int pitch = (int) warp_pitch(CONTIG, n);
  const int bufsz = CONTIG ? tile_lines<CONTIG>() * pitch : n * pitch;
  double2 *const buf0 = (double2 *) smraw;
  auto buf = [&](int b) { return buf0 + (b ? bufsz : 0); };
  long t = blockIdx.x;
  if (t >= ntiles) return;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(&bars[0], (unsigned) (cn_tile_of<CONTIG>(a, t, tpo).nl * a.n * 16));
  }
  __syncthreads();
  cn_tile_copy<CONTIG, true>(psi, buf(0), pitch, cn_tile_of<CONTIG>(a, t, tpo), a, &bars[0], tid);
  const bool pre = (a.pre.kind != GB_POT_NONE || a.pre.g != 0.0);
  const bool post = (a.post.kind != GB_POT_NONE || a.post.g != 0.0);
  for (unsigned it = 0; t < ntiles; t += gridDim.x, it++) {
    const int b = it & 1;
    const long next = t + gridDim.x;
    // prefetch the next tile into the other buffer once the previous tile's
    // stores (issued by the same threads) have read it
    bulk_wait_read_all();
    if (tid == 0 && next < ntiles)
      mbar_arrive_expect_tx(&bars[b ^ 1], (unsigned) (cn_tile_of<CONTIG>(a, next, tpo).nl * a.n * 16));
    __syncthreads();
    if (next < ntiles) cn_tile_copy<CONTIG, true>(psi, buf(b ^ 1), pitch, cn_tile_of<CONTIG>(a, next, tpo), a, &bars[b ^ 1], tid);
    const bool ok = mbar_wait_bounded(&bars[b], (it >> 1) & 1u);
    if (__syncthreads_or(!ok)) {
      // a copy never completed: record it, let the copies in flight land
      // (bounded), drain the stores and leave
      if (tid == 0) {
        atomicExch(a.err, 1);
        mbar_wait_bounded(&bars[b], (it >> 1) & 1u);
        if (next < ntiles) mbar_wait_bounded(&bars[b ^ 1], ((it + 1) >> 1) & 1u);
      }
      bulk_wait_all();
      return;
    }
    const CnTile c = cn_tile_of<CONTIG>(a, t, tpo);
    double2 *sm = buf(b);
    if (pre) {
      cn_tile_pot<CONTIG>(sm, pitch, tile_lines<false>(), c.nl, c.line0, c.o, c.col0, a, a.pre);
      __syncthreads();
    }
    for (int l = warp; l < c.nl; l += kCnWarps) cn_warp_line<CONTIG, SMAX>(sm, pitch, l, a, lane);
    if (post) {
      __syncthreads();
      cn_tile_pot<CONTIG>(sm, pitch, tile_lines<false>(), c.nl, c.line0, c.o, c.col0, a, a.post);
    }
    fence_proxy_async_smem();
    __syncthreads();
    cn_tile_copy<CONTIG, false>(psi, sm, pitch, c, a, nullptr, tid);
    bulk_commit();
  }
  // the CTA may leave once the stores have read shared memory; their global
  // writes complete with the grid
  bulk_wait_read_all();
}

// General path: one thread per line, element (line, i) of a workspace array
// at [i * nlines + line].  Handles rotation (c3) and absorbing boundaries.
__global__ void k_cn_general(double2 *__restrict__ psi, CnAxis a) {
  const long line = blockIdx.x * (long) blockDim.x + threadIdx.x;
  if (line >= a.nlines) return;
  const long n = a.n, NL = a.nlines;
  double2 *V = a.work, *RB = a.work + n * NL, *M = a.work + 2 * n * NL, *Z = a.work + 3 * n * NL;
  // line -> (outer, inner) addressing and element stride
  long base, stride, lid, q;
  if (a.inner == 1) {
    lid = line;
    q = 0;
    base = line * n;
    stride = 1;
  } else {
    lid = line / a.inner;
    q = line - lid * a.inner;
    base = lid * n * a.inner + q;
    stride = a.inner;
  }
  long ix, iy, iz;
  cn_decode(a, lid, 0, q, ix, iy, iz);
  double coord = 0.0;
  if (a.axis == 0) coord = (double) (iy - a.ny / 2) * a.step - a.coord_off;
  else if (a.axis == 1) coord = (double) (ix - a.nx / 2) * a.step - a.coord_off;
  const double2 c3y = csc(a.c3, coord);
  const double2 c2e = ca(a.c2, c3y);
  const double2 cc2p = make_double2(1.0 + c2e.x, c2e.y), cc2m = make_double2(1.0 - c2e.x, -c2e.y);
  const double2 two = make_double2(2.0, 0.0);
  const int bc = a.boundary;

  auto cp_at = [&](long i) -> double2 {
    double2 tim = a.tstep;
    if (a.absorb) {
      long jx, jy, jz;
      cn_decode(a, lid, i, q, jx, jy, jz);
      const double t = cn_absorb(jx, jy, jz, a);
      tim = make_double2((1.0 - t) * a.tstep.x, -a.tstep.x * t);
    }
    return cdiv(a.c, tim);
  };
  auto P = [&](long i) -> double2 { return psi[base + i * stride]; };

  // right-hand side into V, diagonal (with periodic corner changes) into RB
  const double2 pfirst = P(0), plast = P(n - 1);
  double2 pm = plast, p0 = pfirst;
  for (long i = 0; i < n; i++) {
    const double2 pp = (i + 1 < n) ? P(i + 1) : pfirst;
    const double2 cp = cp_at(i);
    V[i * NL + line] = cn_rhs(i, n, bc, cp, a.c2, c3y, pm, p0, pp, pfirst, plast);
    RB[i * NL + line] = cs(cp, two);
    pm = p0;
    p0 = pp;
  }
  double2 gamma = make_double2(0.0, 0.0), alpha = cc2p, beta = cc2m;
  if (bc == 3) {
    const double2 d0 = RB[line];
    gamma = make_double2(-d0.x, -d0.y);
    RB[line] = cs(d0, gamma);
    RB[(n - 1) * NL + line] = cs(RB[(n - 1) * NL + line], cdiv(cm(alpha, beta), gamma));
  }
  // forward elimination; RB becomes 1/b'
  double2 bprev = RB[line];
  RB[line] = cdiv(make_double2(1.0, 0.0), bprev);
  double2 vprev = V[line];
  for (long i = 1; i < n; i++) {
    double2 sub, sup;
    if (bc == 3) {
      sub = cc2m;
      sup = cc2p;
    } else {
      sub = (i == n - 1) ? two : cc2m;
      sup = (i == 1) ? two : cc2p;
    }
    const double2 m = cdiv(sub, bprev);
    const double2 bi = cs(RB[i * NL + line], cm(m, sup));
    M[i * NL + line] = m;
    RB[i * NL + line] = cdiv(make_double2(1.0, 0.0), bi);
    vprev = cs(V[i * NL + line], cm(m, vprev));
    V[i * NL + line] = vprev;
    bprev = bi;
  }
  // back substitution
  double2 x = cm(vprev, RB[(n - 1) * NL + line]);
  V[(n - 1) * NL + line] = x;
  const double2 xlast = x;
  for (long i = n - 2; i >= 0; i--) {
    const double2 ci = (i == 0 && bc != 3) ? two : cc2p;
    x = cm(cs(V[i * NL + line], cm(ci, x)), RB[i * NL + line]);
    V[i * NL + line] = x;
  }
  if (bc == 3) {
    // second system with right-hand side (gamma, 0, ..., 0, alpha)
    double2 zp = gamma;
    Z[line] = zp;
    for (long i = 1; i < n; i++) {
      const double2 rhs = (i == n - 1) ? alpha : make_double2(0.0, 0.0);
      zp = cs(rhs, cm(M[i * NL + line], zp));
      Z[i * NL + line] = zp;
    }
    double2 z = cm(zp, RB[(n - 1) * NL + line]);
    Z[(n - 1) * NL + line] = z;
    const double2 zlast = z;
    for (long i = n - 2; i >= 0; i--) {
      z = cm(cs(Z[i * NL + line], cm(cc2p, z)), RB[i * NL + line]);
      Z[i * NL + line] = z;
    }
    const double2 num = ca(x, cdiv(cm(beta, xlast), gamma));
    const double2 den = ca(ca(make_double2(1.0, 0.0), z), cdiv(cm(beta, zlast), gamma));
    const double2 fact = cdiv(num, den);
    for (long i = 0; i < n; i++) psi[base + i * stride] = cs(V[i * NL + line], cm(fact, Z[i * NL + line]));
  } else {
    for (long i = 0; i < n; i++) psi[base + i * stride] = V[i * NL + line];
  }
}

// Host-side uniform tables for one axis: m, 1/b', z (periodic), and the
// segment responses H (forward) and G (backward) with Q_i = -c_i / b'_i,
// plus the periodic scalars.
struct FastTables {
  std::vector<double2> tab;  // 6 n: m, rb, z, H, Q, G; then (32 segments) the scan tables
  double2 beta, inv_gamma, inv_den;
  long klo, khi;             // rows whose m, rb and Q equal those of row klo bit for bit
  double2 mc, rbc, qc;
};

// nseg segments per line: kSeg for the segment-per-warp kernel, 32 for the
// warp-cooperative one, whose scan tables follow the six per-element tables:
// wf[d][s] = prod_{r = s - 2^d + 1 .. s} A_r with A_r = H at the end of
// segment r, and wb[d][s] = prod_{r = s .. s + 2^d - 1} B_r with B_r = G at
// the start of segment r (1 for empty segments).
static void build_fast_tables(long n, int bc, cd cp, cd c2, int nseg, FastTables &t) {
  const long ntab = 6 * n + (nseg == 32 ? 2 * 5 * 32 : 0);
  t.tab.assign(ntab, make_double2(0.0, 0.0));
  const cd d = cp - 2.0;
  std::vector<cd> bmod(n, d), m(n, 0.0), rb(n), q(n), H(n), G(n);
  cd alpha = 1.0 + c2, beta = 1.0 - c2, gamma = -d;
  if (bc == 3) {
    bmod[0] = d - gamma;
    bmod[n - 1] = bmod[n - 1] - alpha * beta / gamma;
  }
  cd bp = bmod[0];
  rb[0] = 1.0 / bp;
  for (long i = 1; i < n; i++) {
    cd sub, sup;
    if (bc == 3) {
      sub = 1.0 - c2;
      sup = 1.0 + c2;
    } else {
      sub = (i == n - 1) ? cd(2.0) : 1.0 - c2;
      sup = (i == 1) ? cd(2.0) : 1.0 + c2;
    }
    m[i] = sub / bp;
    bp = bmod[i] - m[i] * sup;
    rb[i] = 1.0 / bp;
  }
  for (long i = 0; i < n; i++) {
    const cd ci = (i == 0 && bc != 3) ? cd(2.0) : 1.0 + c2;
    q[i] = -rb[i] * ci;
  }
  const long S = (n + nseg - 1) / nseg;
  std::vector<cd> A(nseg, 1.0), B(nseg, 1.0);
  for (long s = 0; s < nseg; s++) {
    const long as = s * S, es = (as + S < n) ? as + S : n;
    for (long i = as; i < es; i++) H[i] = (i == as) ? -m[i] : H[i - 1] * (-m[i]);
    for (long i = es - 1; i >= as; i--) G[i] = (i == es - 1) ? q[i] : q[i] * G[i + 1];
    if (as < es) {
      A[s] = H[es - 1];
      B[s] = G[as];
    }
  }
  if (nseg == 32) {
    for (int d = 0; d < 5; d++) {
      const int w = 1 << d;
      for (int s = 0; s < 32; s++) {
        cd pf = 1.0, pb = 1.0;
        for (int r = s - w + 1; r <= s; r++) pf = (r >= 0) ? pf * A[r] : cd(0.0);
        for (int r = s; r < s + w; r++) pb = (r < 32) ? pb * B[r] : cd(0.0);
        t.tab[6 * n + d * 32 + s] = make_double2(pf.real(), pf.imag());
        t.tab[6 * n + 5 * 32 + d * 32 + s] = make_double2(pb.real(), pb.imag());
      }
    }
  }
  std::vector<cd> z(n, 0.0);
  cd den = 1.0;
  if (bc == 3) {
    std::vector<cd> v(n, 0.0);
    v[0] = gamma;
    v[n - 1] += alpha;
    for (long i = 1; i < n; i++) v[i] -= m[i] * v[i - 1];
    z[n - 1] = v[n - 1] * rb[n - 1];
    for (long i = n - 2; i >= 0; i--) z[i] = (v[i] - (1.0 + c2) * z[i + 1]) * rb[i];
    den = 1.0 + z[0] + beta * z[n - 1] / gamma;
  }
  auto put = [&](long base, const std::vector<cd> &x) {
    for (long i = 0; i < n; i++) t.tab[base + i] = make_double2(x[i].real(), x[i].imag());
  };
  put(0, m);
  put(n, rb);
  put(2 * n, z);
  put(3 * n, H);
  put(4 * n, q);
  put(5 * n, G);
  // The elimination of a diagonally dominant constant-coefficient matrix
  // reaches a fixed point within a few rows: m, rb and Q of the interior
  // rows are then the same numbers.  The widest such run of rows lets the
  // solver take these three from registers instead of the tables.
  {
    auto same = [&](long i, long j) {
      return m[i] == m[j] && rb[i] == rb[j] && q[i] == q[j];
    };
    long best_lo = n, best_hi = -1;
    for (long i = 0; i < n;) {
      long j = i;
      while (j + 1 < n && same(j + 1, i)) j++;
      if (j - i > best_hi - best_lo) {
        best_lo = i;
        best_hi = j;
      }
      i = j + 1;
    }
    if (best_hi - best_lo < 8) {  // no useful run: tables everywhere
      best_lo = n;
      best_hi = -1;
    }
    t.klo = best_lo;
    t.khi = best_hi;
    const long k = best_lo < n ? best_lo : 0;
    t.mc = make_double2(m[k].real(), m[k].imag());
    t.rbc = make_double2(rb[k].real(), rb[k].imag());
    t.qc = make_double2(q[k].real(), q[k].imag());
  }
  const cd ig = 1.0 / gamma, id = 1.0 / den;
  t.beta = make_double2(beta.real(), beta.imag());
  t.inv_gamma = make_double2(ig.real(), ig.imag());
  t.inv_den = make_double2(id.real(), id.imag());
}

static long largest_pow2_divisor(long v, long cap) {
  long p = 1;
  while (p < cap && v % (p * 2) == 0) p *= 2;
  return p;
}


// Per-axis table cache: rebuilt and uploaded only when (n, bc, cp, c2)
// change, so a run of identical steps issues no host transfers.
struct CnCacheEntry {
  bool valid;
  long n;
  int bc, nseg;
  cd cp, c2;
  FastTables ft;
};
static CnCacheEntry g_cn_cache[3];
static void *g_cn_tab_base = nullptr;

static double2 *fast_tables(int slot, long n, int bc, cd cp, cd c2, int nseg, cudaStream_t st, CnAxis *a) {
  const long nmax = 4096;
  if (n > nmax) {
    gb__set_error(1013, "cn: line length above 4096");
    return nullptr;
  }
  const long per = 6 * nmax + 2 * 5 * 32;
  double2 *base = (double2 *) gb__scratch(GB_SCR_CN, sizeof(double2) * (size_t) per * 3);
  if (!base) return nullptr;
  if (base != g_cn_tab_base) {
    for (int i = 0; i < 3; i++) g_cn_cache[i].valid = false;
    g_cn_tab_base = base;
  }
  double2 *tab = base + (size_t) per * slot;
  CnCacheEntry &e = g_cn_cache[slot];
  if (!(e.valid && e.n == n && e.bc == bc && e.nseg == nseg && e.cp == cp && e.c2 == c2)) {
    build_fast_tables(n, bc, cp, c2, nseg, e.ft);
    if (cudaMemcpyAsync(tab, e.ft.tab.data(), sizeof(double2) * e.ft.tab.size(), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      gb__set_error(3, "cn tables h2d");
      return nullptr;
    }
    e.valid = true;
    e.n = n;
    e.bc = bc;
    e.nseg = nseg;
    e.cp = cp;
    e.c2 = c2;
  }
  a->beta = e.ft.beta;
  a->gamma = e.ft.inv_gamma;
  a->den = e.ft.inv_den;
  a->klo = e.ft.klo;
  a->khi = e.ft.khi;
  a->mc = e.ft.mc;
  a->rbc = e.ft.rbc;
  a->qc = e.ft.qc;
  return tab;
}

// Persistent launch of the warp-cooperative kernel: one resident wave of
// CTAs, each walking the tiles with a stride of the grid.
template <int SMAX> static void *warp_kernel(bool contig) {
  return contig ? (void *) k_cn_warp<true, SMAX> : (void *) k_cn_warp<false, SMAX>;
}

static int launch_cn_warp(void *psi, CnAxis &a, bool contig, int axis, cudaStream_t st) {
  const long pitch = warp_pitch(contig, a.n);
  const long tl = contig ? tile_lines<true>() : tile_lines<false>();
  const size_t sm = 2 * sizeof(double2) * (size_t) (contig ? tl * pitch : a.n * pitch);
  long ntiles, tpo = 1;
  if (contig) {
    ntiles = (a.outer + tl - 1) / tl;
  } else {
    tpo = (a.inner + tl - 1) / tl;
    ntiles = a.outer * tpo;
  }
  // segment length bound: the register arrays hold ceil(n / 32) <= SMAX points
  const int smax = a.n <= 64 ? 2 : a.n <= 128 ? 4 : a.n <= 192 ? 6 : 8;
  const int si = smax / 2 - 1;
  if (ntiles <= 0) return 0;
  // resident CTAs for this (device, kernel, tile size), remembered per kernel
  struct Occ {
    int dev;
    size_t sm;
    int rg;
  };
  static Occ occ[2][4] = {};
  static bool occ_init = false;
  if (!occ_init) {
    for (auto &r : occ)
      for (auto &e : r) e.dev = -1;
    occ_init = true;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  void *kern = si == 0 ? warp_kernel<2>(contig) : si == 1 ? warp_kernel<4>(contig) : si == 2 ? warp_kernel<6>(contig)
                                                                                  : warp_kernel<8>(contig);
  Occ &o = occ[contig ? 1 : 0][si];
  if (o.dev != dev || o.sm != sm) {
    // the attribute covers the largest tile (lines of 32 * kLaneSegMax points)
    const size_t sm_max = 2 * sizeof(double2) * (size_t) (contig ? tl * contig_row(32 * kLaneSegMax)
                                                               : 32 * kLaneSegMax * warp_pitch(false, 0));
    int nsm = 0, per = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm_max);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kCnWarpThreads, sm);
    cudaGetLastError();
    o.dev = dev;
    o.sm = sm;
    o.rg = (nsm > 0 && per > 0) ? nsm * per : -1;
  }
  const int rg = o.rg;
  if (rg < 0) return gb__set_error(1014, "cn: warp kernel does not fit");
  const long grid = ntiles < rg ? ntiles : rg;
  const int slot = gb__pass_begin(15 + axis);
  void *args[] = {&psi, &a, &ntiles, &tpo};
  const cudaError_t e = cudaLaunchKernel(kern, dim3((unsigned) grid), dim3(kCnWarpThreads), args, sm, st);
  if (e != cudaSuccess) {
    gb__pass_end(slot);
    gb__count_launch();
    return gb__set_error((int) e, "cn warp");
  }
  gb__pass_end(slot);
  GB_CHECK_LAUNCH("cn warp");
  return 0;
}

}  // namespace

// Warp-cooperative line solver on (1) or off (0, the default: the
// segment-per-warp kernel, measured faster on B200 at 192^3: 0.447 against
// 0.487 ms per step); -1 only queries.
// The fast kernel unrolled for the segment length of lines of n points.
using FastKernel = void (*)(double2 *, CnAxis);
template <bool CONTIG> static FastKernel fast_kernel(long n) {
  const long S = (n + kSeg - 1) / kSeg;
  if (S <= 4) return k_cn_fast<CONTIG, 4>;
  if (S <= 8) return k_cn_fast<CONTIG, 8>;
  if (S <= 12) return k_cn_fast<CONTIG, 12>;
  if (S <= 16) return k_cn_fast<CONTIG, 16>;
  return k_cn_fast<CONTIG, 0>;
}

static int g_cn_warp_on = 0;
extern "C" int gb_cn_warp_solver(int on) {
  const int old = g_cn_warp_on;
  if (on >= 0) g_cn_warp_on = on ? 1 : 0;
  return old;
}

extern "C" int gb_cn_step(void *psi, const gb_geom *g, const gb_cn_params *p, const gb_potential *pre,
                          const gb_potential *post) {
  if (g->prec != GB_FP64) return gb__set_error(1010, "cn: FP64 storage required");
  int *err_flag = gb__status(GB_STATUS_CN);
  if (!err_flag) return gb_last_error();
  cudaStream_t st = gb__stream();
  const cd c = cd(0.0, 4.0) * p->mass * g->step * g->step / 1.0;  // 4 i m h^2 / hbar (hbar = 1)
  const cd tstep(p->tstep_re, p->tstep_im);
  const bool fast = (p->omega == 0.0) && !p->absorb;
  const long nxyz = g->nx * g->ny * g->nz;
  gb_potential none;
  memset(&none, 0, sizeof(none));
  const gb_potential *prep = pre ? pre : &none, *postp = post ? post : &none;

  // which axes run (reference skips axes of length 1); the first running
  // axis takes the pre potential, the last the post potential
  int axes[3], na = 0;
  if (g->nx != 1) axes[na++] = 0;
  if (g->ny != 1) axes[na++] = 1;
  if (g->nz != 1) axes[na++] = 2;
  if (na == 0) {
    if (prep->kind != GB_POT_NONE || prep->g != 0.0) GB_TRYC(gb_potential_multiply(psi, g, prep));
    if (postp->kind != GB_POT_NONE || postp->g != 0.0) GB_TRYC(gb_potential_multiply(psi, g, postp));
    return 0;
  }

  for (int s = 0; s < na; s++) {
    const int axis = axes[s];
    CnAxis a;
    memset(&a, 0, sizeof(a));
    a.nx = g->nx;
    a.ny = g->ny;
    a.nz = g->nz;
    a.axis = axis;
    a.boundary = p->boundary;
    a.step = g->step;
    a.err = err_flag;
    a.c = make_double2(c.real(), c.imag());
    a.tstep = make_double2(p->tstep_re, p->tstep_im);
    const double k0 = axis == 0 ? p->kx0 : (axis == 1 ? p->ky0 : p->kz0);
    const cd c2 = cd(0.0, -1.0) * g->step * k0;
    cd c3 = 0.0;
    if (axis == 0) c3 = p->mass * p->omega * cd(0.0, 1.0) * g->step / 1.0;
    if (axis == 1) c3 = -p->mass * p->omega * cd(0.0, 1.0) * g->step / 1.0;
    a.c2 = make_double2(c2.real(), c2.imag());
    a.c3 = make_double2(c3.real(), c3.imag());
    a.coord_off = axis == 0 ? p->y0 : p->x0;
    a.absorb = p->absorb;
    a.lx = p->lx;
    a.hx = p->hx;
    a.ly = p->ly;
    a.hy = p->hy;
    a.lz = p->lz;
    a.hz = p->hz;
    if (axis == 2) {
      a.n = g->nz;
      a.inner = 1;
      a.outer = g->nx * g->ny;
    } else if (axis == 1) {
      a.n = g->ny;
      a.inner = g->nz;
      a.outer = g->nx;
    } else {
      a.n = g->nx;
      a.inner = g->ny * g->nz;
      a.outer = 1;
    }
    // the contiguous kernel also covers axes whose inner extent is 1
    const bool contig = (a.inner == 1);
    if (contig) a.outer = nxyz / a.n;
    a.nlines = nxyz / a.n;
    const gb_potential none_pot = none;
    a.pre = (s == 0) ? *prep : none_pot;
    a.post = (s == na - 1) ? *postp : none_pot;

    if (fast && a.n <= 32 * kLaneSegMax && g_cn_warp_on) {
      const cd cp = c / tstep;
      double2 *tab = fast_tables(s, a.n, p->boundary, cp, c2, 32, st, &a);
      if (!tab) return gb_last_error();
      a.tab = tab;
      a.cp = make_double2(cp.real(), cp.imag());
      GB_TRYC(launch_cn_warp(psi, a, contig, axis, st));
    } else if (fast) {
      const cd cp = c / tstep;
      double2 *tab = fast_tables(s, a.n, p->boundary, cp, c2, kSeg, st, &a);
      if (!tab) return gb_last_error();
      a.tab = tab;
      a.cp = make_double2(cp.real(), cp.imag());
      // tile budget: two CTAs per SM, each with its tile, its static
      // shared memory and the per-CTA reservation
      static size_t budget = 0;
      if (!budget) {
        int dev = 0, smpm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&smpm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaFuncAttributes fa0, fa1;
        cudaFuncGetAttributes(&fa0, k_cn_fast<true, 0>);
        cudaFuncGetAttributes(&fa1, k_cn_fast<false, 0>);
        const size_t st_max = fa0.sharedSizeBytes > fa1.sharedSizeBytes ? fa0.sharedSizeBytes : fa1.sharedSizeBytes;
        const long b = (long) smpm / 2 - 1024 - (long) st_max;
        budget = b > 16 * 1024 ? (size_t) b : 16 * 1024;
      }
      if (contig) {
        const long row = contig_row(a.n);
        long lpc = (long) (budget / (row * 16));
        if (lpc > 32) lpc = 32;
        if (lpc < 1) return gb__set_error(1011, "cn: line too long for a shared-memory tile");
        a.lpc = (int) lpc;
        const size_t sm = (size_t) lpc * row * 16;
        const FastKernel kern = fast_kernel<true>(a.n);
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
        const long nb = (a.outer + lpc - 1) / lpc;
        {
          const int slot = gb__pass_begin(15 + axis);
          kern<<<(unsigned) nb, 32 * kSeg, sm, st>>>((double2 *) psi, a);
          gb__pass_end(slot);
        }
      } else {
        long cap = (long) (budget / (a.n * 16));
        if (cap > 32) cap = 32;
        if (cap < 1) return gb__set_error(1011, "cn: line too long for a shared-memory tile");
        const long lpc = largest_pow2_divisor(a.inner, cap);
        a.lpc = (int) lpc;
        const size_t sm = (size_t) lpc * a.n * 16;
        const FastKernel kern = fast_kernel<false>(a.n);
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
        if (a.outer > 65535) return gb__set_error(1012, "cn: outer extent above 65535");
        dim3 grid((unsigned) (a.inner / lpc), (unsigned) a.outer);
        {
          const int slot = gb__pass_begin(15 + axis);
          kern<<<grid, 32 * kSeg, sm, st>>>((double2 *) psi, a);
          gb__pass_end(slot);
        }
      }
      GB_CHECK_LAUNCH("cn fast");
    } else {
      if (a.pre.kind != GB_POT_NONE || a.pre.g != 0.0) GB_TRYC(gb_potential_multiply(psi, g, &a.pre));
      double2 *work = (double2 *) gb__scratch(GB_SCR_WORK, sizeof(double2) * (size_t) nxyz * 4);
      if (!work) return gb_last_error();
      a.work = work;
      if (!contig) a.inner = a.inner;  // strided addressing in the kernel
      const long nb = (a.nlines + 127) / 128;
      {
        const int slot = gb__pass_begin(15 + axis);
        k_cn_general<<<(unsigned) nb, 128, 0, st>>>((double2 *) psi, a);
        gb__pass_end(slot);
      }
      GB_CHECK_LAUNCH("cn general");
      if (a.post.kind != GB_POT_NONE || a.post.g != 0.0) GB_TRYC(gb_potential_multiply(psi, g, &a.post));
    }
  }
  return 0;
}

// Status word written by the bounded copy waits that gave up (0 = none).
extern "C" int gb_cn_error_flag(void) { return gb__status_word(GB_STATUS_CN, 0); }
