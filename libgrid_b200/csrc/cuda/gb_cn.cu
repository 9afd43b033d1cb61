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

// psi * exp(c (cons + V + g |psi|^2)) (src/grid_wf.c:586-598)
__device__ __forceinline__ double2 cn_pot(double2 x, long ix, long iy, long iz, const CnAxis &a, const gb_potential &pt) {
  double wr = pt.cons, wi = 0.0;
  const long vidx = (ix * a.ny + iy) * pt.vrow + iz;
  if (pt.kind == GB_POT_COMPLEX) {
    const double2 v = ((const double2 *) pt.v)[vidx];
    wr += v.x;
    wi += v.y;
  } else if (pt.kind == GB_POT_REAL) {
    wr += ((const double *) pt.v)[vidx];
  }
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

// Fast path.  A CTA of 8 warps owns up to 32 lines (lane = line); warp s
// owns segment s = [s S, (s+1) S) of every line, S = ceil(n / 8).  Both
// Thomas recurrences are linear with line-independent coefficients:
//   forward  v_i = b_i - m_i v_{i-1}
//   backward x_i = rb_i v_i + Q_i x_{i+1},   Q_i = -rb_i c_i
// so each warp runs the particular recurrence of its segment from a zero
// carry-in, one warp chains the 8 segment carries per line, and every
// element then adds (carry-in) x (homogeneous response), whose tables
// H_i = prod(-m_j) and G_i = prod(Q_j) over the segment are precomputed.
template <bool CONTIG> __global__ void __launch_bounds__(32 * kSeg, 2) k_cn_fast(double2 *__restrict__ psi, CnAxis a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ double2 s_end[kSeg][32];
  __shared__ double2 s_in[kSeg][32];
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
  if (a.pre.kind != GB_POT_NONE || a.pre.g != 0.0) {
    for (long e = tid; e < (long) nl * n; e += 32 * kSeg) {
      long l, i;
      if constexpr (CONTIG) {
        l = e / n;
        i = e - l * n;
      } else {
        i = e / nl;
        l = e - i * nl;
      }
      long ix, iy, iz;
      cn_decode(a, CONTIG ? line0 + l : o, i, col0 + l, ix, iy, iz);
      double2 &r = tile_at<CONTIG>(sm, (int) l, i, row);
      r = cn_pot(r, ix, iy, iz, a, a.pre);
    }
  }
  __syncthreads();

  const double2 *tm = a.tab, *trb = a.tab + n, *tz = a.tab + 2 * n, *tH = a.tab + 3 * n, *tQ = a.tab + 4 * n,
                *tG = a.tab + 5 * n;
  const long S = (n + kSeg - 1) / kSeg;
  const long a0 = seg * S, e0 = (a0 + S < n) ? a0 + S : n;
  const bool active = (lane < nl) && (a0 < e0);
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
    for (long i = a0; i < e0; i++) {
      const double2 pp = (i + 1 < e0) ? tile_at<CONTIG>(sm, lane, i + 1, row) : p_after;
      const double2 b = cn_rhs(i, n, bc, a.cp, a.c2, zero, pm, p0, pp, pfirst, plast);
      u = (i == a0) ? b : cs(b, cm(tm[i], u));
      tile_at<CONTIG>(sm, lane, i, row) = u;
      pm = p0;
      p0 = pp;
    }
  }
  if (lane < nl) s_end[seg][lane] = u;
  __syncthreads();
  if (seg == 0 && lane < nl) {
    double2 vin = zero;
    for (int s = 0; s < kSeg; s++) {
      const long as = s * S, es = (as + S < n) ? as + S : n;
      s_in[s][lane] = vin;
      if (as < es) vin = ca(s_end[s][lane], cm(tH[es - 1], vin));
    }
  }
  __syncthreads();

  // ---- forward fix-up fused with the backward particular recurrence
  double2 y = zero;
  if (active) {
    const double2 vin = s_in[seg][lane];
    for (long i = e0 - 1; i >= a0; i--) {
      const double2 v = ca(tile_at<CONTIG>(sm, lane, i, row), cm(tH[i], vin));
      y = (i == e0 - 1) ? cm(trb[i], v) : ca(cm(trb[i], v), cm(tQ[i], y));
      tile_at<CONTIG>(sm, lane, i, row) = y;
    }
  }
  if (lane < nl) s_end[seg][lane] = y;
  __syncthreads();
  if (seg == 0 && lane < nl) {
    double2 xin = zero;
    for (int s = kSeg - 1; s >= 0; s--) {
      const long as = s * S, es = (as + S < n) ? as + S : n;
      s_in[s][lane] = xin;
      if (as < es) xin = ca(s_end[s][lane], cm(tG[as], xin));
    }
    if (bc == 3) {
      // Sherman-Morrison: fact = (x_0 + beta x_{n-1} / gamma) / den; the
      // segment holding n-1 has a zero carry-in, so x_{n-1} = y_{n-1}.
      const double2 xl = tile_at<CONTIG>(sm, lane, n - 1, row);
      s_fact[lane] = cm(ca(xin, cm(a.beta, cm(xl, a.gamma))), a.den);  // gamma, den hold reciprocals
    }
  }
  __syncthreads();

  // ---- backward fix-up, periodic correction, second potential half-step
  const bool post = (a.post.kind != GB_POT_NONE || a.post.g != 0.0);
  if (active) {
    const double2 xin = s_in[seg][lane];
    const double2 fact = (bc == 3) ? s_fact[lane] : zero;
    for (long i = a0; i < e0; i++) {
      double2 x = ca(tile_at<CONTIG>(sm, lane, i, row), cm(tG[i], xin));
      if (bc == 3) x = cs(x, cm(fact, tz[i]));
      if (post) {
        long ix, iy, iz;
        cn_decode(a, CONTIG ? line0 + lane : o, i, col0 + lane, ix, iy, iz);
        x = cn_pot(x, ix, iy, iz, a, a.post);
      }
      tile_at<CONTIG>(sm, lane, i, row) = x;
    }
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
  bulk_wait_all();
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
  std::vector<double2> tab;  // 6 n: m, rb, z, H, Q, G
  double2 beta, inv_gamma, inv_den;
};

static void build_fast_tables(long n, int bc, cd cp, cd c2, FastTables &t) {
  t.tab.assign(6 * n, make_double2(0.0, 0.0));
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
  const long S = (n + kSeg - 1) / kSeg;
  for (long s = 0; s < kSeg; s++) {
    const long as = s * S, es = (as + S < n) ? as + S : n;
    for (long i = as; i < es; i++) H[i] = (i == as) ? -m[i] : H[i - 1] * (-m[i]);
    for (long i = es - 1; i >= as; i--) G[i] = (i == es - 1) ? q[i] : q[i] * G[i + 1];
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
  int bc;
  cd cp, c2;
  FastTables ft;
};
static CnCacheEntry g_cn_cache[3];
static void *g_cn_tab_base = nullptr;

static double2 *fast_tables(int slot, long n, int bc, cd cp, cd c2, cudaStream_t st, CnAxis *a) {
  const long nmax = 4096;
  if (n > nmax) {
    gb__set_error(1013, "cn: line length above 4096");
    return nullptr;
  }
  double2 *base = (double2 *) gb__scratch(GB_SCR_CN, sizeof(double2) * (size_t) (6 * nmax) * 3);
  if (!base) return nullptr;
  if (base != g_cn_tab_base) {
    for (int i = 0; i < 3; i++) g_cn_cache[i].valid = false;
    g_cn_tab_base = base;
  }
  double2 *tab = base + (size_t) (6 * nmax) * slot;
  CnCacheEntry &e = g_cn_cache[slot];
  if (!(e.valid && e.n == n && e.bc == bc && e.cp == cp && e.c2 == c2)) {
    build_fast_tables(n, bc, cp, c2, e.ft);
    if (cudaMemcpyAsync(tab, e.ft.tab.data(), sizeof(double2) * (size_t) (6 * n), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      gb__set_error(3, "cn tables h2d");
      return nullptr;
    }
    e.valid = true;
    e.n = n;
    e.bc = bc;
    e.cp = cp;
    e.c2 = c2;
  }
  a->beta = e.ft.beta;
  a->gamma = e.ft.inv_gamma;
  a->den = e.ft.inv_den;
  return tab;
}

}  // namespace

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

    if (fast) {
      const cd cp = c / tstep;
      double2 *tab = fast_tables(s, a.n, p->boundary, cp, c2, st, &a);
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
        cudaFuncGetAttributes(&fa0, k_cn_fast<true>);
        cudaFuncGetAttributes(&fa1, k_cn_fast<false>);
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
        cudaFuncSetAttribute(k_cn_fast<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
        const long nb = (a.outer + lpc - 1) / lpc;
        {
          const int slot = gb__pass_begin(15 + axis);
          k_cn_fast<true><<<(unsigned) nb, 32 * kSeg, sm, st>>>((double2 *) psi, a);
          gb__pass_end(slot);
        }
      } else {
        long cap = (long) (budget / (a.n * 16));
        if (cap > 32) cap = 32;
        if (cap < 1) return gb__set_error(1011, "cn: line too long for a shared-memory tile");
        const long lpc = largest_pow2_divisor(a.inner, cap);
        a.lpc = (int) lpc;
        const size_t sm = (size_t) lpc * a.n * 16;
        cudaFuncSetAttribute(k_cn_fast<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
        if (a.outer > 65535) return gb__set_error(1012, "cn: outer extent above 65535");
        dim3 grid((unsigned) (a.inner / lpc), (unsigned) a.outer);
        {
          const int slot = gb__pass_begin(15 + axis);
          k_cn_fast<false><<<grid, 32 * kSeg, sm, st>>>((double2 *) psi, a);
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
