// Line-pass FFT engine for the libgrid-b200 split-operator path (sm_100a).
//
// A 3-D grid (nx, ny, nz), z fastest, is viewed per axis as [outer][N][inner]:
//   z: outer = nx*ny, inner = 1      (contiguous lines)
//   y: outer = nx,    inner = nz
//   x: outer = 1,     inner = ny*nz
// One "pass" reads each element of the grid once from HBM, applies a short
// program of line operations (forward/inverse FFT along the axis, kinetic
// factor, potential factor, scale, k^2 reduction) and writes it once.
//
// Each line of N points is transformed by TL = N/P threads.  Thread t always
// holds the P elements at positions t + TL*m (m < P) in registers, both on
// entry and on exit of the transform, so the first radix stage loads straight
// from HBM and the last stage stores straight to HBM with unit stride across
// threads; only the exchanges between radix stages go through shared memory.
// Stages follow the Stockham autosort scheme: with Ns the product of the
// previous radices, butterfly j (k = j mod Ns) takes x[j + r N/R], applies
// exp(s 2 pi i k r / (Ns R)), does a radix-R DFT and writes
// (j - k) R + k + r Ns.  Strided passes interleave BZ adjacent columns in
// shared memory (column index fastest, conflict-free); contiguous passes pad
// one element every R0 so the stride-R0 writes of the first stage are
// conflict-free.
#pragma once

#include <cuda.h>

#include "gb_common.cuh"

// Tensor maps for the pipelined strided passes and their error flag
// (gb_runtime.cu).
int gb__tmap_lines(CUtensorMap *out, const void *base, long outer, long n, long inner, int fp32, int bz, int rows);

namespace gbfft {

// OP_POT_RP is the potential op for one case only, a real V_ext in real
// time without an absorbing region (a pure phase), so a kernel built for it
// carries none of the other potential paths.
enum : int { OP_END = 0, OP_FWD = 1, OP_INV = 2, OP_KIN = 3, OP_POT = 4, OP_SCALE = 5, OP_KSQ = 6, OP_POT_RP = 7 };

template <int... Ops> struct OpL {};
template <int... Rs> struct IL {};

// cos(pi/8), sin(pi/8), sqrt(1/2)
constexpr double kC1 = 0.92387953251128675613;
constexpr double kS1 = 0.38268343236508977173;
constexpr double kSQH = 0.70710678118654752440;

// o * (wr + S i wi)
template <int S, typename T2> __device__ __forceinline__ T2 wmul(T2 o, double wr, double wi) {
  using T = decltype(o.x);
  const T r = (T) wr, i = (T) (S * wi);
  return T2{o.x * r - o.y * i, o.x * i + o.y * r};
}

template <int R, int S, typename T2> struct DFT;
template <int S, typename T2> struct DFT<2, S, T2> {
  static __device__ __forceinline__ void run(T2 *v) {
    T2 a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  }
};
template <int S, typename T2> struct DFT<4, S, T2> {
  static __device__ __forceinline__ void run(T2 *v) {
    T2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    T2 a2 = cadd(v[1], v[3]), a3 = mul_si<S>(csub(v[1], v[3]));
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3);
    v[3] = csub(a1, a3);
  }
};
template <int S, typename T2> struct DFT<8, S, T2> {
  static __device__ __forceinline__ void run(T2 *v) {
    T2 e[4] = {v[0], v[2], v[4], v[6]};
    T2 o[4] = {v[1], v[3], v[5], v[7]};
    DFT<4, S, T2>::run(e);
    DFT<4, S, T2>::run(o);
    o[1] = wmul<S>(o[1], kSQH, kSQH);
    o[2] = mul_si<S>(o[2]);
    o[3] = wmul<S>(o[3], -kSQH, kSQH);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      v[k] = cadd(e[k], o[k]);
      v[k + 4] = csub(e[k], o[k]);
    }
  }
};
// Radix-4 butterfly on four elements of v given by index (in place).
template <int S, typename T2> __device__ __forceinline__ void bfly4(T2 &x0, T2 &x1, T2 &x2, T2 &x3) {
  const T2 a0 = cadd(x0, x2), a1 = csub(x0, x2);
  const T2 a2 = cadd(x1, x3), a3 = mul_si<S>(csub(x1, x3));
  x0 = cadd(a0, a2);
  x2 = csub(a0, a2);
  x1 = cadd(a1, a3);
  x3 = csub(a1, a3);
}

// 16-point DFT as 4 x 4: with input index 4a + b and output index k1 + 4 k2,
//   X[k1 + 4 k2] = sum_b W16^{b k1} W4^{b k2} sum_a x[4a + b] W4^{a k1}.
// Both butterfly layers work in place; the final index transpose is a
// compile-time renaming of registers.
template <int S, typename T2> struct DFT<16, S, T2> {
  static __device__ __forceinline__ void run(T2 *v) {
#pragma unroll
    for (int b = 0; b < 4; b++) bfly4<S>(v[b], v[b + 4], v[b + 8], v[b + 12]);
    // v[b + 4 k1] now holds Y[b][k1]; twiddle by W16^{b k1}
    v[1 + 4] = wmul<S>(v[1 + 4], kC1, kS1);    // b=1,k1=1: W^1
    v[1 + 8] = wmul<S>(v[1 + 8], kSQH, kSQH);  // b=1,k1=2: W^2
    v[1 + 12] = wmul<S>(v[1 + 12], kS1, kC1);  // b=1,k1=3: W^3
    v[2 + 4] = wmul<S>(v[2 + 4], kSQH, kSQH);  // b=2,k1=1: W^2
    v[2 + 8] = mul_si<S>(v[2 + 8]);            // b=2,k1=2: W^4
    v[2 + 12] = wmul<S>(v[2 + 12], -kSQH, kSQH);  // b=2,k1=3: W^6
    v[3 + 4] = wmul<S>(v[3 + 4], kS1, kC1);    // b=3,k1=1: W^3
    v[3 + 8] = wmul<S>(v[3 + 8], -kSQH, kSQH);  // b=3,k1=2: W^6
    v[3 + 12] = wmul<S>(v[3 + 12], -kC1, -kS1);  // b=3,k1=3: W^9
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) bfly4<S>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // v[4 k1 + k2] holds X[k1 + 4 k2]; transpose the 4 x 4 index
    T2 t;
    t = v[1]; v[1] = v[4]; v[4] = t;
    t = v[2]; v[2] = v[8]; v[8] = t;
    t = v[3]; v[3] = v[12]; v[12] = t;
    t = v[6]; v[6] = v[9]; v[9] = t;
    t = v[7]; v[7] = v[13]; v[13] = t;
    t = v[11]; v[11] = v[14]; v[14] = t;
  }
};

// Radix schedule per line length: P = registers (elements) per thread.
template <int N> struct Sched;
template <> struct Sched<2> { static constexpr int P = 2; using R = IL<2>; };
template <> struct Sched<4> { static constexpr int P = 4; using R = IL<4>; };
template <> struct Sched<8> { static constexpr int P = 8; using R = IL<8>; };
template <> struct Sched<16> { static constexpr int P = 16; using R = IL<16>; };
template <> struct Sched<32> { static constexpr int P = 8; using R = IL<8, 4>; };
template <> struct Sched<64> { static constexpr int P = 8; using R = IL<8, 8>; };
template <> struct Sched<128> { static constexpr int P = 16; using R = IL<16, 8>; };
template <> struct Sched<256> { static constexpr int P = 16; using R = IL<16, 16>; };
template <> struct Sched<512> { static constexpr int P = 16; using R = IL<16, 16, 2>; };
template <> struct Sched<1024> { static constexpr int P = 16; using R = IL<16, 16, 4>; };
template <> struct Sched<2048> { static constexpr int P = 16; using R = IL<16, 16, 8>; };
template <> struct Sched<4096> { static constexpr int P = 16; using R = IL<16, 16, 16>; };

template <int R0, int... Rest> __host__ __device__ constexpr int first_radix(IL<R0, Rest...>) { return R0; }

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v / 2); }

// Shared-memory views.  sync() orders the exchange between radix stages
// among the threads that share a line: strided tiles interleave their lines
// across the whole CTA; a contiguous line of TL threads lives inside one
// warp when TL <= 32 (warp barrier), else in TL / 32 consecutive warps
// (named barrier 1 + line, as id 0 is the CTA barrier).
template <typename T2, int BZ> struct SmStrided {
  T2 *p;
  __device__ __forceinline__ T2 &operator()(int pos) const { return p[pos * BZ]; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};
template <typename T2, int SH, int TL> struct SmContig {
  T2 *p;
  __device__ __forceinline__ T2 &operator()(int pos) const { return p[pos + (pos >> SH)]; }
  __device__ __forceinline__ void sync() const {
    if constexpr (TL <= 32) {
      __syncwarp();
    } else {
      static_assert(TL % 32 == 0 && 256 / TL <= 15, "named barriers per line");
      asm volatile("bar.sync %0, %1;" ::"r"(1 + (int) (threadIdx.x / TL)), "r"(TL) : "memory");
    }
  }
};

// One Stockham stage; v holds positions t + TL*m on entry and exit.
template <typename T2, int S, int N, int P, int NS, int R, bool FIRST, bool LAST, class SM>
__device__ __forceinline__ void fft_stage(T2 (&v)[P], int t, const SM &sm, const T2 *__restrict__ tw) {
  constexpr int TL = N / P;
  constexpr int B = P / R;
#pragma unroll
  for (int u = 0; u < B; u++) {
    const int j = t + u * TL;
    const int k = j & (NS - 1);
    T2 w[R];
#pragma unroll
    for (int r = 0; r < R; r++) w[r] = v[u + r * B];
    if constexpr (!FIRST && R == 16) {
      // w^(k r) with r = 4a + b is w^(4 k a) w^(k b): six table values
      // (b, a = 1..3) instead of fifteen keep the register footprint of the
      // stage small; each product is applied as two multiplications
      constexpr int STRIDE = N / (NS * R);
      T2 tb[4], ta[4];
#pragma unroll
      for (int e = 1; e < 4; e++) {
        tb[e] = tw[k * e * STRIDE];
        ta[e] = tw[k * 4 * e * STRIDE];
        if constexpr (S > 0) {
          tb[e].y = -tb[e].y;
          ta[e].y = -ta[e].y;
        }
      }
#pragma unroll
      for (int r = 1; r < R; r++) {
        const int a4 = r >> 2, b4 = r & 3;
        if (b4) w[r] = cmul(w[r], tb[b4]);
        if (a4) w[r] = cmul(w[r], ta[a4]);
      }
    } else if constexpr (!FIRST) {
      constexpr int STRIDE = N / (NS * R);
#pragma unroll
      for (int r = 1; r < R; r++) {
        T2 tt = tw[k * r * STRIDE];
        if constexpr (S > 0) tt.y = -tt.y;
        w[r] = cmul(w[r], tt);
      }
    }
    DFT<R, S, T2>::run(w);
    if constexpr (LAST) {
#pragma unroll
      for (int r = 0; r < R; r++) v[u + r * B] = w[r];
    } else {
      const int base = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; r++) sm(base + r * NS) = w[r];
    }
  }
  if constexpr (!LAST) {
    sm.sync();
#pragma unroll
    for (int m = 0; m < P; m++) v[m] = sm(t + TL * m);
    sm.sync();
  }
}

template <typename T2, int S, int N, int P, int NS, bool FIRST, class SM, int R0, int... Rest>
__device__ __forceinline__ void fft_run(T2 (&v)[P], int t, const SM &sm, const T2 *tw, IL<R0, Rest...>) {
  fft_stage<T2, S, N, P, NS, R0, FIRST, (sizeof...(Rest) == 0), SM>(v, t, sm, tw);
  if constexpr (sizeof...(Rest) > 0) fft_run<T2, S, N, P, NS * R0, false, SM>(v, t, sm, tw, IL<Rest...>{});
}

template <typename T2, int S, int N, class SM>
__device__ __forceinline__ void fft_line(T2 (&v)[Sched<N>::P], int t, const SM &sm, const T2 *tw) {
  fft_run<T2, S, N, Sched<N>::P, 1, true, SM>(v, t, sm, tw, typename Sched<N>::R{});
}

// Arguments shared by all pass kernels (plain data, passed by value).
struct PassArgs {
  long nx, ny, nz;
  int axis;             // 0 = x, 1 = y, 2 = z
  const void *tw;       // twiddle table exp(-2 pi i m / N), element type T2
  const void *kfac[3];  // per-axis kinetic factors exp(tm k_a^2) (T2)
  const double *ksq[3]; // per-axis k_a^2 (double), cutoff only
  double kmax2;
  int cutoff;
  double kscale;        // real scale folded into the kinetic factor
  double scale;         // OP_SCALE
  gb_potential pot;
  double *partial;      // OP_KSQ: one partial sum per block
  int *errflag;         // pipelined passes: set when a bounded wait gives up
};

// Decode (i, j, k) of axis position p for a line given by (o, q).  Grids
// handled by the passes hold fewer than 2^31 points (checked on the host),
// so 32-bit arithmetic suffices.
__device__ __forceinline__ void decode(const PassArgs &a, unsigned o, int p, unsigned q, int &i, int &j, int &k) {
  if (a.axis == 2) {
    i = (int) (o / (unsigned) a.ny);
    j = (int) (o - (unsigned) i * (unsigned) a.ny);
    k = p;
  } else if (a.axis == 1) {
    i = (int) o;
    j = p;
    k = (int) q;
  } else {
    i = p;
    j = (int) (q / (unsigned) a.nz);
    k = (int) (q - (unsigned) j * (unsigned) a.nz);
  }
}

__device__ __forceinline__ double absorb_ramp(long i, long j, long k, const gb_potential &pt) {
  // src/grid_wf.c:185-203
  double t = 0.0;
  if (i < pt.lx) t += (double) (pt.lx - i) / (double) pt.lx;
  else if (i > pt.hx) t += (double) (i - pt.hx) / (double) pt.lx;
  if (j < pt.ly) t += (double) (pt.ly - j) / (double) pt.ly;
  else if (j > pt.hy) t += (double) (j - pt.hy) / (double) pt.ly;
  if (k < pt.lz) t += (double) (pt.lz - k) / (double) pt.lz;
  else if (k > pt.hz) t += (double) (k - pt.hz) / (double) pt.lz;
  t *= 2.0 / 3.0;
  return t > 1.0 ? 1.0 : t;
}

// psi * exp(c (cons + V + g |psi|^2)) for one element (src/grid_wf.c:593-597).
// vidx is the element's index in the potential array.
template <typename T>
__device__ __forceinline__ C2<T> pot_factor_apply(C2<T> x, long i, long j, long k, unsigned vidx, const PassArgs &a) {
  const gb_potential &pt = a.pot;
  double wr = pt.cons, wi = 0.0;
  if (pt.kind == GB_POT_COMPLEX) {
    const C2<T> vv = ((const C2<T> *) pt.v)[vidx];
    wr += (double) vv.x;
    wi += (double) vv.y;
  } else if (pt.kind == GB_POT_REAL) {
    wr += (double) ((const T *) pt.v)[vidx];
  }
  if (pt.g != 0.0) wr += pt.g * ((double) x.x * (double) x.x + (double) x.y * (double) x.y);
  double cr = pt.c_re, ci = pt.c_im;
  if (pt.absorb) {
    const double am = absorb_ramp(i, j, k, pt);
    cr = -pt.treal * am;
    ci = -pt.treal * (1.0 - am);
  }
  const double ar = cr * wr - ci * wi;
  const double ai = cr * wi + ci * wr;
  return cmul(x, cexp_phase<T>(ar, ai, ar != 0.0));
}

// Potential factor on a register line when V is real or absent and there
// is no absorbing region: the exponent c (cons + V + g |psi|^2) is then
// purely imaginary when Re c = 0 (real time: a phase) or purely real when
// Im c = 0 (imaginary time: a decay), and only sincos or exp is needed.
// Same values as pot_factor_apply for these cases.
template <typename T, int P, int TL, bool HAS_V, bool PHASE>
__device__ __forceinline__ void pot_line_simple(C2<T> (&v)[P], int t, const T *vp, unsigned vt, unsigned vm,
                                                double cons, double g, double cc) {
#pragma unroll
  for (int m = 0; m < P; m++) {
    double w = cons;
    if constexpr (HAS_V) w += (double) vp[(unsigned) t * vt + (unsigned) m * vm];
    const double xr = (double) v[m].x, xi = (double) v[m].y;
    w = fma(g, fma(xr, xr, xi * xi), w);
    const double arg = cc * w;
    if constexpr (PHASE) {
      v[m] = cmul(v[m], cexp_phase<T>(0.0, arg, false));
    } else {
      const T f = (T) exp(arg);
      v[m] = C2<T>{v[m].x * f, v[m].y * f};
    }
  }
}

// Start of a line's potential row and its stride along the pass axis
// (potential arrays use the row length pot.vrow, e.g. the rgrid nz2).
__device__ __forceinline__ void pot_row(const PassArgs &a, unsigned o, unsigned q, int &i0, int &j0, int &k0,
                                        unsigned &vbase, unsigned &vstride) {
  decode(a, o, 0, q, i0, j0, k0);
  const unsigned vrow = (unsigned) a.pot.vrow, ny = (unsigned) a.ny;
  if (a.axis == 2) {
    vbase = ((unsigned) i0 * ny + (unsigned) j0) * vrow;
    vstride = 1u;
  } else if (a.axis == 1) {
    vbase = (unsigned) i0 * ny * vrow + (unsigned) k0;
    vstride = vrow;
  } else {
    vbase = (unsigned) j0 * vrow + (unsigned) k0;
    vstride = ny * vrow;
  }
}

__device__ __forceinline__ bool pot_is_simple(const gb_potential &pt) {
  return !pt.absorb && pt.kind != GB_POT_COMPLEX && (pt.c_re == 0.0 || pt.c_im == 0.0);
}

// Issue asynchronous copies (cp.async) of the real potential values this
// thread will need in the potential op into its own shared-memory slots
// stage[m * stride], m < P, so the load latency overlaps the tile load and
// the first transform.  Returns false (nothing issued) when the potential
// op will not read a real V through the simple path.
template <typename T, int P, int TL>
__device__ __forceinline__ bool pot_prefetch(const PassArgs &a, unsigned o, unsigned q, int t, T *stage,
                                             int stride) {
  if (a.pot.kind != GB_POT_REAL || !pot_is_simple(a.pot)) return false;
  int i0, j0, k0;
  unsigned vbase, vstride;
  pot_row(a, o, q, i0, j0, k0, vbase, vstride);
  const T *g = (const T *) a.pot.v + vbase;
#pragma unroll
  for (int m = 0; m < P; m++) cp_async_elem<sizeof(T)>(stage + m * stride, g + (unsigned) (t + TL * m) * vstride);
  cp_async_commit();
  return true;
}

template <int... Ops> __host__ __device__ constexpr bool has_pot(OpL<Ops...>) {
  return ((Ops == OP_POT || Ops == OP_POT_RP) || ...);
}
template <int... Ops> __host__ __device__ constexpr bool has_kin(OpL<Ops...>) { return ((Ops == OP_KIN) || ...); }

template <int Op, int... Rest> struct OpsHead {
  static constexpr int value = Op;
};

// Apply the program OpL<...> to a thread's register line.
template <typename T, int N, class SM, int... Ops> struct Program;

template <typename T, int N, class SM> struct Program<T, N, SM> {
  // o, q identify the line; thread holds positions t + TL*m
  static __device__ __forceinline__ void run(C2<T> (&)[Sched<N>::P], int, const SM &, const PassArgs &, unsigned,
                                             unsigned, double &, const void *, int) {}
};

template <typename T, int N, class SM, int Op, int... Rest> struct Program<T, N, SM, Op, Rest...> {
  // vstage: this thread's prefetched potential values in shared memory
  // (element m at vstage[m * vsstride]), or null to read the potential grid
  static __device__ __forceinline__ void run(C2<T> (&v)[Sched<N>::P], int t, const SM &sm, const PassArgs &a, unsigned o,
                                             unsigned q, double &acc, const void *vstage = nullptr, int vsstride = 0) {
    using T2 = C2<T>;
    constexpr int P = Sched<N>::P;
    constexpr int TL = N / P;
    const T2 *tw = (const T2 *) a.tw;
    if constexpr (Op == OP_FWD) {
      fft_line<T2, -1, N>(v, t, sm, tw);
    } else if constexpr (Op == OP_INV) {
      fft_line<T2, +1, N>(v, t, sm, tw);
    } else if constexpr (Op == OP_SCALE) {
      const T s = (T) a.scale;
#pragma unroll
      for (int m = 0; m < P; m++) v[m] = cscale(v[m], s);
    } else if constexpr (Op == OP_KIN) {
      // Line factor from the two other axes, times kscale; element factor
      // from the pass axis.
      int i, j, k;
      decode(a, o, 0, q, i, j, k);
      const int ax = a.axis;
      const int b0 = (ax == 0) ? 1 : 0, b1 = (ax == 2) ? 1 : 2;
      const int ix0 = (ax == 0) ? j : i, ix1 = (ax == 2) ? j : k;
      const T2 *fa = (const T2 *) a.kfac[ax];
      const T2 f0 = ((const T2 *) a.kfac[b0])[ix0];
      const T2 f1 = ((const T2 *) a.kfac[b1])[ix1];
      T2 lf = cmul(f0, f1);
      lf = cscale(lf, (T) a.kscale);
      double k2line = 0.0;
      if (a.cutoff) k2line = a.ksq[b0][ix0] + a.ksq[b1][ix1];
      if (a.cutoff) {
#pragma unroll
        for (int m = 0; m < P; m++) {
          const int p = t + TL * m;
          T2 f = cmul(lf, fa[p]);
          if (k2line + a.ksq[ax][p] >= a.kmax2) f = T2{(T) 0, (T) 0};
          v[m] = cmul(v[m], f);
        }
      } else {
#pragma unroll
        for (int m = 0; m < P; m++) v[m] = cmul(v[m], cmul(lf, fa[t + TL * m]));
      }
    } else if constexpr (Op == OP_POT) {
      // decode the line once; along the pass axis the potential index
      // advances by a fixed stride
      int i0, j0, k0;
      unsigned vbase, vstride;
      pot_row(a, o, q, i0, j0, k0, vbase, vstride);
      const gb_potential &pt = a.pot;
      if (pot_is_simple(pt)) {
        const bool phase = (pt.c_re == 0.0);
        const double cc = phase ? pt.c_im : pt.c_re;
        // V from this thread's prefetched slots when the kernel staged it,
        // else from the grid: element m of the thread sits at position
        // t + TL m of the line
        const T *vp = (const T *) pt.v + vbase;
        unsigned vt = vstride, vm = TL * vstride;
        if (vstage) {
          cp_async_wait_all();
          vp = (const T *) vstage;
          vt = 0;
          vm = (unsigned) vsstride;
        }
        if (pt.kind == GB_POT_REAL) {
          if (phase) pot_line_simple<T, P, TL, true, true>(v, t, vp, vt, vm, pt.cons, pt.g, cc);
          else pot_line_simple<T, P, TL, true, false>(v, t, vp, vt, vm, pt.cons, pt.g, cc);
        } else {
          if (phase) pot_line_simple<T, P, TL, false, true>(v, t, vp, vt, vm, pt.cons, pt.g, cc);
          else pot_line_simple<T, P, TL, false, false>(v, t, vp, vt, vm, pt.cons, pt.g, cc);
        }
      } else {
#pragma unroll
        for (int m = 0; m < P; m++) {
          const int p = t + TL * m;
          const int i = (a.axis == 0) ? p : i0, j = (a.axis == 1) ? p : j0, k = (a.axis == 2) ? p : k0;
          v[m] = pot_factor_apply<T>(v[m], i, j, k, vbase + (unsigned) p * vstride, a);
        }
      }
    } else if constexpr (Op == OP_POT_RP) {
      // real V_ext, real time, no absorber (the caller checked): the phase
      // loop of the simple path only
      int i0, j0, k0;
      unsigned vbase, vstride;
      pot_row(a, o, q, i0, j0, k0, vbase, vstride);
      const T *vp = (const T *) a.pot.v + vbase;
      unsigned vt = vstride, vm = TL * vstride;
      if (vstage) {
        cp_async_wait_all();
        vp = (const T *) vstage;
        vt = 0;
        vm = (unsigned) vsstride;
      }
      pot_line_simple<T, P, TL, true, true>(v, t, vp, vt, vm, a.pot.cons, a.pot.g, a.pot.c_im);
    } else if constexpr (Op == OP_KSQ) {
      // sum |k|^2 |v|^2 with k from the unshifted frequency grid
      int i, j, k;
      decode(a, o, 0, q, i, j, k);
      const int ax = a.axis;
      const int b0 = (ax == 0) ? 1 : 0, b1 = (ax == 2) ? 1 : 2;
      const int ix0 = (ax == 0) ? j : i, ix1 = (ax == 2) ? j : k;
      const double k2line = a.ksq[b0][ix0] + a.ksq[b1][ix1];
#pragma unroll
      for (int m = 0; m < P; m++) {
        const int p = t + TL * m;
        acc += (k2line + a.ksq[ax][p]) * ((double) v[m].x * (double) v[m].x + (double) v[m].y * (double) v[m].y);
      }
    }
    Program<T, N, SM, Rest...>::run(v, t, sm, a, o, q, acc, vstage, vsstride);
  }
};

template <int... Ops> __host__ __device__ constexpr bool has_ksq(OpL<Ops...>) { return ((Ops == OP_KSQ) || ...); }

// Deterministic block sum (fixed shuffle tree, fixed warp order).
template <int THREADS> __device__ __forceinline__ double block_sum(double v, double *sbuf) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  constexpr int NW = (THREADS + 31) / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sbuf[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
#pragma unroll 1
    for (int q = 0; q < NW; q++) r += sbuf[q];
  }
  return r;
}

// ---------------------------------------------------------------- kernels

// CTA shapes, by line length and element size ES = sizeof(real).  Small
// CTAs (128 threads; four resident per SM in FP64) let the load, transform
// and store phases of neighbouring CTAs interleave; FP32 strided passes keep
// 16 columns (256 threads) so each row segment stays 128 bytes.
// Resident CTAs per SM are bounded below by MINB (the register cap: 128
// per thread in FP64, 85 in FP32).
template <int THREADS, int ES> constexpr int pass_min_blocks() {
  return (ES == 8 ? 512 : 768) / THREADS > 0 ? (ES == 8 ? 512 : 768) / THREADS : 1;
}

template <int N, int ES = 8> struct ContigCfg {
  static constexpr int P = Sched<N>::P;
  static constexpr int TL = N / P;
  static constexpr int L = (128 / TL) > 0 ? (128 / TL) : 1;
  static constexpr int THREADS = TL * L;
  static constexpr int SH = ilog2c(first_radix(typename Sched<N>::R{}));
  static constexpr int LINE = N + (N >> SH);
  static constexpr int MINB = pass_min_blocks<THREADS, ES>();
};

// Contiguous lines (inner == 1): L lines of N per block.
template <typename T, int N, int... Ops>
__global__ void __launch_bounds__(ContigCfg<N, sizeof(T)>::THREADS, ContigCfg<N, sizeof(T)>::MINB)
    k_pass_contig(const C2<T> *__restrict__ src, C2<T> *__restrict__ dst, long nlines, PassArgs a) {
  using T2 = C2<T>;
  using Cfg = ContigCfg<N, sizeof(T)>;
  constexpr int P = Cfg::P, TL = Cfg::TL;
  extern __shared__ __align__(16) unsigned char smraw[];
  T2 *smem = (T2 *) smraw;
  const int t = threadIdx.x % TL;
  const int l = threadIdx.x / TL;
  const unsigned line = blockIdx.x * (unsigned) Cfg::L + (unsigned) l;
  const bool ok = line < (unsigned long) nlines;
  const T2 *s = src + (size_t) line * N;
  const T *vstage = nullptr;
  if constexpr (has_pot(OpL<Ops...>{})) {
    // potential values staged behind the exchange buffer
    T *stage = (T *) (smraw + (size_t) Cfg::L * Cfg::LINE * sizeof(T2)) + threadIdx.x;
    if (pot_prefetch<T, P, TL>(a, ok ? line : 0u, 0u, t, stage, Cfg::THREADS)) vstage = stage;
  }
  T2 v[P];
#pragma unroll
  for (int m = 0; m < P; m++) v[m] = ok ? s[t + TL * m] : T2{(T) 0, (T) 0};
  SmContig<T2, Cfg::SH, TL> sm{smem + l * Cfg::LINE};
  double acc = 0.0;
  Program<T, N, SmContig<T2, Cfg::SH, TL>, Ops...>::run(v, t, sm, a, ok ? line : 0u, 0u, acc, vstage,
                                                        Cfg::THREADS);
  if constexpr (has_ksq(OpL<Ops...>{})) {
    __shared__ double sbuf[(Cfg::THREADS + 31) / 32];
    double r = block_sum<Cfg::THREADS>(ok ? acc : 0.0, sbuf);
    if (threadIdx.x == 0) a.partial[blockIdx.x] = r;
  } else {
    if (ok) {
      T2 *d = dst + (size_t) line * N;
#pragma unroll
      for (int m = 0; m < P; m++) d[t + TL * m] = v[m];
    }
  }
}

template <int N, int ES = 8> struct StridedCfg {
  static constexpr int P = Sched<N>::P;
  static constexpr int TL = N / P;
  static constexpr int BZ = ES == 8 ? ((N <= 512) ? 8 : 4) : ((N <= 256) ? 16 : ((N <= 512) ? 8 : 4));
  static constexpr int THREADS = TL * BZ;
};

// Strided lines: block = (column block of BZ adjacent inner indices, outer).
template <typename T, int N, int BZ, int... Ops>
__global__ void __launch_bounds__((N / Sched<N>::P) * BZ, pass_min_blocks<(N / Sched<N>::P) * BZ, sizeof(T)>())
    k_pass_strided(const C2<T> *__restrict__ src, C2<T> *__restrict__ dst, long inner, PassArgs a) {
  using T2 = C2<T>;
  constexpr int P = Sched<N>::P, TL = N / P;
  constexpr int THREADS = TL * BZ;
  extern __shared__ __align__(16) unsigned char smraw[];
  T2 *smem = (T2 *) smraw;
  const int c = threadIdx.x % BZ;
  const int t = threadIdx.x / BZ;
  const unsigned o = blockIdx.y;
  const unsigned q = blockIdx.x * (unsigned) BZ + (unsigned) c;
  const unsigned in32 = (unsigned) inner;
  // element (line, t + TL m) sits at base + (t + TL m) * inner; the whole
  // grid has fewer than 2^31 points, so the in-tile offsets fit 32 bits
  const size_t off = (size_t) o * (size_t) N * (size_t) inner + q;
  const T2 *s = src + off;
  const T *vstage = nullptr;
  if constexpr (has_pot(OpL<Ops...>{})) {
    T *stage = (T *) (smraw + (size_t) N * BZ * sizeof(T2)) + threadIdx.x;
    if (pot_prefetch<T, P, TL>(a, o, q, t, stage, THREADS)) vstage = stage;
  }
  T2 v[P];
#pragma unroll
  for (int m = 0; m < P; m++) v[m] = s[(unsigned) (t + TL * m) * in32];
  SmStrided<T2, BZ> sm{smem + c};
  double acc = 0.0;
  Program<T, N, SmStrided<T2, BZ>, Ops...>::run(v, t, sm, a, o, q, acc, vstage, THREADS);
  if constexpr (has_ksq(OpL<Ops...>{})) {
    __shared__ double sbuf[(THREADS + 31) / 32];
    double r = block_sum<THREADS>(acc, sbuf);
    if (threadIdx.x == 0) a.partial[(long) blockIdx.y * gridDim.x + blockIdx.x] = r;
  } else {
    T2 *d = dst + off;
#pragma unroll
    for (int m = 0; m < P; m++) d[(unsigned) (t + TL * m) * in32] = v[m];
  }
}

// Pipelined strided passes: a persistent CTA walks over its tiles (BZ
// columns x N rows of one outer index).  Each tile arrives in a landing
// buffer through one tiled tensor copy (TMA, no multicast) per 256 rows,
// completing on an mbarrier; as soon as every thread has its elements in
// registers, the next tile's copy is issued, so the HBM reads of tile t + G
// run under the transforms and stores of tile t.  The radix exchanges use a
// separate buffer.  Waits are bounded: a CTA whose wait gives up sets the
// pass error flag, waits (bounded) for its copy in flight and leaves.
int pipe_enabled();

template <int N> __host__ __device__ constexpr int pipe_rows() { return N < 256 ? N : 256; }

#ifndef GB_PIPE_MINB
#define GB_PIPE_MINB 3
#endif
template <typename T, int N, int BZ, int... Ops>
__global__ void __launch_bounds__((N / Sched<N>::P) * BZ, GB_PIPE_MINB)
    k_pass_strided_pipe(C2<T> *__restrict__ dst, unsigned inner, unsigned ncb, unsigned ntiles, PassArgs a,
                        const __grid_constant__ CUtensorMap tmap) {
  using T2 = C2<T>;
  constexpr int P = Sched<N>::P, TL = N / P;
  constexpr int ROWS = pipe_rows<N>();
  constexpr unsigned TILE_BYTES = (unsigned) (N * BZ * sizeof(T2));
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ __align__(8) uint64_t bar;
  // the dynamic buffer has 128 spare bytes: the landing buffer starts at the
  // first 128-byte boundary in it, as the tensor copy requires
  unsigned char *base = smraw + ((128u - (smem_u32(smraw) & 127u)) & 127u);
  T2 *land = (T2 *) base;
  T2 *xch = (T2 *) (base + TILE_BYTES);
  const int tid = threadIdx.x;
  const int c = tid % BZ, t = tid / BZ;
  // a descriptor that is not 64-byte aligned is recorded (code 3) and the
  // pass skipped
  if (((size_t) &tmap & 63u) != 0) {
    if (tid == 0 && a.errflag) atomicExch(a.errflag, 3);
    return;
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  unsigned tile = blockIdx.x;
  if (tid == 0 && tile < ntiles) {
    const unsigned o = tile / ncb, cb = tile - o * ncb;
    mbar_arrive_expect_tx(&bar, TILE_BYTES);
#pragma unroll
    for (int h = 0; h < N / ROWS; h++) tma_load_3d(land + h * ROWS * BZ, &tmap, (int) (cb * 2 * BZ), h * ROWS, (int) o, &bar);
  }
  for (unsigned it = 0; tile < ntiles; tile += gridDim.x, it++) {
    const bool ok = mbar_wait_bounded(&bar, it & 1u);
    T2 v[P];
#pragma unroll
    for (int m = 0; m < P; m++) v[m] = land[(t + TL * m) * BZ + c];
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        if (a.errflag) atomicExch(a.errflag, 1);
        mbar_wait_bounded(&bar, it & 1u);
      }
      return;
    }
    const unsigned next = tile + gridDim.x;
    if (tid == 0 && next < ntiles) {
      const unsigned o = next / ncb, cb = next - o * ncb;
      mbar_arrive_expect_tx(&bar, TILE_BYTES);
#pragma unroll
      for (int h = 0; h < N / ROWS; h++)
        tma_load_3d(land + h * ROWS * BZ, &tmap, (int) (cb * 2 * BZ), h * ROWS, (int) o, &bar);
    }
    const unsigned o = tile / ncb;
    const unsigned q = (tile - o * ncb) * (unsigned) BZ + (unsigned) c;
    SmStrided<T2, BZ> sm{xch + c};
    double acc = 0.0;
    Program<T, N, SmStrided<T2, BZ>, Ops...>::run(v, t, sm, a, o, q, acc);
    T2 *d = dst + (size_t) o * (size_t) N * inner + q;
#pragma unroll
    for (int m = 0; m < P; m++) d[(unsigned) (t + TL * m) * inner] = v[m];
  }
}

// Launch the pipelined form when it applies (strided lines of 64..256,
// programs with the kinetic op and without a potential or a reduction);
// *launched says whether it did.
template <typename T, int N, int BZ, int... Ops>
int launch_strided_pipe(const void *src, void *dst, const PassArgs &a, long outer, long inner, int *launched) {
  *launched = 0;
  // measured on B200: the prefetch pays off on the fused FWD.K.INV pass
  // (two transforms per tile), while single-transform passes are faster in
  // the plain form, which keeps more warps resident
  if constexpr (N < 64 || N > 256 || has_ksq(OpL<Ops...>{}) || has_pot(OpL<Ops...>{}) || !has_kin(OpL<Ops...>{})) {
    return 0;
  } else {
    using T2 = C2<T>;
    if (!pipe_enabled() || !a.errflag || (size_t) src % 16 != 0 || inner % BZ != 0) return 0;
    const long ncb = inner / BZ, ntiles = outer * ncb;
    if (ntiles >= (1l << 31) || inner >= (1l << 30)) return 0;
    constexpr size_t SM = 2 * (size_t) N * BZ * sizeof(T2) + 128;
    constexpr int THREADS = (N / Sched<N>::P) * BZ;
    auto kern = k_pass_strided_pipe<T, N, BZ, Ops...>;
    // resident CTAs per device (0: not yet known, -1: the kernel does not fit)
    static int rgrids[kMaxDevices] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int &rgrid = rgrids[dev >= 0 && dev < kMaxDevices ? dev : 0];
    if (!rgrid) {
      int nsm = 0, per = 0;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) SM);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, THREADS, SM);
      rgrid = (nsm > 0 && per > 0) ? nsm * per : -1;
    }
    if (rgrid < 0) return 0;
    CUtensorMap tm;
    if (gb__tmap_lines(&tm, src, outer, N, inner, sizeof(T) == 4, BZ, pipe_rows<N>())) return gb_last_error();
    const long g = ntiles < rgrid ? ntiles : rgrid;
    kern<<<(unsigned) g, THREADS, SM, gb__stream()>>>((T2 *) dst, (unsigned) inner, (unsigned) ncb,
                                                       (unsigned) ntiles, a, tm);
    *launched = 1;
    GB_CHECK_LAUNCH("pipelined fft pass");
    return 0;
  }
}

// Launch one pass of program Ops along `axis` for line length N.
template <typename T, int N, int... Ops>
int launch_pass_n(const void *src, void *dst, const PassArgs &a, long outer, long inner, long *nblocks) {
  using T2 = C2<T>;
  // per-thread staging of the potential values (P reals per thread)
  constexpr size_t STAGE = has_pot(OpL<Ops...>{}) ? (size_t) Sched<N>::P * sizeof(T) : 0;
  cudaStream_t st = gb__stream();
  if (inner == 1) {
    using Cfg = ContigCfg<N, sizeof(T)>;
    const size_t sm = (size_t) Cfg::L * Cfg::LINE * sizeof(T2) + STAGE * Cfg::THREADS;
    auto kern = k_pass_contig<T, N, Ops...>;
    static bool attr_set = false;
    if (!attr_set) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
      attr_set = true;
    }
    const long nb = (outer + Cfg::L - 1) / Cfg::L;
    if (nblocks) *nblocks = nb;
    kern<<<(unsigned) nb, Cfg::THREADS, sm, st>>>((const T2 *) src, (T2 *) dst, outer, a);
  } else {
    constexpr int BZ = StridedCfg<N, sizeof(T)>::BZ;
    if (!nblocks) {
      int launched = 0;
      const int rc = launch_strided_pipe<T, N, BZ, Ops...>(src, dst, a, outer, inner, &launched);
      if (rc || launched) return rc;
    }
    if (inner % BZ == 0 && outer <= 65535) {
      const size_t sm = (size_t) N * BZ * sizeof(T2) + STAGE * (N / Sched<N>::P) * BZ;
      auto kern = k_pass_strided<T, N, BZ, Ops...>;
      static bool attr_set = false;
      if (!attr_set) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
        attr_set = true;
      }
      dim3 grid((unsigned) (inner / BZ), (unsigned) outer);
      if (nblocks) *nblocks = (long) grid.x * grid.y;
      kern<<<grid, (N / Sched<N>::P) * BZ, sm, st>>>((const T2 *) src, (T2 *) dst, inner, a);
    } else if (outer <= 65535) {
      const size_t sm = (size_t) N * sizeof(T2) + STAGE * (N / Sched<N>::P);
      auto kern = k_pass_strided<T, N, 1, Ops...>;
      static bool attr_set = false;
      if (!attr_set) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
        attr_set = true;
      }
      dim3 grid((unsigned) inner, (unsigned) outer);
      if (nblocks) *nblocks = (long) grid.x * grid.y;
      kern<<<grid, N / Sched<N>::P, sm, st>>>((const T2 *) src, (T2 *) dst, inner, a);
    } else {
      return gb__set_error(1001, "fft pass: outer extent above 65535");
    }
  }
  GB_CHECK_LAUNCH("fft pass");
  return 0;
}

// Number of blocks a pass will launch (for sizing OP_KSQ partials).
template <int N, int ES> long pass_blocks(long outer, long inner) {
  if (inner == 1) return (outer + ContigCfg<N, ES>::L - 1) / ContigCfg<N, ES>::L;
  constexpr int BZ = StridedCfg<N, ES>::BZ;
  if (inner % BZ == 0) return (inner / BZ) * outer;
  return inner * outer;
}

template <typename T, int... Ops>
int launch_pass(long n, const void *src, void *dst, const PassArgs &a, long outer, long inner, OpL<Ops...>) {
  switch (n) {
    case 2: return launch_pass_n<T, 2, Ops...>(src, dst, a, outer, inner, nullptr);
    case 4: return launch_pass_n<T, 4, Ops...>(src, dst, a, outer, inner, nullptr);
    case 8: return launch_pass_n<T, 8, Ops...>(src, dst, a, outer, inner, nullptr);
    case 16: return launch_pass_n<T, 16, Ops...>(src, dst, a, outer, inner, nullptr);
    case 32: return launch_pass_n<T, 32, Ops...>(src, dst, a, outer, inner, nullptr);
    case 64: return launch_pass_n<T, 64, Ops...>(src, dst, a, outer, inner, nullptr);
    case 128: return launch_pass_n<T, 128, Ops...>(src, dst, a, outer, inner, nullptr);
    case 256: return launch_pass_n<T, 256, Ops...>(src, dst, a, outer, inner, nullptr);
    case 512: return launch_pass_n<T, 512, Ops...>(src, dst, a, outer, inner, nullptr);
    case 1024: return launch_pass_n<T, 1024, Ops...>(src, dst, a, outer, inner, nullptr);
    case 2048: return launch_pass_n<T, 2048, Ops...>(src, dst, a, outer, inner, nullptr);
    case 4096: return launch_pass_n<T, 4096, Ops...>(src, dst, a, outer, inner, nullptr);
    default: return gb__set_error(1002, "fft pass: line length must be a power of two in [2, 4096]");
  }
}

template <int ES> long blocks_for(long n, long outer, long inner) {
  switch (n) {
    case 2: return pass_blocks<2, ES>(outer, inner);
    case 4: return pass_blocks<4, ES>(outer, inner);
    case 8: return pass_blocks<8, ES>(outer, inner);
    case 16: return pass_blocks<16, ES>(outer, inner);
    case 32: return pass_blocks<32, ES>(outer, inner);
    case 64: return pass_blocks<64, ES>(outer, inner);
    case 128: return pass_blocks<128, ES>(outer, inner);
    case 256: return pass_blocks<256, ES>(outer, inner);
    case 512: return pass_blocks<512, ES>(outer, inner);
    case 1024: return pass_blocks<1024, ES>(outer, inner);
    case 2048: return pass_blocks<2048, ES>(outer, inner);
    case 4096: return pass_blocks<4096, ES>(outer, inner);
    default: return 0;
  }
}

}  // namespace gbfft
