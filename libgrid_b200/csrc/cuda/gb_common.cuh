// Shared device helpers for the libgrid-b200 CUDA layer (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gb_cuda.h"

// Complex storage type per arithmetic precision.
template <typename T> struct cplx_of;
template <> struct cplx_of<double> { using type = double2; };
template <> struct cplx_of<float> { using type = float2; };
template <typename T> using C2 = typename cplx_of<T>::type;

template <typename T2> __device__ __forceinline__ T2 cadd(T2 a, T2 b) { return T2{a.x + b.x, a.y + b.y}; }
template <typename T2> __device__ __forceinline__ T2 csub(T2 a, T2 b) { return T2{a.x - b.x, a.y - b.y}; }
template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  return T2{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// conj(a) * b
template <typename T2> __device__ __forceinline__ T2 cconjmul(T2 a, T2 b) {
  return T2{a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x};
}
template <typename T2, typename S> __device__ __forceinline__ T2 cscale(T2 a, S s) { return T2{a.x * s, a.y * s}; }
template <typename T2> __device__ __forceinline__ auto cnorm2(T2 a) { return a.x * a.x + a.y * a.y; }

// Multiply by S*i (S = -1 forward, +1 inverse transform sign).
template <int S, typename T2> __device__ __forceinline__ T2 mul_si(T2 a) {
  if constexpr (S > 0) return T2{-a.y, a.x};
  else return T2{a.y, -a.x};
}

// Complex division a / b with scaling against overflow (FP64 use).
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  double s = fabs(b.x) + fabs(b.y);
  double inv_s = 1.0 / s;
  double br = b.x * inv_s, bi = b.y * inv_s;
  double ar = a.x * inv_s, ai = a.y * inv_s;
  double d = br * br + bi * bi;
  return double2{(ar * br + ai * bi) / d, (ai * br - ar * bi) / d};
}

template <typename T> __device__ __forceinline__ C2<T> to_c2(double re, double im) {
  return C2<T>{(T) re, (T) im};
}

// 2 pi split into a double-rounded leading part and the rounded remainder
// (Cody-Waite style), used to reduce phase arguments in FP64 before the FP32
// sincosf of the FP32 propagation mode.  HI = RN(2 pi); LO = RN(2 pi - HI).
#define GB_TWO_PI_HI 6.283185307179586231995926937088
#define GB_TWO_PI_LO 2.4492935982947063e-16
#define GB_INV_TWO_PI 0.15915494309189533577

// sin and cos of a phase argument in FP64 for |x| <= 1e7 (larger arguments
// use the CUDA library routine).  Cody-Waite reduction by pi/2 (W. J. Cody,
// W. Waite, "Software Manual for the Elementary Functions", 1980): n =
// rint(x 2/pi), r = x - n (P1 + P2 + P3) with P1, P2 holding the leading 30
// significant bits of pi/2 each (so n P1 and n P2 are exact for |n| < 2^23)
// and P3 the rounded remainder, split here from the decimal expansion of pi.
// On |r| <= pi/4 the Taylor series of sin and cos are cut after r^17/17! and
// r^16/16! (truncation below 1e-17) and evaluated in r^2 by Estrin's scheme.  The
// quadrant q = n mod 4 is applied without branches: q odd swaps sin and
// cos, bit 1 of q (of q + 1 for the cosine) flips the sign.
// The library fallback stays out of line, so the unrolled per-element loops
// of the passes hold one copy of it.
static __device__ __noinline__ double2 gb_sincos_lib(double x) {
  double s, c;
  sincos(x, &s, &c);
  return double2{s, c};
}

__device__ __forceinline__ double gb_flip_sign(double v, int bit2) {
  return __hiloint2double(__double2hiint(v) ^ (bit2 << 30), __double2loint(v));
}

// (sin r, cos r) for |r| <= pi/4 by the two series below.
__device__ __forceinline__ double2 gb_sincos_series(double r) {
  // both series in s2 = r^2, evaluated by Estrin's scheme (pairs of terms,
  // then powers s2^2 and s2^4 shared by sine and cosine) for a short
  // dependency chain
  const double s2 = r * r;
  const double s4 = s2 * s2;
  const double s8 = s4 * s4;
  // sin: r + r s2 (-1/3! + s2/5! - s2^2/7! + ... + s2^7/17!)
  const double a01 = fma(0.008333333333333333, s2, -0.16666666666666666);
  const double a23 = fma(2.7557319223985893e-06, s2, -0.0001984126984126984);
  const double a45 = fma(1.6059043836821613e-10, s2, -2.505210838544172e-08);
  const double a67 = fma(2.8114572543455206e-15, s2, -7.647163731819816e-13);
  const double ps = fma(fma(a67, s4, a45), s8, fma(a23, s4, a01));
  // cos: 1 + s2 (-1/2! + s2/4! - ... + s2^7/16!)
  const double b01 = fma(0.041666666666666664, s2, -0.5);
  const double b23 = fma(2.48015873015873e-05, s2, -0.001388888888888889);
  const double b45 = fma(2.08767569878681e-09, s2, -2.755731922398589e-07);
  const double b67 = fma(4.779477332387385e-14, s2, -1.1470745597729725e-11);
  const double pc = fma(fma(b67, s4, b45), s8, fma(b23, s4, b01));
  return double2{fma(r * s2, ps, r), fma(s2, pc, 1.0)};
}

// (sin x, cos x) for |x| <= 1e7; out of line (with the library fallback it
// serves the rare large phases), so the unrolled element loops stay small.
static __device__ __noinline__ double2 gb_sincos_reduced(double x) {
  const double n = rint(x * 0.6366197723675814);
  const int q = __double2int_rn(n);
  double r = fma(-n, 1.570796325802803, x);
  r = fma(-n, 9.920935791635221e-10, r);
  r = fma(-n, 5.170182981794105e-19, r);
  const double2 sc = gb_sincos_series(r);
  const bool swap = (q & 1) != 0;
  const double s = swap ? sc.y : sc.x;
  const double c = swap ? sc.x : sc.y;
  return double2{gb_flip_sign(s, q & 2), gb_flip_sign(c, (q + 1) & 2)};
}

// (sin x, cos x) for any x.  Below pi/4 (n = 0: r = x exactly, quadrant 0)
// the series apply directly, with the same result as the reduced path; this
// is the usual case for split-operator phases dt (V + g |psi|^2).
__device__ __forceinline__ double2 gb_sincos2(double x) {
  if (fabs(x) < 0.0625) {
    // |x| < 1/16: sin to x^9 and cos to x^8 (the next terms are below
    // 3e-19 relative)
    const double x2 = x * x;
    const double ps =
        fma(fma(fma(2.7557319223985893e-06, x2, -1.984126984126984e-4), x2, 0.008333333333333333), x2,
            -0.16666666666666666);
    const double pc =
        fma(fma(fma(2.48015873015873e-05, x2, -0.001388888888888889), x2, 0.041666666666666664), x2, -0.5);
    return double2{fma(x * x2, ps, x), fma(x2, pc, 1.0)};
  }
  if (fabs(x) < 0.78539816339744828) return gb_sincos_series(x);
  if (!(fabs(x) <= 1.0e7)) return gb_sincos_lib(x);
  return gb_sincos_reduced(x);
}

__device__ __forceinline__ void gb_sincos(double x, double *sp, double *cp) {
  const double2 sc = gb_sincos2(x);
  *sp = sc.x;
  *cp = sc.y;
}

// exp(a + i b) as a complex number of type T, with both a and b evaluated in
// FP64.  FP64 mode: exp and sincos in FP64.  FP32 mode: b is reduced into
// [-pi, pi] in FP64, then the hardware sine/cosine and the FP64 exp rounded
// to FP32.
template <typename T> __device__ __forceinline__ C2<T> cexp_phase(double a, double b, bool has_a) {
  if constexpr (sizeof(T) == 8) {
    const double2 sc = gb_sincos2(b);
    if (has_a) {
      const double m = exp(a);
      return C2<T>{m * sc.y, m * sc.x};
    }
    return C2<T>{sc.y, sc.x};
  } else {
    const double n = rint(b * GB_INV_TWO_PI);
    double r = fma(-n, GB_TWO_PI_HI, b);
    r = fma(-n, GB_TWO_PI_LO, r);
    float s, c;
    __sincosf((float) r, &s, &c);
    if (has_a) {
      const float m = (float) exp(a);
      return C2<T>{m * c, m * s};
    }
    return C2<T>{c, s};
  }
}

// Host-side launch bookkeeping (defined in gb_runtime.cu).
extern "C" void gb__count_launch(void);
extern "C" int gb__set_error(int code, const char *where);
extern "C" cudaStream_t gb__stream(void);

#define GB_CHECK_LAUNCH(where)                                     \
  do {                                                             \
    gb__count_launch();                                            \
    cudaError_t e_ = cudaGetLastError();                           \
    if (e_ != cudaSuccess) return gb__set_error((int) e_, where);  \
  } while (0)

// ------------------------------------------------------------------------
// Bulk asynchronous copies (TMA, non-tensor form) and mbarriers.
// All waits are bounded: after GB_WAIT_LIMIT polls the caller gets `false`
// and must record an error and leave without touching the data.
#define GB_WAIT_LIMIT (1u << 22)

// Devices for which per-device launch geometry is cached.
constexpr int kMaxDevices = 64;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned) __cvta_generic_to_shared(p); }

// Per-thread asynchronous global -> shared copy of one 4- or 8-byte element
// (both addresses naturally aligned); completion is awaited by the issuing
// thread with cp_async_wait_all().
template <int BYTES> __device__ __forceinline__ void cp_async_elem(void *sdst, const void *gsrc) {
  static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async size");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(sdst)), "l"(gsrc), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned phase) {
  for (unsigned it = 0; it < GB_WAIT_LIMIT; it++)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}
// global -> shared, completion signalled on bar (bytes multiple of 16,
// both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_g2s(void *sdst, const void *gsrc, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(sdst)),
               "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// 3-D tiled tensor copy global -> shared through a tensor map (no
// multicast); coordinates innermost first, completion signalled on bar.
__device__ __forceinline__ void tma_load_3d(void *sdst, const void *tmap, int c0, int c1, int c2, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(sdst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
// shared -> global in the calling thread's bulk group
__device__ __forceinline__ void bulk_s2g(void *gdst, const void *ssrc, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(ssrc)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// the calling thread's committed bulk stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

#define GB_TRYC(x)          \
  do {                      \
    int rc_ = (x);          \
    if (rc_) return rc_;    \
  } while (0)
