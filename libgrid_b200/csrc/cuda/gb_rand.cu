// Seeded noise on device grids (the reference's src/rand.c and
// src/rand-cuda2.cu:54-300 API), from a counter-based generator: element i of
// call c draws its uniforms from splitmix64 (G. L. Steele, D. Lea, C. H.
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014)
// applied to the counter (seed, c, i), so no generator state is stored per
// thread and a result depends only on the seed, the call number and the
// element.  Normal deviates by the Box-Muller transform.  The reference's
// CPU path (drand48) and GPU path (cuRAND states) already differ from each
// other, so these calls match them in distribution, not in values.
#include <math.h>

#include "gb_common.cuh"
#include "gb_internal_cuda.h"

namespace {

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform in (0, 1) with 53 random bits (never 0, so log() is finite).
__device__ __forceinline__ double u01(unsigned long long z) { return ((double) (z >> 11) + 0.5) * 0x1.0p-53; }

// The two uniforms of element i in call `call`.
__device__ __forceinline__ void draw2(unsigned long long seed, unsigned long long call, unsigned long long i, double &a,
                                      double &b) {
  const unsigned long long base = splitmix64(seed ^ splitmix64(call + 0x632BE59BD9B4E019ull));
  a = u01(splitmix64(base + 2 * i));
  b = u01(splitmix64(base + 2 * i + 1));
}

// Standard normal from two uniforms (Box-Muller; the cosine branch).
__device__ __forceinline__ double normal(double a, double b) { return sqrt(-2.0 * log(a)) * cospi(2.0 * b); }

template <typename T>
__global__ void k_random(int kind, T *data, long nxy, long nz, long row, double sre, double sim,
                         unsigned long long seed, unsigned long long call) {
  const long n = nxy * nz;
  for (long g = blockIdx.x * (long) blockDim.x + threadIdx.x; g < n; g += (long) gridDim.x * blockDim.x) {
    double a, b;
    draw2(seed, call, (unsigned long long) g, a, b);
    if (kind == GB_RAND_R_UNIFORM || kind == GB_RAND_R_NORMAL) {
      const long ij = g / nz, k = g - ij * nz;
      T &r = data[ij * row + k];
      r = (T) ((double) r + (kind == GB_RAND_R_UNIFORM ? 2.0 * sre * (a - 0.5) : sre * normal(a, b)));
      continue;
    }
    C2<T> &z = ((C2<T> *) data)[g];
    double dr = 0.0, di = 0.0;
    switch (kind) {
      case GB_RAND_C_UNIFORM:  // src/rand.c:132-149
        dr = 2.0 * sre * (a - 0.5);
        di = 2.0 * sim * (b - 0.5);
        break;
      case GB_RAND_C_UNIFORM_SP: {  // src/rand.c:159-176: scale u exp(2 pi i u')
        double s, c;
        sincospi(2.0 * b, &s, &c);
        dr = sre * a * c;
        di = sre * a * s;
      } break;
      case GB_RAND_C_NORMAL: {  // src/rand.c:186-214: Re(scale) n1 + i Im(scale) n2
        const double r = sqrt(-2.0 * log(a));
        double s, c;
        sincospi(2.0 * b, &s, &c);
        dr = sre * r * c;
        di = sim * r * s;
      } break;
      default: {  // GB_RAND_C_NORMAL_SP, src/rand.c:224-250: scale n exp(i pi u)
        unsigned long long e = splitmix64((unsigned long long) g ^ 0xD1B54A32D192ED03ull ^ (seed + call));
        const double n1 = normal(a, b);
        double s, c;
        sincospi(u01(e), &s, &c);
        dr = sre * n1 * c;
        di = sre * n1 * s;
      } break;
    }
    z = C2<T>{(T) ((double) z.x + dr), (T) ((double) z.y + di)};
  }
}

}  // namespace

extern "C" int gb_random(int kind, void *data, const gb_geom *g, long row, double scale_re, double scale_im,
                         unsigned long long seed, unsigned long long call) {
  if (kind < GB_RAND_R_UNIFORM || kind > GB_RAND_C_NORMAL_SP) return gb__set_error(1050, "random: unknown kind");
  const long nxy = g->nx * g->ny;
  const long n = nxy * g->nz;
  if (n <= 0) return 0;
  long nb = (n + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  cudaStream_t st = gb__stream();
  if (g->prec == GB_FP32)
    k_random<float><<<(unsigned) nb, 256, 0, st>>>(kind, (float *) data, nxy, g->nz, row, scale_re, scale_im, seed,
                                                    call);
  else
    k_random<double><<<(unsigned) nb, 256, 0, st>>>(kind, (double *) data, nxy, g->nz, row, scale_re, scale_im, seed,
                                                     call);
  GB_CHECK_LAUNCH("random");
  return 0;
}
