// Plane-chained passes: one persistent launch runs a chain of line stages on
// the y and z axes (z FWD then y FWD; y INV then z INV; in FP64 also
// z INV.V.FWD then y FWD), plane by plane, so a plane's intermediate result
// is read back from L2 by the next stage instead of making a full HBM round
// trip: the chain reads and writes psi in HBM once.  An FP64 split step runs
//   [z FWD, y FWD] | x FWD.K.INV | y INV | [z INV.V.FWD, y FWD] | x FWD.K.INV | [y INV, z INV]
//
// Work is a sequence of tickets drawn from a global counter.  Ticket group
// g holds, for every stage s, the tiles of plane g - s * lag, so stage s of
// a plane is issued lag groups after stage s - 1 of the same plane.  A tile
// of stage s > 0 waits until all tiles of stage s - 1 of its plane have
// completed (a per-plane counter).  Tiles it waits for always hold smaller
// tickets, and a ticket is only drawn by a running CTA, so the oldest
// unfinished tile never waits: the chain cannot deadlock.  The wait is
// bounded all the same; when it gives up it sets the pass error flag.
// Reads of psi bypass L1 (another SM wrote them in this launch).
#pragma once

#include "gb_fft_impl.cuh"
#include "gb_internal_cuda.h"

namespace gbfft {


template <int AX, int... Ops> struct Stage {};

// Resident CTAs per SM the FP64 chains are compiled for (register caps of
// 128 threads x 168 / 128 registers); overridable for tuning builds.
#ifndef GB_CHAIN_POT_MINB
#define GB_CHAIN_POT_MINB 3
#endif
#ifndef GB_CHAIN_MINB64
#define GB_CHAIN_MINB64 4
#endif

template <typename T, int N> struct ChainCfg {
  static constexpr int P = Sched<N>::P;
  static constexpr int TL = N / P;
  static constexpr int THREADS = sizeof(T) == 8 ? 128 : 256;
  static constexpr int W = THREADS / TL;  // z lines or y columns per tile
  static constexpr int TILES = N / W;     // tiles per plane and stage
  static constexpr int SH = ilog2c(first_radix(typename Sched<N>::R{}));
  static constexpr int LINE = N + (N >> SH);
  static constexpr int SM_Z = W * LINE, SM_Y = N * W;  // exchange elements
  static constexpr int SM_X = SM_Z > SM_Y ? SM_Z : SM_Y;
  static constexpr int MINB = sizeof(T) == 8 ? GB_CHAIN_MINB64 : 3;
};

struct ChainArgs {
  PassArgs ay, az;    // y-stage and z-stage arguments
  int *cnt;           // [stage][plane] completed tiles
  unsigned *ticket;   // ticket counter
  int nplanes, lag;
  unsigned wait_limit;  // polls before a dependency wait gives up
};

// a stage that carries the potential op between two transforms (the
// register-heaviest stage)
template <int AX, int... Ops> __host__ __device__ constexpr bool stage_heavy(Stage<AX, Ops...>) {
  return ((Ops == OP_POT || Ops == OP_POT_RP) || ...) && (((Ops == OP_FWD || Ops == OP_INV) ? 1 : 0) + ...) >= 2;
}

template <int AX, int... Ops> __host__ __device__ constexpr bool stage_has_pot(Stage<AX, Ops...>) {
  return ((Ops == OP_POT || Ops == OP_POT_RP) || ...);
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add(int *p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename T> __device__ __forceinline__ C2<T> ldcg2(const C2<T> *p) { return __ldcg(p); }

// One tile of a z stage (W contiguous lines of plane p) or a y stage (W
// adjacent columns of plane p); same per-line arithmetic as the line passes.
template <typename T, int N, int AX, int... Ops>
__device__ __forceinline__ void chain_tile(Stage<AX, Ops...>, C2<T> *__restrict__ psi, const ChainArgs &c,
                                           unsigned p, unsigned tile, unsigned char *smraw) {
  using T2 = C2<T>;
  using Cfg = ChainCfg<T, N>;
  constexpr int P = Cfg::P, TL = Cfg::TL, W = Cfg::W, THREADS = Cfg::THREADS;
  T2 *smem = (T2 *) smraw;
  T *stage = (T *) (smraw + (size_t) Cfg::SM_X * sizeof(T2)) + threadIdx.x;
  T2 v[P];
  double acc = 0.0;
  if constexpr (AX == 2) {
    const int l = threadIdx.x / TL, t = threadIdx.x % TL;
    const unsigned line = p * (unsigned) N + tile * (unsigned) W + (unsigned) l;
    const T *vstage = nullptr;
    if constexpr (((Ops == OP_POT || Ops == OP_POT_RP) || ...)) {
      if (pot_prefetch<T, P, TL>(c.az, line, 0u, t, stage, THREADS)) vstage = stage;
    }
    T2 *s = psi + (size_t) line * N;
#pragma unroll
    for (int m = 0; m < P; m++) v[m] = ldcg2<T>(s + t + TL * m);
    SmContig<T2, Cfg::SH, TL> sm{smem + l * Cfg::LINE};
    Program<T, N, SmContig<T2, Cfg::SH, TL>, Ops...>::run(v, t, sm, c.az, line, 0u, acc, vstage, THREADS);
#pragma unroll
    for (int m = 0; m < P; m++) s[t + TL * m] = v[m];
  } else {
    const int cc = threadIdx.x % W, t = threadIdx.x / W;
    const unsigned q = tile * (unsigned) W + (unsigned) cc;
    const T *vstage = nullptr;
    if constexpr (((Ops == OP_POT || Ops == OP_POT_RP) || ...)) {
      if (pot_prefetch<T, P, TL>(c.ay, p, q, t, stage, THREADS)) vstage = stage;
    }
    T2 *s = psi + (size_t) p * N * N + q;
#pragma unroll
    for (int m = 0; m < P; m++) v[m] = ldcg2<T>(s + (unsigned) (t + TL * m) * N);
    SmStrided<T2, W> sm{smem + cc};
    Program<T, N, SmStrided<T2, W>, Ops...>::run(v, t, sm, c.ay, p, q, acc, vstage, THREADS);
#pragma unroll
    for (int m = 0; m < P; m++) s[(unsigned) (t + TL * m) * N] = v[m];
  }
}

// Resident CTAs per SM for the register bound: a chain with a stage that
// carries the potential op between two transforms gets 3 in FP64, so it
// does not spill.
template <typename T, int N, class... Stages> constexpr int chain_minb() {
  return (sizeof(T) == 8 && (stage_heavy(Stages{}) || ...)) ? GB_CHAIN_POT_MINB : ChainCfg<T, N>::MINB;
}

template <typename T, int N, class... Stages>
__global__ void __launch_bounds__(ChainCfg<T, N>::THREADS, chain_minb<T, N, Stages...>())
    k_chain(C2<T> *__restrict__ psi, ChainArgs c) {
  using Cfg = ChainCfg<T, N>;
  constexpr int S = sizeof...(Stages);
  constexpr unsigned TILES = Cfg::TILES;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ unsigned s_tk[2];
  const unsigned np = (unsigned) c.nplanes;
  const unsigned total = (np + (unsigned) ((S - 1) * c.lag)) * S * TILES;
  if (threadIdx.x == 0) s_tk[0] = atomicAdd(c.ticket, 1u);
  __syncthreads();
  for (int it = 0;; it++) {
    const unsigned tk = s_tk[it & 1];
    if (tk >= total) break;
    // the next ticket is drawn now and stored at the end of this tile
    unsigned nxt = 0;
    if (threadIdx.x == 0) nxt = atomicAdd(c.ticket, 1u);
    const unsigned g = tk / (S * TILES), rem = tk % (S * TILES);
    const int s = (int) (rem / TILES);
    const unsigned tile = rem % TILES;
    const int pi = (int) g - s * c.lag;
    const bool valid = pi >= 0 && pi < (int) np;
    const unsigned p = valid ? (unsigned) pi : 0u;
    if (valid && s > 0) {
      if (threadIdx.x == 0) {
        const int *f = c.cnt + (size_t) (s - 1) * np + p;
        unsigned n = 0;
        while (ld_acquire(f) < (int) TILES) {
          if (++n > c.wait_limit) {
            atomicOr(c.ay.errflag, 8);
            break;
          }
          __nanosleep(32);
        }
      }
      __syncthreads();
    }
    if (valid) {
      int idx = 0;
      ((idx++ == s ? chain_tile<T, N>(Stages{}, psi, c, p, tile, smraw) : void()), ...);
    }
    if (threadIdx.x == 0) s_tk[(it + 1) & 1] = nxt;
    __syncthreads();
    // publish the tile: the barrier orders every thread's stores before
    // this release increment
    if (valid && threadIdx.x == 0) red_release_add(c.cnt + (size_t) s * np + p, 1);
  }
}

template <typename T, int N, class... Stages> constexpr size_t chain_smem() {
  using Cfg = ChainCfg<T, N>;
  return (size_t) Cfg::SM_X * sizeof(C2<T>) +
         ((stage_has_pot(Stages{}) || ...) ? (size_t) Cfg::THREADS * Cfg::P * sizeof(T) : 0);
}

// Launch one chain over all nx planes: the counters (S * nx + 1 ints in
// `counters`) are cleared first; grid = resident CTAs (persistent).
template <typename T, int N, class... Stages>
int launch_chain(void *psi, long nx, const ChainArgs &base, int *counters) {
  using Cfg = ChainCfg<T, N>;
  constexpr int S = sizeof...(Stages);
  auto kern = k_chain<T, N, Stages...>;
  constexpr size_t smem = chain_smem<T, N, Stages...>();
  // resident CTAs per device (0: not yet known, -1: the kernel does not fit)
  static int rgrids[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int &rgrid = rgrids[dev >= 0 && dev < kMaxDevices ? dev : 0];
  if (!rgrid) {
    int nsm = 0, per = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, Cfg::THREADS, smem);
    cudaGetLastError();
    rgrid = (nsm > 0 && per > 0) ? nsm * per : -1;
  }
  if (rgrid < 0) return gb__set_error(1062, "chained pass: kernel does not fit");
  // lag: about gb_chain_lag's percentage (default 200) of one resident wave
  // of tickets, so most tiles of a stage find their plane's previous stage
  // complete; any lag >= 0 is free of deadlock
  const long group = (long) S * Cfg::TILES;
  const int lag = (int) (((long) rgrid * gb__chain_lag_pct() / 100 + group - 1) / group);
  ChainArgs c = base;
  c.cnt = counters;
  c.ticket = (unsigned *) (counters + (size_t) S * nx);
  c.nplanes = (int) nx;
  c.lag = lag;
  c.wait_limit = gb__wait_limit(GB_WAIT_LIMIT);
  cudaStream_t st = gb__stream();
  if (cudaMemsetAsync(counters, 0, sizeof(int) * ((size_t) S * nx + 1), st) != cudaSuccess)
    return gb__set_error(1063, "chained pass: counter reset failed");
  const long tickets = (nx + (long) (S - 1) * lag) * S * Cfg::TILES;
  const long grid = tickets < rgrid ? tickets : rgrid;
  kern<<<(unsigned) grid, Cfg::THREADS, smem, st>>>((C2<T> *) psi, c);
  GB_CHECK_LAUNCH("chained pass");
  return 0;
}

}  // namespace gbfft
