// Batched split-operator propagation of many independent 2-D wave functions
// of uneven sizes (sm_100a).
//
// All instances advance through the same five line passes of a 2-D
// second-order split-operator step (z: contiguous lines, y: strided lines):
//   z FWD | y FWD.K.INV | z INV.V.FWD | y FWD.K.INV | z INV
// One cooperative, persistent launch runs K steps: in every pass the CTAs
// walk a flat list of tiles that spans all instances (a tile is a group of
// z lines, or a block of y columns, of one instance; the line length of the
// tile's instance selects the compiled transform), and a grid-wide barrier
// separates the passes.  The barrier is this file's own (atomic arrival
// counter + generation word) with a bounded wait: a CTA that waits too long
// sets the batch's error flag and leaves, so the launch always ends.
// A second plan steps each shape class with the specialised pass kernels
// (instance as a grid dimension), one stream per class, one step captured as
// a CUDA graph.  A small autotuner picks the plan (persistent with 128, 256
// or 512-thread CTAs, or per-class graph) per batch by timing each on the
// first steps of the first call; all plans compute the same values.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "gb_fft_impl.cuh"
#include "gb_internal_cuda.h"

namespace gbfft {

struct BatchInst {
  PassArgs az;  // z (contiguous) passes
  PassArgs ay;  // y (strided) passes
  void *psi;
  int nz, ny;
};

struct BatchTile {
  int inst;
  int tile;
};

struct BatchDev {
  const BatchInst *inst;
  const BatchTile *ctiles;
  const BatchTile *stiles;
  int nct, nst;
  unsigned *bar;  // [0] arrivals, [1] generation
  int *err;       // status word GB_STATUS_BATCH
  unsigned wait_limit;
};

#define GB_GRID_WAIT_LIMIT (1u << 24)

// Grid-wide barrier of a cooperative launch (all CTAs resident).  Returns
// false on every thread of a CTA whose wait gave up (error flag set).
__device__ __forceinline__ bool batch_grid_barrier(unsigned *bar, int *err, unsigned limit) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    volatile unsigned *gen = bar + 1;
    const unsigned g0 = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned it = 0;
      while (*gen == g0) {
        if (++it > limit) {
          atomicExch(err, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  return !__syncthreads_or(!ok);
}

// One tile of contiguous (z) lines: L = THREADS / TL lines of length N.
template <typename T, int N, int THREADS, int... Ops>
__device__ __forceinline__ void batch_tile_contig(const BatchInst &I, int tile, unsigned char *smraw) {
  using T2 = C2<T>;
  using Cfg = ContigCfg<N, sizeof(T)>;
  constexpr int P = Cfg::P, TL = Cfg::TL, L = THREADS / TL;
  static_assert(THREADS % TL == 0, "CTA size must hold whole lines");
  T2 *smem = (T2 *) smraw;
  const int t = threadIdx.x % TL;
  const int l = threadIdx.x / TL;
  const unsigned line = (unsigned) tile * L + (unsigned) l;
  T2 *psi = (T2 *) I.psi;
  const T2 *s = psi + (size_t) line * N;
  const PassArgs &a = I.az;
  const T *vstage = nullptr;
  if constexpr (has_pot(OpL<Ops...>{})) {
    T *stage = (T *) (smraw + (size_t) L * Cfg::LINE * sizeof(T2)) + threadIdx.x;
    if (pot_prefetch<T, P, TL>(a, line, 0u, t, stage, THREADS)) vstage = stage;
  }
  T2 v[P];
#pragma unroll
  for (int m = 0; m < P; m++) v[m] = s[t + TL * m];
  SmContig<T2, Cfg::SH, TL> sm{smem + l * Cfg::LINE};
  double acc = 0.0;
  Program<T, N, SmContig<T2, Cfg::SH, TL>, Ops...>::run(v, t, sm, a, line, 0u, acc, vstage, THREADS);
  T2 *d = psi + (size_t) line * N;
#pragma unroll
  for (int m = 0; m < P; m++) d[t + TL * m] = v[m];
}

// One tile of strided (y) lines of a 2-D instance (outer = 1): BZ = THREADS
// / TL adjacent columns, each a line of length N with stride inner = nz.
template <typename T, int N, int THREADS, int... Ops>
__device__ __forceinline__ void batch_tile_strided(const BatchInst &I, int tile, unsigned char *smraw) {
  using T2 = C2<T>;
  constexpr int P = Sched<N>::P, TL = N / P, BZ = THREADS / TL;
  static_assert(THREADS % TL == 0, "CTA size must hold whole lines");
  T2 *smem = (T2 *) smraw;
  const int c = threadIdx.x % BZ;
  const int t = threadIdx.x / BZ;
  const unsigned q = (unsigned) tile * BZ + (unsigned) c;
  const unsigned in32 = (unsigned) I.nz;
  T2 *psi = (T2 *) I.psi;
  const T2 *s = psi + q;
  const PassArgs &a = I.ay;
  const T *vstage = nullptr;
  if constexpr (has_pot(OpL<Ops...>{})) {
    T *stage = (T *) (smraw + (size_t) N * BZ * sizeof(T2)) + threadIdx.x;
    if (pot_prefetch<T, P, TL>(a, 0u, q, t, stage, THREADS)) vstage = stage;
  }
  T2 v[P];
#pragma unroll
  for (int m = 0; m < P; m++) v[m] = s[(unsigned) (t + TL * m) * in32];
  SmStrided<T2, BZ> sm{smem + c};
  double acc = 0.0;
  Program<T, N, SmStrided<T2, BZ>, Ops...>::run(v, t, sm, a, 0u, q, acc, vstage, THREADS);
  T2 *d = psi + q;
#pragma unroll
  for (int m = 0; m < P; m++) d[(unsigned) (t + TL * m) * in32] = v[m];
}

// Line lengths a batch takes on either axis.
template <typename T, int THREADS, int... Ops>
__device__ __forceinline__ void batch_contig(const BatchInst &I, int tile, unsigned char *sm) {
  switch (I.nz) {
    case 64: batch_tile_contig<T, 64, THREADS, Ops...>(I, tile, sm); break;
    case 128: batch_tile_contig<T, 128, THREADS, Ops...>(I, tile, sm); break;
    case 256: batch_tile_contig<T, 256, THREADS, Ops...>(I, tile, sm); break;
    default: batch_tile_contig<T, 512, THREADS, Ops...>(I, tile, sm); break;
  }
}
template <typename T, int THREADS, int... Ops>
__device__ __forceinline__ void batch_strided(const BatchInst &I, int tile, unsigned char *sm) {
  switch (I.ny) {
    case 64: batch_tile_strided<T, 64, THREADS, Ops...>(I, tile, sm); break;
    case 128: batch_tile_strided<T, 128, THREADS, Ops...>(I, tile, sm); break;
    case 256: batch_tile_strided<T, 256, THREADS, Ops...>(I, tile, sm); break;
    default: batch_tile_strided<T, 512, THREADS, Ops...>(I, tile, sm); break;
  }
}

// `steps` full steps of every instance; one pass = one sweep of the pass's
// tile list by all CTAs, then a grid barrier.
template <typename T, int THREADS>
__global__ void __launch_bounds__(THREADS, pass_min_blocks<THREADS, sizeof(T)>())
    k_batch_steps(BatchDev d, int steps) {
  extern __shared__ __align__(16) unsigned char smraw[];
  for (int s = 0; s < steps; s++) {
#pragma unroll 1
    for (int ps = 0; ps < 5; ps++) {
      if ((ps & 1) == 0) {
        for (int k = blockIdx.x; k < d.nct; k += gridDim.x) {
          const BatchTile bt = d.ctiles[k];
          const BatchInst &I = d.inst[bt.inst];
          if (ps == 0) batch_contig<T, THREADS, OP_FWD>(I, bt.tile, smraw);
          else if (ps == 2) batch_contig<T, THREADS, OP_INV, OP_POT, OP_FWD>(I, bt.tile, smraw);
          else batch_contig<T, THREADS, OP_INV>(I, bt.tile, smraw);
        }
      } else {
        for (int k = blockIdx.x; k < d.nst; k += gridDim.x) {
          const BatchTile bt = d.stiles[k];
          batch_strided<T, THREADS, OP_FWD, OP_KIN, OP_INV>(d.inst[bt.inst], bt.tile, smraw);
        }
      }
      if (!batch_grid_barrier(d.bar, d.err, d.wait_limit)) return;
    }
  }
}

// Dynamic shared memory of a CTA of THREADS threads: the largest exchange
// buffer over the line lengths plus the per-thread potential slots.
template <typename T, int THREADS> constexpr size_t batch_smem() {
  using T2 = C2<T>;
  size_t m = 0;
  const int ns[4] = {64, 128, 256, 512};
  const int ps[4] = {Sched<64>::P, Sched<128>::P, Sched<256>::P, Sched<512>::P};
  const int lines[4] = {ContigCfg<64>::LINE, ContigCfg<128>::LINE, ContigCfg<256>::LINE, ContigCfg<512>::LINE};
  for (int i = 0; i < 4; i++) {
    const int tl = ns[i] / ps[i];
    const size_t c = (size_t) (THREADS / tl) * lines[i] * sizeof(T2);
    const size_t st = (size_t) ns[i] * (THREADS / tl) * sizeof(T2);
    const size_t a = (c > st ? c : st) + (size_t) THREADS * ps[i] * sizeof(T);
    if (a > m) m = a;
  }
  return m;
}

}  // namespace gbfft

namespace gbfft {

// Per-shape-class kernels: every instance of a class has the same (ny, nz),
// so a pass of the class is one launch of the specialised pass kernel with
// the instance as the second grid dimension, in the CTA shapes of the
// single-grid passes.
template <typename T, int N, int... Ops>
__global__ void __launch_bounds__(ContigCfg<N, sizeof(T)>::THREADS, ContigCfg<N, sizeof(T)>::MINB)
    k_bclass_contig(const BatchInst *inst) {
  extern __shared__ __align__(16) unsigned char smraw[];
  batch_tile_contig<T, N, ContigCfg<N, sizeof(T)>::THREADS, Ops...>(inst[blockIdx.y], blockIdx.x, smraw);
}

template <typename T, int N, int... Ops>
__global__ void __launch_bounds__(StridedCfg<N, sizeof(T)>::THREADS,
                                  pass_min_blocks<StridedCfg<N, sizeof(T)>::THREADS, sizeof(T)>())
    k_bclass_strided(const BatchInst *inst) {
  extern __shared__ __align__(16) unsigned char smraw[];
  batch_tile_strided<T, N, StridedCfg<N, sizeof(T)>::THREADS, Ops...>(inst[blockIdx.y], blockIdx.x, smraw);
}

template <typename T, int N, int... Ops>
int launch_bclass_contig(const BatchInst *d, int ninst, long lines, cudaStream_t st) {
  using T2 = C2<T>;
  using Cfg = ContigCfg<N, sizeof(T)>;
  constexpr size_t STAGE = has_pot(OpL<Ops...>{}) ? (size_t) Cfg::P * sizeof(T) : 0;
  constexpr size_t SM = (size_t) Cfg::L * Cfg::LINE * sizeof(T2) + STAGE * Cfg::THREADS;
  auto k = k_bclass_contig<T, N, Ops...>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) SM);
    attr = true;
  }
  k<<<dim3((unsigned) (lines / Cfg::L), (unsigned) ninst), Cfg::THREADS, SM, st>>>(d);
  GB_CHECK_LAUNCH("batch class pass");
  return 0;
}

template <typename T, int N, int... Ops>
int launch_bclass_strided(const BatchInst *d, int ninst, long inner, cudaStream_t st) {
  using T2 = C2<T>;
  using Cfg = StridedCfg<N, sizeof(T)>;
  constexpr size_t SM = (size_t) N * Cfg::BZ * sizeof(T2);
  auto k = k_bclass_strided<T, N, Ops...>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) SM);
    attr = true;
  }
  k<<<dim3((unsigned) (inner / Cfg::BZ), (unsigned) ninst), Cfg::THREADS, SM, st>>>(d);
  GB_CHECK_LAUNCH("batch class pass");
  return 0;
}

// Pass ps (0..4 of the 2-D step) of one shape class.
template <typename T, int N>
int bclass_contig_pass(int ps, const BatchInst *d, int ninst, long ny, cudaStream_t st) {
  if (ps == 0) return launch_bclass_contig<T, N, OP_FWD>(d, ninst, ny, st);
  if (ps == 2) return launch_bclass_contig<T, N, OP_INV, OP_POT, OP_FWD>(d, ninst, ny, st);
  return launch_bclass_contig<T, N, OP_INV>(d, ninst, ny, st);
}

template <typename T>
int bclass_pass(int ps, const BatchInst *d, int ninst, long ny, long nz, cudaStream_t st) {
  if ((ps & 1) == 0) {
    switch (nz) {
      case 64: return bclass_contig_pass<T, 64>(ps, d, ninst, ny, st);
      case 128: return bclass_contig_pass<T, 128>(ps, d, ninst, ny, st);
      case 256: return bclass_contig_pass<T, 256>(ps, d, ninst, ny, st);
      default: return bclass_contig_pass<T, 512>(ps, d, ninst, ny, st);
    }
  }
  switch (ny) {
    case 64: return launch_bclass_strided<T, 64, OP_FWD, OP_KIN, OP_INV>(d, ninst, nz, st);
    case 128: return launch_bclass_strided<T, 128, OP_FWD, OP_KIN, OP_INV>(d, ninst, nz, st);
    case 256: return launch_bclass_strided<T, 256, OP_FWD, OP_KIN, OP_INV>(d, ninst, nz, st);
    default: return launch_bclass_strided<T, 512, OP_FWD, OP_KIN, OP_INV>(d, ninst, nz, st);
  }
}

}  // namespace gbfft

// ------------------------------------------------------------------ host

using namespace gbfft;

struct gb_batch {
  int n, prec;
  BatchInst *d_inst;
  BatchTile *d_tiles[3][2];  // [variant 128 / 256 / 512][contiguous / strided]
  int ntiles[3][2];
  unsigned char *d_kin;
  unsigned *d_bar;
  int grid[3];
  int threads;  // chosen plan: persistent CTA size, -1 for the class graph, 0 until tuned
  // per-shape-class plan: instances ordered by class, one stream per class,
  // one step captured as a graph
  BatchInst *d_cinst;
  int ncls;
  int cls_off[16], cls_n[16];
  long cls_ny[16], cls_nz[16];
  cudaStream_t cls_st[16];
  cudaEvent_t ev_fork, ev_join[16];
  cudaGraphExec_t graph;
};

static bool batch_len_ok(long v) { return v == 64 || v == 128 || v == 256 || v == 512; }

// Threads per line (N / P) of each line length.
static long batch_tl(long n) {
  switch (n) {
    case 64: return 64 / Sched<64>::P;
    case 128: return 128 / Sched<128>::P;
    case 256: return 256 / Sched<256>::P;
    default: return 512 / Sched<512>::P;
  }
}

template <typename T, int THREADS> static int batch_grid() {
  auto k = k_batch_steps<T, THREADS>;
  constexpr size_t sm = batch_smem<T, THREADS>();
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
  int dev = 0, nsm = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, THREADS, sm);
  return nsm * per;
}

template <typename T, int THREADS> static int batch_launch(gb_batch *b, int steps, int v) {
  BatchDev d;
  d.inst = b->d_inst;
  d.ctiles = b->d_tiles[v][0];
  d.stiles = b->d_tiles[v][1];
  d.nct = b->ntiles[v][0];
  d.nst = b->ntiles[v][1];
  d.bar = b->d_bar;
  d.err = gb__status(GB_STATUS_BATCH);
  if (!d.err) return gb_last_error();
  d.wait_limit = gb__wait_limit(GB_GRID_WAIT_LIMIT);
  void *args[] = {&d, &steps};
  constexpr size_t sm = batch_smem<T, THREADS>();
  // every launch starts from a clear barrier: a CTA whose wait gave up in an
  // earlier launch leaves its arrival counted
  if (cudaMemsetAsync(b->d_bar, 0, 2 * sizeof(unsigned), gb__stream()) != cudaSuccess)
    return gb__set_error(1044, "batch: barrier reset");
  const cudaError_t e = cudaLaunchCooperativeKernel((const void *) k_batch_steps<T, THREADS>, dim3(b->grid[v]),
                                                    dim3(THREADS), args, sm, gb__stream());
  gb__count_launch();
  if (e != cudaSuccess) return gb__set_error((int) e, "batch launch");
  return 0;
}

static const int kBatchThreads[3] = {128, 256, 512};

static int batch_run(gb_batch *b, int steps, int v) {
  if (steps <= 0) return 0;
  if (b->prec == GB_FP32) {
    if (v == 0) return batch_launch<float, 128>(b, steps, 0);
    if (v == 1) return batch_launch<float, 256>(b, steps, 1);
    return batch_launch<float, 512>(b, steps, 2);
  }
  if (v == 0) return batch_launch<double, 128>(b, steps, 0);
  if (v == 1) return batch_launch<double, 256>(b, steps, 1);
  return batch_launch<double, 512>(b, steps, 2);
}

extern "C" gb_batch *gb_batch_create(const gb_batch_item *items, int n) {
  if (n <= 0 || !items) {
    gb__set_error(1040, "batch: no instances");
    return nullptr;
  }
  const int prec = items[0].g.prec;
  for (int i = 0; i < n; i++) {
    const gb_geom &g = items[i].g;
    if (g.nx != 1 || !batch_len_ok(g.ny) || !batch_len_ok(g.nz) || g.prec != prec || !items[i].psi) {
      gb__set_error(1041, "batch: instances must be 2-D (1, ny, nz) with ny, nz in {64, 128, 256, 512} and one precision");
      return nullptr;
    }
  }
  const size_t esz = prec == GB_FP32 ? 8 : 16;
  gb_batch *b = (gb_batch *) calloc(1, sizeof(gb_batch));
  b->n = n;
  b->prec = prec;
  // kinetic tables: per instance (1 + ny + nz) factors and k^2 values
  std::vector<size_t> koff(n);
  size_t kbytes = 0;
  for (int i = 0; i < n; i++) {
    koff[i] = kbytes;
    const size_t tot = 1 + (size_t) items[i].g.ny + (size_t) items[i].g.nz;
    kbytes += (tot * (esz + 8) + 255) & ~(size_t) 255;
  }
  if (cudaMalloc(&b->d_kin, kbytes) != cudaSuccess || cudaMalloc(&b->d_inst, sizeof(BatchInst) * n) != cudaSuccess ||
      cudaMalloc(&b->d_bar, 2 * sizeof(unsigned)) != cudaSuccess) {
    cudaGetLastError();
    gb__set_error(2, "batch: cudaMalloc");
    gb_batch_free(b);
    return nullptr;
  }
  cudaStream_t st = gb__stream();
  cudaMemsetAsync(b->d_bar, 0, 2 * sizeof(unsigned), st);
  std::vector<BatchInst> hi(n);
  for (int i = 0; i < n; i++) {
    const gb_batch_item &it = items[i];
    const long tot = 1 + it.g.ny + it.g.nz;
    unsigned char *fac = b->d_kin + koff[i];
    double *ksq = (double *) (fac + (size_t) tot * esz);
    if (gb__kin_tables_at(fac, ksq, &it.g, &it.kin)) {
      gb_batch_free(b);
      return nullptr;
    }
    PassArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = 1;
    a.ny = it.g.ny;
    a.nz = it.g.nz;
    a.scale = 1.0;
    a.kscale = it.kin.scale;
    a.cutoff = it.kin.cutoff;
    a.kmax2 = it.kin.kmax2;
    a.kfac[0] = fac;
    a.kfac[1] = fac + esz;
    a.kfac[2] = fac + esz * (size_t) (1 + it.g.ny);
    a.ksq[0] = ksq;
    a.ksq[1] = ksq + 1;
    a.ksq[2] = ksq + 1 + it.g.ny;
    a.pot = it.pot;
    if (a.pot.kind == GB_POT_NONE && a.pot.g == 0.0 && a.pot.cons == 0.0) a.pot.c_re = a.pot.c_im = 0.0;
    BatchInst &bi = hi[i];
    bi.az = a;
    bi.az.axis = 2;
    bi.az.tw = gb__twiddles(it.g.nz, prec);
    bi.ay = a;
    bi.ay.axis = 1;
    bi.ay.tw = gb__twiddles(it.g.ny, prec);
    if (!bi.az.tw || !bi.ay.tw) {
      gb_batch_free(b);
      return nullptr;
    }
    bi.psi = it.psi;
    bi.nz = (int) it.g.nz;
    bi.ny = (int) it.g.ny;
  }
  cudaMemcpyAsync(b->d_inst, hi.data(), sizeof(BatchInst) * n, cudaMemcpyHostToDevice, st);
  // shape classes for the per-class plan
  {
    std::vector<BatchInst> ci;
    for (int sy = 64; sy <= 512; sy *= 2)
      for (int sz = 64; sz <= 512; sz *= 2) {
        const int off = (int) ci.size();
        for (int i = 0; i < n; i++)
          if (hi[i].ny == sy && hi[i].nz == sz) ci.push_back(hi[i]);
        if ((int) ci.size() > off) {
          b->cls_off[b->ncls] = off;
          b->cls_n[b->ncls] = (int) ci.size() - off;
          b->cls_ny[b->ncls] = sy;
          b->cls_nz[b->ncls] = sz;
          b->ncls++;
        }
      }
    if (cudaMalloc(&b->d_cinst, sizeof(BatchInst) * n) != cudaSuccess) {
      cudaGetLastError();
      gb__set_error(2, "batch: cudaMalloc");
      gb_batch_free(b);
      return nullptr;
    }
    cudaMemcpy(b->d_cinst, ci.data(), sizeof(BatchInst) * n, cudaMemcpyHostToDevice);
  }
  // tile lists for the CTA sizes
  for (int v = 0; v < 3; v++) {
    std::vector<BatchTile> ct, stl;
    for (int i = 0; i < n; i++) {
      const long nz = items[i].g.nz, ny = items[i].g.ny;
      const long tlz = batch_tl(nz), tly = batch_tl(ny);
      const long lz = kBatchThreads[v] / tlz, bzy = kBatchThreads[v] / tly;
      for (long k = 0; k < ny / lz; k++) ct.push_back(BatchTile{i, (int) k});
      for (long k = 0; k < nz / bzy; k++) stl.push_back(BatchTile{i, (int) k});
    }
    b->ntiles[v][0] = (int) ct.size();
    b->ntiles[v][1] = (int) stl.size();
    if (cudaMalloc(&b->d_tiles[v][0], sizeof(BatchTile) * ct.size()) != cudaSuccess ||
        cudaMalloc(&b->d_tiles[v][1], sizeof(BatchTile) * stl.size()) != cudaSuccess) {
      cudaGetLastError();
      gb__set_error(2, "batch: cudaMalloc");
      gb_batch_free(b);
      return nullptr;
    }
    cudaMemcpy(b->d_tiles[v][0], ct.data(), sizeof(BatchTile) * ct.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_tiles[v][1], stl.data(), sizeof(BatchTile) * stl.size(), cudaMemcpyHostToDevice);
  }
  b->grid[0] = prec == GB_FP32 ? batch_grid<float, 128>() : batch_grid<double, 128>();
  b->grid[1] = prec == GB_FP32 ? batch_grid<float, 256>() : batch_grid<double, 256>();
  b->grid[2] = prec == GB_FP32 ? batch_grid<float, 512>() : batch_grid<double, 512>();
  if (b->grid[0] <= 0 || b->grid[1] <= 0 || b->grid[2] <= 0) {
    gb__set_error(1042, "batch: kernel cannot be resident");
    gb_batch_free(b);
    return nullptr;
  }
  return b;
}

// The per-class plan: one step of every class on its own stream (forked from
// and joined back into the library stream), captured once as a graph.
template <typename T> static int batch_capture(gb_batch *b) {
  cudaStream_t main = gb__stream();
  if (!b->cls_st[0]) {
    for (int c = 0; c < b->ncls; c++) {
      cudaStreamCreateWithFlags(&b->cls_st[c], cudaStreamNonBlocking);
      cudaEventCreateWithFlags(&b->ev_join[c], cudaEventDisableTiming);
    }
    cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  }
  if (cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return gb__set_error(1043, "batch: stream capture");
  int rc = 0;
  cudaEventRecord(b->ev_fork, main);
  for (int c = 0; c < b->ncls && !rc; c++) {
    cudaStream_t sc = b->cls_st[c];
    cudaStreamWaitEvent(sc, b->ev_fork, 0);
    for (int ps = 0; ps < 5 && !rc; ps++)
      rc = bclass_pass<T>(ps, b->d_cinst + b->cls_off[c], b->cls_n[c], b->cls_ny[c], b->cls_nz[c], sc);
    cudaEventRecord(b->ev_join[c], sc);
    cudaStreamWaitEvent(main, b->ev_join[c], 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(main, &g);
  if (rc || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return rc ? rc : gb__set_error((int) e, "batch: stream capture");
  }
  const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return gb__set_error((int) ei, "batch: graph instantiate");
  return 0;
}

static int batch_run_classes(gb_batch *b, int steps) {
  if (!b->graph) GB_TRYC(b->prec == GB_FP32 ? batch_capture<float>(b) : batch_capture<double>(b));
  for (int s = 0; s < steps; s++) {
    const cudaError_t e = cudaGraphLaunch(b->graph, gb__stream());
    if (e != cudaSuccess) return gb__set_error((int) e, "batch: graph launch");
    for (int k = 0; k < 5 * b->ncls; k++) gb__count_launch();
  }
  return 0;
}

// Steps of every instance.  The first call with at least nine steps times
// one step of each plan (the persistent launch with 128, 256 and 512-thread
// CTAs, and the per-class graph), each after one warm-up step, and keeps
// the fastest; those eight steps count as steps of the run.  Every plan
// computes the same values.
extern "C" int gb_batch_step(gb_batch *b, int steps) {
  if (!b) return gb__set_error(1040, "batch: null");
  if (steps <= 0) return 0;
  if (!b->threads) {
    if (steps < 9) return batch_run(b, steps, 1);
    cudaEvent_t e[2];
    cudaEventCreate(&e[0]);
    cudaEventCreate(&e[1]);
    cudaStream_t st = gb__stream();
    float best = 0.f;
    int bv = 1;
    for (int v = 0; v < 4; v++) {
      GB_TRYC(v < 3 ? batch_run(b, 1, v) : batch_run_classes(b, 1));
      cudaEventRecord(e[0], st);
      GB_TRYC(v < 3 ? batch_run(b, 1, v) : batch_run_classes(b, 1));
      cudaEventRecord(e[1], st);
      cudaEventSynchronize(e[1]);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e[0], e[1]);
      if (v == 0 || ms < best) {
        best = ms;
        bv = v;
      }
    }
    cudaEventDestroy(e[0]);
    cudaEventDestroy(e[1]);
    b->threads = bv < 3 ? kBatchThreads[bv] : -1;
    steps -= 8;
  }
  if (b->threads < 0) return batch_run_classes(b, steps);
  return batch_run(b, steps, b->threads == 128 ? 0 : (b->threads == 256 ? 1 : 2));
}

extern "C" int gb_batch_threads(const gb_batch *b) { return b ? b->threads : 0; }

// The grid barrier's status word (shared by all batches on the library
// stream); reset != 0 clears it.
extern "C" int gb_batch_error_flag(gb_batch *b, int reset) {
  if (!b) return 0;
  return gb__status_word(GB_STATUS_BATCH, reset);
}

extern "C" void gb_batch_free(gb_batch *b) {
  if (!b) return;
  cudaStreamSynchronize(gb__stream());
  cudaFree(b->d_inst);
  for (int v = 0; v < 3; v++)
    for (int k = 0; k < 2; k++) cudaFree(b->d_tiles[v][k]);
  cudaFree(b->d_kin);
  cudaFree(b->d_bar);
  cudaFree(b->d_cinst);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (int c = 0; c < b->ncls; c++) {
    if (b->cls_st[c]) cudaStreamDestroy(b->cls_st[c]);
    if (b->ev_join[c]) cudaEventDestroy(b->ev_join[c]);
  }
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  free(b);
}
