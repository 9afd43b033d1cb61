// Tensor-core convolutions of the warm-start U-Net (sm_100a).
//
// Forward and data-gradient convolutions (tcgen05).  A 3x3x3 convolution
//   y[p][n] = sum_t sum_c B_t[n][c] x[p + off(t)][c]
// is a GEMM with M = output voxels, N = output channels and K = 27 taps x
// input channels.  It is run without an im2col matrix: a CTA stages a
// zero-padded halo block of the input in shared memory as bf16 channel-chunk
// planes [c8][position][8 channels] (16 bytes per position), and the A
// operand of tap t is the same plane read from a start address shifted by
// off(t) positions.  In the layout tcgen05.mma calls K-major without swizzle,
// eight consecutive positions form one 8 x 16-byte core matrix, so the shift
// needs no data movement.  Two K-chunks of 8 channels (two taps, or two
// channel chunks) make one K = 16 instruction; their distance is the
// descriptor's leading-byte offset.  M-tiles of 128 consecutive staged
// positions also cover the halo rows and pad columns; those rows compute
// values that are never stored, which costs tensor-core time the memory-bound
// layers have to spare.  The accumulators live in tensor memory (TMEM,
// 128 columns per CTA), are read back with tcgen05.ld by four warps (one per
// 32-lane quarter), and the epilogue adds the bias, applies the ReLU and
// stores FP32 outputs of the interior positions.  A CTA computes 16 output
// channels (N = 16); wider layers use one CTA per 16 channels of a block, so
// the weight operand of a CTA (27 taps x input channels x 16) always fits
// shared memory.  One thread issues the MMAs and commits them to an
// mbarrier; every wait is bounded.
//
// Weight gradient (mma.sync m16n8k16 bf16, FP32 accumulate):
//   gw[co][ci][t] += sum_q gy[co][q] x[ci][q + off(t)].
// A CTA stages gy of a voxel block (bf16, [co][q]) and three x-shifted copies
// of the x halo block (dx = -1, 0, 1, bf16, [ci][row][x]), so every tap's
// operand rows are 16-byte aligned for ldmatrix.  Warps split the taps.  A
// voxel block is tz x ty planes and rows of w >= 8 points (one kernel
// instance per shape, chosen on the host by estimated time); the staging
// issues eight loads per lane before any store, with rows of 8 or 16 points
// packed several to a warp.  A resident wave of CTAs loops over the voxel
// blocks (CTA b takes blocks b, b + grid, ...) with the accumulators in
// registers; each CTA's partial sums go to scratch and a fixed-order pass
// (one warp per weight, or one thread per weight when there are few
// partials) adds them to gw.  The bias gradient sums the
// unrounded FP32 gy in its own fixed-order kernel (deterministic, no
// atomics).
//
// Operands are rounded to bf16 (round to nearest even) and accumulated in
// FP32; the numpy oracle applies the same rounding.
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "gb_common.cuh"
#include "gb_internal_cuda.h"

namespace {

// ------------------------------------------------------------ tcgen05 helpers

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D(tmem) (+)= A(smem desc) x B(smem desc), kind::f16 (bf16 inputs, FP32 D)
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
// the MMAs issued so far by this thread arrive on bar when complete
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor, no swizzle (canonical K-major layout of
// 8-row x 16-byte core matrices): start address, leading-byte offset (next
// K-chunk), stride-byte offset (next 8-row group), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t) ((addr >> 4) & 0x3FFFu) | ((uint64_t) ((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t) ((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 D, bf16 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (n >> 3) << 17) | ((uint32_t) (m >> 4) << 24);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *(const uint32_t *) &h;
}

// ---------------------------------------------------------- forward (tcgen05)

constexpr int kTcThreads = 256;  // two warpgroups: staging, epilogue
constexpr int kTcM = 128;
constexpr int kTcN = 16;  // output channels per CTA
constexpr int kStageG = 4;  // staging items whose loads are issued together
constexpr int kTcMaxMma = 256;  // MMAs per M-tile (K = 27 taps x channels / 16)

struct TcConv {
  const float *x;     // [cx][d][h][w] FP32
  float *y;           // [ny][d][h][w] FP32
  const float *bias;  // [ny] or null
  const uint4 *bp;    // packed B: per 16-channel chunk, nmma * 4 core matrices
  int *err;
  int cx, ny;         // input channels (K side), output channels (N side)
  int d, h, w;        // d: all samples' planes (nb x dp)
  int dp;             // planes per sample (depth neighbours never cross samples)
  int relu;
  int tz, ty;         // output block: tz x ty x w voxels
  int c8, np, nmma;   // channel chunks, N per CTA (16), MMAs per M-tile
  int sy, sz;         // staged strides (positions)
  int guard;          // rows before position 0 of a plane
  int plane_rows;
  int ntile, tb;      // M-tiles per CTA, M-tiles per TMEM batch
  int ncols;          // allocated TMEM columns
};

// tap t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1): offset in staged positions
__device__ __forceinline__ int tap_off(int t, int sy, int sz) {
  return (t / 9 - 1) * sz + ((t / 3) % 3 - 1) * sy + (t % 3 - 1);
}

__global__ void __launch_bounds__(kTcThreads) k_conv3_tc(TcConv p) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nby = p.h / p.ty;
  const int z0 = (blockIdx.x / nby) * p.tz, y0 = (blockIdx.x % nby) * p.ty;
  const int n0 = blockIdx.y * kTcN;  // first output channel of this CTA
  const int zlo = (z0 / p.dp) * p.dp;  // first plane of this block's sample
  const long vol = (long) p.d * p.h * p.w;
  const uint32_t plane_bytes = (uint32_t) p.plane_rows * 16u;
  unsigned char *a_sm = smraw;
  unsigned char *b_sm = smraw + (size_t) p.c8 * plane_bytes;
  // A descriptor of MMA j for the first M-tile (m0 = sz): K-chunks 2j and
  // 2j + 1 (tap, channel chunk), their distance as the leading-byte offset
  __shared__ uint64_t s_ad[kTcMaxMma];
  {
    const uint32_t ab = smem_u32(a_sm);
    const int nkc = 27 * p.c8;
    for (int j = threadIdx.x; j < p.nmma; j += kTcThreads) {
      const int k1 = 2 * j, k2 = (2 * j + 1 < nkc) ? 2 * j + 1 : 2 * j;
      const uint32_t a1 =
          ab + (uint32_t) (k1 / 27) * plane_bytes + (uint32_t) (p.guard + p.sz + tap_off(k1 % 27, p.sy, p.sz)) * 16u;
      const uint32_t a2 =
          ab + (uint32_t) (k2 / 27) * plane_bytes + (uint32_t) (p.guard + p.sz + tap_off(k2 % 27, p.sy, p.sz)) * 16u;
      s_ad[j] = smem_desc(a1, a2 - a1, 128u);
    }
  }

  if (warp == 0) {
    tmem_alloc(&tslot, (uint32_t) p.ncols);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  // B operand (this channel chunk's packed weights) into shared memory
  const int nb16 = p.nmma * 2 * (kTcN / 8) * 8;  // 16-byte units
  const uint4 *bsrc = p.bp + (size_t) blockIdx.y * nb16;
  for (int i = tid; i < nb16; i += kTcThreads) ((uint4 *) b_sm)[i] = bsrc[i];
  // A operand: the zero-padded halo block, bf16 channel-chunk planes.  The
  // work items are (staged row, 32-position chunk of the row), lanes along
  // x; a warp takes every 8th item and issues the loads of kStageG items
  // (8 channels each) before packing and storing any of them, so that many
  // loads are in flight per lane instead of one row chunk at a time.
  {
    constexpr int G = kStageG, NW = kTcThreads / 32;
    const int rows_per_plane = (p.tz + 2) * (p.ty + 2);
    const int xch = (p.sy + 31) >> 5;
    const int nitems = p.c8 * rows_per_plane * xch;
    for (int i0 = warp; i0 < nitems; i0 += G * NW) {
      float v[G][8];
      int dpos[G];
#pragma unroll
      for (int g = 0; g < G; g++) {
        const int it = i0 + g * NW;
        dpos[g] = -1;
#pragma unroll
        for (int e = 0; e < 8; e++) v[g][e] = 0.f;
        if (it < nitems) {
          const int row = it / xch, xc = it - row * xch;
          const int c = row / rows_per_plane, rr = row - c * rows_per_plane;
          const int zs = rr / (p.ty + 2), ys = rr - zs * (p.ty + 2);
          const int xs = xc * 32 + lane;
          if (xs < p.sy) {
            dpos[g] = c * p.plane_rows + p.guard + zs * p.sz + ys * p.sy + xs;
            const int z = z0 + zs - 1, y = y0 + ys - 1, x = xs - 1;
            if (z >= zlo && z < zlo + p.dp && y >= 0 && y < p.h && x >= 0 && x < p.w) {
              const float *src = p.x + ((long) z * p.h + y) * p.w + x;
#pragma unroll
              for (int e = 0; e < 8; e++)
                if (c * 8 + e < p.cx) v[g][e] = __ldg(src + (size_t) (c * 8 + e) * vol);
            }
          }
        }
      }
#pragma unroll
      for (int g = 0; g < G; g++)
        if (dpos[g] >= 0)
          ((uint4 *) a_sm)[dpos[g]] = make_uint4(pack_bf16x2(v[g][0], v[g][1]), pack_bf16x2(v[g][2], v[g][3]),
                                                 pack_bf16x2(v[g][4], v[g][5]), pack_bf16x2(v[g][6], v[g][7]));
    }
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tslot;
  const uint32_t b_base = smem_u32(b_sm);
  const uint32_t idesc = idesc_bf16(kTcM, p.np);
  bool ok = true;

  for (int b0 = 0, batch = 0; b0 < p.ntile; b0 += p.tb, batch++) {
    const int nt = min(p.tb, p.ntile - b0);
    if (tid == 0) {
      // tile k of the batch starts (b0 + k) * kTcM positions (16-byte units)
      // after the first tile: added to the start-address field of the
      // tabled A descriptors (the sum stays inside shared memory, below the
      // field's 14-bit range); B of MMA j starts j * 2 * np units after B's
      const uint64_t bd0 = smem_desc(b_base, 16u * (uint32_t) p.np, 128u);
      for (int k = 0; k < nt; k++) {
        const uint64_t moff = (uint64_t) ((b0 + k) * kTcM);
        for (int j = 0; j < p.nmma; j++)
          tc_mma(tmem + (uint32_t) (k * p.np), s_ad[j] + moff, bd0 + (uint64_t) (j * 2 * p.np), idesc, j > 0 ? 1u : 0u);
      }
      tc_commit(&bar);
    }
    if (!mbar_wait_bounded(&bar, (unsigned) (batch & 1))) ok = false;
    if (__syncthreads_or(!ok)) break;
    tc_fence_after();
    // epilogue: warpgroup g takes tiles k = g, g + 2, ...; warp w reads TMEM
    // lanes 32 (w % 4) .. + 31 = those rows of a tile
    const int wq = warp & 3, wg = warp >> 2;
    for (int k = wg; k < nt; k += kTcThreads / 128) {
      const int pos = p.sz + (b0 + k) * kTcM + wq * 32 + lane;
      const int zs = pos / p.sz, rem = pos - zs * p.sz, ys = rem / p.sy, xs = rem - ys * p.sy;
      const bool useful = zs >= 1 && zs <= p.tz && ys >= 1 && ys <= p.ty && xs >= 1 && xs <= p.w;
      const long vox = ((long) (z0 + zs - 1) * p.h + (y0 + ys - 1)) * p.w + (xs - 1);
      for (int nb = 0; nb < p.np; nb += 16) {
        float v[16];
        tc_ld16(tmem + ((uint32_t) (wq * 32) << 16) + (uint32_t) (k * p.np + nb), v);
        if (useful) {
#pragma unroll
          for (int q = 0; q < 16; q++) {
            const int co = n0 + nb + q;
            if (co < p.ny) {
              float r = v[q] + (p.bias ? __ldg(p.bias + co) : 0.f);
              if (p.relu) r = fmaxf(r, 0.f);
              p.y[(size_t) co * vol + vox] = r;
            }
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (!ok) {
    // an MMA batch never completed: record it and let it drain (bounded)
    if (tid == 0) {
      atomicExch(p.err, 4);
      mbar_wait_bounded(&bar, 0);
      mbar_wait_bounded(&bar, 1);
    }
    tc_fence_before();
    __syncthreads();
  }
  if (warp == 0) tmem_dealloc(tmem, (uint32_t) p.ncols);
}

// Packed B operand, per chunk of 16 output channels nc: for MMA j and
// K-chunk h (chunk kc = 2 j + h, tap kc % 27, channel chunk kc / 27), the
// 16 x 8 block of weights as two core matrices of 8 rows (n) x 8 bf16
// (channels), [nc][j][h][ng][row][e].  mode 0 (forward): B_t[n][c] =
// w[n][c][t]; mode 1 (data gradient): B_t[n][c] = w[c][n][26 - t] with n an
// input channel and c an output channel of the layer.
__global__ void k_pack_b(const __nv_bfloat16 *__restrict__ w, __nv_bfloat16 *__restrict__ bp, int cin, int cout,
                         int nch, int c8, int nmma, int mode) {
  const long per = (long) nmma * 2 * kTcN * 8;  // elements per channel chunk
  const long total = per * nch;
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int nc = (int) (i / per);
  const long r0 = i - nc * per;
  const int e = (int) (r0 % 8), row = (int) ((r0 / 8) % 8);
  const long rest = r0 / 64;
  const int ng = (int) (rest % (kTcN / 8));
  const int kc = (int) (rest / (kTcN / 8));  // 2 j + h
  const int n = nc * kTcN + ng * 8 + row;
  __nv_bfloat16 v = __float2bfloat16_rn(0.f);
  if (kc < 27 * c8) {
    const int t = kc % 27, c = (kc / 27) * 8 + e;
    if (mode == 0) {
      if (n < cout && c < cin) v = w[((size_t) n * cin + c) * 27 + t];
    } else {
      if (n < cin && c < cout) v = w[((size_t) c * cin + n) * 27 + (26 - t)];
    }
  }
  bp[i] = v;
}

// ------------------------------------------------ weight gradient (mma.sync)

constexpr int kWgThreads = 256;  // 8 warps, warp w takes taps w, w + 8, ...
constexpr int kWgTaps = 4;       // ceil(27 / 8)
constexpr int kWgCo16 = 4;       // up to 64 output channels
constexpr int kWgItems = 8;      // staging items a warp loads before any store
constexpr int kWgReduceThreadParts = 64;  // up to this many partials: one thread per weight

struct TcWgrad {
  const float *x, *gy;
  float *part;  // [cta][cz][co][8][27] partial sums; bias partials [cta][co] after them
  int cin, cout, d, h, w;  // d: all samples' planes (nb x dp)
  int dp;                  // planes per sample
  int co16;     // output channels / 16, rounded up
  int nblk, ncz;
  int qp;       // gy row pitch (bf16)
  int xrp;      // x staged row pitch (bf16) = w
  int xpp;      // x staged plane pitch (bf16)
  int xcp;      // x staged copy pitch (bf16) = 8 * xpp
  int rpi;      // rows per staging item: 32 / w for w = 8 or 16, else 1
  int lgc;      // log2 of the 32-wide chunks per row (rpi == 1)
};

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2(uint32_t addr, uint32_t &r0, uint32_t &r1) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0, %1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Staging item it of a loop over rows of w points -> this lane's (row, x):
// rows of 32 or more points are split into 2^lgc chunks of 32 lanes; rows of
// 8 or 16 points are packed rpi = 32 / w to an item (lane = sub-row, x).
__device__ __forceinline__ void wg_item(int it, int rpi, int lgc, int lsub, int lx, int &row, int &x) {
  if (rpi > 1) {
    row = it * rpi + lsub;
    x = lx;
  } else {
    row = it >> lgc;
    x = ((it & ((1 << lgc) - 1)) << 5) + lx;
  }
}

// grid: (CTAs, input-channel chunks of 8); each CTA loops over the voxel
// blocks blockIdx.x, + gridDim.x, ... of TZ x TY x w points
template <int TZ, int TY>
__global__ void __launch_bounds__(kWgThreads, 2) k_conv3_wgrad_mma(TcWgrad p) {
  constexpr int BZ = TZ * TY, SY = TY + 2, SROWS = (TZ + 2) * SY, NW = kWgThreads / 32;
  extern __shared__ __align__(128) unsigned char smraw[];
  __nv_bfloat16 *gys = (__nv_bfloat16 *) smraw;                           // [16 co16][qp]
  __nv_bfloat16 *xs = gys + (size_t) 16 * p.co16 * p.qp;                   // [3][8][rows][w]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nby = p.h / TY;
  const int cz = blockIdx.y;
  const long vol = (long) p.d * p.h * p.w;
  const int nq = BZ * p.w;
  const int rpi = p.rpi, lgc = p.lgc;
  const int lsub = rpi > 1 ? lane / p.w : 0, lx = rpi > 1 ? lane - lsub * p.w : lane;
  // accumulators persist over the voxel blocks blockIdx.x, + gridDim.x, ...
  float acc[kWgTaps][kWgCo16][4];
#pragma unroll
  for (int a = 0; a < kWgTaps; a++)
#pragma unroll
    for (int b = 0; b < kWgCo16; b++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[a][b][c] = 0.f;
  for (int blk = blockIdx.x; blk < p.nblk; blk += gridDim.x) {
  const int z0 = (blk / nby) * TZ, y0 = (blk % nby) * TY;
  // gy of the block, bf16 [co][q] (rows past cout are zero), rows
  // (co, zi, yi).  A warp issues the loads of kWgItems items before any
  // store.  Rows of channels past cout are written by the CTA's first block
  // only.
  {
    const int nrows = (blk == (int) blockIdx.x ? 16 * p.co16 : p.cout) * BZ;
    const int nit = rpi > 1 ? (nrows + rpi - 1) / rpi : nrows << lgc;
    for (int i0 = warp; i0 < nit; i0 += kWgItems * NW) {
      float v[kWgItems];
      int off[kWgItems];
#pragma unroll
      for (int q = 0; q < kWgItems; q++) {
        int row, x;
        wg_item(i0 + q * NW, rpi, lgc, lsub, lx, row, x);
        const bool ok = i0 + q * NW < nit && row < nrows && x < p.w;
        const int co = row / BZ, rr = row - co * BZ, zi = rr / TY, yi = rr - zi * TY;
        v[q] = (ok && co < p.cout)
                   ? __ldg(p.gy + (size_t) co * vol + ((long) (z0 + zi) * p.h + (y0 + yi)) * p.w + x)
                   : 0.f;
        off[q] = ok ? co * p.qp + rr * p.w + x : -1;
      }
#pragma unroll
      for (int q = 0; q < kWgItems; q++)
        if (off[q] >= 0) gys[off[q]] = __float2bfloat16_rn(v[q]);
    }
  }
  // three x-shifted copies of the x halo block for this chunk of 8 channels:
  // copy cp holds x[. + cp - 1]; each input value is loaded once and stored
  // into the three copies.  Rows (c, zs, ys) of the (TZ + 2) x (TY + 2) halo;
  // a warp issues the loads of kWgItems items before any store.  off packs
  // the element's offset in a copy with two flags: x == 0 (bit 0) and
  // x == w - 1 (bit 1), where copies 0 and 2 take the zero padding.
  {
    const int nrows = 8 * SROWS;
    const int nit = rpi > 1 ? (nrows + rpi - 1) / rpi : nrows << lgc;
    const int zlo = (z0 / p.dp) * p.dp;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    for (int i0 = warp; i0 < nit; i0 += kWgItems * NW) {
      float v[kWgItems];
      int off[kWgItems];
#pragma unroll
      for (int q = 0; q < kWgItems; q++) {
        int row, x;
        wg_item(i0 + q * NW, rpi, lgc, lsub, lx, row, x);
        const bool ok = i0 + q * NW < nit && row < nrows && x < p.w;
        const int c = row / SROWS, r = row - c * SROWS, zs = r / SY, ys = r - zs * SY;
        const int z = z0 + zs - 1, y = y0 + ys - 1, ci = cz * 8 + c;
        const bool in = ok && ci < p.cin && z >= zlo && z < zlo + p.dp && y >= 0 && y < p.h;
        v[q] = in ? __ldg(p.x + (size_t) ci * vol + ((long) z * p.h + y) * p.w + x) : 0.f;
        off[q] = ok ? ((c * p.xpp + r * p.xrp + x) << 2) | (x == 0 ? 1 : 0) | (x == p.w - 1 ? 2 : 0) : -1;
      }
#pragma unroll
      for (int q = 0; q < kWgItems; q++) {
        if (off[q] < 0) continue;
        const int o = off[q] >> 2;
        const __nv_bfloat16 b = __float2bfloat16_rn(v[q]);
        xs[p.xcp + o] = b;                              // copy 1 at x
        if (!(off[q] & 2)) xs[o + 1] = b;               // copy 0 at x + 1
        else xs[2 * p.xcp + o] = zero;                  // copy 2 at w - 1: padding
        if (!(off[q] & 1)) xs[2 * p.xcp + o - 1] = b;   // copy 2 at x - 1
        else xs[o] = zero;                              // copy 0 at 0: padding
      }
    }
  }
  __syncthreads();
  const uint32_t gys_u = smem_u32(gys), xs_u = smem_u32(xs);
  // ldmatrix row addresses: A (x4) lanes 0-15 rows 0-15 at k 0, lanes 16-31
  // rows 0-15 at k 8; B (x2) lanes 0-7 rows (channels) at k 0, 8-15 at k 8.
  // The byte offsets that depend only on the lane and the warp's taps are
  // formed once per block; a q-step adds the staged position of the lane's
  // first B voxel, q0 + bcol, kept as (qx, qy, qz) and advanced by 16 voxels
  // per step (two rows when w = 8).
  const int arow = lane & 15, acol = (lane >> 4) * 8;
  const int bch = lane & 7, bcol = ((lane >> 3) & 1) * 8;
  const uint32_t a_lane = gys_u + (uint32_t) (arow * p.qp + acol) * 2u;
  uint32_t b_tap[kWgTaps];
#pragma unroll
  for (int k = 0; k < kWgTaps; k++) {
    const int t = min(warp + 8 * k, 26);
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    b_tap[k] = xs_u + (uint32_t) ((dx + 1) * p.xcp + bch * p.xpp + ((1 + dz) * SY + (1 + dy)) * p.xrp) * 2u;
  }
  int qx = bcol, qy = 0, qz = 0;
  while (qx >= p.w) {
    qx -= p.w;
    if (++qy == TY) { qy = 0; ++qz; }
  }
  for (int q0 = 0; q0 < nq; q0 += 16) {
    const uint32_t q_off = (uint32_t) ((qz * SY + qy) * p.xrp + qx) * 2u;
    uint32_t a[kWgCo16][4];
#pragma unroll
    for (int g = 0; g < kWgCo16; g++)
      if (g < p.co16)
        ldsm_x4(a_lane + (uint32_t) (g * 16 * p.qp + q0) * 2u, a[g][0], a[g][1], a[g][2], a[g][3]);
#pragma unroll
    for (int k = 0; k < kWgTaps; k++) {
      if (warp + 8 * k < 27) {
        uint32_t b0, b1;
        ldsm_x2(b_tap[k] + q_off, b0, b1);
#pragma unroll
        for (int g = 0; g < kWgCo16; g++)
          if (g < p.co16) mma_bf16(acc[k][g], a[g][0], a[g][1], a[g][2], a[g][3], b0, b1);
      }
    }
    qx += 16;
    while (qx >= p.w) {
      qx -= p.w;
      if (++qy == TY) { qy = 0; ++qz; }
    }
  }
  __syncthreads();  // the next block's staging overwrites the buffers
  }
  // partials: D[m = co][n = ci]; thread holds rows lane/4 (+8), columns 2 (lane%4) (+1)
  const size_t blkoff = ((size_t) blockIdx.x * p.ncz + cz) * (size_t) p.cout * 8 * 27;
#pragma unroll
  for (int k = 0; k < kWgTaps; k++) {
    const int t = warp + 8 * k;
    if (t >= 27) continue;
#pragma unroll
    for (int g = 0; g < kWgCo16; g++) {
      if (g >= p.co16) continue;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int co = g * 16 + (lane >> 2) + (c >> 1) * 8, n = 2 * (lane & 3) + (c & 1);
        if (co < p.cout) p.part[blkoff + ((size_t) co * 8 + n) * 27 + t] = acc[k][g][c];
      }
    }
  }
}

// Bias partials: pb[b][co] = sum of gy[co] over the b-th of nparts equal
// voxel ranges, unrounded FP32 in a fixed order (thread strides, then a
// fixed shuffle and warp tree), so every run gives the same sums.
__global__ void k_wgrad_bias_part(const float *__restrict__ gy, float *__restrict__ pb, int cout, long vol,
                                  int nparts) {
  const int b = blockIdx.x, co = blockIdx.y;
  const long lo = vol * b / nparts, hi = vol * (b + 1) / nparts;
  const float *g = gy + (size_t) co * vol;
  float s = 0.f;
  for (long i = lo + threadIdx.x; i < hi; i += blockDim.x) s += __ldg(g + i);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ float red[kWgThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < kWgThreads / 32; w++) t += red[w];
    pb[(size_t) b * cout + co] = t;
  }
}

// gw[co][ci][t] += sum over the CTAs' partials: one warp per weight, lanes
// take every 32nd partial in CTA order, then a fixed shuffle tree (the same
// sum on every run).
__global__ void k_wgrad_reduce(const float *__restrict__ part, float *__restrict__ gw, float *__restrict__ gbias,
                               int cin, int cout, int nparts, int ncz, int dobias) {
  const long nw = (long) cout * cin * 27;
  const long i = ((long) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  float s = 0.f;
  if (i < nw) {
    const int t = (int) (i % 27);
    const long rest = i / 27;
    const int ci = (int) (rest % cin), co = (int) (rest / cin);
    const int cz = ci / 8, n = ci % 8;
    for (int b = lane; b < nparts; b += 32) s += part[(((size_t) b * ncz + cz) * cout + co) * 8 * 27 + (size_t) n * 27 + t];
  } else if (dobias && i < nw + cout) {
    const int co = (int) (i - nw);
    const float *bp = part + (size_t) nparts * ncz * cout * 8 * 27;
    for (int b = lane; b < nparts; b += 32) s += bp[(size_t) b * cout + co];
  } else {
    return;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) {
    if (i < nw) gw[i] += s;
    else gbias[i - nw] += s;
  }
}

// The same sums with one thread per weight, for launches with few partials
// (the coarse levels' few CTAs): partials b = 0, 1, ... in order, so every
// run gives the same sum; consecutive threads read consecutive partials.
__global__ void k_wgrad_reduce_t(const float *__restrict__ part, float *__restrict__ gw, float *__restrict__ gbias,
                                 int cin, int cout, int nparts, int ncz, int dobias) {
  const long nw = (long) cout * cin * 27;
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  float s = 0.f;
  if (i < nw) {
    const int t = (int) (i % 27);
    const long rest = i / 27;
    const int ci = (int) (rest % cin), co = (int) (rest / cin);
    const int cz = ci / 8, n = ci % 8;
    const size_t stride = (size_t) ncz * cout * 8 * 27;
    const float *p0 = part + ((size_t) cz * cout + co) * 8 * 27 + (size_t) n * 27 + t;
#pragma unroll 8
    for (int b = 0; b < nparts; b++) s += __ldg(p0 + (size_t) b * stride);
    gw[i] += s;
  } else if (dobias && i < nw + cout) {
    const int co = (int) (i - nw);
    const float *bp = part + (size_t) nparts * ncz * cout * 8 * 27;
#pragma unroll 8
    for (int b = 0; b < nparts; b++) s += __ldg(bp + (size_t) b * cout + co);
    gbias[co] += s;
  }
}

// ------------------------------------------------------------------ host side

int g_tc_on = 1;

struct TcPlan {
  int tz, ty, c8, np, nch, nmma, sy, sz, guard, plane_rows, ntile, tb, ncols;
  size_t smem;
};

int pow2_at_least(int v) {
  int p = 32;
  while (p < v) p <<= 1;
  return p;
}

bool tc_plan(int cx, int ny, int d, int h, int w, TcPlan &pl) {
  pl.c8 = (cx + 7) / 8;
  pl.np = kTcN;
  pl.nch = (ny + kTcN - 1) / kTcN;
  pl.nmma = (27 * pl.c8 + 1) / 2;
  if (pl.nmma > kTcMaxMma) return false;
  const size_t bbytes = (size_t) pl.nmma * 32 * pl.np;
  const int cand[5][2] = {{4, 4}, {4, 2}, {2, 2}, {2, 1}, {1, 1}};
  for (auto &c : cand) {
    const int tz = c[0], ty = c[1];
    if (tz > d || ty > h || d % tz || h % ty) continue;
    const int sy = w + 2, sz = (ty + 2) * sy;
    const int guard = sy + 1;
    const int plane_rows = ((tz + 2) * sz + 2 * sy + 129 + 1) & ~1;
    const size_t smem = (size_t) pl.c8 * plane_rows * 16 + bbytes;
    if (smem > 200 * 1024) continue;
    pl.tz = tz;
    pl.ty = ty;
    pl.sy = sy;
    pl.sz = sz;
    pl.guard = guard;
    pl.plane_rows = plane_rows;
    pl.ntile = (tz * sz + kTcM - 1) / kTcM;
    pl.tb = std::max(1, std::min(pl.ntile, 128 / pl.np));
    pl.ncols = pow2_at_least(pl.tb * pl.np);
    // at least 57 KB of shared memory per CTA: at most four CTAs (4 x 128
    // TMEM columns) share an SM
    pl.smem = std::max(smem, (size_t) 57 * 1024);
    return true;
  }
  return false;
}

int run_conv_tc(const float *x, const uint16_t *w, const float *bias, float *y, int cin, int cout, int nb, int d, int h,
                int wd, int relu, int mode) {
  // mode 0: y[cout] = conv(x[cin]); mode 1: y = gx[cin] from x = gy[cout];
  // nb samples of d planes each, stacked along the depth axis
  const int cx = mode == 0 ? cin : cout, ny = mode == 0 ? cout : cin;
  TcPlan pl;
  if (!tc_plan(cx, ny, d, h, wd, pl)) return gb__set_error(1104, "unet tensor-core conv: no block plan fits");
  const size_t nbp = (size_t) pl.nmma * 2 * kTcN * 8 * pl.nch;  // bf16 elements
  __nv_bfloat16 *bp = (__nv_bfloat16 *) gb__scratch(GB_SCR_UNETB, nbp * sizeof(__nv_bfloat16));
  int *err = gb__status(GB_STATUS_PASS);
  if (!bp || !err) return gb_last_error();
  cudaStream_t st = gb__stream();
  k_pack_b<<<(unsigned) ((nbp + 255) / 256), 256, 0, st>>>((const __nv_bfloat16 *) w, bp, cin, cout, pl.nch, pl.c8,
                                                              pl.nmma, mode);
  GB_CHECK_LAUNCH("unet pack weights");
  TcConv p;
  p.x = x;
  p.y = y;
  p.bias = bias;
  p.bp = (const uint4 *) bp;
  p.err = err;
  p.cx = cx;
  p.ny = ny;
  p.d = nb * d;
  p.dp = d;
  p.h = h;
  p.w = wd;
  p.relu = relu;
  p.tz = pl.tz;
  p.ty = pl.ty;
  p.c8 = pl.c8;
  p.np = pl.np;
  p.nmma = pl.nmma;
  p.sy = pl.sy;
  p.sz = pl.sz;
  p.guard = pl.guard;
  p.plane_rows = pl.plane_rows;
  p.ntile = pl.ntile;
  p.tb = pl.tb;
  p.ncols = pl.ncols;
  static size_t attr = 0;
  if (pl.smem > attr) {
    cudaFuncSetAttribute(k_conv3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) (200 * 1024 + 1024));
    attr = 200 * 1024 + 1024;
  }
  const dim3 grid((unsigned) ((nb * d / pl.tz) * (h / pl.ty)), (unsigned) pl.nch);
  k_conv3_tc<<<grid, kTcThreads, pl.smem, st>>>(p);
  GB_CHECK_LAUNCH("unet tensor-core conv");
  return 0;
}

// Voxel block shapes of the weight gradient (tz x ty planes and rows of w
// points), one kernel instance each.
constexpr int kWgShapes[7][2] = {{4, 4}, {4, 2}, {2, 4}, {2, 2}, {2, 1}, {1, 2}, {1, 1}};

using WgKernel = void (*)(TcWgrad);
WgKernel wg_kernel(int s) {
  switch (s) {
    case 0: return k_conv3_wgrad_mma<4, 4>;
    case 1: return k_conv3_wgrad_mma<4, 2>;
    case 2: return k_conv3_wgrad_mma<2, 4>;
    case 3: return k_conv3_wgrad_mma<2, 2>;
    case 4: return k_conv3_wgrad_mma<2, 1>;
    case 5: return k_conv3_wgrad_mma<1, 2>;
    default: return k_conv3_wgrad_mma<1, 1>;
  }
}

size_t wg_smem(int co16, int tz, int ty, int wd) {
  const size_t qp = (size_t) tz * ty * wd + 8, xpp = (size_t) (tz + 2) * (ty + 2) * wd + 8;
  return (16 * co16 * qp + 3 * 8 * xpp) * 2;
}

// Block shape of the weight gradient: the one with the least estimated time
// per CTA, i.e. rounds of blocks (over the CTAs of one resident wave) times
// a block's staging passes (kWgItems items per warp) and MMA steps; shapes
// whose staging fits 108 KB run two CTAs per SM, up to 160 KB one.  -1 if
// none fits.
int wg_plan(int cin, int cout, int nb, int d, int h, int wd, int nsm, int rpi, int lgc) {
  const int co16 = (cout + 15) / 16, ncz = (cin + 7) / 8;
  int best = -1;
  double best_cost = 0;
  for (int s = 0; s < 7; s++) {
    const int tz = kWgShapes[s][0], ty = kWgShapes[s][1];
    if (tz > d || ty > h || d % tz || h % ty || (tz * ty * wd) % 16) continue;
    const size_t smem = wg_smem(co16, tz, ty, wd);
    if (smem > 160 * 1024) continue;
    const int per = smem <= 108 * 1024 ? 2 : 1;
    const long nctas = std::max(1, per * nsm / ncz);
    const long nblk = (long) (nb * d / tz) * (h / ty);
    const long rounds = (nblk + nctas - 1) / nctas;
    auto passes = [&](long rows) {
      const long items = rpi > 1 ? (rows + rpi - 1) / rpi : rows << lgc;
      return (double) ((items + kWgItems * 8 - 1) / (kWgItems * 8));
    };
    const double block = passes(8L * (tz + 2) * (ty + 2)) + passes((long) cout * tz * ty) +
                         0.15 * co16 * (tz * ty * wd / 16);
    const double cost = rounds * block;
    if (best < 0 || cost < best_cost) {
      best = s;
      best_cost = cost;
    }
  }
  return best;
}

int run_wgrad_mma(const float *x, const float *gy, float *gw, float *gbias, int cin, int cout, int nb, int d, int h,
                  int wd) {
  TcWgrad p;
  p.x = x;
  p.gy = gy;
  p.cin = cin;
  p.cout = cout;
  p.d = nb * d;
  p.dp = d;
  p.h = h;
  p.w = wd;
  p.co16 = (cout + 15) / 16;
  p.ncz = (cin + 7) / 8;
  p.rpi = (wd < 32 && 32 % wd == 0) ? 32 / wd : 1;
  p.lgc = 0;
  if (p.rpi == 1)
    while ((32 << p.lgc) < wd) p.lgc++;
  int nsm = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int s = wg_plan(cin, cout, nb, d, h, wd, nsm, p.rpi, p.lgc);
  if (s < 0) return gb__set_error(1105, "unet weight gradient: no block plan fits");
  const int tz = kWgShapes[s][0], ty = kWgShapes[s][1];
  p.qp = tz * ty * wd + 8;
  p.xrp = wd;
  p.xpp = (tz + 2) * (ty + 2) * wd + 8;
  p.xcp = 8 * p.xpp;
  const size_t smem = wg_smem(p.co16, tz, ty, wd);
  p.nblk = (nb * d / tz) * (h / ty);
  const WgKernel kern = wg_kernel(s);
  static bool attr[7] = {};
  if (!attr[s]) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    attr[s] = true;
  }
  // CTAs per channel chunk: one resident wave over all chunks (all CTAs of
  // the launch on the SMs at once), each CTA looping over its share of the
  // voxel blocks
  int per = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kWgThreads, smem) != cudaSuccess || per < 1) {
    cudaGetLastError();
    per = 1;
  }
  int nctas = per * nsm / p.ncz;
  if (nctas > p.nblk) nctas = p.nblk;
  if (nctas < 1) nctas = 1;
  const size_t nwp = (size_t) nctas * p.ncz * cout * 8 * 27;
  const size_t nparts = nwp + (gbias ? (size_t) nctas * cout : 0);
  p.part = (float *) gb__scratch(GB_SCR_UNET, nparts * sizeof(float));
  if (!p.part) return gb_last_error();
  cudaStream_t st = gb__stream();
  kern<<<dim3((unsigned) nctas, (unsigned) p.ncz), kWgThreads, smem, st>>>(p);
  GB_CHECK_LAUNCH("unet weight gradient");
  if (gbias) {
    k_wgrad_bias_part<<<dim3((unsigned) nctas, (unsigned) cout), kWgThreads, 0, st>>>(gy, p.part + nwp, cout,
                                                                                       (long) p.d * h * wd, nctas);
    GB_CHECK_LAUNCH("unet bias gradient partials");
  }
  const long nw = (long) cout * cin * 27 + (gbias ? cout : 0);
  if (nctas <= kWgReduceThreadParts)
    k_wgrad_reduce_t<<<(unsigned) ((nw + 255) / 256), 256, 0, st>>>(p.part, gw, gbias, cin, cout, nctas, p.ncz,
                                                                     gbias != nullptr);
  else
    k_wgrad_reduce<<<(unsigned) ((nw * 32 + 255) / 256), 256, 0, st>>>(p.part, gw, gbias, cin, cout, nctas, p.ncz,
                                                                         gbias != nullptr);
  GB_CHECK_LAUNCH("unet weight gradient reduce");
  return 0;
}

}  // namespace

// Tensor-core paths of the U-Net convolutions (1, the default) or the SIMT
// kernels (0); -1 only queries.
extern "C" int gb_unet_tensor_cores(int on) {
  const int old = g_tc_on;
  if (on >= 0) g_tc_on = on ? 1 : 0;
  return old;
}

// Entry points used by gb_unet.cu when the tensor-core path is on; return
// -1 when the shape has no tensor-core plan (the caller then runs SIMT).
int gb__unet_conv_tc(const float *x, const uint16_t *w, const float *b, float *y, int cin, int cout, int nb, int d,
                     int h, int wd, int relu, int mode) {
  if (!g_tc_on) return -1;
  TcPlan pl;
  if (!tc_plan(mode == 0 ? cin : cout, mode == 0 ? cout : cin, d, h, wd, pl)) return -1;
  return run_conv_tc(x, w, b, y, cin, cout, nb, d, h, wd, relu, mode);
}

int gb__unet_wgrad_tc(const float *x, const float *gy, float *gw, float *gb, int cin, int cout, int nb, int d, int h,
                      int wd) {
  if (!g_tc_on || cout > 16 * kWgCo16 || wd < 8 || wd % 8) return -1;
  int nsm = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int rpi = (wd < 32 && 32 % wd == 0) ? 32 / wd : 1;
  int lgc = 0;
  if (rpi == 1)
    while ((32 << lgc) < wd) lgc++;
  if (wg_plan(cin, cout, nb, d, h, wd, nsm, rpi, lgc) < 0) return -1;
  return run_wgrad_mma(x, gy, gw, gb, cin, cout, nb, d, h, wd);
}
