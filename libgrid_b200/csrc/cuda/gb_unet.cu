// Kernels of the learned warm start for imaginary-time ground states: a 3-D
// convolutional U-Net that maps an external potential (and the coupling g) to
// a guess of the ground-state amplitude.  Nothing here exists in the
// reference; the network only replaces the Gaussian initial guess of the
// caller-composed imaginary-time loop (propagate(-i dt) -> normalize -> energy
// every M steps).  The plain imaginary-time propagation still decides the
// converged state.
//
// Layout: activations FP32 [C][D][H][W]; the *_nb convolutions take nb
// samples stacked along the depth axis ([C][nb D][H][W], depth neighbours
// never crossing samples), and pooling, upsampling and the pointwise kernels
// take the stacked depth as it is; weights bf16
// [Cout][Cin][27] (3x3x3 taps, zero padding), FP32 master weights and FP32
// gradient accumulators [Cout][Cin][27] owned by the caller.  All
// accumulation is FP32 in a fixed order, so every kernel is deterministic.
// Weight gradients accumulate (+=) so that a minibatch is a sequence of
// backward calls followed by one gb_unet_adam, which clears them.
//
// These are SIMT kernels (one thread per output voxel and a group of output
// channels, the block's weight slice staged in shared memory as FP32).
#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>

#include "gb_common.cuh"
#include "gb_internal_cuda.h"

namespace {

constexpr int kThreads = 256;
constexpr int kCoGroup = 4;                      // output channels per thread (forward)
constexpr int kCiGroup = 4;                      // input channels per thread (data gradient)
constexpr int kSplit = 4;                        // channel-loop slices for small volumes
constexpr long kSplitVolume = 4096;              // volumes up to 16^3 use the sliced kernels
// Shared-memory budget for a weight slice: 48 KB less the slices' reduction buffer.
constexpr size_t kMaxStage = 48 * 1024 - kSplit * 4 * (kThreads / kSplit) * sizeof(float);

// S thread slices per voxel split the input-channel loop (ci = s, s + S, ...)
// and are summed in slice order through shared memory, so small volumes (the
// coarse levels: 4^3 to 16^3 voxels) still fill the SM.  S = 1 for large ones.
template <int S>
__global__ void __launch_bounds__(kThreads) k_conv3_fwd(const float *__restrict__ x, const __nv_bfloat16 *__restrict__ w,
                                                        const float *__restrict__ b, float *__restrict__ y, int cin,
                                                        int cout, int d, int h, int wd, int dp, int relu) {
  constexpr int VB = kThreads / S;  // voxels per block
  extern __shared__ float ws[];     // [kCoGroup][cin][27]
  const int co0 = blockIdx.y * kCoGroup;
  const int nco = min(kCoGroup, cout - co0);
  for (int i = threadIdx.x; i < nco * cin * 27; i += blockDim.x)
    ws[i] = __bfloat162float(w[(size_t) co0 * cin * 27 + i]);
  __syncthreads();
  const long vol = (long) d * h * wd;
  const int sl = threadIdx.x / VB, pl = threadIdx.x % VB;
  const long p = (long) blockIdx.x * VB + pl;
  const bool valid = p < vol;
  float acc[kCoGroup];
#pragma unroll
  for (int j = 0; j < kCoGroup; j++) acc[j] = 0.f;
  if (valid) {
    const int ix = (int) (p % wd), iy = (int) ((p / wd) % h), iz = (int) (p / ((long) wd * h));
    const int zl = iz % dp;  // plane within its sample
    for (int ci = sl; ci < cin; ci += S) {
      const float *xc = x + (size_t) ci * vol;
      const float *wc = ws + ci * 27;
      for (int dz = -1; dz <= 1; dz++) {
        const int z = iz + dz;
        if (zl + dz < 0 || zl + dz >= dp) continue;
        for (int dy = -1; dy <= 1; dy++) {
          const int yy = iy + dy;
          if (yy < 0 || yy >= h) continue;
          for (int dx = -1; dx <= 1; dx++) {
            const int xx = ix + dx;
            if (xx < 0 || xx >= wd) continue;
            const float v = xc[((long) z * h + yy) * wd + xx];
            const int t = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
#pragma unroll
            for (int j = 0; j < kCoGroup; j++)
              if (j < nco) acc[j] = fmaf(v, wc[(size_t) j * cin * 27 + t], acc[j]);
          }
        }
      }
    }
  }
  if constexpr (S > 1) {
    __shared__ float red[S][kCoGroup][VB];
#pragma unroll
    for (int j = 0; j < kCoGroup; j++) red[sl][j][pl] = acc[j];
    __syncthreads();
    if (sl != 0) return;
#pragma unroll
    for (int j = 0; j < kCoGroup; j++) {
      float t = red[0][j][pl];
      for (int k = 1; k < S; k++) t += red[k][j][pl];
      acc[j] = t;
    }
  }
  if (!valid) return;
#pragma unroll
  for (int j = 0; j < kCoGroup; j++) {
    if (j >= nco) break;
    float r = acc[j] + b[co0 + j];
    if (relu) r = fmaxf(r, 0.f);
    y[(size_t) (co0 + j) * vol + p] = r;
  }
}

// gx[ci][q] = sum_co sum_t gy[co][q - off(t)] * w[co][ci][t]; S slices split
// the output-channel loop as in the forward kernel.
template <int S>
__global__ void __launch_bounds__(kThreads) k_conv3_bwd_data(const float *__restrict__ gy,
                                                             const __nv_bfloat16 *__restrict__ w, float *__restrict__ gx,
                                                             int cin, int cout, int d, int h, int wd, int dp) {
  constexpr int VB = kThreads / S;
  extern __shared__ float ws[];  // [kCiGroup][cout][27]
  const int ci0 = blockIdx.y * kCiGroup;
  const int nci = min(kCiGroup, cin - ci0);
  for (int i = threadIdx.x; i < nci * cout * 27; i += blockDim.x) {
    const int j = i / (cout * 27), r = i % (cout * 27), co = r / 27, t = r % 27;
    ws[i] = __bfloat162float(w[((size_t) co * cin + ci0 + j) * 27 + t]);
  }
  __syncthreads();
  const long vol = (long) d * h * wd;
  const int sl = threadIdx.x / VB, pl = threadIdx.x % VB;
  const long q = (long) blockIdx.x * VB + pl;
  const bool valid = q < vol;
  float acc[kCiGroup];
#pragma unroll
  for (int j = 0; j < kCiGroup; j++) acc[j] = 0.f;
  if (valid) {
    const int ix = (int) (q % wd), iy = (int) ((q / wd) % h), iz = (int) (q / ((long) wd * h));
    const int zl = iz % dp;  // plane within its sample
    for (int co = sl; co < cout; co += S) {
      const float *gc = gy + (size_t) co * vol;
      const float *wc = ws + co * 27;
      for (int dz = -1; dz <= 1; dz++) {
        const int z = iz - dz;
        if (zl - dz < 0 || zl - dz >= dp) continue;
        for (int dy = -1; dy <= 1; dy++) {
          const int yy = iy - dy;
          if (yy < 0 || yy >= h) continue;
          for (int dx = -1; dx <= 1; dx++) {
            const int xx = ix - dx;
            if (xx < 0 || xx >= wd) continue;
            const float v = gc[((long) z * h + yy) * wd + xx];
            const int t = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
#pragma unroll
            for (int j = 0; j < kCiGroup; j++)
              if (j < nci) acc[j] = fmaf(v, wc[(size_t) j * cout * 27 + t], acc[j]);
          }
        }
      }
    }
  }
  if constexpr (S > 1) {
    __shared__ float red[S][kCiGroup][VB];
#pragma unroll
    for (int j = 0; j < kCiGroup; j++) red[sl][j][pl] = acc[j];
    __syncthreads();
    if (sl != 0) return;
#pragma unroll
    for (int j = 0; j < kCiGroup; j++) {
      float t = red[0][j][pl];
      for (int k = 1; k < S; k++) t += red[k][j][pl];
      acc[j] = t;
    }
  }
  if (!valid) return;
#pragma unroll
  for (int j = 0; j < kCiGroup; j++) {
    if (j >= nci) break;
    gx[(size_t) (ci0 + j) * vol + q] = acc[j];
  }
}

// Weight gradient dL/dw[co][ci][t] = sum_p gy[co][p] * x[ci][p + off(t)].
// One CTA per (ci, group of kWCo output channels, voxel chunk): each input
// load serves kWCo output channels.  With one chunk the CTA adds its sums to
// gw; with several it writes them to part[chunk][co][ci][27], and
// k_wgrad_finish adds the chunks to gw in chunk order (no atomics).
constexpr int kWThreads = 128;
constexpr int kWCo = 4;

__global__ void __launch_bounds__(kWThreads) k_conv3_bwd_weight(const float *__restrict__ x, const float *__restrict__ gy,
                                                                float *__restrict__ gw, float *__restrict__ gbias,
                                                                float *__restrict__ part, int cin, int cout, int d, int h,
                                                                int wd, int dp, long chunk, int nchunk) {
  __shared__ float red[kWThreads / 32][kWCo * 28];  // 27 taps, then the bias sum, per output channel
  const int ci = blockIdx.x, co0 = blockIdx.y * kWCo, c = blockIdx.z;
  const int nco = min(kWCo, cout - co0);
  const long vol = (long) d * h * wd;
  const long p0 = (long) c * chunk, p1 = min(vol, p0 + chunk);
  const float *xc = x + (size_t) ci * vol;
  const bool dob = gbias != nullptr && ci == 0;  // the ci = 0 CTAs also sum the bias gradient
  float acc[kWCo][27], bs[kWCo];
#pragma unroll
  for (int j = 0; j < kWCo; j++) {
    bs[j] = 0.f;
#pragma unroll
    for (int t = 0; t < 27; t++) acc[j][t] = 0.f;
  }
  for (long p = p0 + threadIdx.x; p < p1; p += kWThreads) {
    float g[kWCo];
#pragma unroll
    for (int j = 0; j < kWCo; j++) g[j] = (j < nco) ? gy[(size_t) (co0 + j) * vol + p] : 0.f;
    if (dob) {
#pragma unroll
      for (int j = 0; j < kWCo; j++) bs[j] += g[j];
    }
    const int ix = (int) (p % wd), iy = (int) ((p / wd) % h), iz = (int) (p / ((long) wd * h));
    const int zl = iz % dp;  // plane within its sample
#pragma unroll
    for (int t = 0; t < 27; t++) {
      const int z = iz + t / 9 - 1, yy = iy + (t / 3) % 3 - 1, xx = ix + t % 3 - 1;
      const bool in = zl + t / 9 - 1 >= 0 && zl + t / 9 - 1 < dp && yy >= 0 && yy < h && xx >= 0 && xx < wd;
      const float v = in ? xc[((long) z * h + yy) * wd + xx] : 0.f;
#pragma unroll
      for (int j = 0; j < kWCo; j++) acc[j][t] = fmaf(g[j], v, acc[j][t]);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < kWCo; j++)
#pragma unroll
    for (int t = 0; t < 27; t++) {
      float v = acc[j][t];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][j * 27 + t] = v;
    }
  if (dob) {
#pragma unroll
    for (int j = 0; j < kWCo; j++) {
      float v = bs[j];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][kWCo * 27 + j] = v;
    }
  }
  __syncthreads();
  const size_t nw = (size_t) cout * cin * 27;
  for (int i = threadIdx.x; i < nco * 27; i += kWThreads) {
    float s = 0.f;
    for (int k = 0; k < kWThreads / 32; k++) s += red[k][i];
    const int j = i / 27, t = i % 27;
    const size_t w = ((size_t) (co0 + j) * cin + ci) * 27 + t;
    if (part) part[(size_t) c * nw + w] = s;
    else gw[w] += s;
  }
  if (dob && threadIdx.x < nco) {
    float s = 0.f;
    for (int k = 0; k < kWThreads / 32; k++) s += red[k][kWCo * 27 + threadIdx.x];
    // bias partials follow the nchunk weight-partial blocks
    if (part) part[(size_t) nchunk * nw + (size_t) c * cout + co0 + threadIdx.x] = s;
    else gbias[co0 + threadIdx.x] += s;
  }
}

__global__ void k_wgrad_finish(const float *__restrict__ part, float *__restrict__ gw, long n, int nchunk) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int c = 0; c < nchunk; c++) s += part[(size_t) c * n + i];
  gw[i] += s;
}

__global__ void k_relu_bwd(float *__restrict__ gy, const float *__restrict__ y, long n) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !(y[i] > 0.f)) gy[i] = 0.f;
}

// Average over 2x2x2 blocks; d, h, wd are the input extents (even).  The
// gradient accumulates (gx +=): a pooled activation is also the skip input of
// the decoder, whose gradient is written first.
__global__ void k_pool2_fwd(const float *__restrict__ x, float *__restrict__ y, long n_out, int d, int h, int wd) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_out) return;
  const int ow = wd / 2, oh = h / 2, od = d / 2;
  const int ox = (int) (i % ow), oy = (int) ((i / ow) % oh), oz = (int) ((i / ((long) ow * oh)) % od);
  const long c = i / ((long) ow * oh * od);
  const float *xc = x + (size_t) c * d * h * wd;
  float s = 0.f;
  for (int k = 0; k < 8; k++) s += xc[((long) (2 * oz + (k >> 2)) * h + 2 * oy + ((k >> 1) & 1)) * wd + 2 * ox + (k & 1)];
  y[i] = 0.125f * s;
}

__global__ void k_pool2_bwd(const float *__restrict__ gy, float *__restrict__ gx, long n_in, int d, int h, int wd) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_in) return;
  const int ix = (int) (i % wd), iy = (int) ((i / wd) % h), iz = (int) ((i / ((long) wd * h)) % d);
  const long c = i / ((long) wd * h * d);
  const int ow = wd / 2, oh = h / 2, od = d / 2;
  gx[i] += 0.125f * gy[(((size_t) c * od + iz / 2) * oh + iy / 2) * ow + ix / 2];
}

// Nearest-neighbour doubling; d, h, wd are the input extents.
__global__ void k_up2_fwd(const float *__restrict__ x, float *__restrict__ y, long n_out, int d, int h, int wd) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_out) return;
  const int W = 2 * wd, H = 2 * h, D = 2 * d;
  const int X = (int) (i % W), Y = (int) ((i / W) % H), Z = (int) ((i / ((long) W * H)) % D);
  const long c = i / ((long) W * H * D);
  y[i] = x[(((size_t) c * d + Z / 2) * h + Y / 2) * wd + X / 2];
}

__global__ void k_up2_bwd(const float *__restrict__ gy, float *__restrict__ gx, long n_in, int d, int h, int wd) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_in) return;
  const int ix = (int) (i % wd), iy = (int) ((i / wd) % h), iz = (int) ((i / ((long) wd * h)) % d);
  const long c = i / ((long) wd * h * d);
  const int W = 2 * wd, H = 2 * h, D = 2 * d;
  const float *gc = gy + (size_t) c * D * H * W;
  float s = 0.f;
  for (int k = 0; k < 8; k++) s += gc[((long) (2 * iz + (k >> 2)) * H + 2 * iy + ((k >> 1) & 1)) * W + 2 * ix + (k & 1)];
  gx[i] = s;
}

__global__ void k_mse_grad(const float *__restrict__ pred, const float *__restrict__ tgt, float *__restrict__ grad, long n,
                           float scale) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) grad[i] = scale * (pred[i] - tgt[i]);
}

// Adam on FP32 master weights; writes the bf16 copy and clears the gradient.
// c1 = 1/(1-b1^t), c2 = 1/(1-b2^t).
__global__ void k_adam(float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, float *__restrict__ m, float *__restrict__ v,
                       float *__restrict__ g, long n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
  g[i] = 0.f;
}

__global__ void k_to_bf16(const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, long n) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

__global__ void k_fill(float *__restrict__ p, long n, float v) {
  const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// ---- warm-start inputs and guesses, built on the device

// V = k r^2 / 2 + sum_b a_b exp(-|r - c_b|^2 / w_b^2) on the grid
// x_i = (i - n/2) step (padded real rows of vrow).
__global__ void k_unet_potential(double *__restrict__ v, int nx, int ny, int nz, long vrow, double step, double k,
                                 gb_unet_bumps bm) {
  const long n = (long) nx * ny * nz;
  for (long i = (long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x) {
    const int iz = (int) (i % nz), iy = (int) ((i / nz) % ny), ix = (int) (i / ((long) nz * ny));
    const double x = (ix - nx / 2) * step, y = (iy - ny / 2) * step, z = (iz - nz / 2) * step;
    double s = 0.5 * k * (x * x + y * y + z * z);
    for (int b = 0; b < bm.n; b++) {
      const double dx = x - bm.c[b][0], dy = y - bm.c[b][1], dz = z - bm.c[b][2];
      s += bm.amp[b] * exp(-(dx * dx + dy * dy + dz * dz) / (bm.w[b] * bm.w[b]));
    }
    v[((long) ix * ny + iy) * vrow + iz] = s;
  }
}

// Network input [3][n]: tanh((V - vmin) / vscale), the constant gfeat, and
// the Thomas-Fermi amplitude sqrt(max(mu - V, 0) / g) / amax.
__global__ void k_unet_features(const double *__restrict__ v, int nx, int ny, int nz, long vrow, double vmin,
                                double vscale, float gfeat, double mu, double g, double amax, float *__restrict__ out) {
  const long n = (long) nx * ny * nz;
  for (long i = (long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x) {
    const long ij = i / nz, k = i - ij * nz;
    const double x = v[ij * vrow + k];
    out[i] = (float) tanh((x - vmin) / vscale);
    out[n + i] = gfeat;
    out[2 * n + i] = (float) (sqrt(fmax(mu - x, 0.0) / g) / amax);
  }
}

// psi = max(amp * scale, 0) + floor (real), into a complex grid
template <typename T>
__global__ void k_unet_amplitude(const float *__restrict__ amp, float scale, float floor, C2<T> *__restrict__ psi,
                                 long n) {
  for (long i = (long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x)
    psi[i] = C2<T>{(T) (fmaxf(amp[i] * scale, 0.f) + floor), (T) 0};
}

// out = |psi| * inv_scale (a training target from a complex grid)
template <typename T>
__global__ void k_unet_abs(const C2<T> *__restrict__ psi, float inv_scale, float *__restrict__ out, long n) {
  for (long i = (long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x) {
    const C2<T> v = psi[i];
    out[i] = (float) sqrt((double) v.x * v.x + (double) v.y * v.y) * inv_scale;
  }
}

// a Gaussian exp(-r^2 / width^2) amplitude
__global__ void k_unet_gaussian(float *__restrict__ out, int nx, int ny, int nz, double step, double width) {
  const long n = (long) nx * ny * nz;
  for (long i = (long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x) {
    const int iz = (int) (i % nz), iy = (int) ((i / nz) % ny), ix = (int) (i / ((long) nz * ny));
    const double x = (ix - nx / 2) * step, y = (iy - ny / 2) * step, z = (iz - nz / 2) * step;
    out[i] = (float) exp(-(x * x + y * y + z * z) / (width * width));
  }
}

inline unsigned blocks_for(long n) { return (unsigned) ((n + kThreads - 1) / kThreads); }
inline unsigned grid_for(long n) { return (unsigned) std::min<long>((n + kThreads - 1) / kThreads, 148L * 16); }

inline int shape_ok(const char *where, long a, long b, long c, long d) {
  if (a <= 0 || b <= 0 || c <= 0 || d <= 0) return gb__set_error(1101, where);
  return 0;
}

}  // namespace

extern "C" int gb_unet_conv3_fwd_nb(const float *x, const uint16_t *w, const float *b, float *y, int cin, int cout, int nb,
                                    int d, int h, int wd, int relu) {
  if (shape_ok("gb_unet_conv3_fwd: bad shape", cin, cout, (long) nb * d * h, wd)) return 1101;
  const int tc = gb__unet_conv_tc(x, w, b, y, cin, cout, nb, d, h, wd, relu, 0);
  if (tc >= 0) return tc;
  const size_t smem = (size_t) kCoGroup * cin * 27 * sizeof(float);
  if (smem > kMaxStage) return gb__set_error(1102, "gb_unet_conv3_fwd: too many input channels for the weight stage");
  const int dt = nb * d;  // all samples' planes
  const long vol = (long) dt * h * wd;
  const unsigned gy = (cout + kCoGroup - 1) / kCoGroup;
  if (vol <= kSplitVolume)
    k_conv3_fwd<kSplit><<<dim3((unsigned) ((vol + kThreads / kSplit - 1) / (kThreads / kSplit)), gy), kThreads, smem,
                          gb__stream()>>>(x, (const __nv_bfloat16 *) w, b, y, cin, cout, dt, h, wd, d, relu);
  else
    k_conv3_fwd<1><<<dim3(blocks_for(vol), gy), kThreads, smem, gb__stream()>>>(x, (const __nv_bfloat16 *) w, b, y, cin,
                                                                               cout, dt, h, wd, d, relu);
  GB_CHECK_LAUNCH("gb_unet_conv3_fwd");
  return 0;
}

extern "C" int gb_unet_conv3_fwd(const float *x, const uint16_t *w, const float *b, float *y, int cin, int cout, int d,
                                 int h, int wd, int relu) {
  return gb_unet_conv3_fwd_nb(x, w, b, y, cin, cout, 1, d, h, wd, relu);
}

extern "C" int gb_unet_conv3_bwd_data_nb(const float *gy, const uint16_t *w, float *gx, int cin, int cout, int nb, int d,
                                         int h, int wd) {
  if (shape_ok("gb_unet_conv3_bwd_data: bad shape", cin, cout, (long) nb * d * h, wd)) return 1101;
  const int tc = gb__unet_conv_tc(gy, w, nullptr, gx, cin, cout, nb, d, h, wd, 0, 1);
  if (tc >= 0) return tc;
  const size_t smem = (size_t) kCiGroup * cout * 27 * sizeof(float);
  if (smem > kMaxStage) return gb__set_error(1102, "gb_unet_conv3_bwd_data: too many output channels for the weight stage");
  const int dt = nb * d;
  const long vol = (long) dt * h * wd;
  const unsigned gyd = (cin + kCiGroup - 1) / kCiGroup;
  if (vol <= kSplitVolume)
    k_conv3_bwd_data<kSplit><<<dim3((unsigned) ((vol + kThreads / kSplit - 1) / (kThreads / kSplit)), gyd), kThreads,
                               smem, gb__stream()>>>(gy, (const __nv_bfloat16 *) w, gx, cin, cout, dt, h, wd, d);
  else
    k_conv3_bwd_data<1><<<dim3(blocks_for(vol), gyd), kThreads, smem, gb__stream()>>>(gy, (const __nv_bfloat16 *) w, gx,
                                                                                     cin, cout, dt, h, wd, d);
  GB_CHECK_LAUNCH("gb_unet_conv3_bwd_data");
  return 0;
}

extern "C" int gb_unet_conv3_bwd_data(const float *gy, const uint16_t *w, float *gx, int cin, int cout, int d, int h,
                                      int wd) {
  return gb_unet_conv3_bwd_data_nb(gy, w, gx, cin, cout, 1, d, h, wd);
}

extern "C" int gb_unet_conv3_bwd_weight_nb(const float *x, const float *gy, float *gw, float *gb, int cin, int cout,
                                           int nb, int d, int h, int wd) {
  if (shape_ok("gb_unet_conv3_bwd_weight: bad shape", cin, cout, (long) nb * d * h, wd)) return 1101;
  const int tc = gb__unet_wgrad_tc(x, gy, gw, gb, cin, cout, nb, d, h, wd);
  if (tc >= 0) return tc;
  const int dt = nb * d;
  const long vol = (long) dt * h * wd;
  // Voxel chunks of at least 2048 (at most 16 chunks): enough CTAs at 32^3,
  // one chunk (no partials) at 8^3 and below.
  const int nchunk = (int) std::min<long>(16, std::max<long>(1, vol / 2048));
  const long chunk = (vol + nchunk - 1) / nchunk;
  float *part = nullptr;
  const long nw = (long) cout * cin * 27;
  if (nchunk > 1) {
    part = (float *) gb__scratch(GB_SCR_UNET, (size_t) nchunk * (nw + cout) * sizeof(float));
    if (!part) return gb_last_error();
  }
  k_conv3_bwd_weight<<<dim3(cin, (cout + kWCo - 1) / kWCo, nchunk), kWThreads, 0, gb__stream()>>>(x, gy, gw, gb, part, cin,
                                                                                               cout, dt, h, wd, d, chunk,
                                                                                               nchunk);
  GB_CHECK_LAUNCH("gb_unet_conv3_bwd_weight");
  if (part) {
    k_wgrad_finish<<<blocks_for(nw), kThreads, 0, gb__stream()>>>(part, gw, nw, nchunk);
    GB_CHECK_LAUNCH("gb_unet_conv3_bwd_weight finish");
    if (gb) {
      k_wgrad_finish<<<blocks_for(cout), kThreads, 0, gb__stream()>>>(part + (size_t) nchunk * nw, gb, cout, nchunk);
      GB_CHECK_LAUNCH("gb_unet_conv3_bwd_bias finish");
    }
  }
  return 0;
}

extern "C" int gb_unet_conv3_bwd_weight(const float *x, const float *gy, float *gw, float *gb, int cin, int cout, int d,
                                        int h, int wd) {
  return gb_unet_conv3_bwd_weight_nb(x, gy, gw, gb, cin, cout, 1, d, h, wd);
}

extern "C" int gb_unet_relu_bwd(float *gy, const float *y, long n) {
  if (n <= 0) return 0;
  k_relu_bwd<<<blocks_for(n), kThreads, 0, gb__stream()>>>(gy, y, n);
  GB_CHECK_LAUNCH("gb_unet_relu_bwd");
  return 0;
}

extern "C" int gb_unet_pool2_fwd(const float *x, float *y, int c, int d, int h, int wd) {
  if (shape_ok("gb_unet_pool2_fwd: bad shape", c, d, h, wd) || (d | h | wd) & 1)
    return gb__set_error(1103, "gb_unet_pool2_fwd: extents must be positive and even");
  const long n = (long) c * (d / 2) * (h / 2) * (wd / 2);
  k_pool2_fwd<<<blocks_for(n), kThreads, 0, gb__stream()>>>(x, y, n, d, h, wd);
  GB_CHECK_LAUNCH("gb_unet_pool2_fwd");
  return 0;
}

extern "C" int gb_unet_pool2_bwd(const float *gy, float *gx, int c, int d, int h, int wd) {
  if (shape_ok("gb_unet_pool2_bwd: bad shape", c, d, h, wd) || (d | h | wd) & 1)
    return gb__set_error(1103, "gb_unet_pool2_bwd: extents must be positive and even");
  const long n = (long) c * d * h * wd;
  k_pool2_bwd<<<blocks_for(n), kThreads, 0, gb__stream()>>>(gy, gx, n, d, h, wd);
  GB_CHECK_LAUNCH("gb_unet_pool2_bwd");
  return 0;
}

extern "C" int gb_unet_up2_fwd(const float *x, float *y, int c, int d, int h, int wd) {
  if (shape_ok("gb_unet_up2_fwd: bad shape", c, d, h, wd)) return 1101;
  const long n = 8L * c * d * h * wd;
  k_up2_fwd<<<blocks_for(n), kThreads, 0, gb__stream()>>>(x, y, n, d, h, wd);
  GB_CHECK_LAUNCH("gb_unet_up2_fwd");
  return 0;
}

extern "C" int gb_unet_up2_bwd(const float *gy, float *gx, int c, int d, int h, int wd) {
  if (shape_ok("gb_unet_up2_bwd: bad shape", c, d, h, wd)) return 1101;
  const long n = (long) c * d * h * wd;
  k_up2_bwd<<<blocks_for(n), kThreads, 0, gb__stream()>>>(gy, gx, n, d, h, wd);
  GB_CHECK_LAUNCH("gb_unet_up2_bwd");
  return 0;
}

extern "C" int gb_unet_mse_grad(const float *pred, const float *tgt, float *grad, long n, float scale) {
  if (n <= 0) return 0;
  k_mse_grad<<<blocks_for(n), kThreads, 0, gb__stream()>>>(pred, tgt, grad, n, scale);
  GB_CHECK_LAUNCH("gb_unet_mse_grad");
  return 0;
}

extern "C" int gb_unet_adam(float *w, uint16_t *wb, float *m, float *v, float *g, long n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  if (n <= 0) return 0;
  k_adam<<<blocks_for(n), kThreads, 0, gb__stream()>>>(w, (__nv_bfloat16 *) wb, m, v, g, n, lr, b1, b2, eps, c1, c2);
  GB_CHECK_LAUNCH("gb_unet_adam");
  return 0;
}

extern "C" int gb_unet_to_bf16(const float *w, uint16_t *wb, long n) {
  if (n <= 0) return 0;
  k_to_bf16<<<blocks_for(n), kThreads, 0, gb__stream()>>>(w, (__nv_bfloat16 *) wb, n);
  GB_CHECK_LAUNCH("gb_unet_to_bf16");
  return 0;
}

extern "C" int gb_unet_fill(float *p, long n, float v) {
  if (n <= 0) return 0;
  k_fill<<<blocks_for(n), kThreads, 0, gb__stream()>>>(p, n, v);
  GB_CHECK_LAUNCH("gb_unet_fill");
  return 0;
}

// Minibatch gather: slot b of a batch-nb network's input ([cin][nb][vol])
// and target ([nb][vol]) from sample ix.i[b] of a device-resident set
// (inputs [N][cin][vol], targets [N][vol]); blockIdx.y = channel (cin: the
// target), blockIdx.z = slot.
struct GatherIdx {
  int i[GB_UNET_MAX_GATHER];
};

__global__ void k_gather(float *__restrict__ in, float *__restrict__ tgt, const float *__restrict__ xs,
                         const float *__restrict__ ys, GatherIdx ix, int cin, long vol, int nb) {
  const int c = blockIdx.y, b = blockIdx.z;
  const long s = ix.i[b];
  const float *src = c < cin ? xs + (s * cin + c) * vol : ys + s * vol;
  float *dst = c < cin ? in + ((long) c * nb + b) * vol : tgt + (long) b * vol;
  for (long k = (long) blockIdx.x * blockDim.x + threadIdx.x; k < vol; k += (long) gridDim.x * blockDim.x)
    dst[k] = __ldg(src + k);
}

extern "C" int gb_unet_gather(float *in, float *tgt, const float *xs, const float *ys, const int *idx, int count,
                              int cin, long vol, int nb, long nset) {
  if (count < 1 || count > GB_UNET_MAX_GATHER || count > nb || cin < 1 || vol < 1 || !idx)
    return gb__set_error(1101, "gb_unet_gather: bad count or shape");
  GatherIdx ix;
  for (int b = 0; b < count; b++) {
    if (idx[b] < 0 || idx[b] >= nset) return gb__set_error(1101, "gb_unet_gather: sample index out of range");
    ix.i[b] = idx[b];
  }
  const unsigned gx = (unsigned) std::min<long>((vol + kThreads - 1) / kThreads, 256);
  k_gather<<<dim3(gx, (unsigned) cin + 1, (unsigned) count), kThreads, 0, gb__stream()>>>(in, tgt, xs, ys, ix, cin,
                                                                                        vol, nb);
  GB_CHECK_LAUNCH("gb_unet_gather");
  return 0;
}

extern "C" int gb_unet_potential(double *v, int nx, int ny, int nz, long vrow, double step, double k,
                                 const gb_unet_bumps *bumps) {
  if (shape_ok("gb_unet_potential: bad shape", nx, ny, nz, vrow) || bumps->n < 0 || bumps->n > GB_UNET_MAX_BUMPS)
    return gb__set_error(1101, "gb_unet_potential: bad shape or bump count");
  k_unet_potential<<<grid_for((long) nx * ny * nz), kThreads, 0, gb__stream()>>>(v, nx, ny, nz, vrow, step, k, *bumps);
  GB_CHECK_LAUNCH("gb_unet_potential");
  return 0;
}

extern "C" int gb_unet_features(const double *v, int nx, int ny, int nz, long vrow, double vmin, double vscale,
                                float gfeat, double mu, double g, double amax, float *out) {
  if (shape_ok("gb_unet_features: bad shape", nx, ny, nz, vrow)) return 1101;
  k_unet_features<<<grid_for((long) nx * ny * nz), kThreads, 0, gb__stream()>>>(v, nx, ny, nz, vrow, vmin, vscale, gfeat,
                                                                                mu, g, amax, out);
  GB_CHECK_LAUNCH("gb_unet_features");
  return 0;
}

extern "C" int gb_unet_amplitude(const float *amp, float scale, float floor, void *psi, long n, int prec) {
  if (n <= 0) return 0;
  if (prec == GB_FP32)
    k_unet_amplitude<float><<<grid_for(n), kThreads, 0, gb__stream()>>>(amp, scale, floor, (float2 *) psi, n);
  else
    k_unet_amplitude<double><<<grid_for(n), kThreads, 0, gb__stream()>>>(amp, scale, floor, (double2 *) psi, n);
  GB_CHECK_LAUNCH("gb_unet_amplitude");
  return 0;
}

extern "C" int gb_unet_gaussian(float *out, int nx, int ny, int nz, double step, double width) {
  if (shape_ok("gb_unet_gaussian: bad shape", nx, ny, nz, 1)) return 1101;
  k_unet_gaussian<<<grid_for((long) nx * ny * nz), kThreads, 0, gb__stream()>>>(out, nx, ny, nz, step, width);
  GB_CHECK_LAUNCH("gb_unet_gaussian");
  return 0;
}

extern "C" int gb_unet_abs(const void *psi, int prec, long n, float inv_scale, float *out) {
  if (n <= 0) return 0;
  if (prec == GB_FP32)
    k_unet_abs<float><<<grid_for(n), kThreads, 0, gb__stream()>>>((const float2 *) psi, inv_scale, out, n);
  else
    k_unet_abs<double><<<grid_for(n), kThreads, 0, gb__stream()>>>((const double2 *) psi, inv_scale, out, n);
  GB_CHECK_LAUNCH("gb_unet_abs");
  return 0;
}
