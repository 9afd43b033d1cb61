/*
 * libgrid-b200 CUDA layer: the thin C ABI between the C host library and the
 * sm_100a kernels.  Plain pointers, sizes and plain-old-data parameter
 * structs only.  Every call is stream-ordered on the library's single CUDA
 * stream and returns 0 on success or a nonzero error code (also latched in
 * gb_last_error()).  Device pointers refer to the library's device-resident
 * grids; the C host layer (libgrid API) maps host grids onto them.
 *
 * These entry points replace the reference's CUDA dispatch layer, whose
 * wrappers return 0 (done on the GPU) or -1 (fall back to the CPU): here there
 * is no fallback, so any nonzero status is an error.  Each declaration cites
 * the reference wrapper or kernel it replaces.
 */
#ifndef LIBGRID_B200_GB_CUDA_H
#define LIBGRID_B200_GB_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Device arithmetic of a device buffer. */
#define GB_FP64 0 /* complex128 / float64 storage */
#define GB_FP32 1 /* complex64 / float32 storage */

/* Grid geometry (row-major, z fastest; reference src/cgrid.c:4-7). */
typedef struct {
  long nx, ny, nz;
  double step;
  int prec; /* GB_FP64 or GB_FP32 */
} gb_geom;

/*
 * Kinetic factor: psi_k *= scale * exp(tm * |k - k0|^2), zeroed where
 * |k - k0|^2 >= kmax2 when cutoff != 0.  k_i = 2 pi (i or i - n) / (n step)
 * with i <= n/2 non-negative (reference src/grid_wf_fft.c:141-193 and the
 * cutoff variant :206-262).
 */
typedef struct {
  double tm_re, tm_im;
  double kx0, ky0, kz0;
  double scale;
  double kmax2;
  int cutoff;
} gb_kinetic;

/* Potential kinds. */
#define GB_POT_NONE 0
#define GB_POT_COMPLEX 1 /* complex grid, rows of nz (16 B/pt in FP64) */
#define GB_POT_REAL 2    /* real grid, padded rows of vrow = nz2 (8 B/pt) */

/*
 * Potential factor: psi *= exp(c * (cons + V + g |psi|^2)) with c complex
 * (reference src/grid_wf.c:569-600: c = -i tstep / hbar).  When absorb != 0
 * the time step becomes position dependent as in src/grid_wf.c:593-595 with
 * the ramp of grid_wf_absorb (src/grid_wf.c:185-203):
 *   c = -i ((1 - a) Re(tstep) - i Re(tstep) a) / hbar.
 */
typedef struct {
  int kind;
  const void *v; /* device pointer, or NULL for kind == GB_POT_NONE */
  long vrow;     /* elements per (i, j) row of v */
  double c_re, c_im;
  double cons;
  double g;
  int absorb;
  long lx, hx, ly, hy, lz, hz;
  double treal; /* Re(tstep) / hbar, used when absorb != 0 */
} gb_potential;

/* ------------------------------------------------------------- runtime */
int gb_init(int device);
int gb_shutdown(void);
int gb_last_error(void);
const char *gb_last_error_where(void);
void gb_clear_error(void);
int gb_synchronize(void);
void *gb_stream_handle(void);
long gb_launch_count(void);
/* CUDA graphs of library calls (no reference counterpart): gb_graph_begin
 * captures the library stream, so the kernels the following calls issue are
 * recorded instead of run; gb_graph_end instantiates them (*graph receives a
 * handle); gb_graph_launch replays them on the library stream with the same
 * arguments and pointers; gb_graph_free releases the handle.  Captured calls
 * must not read results back to the host; run the same calls once without
 * capture first, so that scratch buffers already have their size. */
int gb_graph_begin(void);
int gb_graph_end(void **graph);
int gb_graph_launch(void *graph);
int gb_graph_free(void *graph);
void *gb_device_alloc(size_t bytes);
void gb_device_free(void *p);
void *gb_host_alloc(size_t bytes); /* page-locked when possible */
void gb_host_free(void *p);
int gb_h2d(void *dst, const void *src, size_t bytes);
int gb_d2h(void *dst, const void *src, size_t bytes);
int gb_d2d(void *dst, const void *src, size_t bytes);
int gb_memset(void *dst, int value, size_t bytes);
/* CUDA events on the library stream, slots 0..15 (timing). */
int gb_event_record(int slot);
float gb_event_elapsed_ms(int start_slot, int stop_slot);

/* Per-pass timing of the FFT line passes with CUDA events on the library
 * stream (benchmark instrumentation).  Kinds are 5 * axis + program with
 * axis 0 x, 1 y, 2 z and program 0 forward FFT, 1 inverse FFT,
 * 2 forward + kinetic + inverse, 3 inverse + potential + forward, 4 other;
 * kinds 15 + axis are the Crank-Nicolson line sweeps; kinds 18, 19 and 20
 * the plane-chained passes [z FWD, y FWD], [z INV.V.FWD, y FWD] (FP64) and
 * [y INV, z INV].
 * report() fills ms[k] / count[k] for k < nkinds and returns the number of
 * timed passes. */
int gb_pass_timing(int on);
int gb_pass_timing_report(double *ms, long *count, int nkinds);

/* Precision conversion between FP64 and FP32 copies (n scalars). */
int gb_convert_f64_to_f32(void *dst, const void *src, size_t n);
int gb_convert_f32_to_f64(void *dst, const void *src, size_t n);
/* Host FP64 array <-> device FP32 array (n scalars), staged on the device. */
int gb_upload_f64_as_f32(void *dev32, const void *host64, size_t n);
int gb_download_f32_as_f64(void *host64, const void *dev32, size_t n);
/* Status words of the bounded device-side waits (0 = no wait gave up).
 * Every host sync point of this layer (gb_synchronize, gb_d2h and every
 * reduction that returns a value) reads them and latches a nonzero word into
 * gb_last_error() with code GB_ERR_DEVICE_WAIT; the libgrid entry points then
 * abort with a libgrid message, as for any device failure.  A propagation
 * call itself does not wait for the GPU, so its failure surfaces at the next
 * read of a result (a norm, an energy, a host copy of a grid).
 * gb_clear_error() clears the words.  (No reference counterpart: the
 * reference's kernels have no device-side waits.) */
#define GB_ERR_DEVICE_WAIT 1070
#define GB_STATUS_PASS 0  /* pipelined line pass copy wait, plane-chain dependency wait */
#define GB_STATUS_CN 1    /* Crank-Nicolson sweep copy wait */
#define GB_STATUS_BATCH 2 /* batch grid barrier */
#define GB_STATUS_WORDS 4
int gb_cn_error_flag(void);
/* Same for the pipelined FFT line passes and the plane chains; reset != 0
 * clears it. */
int gb_pass_error_flag(int reset);
/* Poll limit of the waits that only wait for other CTAs' progress (the
 * plane chain's dependency wait and the batch kernel's grid barrier); 0
 * restores each wait's built-in limit (about a second).  Returns the
 * previous setting.  A small limit makes those waits give up early, which is
 * reported as above; it exists so tests can exercise that path.  Copy waits
 * (TMA, bulk copies) always keep their built-in limit.  (No reference
 * counterpart.) */
unsigned gb_wait_limit(unsigned polls);
/* Pipelined (persistent, TMA-prefetching) strided line passes: on = 1
 * enables (the default), 0 disables, -1 only queries.  Returns the previous
 * setting.  Both forms compute the same values.  (No reference counterpart.) */
int gb_pass_pipeline(int on);
/* Plane-chained passes: the leading z FWD + y FWD and the trailing
 * y INV + z INV transforms of a split-operator step (in FP64 also the
 * potential pass with the y FWD after it) each run as one persistent launch
 * that works plane by plane, so the intermediate result stays in L2 (grids
 * with nx >= 2 and ny = nz = 256).  on = 1 enables, 2 also chains the y INV
 * pass in front of the FP64 potential chain (y INV | z INV.V.FWD | y FWD in
 * one launch: five launches per step), 3 runs the FP64 real-time step with a
 * real V_ext as y INV | [z INV, V.y FWD, z FWD] (the potential applied in
 * the y stage), 0 disables, -1 only queries; returns the previous setting.
 * All schedules compute the same values up to rounding.  (No reference
 * counterpart.) */
int gb_plane_passes(int on);
/* Ticket lag of the plane-chained passes, in percent of one resident wave of
 * tiles (default 200): the second stage of a plane is issued that far behind
 * its first stage, so it rarely waits.  Any value >= 0 is free of deadlock and
 * computes the same values; -1 only queries.  Returns the previous setting.
 * (No reference counterpart.) */
int gb_chain_lag(int pct);

/* ----------------------------------------------------------------- FFT */
/* In-place 3-D complex FFT, unnormalised, then multiplied by scale
 * (replaces cuFFT Z2Z/C2C in src/cgrid_fft-cuda.c:41-174).  sign = -1 forward,
 * +1 inverse. */
int gb_fft3d(void *data, const gb_geom *g, int sign, double scale);

/* One 2nd-order split-operator step K(dt/2) V(dt) K(dt/2) in place, with the
 * FFTs, the kinetic factors (1/N folded in), the potential and the optional
 * g |psi|^2 term fused into the line passes
 * (replaces src/grid_wf.c:424-430 = 4 cuFFT calls + 5 kernels).
 * kin->scale must hold the 1/(nx ny nz) normalisation. */
int gb_split_step(void *psi, const gb_geom *g, const gb_kinetic *kin, const gb_potential *pot);
/* nsteps such steps with the k-space state kept between them (the inverse
 * and forward transforms between steps cancel and the two half kinetic
 * factors that meet merge into one K(dt) pass): 4 passes per step instead
 * of 9, the same result to rounding.  No reference counterpart (the
 * reference makes one step per call). */
int gb_split_steps(void *psi, const gb_geom *g, const gb_kinetic *kin, const gb_potential *pot, int nsteps);

/* k-space multipliers on unshifted frequencies (src/cgrid_diff.c:454-807):
 * dst = src * (-k^2) or src * (i k_axis). */
#define GB_K_LAPLACE 1
#define GB_K_GRADIENT_X 2
#define GB_K_GRADIENT_Y 3
#define GB_K_GRADIENT_Z 4
int gb_kspace_op(int op, void *dst, const void *src, const gb_geom *g);

/* Self-test: the propagation kernels' FP64 phase sine/cosine against the
 * CUDA library sincos on n host arguments; max_err[0..1] receives the
 * largest absolute differences of sin and cos.  (Test hook; no counterpart
 * in the reference.) */
int gb_sincos_selftest(const double *x_host, long n, double *max_err);

/* Pointwise kinetic factor on a k-space grid
 * (src/grid_wf_fft-cuda2.cu:23-99 and :108-138). */
int gb_kinetic_multiply(void *psi, const gb_geom *g, const gb_kinetic *kin);
/* Pointwise potential factor on a real-space grid (src/grid_wf-cuda2.cu:26-104). */
int gb_potential_multiply(void *psi, const gb_geom *g, const gb_potential *pot);

/* Sum of |k|^2 |psi_k|^2 over the forward FFT of psi (psi unchanged), no k0
 * shift, times fft_norm2 (src/cgrid_diff.c:817-879 after cgrid_fft).
 * work is a device buffer of the same size as psi. */
int gb_fft_ksq_sum(const void *psi, void *work, const gb_geom *g, double *out);

/* ------------------------------------------------------- pointwise ops */
#define GB_OP_CONST 1          /* c = d */
#define GB_OP_SCALE 2          /* c = c * d */
#define GB_OP_ADD_CONST 3      /* c = c + d */
#define GB_OP_SUM 4            /* c = a + b */
#define GB_OP_DIFF 5           /* c = a - b */
#define GB_OP_PRODUCT 6        /* c = a * b */
#define GB_OP_CONJ_PRODUCT 7   /* c = conj(a) * b */
#define GB_OP_ADD_SCALED 8     /* c = c + d * a */
#define GB_OP_ADD_SCALED_PRODUCT 9 /* c = c + d * a * b */
#define GB_OP_COPY 10          /* c = a */
/* Complex elementwise ops over n elements (src/cgrid-cuda2.cu:41-900). */
int gb_complex_op(int op, void *c, const void *a, const void *b, size_t n, double d_re, double d_im, int prec);
/* Real elementwise ops over n scalars (src/rgrid-cuda2.cu). */
int gb_real_op(int op, void *c, const void *a, const void *b, size_t n, double d, int prec);

/* Mixed real/complex ops on (nx, ny, nz) with real rows of rrow scalars
 * (src/ngrid-cuda2.cu, src/grid_wf-cuda2.cu:111-123). */
#define GB_MIX_REAL_TO_COMPLEX_RE 1   /* c = (complex) r */
#define GB_MIX_PRODUCT_NORM 2         /* r = r1 * |c|^2 */
#define GB_MIX_PRODUCT_COMPLEX_REAL 3 /* c = c * r */
#define GB_MIX_DENSITY 4              /* r = |c|^2 */
int gb_mixed_op(int op, void *c, void *r, const void *r1, const gb_geom *g, long rrow, int cprec, int rprec);

/* Real-FFT layout helpers for the padded rgrid (src/rgrid_fft-cuda.c):
 * pack the kz <= nz/2 half of a complex spectrum into rows of nz2 reals;
 * rebuild the full Hermitian spectrum from such rows; take real parts. */
int gb_r2c_pack(void *r, const void *c, const gb_geom *g);
int gb_c2r_unpack(void *c, const void *r, const gb_geom *g);
int gb_complex_real_part(void *r, const void *c, const gb_geom *g, long rrow);

/* Absorbing-boundary blend dst = (1 - a) wr + a wi (src/grid_wf-cuda2.cu:165-176). */
int gb_wf_merge(void *dst, const void *wr, const void *wi, const gb_geom *g, long lx, long hx, long ly, long hy, long lz, long hz);
/* k-space convolution product c = (-1)^(i+j+k) a b over nx x ny x nzc
 * complex entries (src/cgrid.c:1912-1944 with nzc = nz; src/rgrid.c:1848-1878
 * on the half spectrum, nzc = nz2 / 2); prec of all three arrays. */
int gb_fft_convolute(void *c, const void *a, const void *b, long nx, long ny, long nzc, int prec);
/* Geometry of a grid for gb_interpolate: extents, elements per (i, j) row,
 * step and real-space origin. */
typedef struct {
  long nx, ny, nz, row;
  double step, x0, y0, z0;
} gb_grid_frame;
/* dst(i, j, k) = trilinear interpolation of src at dst's point (i, j, k)
 * (src/cgrid.c:2067-2151, src/rgrid.c:2208-2300), corners outside src
 * taken by the boundary rule bc (GB_BC_*; Dirichlet value out_re + i out_im).
 * FP64 complex (is_real = 0) or FP64 padded real grids. */
int gb_interpolate(void *dst, const gb_grid_frame *d, const void *src, const gb_grid_frame *s, int bc, double out_re,
                   double out_im, int is_real);

/* ---------------------------------------------------------- reductions */
/* Deterministic FP64 reductions over the (nx, ny, nz) grid; out[0..1] gets
 * the (complex) sum without the step^d factor (src/cgrid-cuda2.cu:914-1395,
 * src/ngrid-cuda2.cu:511). */
#define GB_RED_SUM 1          /* sum a (complex) */
#define GB_RED_NORM2 2        /* sum |a|^2 */
#define GB_RED_CONJ_PRODUCT 3 /* sum conj(a) b (complex) */
#define GB_RED_EXPECT_COMPLEX 4 /* sum |a|^2 b, b complex */
#define GB_RED_EXPECT_REAL 5  /* sum |a|^2 b, b real with rows of brow */
#define GB_RED_REAL_SUM 6     /* sum a, a real with rows of arow */
#define GB_RED_KSQ_NORM2 7    /* sum |k|^2 |a|^2 on the unshifted frequency grid */
int gb_reduce(int op, const void *a, const void *b, const gb_geom *g, long arow, long brow, int bprec, double *out);
/* psi *= sqrt(target / (step_factor * sum |psi|^2)) with the sum reduced into
 * a device scalar that the scale kernel reads: no host synchronisation
 * (src/grid_wf.c:681-700 computes the same scale on the host).  FP64 or
 * FP32 storage (g->prec). */
int gb_normalize_device(void *psi, const gb_geom *g, double target, double step_factor);
/* out4 = {sum max(0, mu - V), #points with V < mu, min V, sum V} over a
 * padded real grid (vrow scalars per row): the terms of a Newton iteration
 * for the Thomas-Fermi chemical potential.  (No reference counterpart.) */
int gb_tf_stats(const void *v, const gb_geom *g, long vrow, double mu, double *out4);

/*
 * gb_reduce without any device allocation: no reference counterpart.  For
 * callers that cannot let a library allocate device memory (applications
 * that own all device memory through their own pool or a fixed budget, and
 * latency-critical loops where cudaMalloc or the synchronisation of cudaFree
 * is not acceptable).  Same operations and arguments as gb_reduce; the
 * partial sums live in a fixed file-scope __device__ array (8193 x 16 B) that
 * limits a call to grids of at most 16,777,216 points (larger grids are
 * rejected with an error before any launch).  All calls share that array:
 * calls that overlap on the GPU race.  The first call on a device looks up
 * the array's address (cudaGetSymbolAddress); make it before any stream
 * capture.  Requires gb_init / cuda_enable first.
 */
int gb_reduce_noalloc(int op, const void *a, const void *b, const gb_geom *g, long arow, long brow, int bprec, double *out);

/* --------------------------------------------------- finite differences */
#define GB_BC_DIRICHLET 0
#define GB_BC_NEUMANN 1
#define GB_BC_PERIODIC 2
#define GB_FD_LAPLACE 1
#define GB_FD_LAPLACE_X 2
#define GB_FD_LAPLACE_Y 3
#define GB_FD_LAPLACE_Z 4
#define GB_FD_GRADIENT_X 5
#define GB_FD_GRADIENT_Y 6
#define GB_FD_GRADIENT_Z 7
/* dst = stencil(src) with boundary values per bc (Dirichlet constant
 * outside = (out_re, out_im)); coef = 1/h^2 (Laplacians) or 1/(2h)
 * (gradients).  is_real selects real padded rows of row scalars
 * (src/cgrid_diff.c:201-442, src/rgrid_diff.c:309-343). */
int gb_fd(int op, void *dst, const void *src, const gb_geom *g, int bc, double out_re, double out_im, double coef, int is_real, long row);
/* sum conj(psi) * Laplacian_FD(psi) without writing the Laplacian
 * (src/grid_wf_cn.c:37-49 fused). */
int gb_fd_kinetic_sum(const void *psi, const gb_geom *g, int bc, double out_re, double out_im, double inv_h2, double *out);

/* --------------------------------------------------------- Crank-Nicolson */
/*
 * One dimension-split Crank-Nicolson kinetic step exp(-i T tstep / hbar) on
 * psi in place (src/grid_wf_cn.c:65-469 with src/linalg.c:62-92 and
 * :206-230), including the reference's end-row quirks.  pre and post are
 * optional potential factors applied before the x sweep and after the z
 * sweep (kind GB_POT_NONE to skip).
 */
typedef struct {
  int boundary;             /* WF_DIRICHLET_BOUNDARY=1, NEUMANN=2, PERIODIC=3 */
  double tstep_re, tstep_im;
  double mass;
  double kx0, ky0, kz0;
  double omega;
  double x0, y0;
  int absorb;
  long lx, hx, ly, hy, lz, hz;
} gb_cn_params;
int gb_cn_step(void *psi, const gb_geom *g, const gb_cn_params *p, const gb_potential *pre, const gb_potential *post);
/* Line solver of the Crank-Nicolson fast path (no rotation, no absorbing
 * region, lines of up to 256 points): 0 (the default) the segment-per-warp
 * solver (a lane per line, a warp per segment, carries chained through
 * shared memory), 1 the warp-cooperative solver (one warp per line, segment
 * carries by a warp-shuffle scan, persistent double-buffered tiles; measured
 * slower on B200: 0.487 against 0.447 ms per 192^3 step); -1 only queries.
 * Returns the previous setting.  Both solve the reference's systems; they
 * differ only in rounding.  (No reference counterpart.) */
int gb_cn_warp_solver(int on);

/* --------------------------------------------------------------- noise */
/* Seeded noise added to a device grid (the reference's src/rand.c API and
 * src/rand-cuda2.cu kernels), from a counter-based generator: the values
 * depend only on (seed, call, element), so they are reproducible for a
 * given seed and call sequence.  Real kinds act on a real grid with rows of
 * `row` scalars; complex kinds on a complex grid (row unused).
 *   R_UNIFORM     r += 2 s_re (u - 1/2)                 (src/rand.c:55-74)
 *   R_NORMAL      r += s_re n                           (src/rand.c:84-122)
 *   C_UNIFORM     z += 2 s_re (u - 1/2) + 2 i s_im (u' - 1/2) (src/rand.c:132-149)
 *   C_UNIFORM_SP  z += s_re u exp(2 pi i u')            (src/rand.c:159-176)
 *   C_NORMAL      z += s_re n + i s_im n'               (src/rand.c:186-214)
 *   C_NORMAL_SP   z += s_re n exp(i pi u)               (src/rand.c:224-250)
 * with u, u' uniform in (0, 1) and n, n' standard normal. */
#define GB_RAND_R_UNIFORM 1
#define GB_RAND_R_NORMAL 2
#define GB_RAND_C_UNIFORM 3
#define GB_RAND_C_UNIFORM_SP 4
#define GB_RAND_C_NORMAL 5
#define GB_RAND_C_NORMAL_SP 6
int gb_random(int kind, void *data, const gb_geom *g, long row, double scale_re, double scale_im,
              unsigned long long seed, unsigned long long call);

/* ------------------------------------------------------------- batches */
/*
 * Many independent 2-D wave functions of uneven sizes advanced together by
 * the second-order FFT split-operator step (the step gb_split_step makes for
 * one grid), all instances in one persistent launch per call.  No reference
 * counterpart: the reference steps one grid per grid_wf_propagate call.
 * An instance is psi (device, complex, geometry g with g.nx == 1 and
 * g.ny, g.nz in {64, 128, 256, 512}; one precision for the whole batch), its
 * K(dt/2) factor and its V(dt) step with the meanings of gb_split_step; a
 * potential of kind GB_POT_NONE with g == 0 and cons == 0 leaves the
 * potential step out.  The batch keeps the device pointers: the grids must
 * stay allocated while it exists.
 */
typedef struct {
  void *psi;
  gb_geom g;
  gb_kinetic kin;
  gb_potential pot;
} gb_batch_item;
typedef struct gb_batch gb_batch;
gb_batch *gb_batch_create(const gb_batch_item *items, int n);
/* `steps` steps of every instance, asynchronous on the library stream. */
int gb_batch_step(gb_batch *b, int steps);
/* Plan the autotuner chose: the persistent launch's CTA size (128, 256,
 * 512), -1 for the per-class graph, 0 before the first call of >= 9 steps. */
int gb_batch_threads(const gb_batch *b);
/* Status of the launch's bounded grid barrier (0 = no wait gave up). */
int gb_batch_error_flag(gb_batch *b, int reset);
void gb_batch_free(gb_batch *b);

/* ------------------------------------------ learned warm start (U-Net) */
/*
 * Kernels of the 3-D convolutional U-Net that turns an external potential
 * into a starting guess for imaginary-time ground-state relaxation.  No
 * reference counterpart: the reference's imaginary-time loop is composed by
 * its callers from grid_wf_propagate / grid_wf_normalize / grid_wf_energy
 * (src/grid_wf.c:379-556, 681-700, 215-221) and starts from whatever guess
 * the caller maps in; these kernels only produce that guess.
 *
 * Activations are FP32 [C][D][H][W] (one sample, or nb samples stacked along
 * the depth axis for the *_nb convolutions), weights bf16
 * [Cout][Cin][27] (3x3x3 taps, zero padding, tap t = 9(dz+1)+3(dy+1)+(dx+1)),
 * accumulation FP32.  Gradient buffers accumulate (+=); gb_unet_adam clears
 * them.  All calls are asynchronous on the library stream.
 */
/* y = conv(x, w) + b, optionally ReLU'd.  4*cin*27*4 B must fit 48 KB. */
int gb_unet_conv3_fwd(const float *x, const uint16_t *w, const float *b, float *y, int cin, int cout, int d, int h,
                      int wd, int relu);
/* gx = conv^T(gy, w) (overwrites gx).  4*cout*27*4 B must fit 48 KB. */
int gb_unet_conv3_bwd_data(const float *gy, const uint16_t *w, float *gx, int cin, int cout, int d, int h, int wd);
/* gw += dL/dw, gb += dL/db (gb may be NULL). */
int gb_unet_conv3_bwd_weight(const float *x, const float *gy, float *gw, float *gb, int cin, int cout, int d, int h,
                             int wd);
/* The same three convolutions over nb samples in one call: activations
 * [C][nb*d][h][wd], sample s in planes [s*d, (s+1)*d) of every channel, with
 * no depth neighbours across samples (the weight and bias gradients sum
 * over all samples).  Pooling, upsampling, the ReLU mask and the MSE
 * gradient need no variant: give them depth nb*d or n = nb times the
 * sample's size.  Batches fill the GPU on the coarse levels of small
 * grids. */
int gb_unet_conv3_fwd_nb(const float *x, const uint16_t *w, const float *b, float *y, int cin, int cout, int nb, int d,
                         int h, int wd, int relu);
int gb_unet_conv3_bwd_data_nb(const float *gy, const uint16_t *w, float *gx, int cin, int cout, int nb, int d, int h,
                              int wd);
int gb_unet_conv3_bwd_weight_nb(const float *x, const float *gy, float *gw, float *gb, int cin, int cout, int nb, int d,
                                int h, int wd);
/* gy[i] = 0 where y[i] <= 0 (y is the ReLU output). */
int gb_unet_relu_bwd(float *gy, const float *y, long n);
/* 2x2x2 average pooling and its gradient (gx += ...); d, h, wd = input
 * extents (even). */
int gb_unet_pool2_fwd(const float *x, float *y, int c, int d, int h, int wd);
int gb_unet_pool2_bwd(const float *gy, float *gx, int c, int d, int h, int wd);
/* Nearest-neighbour 2x upsampling and its gradient; d, h, wd = input extents. */
int gb_unet_up2_fwd(const float *x, float *y, int c, int d, int h, int wd);
int gb_unet_up2_bwd(const float *gy, float *gx, int c, int d, int h, int wd);
/* grad = scale * (pred - tgt). */
int gb_unet_mse_grad(const float *pred, const float *tgt, float *grad, long n, float scale);
/* Adam step on FP32 master weights w; refreshes the bf16 copy wb (may be
 * NULL) and clears g.  c1 = 1/(1-b1^t), c2 = 1/(1-b2^t). */
int gb_unet_adam(float *w, uint16_t *wb, float *m, float *v, float *g, long n, float lr, float b1, float b2, float eps,
                 float c1, float c2);
/* wb = bf16(w), round to nearest even. */
int gb_unet_to_bf16(const float *w, uint16_t *wb, long n);
/* p[0..n) = v. */
int gb_unet_fill(float *p, long n, float v);
/* Minibatch gather, one launch: for b < count, sample idx[b] of a
 * device-resident set of nset samples (inputs xs [nset][cin][vol], targets
 * ys [nset][vol]) goes to slot b of a batch-nb network's input in
 * ([cin][nb][vol]) and target tgt ([nb][vol]).  count <= nb and
 * count <= GB_UNET_MAX_GATHER; idx is a host array read during the call;
 * an index outside [0, nset) is an error (1101) and nothing is copied.
 * (No reference counterpart.) */
#define GB_UNET_MAX_GATHER 32
int gb_unet_gather(float *in, float *tgt, const float *xs, const float *ys, const int *idx, int count, int cin,
                   long vol, int nb, long nset);
/* Convolution engine: 1 (the default) runs the forward and data-gradient
 * convolutions as tcgen05 implicit GEMMs (bf16 operands in shared memory,
 * FP32 accumulators in tensor memory) and the weight gradient on mma.sync
 * bf16 tensor-core instructions (FP32 accumulate), with activations and
 * gradients rounded to bf16 as operands; 0 runs the FP32 SIMT kernels
 * (FP32 activations, bf16 weights).  Shapes without a tensor-core plan
 * (weight gradients of volumes narrower than 8 points or not a multiple of
 * 8 wide, more than 64 output channels) always run SIMT.  -1 only queries; returns the previous
 * setting.  (No reference counterpart.) */
int gb_unet_tensor_cores(int on);
/* Warm-start inputs and guesses built on the device (no host round trip of
 * the 3-D arrays):
 *   gb_unet_potential  V = k r^2 / 2 + sum of Gaussian bumps a exp(-|r-c|^2/w^2)
 *                      on x_i = (i - n/2) step, into a padded real grid;
 *   gb_unet_features   the network input [3][n]: tanh((V - vmin)/vscale),
 *                      gfeat, sqrt(max(mu - V, 0)/g) / amax;
 *   gb_unet_amplitude  psi = max(amp * scale, 0) + floor (real) into a
 *                      complex grid of precision prec;
 *   gb_unet_gaussian   exp(-r^2 / width^2).
 * (No reference counterpart.) */
#define GB_UNET_MAX_BUMPS 8
typedef struct {
  int n;
  double amp[GB_UNET_MAX_BUMPS], w[GB_UNET_MAX_BUMPS], c[GB_UNET_MAX_BUMPS][3];
} gb_unet_bumps;
int gb_unet_potential(double *v, int nx, int ny, int nz, long vrow, double step, double k, const gb_unet_bumps *bumps);
int gb_unet_features(const double *v, int nx, int ny, int nz, long vrow, double vmin, double vscale, float gfeat,
                     double mu, double g, double amax, float *out);
int gb_unet_amplitude(const float *amp, float scale, float floor, void *psi, long n, int prec);
int gb_unet_gaussian(float *out, int nx, int ny, int nz, double step, double width);
/* out = |psi| * inv_scale from a complex grid (device pointer, precision prec). */
int gb_unet_abs(const void *psi, int prec, long n, float inv_scale, float *out);

#ifdef __cplusplus
}
#endif

#endif
