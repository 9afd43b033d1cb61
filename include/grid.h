/*
 * libgrid-b200 public C API: a drop-in for libgrid's wavefunction
 * propagation path on one NVIDIA B200.
 *
 * Source compatibility: programs written against libgrid's double-precision
 * CUDA build (REAL = double, INT = long, `#include <grid/grid.h>`) compile
 * unchanged against this header and link against libgrid_b200.so.  The
 * structures below keep the field order, types and sizes of the reference's
 * src/structs.h:24-103 in its USE_CUDA + DOUBLE_PREC configuration (the FFTW
 * plan fields become opaque pointers of the same size; the cuFFT handle field
 * keeps its int type and is used by this library as a device-block slot id).
 *
 * Each prototype cites the reference definition it replaces.  Semantics
 * (argument meaning, in-place rules, abort() on API misuse with a
 * "libgrid:" message) follow those definitions; device data is authoritative
 * after a GPU operation and the host copy `value` is brought up to date by the
 * host-side accessors (value_at_index, write, map, cuda_remove_block), as in
 * the reference's CUDA build (src/cuda.c:477-499).
 */
#ifndef LIBGRID_B200_GRID_H
#define LIBGRID_B200_GRID_H

#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <time.h>

#ifndef REAL
#define REAL double
#endif
#ifndef INT
#define INT long
#endif
#ifndef DOUBLE_PREC
#define DOUBLE_PREC
#endif
#ifndef HBAR
#define HBAR 1.0 /* reference make.conf:45 */
#endif
#ifndef EXPORT
#define EXPORT
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Atomic-unit conversions (reference src/au.h:10-28). */
#define GRID_AUTOANG 0.52917725
#define GRID_AUTOM (GRID_AUTOANG * 1E-10)
#define GRID_AUTOK 3.15773213e5
#define GRID_AUTOJ 4.359748E-18
#define GRID_AUTOKG 9.10938356E-31
#define GRID_AUTOAMU (1.0 / 1822.88853006)
#define GRID_AUTOFS 0.02418884
#define GRID_AUTOS (GRID_AUTOFS * 1E-15)
#define GRID_AUKB 3.1668773658e-06

/* Global parameters and enums (reference src/defs.h:10-32). */
#define GRID_EPS 1.0E-16
#define GRID_ABS_BC_FFT (3.0E4 / GRID_AUTOK)

#define CGRID_DIRICHLET_BOUNDARY cgrid_value_outside_dirichlet
#define CGRID_NEUMANN_BOUNDARY cgrid_value_outside_neumann
#define CGRID_PERIODIC_BOUNDARY cgrid_value_outside_periodic
#define RGRID_DIRICHLET_BOUNDARY rgrid_value_outside_dirichlet
#define RGRID_NEUMANN_BOUNDARY rgrid_value_outside_neumann
#define RGRID_PERIODIC_BOUNDARY rgrid_value_outside_periodic

#define WF_DIRICHLET_BOUNDARY 1
#define WF_NEUMANN_BOUNDARY 2
#define WF_PERIODIC_BOUNDARY 3

#define WF_2ND_ORDER_FFT 1
#define WF_4TH_ORDER_FFT 2
#define WF_2ND_ORDER_CFFT 3
#define WF_4TH_ORDER_CFFT 4
#define WF_2ND_ORDER_CN 5
#define WF_4TH_ORDER_CN 6
#define WF_1ST_ORDER_EULER 7

/* Device-side arithmetic of a wavefunction (B200 extension, no counterpart
 * in the reference): FP64 everywhere, or FP32 storage/FFT/elementwise with
 * FP64 phase-argument range reduction and FP64 reductions. */
#define GRID_PREC_FP64 0
#define GRID_PREC_FP32 1

#define FMT_R "%le"
#define FMT_I "%ld"

/* Complex grid (reference src/structs.h:25-50). */
typedef struct cgrid_struct {
  REAL complex *value;
  char id[32];
  size_t grid_len;
  INT nx, ny, nz;
  REAL step;
  REAL x0, y0, z0;
  REAL kx0, ky0, kz0;
  REAL omega;
  REAL complex (*value_outside)(struct cgrid_struct *grid, INT i, INT j, INT k);
  void *outside_params_ptr;
  REAL complex default_outside_params;
  void *plan, *iplan;   /* fftw_plan in the reference; unused here */
  int cufft_handle;     /* cufftHandle in the reference; device-block slot id here */
  char host_lock;
  REAL fft_norm;
  REAL fft_norm2;
  char flag;
} cgrid;

/* Real grid, padded rows of nz2 = 2 (nz/2 + 1) (reference src/structs.h:56-79). */
typedef struct rgrid_struct {
  REAL *value;
  char id[32];
  size_t grid_len;
  INT nx, ny, nz, nz2;
  REAL step;
  REAL x0, y0, z0;
  REAL kx0, ky0, kz0;
  REAL (*value_outside)(struct rgrid_struct *grid, INT i, INT j, INT k);
  void *outside_params_ptr;
  REAL default_outside_params;
  void *plan, *iplan;
  int cufft_handle_r2c; /* device-block slot id here */
  int cufft_handle_c2r;
  char host_lock;
  REAL fft_norm;
  REAL fft_norm2;
  char flag;
} rgrid;

/* Wavefunction (reference src/structs.h:85-103). */
typedef struct wf_struct {
  cgrid *grid;
  REAL mass;
  REAL norm;
  REAL cfft_width;
  char boundary;
  char propagator;
  cgrid *cworkspace;
  cgrid *cworkspace2;
  cgrid *cworkspace3;
  REAL (*ts_func)(INT, INT, INT, INT, INT, INT, INT, INT, INT);
  INT lx, hx, ly, hy, lz, hz;
  REAL kmax;
} wf;

/* ---------------------------------------------------------------- setup */
/* src/threads.c:89 */
void grid_threads_init(INT threads);
/* src/threads.c:154 */
INT grid_threads(void);
/* src/cuda.c:1168 -- selects the B200 (first entry of gpus, or device 0) */
void cuda_enable(char val, int ngpus, int *gpus);
/* src/cuda.c:1195 */
char cuda_status(void);
/* src/cuda.c:477 -- copy=1 refreshes the host copy before dropping the device copy */
int cuda_remove_block(void *host_mem, char copy);
/* src/cuda.c:1142 */
void cuda_free_all_blocks(char sync);
/* src/grid_wf_analyze.c:21 */
void grid_wf_analyze_method(char method);

/* ---------------------------------------------------------------- cgrid */
/* src/cgrid.c:45 */
cgrid *cgrid_alloc(INT nx, INT ny, INT nz, REAL step, REAL complex (*value_outside)(cgrid *grid, INT i, INT j, INT k), void *outside_params_ptr, char *id);
/* src/cgrid.c:169 */
cgrid *cgrid_clone(cgrid *grid, char *id);
/* src/cgrid.c:332 */
void cgrid_free(cgrid *grid);
/* src/cgrid.c:264,282,303,319 */
void cgrid_set_origin(cgrid *grid, REAL x0, REAL y0, REAL z0);
void cgrid_shift_origin(cgrid *grid, REAL x0, REAL y0, REAL z0);
void cgrid_set_momentum(cgrid *grid, REAL kx0, REAL ky0, REAL kz0);
void cgrid_set_rotation(cgrid *grid, REAL omega);
/* src/cgrid.c:360,383 -- binary format nx, ny, nz (INT), step (REAL), values */
/* Seeded noise (src/rand.c:34-250; GPU src/rand-cuda2.cu:54-300).  Values
 * come from a counter-based generator seeded by grid_random_seed (by the
 * time of day when never seeded, as in the reference); they follow the
 * reference's distributions, not its drand48 / cuRAND sequences. */
void grid_random_seed(INT nx, INT ny, INT nz, INT seed);
void rgrid_random_uniform(rgrid *grid, REAL scale);
void rgrid_random_normal(rgrid *grid, REAL scale);
void cgrid_random_uniform(cgrid *grid, REAL complex scale);
void cgrid_random_uniform_sp(cgrid *grid, REAL scale);
void cgrid_random_normal(cgrid *grid, REAL complex scale);
void cgrid_random_normal_sp(cgrid *grid, REAL scale);
/* src/cgrid.c:360 */
void cgrid_write(cgrid *grid, FILE *out);
/* src/cgrid.c:383 -- a file of another size is interpolated (cgrid_extrapolate) */
cgrid *cgrid_read(cgrid *grid, FILE *in);
/* src/cgrid.c:2126 -- trilinear interpolation of src at dest's points, on the GPU */
void cgrid_extrapolate(cgrid *dest, cgrid *src);
/* src/cgrid.c:1912 -- k-space convolution product (-1)^(i+j+k) a b */
void cgrid_fft_convolute(cgrid *gridc, cgrid *grida, cgrid *gridb);
/* src/cgrid.c:615 */
void cgrid_copy(cgrid *dst, cgrid *src);
/* src/cgrid.c:711,725 */
void cgrid_zero(cgrid *grid);
void cgrid_constant(cgrid *grid, REAL complex c);
/* src/cgrid.c:793 */
void cgrid_map(cgrid *grid, REAL complex (*func)(void *arg, REAL x, REAL y, REAL z), void *farg);
/* src/cgrid.c:934,964,994,1169 */
void cgrid_sum(cgrid *gridc, cgrid *grida, cgrid *gridb);
void cgrid_difference(cgrid *gridc, cgrid *grida, cgrid *gridb);
void cgrid_product(cgrid *gridc, cgrid *grida, cgrid *gridb);
void cgrid_conjugate_product(cgrid *gridc, cgrid *grida, cgrid *gridb);
/* src/cgrid.c:1197,1223 */
void cgrid_add(cgrid *grid, REAL complex c);
void cgrid_multiply(cgrid *grid, REAL complex c);
/* src/cgrid.c:1303,1333 */
void cgrid_add_scaled(cgrid *gridc, REAL complex d, cgrid *grida);
void cgrid_add_scaled_product(cgrid *gridc, REAL complex d, cgrid *grida, cgrid *gridb);
/* src/cgrid.c:1536,1610,1640,1669 */
REAL complex cgrid_integral(cgrid *grid);
REAL cgrid_integral_of_square(cgrid *grid);
REAL complex cgrid_integral_of_conjugate_product(cgrid *grida, cgrid *gridb);
REAL complex cgrid_grid_expectation_value(cgrid *dgrid, cgrid *opgrid);
/* src/cgrid.c:1822,1839,1857,1873,1887 */
void cgrid_fft(cgrid *grid);
void cgrid_inverse_fft(cgrid *grid);
void cgrid_scaled_inverse_fft(cgrid *grid, REAL complex c);
void cgrid_inverse_fft_norm(cgrid *grid);
void cgrid_inverse_fft_norm2(cgrid *grid);
/* src/cgrid.c:1960,2016 */
REAL complex cgrid_value_at_index(cgrid *grid, INT i, INT j, INT k);
void cgrid_value_to_index(cgrid *grid, INT i, INT j, INT k, REAL complex value);
/* src/cgrid_bc.c:21,39,69 */
REAL complex cgrid_value_outside_dirichlet(cgrid *grid, INT i, INT j, INT k);
REAL complex cgrid_value_outside_neumann(cgrid *grid, INT i, INT j, INT k);
REAL complex cgrid_value_outside_periodic(cgrid *grid, INT i, INT j, INT k);
/* src/cgrid_diff.c:201,235,269 */
void cgrid_fd_gradient_x(cgrid *grid, cgrid *gradient);
void cgrid_fd_gradient_y(cgrid *grid, cgrid *gradient);
void cgrid_fd_gradient_z(cgrid *grid, cgrid *gradient);
/* src/cgrid_diff.c:303,342,379,416 */
void cgrid_fd_laplace(cgrid *grid, cgrid *laplace);
void cgrid_fd_laplace_x(cgrid *grid, cgrid *laplacex);
void cgrid_fd_laplace_y(cgrid *grid, cgrid *laplacey);
void cgrid_fd_laplace_z(cgrid *grid, cgrid *laplacez);
/* src/cgrid_diff.c:454,503,552 */
void cgrid_fft_gradient_x(cgrid *grid, cgrid *gradient_x);
void cgrid_fft_gradient_y(cgrid *grid, cgrid *gradient_y);
void cgrid_fft_gradient_z(cgrid *grid, cgrid *gradient_z);
/* src/cgrid_diff.c:601 */
void cgrid_fft_laplace(cgrid *grid, cgrid *laplace);
/* src/cgrid_diff.c:817 */
REAL cgrid_fft_laplace_expectation_value(cgrid *grid);
/* src/cgrid_diff.c:125 -- FD or FFT Laplacian per grid_wf_analyze_method */
void cgrid_laplace(cgrid *grid, cgrid *laplace);

/* ---------------------------------------------------------------- rgrid */
/* src/rgrid.c:38,310 */
rgrid *rgrid_alloc(INT nx, INT ny, INT nz, REAL step, REAL (*value_outside)(rgrid *grid, INT i, INT j, INT k), void *outside_params_ptr, char *id);
void rgrid_free(rgrid *grid);
/* src/rgrid.c:662,727,741,806 */
void rgrid_copy(rgrid *dst, rgrid *src);
void rgrid_zero(rgrid *grid);
void rgrid_constant(rgrid *grid, REAL c);
void rgrid_map(rgrid *grid, REAL (*func)(void *arg, REAL x, REAL y, REAL z), void *farg);
/* src/rgrid.c:945,1003,1169,1248 */
void rgrid_sum(rgrid *gridc, rgrid *grida, rgrid *gridb);
void rgrid_product(rgrid *gridc, rgrid *grida, rgrid *gridb);
void rgrid_multiply(rgrid *grid, REAL c);
void rgrid_add_scaled(rgrid *gridc, REAL d, rgrid *grida);
/* src/rgrid.c:1471 */
REAL rgrid_integral(rgrid *grid);
/* src/rgrid.c:1762,1779,1797,1811 -- R2C/C2R in the padded in-place layout */
void rgrid_fft(rgrid *grid);
void rgrid_inverse_fft(rgrid *grid);
void rgrid_scaled_inverse_fft(rgrid *grid, REAL c);
void rgrid_inverse_fft_norm(rgrid *grid);
/* src/rgrid.c:1824 */
void rgrid_inverse_fft_norm2(rgrid *grid);
/* src/rgrid.c:2020,2064 */
REAL rgrid_value_at_index(rgrid *grid, INT i, INT j, INT k);
void rgrid_value_to_index(rgrid *grid, INT i, INT j, INT k, REAL value);
/* src/rgrid_bc.c:19,35,62 */
REAL rgrid_value_outside_dirichlet(rgrid *grid, INT i, INT j, INT k);
REAL rgrid_value_outside_neumann(rgrid *grid, INT i, INT j, INT k);
REAL rgrid_value_outside_periodic(rgrid *grid, INT i, INT j, INT k);
/* src/rgrid_diff.c:309 */
void rgrid_fd_laplace(rgrid *grid, rgrid *laplace);
/* src/rgrid.c:339,360 -- binary grid I/O; rgrid_read interpolates other sizes */
void rgrid_write(rgrid *grid, FILE *out);
rgrid *rgrid_read(rgrid *grid, FILE *in);
/* src/rgrid.c:2267 -- trilinear interpolation of src at dest's points, on the GPU */
void rgrid_extrapolate(rgrid *dest, rgrid *src);
/* src/rgrid.c:1848 -- k-space convolution product on the half spectrum */
void rgrid_fft_convolute(rgrid *gridc, rgrid *grida, rgrid *gridb);

/* ---------------------------------------------------------------- ngrid */
/* src/ngrid.c:53,186,254,355 */
void grid_real_to_complex_re(cgrid *dest, rgrid *source);
void grid_product_norm(rgrid *dst, rgrid *src1, cgrid *src2);
void grid_product_complex_with_real(cgrid *dst, rgrid *src);
REAL grid_grid_expectation_value(cgrid *dgrid, rgrid *opgrid);

/* ------------------------------------------------------------------- wf */
/* src/grid_wf.c:26,99,131,157,185 */
wf *grid_wf_alloc(INT nx, INT ny, INT nz, REAL step, REAL mass, char boundary, char propagator, char *id);
void grid_wf_boundary(wf *gwf, wf *gwfp, INT lx, INT hx, INT ly, INT hy, INT lz, INT hz);
wf *grid_wf_clone(wf *gwf, char *id);
void grid_wf_free(wf *gwf);
REAL grid_wf_absorb(INT i, INT j, INT k, INT lx, INT hx, INT ly, INT hy, INT lz, INT hz);
/* src/grid_wf.c:215,232,246 */
REAL grid_wf_energy(wf *gwf, rgrid *potential);
REAL grid_wf_kinetic_energy(wf *gwf);
REAL grid_wf_potential_energy(wf *gwf, rgrid *potential);
/* src/grid_wf.c:264,331,379 */
void grid_wf_propagate_predict(wf *gwf, wf *gwfp, cgrid *potential, REAL complex time);
void grid_wf_propagate_correct(wf *gwf, cgrid *potential, REAL complex time);
void grid_wf_propagate(wf *gwf, cgrid *potential, REAL complex time);
/* src/grid_wf.c:569 */
void grid_wf_propagate_potential(wf *gwf, REAL complex tstep, cgrid *potential, REAL cons);
/* src/grid_wf.c:611,637,651,668 */
void grid_wf_density(wf *gwf, rgrid *density);
void grid_wf_zero(wf *gwf);
void grid_wf_constant(wf *gwf, REAL complex c);
void grid_wf_map(wf *gwf, REAL complex (*func)(void *arg, REAL x, REAL y, REAL z), void *farg);
/* src/grid_wf.c:681,694,711,728 */
REAL grid_wf_norm(wf *gwf);
REAL grid_wf_normalize(wf *gwf);
REAL complex grid_wf_overlap(wf *gwfa, wf *gwfb);
void grid_wf_merge(wf *dst, cgrid *wfr, cgrid *wfi);
/* src/grid_wf_fft.c:101,119,141,206,276 */
REAL grid_wf_energy_fft(wf *gwf, rgrid *potential);
REAL grid_wf_kinetic_energy_fft(wf *gwf);
void grid_wf_propagate_kinetic_fft(wf *gwf, REAL complex time);
void grid_wf_propagate_kinetic_cfft(wf *gwf, REAL complex time);
void grid_wf_square_of_potential_gradient(wf *gwf, cgrid *sq_grad_pot, cgrid *potential);
/* src/grid_wf_cn.c:19,37,65 */
REAL grid_wf_energy_cn(wf *gwf, rgrid *potential);
REAL grid_wf_kinetic_energy_cn(wf *gwf);
void grid_wf_propagate_kinetic_cn(wf *gwf, REAL complex tstep);
/* src/grid_wf_diag.c:20 */
REAL grid_wf_energy_and_error(wf *gwf, cgrid *potential, cgrid *workspace, REAL *error);

/* ------------------------------------------- B200 extensions (no reference counterpart) */
/*
 * One Gross-Pitaevskii step with the nonlinear potential V_ext + g |psi|^2
 * built inside the propagation kernels.  Defined as the composition of
 * reference primitives: FFT propagators use K(dt/2) -> V_ext + g|psi_mid|^2
 * -> potential(dt) -> K(dt/2) (src/grid_wf.c:424-430 with the potential built
 * by grid_wf_density + grid_real_to_complex_re + cgrid_sum); CN propagators
 * use potential(dt/2) with |psi(t)|^2 -> grid_wf_propagate_kinetic_cn(dt) ->
 * potential(dt/2) with |psi_CN|^2 (src/grid_wf.c:526-530).  vext may be NULL
 * (pure nonlinearity).
 */
void grid_wf_propagate_gp(wf *gwf, rgrid *vext, REAL g, REAL complex time);
/*
 * nsteps steps in one call (no reference counterpart).  For the 2nd-order
 * FFT and CFFT propagators without an absorbing region the k-space state is
 * kept between the steps: the transforms between steps cancel and the two
 * half kinetic factors that meet merge, about half the memory traffic of
 * nsteps separate calls, with the same result to rounding.  Other
 * propagators make nsteps ordinary steps.
 */
void grid_wf_propagate_n(wf *gwf, cgrid *potential, REAL complex time, INT nsteps);
void grid_wf_propagate_gp_n(wf *gwf, rgrid *vext, REAL g, REAL complex time, INT nsteps);
/*
 * Imaginary-time relaxation steps (no reference counterpart as one call):
 * nsteps of grid_wf_propagate_gp(time), each followed by renormalisation to
 * gwf->norm as grid_wf_normalize makes it (src/grid_wf.c:681-700), with the
 * norm reduced and applied on the device: no host synchronisation.
 */
void grid_wf_relax_gp_n(wf *gwf, rgrid *vext, REAL g, REAL complex time, INT nsteps);
/* psi = max(amp * scale, 0) + floor (real) from a device float array of
 * nx ny nz values (a device-side initial guess; no reference counterpart). */
void grid_wf_set_amplitude_device(wf *gwf, const float *amp, REAL scale, REAL floor);
/* Host/device coherence of a grid's value array (no reference counterpart):
 * refresh the host copy; declare host-side writes; or get the FP64 device
 * copy for device-side producers and consumers (mode 0 read, 1 write (every
 * value is overwritten), 2 read and write). */
void gb_grid_sync_host(void *host_mem);
void gb_grid_host_modified(void *host_mem);
void *gb_grid_device(void *host_mem, int mode);
/* Select GRID_PREC_FP64 (default) or GRID_PREC_FP32 for gwf's device data. */
void grid_wf_precision(wf *gwf, char mode);
char grid_wf_get_precision(wf *gwf);

/*
 * Batched propagation (no reference counterpart; the reference advances one
 * wave function per grid_wf_propagate call).  grid_wf_batch_alloc groups n
 * 2-D wave functions (nx == 1; ny, nz in {64, 128, 256, 512}; periodic
 * boundaries, WF_2ND_ORDER_FFT; one device precision for all) with their
 * complex potentials (an entry may be NULL: no potential step) and one time
 * step; grid_wf_batch_propagate then makes `steps` steps of every wave
 * function, the same step grid_wf_propagate(wfs[i], potentials[i], time)
 * makes, all in one persistent GPU launch.  The wave functions and
 * potentials must stay allocated while the batch exists; host-side changes
 * to them are picked up on the next propagate call.
 */
typedef struct grid_wf_batch grid_wf_batch;
grid_wf_batch *grid_wf_batch_alloc(wf **wfs, cgrid **potentials, INT n, REAL complex time);
void grid_wf_batch_propagate(grid_wf_batch *b, INT steps);
void grid_wf_batch_free(grid_wf_batch *b);
/* Plan the batch autotuner chose: persistent CTA size (128, 256, 512), -1
 * for the per-class CUDA graph, 0 until a call of >= 9 steps. */
int grid_wf_batch_threads(grid_wf_batch *b);

#ifdef __cplusplus
}
#endif

#include "gb_cuda.h"

#endif /* LIBGRID_B200_GRID_H */
