// Internal declarations shared by the libgrid-b200 CUDA translation units.
#pragma once

#include <cuda.h>
#include <stddef.h>

#include "gb_cuda.h"

// Library-owned device scratch slots.
enum {
  GB_SCR_KIN = 0,      // kinetic factor tables
  GB_SCR_PARTIAL = 1,  // reduction partial sums
  GB_SCR_RESULT = 2,   // final reduction results
  GB_SCR_CN = 3,       // line-solver coefficient tables
  GB_SCR_WORK = 4,     // temporary full grids
  GB_SCR_STAGE = 5,    // precision-conversion staging
  GB_SCR_KIN2 = 6,     // kinetic factor tables of the merged K(dt) pass
  GB_SCR_CHAIN = 7,    // tile counters and ticket of the plane-chained passes
  GB_SCR_UNET = 8,     // per-chunk weight-gradient partials of the U-Net kernels
  GB_SCR_UNETB = 9,    // packed weight operand of the U-Net tensor-core convolutions
  GB_SCR_COUNT = 10
};

void *gb__scratch(int slot, size_t bytes);
// Pass timing brackets (no-ops unless gb_pass_timing(1) was called).
int gb__pass_begin(int kind);
void gb__pass_end(int slot);
const void *gb__twiddles(long n, int prec);
// Tensor map (TMA descriptor) over the line view [outer][n][inner] of a
// complex grid (fp32 = 0: double2 elements, 1: float2), read as reals with
// the box 2*bz reals x rows lines x 1.  Cached per argument set.
int gb__tmap_lines(CUtensorMap *out, const void *base, long outer, long n, long inner, int fp32, int bz, int rows);
// Device flag set by a pipelined pass or plane chain whose bounded wait gave
// up (status word GB_STATUS_PASS).
int *gb__pass_errflag(void);
// Device address of a status word (GB_STATUS_*), allocated on first use.
int *gb__status(int word);
// Read (and with reset != 0 clear) one status word after draining the stream.
int gb__status_word(int word, int reset);
// Poll limit for waits on other CTAs' progress: gb_wait_limit's setting, or
// dflt when none is set.
unsigned gb__wait_limit(unsigned dflt);
// Plane-chain lag in percent of one resident wave of tickets (gb_chain_lag).
int gb__chain_lag_pct(void);
// Device slot for a reduction result (32 bytes) and its read-back: one copy
// brings the result and the status words; a nonzero status word latches
// GB_ERR_DEVICE_WAIT.
void *gb__result_slot(void);
int gb__read_result(void *host, size_t bytes);

// Kinetic factor tables for (g, kin): per-axis complex factors exp(tm k_a^2)
// in the storage precision of g and per-axis k_a^2 in FP64.
struct GbKinTables {
  const void *kfac[3];
  const double *ksq[3];
};
int gb__kin_tables(const gb_geom *g, const gb_kinetic *kin, int unshifted, GbKinTables *out);
// The same tables into caller-owned buffers (fac: nx + ny + nz factors in the
// storage precision, then as many k^2 values in ksq).
int gb__kin_tables_at(void *fac, double *ksq, const gb_geom *g, const gb_kinetic *kin);

// Precision-specific drivers (gb_fft_f64.cu / gb_fft_f32.cu).
template <typename T> int gb__fft3d_t(void *data, const gb_geom *g, int sign, double scale);
template <typename T> int gb__split_step_t(void *psi, const gb_geom *g, const gb_kinetic *kin, const gb_potential *pot);
template <typename T>
int gb__split_steps_t(void *psi, const gb_geom *g, const gb_kinetic *kin, const gb_potential *pot, int nsteps);
template <typename T> int gb__ksq_sum_t(const void *psi, void *work, const gb_geom *g, double *out);

// Tensor-core U-Net convolutions (gb_unet_tc.cu): return -1 when the path is
// off or the shape has no plan (the caller runs the SIMT kernel), else a
// status.  mode 0: y = conv(x) (+ bias, ReLU); mode 1: y = data gradient of
// x = gy.  nb samples of d planes each are stacked along the depth axis.
int gb__unet_conv_tc(const float *x, const uint16_t *w, const float *b, float *y, int cin, int cout, int nb, int d,
                     int h, int wd, int relu, int mode);
int gb__unet_wgrad_tc(const float *x, const float *gy, float *gw, float *gb, int cin, int cout, int nb, int d, int h,
                      int wd);

// Deterministic sum of n partials into out (FP64), on the library stream.
int gb__sum_partials(const double *partial, long n, double *out_host);
