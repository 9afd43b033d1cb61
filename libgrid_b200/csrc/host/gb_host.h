/*
 * Internal interface of the libgrid-b200 C host layer.
 *
 * Every grid's host array (grid->value) is the key of a device block.  A
 * block holds the device copy in its storage precision, an optional shadow
 * copy in the other precision (refreshed on demand, invalidated by writes)
 * and two validity bits.  This is the single-GPU, no-swap replacement for the
 * reference's block cache (src/cuda.c:447-686): GPU operations make the
 * device copy authoritative, host-side accessors bring the host copy up to
 * date, and cuda_remove_block() keeps the reference's drop/copy-back meaning.
 */
#ifndef GB_HOST_H
#define GB_HOST_H

#include "grid.h"

#define GBH_HOST_VALID 1
#define GBH_DEV_VALID 2

typedef struct {
  void *host;       /* key */
  size_t nscalar;   /* FP64 scalars in the host array (2 per complex point) */
  int is_real;      /* rgrid (padded real) vs cgrid (complex) */
  int host_pinned;  /* host array allocated page-locked by this library */
  int prec;         /* device storage precision, GB_FP64 or GB_FP32 */
  void *dev;        /* device copy in prec */
  void *shadow;     /* device copy in the other precision */
  int shadow_valid;
  int state;
  int live;
} gbh_block;

/* Abort with a libgrid-style message (API misuse or device failure). */
void gbh_die(const char *fmt, ...);
/* Make sure the GPU is initialised (device from cuda_enable, else 0). */
void gbh_gpu(void);
/* Check the CUDA layer's status after a call; abort on failure. */
void gbh_check(int rc, const char *where);

void *gbh_alloc_host(size_t bytes, int *pinned);
void gbh_free_host(void *p, int pinned);

gbh_block *gbh_register(void *host, size_t nscalar, int is_real, int pinned);
gbh_block *gbh_find(const void *host);
void gbh_unregister(void *host);

/* Device access: the returned pointer holds the data in `prec`.
 * read: upload/convert if stale; write: the caller overwrites everything;
 * rw: read + mark device authoritative. */
void *gbh_dev_read(void *host, int prec);
void *gbh_dev_write(void *host, int prec);
void *gbh_dev_rw(void *host, int prec);
/* Host access. */
void gbh_host_read(void *host);
void gbh_host_modified(void *host);
/* Storage precision of a block (GB_FP64 if unknown). */
int gbh_prec(const void *host);
/* Change a block's storage precision, converting device data if present. */
void gbh_set_prec(void *host, int prec);

/* Geometry helper. */
gb_geom gbh_geom(INT nx, INT ny, INT nz, REAL step, int prec);

/* step^d factor used by the integrals (one step per axis of length != 1). */
REAL gbh_step_factor(INT nx, INT ny, INT nz, REAL step);

/* Boundary-condition code of a cgrid / rgrid (abort on custom functions). */
int gbh_cbc(const cgrid *grid, double *out_re, double *out_im);
int gbh_rbc(const rgrid *grid, double *out);

extern char grid_analyze_method;

#endif
