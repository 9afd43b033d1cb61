/*
 * libgrid-b200 host runtime: device-block table, host/device coherence,
 * GPU selection and the reference's setup entry points
 * (src/threads.c:89-157, src/cuda.c:477-499,1142-1199,
 * src/grid_wf_analyze.c:10-24).
 */
#include <stdarg.h>
#include <stdint.h>
#include <unistd.h>

#include "gb_host.h"

/* 0 = finite difference, 1 = FFT, -1 = not yet chosen (the first grid
 * allocation picks finite difference on one GPU, src/cgrid.c:141-149). */
char grid_analyze_method = (char) -1;

static INT g_threads = 0;
static int g_gpu_ready = 0;
static int g_device = 0;
static char g_cuda_enabled = 0;

void gbh_die(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, "libgrid(b200): ");
  vfprintf(stderr, fmt, ap);
  fprintf(stderr, "\n");
  va_end(ap);
  abort();
}

void gbh_gpu(void) {
  if (g_gpu_ready) return;
  const char *env = getenv("LIBGRID_B200_DEVICE");
  int dev = g_device;
  if (env && *env) dev = atoi(env);
  else if (!g_cuda_enabled && getenv("LOCAL_RANK")) dev = atoi(getenv("LOCAL_RANK"));
  if (gb_init(dev)) gbh_die("cannot initialise CUDA device %d (error %d at %s); this library has no CPU path", dev,
                            gb_last_error(), gb_last_error_where());
  g_device = dev;
  g_gpu_ready = 1;
  g_cuda_enabled = 1;
}

void gbh_check(int rc, const char *where) {
  if (rc) gbh_die("%s failed: CUDA layer error %d (%s)", where, rc, gb_last_error_where());
}

void *gbh_alloc_host(size_t bytes, int *pinned) {
  void *p = NULL;
  *pinned = 0;
  if (g_gpu_ready) {
    p = gb_host_alloc(bytes);
    if (p) {
      *pinned = 1;
      return p;
    }
  }
  if (posix_memalign(&p, 64, bytes ? bytes : 64)) return NULL;
  return p;
}

void gbh_free_host(void *p, int pinned) {
  if (!p) return;
  if (pinned) gb_host_free(p);
  else free(p);
}

/* ------------------------------------------------------------ block table */

static gbh_block *g_tab = NULL;
static size_t g_cap = 0, g_used = 0;

static size_t hash_ptr(const void *p) {
  uint64_t x = (uint64_t) (uintptr_t) p;
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  return (size_t) x;
}

static void tab_grow(void) {
  size_t ncap = g_cap ? 2 * g_cap : 256;
  gbh_block *nt = (gbh_block *) calloc(ncap, sizeof(gbh_block));
  if (!nt) gbh_die("out of host memory for the device-block table");
  for (size_t i = 0; i < g_cap; i++) {
    if (!g_tab[i].live) continue;
    size_t h = hash_ptr(g_tab[i].host) & (ncap - 1);
    while (nt[h].live) h = (h + 1) & (ncap - 1);
    nt[h] = g_tab[i];
  }
  free(g_tab);
  g_tab = nt;
  g_cap = ncap;
}

gbh_block *gbh_find(const void *host) {
  if (!g_cap || !host) return NULL;
  size_t h = hash_ptr(host) & (g_cap - 1);
  for (size_t n = 0; n < g_cap; n++) {
    gbh_block *b = &g_tab[h];
    if (!b->live && !b->host) return NULL; /* empty, never used */
    if (b->live && b->host == host) return b;
    h = (h + 1) & (g_cap - 1);
  }
  return NULL;
}

gbh_block *gbh_register(void *host, size_t nscalar, int is_real, int pinned) {
  if (2 * (g_used + 1) > g_cap) tab_grow();
  size_t h = hash_ptr(host) & (g_cap - 1);
  while (g_tab[h].live) h = (h + 1) & (g_cap - 1);
  gbh_block *b = &g_tab[h];
  memset(b, 0, sizeof(*b));
  b->host = host;
  b->nscalar = nscalar;
  b->is_real = is_real;
  b->host_pinned = pinned;
  b->prec = GB_FP64;
  b->state = GBH_HOST_VALID;
  b->live = 1;
  g_used++;
  return b;
}

void gbh_unregister(void *host) {
  gbh_block *b = gbh_find(host);
  if (!b) return;
  if (b->dev) gb_device_free(b->dev);
  if (b->shadow) gb_device_free(b->shadow);
  b->dev = b->shadow = NULL;
  b->live = 0; /* keep host as a tombstone so probes continue */
  g_used--;
}

static gbh_block *need(const void *host) {
  gbh_block *b = gbh_find(host);
  if (!b) gbh_die("grid data %p is not a grid allocated by this library", host);
  return b;
}

static size_t dev_bytes(const gbh_block *b, int prec) { return b->nscalar * (prec == GB_FP32 ? 4 : 8); }

static void ensure_dev(gbh_block *b) {
  gbh_gpu();
  if (!b->dev) {
    b->dev = gb_device_alloc(dev_bytes(b, b->prec));
    if (!b->dev) gbh_die("out of device memory (%zu bytes)", dev_bytes(b, b->prec));
  }
}

static void upload(gbh_block *b) {
  ensure_dev(b);
  if (b->prec == GB_FP64) gbh_check(gb_h2d(b->dev, b->host, b->nscalar * 8), "host->device copy");
  else gbh_check(gb_upload_f64_as_f32(b->dev, b->host, b->nscalar), "host->device copy");
  b->state |= GBH_DEV_VALID;
}

static void download(gbh_block *b) {
  if (b->prec == GB_FP64) gbh_check(gb_d2h(b->host, b->dev, b->nscalar * 8), "device->host copy");
  else gbh_check(gb_download_f32_as_f64(b->host, b->dev, b->nscalar), "device->host copy");
  b->state |= GBH_HOST_VALID;
}

static void *primary(gbh_block *b, int need_valid) {
  if (need_valid && !(b->state & GBH_DEV_VALID)) upload(b);
  else ensure_dev(b);
  return b->dev;
}

static void *shadow_of(gbh_block *b, int prec) {
  if (!b->shadow_valid) {
    primary(b, 1);
    if (!b->shadow) {
      b->shadow = gb_device_alloc(dev_bytes(b, prec));
      if (!b->shadow) gbh_die("out of device memory (%zu bytes)", dev_bytes(b, prec));
    }
    if (prec == GB_FP32) gbh_check(gb_convert_f64_to_f32(b->shadow, b->dev, b->nscalar), "precision shadow");
    else gbh_check(gb_convert_f32_to_f64(b->shadow, b->dev, b->nscalar), "precision shadow");
    b->shadow_valid = 1;
  }
  return b->shadow;
}

void *gbh_dev_read(void *host, int prec) {
  gbh_block *b = need(host);
  if (prec == b->prec) return primary(b, 1);
  return shadow_of(b, prec);
}

void *gbh_dev_write(void *host, int prec) {
  gbh_block *b = need(host);
  if (prec != b->prec) gbh_set_prec(host, prec);
  primary(b, 0);
  b->state = GBH_DEV_VALID;
  b->shadow_valid = 0;
  return b->dev;
}

void *gbh_dev_rw(void *host, int prec) {
  gbh_block *b = need(host);
  if (prec != b->prec) gbh_set_prec(host, prec);
  primary(b, 1);
  b->state = GBH_DEV_VALID;
  b->shadow_valid = 0;
  return b->dev;
}

void gbh_host_read(void *host) {
  gbh_block *b = need(host);
  if (!(b->state & GBH_HOST_VALID)) download(b);
}

void gbh_host_modified(void *host) {
  gbh_block *b = need(host);
  b->state = GBH_HOST_VALID;
  b->shadow_valid = 0;
}

int gbh_prec(const void *host) {
  gbh_block *b = gbh_find(host);
  return b ? b->prec : GB_FP64;
}

void gbh_set_prec(void *host, int prec) {
  gbh_block *b = need(host);
  if (b->prec == prec) return;
  if (b->state & GBH_DEV_VALID) {
    /* convert the device copy; the old primary becomes the (valid) shadow */
    void *nd = gb_device_alloc(dev_bytes(b, prec));
    if (!nd) gbh_die("out of device memory (%zu bytes)", dev_bytes(b, prec));
    if (prec == GB_FP32) gbh_check(gb_convert_f64_to_f32(nd, b->dev, b->nscalar), "precision change");
    else gbh_check(gb_convert_f32_to_f64(nd, b->dev, b->nscalar), "precision change");
    if (b->shadow) gb_device_free(b->shadow);
    b->shadow = b->dev;
    b->shadow_valid = 1;
    b->dev = nd;
  } else {
    /* host copy is authoritative: drop device buffers, upload later */
    if (b->dev) gb_device_free(b->dev);
    if (b->shadow) gb_device_free(b->shadow);
    b->dev = b->shadow = NULL;
    b->shadow_valid = 0;
  }
  b->prec = prec;
}

gb_geom gbh_geom(INT nx, INT ny, INT nz, REAL step, int prec) {
  gb_geom g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.step = step;
  g.prec = prec;
  return g;
}

REAL gbh_step_factor(INT nx, INT ny, INT nz, REAL step) {
  REAL f = 1.0;
  if (nx != 1) f *= step;
  if (ny != 1) f *= step;
  if (nz != 1) f *= step;
  return f;
}

int gbh_cbc(const cgrid *grid, double *out_re, double *out_im) {
  *out_re = *out_im = 0.0;
  if (grid->value_outside == cgrid_value_outside_dirichlet) {
    REAL complex v = *((REAL complex *) grid->outside_params_ptr);
    *out_re = creal(v);
    *out_im = cimag(v);
    return GB_BC_DIRICHLET;
  }
  if (grid->value_outside == cgrid_value_outside_neumann) return GB_BC_NEUMANN;
  if (grid->value_outside == cgrid_value_outside_periodic) return GB_BC_PERIODIC;
  gbh_die("Incompatible boundary condition (only the Dirichlet, Neumann and periodic functions run on the GPU).");
  return 0;
}

int gbh_rbc(const rgrid *grid, double *out) {
  *out = 0.0;
  if (grid->value_outside == rgrid_value_outside_dirichlet) {
    *out = *((REAL *) grid->outside_params_ptr);
    return GB_BC_DIRICHLET;
  }
  if (grid->value_outside == rgrid_value_outside_neumann) return GB_BC_NEUMANN;
  if (grid->value_outside == rgrid_value_outside_periodic) return GB_BC_PERIODIC;
  gbh_die("Incompatible boundary condition (only the Dirichlet, Neumann and periodic functions run on the GPU).");
  return 0;
}

/* ---------------------------------------------------- reference setup API */

void grid_threads_init(INT threads) {
  if (threads < 0) {
    fprintf(stderr, "libgrid: Error in grid_threads_init(). Number of threads <= 0.\n");
    abort();
  }
  if (threads == 0) threads = (INT) sysconf(_SC_NPROCESSORS_ONLN);
  if (g_threads && g_threads != threads) {
    fprintf(stderr, "libgrid: Error in grid_threads_init(). This function was called twice with different number of threads.\n");
    abort();
  }
  g_threads = threads;
}

INT grid_threads(void) { return g_threads; }

void cuda_enable(char val, int ngpus, int *gpus) {
  if (!val) {
    /* There is no CPU path: disabling is recorded but GPU work continues. */
    fprintf(stderr, "libgrid(b200): cuda_enable(0) ignored: all grid operations run on the GPU.\n");
    return;
  }
  if (ngpus > 1) fprintf(stderr, "libgrid(b200): one GPU per process; using the first of %d requested.\n", ngpus);
  if (ngpus >= 1 && gpus) g_device = gpus[0];
  g_cuda_enabled = 1;
  gbh_gpu();
}

char cuda_status(void) { return (char) (g_gpu_ready ? 1 : 0); }

int cuda_remove_block(void *host_mem, char copy) {
  gbh_block *b = gbh_find(host_mem);
  if (!b) return 0;
  if (copy && !(b->state & GBH_HOST_VALID)) download(b);
  if (b->dev) gb_device_free(b->dev);
  if (b->shadow) gb_device_free(b->shadow);
  b->dev = b->shadow = NULL;
  b->shadow_valid = 0;
  b->state = GBH_HOST_VALID;
  return 0;
}

void cuda_free_all_blocks(char sync) {
  for (size_t i = 0; i < g_cap; i++)
    if (g_tab[i].live) cuda_remove_block(g_tab[i].host, sync);
}

void grid_wf_analyze_method(char method) { grid_analyze_method = method; }

/* Refresh the host copy of a grid without dropping its device copy. */
void gb_grid_sync_host(void *host_mem) {
  if (gbh_find(host_mem)) gbh_host_read(host_mem);
}

/* Declare that the caller rewrote a grid's host array directly. */
void gb_grid_host_modified(void *host_mem) {
  if (gbh_find(host_mem)) gbh_host_modified(host_mem);
}

/* FP64 device copy of a grid for device-side producers and consumers:
 * mode 0 read (uploaded if stale), 1 write (the caller overwrites every
 * value; the device copy becomes authoritative), 2 read and write. */
void *gb_grid_device(void *host_mem, int mode) {
  if (!gbh_find(host_mem)) return NULL;
  if (mode == 1) return gbh_dev_write(host_mem, GB_FP64);
  if (mode == 2) return gbh_dev_rw(host_mem, GB_FP64);
  return gbh_dev_read(host_mem, GB_FP64);
}
