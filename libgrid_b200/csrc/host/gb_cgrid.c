/*
 * Complex grid API of libgrid-b200 (reference src/cgrid.c, src/cgrid_bc.c,
 * src/cgrid_diff.c).  Allocation, metadata and host-side accessors follow
 * the reference; every arithmetic operation runs on the GPU through the
 * gb_* CUDA layer on the grid's device copy.
 */
#include "gb_host.h"

static size_t npts(const cgrid *g) { return (size_t) (g->nx * g->ny * g->nz); }

static gb_geom geom_of(const cgrid *g, int prec) { return gbh_geom(g->nx, g->ny, g->nz, g->step, prec); }

/* Arithmetic precision of an operation over several complex grids: FP32 only
 * when every operand is stored in FP32. */
static int op_prec3(const cgrid *a, const cgrid *b, const cgrid *c) {
  int p = GB_FP32;
  if (a && gbh_prec(a->value) != GB_FP32) p = GB_FP64;
  if (b && gbh_prec(b->value) != GB_FP32) p = GB_FP64;
  if (c && gbh_prec(c->value) != GB_FP32) p = GB_FP64;
  return p;
}

/* Settle the output's storage precision before taking any device pointer,
 * so a conversion cannot free a buffer already handed out. */
static void out_prec(cgrid *c, int p) {
  if (gbh_prec(c->value) != p) gbh_set_prec(c->value, p);
}

static void same_shape(const cgrid *a, const cgrid *b, const char *fn) {
  if (a->nx != b->nx || a->ny != b->ny || a->nz != b->nz) gbh_die("Different grid dimensions in %s.", fn);
}

/* src/cgrid.c:45-158 */
cgrid *cgrid_alloc(INT nx, INT ny, INT nz, REAL step, REAL complex (*value_outside)(cgrid *grid, INT i, INT j, INT k),
                   void *outside_params_ptr, char *id) {
  cgrid *grid;
  int pinned = 0;
  size_t len;

  if (nx < 1 || ny < 1 || nz < 1) {
    fprintf(stderr, "libgrid: Error in cgrid_alloc(). Invalid grid dimensions.\n");
    return NULL;
  }
  if (!(grid = (cgrid *) malloc(sizeof(cgrid)))) {
    fprintf(stderr, "libgrid: Error in cgrid_alloc(). Could not allocate memory for grid structure.\n");
    abort();
  }
  memset(grid, 0, sizeof(cgrid));
  grid->nx = nx;
  grid->ny = ny;
  grid->nz = nz;
  grid->grid_len = len = ((size_t) (nx * ny * nz)) * sizeof(REAL complex);
  grid->step = step;
  if (!(grid->value = (REAL complex *) gbh_alloc_host(len, &pinned))) {
    fprintf(stderr, "libgrid: Error in cgrid_alloc(). Could not allocate memory for cgrid->value.\n");
    abort();
  }
  grid->x0 = grid->y0 = grid->z0 = 0.0;
  grid->kx0 = grid->ky0 = grid->kz0 = 0.0;
  grid->omega = 0.0;
  grid->fft_norm = 1.0 / (REAL) (grid->nx * grid->ny * grid->nz);
  grid->fft_norm2 = grid->fft_norm;
  if (grid->nx > 1) grid->fft_norm2 *= grid->step;
  if (grid->ny > 1) grid->fft_norm2 *= grid->step;
  if (grid->nz > 1) grid->fft_norm2 *= grid->step;
  strncpy(grid->id, id ? id : "", 32);
  grid->id[31] = 0;
  grid->value_outside = value_outside ? value_outside : cgrid_value_outside_dirichlet;
  if (outside_params_ptr) grid->outside_params_ptr = outside_params_ptr;
  else {
    grid->default_outside_params = 0.0;
    grid->outside_params_ptr = &grid->default_outside_params;
  }
  grid->plan = grid->iplan = NULL;
  grid->cufft_handle = -1;
  grid->host_lock = 0;
  memset(grid->value, 0, len);
  grid->flag = 0;
  gbh_register(grid->value, 2 * (size_t) (nx * ny * nz), 0, pinned);
  if (grid_analyze_method == -1) grid_analyze_method = 0; /* finite differences on one GPU */
  return grid;
}

/* src/cgrid.c:169-210 */
cgrid *cgrid_clone(cgrid *grid, char *id) {
  cgrid *ng;
  int pinned = 0;
  if (!(ng = (cgrid *) malloc(sizeof(cgrid)))) {
    fprintf(stderr, "libgrid: Out of memory in cgrid_clone().\n");
    abort();
  }
  memcpy(ng, grid, sizeof(cgrid));
  strncpy(ng->id, id ? id : "", 32);
  ng->id[31] = 0;
  if (!(ng->value = (REAL complex *) gbh_alloc_host(ng->grid_len, &pinned))) {
    fprintf(stderr, "libgrid: Error in cgrid_clone(). Could not allocate memory for grid.\n");
    free(ng);
    abort();
  }
  memset(ng->value, 0, ng->grid_len);
  if (grid->outside_params_ptr == &grid->default_outside_params) ng->outside_params_ptr = &ng->default_outside_params;
  ng->plan = ng->iplan = NULL;
  ng->host_lock = 0;
  ng->flag = 0;
  gbh_register(ng->value, 2 * npts(ng), 0, pinned);
  if (gbh_prec(grid->value) == GB_FP32) gbh_set_prec(ng->value, GB_FP32);
  return ng;
}

/* src/cgrid.c:332-349 */
void cgrid_free(cgrid *grid) {
  if (!grid) return;
  gbh_block *b = gbh_find(grid->value);
  int pinned = b ? b->host_pinned : 0;
  gbh_unregister(grid->value);
  gbh_free_host(grid->value, pinned);
  free(grid);
}

void cgrid_set_origin(cgrid *grid, REAL x0, REAL y0, REAL z0) {
  grid->x0 = x0;
  grid->y0 = y0;
  grid->z0 = z0;
}

void cgrid_shift_origin(cgrid *grid, REAL x0, REAL y0, REAL z0) {
  grid->x0 += x0;
  grid->y0 += y0;
  grid->z0 += z0;
}

void cgrid_set_momentum(cgrid *grid, REAL kx0, REAL ky0, REAL kz0) {
  grid->kx0 = kx0;
  grid->ky0 = ky0;
  grid->kz0 = kz0;
}

void cgrid_set_rotation(cgrid *grid, REAL omega) { grid->omega = omega; }

/* src/cgrid.c:360-370: nx, ny, nz (INT), step (REAL), values */
void cgrid_write(cgrid *grid, FILE *out) {
  gbh_host_read(grid->value);
  fwrite(&grid->nx, sizeof(INT), 1, out);
  fwrite(&grid->ny, sizeof(INT), 1, out);
  fwrite(&grid->nz, sizeof(INT), 1, out);
  fwrite(&grid->step, sizeof(REAL), 1, out);
  fwrite(grid->value, sizeof(REAL complex), npts(grid), out);
}

/* src/cgrid.c:2126-2151: dest = trilinear interpolation of src at dest's
 * points (src's boundary rule outside src), on the GPU. */
void cgrid_extrapolate(cgrid *dest, cgrid *src) {
  if (dest == src) {
    fprintf(stderr, "libgrid: Source and destination grids cannot be the same in cgrid_extrapolate().\n");
    abort();
  }
  double ore, oim;
  const int bc = gbh_cbc(src, &ore, &oim);
  const gb_grid_frame d = {dest->nx, dest->ny, dest->nz, dest->nz, dest->step, dest->x0, dest->y0, dest->z0};
  const gb_grid_frame s = {src->nx, src->ny, src->nz, src->nz, src->step, src->x0, src->y0, src->z0};
  out_prec(dest, GB_FP64);
  const void *ds = gbh_dev_read(src->value, GB_FP64);
  void *dd = gbh_dev_write(dest->value, GB_FP64);
  gbh_check(gb_interpolate(dd, &d, ds, &s, bc, ore, oim, 0), "cgrid_extrapolate");
}

/* src/cgrid.c:383-420: a file of another size or step is read into a
 * temporary grid and interpolated onto `grid` (cgrid_extrapolate). */
cgrid *cgrid_read(cgrid *grid, FILE *in) {
  INT nx, ny, nz;
  REAL step;
  if (fread(&nx, sizeof(INT), 1, in) != 1 || fread(&ny, sizeof(INT), 1, in) != 1 || fread(&nz, sizeof(INT), 1, in) != 1 ||
      fread(&step, sizeof(REAL), 1, in) != 1) {
    fprintf(stderr, "libgrid: Error reading grid header in cgrid_read().\n");
    return NULL;
  }
  if (!grid) {
    if (!(grid = cgrid_alloc(nx, ny, nz, step, CGRID_PERIODIC_BOUNDARY, NULL, "read_grid"))) {
      fprintf(stderr, "libgrid: Failed to allocate grid in cgrid_read().\n");
      return NULL;
    }
  }
  if (nx != grid->nx || ny != grid->ny || nz != grid->nz || step != grid->step) {
    cgrid *tmp;
    fprintf(stderr, "libgrid: Grid in file has different size than grid in memory.\n");
    fprintf(stderr, "libgrid: Interpolating between grids.\n");
    if (!(tmp = cgrid_alloc(nx, ny, nz, step, grid->value_outside, NULL, "cgrid_read_temp"))) {
      fprintf(stderr, "libgrid: Error allocating grid in cgrid_read().\n");
      abort();
    }
    if (fread(tmp->value, sizeof(REAL complex), npts(tmp), in) != npts(tmp))
      fprintf(stderr, "libgrid: Short read in cgrid_read().\n");
    gbh_host_modified(tmp->value);
    cgrid_extrapolate(grid, tmp);
    cgrid_free(tmp);
    return grid;
  }
  if (fread(grid->value, sizeof(REAL complex), npts(grid), in) != npts(grid)) {
    fprintf(stderr, "libgrid: Short read in cgrid_read().\n");
  }
  gbh_host_modified(grid->value);
  return grid;
}

/* src/cgrid.c:615-646 */
void cgrid_copy(cgrid *dst, cgrid *src) {
  if (src->nx != dst->nx || src->ny != dst->ny || src->nz != dst->nz) {
    fprintf(stderr, "libgrid: Different grid dimensions in cgrid_copy.\n");
    abort();
  }
  dst->step = src->step;
  dst->x0 = src->x0;
  dst->y0 = src->y0;
  dst->z0 = src->z0;
  dst->kx0 = src->kx0;
  dst->ky0 = src->ky0;
  dst->kz0 = src->kz0;
  if (dst == src) return;
  gbh_block *bs = gbh_find(src->value);
  if (bs && (bs->state & GBH_DEV_VALID)) {
    const int p = gbh_prec(dst->value);
    const int esz = (p == GB_FP32) ? 8 : 16;
    void *s = gbh_dev_read(src->value, p);
    void *d = gbh_dev_write(dst->value, p);
    gbh_check(gb_d2d(d, s, npts(src) * (size_t) esz), "cgrid_copy");
  } else {
    memcpy(dst->value, src->value, npts(src) * sizeof(REAL complex));
    gbh_host_modified(dst->value);
  }
}

void cgrid_zero(cgrid *grid) { cgrid_constant(grid, 0.0); }

/* src/cgrid.c:725-741 */
void cgrid_constant(cgrid *grid, REAL complex c) {
  const int p = gbh_prec(grid->value);
  void *d = gbh_dev_write(grid->value, p);
  gbh_check(gb_complex_op(GB_OP_CONST, d, NULL, NULL, npts(grid), creal(c), cimag(c), p), "cgrid_constant");
}

/* src/cgrid.c:793-819 (host-side mapping; the device copy is dropped) */
void cgrid_map(cgrid *grid, REAL complex (*func)(void *arg, REAL x, REAL y, REAL z), void *farg) {
  INT i, j, k, nx = grid->nx, ny = grid->ny, nz = grid->nz;
  REAL x, y, z, step = grid->step;
  for (i = 0; i < nx; i++) {
    x = ((REAL) (i - nx / 2)) * step - grid->x0;
    for (j = 0; j < ny; j++) {
      y = ((REAL) (j - ny / 2)) * step - grid->y0;
      for (k = 0; k < nz; k++) {
        z = ((REAL) (k - nz / 2)) * step - grid->z0;
        grid->value[(i * ny + j) * nz + k] = func(farg, x, y, z);
      }
    }
  }
  gbh_host_modified(grid->value);
}

static void binary(int op, cgrid *c, cgrid *a, cgrid *b, const char *fn) {
  same_shape(c, a, fn);
  if (b) same_shape(c, b, fn);
  const int p = op_prec3(c, a, b);
  out_prec(c, p);
  const void *da = gbh_dev_read(a->value, p);
  const void *db = b ? gbh_dev_read(b->value, p) : NULL;
  void *dc = gbh_dev_write(c->value, p);
  gbh_check(gb_complex_op(op, dc, da, db, npts(c), 0.0, 0.0, p), fn);
}

/* src/cgrid.c:1912-1944: c = (-1)^(i+j+k) a b in k-space */
void cgrid_fft_convolute(cgrid *gridc, cgrid *grida, cgrid *gridb) {
  same_shape(gridc, grida, "cgrid_fft_convolute");
  same_shape(gridc, gridb, "cgrid_fft_convolute");
  const int p = op_prec3(gridc, grida, gridb);
  out_prec(gridc, p);
  const void *da = gbh_dev_read(grida->value, p);
  const void *db = gbh_dev_read(gridb->value, p);
  void *dc = gbh_dev_write(gridc->value, p);
  gbh_check(gb_fft_convolute(dc, da, db, gridc->nx, gridc->ny, gridc->nz, p), "cgrid_fft_convolute");
}

/* src/cgrid.c:934,964,994,1169 */
void cgrid_sum(cgrid *gridc, cgrid *grida, cgrid *gridb) { binary(GB_OP_SUM, gridc, grida, gridb, "cgrid_sum"); }
void cgrid_difference(cgrid *gridc, cgrid *grida, cgrid *gridb) { binary(GB_OP_DIFF, gridc, grida, gridb, "cgrid_difference"); }
void cgrid_product(cgrid *gridc, cgrid *grida, cgrid *gridb) { binary(GB_OP_PRODUCT, gridc, grida, gridb, "cgrid_product"); }
void cgrid_conjugate_product(cgrid *gridc, cgrid *grida, cgrid *gridb) {
  binary(GB_OP_CONJ_PRODUCT, gridc, grida, gridb, "cgrid_conjugate_product");
}

/* src/cgrid.c:1197,1223 */
void cgrid_add(cgrid *grid, REAL complex c) {
  const int p = gbh_prec(grid->value);
  gbh_check(gb_complex_op(GB_OP_ADD_CONST, gbh_dev_rw(grid->value, p), NULL, NULL, npts(grid), creal(c), cimag(c), p),
            "cgrid_add");
}

void cgrid_multiply(cgrid *grid, REAL complex c) {
  const int p = gbh_prec(grid->value);
  gbh_check(gb_complex_op(GB_OP_SCALE, gbh_dev_rw(grid->value, p), NULL, NULL, npts(grid), creal(c), cimag(c), p),
            "cgrid_multiply");
}

/* src/cgrid.c:1303,1333 */
void cgrid_add_scaled(cgrid *gridc, REAL complex d, cgrid *grida) {
  same_shape(gridc, grida, "cgrid_add_scaled");
  const int p = op_prec3(gridc, grida, NULL);
  out_prec(gridc, p);
  const void *da = gbh_dev_read(grida->value, p);
  void *dc = gbh_dev_rw(gridc->value, p);
  gbh_check(gb_complex_op(GB_OP_ADD_SCALED, dc, da, NULL, npts(gridc), creal(d), cimag(d), p), "cgrid_add_scaled");
}

void cgrid_add_scaled_product(cgrid *gridc, REAL complex d, cgrid *grida, cgrid *gridb) {
  same_shape(gridc, grida, "cgrid_add_scaled_product");
  same_shape(gridc, gridb, "cgrid_add_scaled_product");
  const int p = op_prec3(gridc, grida, gridb);
  out_prec(gridc, p);
  const void *da = gbh_dev_read(grida->value, p);
  const void *db = gbh_dev_read(gridb->value, p);
  void *dc = gbh_dev_rw(gridc->value, p);
  gbh_check(gb_complex_op(GB_OP_ADD_SCALED_PRODUCT, dc, da, db, npts(gridc), creal(d), cimag(d), p),
            "cgrid_add_scaled_product");
}

/* Reductions (src/cgrid.c:1536-1700): device sum, then the step^d factor. */
static void reduce(int op, cgrid *a, const void *bdev, int bprec, long brow, double out[2], const char *fn) {
  const int p = gbh_prec(a->value);
  gb_geom g = geom_of(a, p);
  gbh_check(gb_reduce(op, gbh_dev_read(a->value, p), bdev, &g, a->nz, brow, bprec, out), fn);
}

REAL complex cgrid_integral(cgrid *grid) {
  double r[2];
  reduce(GB_RED_SUM, grid, NULL, GB_FP64, 0, r, "cgrid_integral");
  return (r[0] + I * r[1]) * gbh_step_factor(grid->nx, grid->ny, grid->nz, grid->step);
}

REAL cgrid_integral_of_square(cgrid *grid) {
  double r[2];
  reduce(GB_RED_NORM2, grid, NULL, GB_FP64, 0, r, "cgrid_integral_of_square");
  return r[0] * gbh_step_factor(grid->nx, grid->ny, grid->nz, grid->step);
}

REAL complex cgrid_integral_of_conjugate_product(cgrid *grida, cgrid *gridb) {
  double r[2];
  same_shape(grida, gridb, "cgrid_integral_of_conjugate_product");
  const int pb = gbh_prec(gridb->value);
  reduce(GB_RED_CONJ_PRODUCT, grida, gbh_dev_read(gridb->value, pb), pb, gridb->nz, r, "cgrid_integral_of_conjugate_product");
  return (r[0] + I * r[1]) * gbh_step_factor(grida->nx, grida->ny, grida->nz, grida->step);
}

REAL complex cgrid_grid_expectation_value(cgrid *dgrid, cgrid *opgrid) {
  double r[2];
  same_shape(dgrid, opgrid, "cgrid_grid_expectation_value");
  const int pb = gbh_prec(opgrid->value);
  reduce(GB_RED_EXPECT_COMPLEX, dgrid, gbh_dev_read(opgrid->value, pb), pb, opgrid->nz, r, "cgrid_grid_expectation_value");
  return (r[0] + I * r[1]) * gbh_step_factor(dgrid->nx, dgrid->ny, dgrid->nz, dgrid->step);
}

/* FFTs (src/cgrid.c:1822-1890) */
void cgrid_fft(cgrid *grid) {
  const int p = gbh_prec(grid->value);
  gb_geom g = geom_of(grid, p);
  gbh_check(gb_fft3d(gbh_dev_rw(grid->value, p), &g, -1, 1.0), "cgrid_fft");
}

void cgrid_inverse_fft(cgrid *grid) {
  const int p = gbh_prec(grid->value);
  gb_geom g = geom_of(grid, p);
  gbh_check(gb_fft3d(gbh_dev_rw(grid->value, p), &g, +1, 1.0), "cgrid_inverse_fft");
}

void cgrid_scaled_inverse_fft(cgrid *grid, REAL complex c) {
  const int p = gbh_prec(grid->value);
  gb_geom g = geom_of(grid, p);
  void *d = gbh_dev_rw(grid->value, p);
  if (cimag(c) == 0.0) {
    gbh_check(gb_fft3d(d, &g, +1, creal(c)), "cgrid_scaled_inverse_fft");
  } else {
    gbh_check(gb_fft3d(d, &g, +1, 1.0), "cgrid_scaled_inverse_fft");
    gbh_check(gb_complex_op(GB_OP_SCALE, d, NULL, NULL, npts(grid), creal(c), cimag(c), p), "cgrid_scaled_inverse_fft");
  }
}

void cgrid_inverse_fft_norm(cgrid *grid) { cgrid_scaled_inverse_fft(grid, grid->fft_norm); }
void cgrid_inverse_fft_norm2(cgrid *grid) { cgrid_scaled_inverse_fft(grid, grid->fft_norm2); }

/* src/cgrid.c:1960-2000 */
REAL complex cgrid_value_at_index(cgrid *grid, INT i, INT j, INT k) {
  if (i < 0 || j < 0 || k < 0 || i >= grid->nx || j >= grid->ny || k >= grid->nz) return grid->value_outside(grid, i, j, k);
  const size_t idx = (size_t) ((i * grid->ny + j) * grid->nz + k);
  gbh_block *b = gbh_find(grid->value);
  if (!b || (b->state & GBH_HOST_VALID)) return grid->value[idx];
  if (b->prec == GB_FP64) {
    REAL complex v;
    gbh_check(gb_d2h(&v, (const char *) b->dev + idx * 16, 16), "cgrid_value_at_index");
    return v;
  } else {
    float v[2];
    gbh_check(gb_d2h(v, (const char *) b->dev + idx * 8, 8), "cgrid_value_at_index");
    return (REAL) v[0] + I * (REAL) v[1];
  }
}

/* src/cgrid.c:2016-2054 */
void cgrid_value_to_index(cgrid *grid, INT i, INT j, INT k, REAL complex value) {
  if (i < 0 || j < 0 || k < 0 || i >= grid->nx || j >= grid->ny || k >= grid->nz) return;
  const size_t idx = (size_t) ((i * grid->ny + j) * grid->nz + k);
  gbh_block *b = gbh_find(grid->value);
  if (b && (b->state & GBH_DEV_VALID)) {
    if (b->prec == GB_FP64) {
      gbh_check(gb_h2d((char *) b->dev + idx * 16, &value, 16), "cgrid_value_to_index");
    } else {
      float v[2] = {(float) creal(value), (float) cimag(value)};
      gbh_check(gb_h2d((char *) b->dev + idx * 8, v, 8), "cgrid_value_to_index");
    }
    gbh_check(gb_synchronize(), "cgrid_value_to_index");
    b->shadow_valid = 0;
    if (b->state & GBH_HOST_VALID) grid->value[idx] = value;
    return;
  }
  grid->value[idx] = value;
  if (b) gbh_host_modified(grid->value);
}

/* src/cgrid_bc.c:21-86 */
REAL complex cgrid_value_outside_dirichlet(cgrid *grid, INT i, INT j, INT k) {
  (void) i;
  (void) j;
  (void) k;
  return *((REAL complex *) grid->outside_params_ptr);
}

REAL complex cgrid_value_outside_neumann(cgrid *grid, INT i, INT j, INT k) {
  INT nx = grid->nx, ny = grid->ny, nz = grid->nz;
  if (i < 0) i = -i;
  if (i > nx - 1) i = 2 * nx - i - 2;
  if (j < 0) j = -j;
  if (j > ny - 1) j = 2 * ny - j - 2;
  if (k < 0) k = -k;
  if (k > nz - 1) k = 2 * nz - k - 2;
  /* an axis of length 1 mirrors back outside; use its single plane */
  if (i < 0 || i >= nx) i = 0;
  if (j < 0 || j >= ny) j = 0;
  if (k < 0 || k >= nz) k = 0;
  return cgrid_value_at_index(grid, i, j, k);
}

REAL complex cgrid_value_outside_periodic(cgrid *grid, INT i, INT j, INT k) {
  INT nx = grid->nx, ny = grid->ny, nz = grid->nz;
  i %= nx;
  if (i < 0) i = nx + i;
  j %= ny;
  if (j < 0) j = ny + j;
  k %= nz;
  if (k < 0) k = nz + k;
  return cgrid_value_at_index(grid, i, j, k);
}

/* Finite differences (src/cgrid_diff.c:201-442). */
static void fd(int op, cgrid *grid, cgrid *out, double coef, const char *fn) {
  if (grid == out) {
    fprintf(stderr, "libgrid: source and destination must be different in %s().\n", fn);
    abort();
  }
  same_shape(grid, out, fn);
  double ore, oim;
  const int bc = gbh_cbc(grid, &ore, &oim);
  const int p = op_prec3(grid, out, NULL);
  out_prec(out, p);
  gb_geom g = geom_of(grid, p);
  const void *s = gbh_dev_read(grid->value, p);
  void *d = gbh_dev_write(out->value, p);
  gbh_check(gb_fd(op, d, s, &g, bc, ore, oim, coef, 0, grid->nz), fn);
}

void cgrid_fd_gradient_x(cgrid *grid, cgrid *gradient) { fd(GB_FD_GRADIENT_X, grid, gradient, 1.0 / (2.0 * grid->step), "cgrid_fd_gradient_x"); }
void cgrid_fd_gradient_y(cgrid *grid, cgrid *gradient) { fd(GB_FD_GRADIENT_Y, grid, gradient, 1.0 / (2.0 * grid->step), "cgrid_fd_gradient_y"); }
void cgrid_fd_gradient_z(cgrid *grid, cgrid *gradient) { fd(GB_FD_GRADIENT_Z, grid, gradient, 1.0 / (2.0 * grid->step), "cgrid_fd_gradient_z"); }
void cgrid_fd_laplace(cgrid *grid, cgrid *laplace) { fd(GB_FD_LAPLACE, grid, laplace, 1.0 / (grid->step * grid->step), "cgrid_fd_laplace"); }
void cgrid_fd_laplace_x(cgrid *grid, cgrid *laplacex) { fd(GB_FD_LAPLACE_X, grid, laplacex, 1.0 / (grid->step * grid->step), "cgrid_fd_laplace_x"); }
void cgrid_fd_laplace_y(cgrid *grid, cgrid *laplacey) { fd(GB_FD_LAPLACE_Y, grid, laplacey, 1.0 / (grid->step * grid->step), "cgrid_fd_laplace_y"); }
void cgrid_fd_laplace_z(cgrid *grid, cgrid *laplacez) { fd(GB_FD_LAPLACE_Z, grid, laplacez, 1.0 / (grid->step * grid->step), "cgrid_fd_laplace_z"); }

/* k-space derivatives (src/cgrid_diff.c:454-807); the destination receives
 * the source's metadata as the reference's cgrid_copy does. */
static void kspace(int op, cgrid *grid, cgrid *out, const char *fn) {
  same_shape(grid, out, fn);
  if (out != grid) {
    out->step = grid->step;
    out->x0 = grid->x0;
    out->y0 = grid->y0;
    out->z0 = grid->z0;
    out->kx0 = grid->kx0;
    out->ky0 = grid->ky0;
    out->kz0 = grid->kz0;
  }
  const int p = op_prec3(grid, out, NULL);
  out_prec(out, p);
  gb_geom g = geom_of(grid, p);
  const void *s = gbh_dev_read(grid->value, p);
  void *d = (out == grid) ? gbh_dev_rw(out->value, p) : gbh_dev_write(out->value, p);
  gbh_check(gb_kspace_op(op, d, s, &g), fn);
}

void cgrid_fft_gradient_x(cgrid *grid, cgrid *gradient_x) { kspace(GB_K_GRADIENT_X, grid, gradient_x, "cgrid_fft_gradient_x"); }
void cgrid_fft_gradient_y(cgrid *grid, cgrid *gradient_y) { kspace(GB_K_GRADIENT_Y, grid, gradient_y, "cgrid_fft_gradient_y"); }
void cgrid_fft_gradient_z(cgrid *grid, cgrid *gradient_z) { kspace(GB_K_GRADIENT_Z, grid, gradient_z, "cgrid_fft_gradient_z"); }
void cgrid_fft_laplace(cgrid *grid, cgrid *laplace) { kspace(GB_K_LAPLACE, grid, laplace, "cgrid_fft_laplace"); }

/* src/cgrid_diff.c:817-879: sum -(k^2) |grid_k|^2 * fft_norm2 on a k-space grid */
REAL cgrid_fft_laplace_expectation_value(cgrid *grid) {
  double r[2];
  reduce(GB_RED_KSQ_NORM2, grid, NULL, GB_FP64, 0, r, "cgrid_fft_laplace_expectation_value");
  return -r[0] * grid->fft_norm2;
}

/* src/cgrid_diff.c:125-133 */
void cgrid_laplace(cgrid *grid, cgrid *laplace) {
  if (grid_analyze_method > 0) {
    cgrid_copy(laplace, grid);
    cgrid_fft(laplace);
    cgrid_fft_laplace(laplace, laplace);
    cgrid_inverse_fft_norm(laplace);
  } else cgrid_fd_laplace(grid, laplace);
}
