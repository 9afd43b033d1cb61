/*
 * Real grid and mixed real/complex API of libgrid-b200 (reference
 * src/rgrid.c, src/rgrid_bc.c, src/rgrid_diff.c, src/ngrid.c).  Real grids
 * keep the reference's padded layout (rows of nz2 = 2 (nz/2 + 1) scalars,
 * src/rgrid.c:46-47) on the host and on the device.
 */
#include "gb_host.h"

static size_t nscal(const rgrid *g) { return (size_t) (g->nx * g->ny * g->nz2); }

static gb_geom geom_of(const rgrid *g, int prec) { return gbh_geom(g->nx, g->ny, g->nz, g->step, prec); }

/* src/rgrid.c:38-158 */
rgrid *rgrid_alloc(INT nx, INT ny, INT nz, REAL step, REAL (*value_outside)(rgrid *grid, INT i, INT j, INT k),
                   void *outside_params_ptr, char *id) {
  rgrid *grid;
  int pinned = 0;
  size_t len;
  if (nx < 1 || ny < 1 || nz < 1) {
    fprintf(stderr, "libgrid: Error in rgrid_alloc(). Invalid grid dimensions.\n");
    return NULL;
  }
  if (!(grid = (rgrid *) malloc(sizeof(rgrid)))) {
    fprintf(stderr, "libgrid: Error in rgrid_alloc(). Could not allocate memory for grid structure.\n");
    return NULL;
  }
  memset(grid, 0, sizeof(rgrid));
  grid->nx = nx;
  grid->ny = ny;
  grid->nz = nz;
  grid->nz2 = 2 * (nz / 2 + 1);
  grid->grid_len = len = ((size_t) (nx * ny * grid->nz2)) * sizeof(REAL);
  if (!(grid->value = (REAL *) gbh_alloc_host(len, &pinned))) {
    fprintf(stderr, "libgrid: Error in rgrid_alloc(). Could not allocate memory for rgrid->value.\n");
    abort();
  }
  grid->step = step;
  grid->value_outside = value_outside ? value_outside : rgrid_value_outside_dirichlet;
  if (outside_params_ptr) grid->outside_params_ptr = outside_params_ptr;
  else {
    grid->default_outside_params = 0.0;
    grid->outside_params_ptr = &grid->default_outside_params;
  }
  grid->plan = grid->iplan = NULL;
  grid->cufft_handle_r2c = grid->cufft_handle_c2r = -1;
  if (grid->value_outside == RGRID_NEUMANN_BOUNDARY)
    grid->fft_norm = 1.0 / (2.0 * ((REAL) grid->nx) * 2.0 * ((REAL) grid->ny) * 2.0 * ((REAL) grid->nz));
  else grid->fft_norm = 1.0 / ((REAL) (grid->nx * grid->ny * grid->nz));
  grid->fft_norm2 = grid->fft_norm;
  if (grid->nx > 1) grid->fft_norm2 *= grid->step;
  if (grid->ny > 1) grid->fft_norm2 *= grid->step;
  if (grid->nz > 1) grid->fft_norm2 *= grid->step;
  strncpy(grid->id, id ? id : "", 32);
  grid->id[31] = 0;
  memset(grid->value, 0, len);
  grid->flag = 0;
  grid->host_lock = 0;
  gbh_register(grid->value, nscal(grid), 1, pinned);
  return grid;
}

/* src/rgrid.c:310-335 */
void rgrid_free(rgrid *grid) {
  if (!grid) return;
  gbh_block *b = gbh_find(grid->value);
  int pinned = b ? b->host_pinned : 0;
  gbh_unregister(grid->value);
  gbh_free_host(grid->value, pinned);
  free(grid);
}

/* src/rgrid.c:662-700 */
void rgrid_copy(rgrid *dst, rgrid *src) {
  if (src->nx != dst->nx || src->ny != dst->ny || src->nz != dst->nz) {
    fprintf(stderr, "libgrid: Different grid dimensions in rgrid_copy.\n");
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
    void *s = gbh_dev_read(src->value, GB_FP64);
    void *d = gbh_dev_write(dst->value, GB_FP64);
    gbh_check(gb_d2d(d, s, nscal(src) * 8), "rgrid_copy");
  } else {
    memcpy(dst->value, src->value, nscal(src) * sizeof(REAL));
    gbh_host_modified(dst->value);
  }
}

void rgrid_zero(rgrid *grid) { rgrid_constant(grid, 0.0); }

void rgrid_constant(rgrid *grid, REAL c) {
  gbh_check(gb_real_op(GB_OP_CONST, gbh_dev_write(grid->value, GB_FP64), NULL, NULL, nscal(grid), c, GB_FP64), "rgrid_constant");
}

/* src/rgrid.c:806-840 */
void rgrid_map(rgrid *grid, REAL (*func)(void *arg, REAL x, REAL y, REAL z), void *farg) {
  INT i, j, k, nx = grid->nx, ny = grid->ny, nz = grid->nz, nz2 = grid->nz2;
  REAL x, y, z, step = grid->step;
  for (i = 0; i < nx; i++) {
    x = ((REAL) (i - nx / 2)) * step - grid->x0;
    for (j = 0; j < ny; j++) {
      y = ((REAL) (j - ny / 2)) * step - grid->y0;
      for (k = 0; k < nz; k++) {
        z = ((REAL) (k - nz / 2)) * step - grid->z0;
        grid->value[(i * ny + j) * nz2 + k] = func(farg, x, y, z);
      }
    }
  }
  gbh_host_modified(grid->value);
}

static void rbinary(int op, rgrid *c, rgrid *a, rgrid *b, double d, const char *fn) {
  const void *da = a ? gbh_dev_read(a->value, GB_FP64) : NULL;
  const void *db = b ? gbh_dev_read(b->value, GB_FP64) : NULL;
  void *dc = (op == GB_OP_SCALE || op == GB_OP_ADD_SCALED || op == GB_OP_ADD_CONST) ? gbh_dev_rw(c->value, GB_FP64)
                                                                                     : gbh_dev_write(c->value, GB_FP64);
  gbh_check(gb_real_op(op, dc, da, db, nscal(c), d, GB_FP64), fn);
}

void rgrid_sum(rgrid *gridc, rgrid *grida, rgrid *gridb) { rbinary(GB_OP_SUM, gridc, grida, gridb, 0.0, "rgrid_sum"); }
void rgrid_product(rgrid *gridc, rgrid *grida, rgrid *gridb) { rbinary(GB_OP_PRODUCT, gridc, grida, gridb, 0.0, "rgrid_product"); }
void rgrid_multiply(rgrid *grid, REAL c) { rbinary(GB_OP_SCALE, grid, NULL, NULL, c, "rgrid_multiply"); }
void rgrid_add_scaled(rgrid *gridc, REAL d, rgrid *grida) { rbinary(GB_OP_ADD_SCALED, gridc, grida, NULL, d, "rgrid_add_scaled"); }

/* src/rgrid.c:1471-1500 */
REAL rgrid_integral(rgrid *grid) {
  double r[2];
  gb_geom g = geom_of(grid, GB_FP64);
  gbh_check(gb_reduce(GB_RED_REAL_SUM, gbh_dev_read(grid->value, GB_FP64), NULL, &g, grid->nz2, 0, GB_FP64, r), "rgrid_integral");
  return r[0] * gbh_step_factor(grid->nx, grid->ny, grid->nz, grid->step);
}

/*
 * R2C / C2R transforms in the padded in-place layout (src/rgrid.c:1762-1824).
 * The real rows are widened into a complex work grid, transformed with the
 * complex line-pass FFT, and the non-redundant half (kz <= nz/2) is packed
 * back; the inverse rebuilds the Hermitian half and keeps the real part.
 */
static cgrid *r_work = NULL;

static cgrid *work_for(rgrid *g) {
  if (r_work && (r_work->nx != g->nx || r_work->ny != g->ny || r_work->nz != g->nz)) {
    cgrid_free(r_work);
    r_work = NULL;
  }
  if (!r_work) r_work = cgrid_alloc(g->nx, g->ny, g->nz, g->step, CGRID_PERIODIC_BOUNDARY, NULL, "rgrid fft work");
  return r_work;
}

void rgrid_fft(rgrid *grid) {
  cgrid *w = work_for(grid);
  gb_geom g = geom_of(grid, GB_FP64);
  void *cw = gbh_dev_write(w->value, GB_FP64);
  void *r = gbh_dev_rw(grid->value, GB_FP64);
  gbh_check(gb_mixed_op(GB_MIX_REAL_TO_COMPLEX_RE, cw, r, NULL, &g, grid->nz2, GB_FP64, GB_FP64), "rgrid_fft");
  gbh_check(gb_fft3d(cw, &g, -1, 1.0), "rgrid_fft");
  gbh_check(gb_r2c_pack(r, cw, &g), "rgrid_fft");
}

void rgrid_inverse_fft(rgrid *grid) {
  cgrid *w = work_for(grid);
  gb_geom g = geom_of(grid, GB_FP64);
  void *cw = gbh_dev_write(w->value, GB_FP64);
  void *r = gbh_dev_rw(grid->value, GB_FP64);
  gbh_check(gb_c2r_unpack(cw, r, &g), "rgrid_inverse_fft");
  gbh_check(gb_fft3d(cw, &g, +1, 1.0), "rgrid_inverse_fft");
  gbh_check(gb_complex_real_part(r, cw, &g, grid->nz2), "rgrid_inverse_fft");
}

void rgrid_scaled_inverse_fft(rgrid *grid, REAL c) {
  rgrid_inverse_fft(grid);
  rgrid_multiply(grid, c);
}

void rgrid_inverse_fft_norm(rgrid *grid) { rgrid_scaled_inverse_fft(grid, grid->fft_norm); }
/* src/rgrid.c:1824 */
void rgrid_inverse_fft_norm2(rgrid *grid) { rgrid_scaled_inverse_fft(grid, grid->fft_norm2); }

/* src/rgrid.c:1848-1878: on the half spectrum (nz2 / 2 complex entries per
 * row) left by rgrid_fft */
void rgrid_fft_convolute(rgrid *gridc, rgrid *grida, rgrid *gridb) {
  if (gridc->nx != grida->nx || gridc->ny != grida->ny || gridc->nz != grida->nz || gridc->nx != gridb->nx ||
      gridc->ny != gridb->ny || gridc->nz != gridb->nz)
    gbh_die("Different grid dimensions in rgrid_fft_convolute.");
  const void *da = gbh_dev_read(grida->value, GB_FP64);
  const void *db = gbh_dev_read(gridb->value, GB_FP64);
  void *dc = gbh_dev_write(gridc->value, GB_FP64);
  gbh_check(gb_fft_convolute(dc, da, db, gridc->nx, gridc->ny, gridc->nz2 / 2, GB_FP64), "rgrid_fft_convolute");
}

/* src/rgrid.c:2267-2291 */
void rgrid_extrapolate(rgrid *dest, rgrid *src) {
  double out;
  const int bc = gbh_rbc(src, &out);
  const gb_grid_frame d = {dest->nx, dest->ny, dest->nz, dest->nz2, dest->step, dest->x0, dest->y0, dest->z0};
  const gb_grid_frame s = {src->nx, src->ny, src->nz, src->nz2, src->step, src->x0, src->y0, src->z0};
  const void *ds = gbh_dev_read(src->value, GB_FP64);
  void *dd = gbh_dev_rw(dest->value, GB_FP64); /* the row padding keeps its values */
  gbh_check(gb_interpolate(dd, &d, ds, &s, bc, out, 0.0, 1), "rgrid_extrapolate");
}

/* src/rgrid.c:339-349: nx, ny, nz (INT), step (REAL), then nx ny nz2 values
 * (the padded rows as stored) */
void rgrid_write(rgrid *grid, FILE *out) {
  gbh_host_read(grid->value);
  fwrite(&grid->nx, sizeof(INT), 1, out);
  fwrite(&grid->ny, sizeof(INT), 1, out);
  fwrite(&grid->nz, sizeof(INT), 1, out);
  fwrite(&grid->step, sizeof(REAL), 1, out);
  fwrite(grid->value, sizeof(REAL), nscal(grid), out);
}

/* src/rgrid.c:360-400: a file of another size or step is read into a
 * temporary grid and interpolated onto `grid` (rgrid_extrapolate). */
rgrid *rgrid_read(rgrid *grid, FILE *in) {
  INT nx, ny, nz, nzz;
  REAL step;
  if (fread(&nx, sizeof(INT), 1, in) != 1 || fread(&ny, sizeof(INT), 1, in) != 1 || fread(&nz, sizeof(INT), 1, in) != 1 ||
      fread(&step, sizeof(REAL), 1, in) != 1) {
    fprintf(stderr, "libgrid: Error reading grid header in rgrid_read().\n");
    return NULL;
  }
  nzz = 2 * (nz / 2 + 1);
  if (!grid) {
    if (!(grid = rgrid_alloc(nx, ny, nz, step, RGRID_PERIODIC_BOUNDARY, NULL, "read_grid"))) {
      fprintf(stderr, "libgrid: Failed to allocate grid in rgrid_read().\n");
      return NULL;
    }
  }
  if (nx != grid->nx || ny != grid->ny || nz != grid->nz || step != grid->step) {
    rgrid *tmp;
    fprintf(stderr, "libgrid: Grid in file has different size than grid in memory.\n");
    fprintf(stderr, "libgrid: Interpolating between grids.\n");
    if (!(tmp = rgrid_alloc(nx, ny, nz, step, grid->value_outside, NULL, "rgrid_read_temp"))) {
      fprintf(stderr, "libgrid: Error allocating grid in rgrid_read().\n");
      abort();
    }
    if (fread(tmp->value, sizeof(REAL), (size_t) (nx * ny * nzz), in) != (size_t) (nx * ny * nzz))
      fprintf(stderr, "libgrid: Short read in rgrid_read().\n");
    gbh_host_modified(tmp->value);
    rgrid_extrapolate(grid, tmp);
    rgrid_free(tmp);
    return grid;
  }
  if (fread(grid->value, sizeof(REAL), (size_t) (nx * ny * nzz), in) != (size_t) (nx * ny * nzz))
    fprintf(stderr, "libgrid: Short read in rgrid_read().\n");
  gbh_host_modified(grid->value);
  return grid;
}

/* src/rgrid.c:2020-2060 */
REAL rgrid_value_at_index(rgrid *grid, INT i, INT j, INT k) {
  if (i < 0 || j < 0 || k < 0 || i >= grid->nx || j >= grid->ny || k >= grid->nz) return grid->value_outside(grid, i, j, k);
  const size_t idx = (size_t) ((i * grid->ny + j) * grid->nz2 + k);
  gbh_block *b = gbh_find(grid->value);
  if (!b || (b->state & GBH_HOST_VALID)) return grid->value[idx];
  REAL v;
  gbh_check(gb_d2h(&v, (const char *) b->dev + idx * 8, 8), "rgrid_value_at_index");
  return v;
}

void rgrid_value_to_index(rgrid *grid, INT i, INT j, INT k, REAL value) {
  if (i < 0 || j < 0 || k < 0 || i >= grid->nx || j >= grid->ny || k >= grid->nz) return;
  const size_t idx = (size_t) ((i * grid->ny + j) * grid->nz2 + k);
  gbh_block *b = gbh_find(grid->value);
  if (b && (b->state & GBH_DEV_VALID)) {
    gbh_check(gb_h2d((char *) b->dev + idx * 8, &value, 8), "rgrid_value_to_index");
    gbh_check(gb_synchronize(), "rgrid_value_to_index");
    b->shadow_valid = 0;
    if (b->state & GBH_HOST_VALID) grid->value[idx] = value;
    return;
  }
  grid->value[idx] = value;
  if (b) gbh_host_modified(grid->value);
}

/* src/rgrid_bc.c:19-74 */
REAL rgrid_value_outside_dirichlet(rgrid *grid, INT i, INT j, INT k) {
  (void) i;
  (void) j;
  (void) k;
  return *((REAL *) grid->outside_params_ptr);
}

REAL rgrid_value_outside_neumann(rgrid *grid, INT i, INT j, INT k) {
  INT nx = grid->nx, ny = grid->ny, nz = grid->nz;
  if (i < 0) i = -i;
  if (i > nx - 1) i = 2 * nx - i - 2;
  if (j < 0) j = -j;
  if (j > ny - 1) j = 2 * ny - j - 2;
  if (k < 0) k = -k;
  if (k > nz - 1) k = 2 * nz - k - 2;
  if (i < 0 || i >= nx) i = 0;
  if (j < 0 || j >= ny) j = 0;
  if (k < 0 || k >= nz) k = 0;
  return rgrid_value_at_index(grid, i, j, k);
}

REAL rgrid_value_outside_periodic(rgrid *grid, INT i, INT j, INT k) {
  INT nx = grid->nx, ny = grid->ny, nz = grid->nz;
  i %= nx;
  if (i < 0) i = nx + i;
  j %= ny;
  if (j < 0) j = ny + j;
  k %= nz;
  if (k < 0) k = nz + k;
  return rgrid_value_at_index(grid, i, j, k);
}

/* src/rgrid_diff.c:309-343 */
void rgrid_fd_laplace(rgrid *grid, rgrid *laplace) {
  if (grid == laplace) {
    fprintf(stderr, "libgrid: source and destination must be different in rgrid_fd_laplace().\n");
    abort();
  }
  double out;
  const int bc = gbh_rbc(grid, &out);
  gb_geom g = geom_of(grid, GB_FP64);
  const void *s = gbh_dev_read(grid->value, GB_FP64);
  void *d = gbh_dev_rw(laplace->value, GB_FP64);
  gbh_check(gb_fd(GB_FD_LAPLACE, d, s, &g, bc, out, 0.0, 1.0 / (grid->step * grid->step), 1, grid->nz2), "rgrid_fd_laplace");
}

/* ------------------------------------------------------------ ngrid.c */

/* src/ngrid.c:53-79 */
void grid_real_to_complex_re(cgrid *dest, rgrid *source) {
  dest->nx = source->nx;
  dest->ny = source->ny;
  dest->nz = source->nz;
  dest->step = source->step;
  const int p = gbh_prec(dest->value);
  gb_geom g = geom_of(source, p);
  const void *r = gbh_dev_read(source->value, p);
  void *c = gbh_dev_write(dest->value, p);
  gbh_check(gb_mixed_op(GB_MIX_REAL_TO_COMPLEX_RE, c, (void *) r, NULL, &g, source->nz2, p, p), "grid_real_to_complex_re");
}

/* src/ngrid.c:186-214 */
void grid_product_norm(rgrid *dst, rgrid *src1, cgrid *src2) {
  const int pc = gbh_prec(src2->value);
  gb_geom g = geom_of(src1, pc);
  const void *c = gbh_dev_read(src2->value, pc);
  const void *r1 = gbh_dev_read(src1->value, GB_FP64);
  void *r = (dst == src1) ? gbh_dev_rw(dst->value, GB_FP64) : gbh_dev_write(dst->value, GB_FP64);
  gbh_check(gb_mixed_op(GB_MIX_PRODUCT_NORM, (void *) c, r, r1, &g, src1->nz2, pc, GB_FP64), "grid_product_norm");
  dst->nx = src1->nx;
  dst->ny = src1->ny;
  dst->nz = src1->nz;
  dst->step = src1->step;
}

/* src/ngrid.c:254-280 */
void grid_product_complex_with_real(cgrid *dst, rgrid *src) {
  const int p = gbh_prec(dst->value);
  gb_geom g = geom_of(src, p);
  const void *r = gbh_dev_read(src->value, p);
  void *c = gbh_dev_rw(dst->value, p);
  gbh_check(gb_mixed_op(GB_MIX_PRODUCT_COMPLEX_REAL, c, (void *) r, NULL, &g, src->nz2, p, p), "grid_product_complex_with_real");
}

/* src/ngrid.c:355-378 */
REAL grid_grid_expectation_value(cgrid *dgrid, rgrid *opgrid) {
  double r[2];
  const int p = gbh_prec(dgrid->value);
  gb_geom g = geom_of(opgrid, p);
  const void *b = gbh_dev_read(opgrid->value, GB_FP64);
  gbh_check(gb_reduce(GB_RED_EXPECT_REAL, gbh_dev_read(dgrid->value, p), b, &g, dgrid->nz, opgrid->nz2, GB_FP64, r),
            "grid_grid_expectation_value");
  return r[0] * gbh_step_factor(dgrid->nx, dgrid->ny, dgrid->nz, dgrid->step);
}
