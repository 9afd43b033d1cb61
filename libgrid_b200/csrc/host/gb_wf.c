/*
 * Wavefunction API of libgrid-b200 (reference src/grid_wf.c,
 * src/grid_wf_fft.c, src/grid_wf_cn.c, src/grid_wf_diag.c).
 *
 * grid_wf_propagate keeps the reference's propagator dispatch and its
 * compositions; the 2nd-order FFT/CFFT step runs as one fused line-pass
 * schedule (gb_split_step) and the 2nd-order Crank-Nicolson step as one
 * fused three-sweep schedule (gb_cn_step) with both potential half-steps
 * folded into the first and last sweep.  The remaining propagators are
 * composed from the same device primitives exactly as the reference composes
 * them.
 */
#include "gb_host.h"

static size_t npts(const cgrid *g) { return (size_t) (g->nx * g->ny * g->nz); }

static int psi_prec(const wf *gwf) { return gbh_prec(gwf->grid->value); }

static gb_geom wf_geom(const wf *gwf) {
  const cgrid *g = gwf->grid;
  return gbh_geom(g->nx, g->ny, g->nz, g->step, psi_prec(gwf));
}

static cgrid *workspace(wf *gwf, cgrid **slot, const char *id) {
  cgrid *grid = gwf->grid;
  if (!*slot) {
    *slot = cgrid_alloc(grid->nx, grid->ny, grid->nz, grid->step, grid->value_outside, grid->outside_params_ptr, (char *) id);
    if (!*slot) gbh_die("out of memory for %s", id);
  }
  if (gbh_prec((*slot)->value) != psi_prec(gwf)) gbh_set_prec((*slot)->value, psi_prec(gwf));
  return *slot;
}

static REAL frame_cons(const wf *gwf) {
  const cgrid *g = gwf->grid;
  return -(HBAR * HBAR / (2.0 * gwf->mass)) * (g->kx0 * g->kx0 + g->ky0 * g->ky0 + g->kz0 * g->kz0);
}

/* src/grid_wf.c:26-82 */
wf *grid_wf_alloc(INT nx, INT ny, INT nz, REAL step, REAL mass, char boundary, char propagator, char *id) {
  wf *gwf;
  REAL complex (*value_outside)(struct cgrid_struct *grid, INT i, INT j, INT k) = NULL;

  if (boundary < WF_DIRICHLET_BOUNDARY || boundary > WF_PERIODIC_BOUNDARY) {
    fprintf(stderr, "libgrid: Error in grid_wf_alloc(). Unknown boundary condition.\n");
    return 0;
  }
  if (propagator < WF_2ND_ORDER_FFT || propagator > WF_1ST_ORDER_EULER) {
    fprintf(stderr, "libgrid: Error in grid_wf_alloc(). Unknown propagator.\n");
    return 0;
  }
  if (boundary == WF_DIRICHLET_BOUNDARY && propagator < WF_2ND_ORDER_CN) {
    fprintf(stderr, "libgrid: Error in grid_wf_alloc(). Invalid boundary condition - propagator combination. Dirichlet condition can only be used with Crank-Nicolson propagator.\n");
    return 0;
  }
  if (!(gwf = (wf *) malloc(sizeof(wf)))) {
    fprintf(stderr, "libgrid: Error in grid_wf_alloc(). Could not allocate memory for wf.\n");
    return 0;
  }
  memset(gwf, 0, sizeof(wf));
  switch (boundary) {
    case WF_DIRICHLET_BOUNDARY: value_outside = CGRID_DIRICHLET_BOUNDARY; break;
    case WF_NEUMANN_BOUNDARY: value_outside = CGRID_NEUMANN_BOUNDARY; break;
    case WF_PERIODIC_BOUNDARY: value_outside = CGRID_PERIODIC_BOUNDARY; break;
  }
  if (!(gwf->grid = cgrid_alloc(nx, ny, nz, step, value_outside, 0, id))) {
    fprintf(stderr, "libgrid: Error in grid_wf_alloc(). Could not allocate memory for wf->grid.\n");
    free(gwf);
    return NULL;
  }
  gwf->mass = mass;
  gwf->norm = 1.0;
  gwf->boundary = boundary;
  gwf->propagator = propagator;
  gwf->cworkspace = gwf->cworkspace2 = gwf->cworkspace3 = NULL;
  gwf->ts_func = NULL;
  gwf->cfft_width = 1.0;
  gwf->kmax = 9999.0;
  return gwf;
}

/* src/grid_wf.c:99-120 (including the reference's clearing statement) */
void grid_wf_boundary(wf *gwf, wf *gwfp, INT lx, INT hx, INT ly, INT hy, INT lz, INT hz) {
  if (!lx && !hx && !ly && !hy && !lz && !hz) {
    gwf->ts_func = NULL;
    gwf->lx = gwf->hx = gwf->ly = gwf->hy = gwf->lz = gwf->hz = 0;
    if (gwfp) {
      gwfp->ts_func = NULL;
      gwfp->lx = gwf->hx = gwf->ly = gwf->hy = gwf->lz = gwf->hz = 0;
    }
    return;
  }
  gwf->lx = lx;
  gwf->hx = hx;
  gwf->ly = ly;
  gwf->hy = hy;
  gwf->lz = lz;
  gwf->hz = hz;
  gwf->ts_func = &grid_wf_absorb;
  if (gwfp) gwfp->ts_func = &grid_wf_absorb;
}

/* src/grid_wf.c:131-147; the clone gets workspaces of its own instead of
 * sharing the original's pointers. */
wf *grid_wf_clone(wf *gwf, char *id) {
  wf *nwf;
  cgrid *grid = gwf->grid;
  if (!(nwf = (wf *) malloc(sizeof(wf)))) {
    fprintf(stderr, "libgrid: Out of memory in grid_wf_clone().\n");
    abort();
  }
  memcpy(nwf, gwf, sizeof(wf));
  nwf->cworkspace = nwf->cworkspace2 = nwf->cworkspace3 = NULL;
  if (!(nwf->grid = cgrid_alloc(grid->nx, grid->ny, grid->nz, grid->step, grid->value_outside, 0, id))) {
    fprintf(stderr, "libgrid: Error in grid_wf_clone(). Could not allocate memory for nwf->grid.\n");
    free(nwf);
    return NULL;
  }
  if (psi_prec(gwf) == GB_FP32) gbh_set_prec(nwf->grid->value, GB_FP32);
  return nwf;
}

/* src/grid_wf.c:157-166 */
void grid_wf_free(wf *gwf) {
  if (gwf) {
    if (gwf->grid) cgrid_free(gwf->grid);
    if (gwf->cworkspace) cgrid_free(gwf->cworkspace);
    if (gwf->cworkspace2) cgrid_free(gwf->cworkspace2);
    if (gwf->cworkspace3) cgrid_free(gwf->cworkspace3);
    free(gwf);
  }
}

/* src/grid_wf.c:185-203 */
REAL grid_wf_absorb(INT i, INT j, INT k, INT lx, INT hx, INT ly, INT hy, INT lz, INT hz) {
  REAL t = 0.0;
  if (i < lx) t += ((REAL) (lx - i)) / (REAL) lx;
  else if (i > hx) t += ((REAL) (i - hx)) / (REAL) lx;
  if (j < ly) t += ((REAL) (ly - j)) / (REAL) ly;
  else if (j > hy) t += ((REAL) (j - hy)) / (REAL) ly;
  if (k < lz) t += ((REAL) (lz - k)) / (REAL) lz;
  else if (k > hz) t += ((REAL) (k - hz)) / (REAL) lz;
  t *= 2.0 / 3.0;
  if (t > 1.0) return 1.0;
  return t;
}

static void need_absorb_fn(const wf *gwf) {
  if (gwf->ts_func && gwf->ts_func != grid_wf_absorb) {
    fprintf(stderr, "libgrid(CUDA): Only grid_wf_absorb function can be used for time().\n");
    abort();
  }
}

/* ------------------------------------------------------------- energies */

/* src/grid_wf.c:215-249 */
REAL grid_wf_energy(wf *gwf, rgrid *potential) {
  if (gwf->propagator == WF_2ND_ORDER_CN || gwf->propagator == WF_4TH_ORDER_CN || !grid_analyze_method)
    return grid_wf_energy_cn(gwf, potential);
  return grid_wf_energy_fft(gwf, potential);
}

REAL grid_wf_kinetic_energy(wf *gwf) { return grid_wf_energy(gwf, NULL); }

REAL grid_wf_potential_energy(wf *gwf, rgrid *potential) { return grid_grid_expectation_value(gwf->grid, potential); }

/* src/grid_wf_fft.c:101-129: T = -hbar^2/2m * (-sum k^2 |psi_k|^2 * fft_norm2).
 * psi itself is left untouched (the reference round-trips it through an
 * FFT pair). */
REAL grid_wf_energy_fft(wf *gwf, rgrid *potential) {
  REAL en = grid_wf_kinetic_energy_fft(gwf);
  if (potential) en += grid_wf_potential_energy(gwf, potential);
  return en;
}

REAL grid_wf_kinetic_energy_fft(wf *gwf) {
  cgrid *grid = gwf->grid;
  const int p = psi_prec(gwf);
  gb_geom g = wf_geom(gwf);
  cgrid *w = workspace(gwf, &gwf->cworkspace, "WF cworkspace");
  const void *psi = gbh_dev_read(grid->value, p);
  void *work = gbh_dev_write(w->value, p);
  double s = 0.0;
  gbh_check(gb_fft_ksq_sum(psi, work, &g, &s), "grid_wf_kinetic_energy_fft");
  return -HBAR * HBAR / (2.0 * gwf->mass) * (-s * grid->fft_norm2);
}

/* src/grid_wf_cn.c:19-49, with the Laplacian and the overlap fused into one
 * read-only pass. */
REAL grid_wf_energy_cn(wf *gwf, rgrid *potential) {
  REAL en = grid_wf_kinetic_energy_cn(gwf);
  if (potential) en += grid_wf_potential_energy(gwf, potential);
  return en;
}

REAL grid_wf_kinetic_energy_cn(wf *gwf) {
  cgrid *grid = gwf->grid;
  double ore, oim, r[2];
  const int bc = gbh_cbc(grid, &ore, &oim);
  gb_geom g = wf_geom(gwf);
  gbh_check(gb_fd_kinetic_sum(gbh_dev_read(grid->value, g.prec), &g, bc, ore, oim, 1.0 / (grid->step * grid->step), r),
            "grid_wf_kinetic_energy_cn");
  return (-HBAR * HBAR / (2.0 * gwf->mass)) * r[0] * gbh_step_factor(grid->nx, grid->ny, grid->nz, grid->step);
}

/* src/grid_wf_diag.c:20-64 */
REAL grid_wf_energy_and_error(wf *gwf, cgrid *potential, cgrid *workspace_grid, REAL *error) {
  REAL energy;
  if (gwf->boundary == WF_DIRICHLET_BOUNDARY || gwf->boundary == WF_NEUMANN_BOUNDARY) {
    cgrid_fd_laplace(gwf->grid, workspace_grid);
    cgrid_multiply(workspace_grid, -HBAR * HBAR / (2.0 * gwf->mass));
  } else if (gwf->boundary == WF_PERIODIC_BOUNDARY) {
    cgrid_copy(workspace_grid, gwf->grid);
    cgrid_fft(workspace_grid);
    cgrid_fft_laplace(workspace_grid, workspace_grid);
    cgrid_scaled_inverse_fft(workspace_grid, -gwf->grid->fft_norm * HBAR * HBAR / (2.0 * gwf->mass));
  } else {
    fprintf(stderr, "libgrid: Error in grid_wf_energy_and_error(). Invalid boundary condition.\n");
    abort();
  }
  cgrid_add_scaled_product(workspace_grid, 1.0, potential, gwf->grid);
  *error = cgrid_integral_of_square(workspace_grid);
  cgrid_conjugate_product(workspace_grid, gwf->grid, workspace_grid);
  energy = creal(cgrid_integral(workspace_grid));
  *error = sqrt(*error - energy * energy);
  return energy;
}

/* ------------------------------------------------------ propagation parts */

static void fill_absorb(gb_potential *pt, const wf *gwf, REAL treal) {
  pt->absorb = 1;
  pt->lx = gwf->lx;
  pt->hx = gwf->hx;
  pt->ly = gwf->ly;
  pt->hy = gwf->hy;
  pt->lz = gwf->lz;
  pt->hz = gwf->hz;
  pt->treal = treal;
}

/* src/grid_wf.c:569-600 */
void grid_wf_propagate_potential(wf *gwf, REAL complex tstep, cgrid *potential, REAL cons) {
  if (!potential) return;
  need_absorb_fn(gwf);
  const int p = psi_prec(gwf);
  gb_geom g = wf_geom(gwf);
  gb_potential pt;
  memset(&pt, 0, sizeof(pt));
  REAL complex c = -I * tstep / HBAR;
  pt.kind = GB_POT_COMPLEX;
  pt.v = gbh_dev_read(potential->value, p);
  pt.vrow = potential->nz;
  pt.c_re = creal(c);
  pt.c_im = cimag(c);
  pt.cons = cons;
  if (gwf->ts_func && gwf->propagator >= WF_2ND_ORDER_CN) fill_absorb(&pt, gwf, creal(tstep) / HBAR);
  gbh_check(gb_potential_multiply(gbh_dev_rw(gwf->grid->value, p), &g, &pt), "grid_wf_propagate_potential");
}

static void kinetic_pointwise(wf *gwf, REAL complex time, int cutoff, const char *fn) {
  const cgrid *grid = gwf->grid;
  const int p = psi_prec(gwf);
  gb_geom g = wf_geom(gwf);
  REAL complex tm = -I * time * HBAR / (gwf->mass * 2.0);
  gb_kinetic k;
  memset(&k, 0, sizeof(k));
  k.tm_re = creal(tm);
  k.tm_im = cimag(tm);
  k.kx0 = grid->kx0;
  k.ky0 = grid->ky0;
  k.kz0 = grid->kz0;
  k.scale = 1.0;
  k.kmax2 = gwf->kmax * gwf->kmax;
  k.cutoff = cutoff;
  gbh_check(gb_kinetic_multiply(gbh_dev_rw(gwf->grid->value, p), &g, &k), fn);
}

/* src/grid_wf_fft.c:141-193, :206-262 */
void grid_wf_propagate_kinetic_fft(wf *gwf, REAL complex time) { kinetic_pointwise(gwf, time, 0, "grid_wf_propagate_kinetic_fft"); }
void grid_wf_propagate_kinetic_cfft(wf *gwf, REAL complex time) { kinetic_pointwise(gwf, time, 1, "grid_wf_propagate_kinetic_cfft"); }

static gb_cn_params cn_params(const wf *gwf, REAL complex tstep) {
  const cgrid *grid = gwf->grid;
  gb_cn_params cp;
  memset(&cp, 0, sizeof(cp));
  cp.boundary = gwf->boundary;
  cp.tstep_re = creal(tstep);
  cp.tstep_im = cimag(tstep);
  cp.mass = gwf->mass;
  cp.kx0 = grid->kx0;
  cp.ky0 = grid->ky0;
  cp.kz0 = grid->kz0;
  cp.omega = grid->omega;
  cp.x0 = grid->x0;
  cp.y0 = grid->y0;
  if (gwf->ts_func) {
    cp.absorb = 1;
    cp.lx = gwf->lx;
    cp.hx = gwf->hx;
    cp.ly = gwf->ly;
    cp.hy = gwf->hy;
    cp.lz = gwf->lz;
    cp.hz = gwf->hz;
  }
  return cp;
}

static void cn_kinetic_fused(wf *gwf, REAL complex tstep, const gb_potential *pre, const gb_potential *post, const char *fn) {
  need_absorb_fn(gwf);
  if (psi_prec(gwf) != GB_FP64) gbh_die("%s: Crank-Nicolson propagation runs in FP64 only (grid_wf_precision)", fn);
  gb_geom g = wf_geom(gwf);
  gb_cn_params cp = cn_params(gwf, tstep);
  /* a copy wait that gave up is reported at the next read of a result */
  gbh_check(gb_cn_step(gbh_dev_rw(gwf->grid->value, GB_FP64), &g, &cp, pre, post), fn);
}

/* src/grid_wf_cn.c:65-79 */
void grid_wf_propagate_kinetic_cn(wf *gwf, REAL complex tstep) {
  cn_kinetic_fused(gwf, tstep, NULL, NULL, "grid_wf_propagate_kinetic_cn");
}

/* One fused 2nd-order FFT/CFFT step K(dt/2) V(dt) K(dt/2).  Either a complex
 * potential grid or a real external potential with g |psi|^2 may be given
 * (both NULL / g == 0 means no potential step, as grid_wf_propagate_potential
 * returns early for a NULL potential). */
static void fused_fft_steps(wf *gwf, REAL complex time, cgrid *cpot, rgrid *vext, REAL gnl, int cutoff, int nsteps) {
  cgrid *grid = gwf->grid;
  const int p = psi_prec(gwf);
  gb_geom g = wf_geom(gwf);
  REAL complex half = 0.5 * time;
  REAL complex tm = -I * half * HBAR / (gwf->mass * 2.0);
  gb_kinetic k;
  memset(&k, 0, sizeof(k));
  k.tm_re = creal(tm);
  k.tm_im = cimag(tm);
  k.kx0 = grid->kx0;
  k.ky0 = grid->ky0;
  k.kz0 = grid->kz0;
  k.scale = grid->fft_norm;
  k.kmax2 = gwf->kmax * gwf->kmax;
  k.cutoff = cutoff;
  gb_potential pt;
  memset(&pt, 0, sizeof(pt));
  REAL complex c = -I * time / HBAR;
  pt.c_re = creal(c);
  pt.c_im = cimag(c);
  pt.cons = frame_cons(gwf);
  int has_pot = 0;
  if (cpot) {
    pt.kind = GB_POT_COMPLEX;
    pt.v = gbh_dev_read(cpot->value, p);
    pt.vrow = cpot->nz;
    has_pot = 1;
  } else if (vext || gnl != 0.0) {
    if (vext) {
      pt.kind = GB_POT_REAL;
      pt.v = gbh_dev_read(vext->value, p);
      pt.vrow = vext->nz2;
    }
    pt.g = gnl;
    has_pot = 1;
  }
  gbh_check(gb_split_steps(gbh_dev_rw(grid->value, p), &g, &k, has_pot ? &pt : NULL, nsteps), "grid_wf_propagate");
}

static void fused_fft_step(wf *gwf, REAL complex time, cgrid *cpot, rgrid *vext, REAL gnl, int cutoff) {
  fused_fft_steps(gwf, time, cpot, vext, gnl, cutoff, 1);
}

/* The reference's FFT absorbing-boundary composition (src/grid_wf.c:396-422):
 * a real-time step on psi, an imaginary-time step on a copy, then the blend. */
static void fft_step_with_absorber(wf *gwf, REAL complex time, cgrid *cpot, rgrid *vext, REAL gnl, int cutoff) {
  REAL (*save)(INT, INT, INT, INT, INT, INT, INT, INT, INT) = gwf->ts_func;
  cgrid *gsave;
  gwf->ts_func = NULL;
  cgrid *ws = workspace(gwf, &gwf->cworkspace, "WF cworkspace 1");
  cgrid_copy(ws, gwf->grid);
  fused_fft_step(gwf, time, cpot, vext, gnl, cutoff);
  gsave = gwf->grid;
  gwf->grid = ws;
  fused_fft_step(gwf, -I * creal(time), cpot, vext, gnl, cutoff);
  gwf->grid = gsave;
  gwf->ts_func = save;
  grid_wf_merge(gwf, gwf->grid, ws);
}

/* src/grid_wf.c:276-306: |grad V|^2 via the analysis method in effect */
void grid_wf_square_of_potential_gradient(wf *gwf, cgrid *sq_grad_pot, cgrid *potential) {
  cgrid *cw = workspace(gwf, &gwf->cworkspace, "WF cworkspace");
  cgrid *cw2 = workspace(gwf, &gwf->cworkspace2, "WF cworkspace 2");
  if (grid_analyze_method > 0) {
    cgrid_copy(sq_grad_pot, potential);
    cgrid_fft(sq_grad_pot);
    cgrid_fft_gradient_x(sq_grad_pot, cw);
    cgrid_fft_gradient_y(sq_grad_pot, cw2);
    cgrid_fft_gradient_z(sq_grad_pot, sq_grad_pot);
    cgrid_inverse_fft_norm(sq_grad_pot);
    cgrid_inverse_fft_norm(cw);
    cgrid_inverse_fft_norm(cw2);
  } else {
    cgrid_fd_gradient_x(potential, cw);
    cgrid_fd_gradient_y(potential, cw2);
    cgrid_fd_gradient_z(potential, sq_grad_pot);
  }
  cgrid_conjugate_product(sq_grad_pot, sq_grad_pot, sq_grad_pot);
  cgrid_conjugate_product(cw, cw, cw);
  cgrid_conjugate_product(cw2, cw2, cw2);
  cgrid_sum(cw, cw, cw2);
  cgrid_sum(sq_grad_pot, sq_grad_pot, cw);
}

static void cn_pot_half(gb_potential *pt, const wf *gwf, REAL complex half, cgrid *cpot, rgrid *vext, REAL gnl) {
  memset(pt, 0, sizeof(*pt));
  REAL complex c = -I * half / HBAR;
  pt->c_re = creal(c);
  pt->c_im = cimag(c);
  pt->cons = 0.0;
  if (cpot) {
    pt->kind = GB_POT_COMPLEX;
    pt->v = gbh_dev_read(cpot->value, GB_FP64);
    pt->vrow = cpot->nz;
  } else if (vext) {
    pt->kind = GB_POT_REAL;
    pt->v = gbh_dev_read(vext->value, GB_FP64);
    pt->vrow = vext->nz2;
  }
  pt->g = gnl;
  if (gwf->ts_func) fill_absorb(pt, gwf, creal(half) / HBAR);
}

/* src/grid_wf.c:379-556 */
void grid_wf_propagate(wf *gwf, cgrid *potential, REAL complex time) {
  REAL complex half_time = 0.5 * time;
  REAL complex one_sixth_time = time / 6.0;
  REAL complex two_thirds_time = 2.0 * time / 3.0;
  REAL cons = frame_cons(gwf);

  switch (gwf->propagator) {
    case WF_2ND_ORDER_FFT:
    case WF_2ND_ORDER_CFFT: {
      const int cutoff = (gwf->propagator == WF_2ND_ORDER_CFFT);
      if (gwf->grid->omega != 0.0) {
        fprintf(stderr, "libgrid: omega != 0.0 allowed only with CN.\n");
        abort();
      }
      if (gwf->ts_func && creal(time) != 0.0) fft_step_with_absorber(gwf, time, potential, NULL, 0.0, cutoff);
      else fused_fft_step(gwf, time, potential, NULL, 0.0, cutoff);
    } break;
    case WF_4TH_ORDER_FFT:
    case WF_4TH_ORDER_CFFT: {
      const int cutoff = (gwf->propagator == WF_4TH_ORDER_CFFT);
      if (gwf->ts_func) {
        fprintf(stderr, "libgrid: 4th order propagator not available for FFT absorbing BC.\n");
        abort();
      }
      if (gwf->grid->omega != 0.0) {
        fprintf(stderr, "libgrid: omega != 0.0 allowed only with CN.\n");
        abort();
      }
      cgrid *cw = workspace(gwf, &gwf->cworkspace, "WF cworkspace 1");
      workspace(gwf, &gwf->cworkspace2, "WF cworkspace 2");
      cgrid *cw3 = workspace(gwf, &gwf->cworkspace3, "WF cworkspace 3");
      grid_wf_propagate_potential(gwf, one_sixth_time, potential, cons);
      cgrid_fft(gwf->grid);
      if (cutoff) grid_wf_propagate_kinetic_cfft(gwf, half_time);
      else grid_wf_propagate_kinetic_fft(gwf, half_time);
      cgrid_inverse_fft_norm(gwf->grid);
      cgrid_copy(cw, potential);
      grid_wf_square_of_potential_gradient(gwf, cw3, potential);
      cgrid_add_scaled(cw, ((1.0 / 48.0) * HBAR * HBAR / gwf->mass) * (creal(time) * creal(time) + cimag(time) * cimag(time)), cw3);
      /* the reference propagates the middle step with `potential`, not the
       * gradient-corrected workspace (src/grid_wf.c:452,520) */
      grid_wf_propagate_potential(gwf, two_thirds_time, potential, cons);
      cgrid_fft(gwf->grid);
      if (cutoff) grid_wf_propagate_kinetic_cfft(gwf, half_time);
      else grid_wf_propagate_kinetic_fft(gwf, half_time);
      cgrid_inverse_fft_norm(gwf->grid);
      grid_wf_propagate_potential(gwf, one_sixth_time, potential, cons);
    } break;
    case WF_2ND_ORDER_CN: {
      gb_potential pre, post;
      if (potential) {
        cn_pot_half(&pre, gwf, half_time, potential, NULL, 0.0);
        post = pre;
        cn_kinetic_fused(gwf, time, &pre, &post, "grid_wf_propagate");
      } else cn_kinetic_fused(gwf, time, NULL, NULL, "grid_wf_propagate");
    } break;
    case WF_4TH_ORDER_CN: {
      cgrid *cw = workspace(gwf, &gwf->cworkspace, "WF cworkspace 1");
      workspace(gwf, &gwf->cworkspace2, "WF cworkspace 2");
      cgrid *cw3 = workspace(gwf, &gwf->cworkspace3, "WF cworkspace 3");
      grid_wf_propagate_potential(gwf, one_sixth_time, potential, 0.0);
      grid_wf_propagate_kinetic_cn(gwf, half_time);
      cgrid_copy(cw, potential);
      grid_wf_square_of_potential_gradient(gwf, cw3, potential);
      cgrid_add_scaled(cw, (1.0 / 48.0 * HBAR * HBAR / gwf->mass) * (creal(time) * creal(time) + cimag(time) * cimag(time)), cw3);
      grid_wf_propagate_potential(gwf, two_thirds_time, cw, 0.0);
      grid_wf_propagate_kinetic_cn(gwf, half_time);
      grid_wf_propagate_potential(gwf, one_sixth_time, potential, 0.0);
    } break;
    case WF_1ST_ORDER_EULER: {
      cgrid *cw = workspace(gwf, &gwf->cworkspace, "WF cworkspace 1");
      cgrid_laplace(gwf->grid, cw);
      cgrid_multiply(cw, -0.5 * HBAR * HBAR / gwf->mass);
      cgrid_add_scaled_product(cw, 1.0, potential, gwf->grid);
      cgrid_multiply(cw, -I * time / HBAR);
      cgrid_sum(gwf->grid, gwf->grid, cw);
    } break;
    default:
      fprintf(stderr, "libgrid: Error in grid_wf_propagate(). Unknown propagator.\n");
      abort();
  }
}

/* src/grid_wf.c:264-319 */
void grid_wf_propagate_predict(wf *gwf, wf *gwfp, cgrid *potential, REAL complex time) {
  REAL complex half_time = 0.5 * time;
  REAL cons = frame_cons(gwf);
  switch (gwfp->propagator) {
    case WF_2ND_ORDER_FFT:
    case WF_2ND_ORDER_CFFT:
      if (gwf->ts_func) {
        fprintf(stderr, "libgrid: Predict-correct not available for FFT absorbing BC.\n");
        abort();
      }
      if (gwfp->grid->omega != 0.0) {
        fprintf(stderr, "libgrid: omega != 0.0 allowed only with WF_XX_ORDER_CN.\n");
        abort();
      }
      cgrid_fft(gwf->grid);
      if (gwfp->propagator == WF_2ND_ORDER_CFFT) grid_wf_propagate_kinetic_cfft(gwf, half_time);
      else grid_wf_propagate_kinetic_fft(gwf, half_time);
      cgrid_inverse_fft_norm(gwf->grid);
      cgrid_copy(gwfp->grid, gwf->grid);
      grid_wf_propagate_potential(gwfp, time, potential, cons);
      break;
    case WF_2ND_ORDER_CN:
      grid_wf_propagate_kinetic_cn(gwf, half_time);
      cgrid_copy(gwfp->grid, gwf->grid);
      grid_wf_propagate_potential(gwfp, time, potential, 0.0);
      break;
    case WF_4TH_ORDER_FFT:
    case WF_4TH_ORDER_CFFT:
    case WF_4TH_ORDER_CN:
    case WF_1ST_ORDER_EULER:
      fprintf(stderr, "libgrid: Propagator not implemented for predict-correct.\n");
      abort();
    default:
      fprintf(stderr, "libgrid: Error in grid_wf_propagate(). Unknown propagator.\n");
      abort();
  }
}

/* src/grid_wf.c:331-367 */
void grid_wf_propagate_correct(wf *gwf, cgrid *potential, REAL complex time) {
  REAL complex half_time = 0.5 * time;
  REAL cons = frame_cons(gwf);
  switch (gwf->propagator) {
    case WF_2ND_ORDER_FFT:
    case WF_2ND_ORDER_CFFT:
      grid_wf_propagate_potential(gwf, time, potential, cons);
      cgrid_fft(gwf->grid);
      if (gwf->propagator == WF_2ND_ORDER_CFFT) grid_wf_propagate_kinetic_cfft(gwf, half_time);
      else grid_wf_propagate_kinetic_fft(gwf, half_time);
      cgrid_inverse_fft_norm(gwf->grid);
      break;
    case WF_4TH_ORDER_FFT:
    case WF_4TH_ORDER_CFFT:
    case WF_4TH_ORDER_CN:
    case WF_1ST_ORDER_EULER:
      fprintf(stderr, "libgrid: Propagator not implemented for predict-correct.\n");
      abort();
    case WF_2ND_ORDER_CN:
      grid_wf_propagate_potential(gwf, time, potential, 0.0);
      grid_wf_propagate_kinetic_cn(gwf, half_time);
      break;
    default:
      fprintf(stderr, "libgrid: Error in grid_wf_propagate(). Unknown propagator.\n");
      abort();
  }
}

/* Gross-Pitaevskii step with V_ext + g |psi|^2 built inside the kernels. */
void grid_wf_propagate_gp(wf *gwf, rgrid *vext, REAL g, REAL complex time) {
  switch (gwf->propagator) {
    case WF_2ND_ORDER_FFT:
    case WF_2ND_ORDER_CFFT: {
      const int cutoff = (gwf->propagator == WF_2ND_ORDER_CFFT);
      if (gwf->grid->omega != 0.0) {
        fprintf(stderr, "libgrid: omega != 0.0 allowed only with CN.\n");
        abort();
      }
      if (gwf->ts_func && creal(time) != 0.0) fft_step_with_absorber(gwf, time, NULL, vext, g, cutoff);
      else fused_fft_step(gwf, time, NULL, vext, g, cutoff);
    } break;
    case WF_2ND_ORDER_CN: {
      gb_potential pre, post;
      cn_pot_half(&pre, gwf, 0.5 * time, NULL, vext, g);
      post = pre;
      cn_kinetic_fused(gwf, time, &pre, &post, "grid_wf_propagate_gp");
    } break;
    default:
      gbh_die("grid_wf_propagate_gp(): only the 2nd-order FFT, CFFT and CN propagators are supported");
  }
}

/* ------------------------------------------------------------- the rest */

/* src/grid_wf.c:611-627 */
void grid_wf_density(wf *gwf, rgrid *density) {
  const int p = psi_prec(gwf);
  gb_geom g = wf_geom(gwf);
  const void *c = gbh_dev_read(gwf->grid->value, p);
  void *r = gbh_dev_rw(density->value, GB_FP64);
  gbh_check(gb_mixed_op(GB_MIX_DENSITY, (void *) c, r, NULL, &g, density->nz2, p, GB_FP64), "grid_wf_density");
}

void grid_wf_zero(wf *gwf) { cgrid_zero(gwf->grid); }
void grid_wf_constant(wf *gwf, REAL complex c) { cgrid_constant(gwf->grid, c); }
void grid_wf_map(wf *gwf, REAL complex (*func)(void *arg, REAL x, REAL y, REAL z), void *farg) { cgrid_map(gwf->grid, func, farg); }

/* src/grid_wf.c:681-714 */
REAL grid_wf_norm(wf *gwf) { return cgrid_integral_of_square(gwf->grid); }

REAL grid_wf_normalize(wf *gwf) {
  REAL norm = grid_wf_norm(gwf);
  cgrid_multiply(gwf->grid, sqrt(gwf->norm / norm));
  return norm;
}

REAL complex grid_wf_overlap(wf *gwfa, wf *gwfb) { return cgrid_integral_of_conjugate_product(gwfa->grid, gwfb->grid); }

/* src/grid_wf.c:728-755 */
void grid_wf_merge(wf *dst, cgrid *wfr, cgrid *wfi) {
  const int p = psi_prec(dst);
  gb_geom g = wf_geom(dst);
  const void *r = gbh_dev_read(wfr->value, p);
  const void *i = gbh_dev_read(wfi->value, p);
  void *d = (wfr == dst->grid) ? gbh_dev_rw(dst->grid->value, p) : gbh_dev_write(dst->grid->value, p);
  gbh_check(gb_wf_merge(d, r, i, &g, dst->lx, dst->hx, dst->ly, dst->hy, dst->lz, dst->hz), "grid_wf_merge");
}

/* B200 extension: device storage precision of a wavefunction. */
void grid_wf_precision(wf *gwf, char mode) {
  if (mode != GRID_PREC_FP64 && mode != GRID_PREC_FP32) gbh_die("grid_wf_precision(): unknown mode %d", (int) mode);
  gbh_set_prec(gwf->grid->value, mode == GRID_PREC_FP32 ? GB_FP32 : GB_FP64);
  if (gwf->cworkspace) gbh_set_prec(gwf->cworkspace->value, gbh_prec(gwf->grid->value));
  if (gwf->cworkspace2) gbh_set_prec(gwf->cworkspace2->value, gbh_prec(gwf->grid->value));
  if (gwf->cworkspace3) gbh_set_prec(gwf->cworkspace3->value, gbh_prec(gwf->grid->value));
}

char grid_wf_get_precision(wf *gwf) { return (char) (psi_prec(gwf) == GB_FP32 ? GRID_PREC_FP32 : GRID_PREC_FP64); }

/* npts is kept for symmetry with the other translation units */
size_t gb__wf_points(const wf *gwf) { return npts(gwf->grid); }

/* ------------------------------------------------------------ batches */

struct grid_wf_batch {
  INT n;
  wf **wfs;
  cgrid **pots;
  REAL complex time;
  gb_batch *b;
  void **psi; /* device pointers the batch was built for */
  const void **vdev;
};

/* One instance of a batch: the step fused_fft_step makes for gwf. */
static void batch_item(gb_batch_item *it, wf *gwf, cgrid *cpot, REAL complex time, void **psi, const void **vdev) {
  cgrid *grid = gwf->grid;
  const int p = psi_prec(gwf);
  memset(it, 0, sizeof(*it));
  it->g = wf_geom(gwf);
  REAL complex half = 0.5 * time;
  REAL complex tm = -I * half * HBAR / (gwf->mass * 2.0);
  it->kin.tm_re = creal(tm);
  it->kin.tm_im = cimag(tm);
  it->kin.kx0 = grid->kx0;
  it->kin.ky0 = grid->ky0;
  it->kin.kz0 = grid->kz0;
  it->kin.scale = grid->fft_norm;
  it->kin.kmax2 = gwf->kmax * gwf->kmax;
  it->kin.cutoff = 0;
  *vdev = NULL;
  if (cpot) {
    REAL complex c = -I * time / HBAR;
    it->pot.c_re = creal(c);
    it->pot.c_im = cimag(c);
    it->pot.cons = frame_cons(gwf);
    it->pot.kind = GB_POT_COMPLEX;
    *vdev = gbh_dev_read(cpot->value, p);
    it->pot.v = *vdev;
    it->pot.vrow = cpot->nz;
  }
  *psi = gbh_dev_rw(grid->value, p);
  it->psi = *psi;
}

static gb_batch *batch_build(grid_wf_batch *bb) {
  gb_batch_item *items = (gb_batch_item *) malloc(sizeof(gb_batch_item) * (size_t) bb->n);
  for (INT i = 0; i < bb->n; i++)
    batch_item(&items[i], bb->wfs[i], bb->pots ? bb->pots[i] : NULL, bb->time, &bb->psi[i], &bb->vdev[i]);
  gb_batch *b = gb_batch_create(items, (int) bb->n);
  free(items);
  return b;
}

grid_wf_batch *grid_wf_batch_alloc(wf **wfs, cgrid **potentials, INT n, REAL complex time) {
  if (n <= 0 || !wfs) gbh_die("grid_wf_batch_alloc(): no wave functions");
  const int p = psi_prec(wfs[0]);
  for (INT i = 0; i < n; i++) {
    wf *w = wfs[i];
    if (w->propagator != WF_2ND_ORDER_FFT || w->boundary != WF_PERIODIC_BOUNDARY)
      gbh_die("grid_wf_batch_alloc(): wave functions must use WF_2ND_ORDER_FFT with periodic boundaries");
    if (w->ts_func) gbh_die("grid_wf_batch_alloc(): absorbing boundaries are not batched");
    if (psi_prec(w) != p) gbh_die("grid_wf_batch_alloc(): all wave functions must have one precision");
  }
  grid_wf_batch *bb = (grid_wf_batch *) calloc(1, sizeof(grid_wf_batch));
  bb->n = n;
  bb->time = time;
  bb->wfs = (wf **) malloc(sizeof(wf *) * (size_t) n);
  memcpy(bb->wfs, wfs, sizeof(wf *) * (size_t) n);
  if (potentials) {
    bb->pots = (cgrid **) malloc(sizeof(cgrid *) * (size_t) n);
    memcpy(bb->pots, potentials, sizeof(cgrid *) * (size_t) n);
  }
  bb->psi = (void **) calloc((size_t) n, sizeof(void *));
  bb->vdev = (const void **) calloc((size_t) n, sizeof(void *));
  bb->b = batch_build(bb);
  if (!bb->b) gbh_check(gb_last_error() ? gb_last_error() : -1, "grid_wf_batch_alloc");
  return bb;
}

void grid_wf_batch_propagate(grid_wf_batch *bb, INT steps) {
  /* bring device copies up to date (host-side changes) and rebuild the
   * batch if any device buffer moved */
  int moved = 0;
  for (INT i = 0; i < bb->n; i++) {
    const int p = psi_prec(bb->wfs[i]);
    if (gbh_dev_rw(bb->wfs[i]->grid->value, p) != bb->psi[i]) moved = 1;
    if (bb->pots && bb->pots[i] && gbh_dev_read(bb->pots[i]->value, p) != bb->vdev[i]) moved = 1;
  }
  if (moved) {
    gb_batch_free(bb->b);
    bb->b = batch_build(bb);
    if (!bb->b) gbh_check(gb_last_error() ? gb_last_error() : -1, "grid_wf_batch_propagate");
  }
  gbh_check(gb_batch_step(bb->b, (int) steps), "grid_wf_batch_propagate");
}

int grid_wf_batch_threads(grid_wf_batch *bb) { return bb ? gb_batch_threads(bb->b) : 0; }

void grid_wf_batch_free(grid_wf_batch *bb) {
  if (!bb) return;
  gb_batch_free(bb->b);
  free(bb->wfs);
  free(bb->pots);
  free(bb->psi);
  free(bb->vdev);
  free(bb);
}

/* ------------------------------------------------------ multi-step calls */

/* nsteps steps with the k-space state kept between them when the propagator
 * allows it (2nd-order FFT / CFFT without an absorbing region): the same
 * result as nsteps calls of grid_wf_propagate to rounding, with about half
 * the memory traffic.  Other propagators make nsteps ordinary steps. */
void grid_wf_propagate_n(wf *gwf, cgrid *potential, REAL complex time, INT nsteps) {
  const int fft2 = gwf->propagator == WF_2ND_ORDER_FFT || gwf->propagator == WF_2ND_ORDER_CFFT;
  if (fft2 && !(gwf->ts_func && creal(time) != 0.0) && gwf->grid->omega == 0.0 && nsteps > 1 && nsteps < (1L << 30)) {
    fused_fft_steps(gwf, time, potential, NULL, 0.0, gwf->propagator == WF_2ND_ORDER_CFFT, (int) nsteps);
    return;
  }
  for (INT s = 0; s < nsteps; s++) grid_wf_propagate(gwf, potential, time);
}

void grid_wf_propagate_gp_n(wf *gwf, rgrid *vext, REAL g, REAL complex time, INT nsteps) {
  const int fft2 = gwf->propagator == WF_2ND_ORDER_FFT || gwf->propagator == WF_2ND_ORDER_CFFT;
  if (fft2 && !(gwf->ts_func && creal(time) != 0.0) && gwf->grid->omega == 0.0 && nsteps > 1 && nsteps < (1L << 30)) {
    fused_fft_steps(gwf, time, NULL, vext, g, gwf->propagator == WF_2ND_ORDER_CFFT, (int) nsteps);
    return;
  }
  for (INT s = 0; s < nsteps; s++) grid_wf_propagate_gp(gwf, vext, g, time);
}

/* Imaginary-time relaxation steps (no reference counterpart as one call; the
 * reference's callers compose grid_wf_propagate(-i dt) and grid_wf_normalize,
 * src/grid_wf.c:379-556, 681-700): nsteps of grid_wf_propagate_gp(time), each
 * followed by renormalisation to gwf->norm, with the norm reduced and applied
 * on the device, so the whole loop runs without a host synchronisation. */
void grid_wf_relax_gp_n(wf *gwf, rgrid *vext, REAL g, REAL complex time, INT nsteps) {
  cgrid *grid = gwf->grid;
  for (INT s = 0; s < nsteps; s++) {
    grid_wf_propagate_gp(gwf, vext, g, time);
    const int p = psi_prec(gwf);
    gb_geom geo = wf_geom(gwf);
    gbh_check(gb_normalize_device(gbh_dev_rw(grid->value, p), &geo, gwf->norm,
                                  gbh_step_factor(grid->nx, grid->ny, grid->nz, grid->step)),
              "grid_wf_relax_gp_n");
  }
}

/* psi = max(amp * scale, 0) + floor (real) from a device float array of
 * nx ny nz values, e.g. a network's guess (no reference counterpart). */
void grid_wf_set_amplitude_device(wf *gwf, const float *amp, REAL scale, REAL floor) {
  cgrid *grid = gwf->grid;
  const int p = psi_prec(gwf);
  gbh_check(gb_unet_amplitude(amp, (float) scale, (float) floor, gbh_dev_write(grid->value, p), (long) npts(grid), p),
            "grid_wf_set_amplitude_device");
}
