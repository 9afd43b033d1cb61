/*
 * Seeded noise on grids: the reference's src/rand.c API (grid_random_seed
 * and the rgrid / cgrid random_* calls) on the device, through gb_random.
 * One process-wide seed and call counter: every call draws a fresh stream
 * (seed, call number), so a given seed and call sequence reproduces its
 * values.  Unseeded use seeds from the time of day, as the reference does
 * (src/rand.c:57-60).
 */
#include <time.h>

#include "gb_host.h"

static int rand_init = 0;
static unsigned long long rand_seed = 0, rand_call = 0;

static void rand_check(void) {
  if (!rand_init) {
    rand_seed = (unsigned long long) time(0);
    rand_call = 0;
    rand_init = 1;
  }
}

/* src/rand.c:34-45 (the grid dimensions only sized the reference's cuRAND
 * state arrays; a counter-based generator keeps no state) */
void grid_random_seed(INT nx, INT ny, INT nz, INT seed) {
  (void) nx;
  (void) ny;
  (void) nz;
  rand_seed = (unsigned long long) seed;
  rand_call = 0;
  rand_init = 1;
}

static void rgrid_noise(rgrid *grid, int kind, REAL scale) {
  rand_check();
  const int p = gbh_prec(grid->value);
  gb_geom g = gbh_geom(grid->nx, grid->ny, grid->nz, grid->step, p);
  gbh_check(gb_random(kind, gbh_dev_rw(grid->value, p), &g, grid->nz2, scale, 0.0, rand_seed, rand_call++),
            "rgrid_random");
}

static void cgrid_noise(cgrid *grid, int kind, REAL complex scale) {
  rand_check();
  const int p = gbh_prec(grid->value);
  gb_geom g = gbh_geom(grid->nx, grid->ny, grid->nz, grid->step, p);
  gbh_check(gb_random(kind, gbh_dev_rw(grid->value, p), &g, grid->nz, creal(scale), cimag(scale), rand_seed,
                      rand_call++),
            "cgrid_random");
}

/* src/rand.c:55-74 */
void rgrid_random_uniform(rgrid *grid, REAL scale) { rgrid_noise(grid, GB_RAND_R_UNIFORM, scale); }
/* src/rand.c:84-122 */
void rgrid_random_normal(rgrid *grid, REAL scale) { rgrid_noise(grid, GB_RAND_R_NORMAL, scale); }
/* src/rand.c:132-149 */
void cgrid_random_uniform(cgrid *grid, REAL complex scale) { cgrid_noise(grid, GB_RAND_C_UNIFORM, scale); }
/* src/rand.c:159-176 */
void cgrid_random_uniform_sp(cgrid *grid, REAL scale) { cgrid_noise(grid, GB_RAND_C_UNIFORM_SP, scale); }
/* src/rand.c:186-214 */
void cgrid_random_normal(cgrid *grid, REAL complex scale) { cgrid_noise(grid, GB_RAND_C_NORMAL, scale); }
/* src/rand.c:224-250 */
void cgrid_random_normal_sp(cgrid *grid, REAL scale) { cgrid_noise(grid, GB_RAND_C_NORMAL_SP, scale); }
