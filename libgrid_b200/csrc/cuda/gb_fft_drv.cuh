// Pass schedules built on the line-pass engine (gb_fft_impl.cuh).
#pragma once

#include "gb_fft_impl.cuh"
#include "gb_plane.cuh"
#include "gb_internal_cuda.h"

namespace gbfft {

struct View {
  long outer, n, inner;
};

inline View axis_view(const gb_geom *g, int axis) {
  if (axis == 2) return View{g->nx * g->ny, g->nz, 1};
  if (axis == 1) return View{g->nx, g->ny, g->nz};
  return View{1, g->nx, g->ny * g->nz};
}

inline int active_axes(const gb_geom *g, int *ax) {
  int na = 0;
  if (g->nz > 1) ax[na++] = 2;
  if (g->ny > 1) ax[na++] = 1;
  if (g->nx > 1) ax[na++] = 0;
  return na;
}

inline PassArgs base_args(const gb_geom *g) {
  PassArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = g->nx;
  a.ny = g->ny;
  a.nz = g->nz;
  a.scale = 1.0;
  a.kscale = 1.0;
  return a;
}

// Program id for pass timing: 0 {FWD}, 1 {INV}, 2 {FWD,KIN,INV},
// 3 {INV,POT,FWD}, 4 anything else; kind = 5 * axis + id.
template <int... Ops> constexpr int prog_id(OpL<Ops...>) {
  constexpr int n = sizeof...(Ops);
  constexpr int o[] = {Ops...};
  if (n == 1 && o[0] == OP_FWD) return 0;
  if (n == 1 && o[0] == OP_INV) return 1;
  if (n == 3 && o[0] == OP_FWD && o[1] == OP_KIN && o[2] == OP_INV) return 2;
  if (n == 3 && o[0] == OP_INV && o[1] == OP_POT && o[2] == OP_FWD) return 3;
  return 4;
}

template <typename T, int... Ops>
int pass(const gb_geom *g, int axis, const void *src, void *dst, PassArgs a, OpL<Ops...> ops) {
  const View v = axis_view(g, axis);
  a.axis = axis;
  a.tw = gb__twiddles(v.n, g->prec);
  if (!a.tw) return gb_last_error();
  a.errflag = gb__pass_errflag();
  if (!a.errflag) return gb_last_error();
  const int slot = gb__pass_begin(5 * axis + prog_id(ops));
  const int rc = launch_pass<T>(v.n, src, dst, a, v.outer, v.inner, ops);
  gb__pass_end(slot);
  return rc;
}

// Plane-chained passes (gb_plane.cuh) for grids whose y and z lines are
// 256 long.  The chain counters live in a scratch slot (stages x planes + 1
// ints).
constexpr int kPlaneN = 256;
int plane_enabled();

template <typename T> bool plane_ok(const gb_geom *g) {
  return plane_enabled() && g->nx >= 2 && g->ny == kPlaneN && g->nz == kPlaneN;
}

// Timing kinds of the chains: 18 [z FWD, y FWD], 19 [z INV.V.FWD (or
// INV.FWD), y FWD], 20 [y INV, z INV], 21 [y INV, z INV.V.FWD, y FWD],
// 22 [z INV, V.y FWD, z FWD].
template <typename T, class... Stages>
int plane_chain(const gb_geom *g, void *psi, const PassArgs &a, int kind, Stages...) {
  ChainArgs c;
  memset(&c, 0, sizeof(c));
  c.ay = a;
  c.az = a;
  c.ay.axis = 1;
  c.az.axis = 2;
  c.ay.tw = c.az.tw = gb__twiddles(kPlaneN, g->prec);
  if (!c.ay.tw) return gb_last_error();
  c.ay.errflag = c.az.errflag = gb__pass_errflag();
  if (!c.ay.errflag) return gb_last_error();
  int *cnt = (int *) gb__scratch(GB_SCR_CHAIN, sizeof(int) * (size_t) (3 * g->nx + 1));
  if (!cnt) return gb_last_error();
  const int slot = gb__pass_begin(kind);
  const int rc = launch_chain<T, kPlaneN, Stages...>(psi, g->nx, c, cnt);
  gb__pass_end(slot);
  return rc;
}

// The middle of the step, y INV | z INV.V.FWD | y FWD.  In FP64 the last
// two run as one chain (the potential stage at 3 CTAs per SM); in FP32 the
// chain is slower than the two passes, and all three stay line passes.
template <typename T> int plane_mid(const gb_geom *g, void *psi, const PassArgs &a, bool has_pot) {
  if constexpr (sizeof(T) == 8) {
    // schedule 3 (real-time steps with a real V_ext): y INV | [z INV, V.y FWD, z FWD]
    // (kind 22), the potential applied in the y stage before its forward
    // transform, so no stage carries two transforms
    if (plane_enabled() == 3 && has_pot && a.pot.kind == GB_POT_REAL && !a.pot.absorb && a.pot.c_re == 0.0) {
      const int rc = pass<T>(g, 1, psi, psi, a, OpL<OP_INV>{});
      if (rc) return rc;
      return plane_chain<T>(g, psi, a, 22, Stage<2, OP_INV>{}, Stage<1, OP_POT_RP, OP_FWD>{}, Stage<2, OP_FWD>{});
    }
    // schedule 2: the y INV pass joins the chain as its first stage (kind 21)
    if (plane_enabled() == 2) {
      if (has_pot && a.pot.kind == GB_POT_REAL && !a.pot.absorb && a.pot.c_re == 0.0)
        return plane_chain<T>(g, psi, a, 21, Stage<1, OP_INV>{}, Stage<2, OP_INV, OP_POT_RP, OP_FWD>{},
                              Stage<1, OP_FWD>{});
      return has_pot ? plane_chain<T>(g, psi, a, 21, Stage<1, OP_INV>{}, Stage<2, OP_INV, OP_POT, OP_FWD>{},
                                      Stage<1, OP_FWD>{})
                     : plane_chain<T>(g, psi, a, 21, Stage<1, OP_INV>{}, Stage<2, OP_INV, OP_FWD>{},
                                      Stage<1, OP_FWD>{});
    }
  }
  int rc = pass<T>(g, 1, psi, psi, a, OpL<OP_INV>{});
  if (rc) return rc;
  if constexpr (sizeof(T) == 8) {
    // real-time steps with a real V_ext (the GP workload) get a chain built
    // for that potential case alone
    if (has_pot && a.pot.kind == GB_POT_REAL && !a.pot.absorb && a.pot.c_re == 0.0)
      return plane_chain<T>(g, psi, a, 19, Stage<2, OP_INV, OP_POT_RP, OP_FWD>{}, Stage<1, OP_FWD>{});
    return has_pot ? plane_chain<T>(g, psi, a, 19, Stage<2, OP_INV, OP_POT, OP_FWD>{}, Stage<1, OP_FWD>{})
                   : plane_chain<T>(g, psi, a, 19, Stage<2, OP_INV, OP_FWD>{}, Stage<1, OP_FWD>{});
  } else {
    rc = has_pot ? pass<T>(g, 2, psi, psi, a, OpL<OP_INV, OP_POT, OP_FWD>{})
                 : pass<T>(g, 2, psi, psi, a, OpL<OP_INV, OP_FWD>{});
    if (!rc) rc = pass<T>(g, 1, psi, psi, a, OpL<OP_FWD>{});
    return rc;
  }
}

#define GB_TRY(x)               \
  do {                          \
    int rc_ = (x);              \
    if (rc_) return rc_;        \
  } while (0)

}  // namespace gbfft

template <typename T> int gb__fft3d_t(void *data, const gb_geom *g, int sign, double scale) {
  using namespace gbfft;
  int ax[3];
  const int na = active_axes(g, ax);
  if (na == 0) {
    if (scale != 1.0) return gb_complex_op(GB_OP_SCALE, data, nullptr, nullptr, 1, scale, 0.0, g->prec);
    return 0;
  }
  PassArgs a = base_args(g);
  a.scale = scale;
  for (int s = 0; s < na; s++) {
    const bool last = (s == na - 1);
    if (sign < 0) {
      if (last && scale != 1.0) GB_TRY((pass<T>(g, ax[s], data, data, a, OpL<OP_FWD, OP_SCALE>{})));
      else GB_TRY((pass<T>(g, ax[s], data, data, a, OpL<OP_FWD>{})));
    } else {
      if (last && scale != 1.0) GB_TRY((pass<T>(g, ax[s], data, data, a, OpL<OP_INV, OP_SCALE>{})));
      else GB_TRY((pass<T>(g, ax[s], data, data, a, OpL<OP_INV>{})));
    }
  }
  return 0;
}

template <typename T>
int gb__split_step_t(void *psi, const gb_geom *g, const gb_kinetic *kin, const gb_potential *pot) {
  using namespace gbfft;
  int ax[3];
  const int na = active_axes(g, ax);
  PassArgs a = base_args(g);
  GbKinTables kt;
  GB_TRY(gb__kin_tables(g, kin, 0, &kt));
  for (int d = 0; d < 3; d++) {
    a.kfac[d] = kt.kfac[d];
    a.ksq[d] = kt.ksq[d];
  }
  a.kscale = kin->scale;
  a.cutoff = kin->cutoff;
  a.kmax2 = kin->kmax2;
  const bool has_pot = (pot != nullptr);
  if (has_pot) a.pot = *pot;
  if (na == 0) return gb__set_error(1004, "split step: empty grid");
  if (na == 1) {
    if (has_pot)
      return pass<T>(g, ax[0], psi, psi, a, OpL<OP_FWD, OP_KIN, OP_INV, OP_POT, OP_FWD, OP_KIN, OP_INV>{});
    return pass<T>(g, ax[0], psi, psi, a, OpL<OP_FWD, OP_KIN, OP_INV, OP_FWD, OP_KIN, OP_INV>{});
  }
  if (na == 3 && plane_ok<T>(g)) {
    // [z FWD, y FWD] | x FWD.K.INV | y INV | [z INV.V.FWD, y FWD] (FP64; FP32: two passes) | x FWD.K.INV |
    // [y INV, z INV]
    GB_TRY((plane_chain<T>(g, psi, a, 18, Stage<2, OP_FWD>{}, Stage<1, OP_FWD>{})));
    GB_TRY((pass<T>(g, 0, psi, psi, a, OpL<OP_FWD, OP_KIN, OP_INV>{})));
    GB_TRY(plane_mid<T>(g, psi, a, has_pot));
    GB_TRY((pass<T>(g, 0, psi, psi, a, OpL<OP_FWD, OP_KIN, OP_INV>{})));
    return plane_chain<T>(g, psi, a, 20, Stage<1, OP_INV>{}, Stage<2, OP_INV>{});
  }
  const int last = ax[na - 1];
  // forward along all but the outermost axis
  for (int s = 0; s < na - 1; s++) GB_TRY((pass<T>(g, ax[s], psi, psi, a, OpL<OP_FWD>{})));
  // outermost axis: forward, kinetic factor (1/N folded in), inverse
  GB_TRY((pass<T>(g, last, psi, psi, a, OpL<OP_FWD, OP_KIN, OP_INV>{})));
  for (int s = na - 2; s >= 1; s--) GB_TRY((pass<T>(g, ax[s], psi, psi, a, OpL<OP_INV>{})));
  // innermost axis: back to real space, potential factor, forward again
  if (has_pot) GB_TRY((pass<T>(g, ax[0], psi, psi, a, OpL<OP_INV, OP_POT, OP_FWD>{})));
  else GB_TRY((pass<T>(g, ax[0], psi, psi, a, OpL<OP_INV, OP_FWD>{})));
  for (int s = 1; s < na - 1; s++) GB_TRY((pass<T>(g, ax[s], psi, psi, a, OpL<OP_FWD>{})));
  GB_TRY((pass<T>(g, last, psi, psi, a, OpL<OP_FWD, OP_KIN, OP_INV>{})));
  for (int s = na - 2; s >= 1; s--) GB_TRY((pass<T>(g, ax[s], psi, psi, a, OpL<OP_INV>{})));
  GB_TRY((pass<T>(g, ax[0], psi, psi, a, OpL<OP_INV>{})));
  return 0;
}

// nsteps consecutive split-operator steps with the k-space state kept
// between them: the trailing inverse transforms of one step and the leading
// forward transforms of the next cancel, and the two K(dt/2) factors that
// then meet on the outermost axis merge into one K(dt) pass.  Every FWD.K.INV
// pass closes one round trip per axis, so each keeps the 1/N factor.  Steady
// state: outermost FWD.K(dt).INV, middle INV, innermost INV.V.FWD, middle FWD.
template <typename T>
int gb__split_steps_t(void *psi, const gb_geom *g, const gb_kinetic *kin, const gb_potential *pot, int nsteps) {
  using namespace gbfft;
  int ax[3];
  const int na = active_axes(g, ax);
  if (nsteps <= 0) return 0;
  if (na < 2 || nsteps == 1) {
    for (int s = 0; s < nsteps; s++) GB_TRY(gb__split_step_t<T>(psi, g, kin, pot));
    return 0;
  }
  PassArgs ah = base_args(g);
  GbKinTables kt;
  GB_TRY(gb__kin_tables(g, kin, 0, &kt));
  for (int d = 0; d < 3; d++) {
    ah.kfac[d] = kt.kfac[d];
    ah.ksq[d] = kt.ksq[d];
  }
  ah.kscale = kin->scale;
  ah.cutoff = kin->cutoff;
  ah.kmax2 = kin->kmax2;
  const bool has_pot = (pot != nullptr);
  if (has_pot) ah.pot = *pot;
  // K(dt): the same factor with twice the exponent, in its own tables
  gb_kinetic kf = *kin;
  kf.tm_re *= 2.0;
  kf.tm_im *= 2.0;
  const long tot = g->nx + g->ny + g->nz;
  const size_t esz = sizeof(C2<T>);
  unsigned char *fb = (unsigned char *) gb__scratch(GB_SCR_KIN2, (size_t) tot * (esz + 8));
  if (!fb) return gb_last_error();
  double *fsq = (double *) (fb + (size_t) tot * esz);
  GB_TRY(gb__kin_tables_at(fb, fsq, g, &kf));
  PassArgs af = ah;
  af.kfac[0] = fb;
  af.kfac[1] = fb + esz * (size_t) g->nx;
  af.kfac[2] = fb + esz * (size_t) (g->nx + g->ny);
  af.ksq[0] = fsq;
  af.ksq[1] = fsq + g->nx;
  af.ksq[2] = fsq + g->nx + g->ny;
  if (na == 3 && plane_ok<T>(g)) {
    // steady state x FWD.K(dt).INV | y INV | [z INV.V.FWD, y FWD] (FP64), with the leading
    // and trailing transform pairs chained
    GB_TRY((plane_chain<T>(g, psi, ah, 18, Stage<2, OP_FWD>{}, Stage<1, OP_FWD>{})));
    for (int st = 0; st < nsteps; st++) {
      GB_TRY((pass<T>(g, 0, psi, psi, st == 0 ? ah : af, OpL<OP_FWD, OP_KIN, OP_INV>{})));
      GB_TRY(plane_mid<T>(g, psi, ah, has_pot));
    }
    GB_TRY((pass<T>(g, 0, psi, psi, ah, OpL<OP_FWD, OP_KIN, OP_INV>{})));
    return plane_chain<T>(g, psi, ah, 20, Stage<1, OP_INV>{}, Stage<2, OP_INV>{});
  }
  const int last = ax[na - 1];
  for (int s = 0; s < na - 1; s++) GB_TRY((pass<T>(g, ax[s], psi, psi, ah, OpL<OP_FWD>{})));
  for (int st = 0; st < nsteps; st++) {
    GB_TRY((pass<T>(g, last, psi, psi, st == 0 ? ah : af, OpL<OP_FWD, OP_KIN, OP_INV>{})));
    for (int s = na - 2; s >= 1; s--) GB_TRY((pass<T>(g, ax[s], psi, psi, ah, OpL<OP_INV>{})));
    if (has_pot) GB_TRY((pass<T>(g, ax[0], psi, psi, ah, OpL<OP_INV, OP_POT, OP_FWD>{})));
    else GB_TRY((pass<T>(g, ax[0], psi, psi, ah, OpL<OP_INV, OP_FWD>{})));
    for (int s = 1; s < na - 1; s++) GB_TRY((pass<T>(g, ax[s], psi, psi, ah, OpL<OP_FWD>{})));
  }
  GB_TRY((pass<T>(g, last, psi, psi, ah, OpL<OP_FWD, OP_KIN, OP_INV>{})));
  for (int s = na - 2; s >= 0; s--) GB_TRY((pass<T>(g, ax[s], psi, psi, ah, OpL<OP_INV>{})));
  return 0;
}

template <typename T> int gb__ksq_sum_t(const void *psi, void *work, const gb_geom *g, double *out) {
  using namespace gbfft;
  int ax[3];
  const int na = active_axes(g, ax);
  if (na == 0) {
    *out = 0.0;
    return 0;
  }
  gb_kinetic kin;
  memset(&kin, 0, sizeof(kin));
  kin.scale = 1.0;
  GbKinTables kt;
  GB_TRY(gb__kin_tables(g, &kin, 1, &kt));
  PassArgs a = base_args(g);
  for (int d = 0; d < 3; d++) {
    a.kfac[d] = kt.kfac[d];
    a.ksq[d] = kt.ksq[d];
  }
  const void *src = psi;
  for (int s = 0; s < na - 1; s++) {
    GB_TRY((pass<T>(g, ax[s], src, work, a, OpL<OP_FWD>{})));
    src = work;
  }
  const View v = axis_view(g, ax[na - 1]);
  const long nb = blocks_for<(int) sizeof(T)>(v.n, v.outer, v.inner);
  double *partial = (double *) gb__scratch(GB_SCR_PARTIAL, sizeof(double) * (size_t) nb);
  if (!partial) return gb_last_error();
  a.partial = partial;
  GB_TRY((pass<T>(g, ax[na - 1], src, nullptr, a, OpL<OP_FWD, OP_KSQ>{})));
  return gb__sum_partials(partial, nb, out);
}
