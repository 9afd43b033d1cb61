"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs libgrid's own CPU sources (compiled unchanged into oracle/_ref by
oracle/build_ref.sh) on small seeded cases and records the outputs.  Inputs
are rebuilt from libgrid_b200.workloads with the seeds stored alongside, so
only outputs are saved.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libgrid_b200 import capi, workloads  # noqa: E402
from oracle import pyoracle  # noqa: E402


def wavepacket_case(ref):
    # The real-time harmonic wavepacket at 16^3 (box 25.6 bohr as at 128^3).
    n, step, mass, dt = 16, 1.6, 1.0, 0.05
    psi0, v = workloads.wavepacket(n, step)
    w = ref.wf(n, n, n, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT, values=psi0)
    ref.lib.grid_wf_normalize(w.ptr)
    pot = ref.cgrid(n, n, n, step, values=v)
    vr = ref.rgrid(n, n, n, step, values=v.real)
    out = {"psi_start": w.grid.get()}
    ref.lib.grid_wf_analyze_method(b"\x01")
    for s in range(1, 21):
        w.propagate(pot, dt)
        if s % 10 == 0:
            out["psi_%d" % s] = w.grid.get()
            out["norm_%d" % s] = ref.lib.grid_wf_norm(w.ptr)
            out["ekin_fft_%d" % s] = ref.lib.grid_wf_kinetic_energy_fft(w.ptr)
            out["epot_%d" % s] = ref.lib.grid_wf_potential_energy(w.ptr, vr.ptr)
    ref.lib.grid_wf_analyze_method(b"\x00")
    out["ekin_fd_20"] = ref.lib.grid_wf_kinetic_energy_cn(w.ptr)
    meta = dict(n=n, step=step, mass=mass, dt=dt)
    return out, meta


def gp_case(ref):
    # GP split step with V_ext + g |psi|^2 composed from reference primitives:
    # K(dt/2) -> V_ext + g |psi_mid|^2 -> potential(dt) -> K(dt/2).
    shape, step, g, dt, seed = (16, 16, 16), 0.5, 0.0025, 1.0, 21
    mass = 4.0 / capi.GRID_AUTOAMU
    psi0, v = workloads.gp_wells(shape, step, g, seed)
    w = ref.wf(*shape, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT, values=psi0)
    vext = ref.rgrid(*shape, step, values=v)
    dens = ref.rgrid(*shape, step)
    pot = ref.cgrid(*shape, step)
    vc = ref.cgrid(*shape, step)
    ref.lib.grid_real_to_complex_re(vc.ptr, vext.ptr)
    for _ in range(5):
        ref.lib.cgrid_fft(w.s.grid)
        ref.lib.grid_wf_propagate_kinetic_fft(w.ptr, capi.Complex.of(0.5 * dt))
        ref.lib.cgrid_inverse_fft_norm(w.s.grid)
        ref.lib.grid_wf_density(w.ptr, dens.ptr)
        ref.lib.grid_real_to_complex_re(pot.ptr, dens.ptr)
        ref.lib.cgrid_multiply(pot.ptr, capi.Complex.of(g))
        ref.lib.cgrid_sum(pot.ptr, pot.ptr, vc.ptr)
        ref.lib.grid_wf_propagate_potential(w.ptr, capi.Complex.of(dt), pot.ptr, 0.0)
        ref.lib.cgrid_fft(w.s.grid)
        ref.lib.grid_wf_propagate_kinetic_fft(w.ptr, capi.Complex.of(0.5 * dt))
        ref.lib.cgrid_inverse_fft_norm(w.s.grid)
    out = {"psi_5": w.grid.get(), "norm_5": ref.lib.grid_wf_norm(w.ptr)}
    return out, dict(shape=shape, step=step, g=g, dt=dt, seed=seed, mass=mass)


def cn_case(ref):
    # Dirichlet CN (GP form): V(dt/2) with |psi(t)|^2, CN(dt), V(dt/2) with
    # |psi_CN|^2, composed from reference primitives.
    shape, step, g, dt, seed = (12, 10, 14), 0.3, 0.001, 0.5, 31
    mass = 4.0 / capi.GRID_AUTOAMU
    psi0, v = workloads.cn_wells(shape, step, g, seed)
    w = ref.wf(*shape, step, mass, capi.WF_DIRICHLET_BOUNDARY, capi.WF_2ND_ORDER_CN, values=psi0)
    # the reference's non-periodic CN sweeps dereference the third workspace
    # pointer even though only the periodic case allocates it
    # (src/grid_wf_cn.c:72-74,126); the caller provides it
    ws3 = ref.cgrid(*shape, step, bc="dirichlet")
    w.s.cworkspace3 = ws3.ptr
    vext = ref.rgrid(*shape, step, values=v)
    dens = ref.rgrid(*shape, step)
    pot = ref.cgrid(*shape, step)
    vc = ref.cgrid(*shape, step)
    ref.lib.grid_real_to_complex_re(vc.ptr, vext.ptr)

    def half_potential():
        ref.lib.grid_wf_density(w.ptr, dens.ptr)
        ref.lib.grid_real_to_complex_re(pot.ptr, dens.ptr)
        ref.lib.cgrid_multiply(pot.ptr, capi.Complex.of(g))
        ref.lib.cgrid_sum(pot.ptr, pot.ptr, vc.ptr)
        ref.lib.grid_wf_propagate_potential(w.ptr, capi.Complex.of(0.5 * dt), pot.ptr, 0.0)

    for _ in range(5):
        half_potential()
        ref.lib.grid_wf_propagate_kinetic_cn(w.ptr, capi.Complex.of(dt))
        half_potential()
    out = {"psi_5": w.grid.get(), "norm_5": ref.lib.grid_wf_norm(w.ptr)}
    ref.lib.grid_wf_analyze_method(b"\x00")
    out["ekin_fd_5"] = ref.lib.grid_wf_kinetic_energy_cn(w.ptr)
    return out, dict(shape=shape, step=step, g=g, dt=dt, seed=seed, mass=mass)


def main():
    ref = pyoracle.reference(4)
    for name, fn in (("wavepacket16", wavepacket_case), ("gp16", gp_case), ("cn_dirichlet", cn_case)):
        out, meta = fn(ref)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out, **{"meta_" + k: np.asarray(v) for k, v in meta.items()})
        print("wrote", name)


if __name__ == "__main__":
    main()
