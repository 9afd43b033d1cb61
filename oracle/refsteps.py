"""ORACLE (test infrastructure only).

Steppers that advance a wavefunction of the reference's own CPU build
(oracle/_ref, libgrid's src/*.c compiled unchanged) through the propagation
workloads, composed from the reference's exported primitives exactly as the
GPU path's definitions state.  Used by tests/, by the fixture scripts under
tests/golden/ and by bench.py's CPU-baseline leg; never by the library.

  WavepacketStepper  grid_wf_propagate (2nd-order FFT) with a complex
                     potential grid: src/grid_wf.c:424-430
  GPStepper          the Gross-Pitaevskii FFT split step:
                     FFT, K(dt/2), IFFT/N, rho = |psi|^2, V = V_ext + g rho,
                     grid_wf_propagate_potential(dt), FFT, K(dt/2), IFFT/N
                     (src/grid_wf_fft.c:141-193, src/grid_wf.c:569-600,
                     src/grid_wf.c:611-627, src/ngrid.c:53, src/cgrid.c:934,1223)
  CNGPStepper        the Gross-Pitaevskii Crank-Nicolson step:
                     V(dt/2) with |psi(t)|^2, grid_wf_propagate_kinetic_cn(dt),
                     V(dt/2) with |psi after CN|^2 (src/grid_wf.c:526-530,
                     src/grid_wf_cn.c:65-79)

Observables (`observables()`): the norm (grid_wf_norm), the kinetic energy
by the stepper's analysis method (FFT: grid_wf_kinetic_energy_fft; CN:
grid_wf_kinetic_energy_cn, the finite-difference one), <V> by
grid_grid_expectation_value, and for the GP forms the interaction term
(g/2) sum |psi|^4 h^3 evaluated in numpy from the full psi.
"""
from __future__ import annotations

import numpy as np

from libgrid_b200 import capi


def interaction_energy(psi: np.ndarray, step: float, g: float) -> float:
    """(g/2) * integral |psi|^4, every axis of length > 1 contributing one
    step factor (the reference's integral convention, src/cgrid.c:1610-1629)."""
    rho = psi.real * psi.real + psi.imag * psi.imag
    h = step ** sum(1 for n in psi.shape if n > 1)
    return 0.5 * g * float(np.sum(rho * rho)) * h


class _Base:
    def __init__(self, ref, psi0, step, mass, bc, prop):
        self.ref, self.lib, self.step, self.mass = ref, ref.lib, step, mass
        self.shape = psi0.shape
        bcname = {capi.WF_DIRICHLET_BOUNDARY: "dirichlet", capi.WF_NEUMANN_BOUNDARY: "neumann"}.get(bc, "periodic")
        self.bcname = bcname
        self.w = ref.wf(*self.shape, step, mass, bc, prop, values=psi0)
        self._owned = [self.w]
        if bc != capi.WF_PERIODIC_BOUNDARY:
            # the reference's non-periodic CN sweeps dereference the third
            # workspace pointer although only the periodic case allocates it
            # (src/grid_wf_cn.c:72-74,126); the caller provides it
            # (grid_wf_free releases it with the wavefunction, src/grid_wf.c:157-166)
            ws3 = ref.cgrid(*self.shape, step, bc=bcname)
            self.w.s.cworkspace3 = ws3.ptr

    def psi(self) -> np.ndarray:
        return self.w.grid.get()

    def norm(self) -> float:
        return self.lib.grid_wf_norm(self.w.ptr)

    def free(self):
        for o in self._owned:
            self.ref.free(o)
        self._owned = []


class WavepacketStepper(_Base):
    """2nd-order FFT propagation with a complex potential grid (the harmonic
    wavepacket workload); the real part of V is kept as an rgrid for <V>."""

    def __init__(self, ref, psi0, v, step, mass, dt, normalize=True):
        super().__init__(ref, psi0, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT)
        self.dt = dt
        if normalize:
            self.lib.grid_wf_normalize(self.w.ptr)
        self.pot = ref.cgrid(*self.shape, step, values=v)
        self.vr = ref.rgrid(*self.shape, step, values=np.asarray(v).real)
        self._owned += [self.pot, self.vr]

    def step_once(self):
        self.w.propagate(self.pot, self.dt)

    def observables(self, psi=None) -> dict:
        self.lib.grid_wf_analyze_method(b"\x01")
        return {
            "norm": self.norm(),
            "ekin": self.lib.grid_wf_kinetic_energy_fft(self.w.ptr),
            "epot": self.lib.grid_grid_expectation_value(self.w.s.grid, self.vr.ptr),
        }


class GPStepper(_Base):
    def __init__(self, ref, psi0, v, step, mass, g, dt):
        super().__init__(ref, psi0, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT)
        self.g, self.dt = g, dt
        sh = self.shape
        self.vext = ref.rgrid(*sh, step, values=v)
        self.dens = ref.rgrid(*sh, step)
        self.pot = ref.cgrid(*sh, step)
        self.vc = ref.cgrid(*sh, step)
        self._owned += [self.vext, self.dens, self.pot, self.vc]
        self.lib.grid_real_to_complex_re(self.vc.ptr, self.vext.ptr)
        self.half = capi.Complex.of(0.5 * dt)

    def step_once(self):
        lib, w = self.lib, self.w
        lib.cgrid_fft(w.s.grid)
        lib.grid_wf_propagate_kinetic_fft(w.ptr, self.half)
        lib.cgrid_inverse_fft_norm(w.s.grid)
        lib.grid_wf_density(w.ptr, self.dens.ptr)
        lib.grid_real_to_complex_re(self.pot.ptr, self.dens.ptr)
        lib.cgrid_multiply(self.pot.ptr, capi.Complex.of(self.g))
        lib.cgrid_sum(self.pot.ptr, self.pot.ptr, self.vc.ptr)
        lib.grid_wf_propagate_potential(w.ptr, capi.Complex.of(self.dt), self.pot.ptr, 0.0)
        lib.cgrid_fft(w.s.grid)
        lib.grid_wf_propagate_kinetic_fft(w.ptr, self.half)
        lib.cgrid_inverse_fft_norm(w.s.grid)

    def observables(self, psi=None) -> dict:
        psi = self.psi() if psi is None else psi
        return {
            "norm": self.norm(),
            "ekin": self.lib.grid_wf_kinetic_energy_fft(self.w.ptr),
            "epot": self.lib.grid_grid_expectation_value(self.w.s.grid, self.vext.ptr),
            "eint": interaction_energy(psi, self.step, self.g),
        }


class CNGPStepper(_Base):
    def __init__(self, ref, psi0, v, step, mass, g, dt, bc=capi.WF_DIRICHLET_BOUNDARY):
        super().__init__(ref, psi0, step, mass, bc, capi.WF_2ND_ORDER_CN)
        self.g, self.dt = g, dt
        sh = self.shape
        self.vext = ref.rgrid(*sh, step, values=v)
        self.dens = ref.rgrid(*sh, step)
        self.pot = ref.cgrid(*sh, step)
        self.vc = ref.cgrid(*sh, step)
        self._owned += [self.vext, self.dens, self.pot, self.vc]
        self.lib.grid_real_to_complex_re(self.vc.ptr, self.vext.ptr)

    def _half_potential(self):
        lib = self.lib
        lib.grid_wf_density(self.w.ptr, self.dens.ptr)
        lib.grid_real_to_complex_re(self.pot.ptr, self.dens.ptr)
        lib.cgrid_multiply(self.pot.ptr, capi.Complex.of(self.g))
        lib.cgrid_sum(self.pot.ptr, self.pot.ptr, self.vc.ptr)
        lib.grid_wf_propagate_potential(self.w.ptr, capi.Complex.of(0.5 * self.dt), self.pot.ptr, 0.0)

    def step_once(self):
        self._half_potential()
        self.lib.grid_wf_propagate_kinetic_cn(self.w.ptr, capi.Complex.of(self.dt))
        self._half_potential()

    def observables(self, psi=None) -> dict:
        psi = self.psi() if psi is None else psi
        self.lib.grid_wf_analyze_method(b"\x00")
        return {
            "norm": self.norm(),
            "ekin": self.lib.grid_wf_kinetic_energy_cn(self.w.ptr),
            "epot": self.lib.grid_grid_expectation_value(self.w.s.grid, self.vext.ptr),
            "eint": interaction_energy(psi, self.step, self.g),
        }


def sample_indices(npts: int, count: int, seed: int = 12345) -> np.ndarray:
    """A fixed, sorted set of flat grid indices at which long trajectories
    store psi (the relative L2 distance over a uniform random subset
    estimates the full-grid one)."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(npts, size=min(count, npts), replace=False))
