"""Multi-step calls (grid_wf_propagate_n / grid_wf_propagate_gp_n): the
k-space state is kept between steps (4 passes per step instead of 9), which
changes only the rounding: against nsteps single-step calls the result agrees
to 1e-12 relative L2, and against the oracle to the parity tolerance."""
import numpy as np
import pytest

from conftest import rel
from libgrid_b200 import capi, workloads

pytestmark = pytest.mark.gpu

PER, DIR = capi.WF_PERIODIC_BOUNDARY, capi.WF_DIRICHLET_BOUNDARY
FFT2, CFFT2, CN2 = capi.WF_2ND_ORDER_FFT, capi.WF_2ND_ORDER_CFFT, capi.WF_2ND_ORDER_CN


def _gp(b200, shape, time, n, multi, prec=0, seed=21):
    step, g = 0.5, 0.0025
    mass = 4.0 / workloads.GRID_AUTOAMU
    psi0, v = workloads.gp_wells(shape, step, g, seed=seed)
    w = b200.wf(*shape, step, mass, PER, FFT2, values=psi0)
    if prec:
        w.precision(prec)
    vx = b200.rgrid(*shape, step, values=v)
    if multi:
        w.propagate_gp_n(vx, g, time, n)
    else:
        for _ in range(n):
            w.propagate_gp(vx, g, time)
    out = w.grid.get()
    b200.free(w)
    b200.free(vx)
    return out, psi0, v


@pytest.mark.parametrize("shape", [(32, 64, 128), (1, 64, 128), (64, 64, 64)])
@pytest.mark.parametrize("time", [1.0, -1.0j])
def test_gp_n_matches_single_steps(b200, shape, time):
    got, _, _ = _gp(b200, shape, time, 10, True)
    want, _, _ = _gp(b200, shape, time, 10, False)
    assert rel(got, want) < 1e-12


def test_gp_n_against_oracle(b200, restate):
    shape, step, g = (32, 32, 64), 0.5, 0.0025
    mass = 4.0 / workloads.GRID_AUTOAMU
    got, psi0, v = _gp(b200, shape, 1.0, 12, True)
    want = psi0.copy()
    vr = workloads.padded(v)
    for _ in range(12):
        want = restate.fft_step(want, step, mass, 1.0, vr=vr, g=g)
    assert rel(got, want) < 1e-11


def test_gp_n_fp32(b200):
    got, _, _ = _gp(b200, (32, 64, 128), 1.0, 10, True, prec=capi.GRID_PREC_FP32)
    want, _, _ = _gp(b200, (32, 64, 128), 1.0, 10, False, prec=capi.GRID_PREC_FP32)
    assert rel(got, want) < 1e-5


def test_propagate_n_cfft_complex_potential(b200, restate):
    shape, step, mass, kmax = (16, 32, 64), 0.3, 1.0, 5.0
    rng = np.random.default_rng(8)
    psi0 = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    v = 0.1 * rng.standard_normal(shape) + 0.01j * rng.standard_normal(shape)
    outs = []
    for multi in (True, False):
        w = b200.wf(*shape, step, mass, PER, CFFT2, values=psi0)
        w.s.kmax = kmax
        b200.lib.cgrid_set_momentum(w.s.grid, 0.2, -0.1, 0.05)
        pot = b200.cgrid(*shape, step, values=v)
        if multi:
            w.propagate_n(pot, 0.05, 7)
        else:
            for _ in range(7):
                w.propagate(pot, 0.05)
        outs.append(w.grid.get())
        b200.free(w)
        b200.free(pot)
    assert rel(outs[0], outs[1]) < 1e-12
    want = psi0.copy()
    for _ in range(7):
        want = restate.fft_step(want, step, mass, 0.05, k0=(0.2, -0.1, 0.05), vc=v, cutoff=1, kmax=kmax)
    assert rel(outs[0], want) < 1e-11


def test_propagate_n_single_step_and_cn_fallback(b200):
    """nsteps == 1 is the ordinary step exactly; a CN wave function makes
    ordinary steps."""
    a, _, _ = _gp(b200, (16, 32, 32), 1.0, 1, True)
    b, _, _ = _gp(b200, (16, 32, 32), 1.0, 1, False)
    assert np.array_equal(a, b)
    shape, step, g = (12, 16, 20), 0.3, 0.001
    psi0, v = workloads.cn_wells(shape, step, g)
    outs = []
    for multi in (True, False):
        w = b200.wf(*shape, step, 4.0 / workloads.GRID_AUTOAMU, DIR, CN2, values=psi0)
        vx = b200.rgrid(*shape, step, values=v)
        if multi:
            w.propagate_gp_n(vx, g, 0.5, 3)
        else:
            for _ in range(3):
                w.propagate_gp(vx, g, 0.5)
        outs.append(w.grid.get())
        b200.free(w)
        b200.free(vx)
    assert np.array_equal(outs[0], outs[1])
