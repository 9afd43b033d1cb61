"""CPU checks of the oracle itself (no GPU).

The restatement (oracle/gbo_path.c) is pinned three ways:
  * its FFT against numpy's (independent pocketfft) on mixed-radix shapes,
  * against golden fixtures written by the reference's own compiled sources
    (tests/golden/make_golden.py),
  * directly against the compiled reference (oracle/_ref) where present.
"""
import os

import numpy as np
import pytest

from conftest import rel
from libgrid_b200 import capi, workloads

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("shape", [(1, 1, 8), (4, 6, 10), (3, 5, 7), (16, 16, 16), (1, 12, 96), (2, 3, 49), (8, 192, 5)])
def test_fft_vs_numpy(restate, shape):
    rng = np.random.default_rng(sum(shape))
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    assert rel(restate.fft3d(a, -1), np.fft.fftn(a)) < 1e-14
    assert rel(restate.fft3d(a, +1), np.fft.ifftn(a) * a.size) < 1e-14


def test_fft_known_answers(restate):
    # plane wave -> single spike; Gaussian -> Gaussian (Parseval)
    n = 32
    k = np.arange(n)
    pw = np.exp(2j * np.pi * 5 * k / n).reshape(1, 1, n)
    f = restate.fft3d(pw, -1)
    spike = np.zeros_like(f)
    spike[0, 0, 5] = n
    assert np.max(np.abs(f - spike)) < 1e-12
    rng = np.random.default_rng(1)
    a = rng.standard_normal((8, 8, 8)) + 0j
    f = restate.fft3d(a, -1)
    assert abs(np.sum(np.abs(f) ** 2) / a.size - np.sum(np.abs(a) ** 2)) < 1e-10


def _load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def test_golden_wavepacket(restate):
    z = _load("wavepacket16")
    n, step, mass, dt = int(z["meta_n"]), float(z["meta_step"]), float(z["meta_mass"]), float(z["meta_dt"])
    psi0, v = workloads.wavepacket(n, step)
    psi = z["psi_start"]
    # the fixture starts from the reference-normalized packet
    assert rel(psi, psi0 * np.sqrt(1.0 / restate.norm(psi0, step))) < 1e-14
    for s in range(1, 21):
        psi = restate.fft_step(psi, step, mass, dt, vc=v)
        if s % 10 == 0:
            assert rel(psi, z["psi_%d" % s]) < 1e-14
            assert abs(restate.norm(psi, step) - float(z["norm_%d" % s])) < 1e-14
            assert abs(restate.kinetic_energy_fft(psi, step, mass) - float(z["ekin_fft_%d" % s])) < 1e-13
            assert abs(restate.potential_energy(psi, workloads.padded(v.real), step) - float(z["epot_%d" % s])) < 1e-13
    assert abs(restate.kinetic_energy_fd(psi, step, mass, 2) - float(z["ekin_fd_20"])) < 1e-13


def test_golden_gp(restate):
    z = _load("gp16")
    shape = tuple(int(q) for q in z["meta_shape"])
    step, g, dt, seed, mass = (float(z["meta_" + k]) for k in ("step", "g", "dt", "seed", "mass"))
    psi, v = workloads.gp_wells(shape, step, g, int(seed))
    for _ in range(5):
        psi = restate.fft_step(psi, step, mass, dt, vr=workloads.padded(v), g=g)
    assert rel(psi, z["psi_5"]) < 1e-14
    assert abs(restate.norm(psi, step) - float(z["norm_5"])) <= 1e-14 * float(z["norm_5"])


def test_golden_cn_dirichlet(restate):
    z = _load("cn_dirichlet")
    shape = tuple(int(q) for q in z["meta_shape"])
    step, g, dt, seed, mass = (float(z["meta_" + k]) for k in ("step", "g", "dt", "seed", "mass"))
    psi, v = workloads.cn_wells(shape, step, g, int(seed))
    for _ in range(5):
        psi = restate.cn_step(psi, step, mass, dt, capi.WF_DIRICHLET_BOUNDARY, vr=workloads.padded(v), g=g)
    assert rel(psi, z["psi_5"]) < 1e-14
    assert abs(restate.kinetic_energy_fd(psi, step, mass, 0) - float(z["ekin_fd_5"])) <= 1e-13 * abs(float(z["ekin_fd_5"]))


# ------------------------------------------- restatement vs compiled reference


@pytest.mark.parametrize("shape", [(8, 8, 8), (1, 16, 32), (4, 6, 10)])
@pytest.mark.parametrize("time", [0.05, -0.1j, 0.03 - 0.01j])
def test_restatement_fft_step_vs_reference(restate, ref, shape, time):
    rng = np.random.default_rng(5)
    step, mass = 0.3, 1.3
    psi0 = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    v = 0.1 * rng.standard_normal(shape) + 0.01j * rng.standard_normal(shape)
    w = ref.wf(*shape, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT, values=psi0)
    ref.lib.cgrid_set_momentum(w.s.grid, 0.1, 0.0, -0.2)
    pot = ref.cgrid(*shape, step, values=v)
    b = psi0.copy()
    for _ in range(3):
        w.propagate(pot, time)
        b = restate.fft_step(b, step, mass, time, k0=(0.1, 0.0, -0.2), vc=v)
    assert rel(b, w.grid.get()) < 1e-15


@pytest.mark.parametrize("bc", [1, 2, 3])
@pytest.mark.parametrize("extras", ["plain", "rotation", "absorber"])
def test_restatement_cn_vs_reference(restate, ref, bc, extras):
    rng = np.random.default_rng(6)
    shape, step, mass = (9, 8, 10), 0.3, 1.1
    psi0 = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    v = 0.1 * rng.standard_normal(shape) + 0.01j * rng.standard_normal(shape)
    w = ref.wf(*shape, step, mass, bc, capi.WF_2ND_ORDER_CN, values=psi0)
    ws3 = ref.cgrid(*shape, step)
    w.s.cworkspace3 = ws3.ptr
    ref.lib.cgrid_set_momentum(w.s.grid, 0.1, -0.3, 0.2)
    omega, lh = 0.0, None
    if extras == "rotation":
        omega = 0.4
        ref.lib.cgrid_set_rotation(w.s.grid, omega)
    if extras == "absorber":
        lh = (2, 6, 2, 5, 3, 6)
        ref.lib.grid_wf_boundary(w.ptr, None, *lh)
    pot = ref.cgrid(*shape, step, values=v)
    b = psi0.copy()
    for _ in range(2):
        w.propagate(pot, 0.07)
        b = restate.cn_step(b, step, mass, 0.07, bc, k0=(0.1, -0.3, 0.2), omega=omega, vc=v, absorb=lh)
    assert rel(b, w.grid.get()) < 1e-15


def test_restatement_energies_vs_reference(restate, ref):
    rng = np.random.default_rng(8)
    shape, step, mass = (8, 10, 12), 0.4, 1.7
    psi = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    v = rng.standard_normal(shape)
    for bc, obc in ((1, 0), (2, 1), (3, 2)):
        prop = capi.WF_2ND_ORDER_CN if bc != 3 else capi.WF_2ND_ORDER_FFT
        w = ref.wf(*shape, step, mass, bc, prop, values=psi)
        vr = ref.rgrid(*shape, step, values=v)
        ref.lib.grid_wf_analyze_method(b"\x00")
        assert abs(ref.lib.grid_wf_kinetic_energy_cn(w.ptr) - restate.kinetic_energy_fd(psi, step, mass, obc)) < 1e-10
        assert abs(ref.lib.grid_wf_potential_energy(w.ptr, vr.ptr) - restate.potential_energy(psi, workloads.padded(v), step)) < 1e-10
        assert abs(ref.lib.grid_wf_norm(w.ptr) - restate.norm(psi, step)) < 1e-10
        if bc == 3:
            assert abs(ref.lib.grid_wf_kinetic_energy_fft(w.ptr) - restate.kinetic_energy_fft(psi, step, mass)) < 1e-10
