"""Parity on the full-size workloads, through the C ABI, against the
reference's own CPU build (oracle/_ref: libgrid's src/*.c compiled unchanged)
on the same seeded inputs (libgrid_b200.workloads).

  wavepacket 128^3   harmonic trap, Gaussian packet with kx = 0.5, 2nd-order
                     FFT, dt 0.05, 200 steps; psi, norm, kinetic (FFT
                     method) and potential energy every 50 steps, inline
  GP 256^3           Gross-Pitaevskii FFT split step (V_ext + g|psi|^2),
                     dt 1: 50 steps inline (full psi), 1000 steps against
                     the committed reference trajectory
                     (tests/golden/gp256_traj.npz: psi at a seeded subset of
                     points plus full-grid observables), in FP64 and in the
                     FP32 mode
  CN 192^3           Gross-Pitaevskii Crank-Nicolson with Dirichlet walls,
                     dt 0.5: 20 steps inline, 500 against
                     tests/golden/cn192_traj.npz

Tolerances (FP64): psi relative L2 <= 1e-11; total energy relative <= 1e-12
(components: kinetic, <V_ext>, interaction, each <= 1e-11 relative);
norm relative to the reference <= 1e-12 and its drift over the run <= 1e-12.
FP32 mode: the errors against the FP64 reference are asserted against the
stated bounds below, relative, at every checkpoint up to 1000 steps (measured
on a B200 after 1000 steps: psi 1.1e-4, energy 1.4e-4, norm 6.7e-5; the FP32
rounding of the FFTs accumulates as a random walk).
"""
import os

import numpy as np
import pytest

from conftest import ROOT, rel
from libgrid_b200 import capi, workloads
from oracle import refsteps

pytestmark = pytest.mark.gpu

PER, DIR = capi.WF_PERIODIC_BOUNDARY, capi.WF_DIRICHLET_BOUNDARY
FFT2, CN2 = capi.WF_2ND_ORDER_FFT, capi.WF_2ND_ORDER_CN
GOLDEN = os.path.join(ROOT, "tests", "golden")
MASS4 = 4.0 / workloads.GRID_AUTOAMU

TOL_PSI, TOL_E, TOL_E_PART, TOL_NORM = 1e-11, 1e-12, 1e-11, 1e-12
FP32_TOL = {"psi": 5e-4, "energy": 5e-4, "norm": 3e-4}


def relerr(a, b):
    return abs(a - b) / abs(b)


def gpu_observables(b200, w, vx, g, kinetic="fft"):
    lib = b200.lib
    psi = w.grid.get()
    ob = {
        "norm": w.norm(),
        "ekin": lib.grid_wf_kinetic_energy_fft(w.ptr) if kinetic == "fft" else lib.grid_wf_kinetic_energy_cn(w.ptr),
        "epot": lib.grid_grid_expectation_value(w.s.grid, vx.ptr),
    }
    if g:
        ob["eint"] = refsteps.interaction_energy(psi, w.s.grid.contents.step, g)
    return psi, ob


def total(ob):
    return ob["ekin"] + ob["epot"] + ob.get("eint", 0.0)


def check_observables(got, want, where):
    assert relerr(got["norm"], want["norm"]) <= TOL_NORM, (where, got["norm"], want["norm"])
    for k in ("ekin", "epot", "eint"):
        if k in want:
            assert relerr(got[k], want[k]) <= TOL_E_PART, (where, k, got[k], want[k])
    assert relerr(total(got), total(want)) <= TOL_E, (where, total(got), total(want))


# ------------------------------------------------------------ wavepacket 128^3


def test_wavepacket_128_vs_reference(b200, ref):
    n, step, mass, dt = 128, 0.2, 1.0, 0.05
    psi0, v = workloads.wavepacket(n, step)
    st = refsteps.WavepacketStepper(ref, psi0, v, step, mass, dt)
    w = b200.wf(n, n, n, step, mass, PER, FFT2, values=psi0)
    b200.lib.grid_wf_normalize(w.ptr)
    pot = b200.cgrid(n, n, n, step, values=v)
    vr = b200.rgrid(n, n, n, step, values=v.real)
    n0 = w.norm()
    try:
        for s in range(1, 201):
            w.propagate(pot, dt)
            st.step_once()
            if s % 50 == 0:
                psi, got = gpu_observables(b200, w, vr, 0.0)
                want = st.observables()
                assert rel(psi, st.psi()) < TOL_PSI, s
                check_observables(got, want, "step %d" % s)
        assert relerr(w.norm(), n0) <= TOL_NORM
    finally:
        st.free()
        for o in (w, pot, vr):
            b200.free(o)


# ------------------------------------------------------------------ GP 256^3


def _gp256(b200, prec=0):
    shape, step, g = (256, 256, 256), 0.5, 0.0025
    psi0, v = workloads.gp_wells(shape, step, g, seed=2)
    w = b200.wf(*shape, step, MASS4, PER, FFT2, values=psi0)
    if prec:
        w.precision(prec)
    vx = b200.rgrid(*shape, step, values=v)
    return psi0, v, w, vx, g


def test_gp256_50_steps_vs_reference(b200, ref):
    psi0, v, w, vx, g = _gp256(b200)
    st = refsteps.GPStepper(ref, psi0, v, 0.5, MASS4, g, 1.0)
    try:
        for _ in range(50):
            w.propagate_gp(vx, g, 1.0)
            st.step_once()
        psi, got = gpu_observables(b200, w, vx, g)
        want_psi = st.psi()
        assert rel(psi, want_psi) < TOL_PSI
        check_observables(got, st.observables(want_psi), "step 50")
    finally:
        st.free()
        b200.free(w)
        b200.free(vx)


def _traj(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.fail("missing fixture %s (python tests/golden/make_baseline_traj.py)" % path)
    return np.load(path)


def _fixture_obs(z, s):
    return {k: float(z["%s_%d" % (k, s)]) for k in ("norm", "ekin", "epot", "eint") if "%s_%d" % (k, s) in z}


def _run_against_traj(b200, z, w, vx, g, step_fn, kinetic):
    """Advance w to every checkpoint of the trajectory z; return per
    checkpoint (psi subset rel L2, observables, fixture observables) and the
    norm at step 0."""
    idx = z["idx"]
    _, ob0 = gpu_observables(b200, w, vx, g, kinetic)
    cps = sorted(int(k[4:]) for k in z.files if k.startswith("psi_") and k != "psi_0")
    out, done = {}, 0
    for s in cps:
        for _ in range(s - done):
            step_fn()
        done = s
        psi, ob = gpu_observables(b200, w, vx, g, kinetic)
        out[s] = (rel(psi.ravel()[idx], z["psi_%d" % s]), ob, _fixture_obs(z, s))
    return ob0, out


def test_gp256_1000_steps_vs_reference_trajectory(b200):
    z = _traj("gp256_traj.npz")
    psi0, v, w, vx, g = _gp256(b200)
    try:
        ob0, res = _run_against_traj(b200, z, w, vx, g, lambda: w.propagate_gp(vx, g, 1.0), "fft")
    finally:
        b200.free(w)
        b200.free(vx)
    check_observables(ob0, _fixture_obs(z, 0), "step 0")
    for s, (e_psi, got, want) in res.items():
        assert e_psi < TOL_PSI, (s, e_psi)
        check_observables(got, want, "step %d" % s)
    last = max(res)
    assert relerr(res[last][1]["norm"], ob0["norm"]) <= TOL_NORM  # drift over 1000 real-time steps


def test_gp256_fp32_mode_error_vs_reference_trajectory(b200):
    """The FP32 mode (FP32 storage and FFTs, FP64 phase reduction and FP64
    reductions) against the FP64 reference after 50, 500 and 1000 steps."""
    z = _traj("gp256_traj.npz")
    psi0, v, w, vx, g = _gp256(b200, capi.GRID_PREC_FP32)
    try:
        ob0, res = _run_against_traj(b200, z, w, vx, g, lambda: w.propagate_gp(vx, g, 1.0), "fft")
    finally:
        b200.free(w)
        b200.free(vx)
    for s, (e_psi, got, want) in res.items():
        assert e_psi < FP32_TOL["psi"], (s, e_psi)
        assert relerr(total(got), total(want)) < FP32_TOL["energy"], (s, total(got), total(want))
        assert relerr(got["norm"], want["norm"]) < FP32_TOL["norm"], (s, got["norm"], want["norm"])


# ---------------------------------------------------------------- CN 192^3


def _cn192(b200):
    shape, step, g = (192, 192, 192), 0.3, 0.001
    psi0, v = workloads.cn_wells(shape, step, g, seed=3)
    w = b200.wf(*shape, step, MASS4, DIR, CN2, values=psi0)
    vx = b200.rgrid(*shape, step, values=v)
    return psi0, v, w, vx, g


def test_cn192_20_steps_vs_reference(b200, ref):
    psi0, v, w, vx, g = _cn192(b200)
    st = refsteps.CNGPStepper(ref, psi0, v, 0.3, MASS4, g, 0.5)
    try:
        for _ in range(20):
            w.propagate_gp(vx, g, 0.5)
            st.step_once()
        psi, got = gpu_observables(b200, w, vx, g, kinetic="fd")
        want_psi = st.psi()
        assert rel(psi, want_psi) < TOL_PSI
        check_observables(got, st.observables(want_psi), "step 20")
    finally:
        st.free()
        b200.free(w)
        b200.free(vx)


def test_cn192_500_steps_vs_reference_trajectory(b200):
    z = _traj("cn192_traj.npz")
    psi0, v, w, vx, g = _cn192(b200)
    try:
        ob0, res = _run_against_traj(b200, z, w, vx, g, lambda: w.propagate_gp(vx, g, 0.5), "fd")
    finally:
        b200.free(w)
        b200.free(vx)
    check_observables(ob0, _fixture_obs(z, 0), "step 0")
    for s, (e_psi, got, want) in res.items():
        assert e_psi < TOL_PSI, (s, e_psi)
        check_observables(got, want, "step %d" % s)
