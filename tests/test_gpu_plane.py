"""Plane-chained passes (the leading z FWD + y FWD and the trailing y INV +
z INV of a split step, each one persistent launch working plane by plane
with per-plane completion counters) against the nine-pass schedule and the
oracle.  Schedules 1 and 2 run the same per-line arithmetic in the same
order, so they agree to the last bit up to contraction differences (<= 1e-15
relative L2; FP32 <= 1e-7); schedule 3 applies the forward y and z
transforms after the potential in the other order (<= 1e-14)."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel
from libgrid_b200 import capi, workloads

pytestmark = pytest.mark.gpu

PER, FFT2 = capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT


def _lib(b200):
    lib = b200.lib
    lib.gb_plane_passes.argtypes = [C.c_int]
    lib.gb_plane_passes.restype = C.c_int
    return lib


def _run(b200, shape, prec, time, steps=3, multi=False, g=0.0025, kind="gp"):
    step = 0.5
    mass = 4.0 / workloads.GRID_AUTOAMU
    psi0, v = workloads.gp_wells(shape, step, g, seed=37)
    w = b200.wf(*shape, step, mass, PER, FFT2, values=psi0)
    if prec:
        w.precision(prec)
    if kind == "gp":
        pot = b200.rgrid(*shape, step, values=v)
        if multi:
            w.propagate_gp_n(pot, g, time, steps)
        else:
            for _ in range(steps):
                w.propagate_gp(pot, g, time)
    elif kind == "complex":
        rng = np.random.default_rng(5)
        vc = v + 0.01j * rng.standard_normal(shape)
        pot = b200.cgrid(*shape, step, values=vc)
        for _ in range(steps):
            w.propagate(pot, time)
        v = vc
    else:
        pot = None
        if multi:
            w.propagate_n(None, time, steps)
        else:
            for _ in range(steps):
                w.propagate(None, time)
    out = w.grid.get()
    b200.free(w)
    if pot is not None:
        b200.free(pot)
    return out, psi0, v


def _both(b200, *args, mode=1, **kw):
    lib = _lib(b200)
    old = lib.gb_plane_passes(0)
    try:
        nine, psi0, v = _run(b200, *args, **kw)
        lib.gb_plane_passes(mode)
        plane, _, _ = _run(b200, *args, **kw)
    finally:
        lib.gb_plane_passes(old)
    return plane, nine, psi0, v


MODES = [1, 2, 3]  # 2: y INV chained in front of the potential chain; 3: potential in the y stage


def tol64(mode):
    # schedule 3 applies the y and z forward transforms after the potential
    # in the other order: the same values up to rounding
    return 1e-15 if mode != 3 else 1e-14


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", [(2, 256, 256), (16, 256, 256)])
@pytest.mark.parametrize("time", [1.0, -1.0j])
@pytest.mark.parametrize("prec", [0, capi.GRID_PREC_FP32])
def test_plane_matches_nine_pass(b200, shape, time, prec, mode):
    plane, nine, _, _ = _both(b200, shape, prec, time, mode=mode)
    assert rel(plane, nine) <= (tol64(mode) if not prec else 1e-7)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("kind", ["free", "complex"])
def test_plane_other_programs(b200, kind, mode):
    plane, nine, _, _ = _both(b200, (4, 256, 256), 0, 1.0, kind=kind, mode=mode)
    assert rel(plane, nine) <= tol64(mode)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("kind", ["gp", "free"])
@pytest.mark.parametrize("prec", [0, capi.GRID_PREC_FP32])
def test_plane_multistep(b200, kind, prec, mode):
    plane, nine, _, _ = _both(b200, (8, 256, 256), prec, 1.0, steps=7, multi=True, kind=kind, mode=mode)
    assert rel(plane, nine) <= (tol64(mode) if not prec else 1e-7)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("prec", [0, capi.GRID_PREC_FP32])
def test_plane_chains_full_size(b200, prec, mode):
    """The 256^3 workload: 256 planes per chain, two steps and a multi-step
    call, bit for bit against the nine-pass schedule."""
    plane, nine, _, _ = _both(b200, (256, 256, 256), prec, 1.0, steps=2, mode=mode)
    assert rel(plane, nine) <= (tol64(mode) if not prec else 1e-7)
    plane, nine, _, _ = _both(b200, (256, 256, 256), prec, -1.0j, steps=4, multi=True, mode=mode)
    assert rel(plane, nine) <= (tol64(mode) if not prec else 1e-7)


def test_plane_against_oracle(b200, restate):
    lib = _lib(b200)
    old = lib.gb_plane_passes(1)
    try:
        got, psi0, v = _run(b200, (4, 256, 256), 0, 1.0, steps=2)
    finally:
        lib.gb_plane_passes(old)
    want = psi0.copy()
    vr = workloads.padded(v)
    for _ in range(2):
        want = restate.fft_step(want, 0.5, 4.0 / workloads.GRID_AUTOAMU, 1.0, vr=vr, g=0.0025)
    assert rel(got, want) < 1e-11


@pytest.mark.parametrize("mode", MODES)
def test_plane_timing_kinds(b200, mode):
    """A chained FP64 step runs six launches: the three chains (kinds 18, 19
    and 20), the x FWD.K.INV pass twice and the y INV pass; with the y INV
    pass chained in front of the potential chain (kind 21) five launches;
    the pass error flag stays clear."""
    lib = _lib(b200)
    lib.gb_pass_timing.argtypes = [C.c_int]
    lib.gb_pass_timing_report.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_long), C.c_int]
    lib.gb_pass_error_flag.argtypes = [C.c_int]
    lib.gb_pass_error_flag.restype = C.c_int
    old = lib.gb_plane_passes(mode)
    try:
        lib.gb_pass_timing(1)
        _run(b200, (4, 256, 256), 0, 1.0, steps=1)
        ms = (C.c_double * 23)()
        cnt = (C.c_long * 23)()
        lib.gb_pass_timing_report(ms, cnt, 23)
        lib.gb_pass_timing(0)
    finally:
        lib.gb_plane_passes(old)
    counts = list(cnt)
    assert counts[18] == 1 and counts[20] == 1
    assert counts[2] == 2  # x FWD.K.INV
    if mode == 1:
        assert counts[19] == 1 and counts[6] == 1  # y INV
        assert sum(counts) == 6
    elif mode == 2:
        assert counts[21] == 1
        assert sum(counts) == 5
    else:
        assert counts[22] == 1 and counts[6] == 1
        assert sum(counts) == 6
    assert lib.gb_pass_error_flag(1) == 0
