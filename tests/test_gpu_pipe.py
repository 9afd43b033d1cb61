"""Pipelined (persistent, TMA-prefetching) strided FWD.K.INV passes against
the plain passes and the oracle: the same per-element arithmetic, so the results agree
to rounding of a different schedule (<= 1e-15 relative L2; FP32 <= 1e-7), and
the bounded-wait error flag stays clear."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel
from libgrid_b200 import capi, workloads

pytestmark = pytest.mark.gpu

PER, FFT2 = capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT


def _lib(b200):
    lib = b200.lib
    lib.gb_pass_pipeline.argtypes = [C.c_int]
    lib.gb_pass_pipeline.restype = C.c_int
    lib.gb_pass_error_flag.argtypes = [C.c_int]
    lib.gb_pass_error_flag.restype = C.c_int
    return lib


def _gp(b200, shape, prec, steps=3):
    step, g = 0.5, 0.0025
    mass = 4.0 / workloads.GRID_AUTOAMU
    psi0, v = workloads.gp_wells(shape, step, g, seed=31)
    w = b200.wf(*shape, step, mass, PER, FFT2, values=psi0)
    if prec:
        w.precision(prec)
    vx = b200.rgrid(*shape, step, values=v)
    for _ in range(steps):
        w.propagate_gp(vx, g, 1.0)
    out = w.grid.get()
    b200.free(w)
    b200.free(vx)
    return out, psi0, v


@pytest.mark.parametrize("shape", [(64, 64, 64), (128, 256, 32), (256, 64, 128), (16, 128, 256)])
@pytest.mark.parametrize("prec", [0, capi.GRID_PREC_FP32])
def test_pipelined_matches_plain(b200, shape, prec):
    lib = _lib(b200)
    old = lib.gb_pass_pipeline(0)
    try:
        plain, _, _ = _gp(b200, shape, prec)
        lib.gb_pass_pipeline(1)
        piped, _, _ = _gp(b200, shape, prec)
    finally:
        lib.gb_pass_pipeline(old)
    assert lib.gb_pass_error_flag(1) == 0
    assert rel(piped, plain) <= (1e-15 if not prec else 1e-7)


def test_pipelined_against_oracle(b200, restate):
    lib = _lib(b200)
    old = lib.gb_pass_pipeline(1)
    try:
        got, psi0, v = _gp(b200, (32, 64, 128), 0)
    finally:
        lib.gb_pass_pipeline(old)
    want = psi0.copy()
    vr = workloads.padded(v)
    for _ in range(3):
        want = restate.fft_step(want, 0.5, 4.0 / workloads.GRID_AUTOAMU, 1.0, vr=vr, g=0.0025)
    assert rel(got, want) < 1e-11
    assert lib.gb_pass_error_flag(1) == 0


def test_pipelined_fft3d(b200):
    lib = _lib(b200)
    rng = np.random.default_rng(4)
    shape = (128, 64, 256)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    old = lib.gb_pass_pipeline(1)
    try:
        gr = b200.cgrid(*shape, 1.0, values=x)
        lib.cgrid_fft(gr.ptr)
        got = gr.get()
        b200.free(gr)
    finally:
        lib.gb_pass_pipeline(old)
    assert rel(got, np.fft.fftn(x)) < 1e-14
