"""Bounded device-side waits that give up are reported, not hidden.

Two waits in the propagation kernels only wait for other CTAs' progress:
the plane chain's dependency wait (a y-stage tile waits until every z-stage
tile of its x-plane has completed) and the batch kernel's grid barrier.
gb_wait_limit() shortens their poll limit so that the wait runs out on a
healthy GPU (no fault, no hang: the kernel gives up, sets its status word
and carries on or returns).  The tests check that
  * the library reports the failure at its next host sync point
    (gb_synchronize returns GB_ERR_DEVICE_WAIT and the status word is set),
  * the libgrid entry points then abort with a libgrid message instead of
    returning a wrong result (run in a child process), and
  * after gb_clear_error() and the default limit, the same call computes the
    oracle's values again (the context stays usable; the batch barrier's
    arrival counter starts clean in every launch).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, rel
from libgrid_b200 import capi, workloads

pytestmark = pytest.mark.gpu

ERR_DEVICE_WAIT = 1070
STATUS_PASS_CHAIN = 8  # code the chain's dependency wait writes


def _gp_case():
    shape, step, g = (4, 256, 256), 0.5, 0.0025
    mass = 4.0 / workloads.GRID_AUTOAMU
    psi0, v = workloads.gp_wells(shape, step, g, seed=19)
    return shape, step, g, mass, psi0, v


def test_chain_wait_gives_up_and_is_reported(b200, restate):
    lib = b200.lib
    lib.cuda_enable(b"\x01", 0, None)
    shape, step, g, mass, psi0, v = _gp_case()
    w = b200.wf(*shape, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT, values=psi0)
    vx = b200.rgrid(*shape, step, values=v)
    old_lag = lib.gb_chain_lag(0)  # second stages drawn right behind their first stage
    old_lim = lib.gb_wait_limit(2)
    try:
        w.propagate_gp(vx, g, 1.0)
        assert lib.gb_synchronize() == ERR_DEVICE_WAIT
        assert lib.gb_last_error() == ERR_DEVICE_WAIT
        assert b"device-side wait" in lib.gb_last_error_where()
        assert lib.gb_pass_error_flag(0) & STATUS_PASS_CHAIN
    finally:
        lib.gb_wait_limit(old_lim)
        lib.gb_chain_lag(old_lag)
        lib.gb_clear_error()
    assert lib.gb_last_error() == 0 and lib.gb_pass_error_flag(0) == 0
    # the same step with the default limit matches the oracle again
    w.grid.set(psi0)
    w.propagate_gp(vx, g, 1.0)
    got = w.grid.get()
    assert lib.gb_last_error() == 0
    want = restate.fft_step(psi0, step, mass, 1.0, vr=workloads.padded(v), g=g)
    assert rel(got, want) < 1e-11
    b200.free(w)
    b200.free(vx)


def test_chain_wait_failure_aborts_libgrid_call():
    """Through the libgrid API the failure aborts at the next result read
    (grid_wf_norm), with a libgrid message; the propagation call itself
    returned before the GPU finished."""
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import libgrid_b200 as gb\n"
        "from libgrid_b200 import capi, workloads\n"
        "api = gb.load(); lib = api.lib\n"
        "lib.cuda_enable(b'\\x01', 0, None)\n"
        "psi0, v = workloads.gp_wells((4, 256, 256), 0.5, 0.0025, seed=19)\n"
        "w = api.wf(4, 256, 256, 0.5, 4.0 / workloads.GRID_AUTOAMU, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT, values=psi0)\n"
        "vx = api.rgrid(4, 256, 256, 0.5, values=v)\n"
        "lib.gb_chain_lag(0); lib.gb_wait_limit(2)\n"
        "w.propagate_gp(vx, 0.0025, 1.0)\n"
        "print('propagate returned', flush=True)\n"
        "n = w.norm()\n"
        "print('norm returned', n, flush=True)\n"
    ) % (ROOT,)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert "propagate returned" in p.stdout
    assert "norm returned" not in p.stdout
    assert p.returncode != 0
    assert "libgrid" in p.stderr and "device-side wait" in p.stderr, p.stderr[-2000:]


def _batch_case():
    rng = np.random.default_rng(29)
    out = []
    for n in (64, 128, 64, 256, 128, 64):
        _, y, z = workloads.mesh(1, n, n, 0.2)
        r2 = y * y + z * z
        v = (0.5 * 0.01 * r2 + 0.002 * rng.standard_normal((1, n, n))).astype(complex)
        psi = np.exp(-r2 / 4.0 + 1j * rng.uniform(-1, 1) * y)
        out.append(((1, n, n), psi.astype(complex), v))
    return out


def test_batch_barrier_gives_up_then_recovers(b200, restate):
    lib = b200.lib
    lib.cuda_enable(b"\x01", 0, None)
    inst = _batch_case()
    step, mass, dt = 0.2, 1.0, 0.05
    wfs = [b200.wf(*sh, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT, values=p) for sh, p, _ in inst]
    pots = [b200.cgrid(*sh, step, values=v) for sh, _, v in inst]
    b = b200.batch(wfs, pots, dt)
    old_lim = lib.gb_wait_limit(2)
    try:
        b.propagate(3)  # fewer than 9 steps: the persistent launch with its grid barrier
        assert lib.gb_synchronize() == ERR_DEVICE_WAIT
        assert lib.gb_batch_error_flag(b.ptr, 0) != 0
    finally:
        lib.gb_wait_limit(old_lim)
        lib.gb_clear_error()
    assert lib.gb_batch_error_flag(b.ptr, 0) == 0
    # a normal call after the failed launch: the barrier starts clean
    for w, (_, p, _) in zip(wfs, inst):
        w.grid.set(p)
    b.propagate(3)
    assert lib.gb_synchronize() == 0
    for w, (sh, p, v) in zip(wfs, inst):
        want = p.copy()
        for _ in range(3):
            want = restate.fft_step(want, step, mass, dt, vc=v)
        assert rel(w.grid.get(), want) < 1e-11
    b200.free(b)
    for o in wfs + pots:
        b200.free(o)
