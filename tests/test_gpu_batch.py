"""Batched 2-D propagation (grid_wf_batch_*): one persistent launch advances
many wave functions of uneven sizes.  Each instance must come out as
grid_wf_propagate leaves it (same per-line arithmetic: relative L2 <= 1e-15,
in practice bit-identical), and agree with the oracle's FFT step to 1e-11."""
import numpy as np
import pytest

from conftest import rel
from libgrid_b200 import capi, workloads

pytestmark = pytest.mark.gpu

PER, FFT2 = capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT
SHAPES = [(1, 64, 64), (1, 128, 64), (1, 64, 256), (1, 256, 256), (1, 512, 64), (1, 128, 128), (1, 64, 512)]


def _instances(shapes, seed):
    rng = np.random.default_rng(seed)
    out = []
    for sh in shapes:
        _, y, z = workloads.mesh(*sh, 0.2)
        psi = np.exp(-(y * y + z * z) / 4.0 + 1j * (rng.uniform(-1, 1) * y + rng.uniform(-1, 1) * z))
        v = 0.01 * (y * y + z * z) + 0.002 * rng.standard_normal(sh) + 1e-4j * rng.standard_normal(sh)
        out.append((sh, psi, v))
    return out


def _run(b200, inst, time, steps, batched, prec=0, skip_pot=()):
    step, mass = 0.2, 1.3
    wfs, pots = [], []
    for i, (sh, psi, v) in enumerate(inst):
        w = b200.wf(*sh, step, mass, PER, FFT2, values=psi)
        if prec:
            w.precision(prec)
        wfs.append(w)
        pots.append(None if i in skip_pot else b200.cgrid(*sh, step, values=v))
    if batched:
        b = b200.batch(wfs, pots, time)
        b.propagate(steps)
        threads = b200.lib.grid_wf_batch_threads(b.ptr)
        b200.free(b)
    else:
        threads = 0
        for w, p in zip(wfs, pots):
            for _ in range(steps):
                w.propagate(p, time)
    out = [w.grid.get() for w in wfs]
    for w in wfs:
        b200.free(w)
    for p in pots:
        if p is not None:
            b200.free(p)
    return out, threads


@pytest.mark.parametrize("time", [0.05, -0.05j])
def test_batch_matches_single(b200, time):
    inst = _instances(SHAPES, 3)
    got, threads = _run(b200, inst, time, 11, True, skip_pot=(2,))
    want, _ = _run(b200, inst, time, 11, False, skip_pot=(2,))
    assert threads in (128, 256, 512, -1)
    for g, w in zip(got, want):
        assert rel(g, w) <= 1e-15


def test_batch_fp32_matches_single(b200):
    inst = _instances(SHAPES[:4], 5)
    got, _ = _run(b200, inst, 0.05, 10, True, prec=capi.GRID_PREC_FP32)
    want, _ = _run(b200, inst, 0.05, 10, False, prec=capi.GRID_PREC_FP32)
    for g, w in zip(got, want):
        assert rel(g, w) <= 1e-7


def test_batch_short_call_and_repeat(b200):
    """Calls of fewer than nine steps (no tuning) and repeated calls."""
    inst = _instances(SHAPES[:3], 9)
    step, mass = 0.2, 1.3
    wfs = [b200.wf(*sh, step, mass, PER, FFT2, values=psi) for sh, psi, _ in inst]
    pots = [b200.cgrid(*sh, step, values=v) for sh, _, v in inst]
    b = b200.batch(wfs, pots, 0.05)
    b.propagate(2)
    b.propagate(3)
    b.propagate(10)
    got = [w.grid.get() for w in wfs]
    b200.free(b)
    want, _ = _run(b200, inst, 0.05, 15, False)
    for g, w in zip(got, want):
        assert rel(g, w) <= 1e-15
    for o in wfs + pots:
        b200.free(o)


@pytest.mark.parametrize("steps", [5, 12])  # 12: the autotuned plan runs after the tuning steps
def test_batch_against_oracle(b200, restate, steps):
    """Every line length (64 to 512, the 512-point lines as radix 16.16.2),
    mixed shapes and a time step with an imaginary part, against the FP64
    oracle."""
    inst = _instances([(1, 64, 128), (1, 128, 256), (1, 512, 512), (1, 512, 64), (1, 64, 512), (1, 256, 256)], 11)
    time = 0.05 - 0.01j
    got, _ = _run(b200, inst, time, steps, True)
    for (sh, psi, v), g in zip(inst, got):
        want = psi.copy()
        for _ in range(steps):
            want = restate.fft_step(want, 0.2, 1.3, time, vc=v)
        assert rel(g, want) < 1e-11, sh


def test_batch_fp32_against_oracle(b200, restate):
    """The FP32 batch (FP32 storage and FFTs, FP64 phase reduction) against
    the FP64 oracle, within the FP32 mode's stated bound after 10 steps."""
    inst = _instances([(1, 64, 64), (1, 128, 512), (1, 512, 512), (1, 256, 128)], 13)
    got, _ = _run(b200, inst, 0.05, 10, True, prec=capi.GRID_PREC_FP32)
    for (sh, psi, v), g in zip(inst, got):
        want = psi.copy()
        for _ in range(10):
            want = restate.fft_step(want, 0.2, 1.3, 0.05, vc=v)
        assert rel(g, want) < 2e-5, sh


def test_batch_rejects_unsupported(b200):
    import subprocess
    import sys

    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import libgrid_b200 as gb\n"
        "from libgrid_b200 import capi\n"
        "api = gb.load()\n"
        "w = api.wf(2, 64, 64, 0.2, 1.0, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT)\n"
        "api.batch([w], [None], 0.1)\n"
        "print('returned')\n"
    ) % (__import__("conftest").ROOT,)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert p.returncode != 0 and "returned" not in p.stdout
    assert "2-D" in p.stderr
