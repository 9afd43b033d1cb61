"""Seeded noise (grid_random_seed, rgrid_/cgrid_random_*): the reference's
CPU (drand48) and GPU (cuRAND) paths give different sequences, so parity is
in distribution: means and variances within 5 standard errors of the
reference's distributions, ranges, untouched rgrid padding, and exact
reproducibility for a given seed and call sequence."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (64, 48, 40)


def _zeros_r(b200):
    return b200.rgrid(*SHAPE, 0.1, values=np.zeros(SHAPE))


def _zeros_c(b200):
    return b200.cgrid(*SHAPE, 0.1, values=np.zeros(SHAPE, complex))


def _close(x, want, se):
    assert abs(x - want) < 5 * se, (x, want, se)


def test_rgrid_uniform_and_normal(b200):
    n = np.prod(SHAPE)
    b200.lib.grid_random_seed(64, 48, 40, 11)
    r = _zeros_r(b200)
    b200.lib.rgrid_random_uniform(r.ptr, 0.5)
    v = r.get()
    assert np.all(np.abs(v) <= 0.5)
    _close(v.mean(), 0.0, 0.5 / np.sqrt(3 * n))
    _close(v.var(), 0.25 / 3, 0.25 / 3 * np.sqrt(0.8 / n))
    # padding columns of the rgrid rows stay untouched
    pad = r._view()[:, :, SHAPE[2]:]
    assert np.all(pad == 0.0)
    b200.free(r)
    r = _zeros_r(b200)
    b200.lib.rgrid_random_normal(r.ptr, 2.0)
    v = r.get()
    _close(v.mean(), 0.0, 2.0 / np.sqrt(n))
    _close(v.var(), 4.0, 4.0 * np.sqrt(2.0 / n))
    b200.free(r)


def test_cgrid_kinds(b200):
    from libgrid_b200.capi import Complex

    n = np.prod(SHAPE)
    b200.lib.grid_random_seed(64, 48, 40, 12)
    c = _zeros_c(b200)
    b200.lib.cgrid_random_uniform(c.ptr, Complex.of(1.0 + 3.0j))
    z = c.get()
    assert np.all(np.abs(z.real) <= 1.0) and np.all(np.abs(z.imag) <= 3.0)
    _close(z.real.var(), 1.0 / 3, 1.0 / 3 * np.sqrt(0.8 / n))
    _close(z.imag.var(), 9.0 / 3, 9.0 / 3 * np.sqrt(0.8 / n))
    b200.free(c)
    c = _zeros_c(b200)
    b200.lib.cgrid_random_uniform_sp(c.ptr, 2.0)
    z = c.get()
    assert np.all(np.abs(z) <= 2.0 + 1e-12)
    _close(np.mean(np.abs(z) ** 2), 4.0 / 3, 4.0 * np.sqrt(4.0 / 45 / n))
    _close(z.real.mean(), 0.0, 2.0 / np.sqrt(6 * n))
    b200.free(c)
    c = _zeros_c(b200)
    b200.lib.cgrid_random_normal(c.ptr, Complex.of(0.5 + 2.0j))
    z = c.get()
    _close(z.real.var(), 0.25, 0.25 * np.sqrt(2.0 / n))
    _close(z.imag.var(), 4.0, 4.0 * np.sqrt(2.0 / n))
    _close(np.corrcoef(z.real.ravel(), z.imag.ravel())[0, 1], 0.0, 1.0 / np.sqrt(n))
    b200.free(c)
    c = _zeros_c(b200)
    b200.lib.cgrid_random_normal_sp(c.ptr, 1.5)
    z = c.get()
    _close(np.mean(np.abs(z) ** 2), 2.25, 2.25 * np.sqrt(2.0 / n))
    b200.free(c)


def test_seed_reproducibility(b200):
    outs = []
    for seed in (5, 5, 6):
        b200.lib.grid_random_seed(64, 48, 40, seed)
        r = _zeros_r(b200)
        b200.lib.rgrid_random_uniform(r.ptr, 1.0)
        b200.lib.rgrid_random_uniform(r.ptr, 1.0)  # second call: a new stream
        outs.append(r.get())
        b200.free(r)
    assert np.array_equal(outs[0], outs[1])
    assert not np.array_equal(outs[0], outs[2])
    # two calls are two independent streams: the sum has twice the variance
    n = np.prod(SHAPE)
    # (triangular distribution: excess kurtosis -0.6)
    _close(outs[0].var(), 2.0 / 3, 2.0 / 3 * np.sqrt(1.4 / n))
