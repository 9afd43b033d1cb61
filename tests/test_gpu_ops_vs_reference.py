"""GPU grid operations, through the C ABI, against the reference's own CPU
build (oracle/_ref) on the same seeded inputs:

  * finite differences: cgrid_fd_laplace_{x,y,z}, cgrid_fd_gradient_{x,y,z}
    (src/cgrid_diff.c:201-442) and rgrid_fd_laplace (src/rgrid_diff.c:309),
    under all three boundary conditions;
  * k-space operators: cgrid_fft_laplace, cgrid_fft_gradient_{x,y,z},
    cgrid_fft_laplace_expectation_value (src/cgrid_diff.c:454-879);
  * pointwise products and sums (src/cgrid.c:934-1333, src/ngrid.c:53-254,
    src/rgrid.c:945-1003);
  * FFT convolution (src/cgrid.c:1912, src/rgrid.c:1848);
  * interpolation between grids (src/cgrid.c:2126, src/rgrid.c:2267) and the
    binary grid files with interpolating reads (src/cgrid.c:360-420,
    src/rgrid.c:339-400).

Pointwise and stencil results follow the reference's arithmetic order, so
they agree to rounding (<= 1e-14 relative L2; FFT-based ones <= 1e-13).

The reference's Neumann boundary value (src/cgrid_bc.c:39-57) mirrors an
index and looks the mirrored index up again; on an axis of length 1 the
mirror lands outside the grid again and the lookup never ends.  Those
combinations are compared with the restatement's definition instead (the
library takes the single plane there) and never run on the reference.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

BCS = ["dirichlet", "neumann", "periodic"]
_libc = C.CDLL(None)
_libc.fopen.restype = C.c_void_p
_libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
_libc.fclose.argtypes = [C.c_void_p]


def rand_c(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def both(b200, ref, fn):
    """fn(api) -> result, for the GPU library and the reference."""
    return fn(b200), fn(ref)


# ------------------------------------------------------- finite differences


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("shape", [(9, 10, 11), (16, 8, 32), (1, 24, 20)])
@pytest.mark.parametrize("op", ["fd_laplace_x", "fd_laplace_y", "fd_laplace_z", "fd_gradient_x", "fd_gradient_y",
                                "fd_gradient_z", "fd_laplace"])
def test_cgrid_fd_ops(b200, ref, restate, bc, shape, op):
    a = rand_c(np.random.default_rng(3), shape)
    if bc == "neumann" and 1 in shape:
        if op != "fd_laplace":
            pytest.skip("the reference's Neumann boundary does not terminate on an axis of length 1")
        g = b200.cgrid(*shape, 0.3, bc=bc, values=a)
        o = b200.cgrid(*shape, 0.3, bc=bc)
        b200.lib.cgrid_fd_laplace(g.ptr, o.ptr)
        assert rel(o.get(), restate.fd_laplace(a, 0.3, 1)) <= 1e-14
        b200.free(g)
        b200.free(o)
        return

    def run(api):
        g = api.cgrid(*shape, 0.3, bc=bc, values=a)
        o = api.cgrid(*shape, 0.3, bc=bc)
        getattr(api.lib, "cgrid_" + op)(g.ptr, o.ptr)
        r = o.get()
        api.free(g)
        api.free(o)
        return r

    got, want = both(b200, ref, run)
    assert rel(got, want) <= 1e-14


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("shape", [(9, 10, 11), (16, 8, 32)])
def test_rgrid_fd_laplace(b200, ref, bc, shape):
    a = np.random.default_rng(4).standard_normal(shape)

    def run(api):
        g = api.rgrid(*shape, 0.25, bc=bc, values=a)
        o = api.rgrid(*shape, 0.25, bc=bc)
        api.lib.rgrid_fd_laplace(g.ptr, o.ptr)
        r = o.get()
        api.free(g)
        api.free(o)
        return r

    got, want = both(b200, ref, run)
    assert rel(got, want) <= 1e-14


# ------------------------------------------------------ k-space operators


@pytest.mark.parametrize("shape", [(8, 16, 32), (1, 32, 64), (16, 16, 16)])
@pytest.mark.parametrize("op", ["fft_laplace", "fft_gradient_x", "fft_gradient_y", "fft_gradient_z"])
def test_cgrid_kspace_ops(b200, ref, shape, op):
    a = rand_c(np.random.default_rng(5), shape)

    def run(api):
        g = api.cgrid(*shape, 0.35, values=a)
        api.lib.cgrid_set_momentum(g.ptr, 0.2, -0.1, 0.3)
        o = api.cgrid(*shape, 0.35)
        api.lib.cgrid_fft(g.ptr)
        getattr(api.lib, "cgrid_" + op)(g.ptr, o.ptr)
        api.lib.cgrid_inverse_fft_norm(o.ptr)
        r = o.get()
        api.free(g)
        api.free(o)
        return r

    got, want = both(b200, ref, run)
    assert rel(got, want) <= 1e-13


@pytest.mark.parametrize("shape", [(8, 16, 32), (16, 16, 16)])
def test_cgrid_fft_laplace_expectation_value(b200, ref, shape):
    a = rand_c(np.random.default_rng(6), shape)

    def run(api):
        g = api.cgrid(*shape, 0.35, values=a)
        api.lib.cgrid_fft(g.ptr)
        v = api.lib.cgrid_fft_laplace_expectation_value(g.ptr)
        api.free(g)
        return v

    got, want = both(b200, ref, run)
    assert abs(got - want) <= 1e-12 * abs(want)


# ----------------------------------------------------------- pointwise ops


def test_cgrid_pointwise_ops(b200, ref):
    shape = (12, 10, 14)
    rng = np.random.default_rng(7)
    a, b, c0 = rand_c(rng, shape), rand_c(rng, shape), rand_c(rng, shape)
    d = 0.7 - 0.3j
    ops = [
        ("cgrid_sum", lambda L, c, x, y: L.cgrid_sum(c, x, y)),
        ("cgrid_difference", lambda L, c, x, y: L.cgrid_difference(c, x, y)),
        ("cgrid_product", lambda L, c, x, y: L.cgrid_product(c, x, y)),
        ("cgrid_conjugate_product", lambda L, c, x, y: L.cgrid_conjugate_product(c, x, y)),
        ("cgrid_add_scaled", lambda L, c, x, y: L.cgrid_add_scaled(c, _cx(d), x)),
        ("cgrid_add_scaled_product", lambda L, c, x, y: L.cgrid_add_scaled_product(c, _cx(d), x, y)),
        ("cgrid_multiply", lambda L, c, x, y: L.cgrid_multiply(c, _cx(d))),
        ("cgrid_add", lambda L, c, x, y: L.cgrid_add(c, _cx(d))),
    ]
    for name, fn in ops:

        def run(api):
            ga, gb, gc = (api.cgrid(*shape, 0.2, values=v) for v in (a, b, c0))
            fn(api.lib, gc.ptr, ga.ptr, gb.ptr)
            r = gc.get()
            for x in (ga, gb, gc):
                api.free(x)
            return r

        got, want = both(b200, ref, run)
        assert rel(got, want) <= 1e-15, name


def _cx(z):
    from libgrid_b200 import capi

    return capi.Complex.of(z)


def test_mixed_and_real_ops(b200, ref):
    shape = (8, 12, 10)
    rng = np.random.default_rng(8)
    psi = rand_c(rng, shape)
    r1, r2 = rng.standard_normal(shape), rng.standard_normal(shape)

    def run(api):
        c = api.cgrid(*shape, 0.3, values=psi)
        ra, rb = api.rgrid(*shape, 0.3, values=r1), api.rgrid(*shape, 0.3, values=r2)
        out = api.rgrid(*shape, 0.3)
        res = {}
        api.lib.grid_product_norm(out.ptr, ra.ptr, c.ptr)
        res["product_norm"] = out.get()
        api.lib.rgrid_product(out.ptr, ra.ptr, rb.ptr)
        res["rgrid_product"] = out.get()
        api.lib.rgrid_sum(out.ptr, ra.ptr, rb.ptr)
        res["rgrid_sum"] = out.get()
        res["integral"] = api.lib.rgrid_integral(ra.ptr)
        for x in (c, ra, rb, out):
            api.free(x)
        return res

    got, want = both(b200, ref, run)
    for k in ("product_norm", "rgrid_product", "rgrid_sum"):
        assert rel(got[k], want[k]) <= 1e-15, k
    assert abs(got["integral"] - want["integral"]) <= 1e-12 * abs(want["integral"])


# --------------------------------------------------------- FFT convolution


@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 32, 16), (1, 64, 32)])
def test_cgrid_fft_convolute(b200, ref, shape):
    rng = np.random.default_rng(9)
    a, b = rand_c(rng, shape), rand_c(rng, shape)

    def run(api):
        ga, gb, gc = api.cgrid(*shape, 0.4, values=a), api.cgrid(*shape, 0.4, values=b), api.cgrid(*shape, 0.4)
        api.lib.cgrid_fft(ga.ptr)
        api.lib.cgrid_fft(gb.ptr)
        api.lib.cgrid_fft_convolute(gc.ptr, ga.ptr, gb.ptr)
        api.lib.cgrid_inverse_fft_norm2(gc.ptr)
        r = gc.get()
        for x in (ga, gb, gc):
            api.free(x)
        return r

    got, want = both(b200, ref, run)
    assert rel(got, want) <= 1e-13
    # the convolution theorem with the origin at the grid centre
    n = np.array(shape)
    direct = np.fft.ifftn(np.fft.fftn(a) * np.fft.fftn(b))
    direct = np.roll(direct, tuple(n // 2), axis=(0, 1, 2)) * 0.4 ** sum(1 for m in shape if m > 1)
    assert rel(got, direct) <= 1e-12


@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 16, 32)])
def test_rgrid_fft_convolute(b200, ref, shape):
    rng = np.random.default_rng(10)
    a, b = rng.standard_normal(shape), rng.standard_normal(shape)

    def run(api):
        ga, gb, gc = api.rgrid(*shape, 0.4, values=a), api.rgrid(*shape, 0.4, values=b), api.rgrid(*shape, 0.4)
        api.lib.rgrid_fft(ga.ptr)
        api.lib.rgrid_fft(gb.ptr)
        api.lib.rgrid_fft_convolute(gc.ptr, ga.ptr, gb.ptr)
        api.lib.rgrid_inverse_fft_norm2(gc.ptr)
        r = gc.get()
        for x in (ga, gb, gc):
            api.free(x)
        return r

    got, want = both(b200, ref, run)
    assert rel(got, want) <= 1e-13


# ------------------------------------------------ interpolation and files


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("dst,src", [((20, 18, 22), (16, 16, 16)), ((12, 12, 12), (24, 20, 16)), ((1, 30, 30), (1, 16, 20))])
def test_cgrid_extrapolate(b200, ref, bc, dst, src):
    if bc == "neumann" and 1 in src:
        pytest.skip("the reference's Neumann boundary does not terminate on an axis of length 1")
    a = rand_c(np.random.default_rng(11), src)

    def run(api):
        s = api.cgrid(*src, 0.5, bc=bc, values=a)
        api.lib.cgrid_set_origin(s.ptr, 0.3, -0.2, 0.1)
        d = api.cgrid(*dst, 0.37, bc=bc)
        api.lib.cgrid_set_origin(d.ptr, -0.15, 0.05, 0.2)
        api.lib.cgrid_extrapolate(d.ptr, s.ptr)
        r = d.get()
        api.free(s)
        api.free(d)
        return r

    got, want = both(b200, ref, run)
    assert rel(got, want) <= 1e-15


@pytest.mark.parametrize("bc", BCS)
def test_rgrid_extrapolate(b200, ref, bc):
    src, dst = (12, 14, 16), (18, 16, 15)
    a = np.random.default_rng(12).standard_normal(src)

    def run(api):
        s = api.rgrid(*src, 0.5, bc=bc, values=a)
        d = api.rgrid(*dst, 0.41, bc=bc)
        api.lib.rgrid_extrapolate(d.ptr, s.ptr)
        r = d.get()
        api.free(s)
        api.free(d)
        return r

    got, want = both(b200, ref, run)
    assert rel(got, want) <= 1e-15


def _write(api, g, path, real):
    fp = _libc.fopen(path.encode(), b"wb")
    (api.lib.rgrid_write if real else api.lib.cgrid_write)(g.ptr, fp)
    _libc.fclose(fp)


def _read(api, g, path, real):
    fp = _libc.fopen(path.encode(), b"rb")
    r = (api.lib.rgrid_read if real else api.lib.cgrid_read)(g.ptr, fp)
    _libc.fclose(fp)
    assert r


@pytest.mark.parametrize("real", [False, True])
def test_grid_files_and_interpolating_read(b200, ref, tmp_path, real):
    """Files written by either library are byte-identical; reading a file of
    another size interpolates it onto the grid in memory as the reference
    does."""
    shape, other = (10, 12, 14), (16, 12, 10)
    rng = np.random.default_rng(13)
    a = rng.standard_normal(shape) if real else rand_c(rng, shape)
    mk = (lambda api, sh, st, v=None: api.rgrid(*sh, st, values=v)) if real else \
        (lambda api, sh, st, v=None: api.cgrid(*sh, st, values=v))
    files = {}
    for api in (b200, ref):
        g = mk(api, shape, 0.3, a)
        p = str(tmp_path / ("%s_%s.grd" % (api.kind, "r" if real else "c")))
        _write(api, g, p, real)
        files[api.kind] = p
        api.free(g)
    assert open(files["b200"], "rb").read() == open(files["ref"], "rb").read()
    out = {}
    for api in (b200, ref):
        same = mk(api, shape, 0.3)
        _read(api, same, files["ref"], real)
        diff = mk(api, other, 0.25)
        _read(api, diff, files["ref"], real)
        out[api.kind] = (same.get(), diff.get())
        api.free(same)
        api.free(diff)
    assert rel(out["b200"][0], a) == 0.0
    assert rel(out["b200"][1], out["ref"][1]) <= 1e-15
