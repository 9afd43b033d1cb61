"""gb_reduce_noalloc: the reduction entry point that allocates no device memory.

It is meant for callers that cannot let a library allocate on the device: an
application that hands out every byte of device memory from its own pool or
budget, or a latency-critical loop where a cudaMalloc, or the device-wide
synchronisation of cudaFree, is not acceptable.  It must compute the same
sums as gb_reduce up to rounding (it adds the terms in a different order, so
the two agree to about 1e-12 relative, not bit for bit; each is deterministic
from call to call).  This test calls both through the C ABI on the same
device data, two calls in a row, for every reduction op and for mixed-
precision operands, with the relative tolerance the other reduction tests
use, and checks that oversized grids and unknown ops are refused before any
launch.
"""
import ctypes as C

import numpy as np
import pytest

from libgrid_b200 import capi

pytestmark = pytest.mark.gpu

RED_SUM, RED_NORM2, RED_CONJ_PRODUCT, RED_EXPECT_COMPLEX, RED_EXPECT_REAL, RED_REAL_SUM, RED_KSQ_NORM2 = 1, 2, 3, 4, 5, 6, 7
TOL = 1e-12


class Geom(C.Structure):
    _fields_ = [("nx", C.c_long), ("ny", C.c_long), ("nz", C.c_long), ("step", C.c_double), ("prec", C.c_int)]


def _bind(lib):
    V, L, I = C.c_void_p, C.c_long, C.c_int
    for name in ("gb_reduce", "gb_reduce_noalloc"):
        fn = getattr(lib, name)
        fn.restype = I
        fn.argtypes = [I, V, V, C.POINTER(Geom), L, L, I, C.POINTER(C.c_double)]
    lib.gb_device_alloc.restype = V
    lib.gb_device_alloc.argtypes = [C.c_size_t]
    lib.gb_device_free.argtypes = [V]
    lib.gb_h2d.restype = I
    lib.gb_h2d.argtypes = [V, V, C.c_size_t]
    lib.gb_clear_error.restype = None
    lib.gb_last_error.restype = I


def _to_device(lib, arr):
    arr = np.ascontiguousarray(arr)
    p = lib.gb_device_alloc(arr.nbytes)
    assert p
    assert lib.gb_h2d(p, arr.ctypes.data, arr.nbytes) == 0
    assert lib.gb_synchronize() == 0
    return p


def _call(fn, op, a, b, geom, arow, brow, bprec):
    out = (C.c_double * 2)()
    rc = fn(op, a, b, C.byref(geom), arow, brow, bprec, out)
    assert rc == 0
    return complex(out[0], out[1])


def test_noalloc_matches_gb_reduce(b200):
    lib = b200.lib
    _bind(lib)
    lib.cuda_enable(b"\x01", 0, None)
    rng = np.random.default_rng(123)
    nx, ny, nz = 48, 40, 36
    nz2 = 2 * (nz // 2 + 1)
    a = rng.standard_normal((nx, ny, nz)) + 1j * rng.standard_normal((nx, ny, nz))
    b = rng.standard_normal((nx, ny, nz)) + 1j * rng.standard_normal((nx, ny, nz))
    r = np.zeros((nx, ny, nz2))
    r[:, :, :nz] = rng.standard_normal((nx, ny, nz))
    a32 = a.astype(np.complex64)
    b32 = b.astype(np.complex64)
    r32 = r.astype(np.float32)
    da, db, dr, da32, db32, dr32 = (_to_device(lib, x) for x in (a, b, r, a32, b32, r32))
    g64 = Geom(nx, ny, nz, 0.3, capi.GRID_PREC_FP64)
    g32 = Geom(nx, ny, nz, 0.3, capi.GRID_PREC_FP32)
    cases = [
        (RED_SUM, da, None, g64, nz, 0, 0),
        (RED_NORM2, da, None, g64, nz, 0, 0),
        (RED_CONJ_PRODUCT, da, db, g64, nz, nz, 0),
        (RED_EXPECT_COMPLEX, da, db, g64, nz, nz, 0),
        (RED_EXPECT_REAL, da, dr, g64, nz, nz2, 0),
        (RED_REAL_SUM, dr, None, g64, nz2, 0, 0),
        (RED_KSQ_NORM2, da, None, g64, nz, 0, 0),
        (RED_NORM2, da32, None, g32, nz, 0, 0),
        # mixed precision: FP64 a with an FP32 second operand, and the reverse
        (RED_CONJ_PRODUCT, da, db32, g64, nz, nz, capi.GRID_PREC_FP32),
        (RED_EXPECT_REAL, da, dr32, g64, nz, nz2, capi.GRID_PREC_FP32),
        (RED_EXPECT_COMPLEX, da32, db, g32, nz, nz, capi.GRID_PREC_FP64),
    ]
    try:
        for op, x, y, geom, arow, brow, bprec in cases:
            want = _call(lib.gb_reduce, op, x, y, geom, arow, brow, bprec)
            for _ in range(2):  # two calls in a row share the static scratch
                got = _call(lib.gb_reduce_noalloc, op, x, y, geom, arow, brow, bprec)
                assert abs(got - want) <= TOL * max(abs(want), 1e-300), (op, got, want)
        # numpy cross-check of one of them
        n2 = _call(lib.gb_reduce_noalloc, RED_NORM2, da, None, g64, nz, 0, 0).real
        assert abs(n2 - np.sum(np.abs(a) ** 2)) <= TOL * n2
    finally:
        for p in (da, db, dr, da32, db32, dr32):
            lib.gb_device_free(p)


def test_noalloc_rejects_grids_above_its_limit(b200):
    lib = b200.lib
    _bind(lib)
    lib.cuda_enable(b"\x01", 0, None)
    out = (C.c_double * 2)()
    big = Geom(257, 256, 256, 0.5, capi.GRID_PREC_FP64)  # one plane past 16,777,216 points
    rc = lib.gb_reduce_noalloc(RED_NORM2, None, None, C.byref(big), 256, 0, 0, out)
    assert rc != 0
    assert lib.gb_last_error() != 0
    lib.gb_clear_error()
    assert lib.gb_last_error() == 0


def test_noalloc_rejects_unknown_op(b200):
    lib = b200.lib
    _bind(lib)
    lib.cuda_enable(b"\x01", 0, None)
    out = (C.c_double * 2)()
    g = Geom(8, 8, 8, 0.5, capi.GRID_PREC_FP64)
    for fn in (lib.gb_reduce_noalloc, lib.gb_reduce):
        for op in (0, 8, -1):
            assert fn(op, None, None, C.byref(g), 8, 0, 0, out) != 0
            assert lib.gb_last_error() != 0
            lib.gb_clear_error()
