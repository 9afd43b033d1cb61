"""libgrid_b200: a B200 (sm_100a) implementation of libgrid's wavefunction
propagation path behind libgrid's own C API.

The product is the C library ``libgrid_b200.so`` (headers in ``include/``).
This module loads it through ctypes and adds thin numpy conveniences used by
the tests, the benchmark and Python callers.  Everything computes on the GPU;
if the shared library is missing, loading fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import capi
from .capi import Complex  # noqa: F401  (re-exported)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgrid_b200.so")

_lib = None


def load(path: str | None = None) -> "Api":
    """Load libgrid_b200.so and return the Python view of its API."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError(
            "libgrid_b200.so not found at %s; build it with `python -m libgrid_b200.build` "
            "(this package has no CPU fallback)" % p
        )
    api = Api(C.CDLL(p), cuda_layout=True, extensions=True, kind="b200")
    if path is None:
        _lib = api
    return api


class Grid:
    """A cgrid or rgrid pointer plus numpy views of its host array."""

    def __init__(self, api: "Api", ptr, real: bool):
        self.api, self.ptr, self.real = api, ptr, real

    @property
    def s(self):
        return self.ptr.contents

    @property
    def shape(self):
        s = self.s
        return (s.nx, s.ny, s.nz)

    def _view(self):
        s = self.s
        if self.real:
            n = s.nx * s.ny * s.nz2
            buf = (C.c_double * n).from_address(s.value)
            return np.frombuffer(buf, dtype=np.float64).reshape(s.nx, s.ny, s.nz2)
        n = s.nx * s.ny * s.nz
        buf = (C.c_double * (2 * n)).from_address(s.value)
        return np.frombuffer(buf, dtype=np.complex128).reshape(s.nx, s.ny, s.nz)

    def get(self) -> np.ndarray:
        """Copy of the grid values (host copy refreshed first)."""
        self.api.sync_host(self)
        v = self._view()
        return (v[:, :, : self.s.nz] if self.real else v).copy()

    def set(self, arr) -> None:
        """Overwrite the grid values from a numpy array of the logical shape."""
        v = self._view()
        if self.real:
            v[:, :, : self.s.nz] = np.asarray(arr, dtype=np.float64)
        else:
            v[...] = np.asarray(arr, dtype=np.complex128)
        self.api.host_modified(self)


class Api:
    """Thin Python face of a libgrid-compatible shared library."""

    def __init__(self, lib: C.CDLL, cuda_layout: bool, extensions: bool, kind: str):
        self.lib, self.kind = lib, kind
        self.CGrid, self.RGrid, self.WF, _ = capi.bind(lib, cuda_layout, extensions)
        self.extensions = extensions

    # boundary-condition function pointers of the library itself
    def cbc(self, name: str):
        return C.cast(getattr(self.lib, "cgrid_value_outside_" + name), C.c_void_p)

    def rbc(self, name: str):
        return C.cast(getattr(self.lib, "rgrid_value_outside_" + name), C.c_void_p)

    def sync_host(self, g: Grid) -> None:
        if self.kind == "b200":
            self.lib.gb_grid_sync_host(C.c_void_p(g.s.value))

    def host_modified(self, g: Grid) -> None:
        if self.kind == "b200":
            self.lib.gb_grid_host_modified(C.c_void_p(g.s.value))

    def cgrid(self, nx, ny, nz, step, bc="periodic", values=None, id=b"grid") -> Grid:
        p = self.lib.cgrid_alloc(nx, ny, nz, step, self.cbc(bc), None, id)
        if not p:
            raise MemoryError("cgrid_alloc failed")
        g = Grid(self, p, False)
        if values is not None:
            g.set(values)
        return g

    def rgrid(self, nx, ny, nz, step, bc="periodic", values=None, id=b"rgrid") -> Grid:
        p = self.lib.rgrid_alloc(nx, ny, nz, step, self.rbc(bc), None, id)
        if not p:
            raise MemoryError("rgrid_alloc failed")
        g = Grid(self, p, True)
        if values is not None:
            g.set(values)
        return g

    def wf(self, nx, ny, nz, step, mass, boundary, propagator, values=None, id=b"wf"):
        p = self.lib.grid_wf_alloc(nx, ny, nz, step, mass, bytes([boundary]), bytes([propagator]), id)
        if not p:
            raise ValueError("grid_wf_alloc failed")
        w = WaveFunction(self, p)
        if values is not None:
            w.grid.set(values)
        return w

    def batch(self, wfs, potentials, time) -> "Batch":
        """grid_wf_batch_alloc over WaveFunction objects and complex potential
        Grids (entries may be None)."""
        n = len(wfs)
        PW, PC = C.POINTER(self.WF), C.POINTER(self.CGrid)
        warr = (PW * n)(*[w.ptr for w in wfs])
        parr = (PC * n)(*[(p.ptr if p is not None else PC()) for p in potentials]) if potentials else None
        b = self.lib.grid_wf_batch_alloc(warr, parr, n, capi.Complex.of(time))
        if not b:
            raise RuntimeError("grid_wf_batch_alloc failed")
        return Batch(self, b)

    def free(self, obj) -> None:
        if isinstance(obj, WaveFunction):
            self.lib.grid_wf_free(obj.ptr)
        elif isinstance(obj, Grid):
            (self.lib.rgrid_free if obj.real else self.lib.cgrid_free)(obj.ptr)
        elif isinstance(obj, Batch):
            self.lib.grid_wf_batch_free(obj.ptr)


class Batch:
    def __init__(self, api: Api, ptr):
        self.api, self.ptr = api, ptr

    def propagate(self, steps: int) -> None:
        self.api.lib.grid_wf_batch_propagate(self.ptr, steps)


class WaveFunction:
    def __init__(self, api: Api, ptr):
        self.api, self.ptr = api, ptr

    @property
    def s(self):
        return self.ptr.contents

    @property
    def grid(self) -> Grid:
        return Grid(self.api, self.s.grid, False)

    def propagate(self, potential: Grid | None, time) -> None:
        self.api.lib.grid_wf_propagate(self.ptr, potential.ptr if potential else None, Complex.of(time))

    def propagate_gp(self, vext: Grid | None, g: float, time) -> None:
        self.api.lib.grid_wf_propagate_gp(self.ptr, vext.ptr if vext else None, g, Complex.of(time))

    def propagate_n(self, potential: Grid | None, time, nsteps: int) -> None:
        self.api.lib.grid_wf_propagate_n(self.ptr, potential.ptr if potential else None, Complex.of(time), nsteps)

    def propagate_gp_n(self, vext: Grid | None, g: float, time, nsteps: int) -> None:
        self.api.lib.grid_wf_propagate_gp_n(self.ptr, vext.ptr if vext else None, g, Complex.of(time), nsteps)

    def norm(self) -> float:
        return self.api.lib.grid_wf_norm(self.ptr)

    def normalize(self) -> float:
        return self.api.lib.grid_wf_normalize(self.ptr)

    def energy(self, potential: Grid | None) -> float:
        return self.api.lib.grid_wf_energy(self.ptr, potential.ptr if potential else None)

    def precision(self, mode: int) -> None:
        self.api.lib.grid_wf_precision(self.ptr, bytes([mode]))
