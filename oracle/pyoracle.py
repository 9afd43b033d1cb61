"""ORACLE (test infrastructure only).

Python access to the two CPU oracles of the propagation path:
  * the project's plain-C restatement (oracle/gbo_path.c + oracle/gbo_fft.c),
    built into oracle/_build/libgbo.so, and
  * the reference's own CPU sources compiled unchanged against the FFTW
    stand-in (oracle/_ref/libgrid_ref.so, built by oracle/build_ref.sh where
    the reference sources are available).
Only the tests, the smoke check and the benchmark's CPU-baseline leg use this
module, and only as the thing checked against or timed beside the GPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
GBO_LIB = os.path.join(BUILD, "libgbo.so")
REF_LIB = os.path.join(HERE, "_ref", "libgrid_ref.so")

_gbo = None
_ref = None


def build_gbo(force: bool = False) -> str:
    """Compile the restatement (plain C, OpenMP, no FMA contraction)."""
    srcs = [os.path.join(HERE, "gbo_fft.c"), os.path.join(HERE, "gbo_path.c")]
    if not force and os.path.exists(GBO_LIB):
        m = os.path.getmtime(GBO_LIB)
        if all(os.path.getmtime(s) <= m for s in srcs + [os.path.join(HERE, "gbo_fft.h")]):
            return GBO_LIB
    os.makedirs(BUILD, exist_ok=True)
    cmd = ["gcc", "-std=gnu11", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-shared", "-o", GBO_LIB] + srcs + ["-lm"]
    subprocess.run(cmd, check=True)
    return GBO_LIB


def _cp(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Restatement:
    """Wrappers over oracle/gbo_path.c on numpy arrays (complex128, C order)."""

    def __init__(self, lib: C.CDLL):
        self.lib = lib
        D, L, V, I = C.c_double, C.c_long, C.c_void_p, C.c_int
        cx = _Cx
        lib.gbo_fft3d.argtypes = [V, L, L, L, I]
        lib.gbo_fft3d.restype = None
        lib.gbo_fft_step.argtypes = [V, L, L, L, D, D, cx, D, D, D, V, V, D, I, D]
        lib.gbo_fft_step.restype = None
        lib.gbo_cn_step.argtypes = [V, L, L, L, D, D, cx, I, D, D, D, D, D, D, V, V, D, V]
        lib.gbo_cn_step.restype = None
        lib.gbo_cn_kinetic.argtypes = [V, L, L, L, D, D, cx, I, D, D, D, D, D, D, V]
        lib.gbo_cn_kinetic.restype = None
        lib.gbo_potential.argtypes = [V, L, L, L, cx, V, V, D, D, V]
        lib.gbo_potential.restype = None
        lib.gbo_kinetic_fft.argtypes = [V, L, L, L, D, D, cx, D, D, D, I, D]
        lib.gbo_kinetic_fft.restype = None
        lib.gbo_norm.argtypes = [V, L, L, L, D]
        lib.gbo_norm.restype = D
        lib.gbo_fd_laplace.argtypes = [V, V, L, L, L, D, I, cx]
        lib.gbo_fd_laplace.restype = None
        lib.gbo_kinetic_energy_fd.argtypes = [V, L, L, L, D, D, I, cx]
        lib.gbo_kinetic_energy_fd.restype = D
        lib.gbo_kinetic_energy_fft.argtypes = [V, L, L, L, D, D]
        lib.gbo_kinetic_energy_fft.restype = D
        lib.gbo_potential_energy.argtypes = [V, V, L, L, L, D]
        lib.gbo_potential_energy.restype = D

    @staticmethod
    def _c(a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        return a

    def fft3d(self, a, sign=-1):
        a = self._c(a).copy()
        self.lib.gbo_fft3d(_cp(a), *a.shape, sign)
        return a

    def fft_step(self, psi, step, mass, time, k0=(0.0, 0.0, 0.0), vc=None, vr=None, g=0.0, cutoff=0, kmax=9999.0):
        psi = self._c(psi)
        vcp = _cp(self._c(vc)) if vc is not None else None
        vra = np.ascontiguousarray(vr, dtype=np.float64) if vr is not None else None
        self.lib.gbo_fft_step(_cp(psi), *psi.shape, step, mass, _Cx.of(time), *k0, vcp,
                              _cp(vra) if vra is not None else None, g, cutoff, kmax)
        return psi

    def cn_step(self, psi, step, mass, time, bc, k0=(0.0, 0.0, 0.0), omega=0.0, x0=0.0, y0=0.0, vc=None, vr=None, g=0.0,
                absorb=None):
        psi = self._c(psi)
        vca = self._c(vc) if vc is not None else None
        vra = np.ascontiguousarray(vr, dtype=np.float64) if vr is not None else None
        lh = np.asarray(absorb, dtype=np.int64) if absorb is not None else None
        self.lib.gbo_cn_step(_cp(psi), *psi.shape, step, mass, _Cx.of(time), bc, *k0, omega, x0, y0,
                             _cp(vca) if vca is not None else None, _cp(vra) if vra is not None else None, g,
                             _cp(lh) if lh is not None else None)
        return psi

    def norm(self, psi, step):
        psi = self._c(psi)
        return self.lib.gbo_norm(_cp(psi), *psi.shape, step)

    def fd_laplace(self, a, step, bc, outside=0.0):
        a = self._c(a)
        out = np.empty_like(a)
        self.lib.gbo_fd_laplace(_cp(a), _cp(out), *a.shape, step, bc, _Cx.of(outside))
        return out

    def kinetic_energy_fd(self, psi, step, mass, bc, outside=0.0):
        psi = self._c(psi)
        return self.lib.gbo_kinetic_energy_fd(_cp(psi), *psi.shape, step, mass, bc, _Cx.of(outside))

    def kinetic_energy_fft(self, psi, step, mass):
        psi = self._c(psi)
        return self.lib.gbo_kinetic_energy_fft(_cp(psi), *psi.shape, step, mass)

    def potential_energy(self, psi, vr, step):
        psi = self._c(psi)
        vr = np.ascontiguousarray(vr, dtype=np.float64)
        return self.lib.gbo_potential_energy(_cp(psi), _cp(vr), *psi.shape, step)


class _Cx(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]

    @classmethod
    def of(cls, z):
        z = complex(z)
        return cls(z.real, z.imag)


def restatement() -> Restatement:
    global _gbo
    if _gbo is None:
        _gbo = Restatement(C.CDLL(build_gbo()))
    return _gbo


def reference_available() -> bool:
    return os.path.exists(REF_LIB)


def reference(threads: int | None = None):
    """The reference's CPU build as a libgrid_b200.Api (kind 'ref').

    grid_threads_init arms floating-point traps (src/threads.c:125); they are
    switched off again so the host process keeps IEEE semantics.
    """
    global _ref
    if _ref is not None:
        return _ref
    if not reference_available():
        raise FileNotFoundError(REF_LIB)
    from libgrid_b200 import Api

    api = Api(C.CDLL(REF_LIB), cuda_layout=False, extensions=False, kind="ref")
    api.lib.grid_threads_init(threads or os.cpu_count() or 1)
    libm = C.CDLL("libm.so.6")
    libm.fedisableexcept(0x3D)
    _ref = api
    return api
