"""Seeded synthetic inputs for the propagation workloads.

All coordinates follow the reference's grid convention
x_i = (i - nx/2) step - x0 (src/cgrid.c:808-812).  Random draws use
numpy.random.default_rng(seed); the seeds and the unspecified distribution
choices are fixed here and recorded in the workload descriptions.

  wavepacket  -- harmonic trap V = k r^2 / 2 with a Gaussian packet
                 exp(-r^2/w^2 + i kx x) (the FFT real-time case, 128^3 at full
                 size)
  gp_wells    -- V_ext = -sum_i d_i exp(-|r - c_i|^2 / w_i^2), 8 wells,
                 d ~ U(1e-4, 1e-3) Ha, w ~ U(3, 10) bohr, c ~ U(-L/4, L/4)^3;
                 Thomas-Fermi start sqrt(max(0, (mu - V)/g)) (1 + 0.01 (xi1 + i xi2))
                 with mu = 2 max(d) (the GP case, 256^3 at full size)
  cn_wells    -- the same well family with a window vanishing at the
                 Dirichlet walls (the CN case, 192^3 at full size)
"""
from __future__ import annotations

import numpy as np

GRID_AUTOAMU = 1.0 / 1822.88853006  # src/au.h:17


def coords(n: int, step: float, origin: float = 0.0) -> np.ndarray:
    return (np.arange(n) - n // 2) * step - origin


def mesh(nx, ny, nz, step):
    return np.meshgrid(coords(nx, step), coords(ny, step), coords(nz, step), indexing="ij")


def padded(v: np.ndarray) -> np.ndarray:
    """Real (nx, ny, nz) -> the reference's padded rgrid layout (nz2 rows)."""
    nx, ny, nz = v.shape
    out = np.zeros((nx, ny, 2 * (nz // 2 + 1)))
    out[:, :, :nz] = v
    return out


def wavepacket(n=128, step=0.2, k=0.01, width=2.0, kx=0.5):
    x, y, z = mesh(n, n, n, step)
    r2 = x * x + y * y + z * z
    v = 0.5 * k * r2
    psi = np.exp(-r2 / width**2 + 1j * kx * x)
    return psi, v.astype(np.complex128)


def wells(shape, step, seed, nwells=8):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    L = max(nx, ny, nz) * step
    d = rng.uniform(1e-4, 1e-3, nwells)
    w = rng.uniform(3.0, 10.0, nwells)
    c = rng.uniform(-L / 4, L / 4, (nwells, 3))
    x, y, z = mesh(nx, ny, nz, step)
    v = np.zeros(shape)
    for i in range(nwells):
        v -= d[i] * np.exp(-((x - c[i, 0]) ** 2 + (y - c[i, 1]) ** 2 + (z - c[i, 2]) ** 2) / w[i] ** 2)
    return v, d


def gp_wells(shape=(256, 256, 256), step=0.5, g=0.0025, seed=2):
    v, d = wells(shape, step, seed)
    mu = 2.0 * d.max()
    rng = np.random.default_rng(seed + 1000)
    xi1 = rng.standard_normal(shape)
    xi2 = rng.standard_normal(shape)
    psi = np.sqrt(np.maximum(0.0, (mu - v) / g)) * (1.0 + 0.01 * (xi1 + 1j * xi2))
    return psi.astype(np.complex128), v


def cn_wells(shape=(192, 192, 192), step=0.3, g=0.001, seed=3):
    psi, v = gp_wells(shape, step, g, seed)
    win = np.ones(shape)
    for ax, n in enumerate(shape):
        s = np.sin(np.pi * (np.arange(n) + 1) / (n + 1))
        sh = [1, 1, 1]
        sh[ax] = n
        win = win * s.reshape(sh)
    return (psi * win).astype(np.complex128), v


def batch2d(seed: int = 7, sizes=(64, 128, 256, 512), per_size: int = 24, step: float = 0.2):
    """The batched 2-D workload: per_size instances of each n x n size (order
    shuffled with the seed), each with V = k r^2 / 2 (k ~ U(0.005, 0.02)) plus
    1..6 Gaussian bumps (height ~ U(1e-3, 1e-2) Ha, width ~ U(1, 4) bohr,
    centre ~ U(-L/4, L/4)^2) as a complex potential, and a Gaussian start
    exp(-r^2/w^2 + i (k_y y + k_z z)) with w = 2 and k ~ U(-1, 1)^2.
    Returns a list of (shape, psi0, v)."""
    rng = np.random.default_rng(seed)
    ns = [n for n in sizes for _ in range(per_size)]
    rng.shuffle(ns)
    out = []
    for n in ns:
        _, y, z = mesh(1, n, n, step)
        r2 = y * y + z * z
        v = 0.5 * rng.uniform(0.005, 0.02) * r2
        L = n * step
        for _ in range(int(rng.integers(1, 7))):
            h, w = rng.uniform(1e-3, 1e-2), rng.uniform(1.0, 4.0)
            cy, cz = rng.uniform(-L / 4, L / 4, 2)
            v = v + h * np.exp(-((y - cy) ** 2 + (z - cz) ** 2) / w**2)
        ky, kz = rng.uniform(-1.0, 1.0, 2)
        psi = np.exp(-r2 / 4.0 + 1j * (ky * y + kz * z))
        out.append(((1, n, n), psi.astype(np.complex128), v.astype(np.complex128)))
    return out
