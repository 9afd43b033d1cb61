"""GPU parity: libgrid_b200 (sm_100a kernels, through the C ABI) against the
CPU oracles on the same seeded inputs.

Tolerances (FP64 mode): psi relative L2 <= 1e-11, energies relative <= 1e-12
(1e-10 absolute-relative for sums that cancel), norms relative <= 1e-12.
FP32 mode is checked against the FP64 oracle with its stated error bound.
"""
import numpy as np
import pytest

from conftest import rel
from libgrid_b200 import capi, workloads

pytestmark = pytest.mark.gpu

PER, DIR, NEU = capi.WF_PERIODIC_BOUNDARY, capi.WF_DIRICHLET_BOUNDARY, capi.WF_NEUMANN_BOUNDARY
FFT2, CFFT2, CN2 = capi.WF_2ND_ORDER_FFT, capi.WF_2ND_ORDER_CFFT, capi.WF_2ND_ORDER_CN
TOL_PSI = 1e-11


def rand_c(rng, shape, scale=1.0):
    return scale * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


def smooth_state(shape, step, kx=0.3):
    x, y, z = workloads.mesh(*shape, step)
    w = 0.25 * max(shape) * step
    return np.exp(-(x * x + y * y + z * z) / w**2 + 1j * kx * x)


# ------------------------------------------------------------------- FFT


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 32, 64), (1, 64, 128), (1, 1, 256), (32, 16, 2), (4, 2, 512), (2, 1024, 4)])
def test_fft3d_matches_numpy(b200, shape):
    rng = np.random.default_rng(sum(shape))
    a = rand_c(rng, shape)
    g = b200.cgrid(*shape, 0.1, values=a)
    b200.lib.cgrid_fft(g.ptr)
    f = g.get()
    assert rel(f, np.fft.fftn(a)) < 1e-13
    b200.lib.cgrid_inverse_fft_norm(g.ptr)
    assert rel(g.get(), a) < 1e-13
    b200.free(g)


def test_fft_non_power_of_two_fails_loudly():
    """The GPU FFT takes power-of-two line lengths (as the reference's CUDA
    build, src/cgrid.c:113-116); other lengths abort with a libgrid message
    instead of computing anything on a fallback path."""
    import subprocess
    import sys

    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import libgrid_b200 as gb\n"
        "api = gb.load()\n"
        "g = api.cgrid(12, 10, 14, 0.1)\n"
        "api.lib.cgrid_fft(g.ptr)\n"
        "print('returned')\n"
    ) % (__import__("conftest").ROOT,)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert p.returncode != 0
    assert "returned" not in p.stdout
    assert "power of two" in p.stderr


# ----------------------------------------------------- split-operator step


def b200_fft_run(b200, psi0, v, step, mass, time, nsteps, k0=(0.0, 0.0, 0.0), prop=FFT2, kmax=None, prec=0):
    w = b200.wf(*psi0.shape, step, mass, PER, prop, values=psi0)
    b200.lib.cgrid_set_momentum(w.s.grid, *k0)
    if kmax is not None:
        w.s.kmax = kmax
    if prec:
        w.precision(prec)
    pot = b200.cgrid(*psi0.shape, step, values=v) if v is not None else None
    for _ in range(nsteps):
        w.propagate(pot, time)
    out = w.grid.get()
    b200.free(w)
    if pot:
        b200.free(pot)
    return out


@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 16, 64), (1, 32, 64), (1, 1, 128), (8, 64, 1)])
@pytest.mark.parametrize("time", [0.05, -0.05j, 0.04 - 0.01j])
def test_split_step_fft(b200, restate, shape, time):
    rng = np.random.default_rng(7)
    step, mass = 0.4, 1.7
    psi0 = smooth_state(shape, step) + 0.01 * rand_c(rng, shape)
    v = 0.05 * rng.standard_normal(shape) + 0.002j * rng.standard_normal(shape)
    k0 = (0.2, -0.1, 0.05)
    got = b200_fft_run(b200, psi0, v, step, mass, time, 5, k0)
    want = psi0.copy()
    for _ in range(5):
        want = restate.fft_step(want, step, mass, time, k0=k0, vc=v)
    assert rel(got, want) < TOL_PSI


def test_split_step_no_potential(b200, restate):
    shape, step, mass = (16, 8, 32), 0.3, 1.0
    psi0 = smooth_state(shape, step)
    got = b200_fft_run(b200, psi0, None, step, mass, 0.1, 3)
    want = psi0.copy()
    for _ in range(3):
        want = restate.fft_step(want, step, mass, 0.1)
    assert rel(got, want) < TOL_PSI


def test_split_step_cfft_cutoff(b200, restate):
    shape, step, mass = (16, 16, 32), 0.3, 1.0
    rng = np.random.default_rng(3)
    psi0 = rand_c(rng, shape)
    v = 0.1 * rng.standard_normal(shape).astype(complex)
    kmax = 5.0  # below the largest |k| = pi/step so the cutoff is active
    got = b200_fft_run(b200, psi0, v, step, mass, 0.05, 4, prop=CFFT2, kmax=kmax)
    want = psi0.copy()
    for _ in range(4):
        want = restate.fft_step(want, step, mass, 0.05, vc=v, cutoff=1, kmax=kmax)
    assert rel(got, want) < TOL_PSI


@pytest.mark.parametrize("shape,time", [((32, 32, 32), 1.0), ((16, 32, 64), -1.0j), ((1, 64, 64), 0.5),
                                        ((32, 64, 256), 1.0), ((256, 16, 32), -1.0j)])
def test_gp_step_fft(b200, restate, shape, time):
    step, g = 0.5, 0.0025
    mass = 4.0 / workloads.GRID_AUTOAMU
    psi0, v = workloads.gp_wells(shape, step, g, seed=11)
    vr = workloads.padded(v)
    w = b200.wf(*shape, step, mass, PER, FFT2, values=psi0)
    vx = b200.rgrid(*shape, step, values=v)
    for _ in range(4):
        w.propagate_gp(vx, g, time)
    got = w.grid.get()
    want = psi0.copy()
    for _ in range(4):
        want = restate.fft_step(want, step, mass, time, vr=vr, g=g)
    assert rel(got, want) < TOL_PSI
    b200.free(w)
    b200.free(vx)


def test_long_run_gp_parity_and_norm(b200, restate):
    """1000 FP64 GP steps: psi within 1e-11 relative L2 of the oracle and the
    norm conserved to 1e-12 (real time)."""
    shape, step, g = (32, 32, 32), 0.5, 0.0025
    mass = 4.0 / workloads.GRID_AUTOAMU
    psi0, v = workloads.gp_wells(shape, step, g, seed=13)
    w = b200.wf(*shape, step, mass, PER, FFT2, values=psi0)
    vx = b200.rgrid(*shape, step, values=v)
    n0 = w.norm()
    for _ in range(1000):
        w.propagate_gp(vx, g, 1.0)
    got = w.grid.get()
    n1 = w.norm()
    want = psi0.copy()
    vr = workloads.padded(v)
    for _ in range(1000):
        want = restate.fft_step(want, step, mass, 1.0, vr=vr, g=g)
    assert rel(got, want) < TOL_PSI
    assert abs(n1 - n0) / n0 < 1e-12
    b200.free(w)
    b200.free(vx)


def test_fp32_mode_error_bound(b200, restate):
    shape, step, g = (32, 32, 32), 0.5, 0.0025
    mass = 4.0 / workloads.GRID_AUTOAMU
    psi0, v = workloads.gp_wells(shape, step, g, seed=5)
    w = b200.wf(*shape, step, mass, PER, FFT2, values=psi0)
    w.precision(capi.GRID_PREC_FP32)
    vx = b200.rgrid(*shape, step, values=v)
    for _ in range(10):
        w.propagate_gp(vx, g, 1.0)
    got = w.grid.get()
    n32 = w.norm()
    want = psi0.copy()
    for _ in range(10):
        want = restate.fft_step(want, step, mass, 1.0, vr=workloads.padded(v), g=g)
    # stated FP32-mode bound after 10 steps (FP32 storage and FFTs)
    assert rel(got, want) < 2e-5
    assert abs(n32 - restate.norm(want, step)) / restate.norm(want, step) < 1e-5
    b200.free(w)
    b200.free(vx)


# ------------------------------------------------------------ Crank-Nicolson


def b200_cn_run(b200, psi0, v, step, mass, time, bc, nsteps, k0=(0.0, 0.0, 0.0), omega=0.0, absorb=None, gp=None):
    w = b200.wf(*psi0.shape, step, mass, bc, CN2, values=psi0)
    b200.lib.cgrid_set_momentum(w.s.grid, *k0)
    if omega:
        b200.lib.cgrid_set_rotation(w.s.grid, omega)
    if absorb is not None:
        b200.lib.grid_wf_boundary(w.ptr, None, *absorb)
    pot = b200.cgrid(*psi0.shape, step, values=v) if v is not None else None
    vx = b200.rgrid(*psi0.shape, step, values=gp[0]) if gp is not None else None
    for _ in range(nsteps):
        if gp is not None:
            w.propagate_gp(vx, gp[1], time)
        else:
            w.propagate(pot, time)
    out = w.grid.get()
    b200.free(w)
    for o in (pot, vx):
        if o:
            b200.free(o)
    return out


@pytest.mark.parametrize("bc", [DIR, NEU, PER])
@pytest.mark.parametrize("shape", [(12, 10, 14), (24, 24, 24), (1, 40, 48), (2, 3, 64), (3, 2, 300), (33, 5, 7)])
@pytest.mark.parametrize("time", [0.05, -0.2j])
def test_cn_step(b200, restate, bc, shape, time):
    rng = np.random.default_rng(17)
    step, mass = 0.3, 1.3
    psi0 = smooth_state(shape, step) + 0.01 * rand_c(rng, shape)
    v = 0.05 * rng.standard_normal(shape) + 0.001j * rng.standard_normal(shape)
    k0 = (0.1, -0.2, 0.3)
    got = b200_cn_run(b200, psi0, v, step, mass, time, bc, 3, k0)
    want = psi0.copy()
    for _ in range(3):
        want = restate.cn_step(want, step, mass, time, bc, k0=k0, vc=v)
    assert rel(got, want) < TOL_PSI


@pytest.mark.parametrize("bc", [DIR, PER])
def test_cn_rotation_and_absorber(b200, restate, bc):
    """General line-solver path: rotating frame and absorbing ramp."""
    shape, step, mass = (16, 12, 10), 0.3, 1.0
    rng = np.random.default_rng(23)
    psi0 = smooth_state(shape, step) + 0.01 * rand_c(rng, shape)
    v = 0.02 * rng.standard_normal(shape).astype(complex)
    absorb = (3, 12, 2, 9, 2, 7)
    got = b200_cn_run(b200, psi0, v, step, mass, 0.05, bc, 3, omega=0.3, absorb=absorb)
    want = psi0.copy()
    for _ in range(3):
        want = restate.cn_step(want, step, mass, 0.05, bc, omega=0.3, vc=v, absorb=absorb)
    assert rel(got, want) < TOL_PSI


@pytest.mark.parametrize("bc", [DIR, NEU, PER])
@pytest.mark.parametrize("shape", [(16, 192, 200), (256, 4, 33)])
def test_cn_line_solvers_agree(b200, bc, shape):
    """The warp-cooperative line solver (lines up to 256 points, segment
    carries by a warp-shuffle scan) and the segment-per-warp solver solve the
    same systems; they differ only in rounding."""
    lib = b200.lib
    step, g = 0.3, 0.001
    mass = 4.0 / workloads.GRID_AUTOAMU
    psi0, v = workloads.cn_wells(shape, step, g, seed=21)
    out = []
    old = lib.gb_cn_warp_solver(-1)
    try:
        for on in (1, 0):
            lib.gb_cn_warp_solver(on)
            out.append(b200_cn_run(b200, psi0, None, step, mass, 0.5, bc, 3, k0=(0.1, 0.0, -0.2), gp=(v, g)))
    finally:
        lib.gb_cn_warp_solver(old)
    assert rel(out[0], out[1]) < 1e-13


def test_cn_gp_dirichlet(b200, restate):
    shape, step, g = (24, 20, 28), 0.3, 0.001
    mass = 4.0 / workloads.GRID_AUTOAMU
    psi0, v = workloads.cn_wells(shape, step, g, seed=9)
    got = b200_cn_run(b200, psi0, None, step, mass, 0.5, DIR, 4, gp=(v, g))
    want = psi0.copy()
    for _ in range(4):
        want = restate.cn_step(want, step, mass, 0.5, DIR, vr=workloads.padded(v), g=g)
    assert rel(got, want) < TOL_PSI


# -------------------------------------------------------------- analysis


@pytest.mark.parametrize("shape", [(16, 16, 16), (1, 32, 64), (12, 10, 14)])
def test_norm_and_energies(b200, restate, shape):
    step, mass = 0.35, 2.0
    rng = np.random.default_rng(31)
    psi = smooth_state(shape, step) + 0.05 * rand_c(rng, shape)
    v = 0.1 * rng.standard_normal(shape)
    for bc, bcname, obc in ((PER, "periodic", 2), (DIR, "dirichlet", 0), (NEU, "neumann", 1)):
        prop = CN2 if bc != PER else FFT2
        w = b200.wf(*shape, step, mass, bc, prop, values=psi)
        vx = b200.rgrid(*shape, step, values=v)
        assert abs(w.norm() - restate.norm(psi, step)) / restate.norm(psi, step) < 1e-12
        b200.lib.grid_wf_analyze_method(b"\x00")
        t_fd = b200.lib.grid_wf_kinetic_energy_cn(w.ptr)
        t_ref = restate.kinetic_energy_fd(psi, step, mass, obc)
        assert abs(t_fd - t_ref) <= 1e-12 * abs(t_ref) + 1e-13
        e = b200.lib.grid_wf_energy(w.ptr, vx.ptr)
        e_ref = t_ref + restate.potential_energy(psi, workloads.padded(v), step)
        assert abs(e - e_ref) <= 1e-12 * abs(e_ref) + 1e-13
        if bc == PER and all(n & (n - 1) == 0 for n in shape):
            t_fft = b200.lib.grid_wf_kinetic_energy_fft(w.ptr)
            t_fft_ref = restate.kinetic_energy_fft(psi, step, mass)
            assert abs(t_fft - t_fft_ref) <= 1e-12 * abs(t_fft_ref)
            # psi is left untouched by the FFT energy
            assert rel(w.grid.get(), psi) == 0.0
        b200.free(w)
        b200.free(vx)


@pytest.mark.parametrize("bcname,obc", [("periodic", 2), ("dirichlet", 0), ("neumann", 1)])
@pytest.mark.parametrize("shape", [(8, 9, 10), (1, 16, 32), (20, 20, 20)])
def test_fd_laplace(b200, restate, bcname, obc, shape):
    rng = np.random.default_rng(41)
    a = rand_c(rng, shape)
    g = b200.cgrid(*shape, 0.25, bc=bcname, values=a)
    o = b200.cgrid(*shape, 0.25, bc=bcname)
    b200.lib.cgrid_fd_laplace(g.ptr, o.ptr)
    assert rel(o.get(), restate.fd_laplace(a, 0.25, obc)) < 1e-14
    b200.free(g)
    b200.free(o)


def test_imaginary_time_normalize(b200, restate):
    shape, step, mass = (16, 16, 16), 0.5, 1.0
    x, y, z = workloads.mesh(*shape, step)
    v = (0.5 * 0.2 * (x * x + y * y + z * z)).astype(complex)
    psi0 = np.exp(-(x * x + y * y + z * z) / 4.0) * (1 + 0.1 * x)
    w = b200.wf(*shape, step, mass, PER, FFT2, values=psi0)
    pot = b200.cgrid(*shape, step, values=v)
    want = psi0.copy()
    for _ in range(10):
        w.propagate(pot, -0.1j)
        w.normalize()
        want = restate.fft_step(want, step, mass, -0.1j, vc=v)
        want = want * np.sqrt(1.0 / restate.norm(want, step))
    assert rel(w.grid.get(), want) < TOL_PSI
    b200.free(w)
    b200.free(pot)


def test_fft_absorbing_boundary_composition(b200, restate):
    """Real-time step + imaginary-time step + ramp blend (src/grid_wf.c:396-422)."""
    shape, step, mass = (16, 16, 16), 0.4, 1.0
    rng = np.random.default_rng(51)
    psi0 = smooth_state(shape, step) + 0.01 * rand_c(rng, shape)
    v = 0.05 * rng.standard_normal(shape).astype(complex)
    lh = (3, 12, 3, 12, 3, 12)
    w = b200.wf(*shape, step, mass, PER, FFT2, values=psi0)
    b200.lib.grid_wf_boundary(w.ptr, None, *lh)
    pot = b200.cgrid(*shape, step, values=v)
    w.propagate(pot, 0.05)
    got = w.grid.get()
    real = restate.fft_step(psi0.copy(), step, mass, 0.05, vc=v)
    imag = restate.fft_step(psi0.copy(), step, mass, -0.05j, vc=v)
    i, j, k = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")

    def ramp(q, lo, hi):
        return np.where(q < lo, (lo - q) / lo, np.where(q > hi, (q - hi) / lo, 0.0))

    t = (ramp(i, lh[0], lh[1]) + ramp(j, lh[2], lh[3]) + ramp(k, lh[4], lh[5])) * (2.0 / 3.0)
    a = np.minimum(t, 1.0)
    want = (1 - a) * real + a * imag
    assert rel(got, want) < TOL_PSI
    b200.free(w)
    b200.free(pot)


# ----------------------------------------- against the compiled reference


def _ref_wf(ref, psi0, step, mass, bc, prop):
    w = ref.wf(*psi0.shape, step, mass, bc, prop, values=psi0)
    return w


@pytest.mark.parametrize("prop", [capi.WF_4TH_ORDER_FFT, capi.WF_4TH_ORDER_CN, capi.WF_1ST_ORDER_EULER])
def test_other_propagators_vs_reference(b200, ref, prop):
    shape, step, mass = (16, 16, 16), 0.4, 1.0
    rng = np.random.default_rng(61)
    psi0 = smooth_state(shape, step) + 0.01 * rand_c(rng, shape)
    v = (0.05 * rng.standard_normal(shape)).astype(complex)
    out = []
    for api in (b200, ref):
        api.lib.grid_wf_analyze_method(b"\x00")
        w = api.wf(*shape, step, mass, PER, prop, values=psi0)
        pot = api.cgrid(*shape, step, values=v)
        for _ in range(3):
            w.propagate(pot, 0.01)
        out.append(w.grid.get())
    assert rel(out[0], out[1]) < TOL_PSI


def test_predict_correct_vs_reference(b200, ref):
    shape, step, mass = (16, 8, 32), 0.4, 1.0
    rng = np.random.default_rng(71)
    psi0 = smooth_state(shape, step) + 0.01 * rand_c(rng, shape)
    v = (0.05 * rng.standard_normal(shape)).astype(complex)
    out = []
    for api in (b200, ref):
        w = api.wf(*shape, step, mass, PER, FFT2, values=psi0)
        wp = api.wf(*shape, step, mass, PER, FFT2)
        pot = api.cgrid(*shape, step, values=v)
        api.lib.grid_wf_propagate_predict(w.ptr, wp.ptr, pot.ptr, capi.Complex.of(0.05))
        api.lib.grid_wf_propagate_correct(w.ptr, pot.ptr, capi.Complex.of(0.05))
        out.append((w.grid.get(), wp.grid.get()))
    assert rel(out[0][0], out[1][0]) < TOL_PSI
    assert rel(out[0][1], out[1][1]) < TOL_PSI


@pytest.mark.parametrize("prop,tstep,cons,absorb", [
    (FFT2, 0.05, 0.0, None),
    (FFT2, 0.05, 0.013, None),
    (FFT2, -0.05j, 0.0, None),
    (FFT2, 0.04 - 0.01j, 0.002, None),
    (FFT2, 0.05, 0.0, (3, 12, 2, 5, 4, 25)),  # FFT ignores the absorbing ramp here (src/grid_wf.c:593)
    (CN2, 0.05, 0.0, (3, 12, 2, 5, 4, 25)),
    (CN2, -0.05j, 0.01, None),
])
def test_propagate_potential_vs_reference(b200, ref, prop, tstep, cons, absorb):
    """grid_wf_propagate_potential on its own (src/grid_wf.c:569-602):
    psi *= exp(-i c (cons + V) / hbar), with the absorbing-region time
    ramp of the CN propagators, against the compiled reference."""
    shape, step, mass = (16, 8, 32), 0.4, 1.0
    rng = np.random.default_rng(91)
    psi0 = smooth_state(shape, step) + 0.01 * rand_c(rng, shape)
    v = 0.05 * rng.standard_normal(shape) + 0.01j * rng.standard_normal(shape)
    out = []
    for api in (b200, ref):
        w = api.wf(*shape, step, mass, PER, prop, values=psi0)
        if absorb is not None:
            api.lib.grid_wf_boundary(w.ptr, None, *absorb)
        pot = api.cgrid(*shape, step, values=v)
        api.lib.grid_wf_propagate_potential(w.ptr, capi.Complex.of(tstep), pot.ptr, cons)
        out.append(w.grid.get())
    assert rel(out[0], out[1]) < TOL_PSI


def test_energy_and_error_vs_reference(b200, ref):
    shape, step, mass = (16, 16, 16), 0.4, 1.0
    x, y, z = workloads.mesh(*shape, step)
    v = (0.5 * 0.3 * (x * x + y * y + z * z)).astype(complex)
    psi = np.exp(-(x * x + y * y + z * z) / 5.0) * (1 + 0.2 * y)
    # the error formula assumes a normalized state (src/grid_wf_diag.c:49-60)
    psi = psi / np.sqrt(np.sum(np.abs(psi) ** 2) * step**3)
    res = []
    for api in (b200, ref):
        w = api.wf(*shape, step, mass, PER, FFT2, values=psi)
        pot = api.cgrid(*shape, step, values=v)
        ws = api.cgrid(*shape, step)
        import ctypes as C

        err = C.c_double()
        e = api.lib.grid_wf_energy_and_error(w.ptr, pot.ptr, ws.ptr, C.byref(err))
        res.append((e, err.value))
    assert abs(res[0][0] - res[1][0]) <= 1e-12 * abs(res[1][0])
    assert abs(res[0][1] - res[1][1]) <= 1e-8 * abs(res[1][1]) + 1e-12


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 4, 32), (1, 16, 64)])
def test_rgrid_fft_roundtrip(b200, ref, shape):
    rng = np.random.default_rng(81)
    a = rng.standard_normal(shape)
    out = []
    for api in (b200, ref):
        g = api.rgrid(*shape, 0.2, values=a)
        api.lib.rgrid_fft(g.ptr)
        api.sync_host(g)
        spec = g._view().copy()
        api.lib.rgrid_inverse_fft_norm(g.ptr)
        out.append((spec, g.get()))
    nzh = shape[2] // 2 + 1
    s0 = out[0][0].view(np.complex128)[:, :, :nzh]
    s1 = out[1][0].view(np.complex128)[:, :, :nzh]
    assert rel(s0, s1) < 1e-13
    assert rel(out[0][1], a) < 1e-13


def test_mixed_ops_vs_reference(b200, ref):
    shape, step = (8, 12, 10), 0.3
    rng = np.random.default_rng(91)
    psi = rand_c(rng, shape)
    r = rng.standard_normal(shape)
    res = []
    for api in (b200, ref):
        w = api.wf(*shape, step, 1.0, PER, FFT2, values=psi)
        rg = api.rgrid(*shape, step, values=r)
        d = api.rgrid(*shape, step)
        api.lib.grid_wf_density(w.ptr, d.ptr)
        c = api.cgrid(*shape, step)
        api.lib.grid_real_to_complex_re(c.ptr, rg.ptr)
        api.lib.grid_product_complex_with_real(c.ptr, d.ptr)
        ev = api.lib.grid_grid_expectation_value(w.s.grid, rg.ptr)
        res.append((d.get(), c.get(), ev))
    assert rel(res[0][0], res[1][0]) < 1e-15
    assert rel(res[0][1], res[1][1]) < 1e-15
    assert abs(res[0][2] - res[1][2]) <= 1e-12 * abs(res[1][2])


def test_phase_sincos_against_cuda(b200):
    """The propagation kernels' FP64 phase sine/cosine (Cody-Waite reduction
    + Taylor polynomials, library routine beyond 1e7) against the CUDA
    library sincos."""
    import ctypes as C

    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(-1e-3, 1e-3, 4000), rng.uniform(-0.07, 0.07, 4000), rng.uniform(-4, 4, 4000), rng.uniform(-1e4, 1e4, 4000),
                        rng.uniform(-1e7, 1e7, 2000), rng.uniform(-1e9, 1e9, 500),
                        np.array([0.0, -0.0, np.pi / 4, -np.pi / 4, np.pi / 2, np.pi, 3e6 * np.pi])])
    err = (C.c_double * 2)()
    b200.lib.gb_sincos_selftest.argtypes = [C.c_void_p, C.c_long, C.POINTER(C.c_double)]
    assert b200.lib.gb_sincos_selftest(x.ctypes.data, len(x), err) == 0
    # a few ulp of 1 (arguments up to 1e7 keep the reduced argument accurate
    # to ~1e-16)
    assert err[0] < 1e-15 and err[1] < 1e-15, (err[0], err[1])
