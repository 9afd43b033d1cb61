"""Small drivers of the propagation workloads for profilers (ncu) and
manual runs; each builds a workload from libgrid_b200.workloads, steps it
through the C API on the current GPU and returns.

    python tests/drivers.py gp [n] [steps] [prec: 0 FP64, 1 FP32]
    python tests/drivers.py cn [n] [steps]
    python tests/drivers.py batch [steps] [prec]
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from libgrid_b200.workloads import GRID_AUTOAMU, batch2d, cn_wells, gp_wells  # noqa: E402


def run_gp_steps(n: int = 256, steps: int = 3, prec: int = 0) -> float:
    """Propagate the GP workload at n^3 for `steps` steps through the C API on
    the current GPU and return the final norm (a small driver for profilers:
    ``python tests/drivers.py gp 256 3``)."""
    import libgrid_b200 as gb
    from libgrid_b200 import capi

    api = gb.load()
    api.lib.cuda_enable(b"\x01", 0, None)
    shape, step, g = (n, n, n), 0.5, 0.0025
    mass = 4.0 / GRID_AUTOAMU
    psi0, v = gp_wells(shape, step, g, seed=2)
    w = api.wf(*shape, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT, values=psi0)
    if prec:
        w.precision(prec)
    vx = api.rgrid(*shape, step, values=v)
    for _ in range(steps):
        w.propagate_gp(vx, g, 1.0)
    api.lib.gb_synchronize()
    nrm = w.norm()
    api.free(w)
    api.free(vx)
    return nrm


def run_cn_steps(n: int = 192, steps: int = 3) -> float:
    """The Crank-Nicolson GP workload at n^3 (Dirichlet walls, step 0.3,
    g 0.001, 4 amu, dt 0.5) for `steps` steps; returns the final norm."""
    import libgrid_b200 as gb
    from libgrid_b200 import capi

    api = gb.load()
    api.lib.cuda_enable(b"\x01", 0, None)
    shape, step, g = (n, n, n), 0.3, 0.001
    psi0, v = cn_wells(shape, step, g)
    w = api.wf(*shape, step, 4.0 / GRID_AUTOAMU, capi.WF_DIRICHLET_BOUNDARY, capi.WF_2ND_ORDER_CN, values=psi0)
    vx = api.rgrid(*shape, step, values=v)
    for _ in range(steps):
        w.propagate_gp(vx, g, 0.5)
    api.lib.gb_synchronize()
    nrm = w.norm()
    api.free(w)
    api.free(vx)
    return nrm


def run_batch_steps(steps: int = 8, prec: int = 0) -> None:
    """The batched 2-D workload (batch2d) for `steps` steps in one call."""
    import libgrid_b200 as gb
    from libgrid_b200 import capi

    api = gb.load()
    api.lib.cuda_enable(b"\x01", 0, None)
    inst = batch2d(seed=7)
    wfs = [api.wf(*sh, 0.2, 1.0, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT, values=p) for sh, p, _ in inst]
    pots = [api.cgrid(*sh, 0.2, values=v) for sh, _, v in inst]
    if prec:
        for w in wfs:
            w.precision(prec)
    b = api.batch(wfs, pots, 0.05)
    b.propagate(steps)
    api.lib.gb_synchronize()
    api.free(b)
    for o in wfs + pots:
        api.free(o)


def run_unet_step(n: int = 128, tensor_cores: int = 1, reps: int = 1, batch: int = 1) -> None:
    """One forward and backward pass of the warm-start U-Net at n^3 with
    random weights and inputs (tensor-core or SIMT convolutions), over
    `batch` samples stacked in one launch per layer."""
    import ctypes as C

    import numpy as np

    import libgrid_b200 as gb
    from libgrid_b200 import warmstart as ws

    api = gb.load()
    api.lib.cuda_enable(b"\x01", 0, None)
    api.lib.gb_unet_tensor_cores.argtypes = [C.c_int]
    api.lib.gb_unet_tensor_cores(tensor_cores)
    rng = np.random.default_rng(1)
    net = ws.DeviceUNet(api, n, cin=3, seed=0, batch=batch)
    x = rng.standard_normal((3, batch, n, n, n)).astype(np.float32)
    api.lib.gb_h2d(net._act("in"), x.ctypes.data, x.nbytes)
    tgt = net.set_target(rng.standard_normal((batch, n, n, n)).astype(np.float32))
    for _ in range(reps):
        net.forward()
        net.loss_grad(tgt)
        net.backward()
    api.lib.gb_synchronize()
    net.free()


def run_ops(n: int = 256) -> None:
    """One call of each grid operation of the path at n^3 (FD stencils,
    k-space operators, pointwise products, FFT, convolution, interpolation,
    density, reductions), for an ncu launch list of those kernels."""
    import numpy as np

    import libgrid_b200 as gb
    from libgrid_b200 import capi

    api = gb.load()
    lib = api.lib
    lib.cuda_enable(b"\x01", 0, None)
    rng = np.random.default_rng(2)
    shape = (n, n, n)
    a = api.cgrid(*shape, 0.2, values=rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    b = api.cgrid(*shape, 0.2, values=rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    c = api.cgrid(*shape, 0.2)
    d = api.cgrid(*shape, 0.17)
    r = api.rgrid(*shape, 0.2, values=rng.standard_normal(shape))
    r2 = api.rgrid(*shape, 0.2)
    w = api.wf(*shape, 0.2, 1.0, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT)
    lib.cgrid_copy(w.s.grid, a.ptr)
    lib.cgrid_fd_laplace(a.ptr, c.ptr)
    lib.cgrid_fd_gradient_x(a.ptr, c.ptr)
    lib.rgrid_fd_laplace(r.ptr, r2.ptr)
    lib.cgrid_product(c.ptr, a.ptr, b.ptr)
    lib.cgrid_multiply(c.ptr, capi.Complex.of(0.5 - 0.25j))
    lib.grid_wf_density(w.ptr, r2.ptr)
    lib.cgrid_integral_of_square(a.ptr)
    lib.cgrid_fft(a.ptr)
    lib.cgrid_fft(b.ptr)
    lib.cgrid_fft_laplace(a.ptr, c.ptr)
    lib.cgrid_fft_convolute(c.ptr, a.ptr, b.ptr)
    lib.cgrid_inverse_fft_norm(c.ptr)
    lib.cgrid_extrapolate(d.ptr, c.ptr)
    lib.gb_synchronize()
    for o in (a, b, c, d, r, r2, w):
        api.free(o)


if __name__ == "__main__":
    import sys

    usage = ("usage: python tests/drivers.py gp [n] [steps] [prec: 0 FP64, 1 FP32]\n"
             "       python tests/drivers.py cn [n] [steps]\n"
             "       python tests/drivers.py batch [steps] [prec]\n"
             "       python tests/drivers.py unet [n] [tensor cores: 1 or 0] [reps] [batch]\n"
             "       python tests/drivers.py ops [n]")
    if len(sys.argv) < 2 or sys.argv[1] not in ("gp", "cn", "batch", "unet", "ops"):
        sys.exit(usage)
    a = [int(x) for x in sys.argv[2:]]
    if sys.argv[1] == "gp":
        print("norm", run_gp_steps(*a))
    elif sys.argv[1] == "cn":
        print("norm", run_cn_steps(*a))
    elif sys.argv[1] == "unet":
        run_unet_step(*a)
        print("ok")
    elif sys.argv[1] == "ops":
        run_ops(*a)
        print("ok")
    else:
        run_batch_steps(*a)
        print("ok")
