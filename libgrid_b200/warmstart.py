"""Learned warm start for imaginary-time Gross-Pitaevskii ground states.

The reference relaxes to a ground state with a caller-composed loop:
grid_wf_propagate(wf, V, -i dt) -> grid_wf_normalize -> grid_wf_energy every M
steps (src/grid_wf.c:379-556, 681-700, 215-221), started from a guess the
caller maps in (a Gaussian in examples/).  This module keeps that loop as the
judge and only replaces the guess: a small 3-D convolutional U-Net, run and
trained entirely by this library's own device kernels (gb_unet_* in
csrc/cuda/gb_unet.cu: bf16 weights, FP32 activations and accumulation, Adam on
FP32 master weights), maps the external potential, the coupling g and the
Thomas-Fermi profile to the ground-state amplitude.  Training data are ground
states produced by the plain imaginary-time propagator of this library.

Workload (seeded, reduced from the 128^3 family so that data generation and
training fit a short run): 32^3 grid, step 0.1 bohr, mass 4 amu,
g ~ U(0.001, 0.01), V = k r^2 / 2 with k ~ U(0.005, 0.02) plus 1-6 Gaussian
bumps (amplitude +-U(0.5, 2) mHa, width U(0.2, 0.6) bohr, centre
U(-0.8, 0.8)^3 bohr).  Imaginary time dt = -2i au with renormalisation every
step; converged when |E_n - E_(n-M)| < 1e-8 Ha with M = 10, E the GP energy
functional T + <V> + g/2 int |psi|^4 (FFT kinetic energy).
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import capi, workloads

AMU = capi.GRID_AUTOAMU
C_LEVELS = (8, 16, 32, 64)


# --------------------------------------------------------------- network


def unet_spec(cin: int = 3, ch=C_LEVELS):
    """Ops of the 4-level U-Net: ("conv", sources, out, layer, relu),
    ("pool", sources, out), ("up", sources, out).  A conv with two sources
    reads their channel concatenation (decoder input, then skip)."""
    c0, c1, c2, c3 = ch
    return [
        ("conv", ["in"], "e0a", "e0a", True),
        ("conv", ["e0a"], "e0b", "e0b", True),
        ("pool", ["e0b"], "p1"),
        ("conv", ["p1"], "e1a", "e1a", True),
        ("conv", ["e1a"], "e1b", "e1b", True),
        ("pool", ["e1b"], "p2"),
        ("conv", ["p2"], "e2a", "e2a", True),
        ("conv", ["e2a"], "e2b", "e2b", True),
        ("pool", ["e2b"], "p3"),
        ("conv", ["p3"], "ba", "ba", True),
        ("conv", ["ba"], "bb", "bb", True),
        ("up", ["bb"], "u2"),
        ("conv", ["u2", "e2b"], "d2a", "d2a", True),
        ("conv", ["d2a"], "d2b", "d2b", True),
        ("up", ["d2b"], "u1"),
        ("conv", ["u1", "e1b"], "d1a", "d1a", True),
        ("conv", ["d1a"], "d1b", "d1b", True),
        ("up", ["d1b"], "u0"),
        ("conv", ["u0", "e0b"], "d0a", "d0a", True),
        ("conv", ["d0a"], "d0b", "d0b", True),
        ("conv", ["d0b"], "out", "out", False),
    ], {"in": cin, "e0a": c0, "e0b": c0, "p1": c0, "e1a": c1, "e1b": c1, "p2": c1, "e2a": c2, "e2b": c2,
        "p3": c2, "ba": c3, "bb": c3, "u2": c3, "d2a": c2, "d2b": c2, "u1": c2, "d1a": c1, "d1b": c1,
        "u0": c1, "d0a": c0, "d0b": c0, "out": 1}


_LEVEL = {"in": 0, "e0a": 0, "e0b": 0, "p1": 1, "e1a": 1, "e1b": 1, "p2": 2, "e2a": 2, "e2b": 2, "p3": 3,
          "ba": 3, "bb": 3, "u2": 2, "d2a": 2, "d2b": 2, "u1": 1, "d1a": 1, "d1b": 1, "u0": 0, "d0a": 0,
          "d0b": 0, "out": 0}


def _bind(lib):
    V, I, L, F = C.c_void_p, C.c_int, C.c_long, C.c_float
    sig = {
        "gb_unet_conv3_fwd": [V, V, V, V, I, I, I, I, I, I],
        "gb_unet_conv3_bwd_data": [V, V, V, I, I, I, I, I],
        "gb_unet_conv3_bwd_weight": [V, V, V, V, I, I, I, I, I],
        "gb_unet_relu_bwd": [V, V, L],
        "gb_unet_pool2_fwd": [V, V, I, I, I, I],
        "gb_unet_pool2_bwd": [V, V, I, I, I, I],
        "gb_unet_up2_fwd": [V, V, I, I, I, I],
        "gb_unet_up2_bwd": [V, V, I, I, I, I],
        "gb_unet_mse_grad": [V, V, V, L, F],
        "gb_unet_adam": [V, V, V, V, V, L, F, F, F, F, F, F],
        "gb_unet_to_bf16": [V, V, L],
        "gb_unet_fill": [V, L, F],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.restype = I
        fn.argtypes = args
    lib.gb_device_alloc.restype = V
    lib.gb_device_alloc.argtypes = [C.c_size_t]
    lib.gb_device_free.argtypes = [V]
    lib.gb_device_free.restype = None
    lib.gb_h2d.restype = I
    lib.gb_h2d.argtypes = [V, V, C.c_size_t]
    lib.gb_d2h.restype = I
    lib.gb_d2h.argtypes = [V, V, C.c_size_t]
    lib.gb_d2d.restype = I
    lib.gb_d2d.argtypes = [V, V, C.c_size_t]
    lib.gb_synchronize.restype = I
    lib.rgrid_product.restype = None
    lib.rgrid_product.argtypes = [V, V, V]


def _ok(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed with status %d" % (what, rc))


class DeviceUNet:
    """The U-Net on the device: parameter slabs (FP32 master, bf16 copy,
    Adam moments, gradient), one activation slab and one gradient slab with
    the same offsets.  Everything runs on the library stream."""

    def __init__(self, api, n: int, cin: int = 3, seed: int = 0, ch=C_LEVELS):
        if n % 8:
            raise ValueError("grid extent must be a multiple of 8 (three poolings)")
        self.api, self.lib, self.n = api, api.lib, n
        _bind(self.lib)
        self.spec, self.chan = unet_spec(cin, ch)
        # parameters
        self.layers = {}
        off = 0
        for op in self.spec:
            if op[0] == "conv":
                ci = sum(self.chan[s] for s in op[1])
                co = self.chan[op[2]]
                self.layers[op[3]] = (off, co, ci)
                off += co * ci * 27 + co
        self.nparam = off
        rng = np.random.default_rng(seed)
        p = np.zeros(off, np.float32)
        for name, (o, co, ci) in self.layers.items():
            std = math.sqrt(2.0 / (ci * 27)) * (0.1 if name == "out" else 1.0)
            p[o : o + co * ci * 27] = rng.standard_normal(co * ci * 27) * std
        self._p = self._alloc(4 * off)
        self._pb = self._alloc(2 * off)
        self._m = self._alloc(4 * off)
        self._v = self._alloc(4 * off)
        self._g = self._alloc(4 * off)
        self.set_params(p)
        for b in (self._m, self._v, self._g):
            _ok(self.lib.gb_unet_fill(b, off, 0.0), "fill")
        self.t = 0
        # activations: a conv with two sources reads them as one contiguous block
        self.vol = [(n >> l) ** 3 for l in range(4)]
        place, off = {}, 0
        for op in self.spec:
            if op[0] == "conv" and len(op[1]) == 2:
                a, b = op[1]
                place[a] = off
                place[b] = off + self.chan[a] * self.vol[_LEVEL[a]]
                off += (self.chan[a] + self.chan[b]) * self.vol[_LEVEL[a]]
        for name, c in self.chan.items():
            if name not in place:
                place[name] = off
                off += c * self.vol[_LEVEL[name]]
        self.place, self.nact = place, off
        self._a = self._alloc(4 * off)
        self._ga = self._alloc(4 * off)
        self._tgt = self._alloc(4 * self.vol[0])

    def _alloc(self, nbytes):
        p = self.lib.gb_device_alloc(nbytes)
        if not p:
            raise MemoryError("gb_device_alloc(%d) failed" % nbytes)
        return p

    def free(self):
        for b in (self._p, self._pb, self._m, self._v, self._g, self._a, self._ga, self._tgt):
            self.lib.gb_device_free(b)

    # -- parameters
    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        _ok(self.lib.gb_h2d(self._p, p.ctypes.data, p.nbytes), "h2d")
        _ok(self.lib.gb_unet_to_bf16(self._p, self._pb, self.nparam), "to_bf16")
        _ok(self.lib.gb_synchronize(), "sync")

    def get(self, which: str = "p") -> np.ndarray:
        buf = {"p": self._p, "g": self._g}[which]
        out = np.empty(self.nparam, np.float32)
        _ok(self.lib.gb_d2h(out.ctypes.data, buf, out.nbytes), "d2h")
        _ok(self.lib.gb_synchronize(), "sync")
        return out

    def layer_arrays(self, flat: np.ndarray):
        """{layer: (w [co, ci, 27], b [co])} views of a flat parameter vector."""
        out = {}
        for name, (o, co, ci) in self.layers.items():
            out[name] = (flat[o : o + co * ci * 27].reshape(co, ci, 27), flat[o + co * ci * 27 : o + co * ci * 27 + co])
        return out

    # -- activations
    def _act(self, name, base=None):
        return (self._a if base is None else base) + 4 * self.place[name]

    def set_input(self, x: np.ndarray):
        x = np.ascontiguousarray(x, np.float32)
        assert x.shape == (self.chan["in"], self.n, self.n, self.n)
        _ok(self.lib.gb_h2d(self._act("in"), x.ctypes.data, x.nbytes), "h2d")

    def set_input_device(self, dptr):
        """Input already on the device (cin x n^3 float32)."""
        _ok(self.lib.gb_d2d(self._act("in"), dptr, 4 * self.chan["in"] * self.vol[0]), "d2d")

    def activation(self, name: str) -> np.ndarray:
        lv = _LEVEL[name]
        m = self.n >> lv
        out = np.empty((self.chan[name], m, m, m), np.float32)
        _ok(self.lib.gb_d2h(out.ctypes.data, self._act(name), out.nbytes), "d2h")
        _ok(self.lib.gb_synchronize(), "sync")
        return out

    def forward(self):
        lib = self.lib
        for op in self.spec:
            kind, srcs, out = op[0], op[1], op[2]
            m = self.n >> _LEVEL[srcs[0]]
            cin = sum(self.chan[s] for s in srcs)
            if kind == "conv":
                o, co, ci = self.layers[op[3]]
                _ok(lib.gb_unet_conv3_fwd(self._act(srcs[0]), self._pb + 2 * o, self._p + 4 * (o + co * ci * 27),
                                          self._act(out), ci, co, m, m, m, int(op[4])), "conv3_fwd")
            elif kind == "pool":
                _ok(lib.gb_unet_pool2_fwd(self._act(srcs[0]), self._act(out), cin, m, m, m), "pool2_fwd")
            else:
                _ok(lib.gb_unet_up2_fwd(self._act(srcs[0]), self._act(out), cin, m, m, m), "up2_fwd")

    def backward(self):
        """Accumulate parameter gradients of the loss whose gradient with
        respect to the output is already in the gradient slab."""
        lib = self.lib
        ga = self._ga
        for op in reversed(self.spec):
            kind, srcs, out = op[0], op[1], op[2]
            m = self.n >> _LEVEL[srcs[0]]
            cin = sum(self.chan[s] for s in srcs)
            if kind == "conv":
                o, co, ci = self.layers[op[3]]
                if op[4]:
                    _ok(lib.gb_unet_relu_bwd(self._act(out, ga), self._act(out), co * m ** 3), "relu_bwd")
                _ok(lib.gb_unet_conv3_bwd_weight(self._act(srcs[0]), self._act(out, ga), self._g + 4 * o,
                                                 self._g + 4 * (o + co * ci * 27), ci, co, m, m, m), "bwd_weight")
                if srcs[0] != "in":
                    _ok(lib.gb_unet_conv3_bwd_data(self._act(out, ga), self._pb + 2 * o, self._act(srcs[0], ga),
                                                   ci, co, m, m, m), "bwd_data")
            elif kind == "pool":
                _ok(lib.gb_unet_pool2_bwd(self._act(out, ga), self._act(srcs[0], ga), cin, m, m, m), "pool2_bwd")
            else:
                _ok(lib.gb_unet_up2_bwd(self._act(out, ga), self._act(srcs[0], ga), cin, m, m, m), "up2_bwd")

    def loss_grad(self, tgt_dptr, scale=None):
        n = self.vol[0]
        s = 2.0 / n if scale is None else scale
        _ok(self.lib.gb_unet_mse_grad(self._act("out"), tgt_dptr, self._act("out", self._ga), n, s), "mse_grad")

    def set_target(self, tgt: np.ndarray):
        t = np.ascontiguousarray(tgt, np.float32)
        _ok(self.lib.gb_h2d(self._tgt, t.ctypes.data, t.nbytes), "h2d")
        return self._tgt

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        c1, c2 = 1.0 / (1.0 - b1 ** self.t), 1.0 / (1.0 - b2 ** self.t)
        _ok(self.lib.gb_unet_adam(self._p, self._pb, self._m, self._v, self._g, self.nparam, lr, b1, b2, eps, c1, c2),
            "adam")

    def predict(self, x: np.ndarray) -> np.ndarray:
        self.set_input(x)
        self.forward()
        return self.activation("out")[0]


# --------------------------------------------------------------- physics


def sample_problem(seed: int, n: int = 32, step: float = 0.1):
    """(V, g, k) of one seeded potential of the family above."""
    rng = np.random.default_rng(seed)
    k = rng.uniform(0.005, 0.02)
    g = rng.uniform(0.001, 0.01)
    x, y, z = workloads.mesh(n, n, n, step)
    v = 0.5 * k * (x * x + y * y + z * z)
    for _ in range(int(rng.integers(1, 7))):
        amp = rng.uniform(0.5e-3, 2e-3) * (1 if rng.random() < 0.5 else -1)
        w = rng.uniform(0.2, 0.6)
        c = rng.uniform(-0.8, 0.8, 3)
        v += amp * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / w**2)
    return v, g, k


def thomas_fermi(v, g, step):
    """Normalised Thomas-Fermi amplitude sqrt(max(mu - V, 0) / g).  The norm
    sum_{V_i < mu} (mu - V_i) dv / g is piecewise linear in mu: with the
    potential sorted, the k lowest points give mu_k = (g / dv + S_k) / k, and
    mu is the first mu_k that does not pass the next potential value."""
    dv = step**3
    vs = np.sort(v, axis=None)
    k = np.arange(1, vs.size + 1)
    mus = (g / dv + np.cumsum(vs)) / k
    nxt = np.append(vs[1:], np.inf)
    mu = mus[int(np.argmax(mus <= nxt))]
    return np.sqrt(np.maximum(mu - v, 0) / g)


def features(v, g, step):
    """Network input [3, n, n, n] and the amplitude scale s (targets and
    predictions are amplitudes / s)."""
    tf = thomas_fermi(v, g, step)
    s = float(tf.max())
    x = np.stack([np.tanh((v - v.min()) / 0.01), np.full_like(v, g / 0.01), tf / s]).astype(np.float32)
    return x, s


def gaussian_guess(n, step, width=1.0):
    x, y, z = workloads.mesh(n, n, n, step)
    return np.exp(-(x * x + y * y + z * z) / width**2)


class Relaxer:
    """The plain imaginary-time loop on the device through the libgrid API:
    grid_wf_propagate_gp(-i dt) -> grid_wf_normalize every step, the GP
    energy every M steps."""

    def __init__(self, api, n: int, step: float, mass: float = 4.0 / AMU):
        self.api, self.lib, self.n, self.step = api, api.lib, n, step
        _bind(self.lib)
        self.lib.grid_wf_analyze_method(b"\x01")
        self.w = api.wf(n, n, n, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT)
        self.vx = api.rgrid(n, n, n, step)
        self.rho = api.rgrid(n, n, n, step)
        self.rho2 = api.rgrid(n, n, n, step)

    def free(self):
        for o in (self.w, self.vx, self.rho, self.rho2):
            self.api.free(o)

    def energy(self, g):
        lib = self.lib
        e = self.w.energy(self.vx)
        lib.grid_wf_density(self.w.ptr, self.rho.ptr)
        lib.rgrid_product(C.cast(self.rho2.ptr, C.c_void_p), C.cast(self.rho.ptr, C.c_void_p),
                          C.cast(self.rho.ptr, C.c_void_p))
        return e + 0.5 * g * lib.rgrid_integral(self.rho2.ptr)

    def relax(self, v, g, psi0, dt=2.0, m=10, tol=1e-8, max_steps=20000):
        """Returns (psi, E, steps, seconds); seconds covers the loop only."""
        self.vx.set(v)
        self.w.grid.set(psi0.astype(np.complex128))
        self.w.normalize()
        t0 = time.perf_counter()
        e_prev = self.energy(g)
        steps = 0
        while steps < max_steps:
            for _ in range(m):
                self.w.propagate_gp(self.vx, g, complex(0.0, -dt))
                self.w.normalize()
            steps += m
            e = self.energy(g)
            if abs(e - e_prev) < tol:
                break
            e_prev = e
        secs = time.perf_counter() - t0
        return self.w.grid.get(), e, steps, secs


def make_dataset(api, seeds, n=32, step=0.1, **kw):
    """Ground states of the seeded potentials from a Gaussian start."""
    r = Relaxer(api, n, step)
    xs, ys, meta = [], [], []
    try:
        for sd in seeds:
            v, g, _ = sample_problem(sd, n, step)
            psi, e, steps, secs = r.relax(v, g, gaussian_guess(n, step), **kw)
            x, s = features(v, g, step)
            xs.append(x)
            ys.append((np.abs(psi) / s).astype(np.float32))
            meta.append(dict(seed=sd, g=g, energy=e, steps=steps, seconds=secs, scale=s))
    finally:
        r.free()
    return np.stack(xs), np.stack(ys), meta


def train(net: DeviceUNet, xs, ys, epochs=60, batch=8, lr=2e-3, seed=0, log=None):
    """Adam over minibatches of samples; inputs and targets live on the
    device for the whole run.  Returns the mean loss of the last epoch."""
    lib = net.lib
    nb, vol = xs.shape[0], net.vol[0]
    dx = net._alloc(xs.nbytes)
    dy = net._alloc(ys.nbytes)
    try:
        _ok(lib.gb_h2d(dx, np.ascontiguousarray(xs).ctypes.data, xs.nbytes), "h2d")
        _ok(lib.gb_h2d(dy, np.ascontiguousarray(ys).ctypes.data, ys.nbytes), "h2d")
        rng = np.random.default_rng(seed)
        xbytes = xs[0].nbytes
        last = float("nan")
        for ep in range(epochs):
            order = rng.permutation(nb)
            for b0 in range(0, nb, batch):
                idx = order[b0 : b0 + batch]
                for i in idx:
                    net.set_input_device(dx + int(i) * xbytes)
                    net.forward()
                    net.loss_grad(dy + int(i) * 4 * vol, 2.0 / (vol * len(idx)))
                    net.backward()
                net.adam(lr * (0.5 * (1 + math.cos(math.pi * ep / epochs)) * 0.95 + 0.05))
            if log is not None or ep == epochs - 1:
                errs = []
                for i in range(min(nb, 8)):
                    net.set_input_device(dx + i * xbytes)
                    net.forward()
                    errs.append(float(((net.activation("out")[0] - ys[i]) ** 2).mean()))
                last = float(np.mean(errs))
                if log is not None:
                    log(ep, last)
    finally:
        lib.gb_device_free(dx)
        lib.gb_device_free(dy)
    return last


def evaluate(api, net: DeviceUNet, seeds, n=32, step=0.1):
    """Per held-out potential: steps and seconds to convergence from the
    Gaussian guess, from the Thomas-Fermi profile and from the network guess
    (each including the host time to build its guess; for the network that is
    the features and the inference), and the energy differences."""
    r = Relaxer(api, n, step)
    rows = []
    try:
        for sd in seeds:
            v, g, _ = sample_problem(sd, n, step)
            # each start is charged the time to prepare its guess on the host
            t0 = time.perf_counter()
            guess = gaussian_guess(n, step)
            t_g0 = time.perf_counter() - t0
            _, e_g, st_g, t_g = r.relax(v, g, guess)
            t0 = time.perf_counter()
            x, s = features(v, g, step)
            guess = x[2] * s
            t_tf0 = time.perf_counter() - t0
            _, e_tf, st_tf, t_tf = r.relax(v, g, guess)
            t0 = time.perf_counter()
            x, s = features(v, g, step)
            amp = np.maximum(net.predict(x), 0.0) * s + 1e-6
            t_inf = time.perf_counter() - t0
            _, e_n, st_n, t_n = r.relax(v, g, amp)
            t_g += t_g0
            t_tf += t_tf0
            rows.append(dict(seed=sd, steps_gauss=st_g, sec_gauss=t_g, steps_tf=st_tf, sec_tf=t_tf, steps_net=st_n,
                             sec_net=t_n + t_inf, e_gauss=e_g, e_net=e_n, de=abs(e_n - e_g)))
    finally:
        r.free()
    return rows


def time_training_step(net: DeviceUNet, x, y, reps: int = 20):
    """(forward ms, forward + loss + backward ms) per sample, CUDA events on
    the library stream, after 3 warm-up repetitions."""
    lib = net.lib
    lib.gb_event_record.restype = C.c_int
    lib.gb_event_record.argtypes = [C.c_int]
    lib.gb_event_elapsed_ms.restype = C.c_float
    lib.gb_event_elapsed_ms.argtypes = [C.c_int, C.c_int]
    net.set_input(x)
    tgt = net.set_target(y)
    out = []
    for with_bwd in (False, True):
        for r in range(reps + 3):
            if r == 3:
                _ok(lib.gb_event_record(0), "event")
            net.forward()
            if with_bwd:
                net.loss_grad(tgt)
                net.backward()
        _ok(lib.gb_event_record(1), "event")
        _ok(lib.gb_synchronize(), "sync")
        out.append(lib.gb_event_elapsed_ms(0, 1) / reps)
    _ok(lib.gb_unet_fill(net._g, net.nparam, 0.0), "fill")  # drop the timing runs' gradients
    return out


def main(argv=None):
    """python -m libgrid_b200.warmstart [--train N] [--test N] [--epochs E]
    [--out report.json]: generate, train, evaluate and print one JSON report."""
    import argparse
    import json

    import libgrid_b200

    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=128)
    ap.add_argument("--test", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=100)
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--step", type=float, default=0.1)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    api = libgrid_b200.load()
    api.lib.cuda_enable(b"\x01", 0, None)
    t0 = time.perf_counter()
    xs, ys, meta = make_dataset(api, range(1000, 1000 + a.train), a.n, a.step)
    t_data = time.perf_counter() - t0
    net = DeviceUNet(api, a.n, cin=3, seed=0)
    try:
        t0 = time.perf_counter()
        loss = train(net, xs, ys, epochs=a.epochs, batch=8, lr=2e-3)
        t_train = time.perf_counter() - t0
        step_ms = time_training_step(net, xs[0], ys[0])
        rows = evaluate(api, net, range(5000, 5000 + a.test), a.n, a.step)
    finally:
        net.free()
    mean = lambda k: float(np.mean([r[k] for r in rows]))
    rep = dict(
        workload="learned warm start, GP imaginary time %d^3 step %.2f, %d training / %d held-out potentials"
        % (a.n, a.step, a.train, a.test),
        params=int(net.nparam), epochs=a.epochs, train_loss=loss, target_ms=float((ys**2).mean()),
        data_seconds=t_data, train_seconds=t_train, forward_ms=step_ms[0], forward_backward_ms=step_ms[1],
        steps_gauss=mean("steps_gauss"), steps_tf=mean("steps_tf"), steps_net=mean("steps_net"),
        sec_gauss=mean("sec_gauss"), sec_tf=mean("sec_tf"), sec_net=mean("sec_net"),
        step_ratio=mean("steps_gauss") / mean("steps_net"), time_ratio=mean("sec_gauss") / mean("sec_net"),
        max_de=float(max(r["de"] for r in rows)), rows=rows,
    )
    line = json.dumps(rep)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")
    print(line)


if __name__ == "__main__":
    main()
