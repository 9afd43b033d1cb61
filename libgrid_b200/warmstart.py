"""Learned warm start for imaginary-time Gross-Pitaevskii ground states.

The reference relaxes to a ground state with a caller-composed loop:
grid_wf_propagate(wf, V, -i dt) -> grid_wf_normalize -> grid_wf_energy every M
steps (src/grid_wf.c:379-556, 681-700, 215-221), started from a guess the
caller maps in (a Gaussian in examples/).  This module keeps that loop as the
arbiter of convergence and only replaces the guess: a small 3-D convolutional U-Net, run and
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
import sys
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
        "gb_unet_conv3_fwd_nb": [V, V, V, V, I, I, I, I, I, I, I],
        "gb_unet_conv3_bwd_data_nb": [V, V, V, I, I, I, I, I, I],
        "gb_unet_conv3_bwd_weight_nb": [V, V, V, V, I, I, I, I, I, I],
        "gb_unet_relu_bwd": [V, V, L],
        "gb_unet_pool2_fwd": [V, V, I, I, I, I],
        "gb_unet_pool2_bwd": [V, V, I, I, I, I],
        "gb_unet_up2_fwd": [V, V, I, I, I, I],
        "gb_unet_up2_bwd": [V, V, I, I, I, I],
        "gb_unet_mse_grad": [V, V, V, L, F],
        "gb_unet_adam": [V, V, V, V, V, L, F, F, F, F, F, F],
        "gb_unet_to_bf16": [V, V, L],
        "gb_unet_fill": [V, L, F],
        "gb_unet_gather": [V, V, V, V, C.POINTER(C.c_int), I, I, L, I, L],
        "gb_unet_tensor_cores": [I],
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
    lib.gb_graph_begin.restype = I
    lib.gb_graph_begin.argtypes = []
    lib.gb_graph_end.restype = I
    lib.gb_graph_end.argtypes = [C.POINTER(V)]
    lib.gb_graph_launch.restype = I
    lib.gb_graph_launch.argtypes = [V]
    lib.gb_graph_free.restype = I
    lib.gb_graph_free.argtypes = [V]
    lib.rgrid_product.restype = None
    lib.rgrid_product.argtypes = [V, V, V]


def _ok(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed with status %d" % (what, rc))


class DeviceUNet:
    """The U-Net on the device: parameter slabs (FP32 master, bf16 copy,
    Adam moments, gradient), one activation slab and one gradient slab with
    the same offsets.  With batch = nb > 1 every activation holds nb samples
    stacked along the depth axis ([C][nb n][n][n]) and each layer is one
    launch over all of them (gb_unet_conv3_*_nb), which fills the GPU on the
    coarse levels.  Everything runs on the library stream."""

    def __init__(self, api, n: int, cin: int = 3, seed: int = 0, ch=C_LEVELS, batch: int = 1):
        if n % 8:
            raise ValueError("grid extent must be a multiple of 8 (three poolings)")
        if batch < 1:
            raise ValueError("batch must be at least 1")
        self.api, self.lib, self.n, self.nb = api, api.lib, n, batch
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
        self._graphs = {}
        # activations: a conv with two sources reads them as one contiguous
        # block; every channel holds nb samples
        self.vol = [(n >> l) ** 3 for l in range(4)]
        nb = self.nb
        place, off = {}, 0
        for op in self.spec:
            if op[0] == "conv" and len(op[1]) == 2:
                a, b = op[1]
                place[a] = off
                place[b] = off + self.chan[a] * self.vol[_LEVEL[a]] * nb
                off += (self.chan[a] + self.chan[b]) * self.vol[_LEVEL[a]] * nb
        for name, c in self.chan.items():
            if name not in place:
                place[name] = off
                off += c * self.vol[_LEVEL[name]] * nb
        self.place, self.nact = place, off
        self._a = self._alloc(4 * off)
        self._ga = self._alloc(4 * off)
        self._tgt = self._alloc(4 * self.vol[0] * nb)

    def _alloc(self, nbytes):
        p = self.lib.gb_device_alloc(nbytes)
        if not p:
            raise MemoryError("gb_device_alloc(%d) failed" % nbytes)
        return p

    def free(self):
        for h in self.__dict__.get("_graphs", {}).values():
            self.lib.gb_graph_free(h)
        self._graphs = {}
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
        assert self.nb == 1 and x.shape == (self.chan["in"], self.n, self.n, self.n)
        _ok(self.lib.gb_h2d(self._act("in"), x.ctypes.data, x.nbytes), "h2d")

    def set_input_device(self, dptr):
        """Input already on the device (cin x n^3 float32), into sample 0."""
        self.load_slot(0, dptr)

    def load_slot(self, b, x_dptr, y_dptr=None):
        """Copy one sample's input (cin x n^3) and optionally its target
        (n^3), both in device memory, into batch slot b."""
        v, nb = self.vol[0], self.nb
        base = self._act("in")
        for c in range(self.chan["in"]):
            _ok(self.lib.gb_d2d(base + 4 * (c * nb + b) * v, x_dptr + 4 * c * v, 4 * v), "d2d")
        if y_dptr is not None:
            _ok(self.lib.gb_d2d(self._tgt + 4 * b * v, y_dptr, 4 * v), "d2d")

    def activation(self, name: str) -> np.ndarray:
        """An activation, [C][m][m][m] (batch 1) or [C][nb][m][m][m]."""
        lv = _LEVEL[name]
        m = self.n >> lv
        shape = (self.chan[name], m, m, m) if self.nb == 1 else (self.chan[name], self.nb, m, m, m)
        out = np.empty(shape, np.float32)
        _ok(self.lib.gb_d2h(out.ctypes.data, self._act(name), out.nbytes), "d2h")
        _ok(self.lib.gb_synchronize(), "sync")
        return out

    def forward(self):
        lib, nb = self.lib, self.nb
        for op in self.spec:
            kind, srcs, out = op[0], op[1], op[2]
            m = self.n >> _LEVEL[srcs[0]]
            cin = sum(self.chan[s] for s in srcs)
            if kind == "conv":
                o, co, ci = self.layers[op[3]]
                _ok(lib.gb_unet_conv3_fwd_nb(self._act(srcs[0]), self._pb + 2 * o, self._p + 4 * (o + co * ci * 27),
                                             self._act(out), ci, co, nb, m, m, m, int(op[4])), "conv3_fwd")
            elif kind == "pool":
                _ok(lib.gb_unet_pool2_fwd(self._act(srcs[0]), self._act(out), cin, nb * m, m, m), "pool2_fwd")
            else:
                _ok(lib.gb_unet_up2_fwd(self._act(srcs[0]), self._act(out), cin, nb * m, m, m), "up2_fwd")

    def backward(self):
        """Accumulate parameter gradients of the loss whose gradient with
        respect to the output is already in the gradient slab."""
        lib, nb = self.lib, self.nb
        ga = self._ga
        for op in reversed(self.spec):
            kind, srcs, out = op[0], op[1], op[2]
            m = self.n >> _LEVEL[srcs[0]]
            cin = sum(self.chan[s] for s in srcs)
            if kind == "conv":
                o, co, ci = self.layers[op[3]]
                if op[4]:
                    _ok(lib.gb_unet_relu_bwd(self._act(out, ga), self._act(out), co * nb * m ** 3), "relu_bwd")
                _ok(lib.gb_unet_conv3_bwd_weight_nb(self._act(srcs[0]), self._act(out, ga), self._g + 4 * o,
                                                    self._g + 4 * (o + co * ci * 27), ci, co, nb, m, m, m),
                    "bwd_weight")
                if srcs[0] != "in":
                    _ok(lib.gb_unet_conv3_bwd_data_nb(self._act(out, ga), self._pb + 2 * o, self._act(srcs[0], ga),
                                                      ci, co, nb, m, m, m), "bwd_data")
            elif kind == "pool":
                _ok(lib.gb_unet_pool2_bwd(self._act(out, ga), self._act(srcs[0], ga), cin, nb * m, m, m), "pool2_bwd")
            else:
                _ok(lib.gb_unet_up2_bwd(self._act(out, ga), self._act(srcs[0], ga), cin, nb * m, m, m), "up2_bwd")

    def loss_grad(self, tgt_dptr, scale=None, count=None):
        """Output gradient of the MSE loss for the first `count` samples
        (default all nb) against targets at tgt_dptr ([count][n^3]); the
        other slots get a zero gradient, so they add nothing."""
        v, nb = self.vol[0], self.nb
        count = nb if count is None else count
        s = 2.0 / v if scale is None else scale
        _ok(self.lib.gb_unet_mse_grad(self._act("out"), tgt_dptr, self._act("out", self._ga), count * v, s), "mse_grad")
        if count < nb:
            _ok(self.lib.gb_unet_fill(self._act("out", self._ga) + 4 * count * v, (nb - count) * v, 0.0), "fill")

    def set_target(self, tgt: np.ndarray):
        t = np.ascontiguousarray(tgt, np.float32)
        _ok(self.lib.gb_h2d(self._tgt, t.ctypes.data, t.nbytes), "h2d")
        return self._tgt

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        c1, c2 = 1.0 / (1.0 - b1 ** self.t), 1.0 / (1.0 - b2 ** self.t)
        _ok(self.lib.gb_unet_adam(self._p, self._pb, self._m, self._v, self._g, self.nparam, lr, b1, b2, eps, c1, c2),
            "adam")

    def _graph(self, key, build):
        """The CUDA graph of the calls `build` makes, captured on first use
        (after one uncaptured run that sizes the library's scratch buffers)
        and cached under key."""
        g = self._graphs.get(key)
        if g is None:
            build()
            _ok(self.lib.gb_synchronize(), "sync")
            _ok(self.lib.gb_graph_begin(), "graph begin")
            try:
                build()
            finally:
                h = C.c_void_p()
                rc = self.lib.gb_graph_end(C.byref(h))
            _ok(rc, "graph end")
            g = self._graphs[key] = h
        return g

    def train_sample(self, x_dptr, y_dptr, scale):
        """Forward, MSE gradient (times scale) and backward of one sample
        whose input and target sit in device memory (batch-1 network): two
        device copies into the network's input and target slots, then one
        graph launch (the captured forward, loss gradient and backward;
        weight gradients accumulate)."""
        self.train_batch([x_dptr], [y_dptr], scale)

    def train_batch(self, x_dptrs, y_dptrs, scale):
        """The same for up to nb samples at once: each sample is copied into
        its batch slot, then one graph launch runs forward, loss gradient and
        backward over the batch (slots past the given samples get a zero
        output gradient)."""
        count = len(x_dptrs)
        if not 1 <= count <= self.nb:
            raise ValueError("train_batch: %d samples for a batch of %d" % (count, self.nb))
        g = self._graphs.get(("train", float(scale), count))
        if g is None:
            raise RuntimeError("train_batch: no graph for loss scale %r and %d samples (call prepare_training first)"
                               % (scale, count))
        for b, (xp, yp) in enumerate(zip(x_dptrs, y_dptrs)):
            self.load_slot(b, xp, yp)
        _ok(self.lib.gb_graph_launch(g), "graph launch")

    def train_set_batch(self, ds, idx, scale):
        """train_batch for samples idx of a device-resident set (DeviceSet):
        one gather launch fills the batch slots (inputs and targets), then
        one graph launch runs forward, loss gradient and backward."""
        count = len(idx)
        if not 1 <= count <= self.nb:
            raise ValueError("train_set_batch: %d samples for a batch of %d" % (count, self.nb))
        g = self._graphs.get(("train", float(scale), count))
        if g is None:
            raise RuntimeError("train_set_batch: no graph for loss scale %r and %d samples (call prepare_training "
                               "first)" % (scale, count))
        ix = (C.c_int * count)(*[int(i) for i in idx])
        _ok(self.lib.gb_unet_gather(self._act("in"), self._tgt, ds.x, ds.y, ix, count, self.chan["in"], self.vol[0],
                                    self.nb, ds.count), "gather")
        _ok(self.lib.gb_graph_launch(g), "graph launch")

    def prepare_training(self, scales, counts=None):
        """Capture the training graphs of the given loss scales (and batch
        fills, default a full batch) before the first sample; their sizing
        runs' gradients are cleared."""
        counts = [self.nb] * len(scales) if counts is None else counts
        for sc, cnt in zip(scales, counts):
            def build(sc=sc, cnt=cnt):
                self.forward()
                self.loss_grad(self._tgt, sc, cnt)
                self.backward()

            self._graph(("train", float(sc), int(cnt)), build)
        _ok(self.lib.gb_unet_fill(self._g, self.nparam, 0.0), "fill")

    def clone(self, batch: int = 1):
        """A network of the same shape and parameters with another batch
        size (e.g. batch 1 for inference after batched training)."""
        other = DeviceUNet(self.api, self.n, cin=self.chan["in"], seed=0, batch=batch)
        _ok(self.lib.gb_d2d(other._p, self._p, 4 * self.nparam), "d2d")
        _ok(self.lib.gb_d2d(other._pb, self._pb, 2 * self.nparam), "d2d")
        return other

    def forward_graph(self):
        """Forward of the input already in the activation slab, as one
        graph launch."""
        _ok(self.lib.gb_graph_launch(self._graph(("fwd",), self.forward)), "graph launch")

    def infer_device(self, x_dptr):
        """Forward of one device-resident input in batch slot 0 (a graph
        launch); the output stays in the activation slab ("out")."""
        self.load_slot(0, x_dptr)
        _ok(self.lib.gb_graph_launch(self._graph(("fwd",), self.forward)), "graph launch")

    def predict(self, x: np.ndarray) -> np.ndarray:
        self.set_input(x)
        self.forward()
        return self.activation("out")[0]


# --------------------------------------------------------------- physics


def problem_params(seed: int):
    """(k, g, bumps) of one seeded potential of the family above; bumps is a
    list of (amplitude, width, centre[3])."""
    rng = np.random.default_rng(seed)
    k = rng.uniform(0.005, 0.02)
    g = rng.uniform(0.001, 0.01)
    bumps = []
    for _ in range(int(rng.integers(1, 7))):
        amp = rng.uniform(0.5e-3, 2e-3) * (1 if rng.random() < 0.5 else -1)
        w = rng.uniform(0.2, 0.6)
        c = rng.uniform(-0.8, 0.8, 3)
        bumps.append((amp, w, c))
    return k, g, bumps


def sample_problem(seed: int, n: int = 32, step: float = 0.1):
    """(V, g, k) of one seeded potential on the host (the definition the
    device potential kernel follows)."""
    k, g, bumps = problem_params(seed)
    x, y, z = workloads.mesh(n, n, n, step)
    v = 0.5 * k * (x * x + y * y + z * z)
    for amp, w, c in bumps:
        v += amp * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / w**2)
    return v, g, k


def thomas_fermi_mu(v, g, step):
    """Chemical potential of the normalised Thomas-Fermi profile: the norm
    sum_{V_i < mu} (mu - V_i) dv / g is piecewise linear in mu; with the
    potential sorted, the k lowest points give mu_k = (g / dv + S_k) / k, and
    mu is the first mu_k that does not pass the next potential value."""
    dv = step**3
    vs = np.sort(v, axis=None)
    k = np.arange(1, vs.size + 1)
    mus = (g / dv + np.cumsum(vs)) / k
    nxt = np.append(vs[1:], np.inf)
    return float(mus[int(np.argmax(mus <= nxt))])


def thomas_fermi(v, g, step):
    """Normalised Thomas-Fermi amplitude sqrt(max(mu - V, 0) / g)."""
    return np.sqrt(np.maximum(thomas_fermi_mu(v, g, step) - v, 0) / g)


def features(v, g, step):
    """Network input [3, n, n, n] and the amplitude scale s (targets and
    predictions are amplitudes / s) on the host (the definition the device
    features kernel follows)."""
    tf = thomas_fermi(v, g, step)
    s = float(tf.max())
    x = np.stack([np.tanh((v - v.min()) / 0.01), np.full_like(v, g / 0.01), tf / s]).astype(np.float32)
    return x, s


def gaussian_guess(n, step, width=1.0):
    x, y, z = workloads.mesh(n, n, n, step)
    return np.exp(-(x * x + y * y + z * z) / width**2)


class Bumps(C.Structure):
    _fields_ = [("n", C.c_int), ("amp", C.c_double * 8), ("w", C.c_double * 8), ("c", (C.c_double * 3) * 8)]


def _bind_device(lib):
    V, I, L, D, F = C.c_void_p, C.c_int, C.c_long, C.c_double, C.c_float
    sig = {
        "gb_unet_potential": (I, [V, I, I, I, L, D, D, C.POINTER(Bumps)]),
        "gb_unet_features": (I, [V, I, I, I, L, D, D, F, D, D, D, V]),
        "gb_unet_gaussian": (I, [V, I, I, I, D, D]),
        "gb_unet_abs": (I, [V, I, L, F, V]),
        "gb_tf_stats": (I, [V, V, L, D, C.POINTER(D)]),
        "gb_grid_device": (V, [V, I]),
        "grid_wf_set_amplitude_device": (None, [V, V, D, D]),
        "grid_wf_relax_gp_n": (None, [V, V, D, capi.Complex, L]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


class Geom(C.Structure):
    _fields_ = [("nx", C.c_long), ("ny", C.c_long), ("nz", C.c_long), ("step", C.c_double), ("prec", C.c_int)]


def converged(a, a_prev, tol, rule="remainder"):
    """One check of the imaginary-time stopping rule on the decrement
    a = E_(k-1) - E_k over the last m steps (a_prev: the previous positive
    decrement or None).  Returns (stop, a_prev for the next check).  "change":
    |a| < tol.  "remainder": the energy falls geometrically, so the distance
    left to the limit is about a q / (1 - q) with q = a / a_prev; stop when
    it and a are below tol / 2, or when the energy stops moving (|a| below
    1e-3 tol)."""
    if rule == "change":
        return abs(a) < tol, a_prev
    if abs(a) < 1e-3 * tol:
        return True, a_prev
    if a_prev is not None and 0.0 < a < a_prev:
        q = a / a_prev
        if a < 0.5 * tol and a * q / (1.0 - q) < 0.5 * tol:
            return True, a_prev
    return False, (a if a > 0.0 else None)


class Relaxer:
    """The plain imaginary-time loop on the device through the libgrid API:
    grid_wf_propagate_gp(-i dt) and a renormalisation every step
    (grid_wf_relax_gp_n: the norm is reduced and applied on the device), the
    GP energy E = T (FFT) + <V> + g/2 int |psi|^4 every M steps.  The
    potential, the Thomas-Fermi features and every initial guess are built on
    the device too, so a relaxation moves no 3-D array across PCIe."""

    def __init__(self, api, n: int, step: float, mass: float = 4.0 / AMU):
        self.api, self.lib, self.n, self.step = api, api.lib, n, step
        _bind(self.lib)
        _bind_device(self.lib)
        self.lib.grid_wf_analyze_method(b"\x01")
        self.w = api.wf(n, n, n, step, mass, capi.WF_PERIODIC_BOUNDARY, capi.WF_2ND_ORDER_FFT)
        self.vx = api.rgrid(n, n, n, step)
        self.rho = api.rgrid(n, n, n, step)
        self.rho2 = api.rgrid(n, n, n, step)
        self.vol = n**3
        self.work = self.lib.gb_device_alloc(4 * self.vol)
        self.feat = self.lib.gb_device_alloc(4 * 3 * self.vol)
        if not self.work or not self.feat:
            raise MemoryError("gb_device_alloc failed")
        self.g = 0.0

    def free(self):
        for o in (self.w, self.vx, self.rho, self.rho2):
            self.api.free(o)
        self.lib.gb_device_free(self.work)
        self.lib.gb_device_free(self.feat)

    def _vdev(self, mode=0):
        return self.lib.gb_grid_device(C.c_void_p(self.vx.s.value), mode)

    def set_problem(self, seed):
        """The seeded potential on the device; returns g."""
        k, g, bumps = problem_params(seed)
        b = Bumps()
        b.n = len(bumps)
        for i, (amp, w, c) in enumerate(bumps):
            b.amp[i], b.w[i] = amp, w
            for j in range(3):
                b.c[i][j] = c[j]
        n = self.n
        _ok(self.lib.gb_unet_potential(self._vdev(1), n, n, n, self.vx.s.nz2, self.step, k, C.byref(b)), "potential")
        self.g = g
        return g

    def tf_features(self, out=None):
        """Thomas-Fermi chemical potential by Newton's method on the device
        sums (sum max(0, mu - V) is convex and piecewise linear in mu, so
        Newton from above ends on the exact root), then the network input
        [3][n^3] into `out` (default: the relaxer's own buffer).  Returns
        (out, amplitude scale s)."""
        lib, n, g = self.lib, self.n, self.g
        geo = Geom(n, n, n, self.step, 0)
        st = (C.c_double * 4)()
        vd = self._vdev(0)
        target = g / self.step**3
        _ok(lib.gb_tf_stats(vd, C.byref(geo), self.vx.s.nz2, -1e300, st), "tf stats")
        vmin, vsum = st[2], st[3]
        mu = (target + vsum) / self.vol  # at or above the root
        for _ in range(64):
            _ok(lib.gb_tf_stats(vd, C.byref(geo), self.vx.s.nz2, mu, st), "tf stats")
            f, cnt = st[0], st[1]
            if cnt <= 0:
                break
            nmu = mu - (f - target) / cnt
            if not (nmu < mu) or abs(f - target) <= 1e-13 * target:
                break
            mu = nmu
        s = math.sqrt(max(mu - vmin, 0.0) / g)
        out = self.feat if out is None else out
        _ok(lib.gb_unet_features(vd, n, n, n, self.vx.s.nz2, vmin, 0.01, g / 0.01, mu, g, s, out), "features")
        return out, s

    def set_guess(self, amp_dev, scale, floor=0.0):
        self.lib.grid_wf_set_amplitude_device(self.w.ptr, amp_dev, scale, floor)
        self.w.normalize()

    def gaussian(self, width=1.0):
        n = self.n
        _ok(self.lib.gb_unet_gaussian(self.work, n, n, n, self.step, width), "gaussian")
        self.set_guess(self.work, 1.0)

    def energy(self):
        lib, g = self.lib, self.g
        e = self.w.energy(self.vx)
        lib.grid_wf_density(self.w.ptr, self.rho.ptr)
        lib.rgrid_product(C.cast(self.rho2.ptr, C.c_void_p), C.cast(self.rho.ptr, C.c_void_p),
                          C.cast(self.rho.ptr, C.c_void_p))
        return e + 0.5 * g * lib.rgrid_integral(self.rho2.ptr)

    def relax(self, dt=2.0, m=10, tol=1e-8, max_steps=50000, rule="remainder"):
        """From the guess in place: returns (E, steps).  The energy is read
        every m steps.  rule "change": stop when it changed by less than tol
        over m steps.  rule "remainder" (default): imaginary time lowers the
        energy geometrically, E_k - E_inf ~ c q^k, so with the decrements
        a_k = E_(k-1) - E_k over m steps the remaining distance to the limit
        is about a_k q / (1 - q), q = a_k / a_(k-1); stop when that estimate
        and a_k are below tol / 2 (or the energy stops moving), so that a
        converged energy lies within about tol of the limit.  self.trace
        holds (steps, energy, perf_counter time) of every energy read."""
        e_prev = self.energy()
        self.trace = [(0, e_prev, time.perf_counter())]
        a_prev = None
        steps = 0
        while steps < max_steps:
            self.lib.grid_wf_relax_gp_n(self.w.ptr, self.vx.ptr, self.g, capi.Complex.of(complex(0.0, -dt)), m)
            steps += m
            e = self.energy()
            self.trace.append((steps, e, time.perf_counter()))
            a = e_prev - e
            stop, a_prev = converged(a, a_prev, tol, rule)
            if stop:
                break
            e_prev = e
        return e, steps

    def target(self, out, s):
        """|psi| / s of the relaxed state into a device float array."""
        _ok(self.lib.gb_unet_abs(self.lib.gb_grid_device(C.c_void_p(self.w.s.grid.contents.value), 0), 0, self.vol,
                                 1.0 / s, out), "abs")


class DeviceSet:
    """Inputs [N][3][n^3] and targets [N][n^3] of a training set, resident on
    the device."""

    def __init__(self, lib, count, vol):
        self.lib, self.count, self.vol = lib, count, vol
        self.x = lib.gb_device_alloc(4 * 3 * vol * count)
        self.y = lib.gb_device_alloc(4 * vol * count)
        if not self.x or not self.y:
            raise MemoryError("training set does not fit the device")

    def xp(self, i):
        return self.x + 4 * 3 * self.vol * int(i)

    def yp(self, i):
        return self.y + 4 * self.vol * int(i)

    def free(self):
        self.lib.gb_device_free(self.x)
        self.lib.gb_device_free(self.y)


def make_dataset(api, seeds, n=32, step=0.1, tol=1e-8):
    """Ground states of the seeded potentials, relaxed by the plain
    imaginary-time loop from the Thomas-Fermi profile; features and targets
    (the ground-state amplitude in units of the Thomas-Fermi maximum) stay on
    the device.  Returns (DeviceSet, meta)."""
    seeds = list(seeds)
    r = Relaxer(api, n, step)
    ds = DeviceSet(r.lib, len(seeds), n**3)
    meta = []
    try:
        for i, sd in enumerate(seeds):
            g = r.set_problem(sd)
            _, s = r.tf_features(ds.xp(i))
            r.set_guess(ds.xp(i) + 4 * 2 * r.vol, s)
            e, steps = r.relax(tol=tol)
            r.target(ds.yp(i), s)
            meta.append(dict(seed=sd, g=g, energy=e, steps=steps, scale=s))
        _ok(r.lib.gb_synchronize(), "sync")
    finally:
        r.free()
    return ds, meta


def host_dataset(api, xs, ys):
    """A DeviceSet from host arrays (tests)."""
    _bind(api.lib)
    ds = DeviceSet(api.lib, xs.shape[0], int(np.prod(ys.shape[1:])))
    _ok(api.lib.gb_h2d(ds.x, np.ascontiguousarray(xs, np.float32).ctypes.data, xs.nbytes), "h2d")
    _ok(api.lib.gb_h2d(ds.y, np.ascontiguousarray(ys, np.float32).ctypes.data, ys.nbytes), "h2d")
    return ds


def train(net: DeviceUNet, ds: DeviceSet, epochs=60, batch=8, lr=2e-3, seed=0, log=None, monitor=8):
    """Adam over minibatches of samples of a device-resident set: a batch-nb
    network takes each minibatch (of nb samples) in one graph launch, a
    batch-1 network one sample per launch.  Returns the mean squared error
    on the first `monitor` samples after the last epoch."""
    nb, vol = ds.count, net.vol[0]
    rng = np.random.default_rng(seed)
    last = float("nan")
    if net.nb > 1:
        batch = net.nb  # a batched network takes whole minibatches per launch
    # one captured graph (forward, loss gradient, backward) per minibatch
    # length: the full batch and the remainder
    lens = sorted({min(batch, nb - b0) for b0 in range(0, nb, batch)})
    if net.nb > 1:
        net.prepare_training([2.0 / (vol * L) for L in lens], lens)
    else:
        net.prepare_training([2.0 / (vol * L) for L in lens])
    # learning rate: linear warm-up over the first epoch's minibatches (from
    # a tenth), then a cosine decay to 5% by epoch
    warm = max(1, (nb + batch - 1) // batch)
    step = 0
    for ep in range(epochs):
        order = rng.permutation(nb)
        for b0 in range(0, nb, batch):
            idx = order[b0 : b0 + batch]
            if net.nb > 1:
                net.train_set_batch(ds, idx, 2.0 / (vol * len(idx)))
            else:
                for i in idx:
                    net.train_sample(ds.xp(i), ds.yp(i), 2.0 / (vol * len(idx)))
            ramp = min(1.0, 0.1 + 0.9 * step / warm)
            net.adam(lr * ramp * (0.5 * (1 + math.cos(math.pi * ep / epochs)) * 0.95 + 0.05))
            step += 1
        if log is not None or ep == epochs - 1:
            errs = []
            for i in range(min(nb, monitor)):
                net.infer_device(ds.xp(i))
                y = np.empty(vol, np.float32)
                _ok(net.lib.gb_d2h(y.ctypes.data, ds.yp(i), y.nbytes), "d2h")
                errs.append(float(((net.activation("out")[0].reshape(net.nb, -1)[0] - y) ** 2).mean()))
            last = float(np.mean(errs))
            if log is not None:
                log(ep, last)
    return last


def evaluate(api, net: DeviceUNet, seeds, n=32, step=0.1, tol=1e-8, ref_tol=1e-12):
    """Per held-out potential: steps and seconds to convergence from the
    Gaussian guess, from the Thomas-Fermi profile and from the network guess,
    and (*_1e8) the steps and seconds until the energy first lies within
    1e-8 Ha of the tightly converged limit (read every 10 steps).
    Each start's seconds run from the potential on the device to the
    converged state and include building its guess (for the network: the
    Thomas-Fermi features and the inference).  The converged energies are
    compared with each other and with a reference relaxed to ref_tol."""
    if net.nb != 1:
        raise ValueError("evaluate: the inference network must have batch 1 (use net.clone(1))")
    r = Relaxer(api, n, step)
    lib = r.lib
    rows = []
    try:
        for sd in seeds:
            r.set_problem(sd)
            _ok(lib.gb_synchronize(), "sync")
            t0 = time.perf_counter()
            r.gaussian()
            e_g, st_g = r.relax(tol=tol)
            _ok(lib.gb_synchronize(), "sync")
            t_g = time.perf_counter() - t0
            tr_g = [(k, e, t - t0) for k, e, t in r.trace]
            t0 = time.perf_counter()
            _, s = r.tf_features()
            r.set_guess(r.feat + 4 * 2 * r.vol, s)
            e_tf, st_tf = r.relax(tol=tol)
            _ok(lib.gb_synchronize(), "sync")
            t_tf = time.perf_counter() - t0
            t0 = time.perf_counter()
            _, s = r.tf_features(net._act("in"))
            net.forward_graph()
            r.set_guess(net._act("out"), s, 1e-6)
            e_n, st_n = r.relax(tol=tol)
            _ok(lib.gb_synchronize(), "sync")
            t_n = time.perf_counter() - t0
            tr_n = [(k, e, t - t0) for k, e, t in r.trace]
            e_ref, st_ref = r.relax(tol=ref_tol, rule="change")  # continue to a far tighter limit

            def reach(tr):
                # first energy read within 1e-8 Ha of the tightly converged limit
                for k, e, t in tr:
                    if abs(e - e_ref) < 1e-8:
                        return k, t
                return tr[-1][0], tr[-1][2]

            (k_g, s_g), (k_n, s_n) = reach(tr_g), reach(tr_n)
            rows.append(dict(seed=sd, steps_gauss=st_g, sec_gauss=t_g, steps_tf=st_tf, sec_tf=t_tf, steps_net=st_n,
                             sec_net=t_n, e_gauss=e_g, e_net=e_n, e_ref=e_ref, de=abs(e_n - e_g),
                             de_net_ref=abs(e_n - e_ref), de_gauss_ref=abs(e_g - e_ref),
                             steps_gauss_1e8=k_g, sec_gauss_1e8=s_g, steps_net_1e8=k_n, sec_net_1e8=s_n))
    finally:
        r.free()
    return rows


def time_training_step(net: DeviceUNet, ds: DeviceSet, reps: int = 10):
    """(forward ms, forward + loss + backward ms) per sample as training and
    inference run them (captured graphs replayed on the library stream; a
    batched network runs nb samples per launch and the time is divided by
    nb), CUDA events after 3 warm-up repetitions."""
    lib = net.lib
    lib.gb_event_record.restype = C.c_int
    lib.gb_event_record.argtypes = [C.c_int]
    lib.gb_event_elapsed_ms.restype = C.c_float
    lib.gb_event_elapsed_ms.argtypes = [C.c_int, C.c_int]
    nb, v = net.nb, net.vol[0]
    net.prepare_training([2.0 / (v * nb)], [nb])
    xs, ys = [ds.xp(0)] * nb, [ds.yp(0)] * nb
    out = []
    for with_bwd in (False, True):
        for r in range(reps + 3):
            if r == 3:
                _ok(lib.gb_event_record(0), "event")
            if with_bwd:
                net.train_set_batch(ds, [0] * nb, 2.0 / (v * nb))
            else:
                for b in range(nb):
                    net.load_slot(b, xs[b])
                net.forward_graph()
        _ok(lib.gb_event_record(1), "event")
        _ok(lib.gb_synchronize(), "sync")
        out.append(lib.gb_event_elapsed_ms(0, 1) / reps / nb)
    _ok(lib.gb_unet_fill(net._g, net.nparam, 0.0), "fill")  # drop the timing runs' gradients
    return out


def time_simt_step(api, n, ds, reps: int = 10):
    """Forward + loss + backward ms per sample of a batch-1 network on the
    FP32 SIMT convolutions (gb_unet_tensor_cores(0)), the per-sample
    training the tensor-core kernels and minibatch launches replace; the
    tensor-core setting is restored afterwards."""
    lib = api.lib
    old = lib.gb_unet_tensor_cores(0)
    net = DeviceUNet(api, n, cin=3, seed=0)
    try:
        return time_training_step(net, ds, reps)[1]
    finally:
        lib.gb_unet_tensor_cores(old)
        net.free()


def main(argv=None):
    """python -m libgrid_b200.warmstart [--n N] [--step H] [--train N] [--test N]
    [--epochs E] [--out report.json]: generate, train, evaluate and print one
    JSON report."""
    import argparse
    import json

    import libgrid_b200

    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=512)
    ap.add_argument("--test", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=100)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--step", type=float, default=0.1)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--out", default=None)
    ap.add_argument("--quiet", action="store_true", help="no progress lines on stderr")
    ap.add_argument("--per-sample", action="store_true",
                    help="train one sample per launch (default: the whole minibatch per launch)")
    a = ap.parse_args(argv)

    def note(msg):
        if not a.quiet:
            print("[warmstart %.0fs] %s" % (time.perf_counter() - t_start, msg), file=sys.stderr, flush=True)

    t_start = time.perf_counter()
    api = libgrid_b200.load()
    api.lib.cuda_enable(b"\x01", 0, None)
    t0 = time.perf_counter()
    ds, meta = make_dataset(api, range(1000, 1000 + a.train), a.n, a.step, tol=a.tol)
    t_data = time.perf_counter() - t0
    note("%d ground states in %.1f s (mean %.0f steps)" % (a.train, t_data, np.mean([m["steps"] for m in meta])))
    net = DeviceUNet(api, a.n, cin=3, seed=0, batch=1 if a.per_sample else a.batch)
    inf = None
    try:
        t0 = time.perf_counter()
        loss = train(net, ds, epochs=a.epochs, batch=a.batch, lr=a.lr,
                     log=None if a.quiet else (lambda ep, l: note("epoch %d loss %.3e" % (ep, l))))
        api.lib.gb_synchronize()
        t_train = time.perf_counter() - t0
        step_ms = time_training_step(net, ds)
        simt_ms = time_simt_step(api, a.n, ds)
        ds.free()
        note("trained in %.1f s" % t_train)
        inf = net.clone(1) if net.nb > 1 else net  # inference one potential at a time
        rows = evaluate(api, inf, range(5000, 5000 + a.test), a.n, a.step, tol=a.tol)
    finally:
        if inf is not None and inf is not net:
            inf.free()
        net.free()
    mean = lambda k: float(np.mean([r[k] for r in rows]))
    rep = dict(
        workload="learned warm start, GP imaginary time %d^3 step %.3f bohr, %d training / %d held-out potentials"
        % (a.n, a.step, a.train, a.test),
        stopping="energy read every 10 steps; stop when the geometric estimate of the remaining distance to "
        "the limit and the last 10-step decrement are below %.0e Ha" % (a.tol / 2),
        params=int(net.nparam), epochs=a.epochs, batch=a.batch, samples_per_launch=net.nb, train_loss=loss,
        data_seconds=t_data, train_seconds=t_train, train_samples=a.train * a.epochs,
        train_ms_per_sample=1e3 * t_train / (a.train * a.epochs),
        forward_ms=step_ms[0], forward_backward_ms=step_ms[1],
        simt_forward_backward_ms=simt_ms, training_speedup_vs_simt=simt_ms / step_ms[1],
        data_steps_mean=float(np.mean([m["steps"] for m in meta])),
        steps_gauss=mean("steps_gauss"), steps_tf=mean("steps_tf"), steps_net=mean("steps_net"),
        sec_gauss=mean("sec_gauss"), sec_tf=mean("sec_tf"), sec_net=mean("sec_net"),
        step_ratio=mean("steps_gauss") / mean("steps_net"), time_ratio=mean("sec_gauss") / mean("sec_net"),
        steps_gauss_1e8=mean("steps_gauss_1e8"), steps_net_1e8=mean("steps_net_1e8"),
        sec_gauss_1e8=mean("sec_gauss_1e8"), sec_net_1e8=mean("sec_net_1e8"),
        step_ratio_1e8=mean("steps_gauss_1e8") / mean("steps_net_1e8"),
        time_ratio_1e8=mean("sec_gauss_1e8") / mean("sec_net_1e8"),
        max_de=float(max(r["de"] for r in rows)), max_de_net_ref=float(max(r["de_net_ref"] for r in rows)),
        max_de_gauss_ref=float(max(r["de_gauss_ref"] for r in rows)), rows=rows,
    )
    line = json.dumps(rep)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")
    print(line)


if __name__ == "__main__":
    main()
