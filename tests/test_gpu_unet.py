"""U-Net warm-start kernels (gb_unet_*) against the numpy oracle, the whole
network's gradients against the oracle's reverse mode, and the warm start
itself: ground states relaxed from the network's guess need fewer
imaginary-time steps than from a Gaussian and reach the same energy."""
import ctypes as C

import numpy as np
import pytest

from libgrid_b200 import warmstart as ws
from oracle import unet_oracle as uo

pytestmark = pytest.mark.gpu

TOL = 2e-6  # FP32 accumulation against the float64 oracle, relative L2
TOL_TC = 1e-5  # tensor-core accumulation order (FP32) against the float64 oracle


@pytest.fixture(params=[1, 0], ids=["tensor_cores", "simt"])
def engine(request, b200):
    """Run a test with the tensor-core convolutions (tcgen05 forward and data
    gradient, mma.sync weight gradient) and with the SIMT kernels."""
    lib = b200.lib
    lib.gb_unet_tensor_cores.restype = C.c_int
    lib.gb_unet_tensor_cores.argtypes = [C.c_int]
    old = lib.gb_unet_tensor_cores(request.param)
    yield request.param
    lib.gb_unet_tensor_cores(old)


def _rel(a, b):
    return float(np.linalg.norm((np.asarray(a, np.float64) - b).ravel()) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.fixture(scope="module")
def lib(b200):
    b200.lib.cuda_enable(b"\x01", 0, None)
    ws._bind(b200.lib)
    return b200.lib


class Dev:
    def __init__(self, lib):
        self.lib, self.ptrs = lib, []

    def put(self, a):
        a = np.ascontiguousarray(a)
        p = self.lib.gb_device_alloc(max(a.nbytes, 4))
        assert p
        assert self.lib.gb_h2d(p, a.ctypes.data, a.nbytes) == 0
        self.ptrs.append(p)
        return p

    def get(self, p, shape, dtype=np.float32):
        out = np.empty(shape, dtype)
        assert self.lib.gb_d2h(out.ctypes.data, p, out.nbytes) == 0
        assert self.lib.gb_synchronize() == 0
        return out

    def free(self):
        for p in self.ptrs:
            self.lib.gb_device_free(p)


def _wgrad_on_tensor_cores(cout, shape):
    d, h, w = shape
    return (cout <= 64 and w % 8 == 0 and
            any(d % tz == 0 and h % ty == 0 and (tz * ty * w) % 16 == 0 for tz in (1, 2, 4) for ty in (1, 2, 4)))


@pytest.mark.parametrize("cin,cout,shape", [(5, 6, (6, 8, 10)), (24, 8, (8, 8, 8)), (96, 32, (4, 4, 4)), (3, 1, (5, 7, 3)),
                                            (8, 7, (16, 16, 20)), (64, 64, (4, 4, 4)), (8, 8, (4, 4, 128)),
                                            (24, 8, (4, 2, 32)), (16, 32, (2, 8, 16)), (96, 32, (4, 4, 32)),
                                            (64, 64, (2, 2, 16)), (3, 8, (8, 4, 64)), (8, 1, (2, 4, 48)),
                                            (96, 32, (8, 8, 8)), (16, 17, (1, 2, 8)), (5, 9, (2, 1, 40)),
                                            (8, 8, (2, 2, 24)), (32, 64, (2, 2, 8))])
def test_conv_kernels_vs_oracle(lib, engine, cin, cout, shape):
    rng = np.random.default_rng(cin * 100 + cout)
    d = Dev(lib)
    x = rng.standard_normal((cin,) + shape).astype(np.float32)
    w = (rng.standard_normal((cout, cin, 27)) * 0.2).astype(np.float32)
    b = rng.standard_normal(cout).astype(np.float32)
    gy = rng.standard_normal((cout,) + shape).astype(np.float32)
    wr = uo.bf16_round(w)
    tc, tol = bool(engine), (TOL_TC if engine else TOL)
    # the weight gradient runs on tensor cores for volumes a multiple of 8
    # points wide with a voxel block of a multiple of 16 points (tz x ty
    # planes and rows, tz, ty in 1, 2, 4) and up to 64 output channels
    tc_w = tc and _wgrad_on_tensor_cores(cout, shape)
    dx, dw, db, dgy = d.put(x), d.put(uo.bf16_bits(w)), d.put(b), d.put(gy)
    dy = d.put(np.zeros((cout,) + shape, np.float32))
    for relu in (0, 1):
        assert lib.gb_unet_conv3_fwd(dx, dw, db, dy, cin, cout, *shape, relu) == 0
        assert _rel(d.get(dy, (cout,) + shape), uo.conv3_fwd(x, wr, b, relu, tc)) < tol
    dgx = d.put(np.full((cin,) + shape, 7.0, np.float32))
    assert lib.gb_unet_conv3_bwd_data(dgy, dw, dgx, cin, cout, *shape) == 0
    assert _rel(d.get(dgx, (cin,) + shape), uo.conv3_bwd_data(gy, wr, tc)) < tol
    gw0 = rng.standard_normal((cout, cin, 27)).astype(np.float32)
    gb0 = rng.standard_normal(cout).astype(np.float32)
    dgw, dgb = d.put(gw0), d.put(gb0)
    assert lib.gb_unet_conv3_bwd_weight(dx, dgy, dgw, dgb, cin, cout, *shape) == 0
    gw, gb = uo.conv3_bwd_weight(x, gy, tc_w)
    assert _rel(d.get(dgw, gw.shape), gw + gw0) < (TOL_TC if tc_w else TOL)
    assert _rel(d.get(dgb, gb.shape), gb + gb0) < TOL
    assert lib.gb_last_error() == 0
    d.free()


@pytest.mark.parametrize("cin,cout,shape", [(24, 8, (4, 4, 8)), (16, 32, (4, 2, 16)), (8, 8, (2, 4, 32)),
                                            (5, 3, (2, 3, 10))])
def test_batched_weight_gradient_vs_oracle(lib, engine, cin, cout, shape):
    """gb_unet_conv3_bwd_weight_nb over 3 samples stacked along depth gives
    the sum of the samples' own weight and bias gradients: no tap reaches
    across a sample boundary."""
    rng = np.random.default_rng(cin + 7 * cout)
    nb = 3
    d = Dev(lib)
    x = rng.standard_normal((cin, nb) + shape).astype(np.float32)
    gy = rng.standard_normal((cout, nb) + shape).astype(np.float32)
    tc_w = bool(engine) and _wgrad_on_tensor_cores(cout, shape)
    gw = np.zeros((cout, cin, 27))
    gb = np.zeros(cout)
    for s in range(nb):
        w_s, b_s = uo.conv3_bwd_weight(x[:, s], gy[:, s], tc_w)
        gw += w_s
        gb += b_s
    dgw, dgb = d.put(np.zeros((cout, cin, 27), np.float32)), d.put(np.zeros(cout, np.float32))
    dx, dgy = d.put(x), d.put(gy)
    assert lib.gb_unet_conv3_bwd_weight_nb(dx, dgy, dgw, dgb, cin, cout, nb, *shape) == 0
    assert _rel(d.get(dgw, gw.shape), gw) < (TOL_TC if tc_w else TOL)
    assert _rel(d.get(dgb, gb.shape), gb) < TOL
    assert lib.gb_last_error() == 0
    d.free()


def test_pool_up_relu_adam_vs_oracle(lib):
    rng = np.random.default_rng(3)
    d = Dev(lib)
    c, shape = 5, (6, 8, 4)
    half = tuple(s // 2 for s in shape)
    x = rng.standard_normal((c,) + shape).astype(np.float32)
    dx = d.put(x)
    dp = d.put(np.zeros((c,) + half, np.float32))
    assert lib.gb_unet_pool2_fwd(dx, dp, c, *shape) == 0
    assert _rel(d.get(dp, (c,) + half), uo.pool2_fwd(x)) < TOL
    gy = rng.standard_normal((c,) + half).astype(np.float32)
    g0 = rng.standard_normal((c,) + shape).astype(np.float32)
    dgy, dg0 = d.put(gy), d.put(g0)
    assert lib.gb_unet_pool2_bwd(dgy, dg0, c, *shape) == 0  # accumulates
    assert _rel(d.get(dg0, (c,) + shape), g0 + uo.pool2_bwd(gy)) < TOL
    xs = rng.standard_normal((c,) + half).astype(np.float32)
    dxs, dup = d.put(xs), d.put(np.zeros((c,) + shape, np.float32))
    assert lib.gb_unet_up2_fwd(dxs, dup, c, *half) == 0
    assert np.array_equal(d.get(dup, (c,) + shape), uo.up2_fwd(xs).astype(np.float32))
    gup = rng.standard_normal((c,) + shape).astype(np.float32)
    dgup, dgs = d.put(gup), d.put(np.zeros((c,) + half, np.float32))
    assert lib.gb_unet_up2_bwd(dgup, dgs, c, *half) == 0
    assert _rel(d.get(dgs, (c,) + half), uo.up2_bwd(gup)) < TOL
    y = rng.standard_normal(1000).astype(np.float32)
    g = rng.standard_normal(1000).astype(np.float32)
    dyy, dg = d.put(np.maximum(y, 0)), d.put(g)
    assert lib.gb_unet_relu_bwd(dg, dyy, 1000) == 0
    assert np.array_equal(d.get(dg, 1000), np.where(y > 0, g, 0).astype(np.float32))
    # Adam
    n = 777
    w, m, v, gr = (rng.standard_normal(n).astype(np.float32) for _ in range(4))
    v = np.abs(v)
    dw, dm, dv, dgr = d.put(w), d.put(m), d.put(v), d.put(gr)
    dwb = d.put(np.zeros(n, np.uint16))
    lr, b1, b2, eps, c1, c2 = 1e-2, 0.9, 0.999, 1e-8, 1 / (1 - 0.9**3), 1 / (1 - 0.999**3)
    assert lib.gb_unet_adam(dw, dwb, dm, dv, dgr, n, lr, b1, b2, eps, c1, c2) == 0
    m1 = b1 * m.astype(np.float64) + (1 - b1) * gr
    v1 = b2 * v.astype(np.float64) + (1 - b2) * gr.astype(np.float64) ** 2
    w1 = w - lr * (m1 * c1) / (np.sqrt(v1 * c2) + eps)
    got = d.get(dw, n)
    assert _rel(got, w1) < 1e-6
    assert np.array_equal(d.get(dwb, n, np.uint16), uo.bf16_bits(got))
    assert not np.any(d.get(dgr, n))
    d.free()


@pytest.mark.parametrize("n", [16, 32])
def test_unet_gradients_vs_oracle(b200, lib, engine, n):
    rng = np.random.default_rng(11)
    net = ws.DeviceUNet(b200, n, cin=3, seed=4)
    try:
        p = net.get("p")
        bias = rng.standard_normal(p.shape).astype(np.float32) * 0.05
        for o, co, ci in net.layers.values():  # give the biases nonzero values
            p[o + co * ci * 27 : o + co * ci * 27 + co] = bias[:co]
        net.set_params(p)
        x = rng.standard_normal((3, n, n, n)).astype(np.float32)
        tgt = rng.standard_normal((n, n, n)).astype(np.float32) * 0.1
        net.set_input(x)
        net.forward()
        net.loss_grad(net.set_target(tgt), 2.0 / n**3)
        net.backward()
        g = net.get("g")
        pred = net.activation("out")[0]
        params = {k: (uo.bf16_round(w), b.astype(np.float64)) for k, (w, b) in net.layer_arrays(p).items()}
        tc = bool(engine)
        want_pred, _ = uo.unet_forward(net.spec, params, x, tc)
        # tensor cores: every convolution rounds its operands to bf16; where an
        # intermediate activation lies near a bf16 rounding boundary, the
        # device (FP32 accumulation) and the oracle (float64) round it to
        # neighbouring bf16 values, and such one-ulp (2^-8) differences
        # compound through the 21 layers.  Each kernel alone is pinned to
        # 1e-5 in test_conv_kernels_vs_oracle.
        assert _rel(pred, want_pred[0]) < (2e-2 if tc else 1e-5)
        _, grads = uo.unet_loss_grads(net.spec, params, x, tgt[None], tc)
        got = net.layer_arrays(g)
        for layer, (gw, gb) in grads.items():
            assert _rel(got[layer][0], gw) < (5e-2 if tc else 1e-4), layer
            assert _rel(got[layer][1], gb) < (5e-2 if tc else 1e-4), layer
    finally:
        net.free()


def test_warm_start_cuts_imaginary_time_steps(b200, lib):
    n, step = 32, 0.1
    ds, meta = ws.make_dataset(b200, range(1000, 1032), n, step)
    assert all(m["steps"] < 20000 for m in meta)
    net = ws.DeviceUNet(b200, n, cin=3, seed=0)
    try:
        ys = np.empty((ds.count, n**3), np.float32)
        assert lib.gb_d2h(ys.ctypes.data, ds.y, ys.nbytes) == 0
        loss = ws.train(net, ds, epochs=40, batch=8, lr=2e-3)
        assert loss < 0.05 * float((ys**2).mean())
        rows = ws.evaluate(b200, net, range(5000, 5006), n, step)
    finally:
        ds.free()
        net.free()
    steps_g = np.mean([r["steps_gauss"] for r in rows])
    steps_n = np.mean([r["steps_net"] for r in rows])
    print("warm start: steps %.0f (Gaussian) -> %.0f (network); TF start %.0f; max |dE| %.2e"
          % (steps_g, steps_n, np.mean([r["steps_tf"] for r in rows]), max(r["de"] for r in rows)))
    assert steps_n < steps_g
    # the stopping rule estimates the remaining distance to the limit: the
    # network and the Gaussian start converge to energies within 1e-8 Ha of
    # each other and of the limit a far tighter rule (1e-12 change) reaches
    assert max(r["de"] for r in rows) < 1e-8
    assert max(r["de_net_ref"] for r in rows) < 1e-8


def test_device_problem_features_match_host(b200, lib):
    """The device potential, Thomas-Fermi chemical potential (Newton on
    device sums) and network input against their host definitions."""
    n, step = 32, 0.1
    r = ws.Relaxer(b200, n, step)
    try:
        for seed in (1000, 1234, 5003):
            v, g, _ = ws.sample_problem(seed, n, step)
            assert r.set_problem(seed) == g
            assert np.max(np.abs(r.vx.get() - v)) <= 1e-15 * np.max(np.abs(v)) + 1e-18
            out, s = r.tf_features()
            x, s_host = ws.features(v, g, step)
            assert abs(s - s_host) <= 1e-10 * s_host
            got = np.empty((3, n, n, n), np.float32)
            assert lib.gb_d2h(got.ctypes.data, out, got.nbytes) == 0
            assert lib.gb_synchronize() == 0
            assert np.max(np.abs(got - x)) < 1e-6
    finally:
        r.free()


def test_training_is_deterministic(b200, lib):
    """No kernel uses atomics and every sum has a fixed order, so two
    training runs from the same seed give bit-identical weights."""
    rng = np.random.default_rng(21)
    n = 16
    xs = rng.standard_normal((4, 3, n, n, n)).astype(np.float32)
    ys = np.abs(rng.standard_normal((4, n, n, n))).astype(np.float32)
    out = []
    for _ in range(2):
        net = ws.DeviceUNet(b200, n, cin=3, seed=7)
        ds = ws.host_dataset(b200, xs, ys)
        try:
            ws.train(net, ds, epochs=3, batch=2, lr=1e-3, seed=3, monitor=2)
            out.append(net.get("p"))
        finally:
            ds.free()
            net.free()
    assert np.array_equal(out[0], out[1])
    assert np.any(out[0] != 0)


def test_graph_training_step_matches_eager(b200, lib, engine):
    """The captured training step (forward, loss gradient and backward replayed
    as one CUDA graph) and the captured forward give bit-identical
    gradients and outputs to the same calls made one by one; the graphs'
    kernels are counted in gb_launch_count on every replay."""
    rng = np.random.default_rng(31)
    n = 16
    x = rng.standard_normal((3, n, n, n)).astype(np.float32)
    y = np.abs(rng.standard_normal((n, n, n))).astype(np.float32)
    scale = 2.0 / n**3
    net = ws.DeviceUNet(b200, n, cin=3, seed=5)
    dev = Dev(lib)
    try:
        dx, dy = dev.put(x), dev.put(y)
        net.set_input(x)
        net.forward()
        out_eager = net.activation("out")
        net.loss_grad(net.set_target(y), scale)
        net.backward()
        g_eager = net.get("g")
        assert lib.gb_unet_fill(net._g, net.nparam, 0.0) == 0
        with pytest.raises(RuntimeError):
            net.train_sample(dx, dy, scale)  # graphs are prepared first
        net.prepare_training([scale])
        assert not np.any(net.get("g"))  # the sizing run's gradient is cleared
        lib.gb_launch_count.restype = C.c_long
        before = lib.gb_launch_count()
        net.train_sample(dx, dy, scale)
        per_replay = lib.gb_launch_count() - before
        assert per_replay > 20
        g_graph = net.get("g")
        assert np.array_equal(g_graph, g_eager)
        net.train_sample(dx, dy, scale)  # gradients accumulate across replays
        assert _rel(net.get("g"), 2.0 * g_eager.astype(np.float64)) < 1e-6
        assert lib.gb_launch_count() - before == 2 * per_replay
        net.infer_device(dx)
        assert np.array_equal(net.activation("out"), out_eager)
    finally:
        dev.free()
        net.free()


def test_batched_network_matches_per_sample(b200, lib, engine):
    """A batch-4 network (samples stacked along depth, one launch per layer)
    fed 3 samples gives each sample's output as the batch-1 network does,
    and the same summed weight and bias gradients up to the FP32 summation
    order (the fourth slot gets a zero output gradient); no depth neighbour
    crosses a sample boundary."""
    rng = np.random.default_rng(41)
    n = 16
    xs = rng.standard_normal((3, 3, n, n, n)).astype(np.float32)
    ys = np.abs(rng.standard_normal((3, n, n, n))).astype(np.float32)
    scale = 2.0 / (3 * n**3)
    one = ws.DeviceUNet(b200, n, cin=3, seed=9)
    four = ws.DeviceUNet(b200, n, cin=3, seed=9, batch=4)
    dev = Dev(lib)
    try:
        dx = [dev.put(x) for x in xs]
        dy = [dev.put(y) for y in ys]
        one.prepare_training([scale])
        outs = []
        for i in range(3):
            one.train_sample(dx[i], dy[i], scale)
            outs.append(one.activation("out")[0])
        g_one = one.get("g")
        four.prepare_training([scale], [3])
        four.train_batch(dx, dy, scale)
        g_four = four.get("g")
        out4 = four.activation("out")[0]  # [4][n][n][n]
        for i in range(3):
            assert _rel(out4[i], outs[i].astype(np.float64)) < 1e-6, i
        assert _rel(g_four, g_one.astype(np.float64)) < 1e-5
        inf = four.clone(1)
        try:
            inf.infer_device(dx[1])
            assert _rel(inf.activation("out")[0], outs[1].astype(np.float64)) < 1e-6
        finally:
            inf.free()
    finally:
        dev.free()
        one.free()
        four.free()


def test_gather_fills_batch_slots(b200, lib):
    """gb_unet_gather puts samples idx[b] of a device set into batch slots b
    (inputs [cin][nb][vol], target [nb][vol]) as per-sample copies do, and
    rejects an index outside the set without copying."""
    rng = np.random.default_rng(5)
    n, nset = 16, 5
    vol = n**3
    net = ws.DeviceUNet(b200, n, cin=3, seed=0, batch=4)
    ds = ws.DeviceSet(lib, nset, vol)
    try:
        xs = rng.standard_normal((nset, 3, vol)).astype(np.float32)
        ys = rng.standard_normal((nset, vol)).astype(np.float32)
        assert lib.gb_h2d(ds.x, xs.ctypes.data, xs.nbytes) == 0
        assert lib.gb_h2d(ds.y, ys.ctypes.data, ys.nbytes) == 0
        idx = [4, 0, 4]
        assert lib.gb_unet_fill(net._act("in"), 3 * 4 * vol, -1.0) == 0
        assert lib.gb_unet_gather(net._act("in"), net._tgt, ds.x, ds.y, (C.c_int * 3)(*idx), 3, 3, vol, 4, nset) == 0
        got = net.activation("in").reshape(3, 4, vol)
        tgt = np.empty((4, vol), np.float32)
        assert lib.gb_d2h(tgt.ctypes.data, net._tgt, tgt.nbytes) == 0
        assert lib.gb_synchronize() == 0
        for b, i in enumerate(idx):
            assert np.array_equal(got[:, b], xs[i])
            assert np.array_equal(tgt[b], ys[i])
        assert np.all(got[:, 3] == -1.0)  # slot past count untouched
        bad = (C.c_int * 2)(1, nset)
        assert lib.gb_unet_gather(net._act("in"), net._tgt, ds.x, ds.y, bad, 2, 3, vol, 4, nset) == 1101
        assert lib.gb_last_error() == 1101
        lib.gb_clear_error()
        assert np.array_equal(net.activation("in").reshape(3, 4, vol), got)
    finally:
        ds.free()
        net.free()
