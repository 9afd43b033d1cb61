"""CPU checks of the U-Net oracle: its analytic gradients against central
finite differences on a tiny network, and its bf16 rounding (nearest, ties
to even)."""
import numpy as np

from libgrid_b200.warmstart import unet_spec
from oracle import unet_oracle as uo


def _params(spec, chan, rng):
    out = {}
    for op in spec:
        if op[0] == "conv":
            ci = sum(chan[s] for s in op[1])
            co = chan[op[2]]
            out[op[3]] = (rng.standard_normal((co, ci, 27)) * np.sqrt(2.0 / (ci * 27)), rng.standard_normal(co) * 0.1)
    return out


def test_bf16_round_nearest_even():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, -2.5, 1e-3, 3.0e38], np.float32)
    got = uo.bf16_round(x)
    assert got[0] == 1.0
    assert got[1] == 1.0  # halfway: ties to even (mantissa ...0)
    assert got[2] == 1.0 + 2 * 2**-7  # halfway: rounds up to the even neighbour
    assert got[3] == -2.5
    assert abs(got[4] - 1e-3) / 1e-3 < 2**-8
    bits = uo.bf16_bits(x)
    back = (bits.astype(np.uint32) << 16).view(np.float32)
    assert np.array_equal(back.astype(np.float64), got)


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(5)
    spec, chan = unet_spec(cin=2, ch=(2, 3, 3, 4))
    params = _params(spec, chan, rng)
    n = 8
    x = rng.standard_normal((2, n, n, n))
    tgt = rng.standard_normal((1, n, n, n)) * 0.1
    loss, grads = uo.unet_loss_grads(spec, params, x, tgt)
    eps = 1e-6
    for layer in ("e0a", "ba", "d1a", "d0a", "out"):
        w, b = params[layer]
        for idx in [tuple(rng.integers(0, s) for s in w.shape) for _ in range(3)]:
            old = w[idx]
            w[idx] = old + eps
            lp, _ = uo.unet_loss_grads(spec, params, x, tgt)
            w[idx] = old - eps
            lm, _ = uo.unet_loss_grads(spec, params, x, tgt)
            w[idx] = old
            fd = (lp - lm) / (2 * eps)
            an = grads[layer][0][idx]
            assert abs(fd - an) <= 1e-5 * max(1.0, abs(fd)) + 1e-8, (layer, idx, fd, an)
        j = int(rng.integers(0, b.shape[0]))
        old = b[j]
        b[j] = old + eps
        lp, _ = uo.unet_loss_grads(spec, params, x, tgt)
        b[j] = old - eps
        lm, _ = uo.unet_loss_grads(spec, params, x, tgt)
        b[j] = old
        assert abs((lp - lm) / (2 * eps) - grads[layer][1][j]) <= 1e-5 * max(1.0, abs(grads[layer][1][j])) + 1e-8


def test_warm_start_host_logic():
    from libgrid_b200 import warmstart as ws

    # the seeded problem family is reproducible and in its stated ranges
    v1, g1, k1 = ws.sample_problem(1234, 16, 0.1)
    v2, g2, k2 = ws.sample_problem(1234, 16, 0.1)
    assert np.array_equal(v1, v2) and g1 == g2 and k1 == k2
    assert 0.001 <= g1 <= 0.01 and 0.005 <= k1 <= 0.02
    # Thomas-Fermi amplitude is normalised and vanishes where V > mu
    v, g, _ = ws.sample_problem(7, 32, 0.1)
    tf = ws.thomas_fermi(v, g, 0.1)
    assert abs((tf**2).sum() * 0.1**3 - 1.0) < 1e-9
    assert tf.min() == 0.0 and tf.max() > 0
    x, s = ws.features(v, g, 0.1)
    assert x.shape == (3, 32, 32, 32) and x.dtype == np.float32
    assert abs(x[2].max() - 1.0) < 1e-6 and abs(s - tf.max()) < 1e-12
    # network: every conv's input channels are its sources' channels, the
    # skip concatenations pair equal resolutions, and the size is as stated
    spec, chan = ws.unet_spec()
    nparam = 0
    for op in spec:
        if op[0] == "conv":
            ci = sum(chan[src] for src in op[1])
            nparam += chan[op[2]] * ci * 27 + chan[op[2]]
            assert len({ws._LEVEL[src] for src in op[1]}) == 1
            assert ws._LEVEL[op[2]] == ws._LEVEL[op[1][0]]
        elif op[0] == "pool":
            assert ws._LEVEL[op[2]] == ws._LEVEL[op[1][0]] + 1
        else:
            assert ws._LEVEL[op[2]] == ws._LEVEL[op[1][0]] - 1
    assert nparam == 365825
