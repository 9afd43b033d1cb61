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
