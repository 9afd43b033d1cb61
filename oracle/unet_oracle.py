"""CPU oracle (test infrastructure only) for the U-Net warm-start kernels.

Plain numpy, float64 accumulation, bf16 weights rounded to nearest even as the
device kernels round them.  With tc=True the convolution operands are also
rounded to bf16 (activations in the forward and data-gradient convolutions,
activations and output gradients in the weight gradient), as the library's
tensor-core convolutions do; with tc=False they stay as given (the SIMT
kernels: FP32 activations).  The reference has no learned part, so nothing
here follows a reference file: these are the textbook definitions of a 3x3x3
zero-padded convolution, its two gradients, 2x2x2 average pooling and
nearest-neighbour upsampling.  Layouts match the device kernels: activations
[C][D][H][W], weights [Cout][Cin][27] with tap t = 9(dz+1) + 3(dy+1) + (dx+1).
Only tests import this module.
"""
from __future__ import annotations

import numpy as np

TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def bf16_round(w) -> np.ndarray:
    """float32 -> nearest bf16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(w) -> np.ndarray:
    """float32 -> bf16 bit patterns (uint16), nearest even."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def _shift(x, dz, dy, dx):
    """s[..., z, y, x] = x[..., z+dz, y+dy, x+dx], zero outside."""
    p = np.pad(x, [(0, 0)] * (x.ndim - 3) + [(1, 1)] * 3)
    d, h, w = x.shape[-3:]
    return p[..., 1 + dz : 1 + dz + d, 1 + dy : 1 + dy + h, 1 + dx : 1 + dx + w]


def _op(a, tc):
    return bf16_round(a) if tc else np.asarray(a, np.float64)


def conv3_fwd(x, w, b, relu, tc=False):
    """y[co] = sum_ci sum_t x[ci](p + off t) w[co, ci, t] + b[co]."""
    x = _op(x, tc)
    y = np.zeros((w.shape[0],) + x.shape[1:])
    for t, (dz, dy, dx) in enumerate(TAPS):
        y += np.tensordot(w[:, :, t], _shift(x, dz, dy, dx), axes=(1, 0))
    y += np.asarray(b, np.float64)[:, None, None, None]
    return np.maximum(y, 0.0) if relu else y


def conv3_bwd_data(gy, w, tc=False):
    gy = _op(gy, tc)
    gx = np.zeros((w.shape[1],) + gy.shape[1:])
    for t, (dz, dy, dx) in enumerate(TAPS):
        gx += np.tensordot(w[:, :, t].T, _shift(gy, -dz, -dy, -dx), axes=(1, 0))
    return gx


def conv3_bwd_weight(x, gy, tc=False):
    """Weight and bias gradients; the bias gradient sums the unrounded gy."""
    gsum = np.asarray(gy, np.float64).sum(axis=(1, 2, 3))
    x = _op(x, tc)
    gy = _op(gy, tc)
    gw = np.zeros((gy.shape[0], x.shape[0], 27))
    for t, (dz, dy, dx) in enumerate(TAPS):
        gw[:, :, t] = np.tensordot(gy, _shift(x, dz, dy, dx), axes=([1, 2, 3], [1, 2, 3]))
    return gw, gsum


def pool2_fwd(x):
    c, d, h, w = x.shape
    return np.asarray(x, np.float64).reshape(c, d // 2, 2, h // 2, 2, w // 2, 2).mean(axis=(2, 4, 6))


def pool2_bwd(gy):
    return np.repeat(np.repeat(np.repeat(np.asarray(gy, np.float64), 2, 1), 2, 2), 2, 3) / 8.0


def up2_fwd(x):
    return np.repeat(np.repeat(np.repeat(np.asarray(x, np.float64), 2, 1), 2, 2), 2, 3)


def up2_bwd(gy):
    c, d, h, w = gy.shape
    return np.asarray(gy, np.float64).reshape(c, d // 2, 2, h // 2, 2, w // 2, 2).sum(axis=(2, 4, 6))


def unet_forward(spec, params, x, tc=False):
    """Whole network on the CPU.  spec: list of ops as built by
    libgrid_b200.warmstart.unet_spec; params: {layer: (w float64 [co,ci,27]
    already bf16-rounded, b)}.  Returns (prediction, activations)."""
    acts = {"in": np.asarray(x, np.float64)}
    for op in spec:
        kind = op[0]
        src = np.concatenate([acts[n] for n in op[1]], axis=0)
        if kind == "conv":
            w, b = params[op[3]]
            acts[op[2]] = conv3_fwd(src, w, b, op[4], tc)
        elif kind == "pool":
            acts[op[2]] = pool2_fwd(src)
        elif kind == "up":
            acts[op[2]] = up2_fwd(src)
    return acts[spec[-1][2]], acts


def unet_loss_grads(spec, params, x, tgt, tc=False):
    """Loss = sum (pred - tgt)^2 / n and its gradients for every layer, by
    reverse-mode through the same ops (float64)."""
    pred, acts = unet_forward(spec, params, x, tc)
    n = pred.size
    loss = float(((pred - tgt) ** 2).sum() / n)
    grads = {k: np.zeros_like(v) for k, v in acts.items()}
    grads[spec[-1][2]] = 2.0 * (pred - tgt) / n
    pgrads = {}
    for op in reversed(spec):
        kind, srcs, out = op[0], op[1], op[2]
        g = grads[out]
        src = np.concatenate([acts[s] for s in srcs], axis=0)
        if kind == "conv":
            if op[4]:
                g = g * (acts[out] > 0)
            w, _ = params[op[3]]
            gw, gb = conv3_bwd_weight(src, g, tc)
            pgrads[op[3]] = (gw, gb)
            gsrc = conv3_bwd_data(g, w, tc)
        elif kind == "pool":
            gsrc = pool2_bwd(g)
        else:
            gsrc = up2_bwd(g)
        c0 = 0
        for s in srcs:
            c = acts[s].shape[0]
            grads[s] = grads[s] + gsrc[c0 : c0 + c]
            c0 += c
    return loss, pgrads
