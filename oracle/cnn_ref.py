"""CPU restatement of the warm-start CNN (test oracle for its CUDA kernels).

3x3 convolutions with zero padding, ReLU after every layer but the last,
weights rounded to FP16 as the device uses them, arithmetic in float64;
loss = mean squared error.  forward() and gradients() follow the layer
definitions of verb-4d_b200/csrc/cnn.cu operation for operation in exact
arithmetic (the device sums in FP32, in another order)."""
import numpy as np


def unpack(params, channels):
    out, off = [], 0
    for ci, co in zip(channels[:-1], channels[1:]):
        w = params[off:off + co * ci * 9].reshape(co, ci, 3, 3)
        off += co * ci * 9
        b = params[off:off + co]
        off += co
        out.append((w.astype(np.float16).astype(np.float64), b.astype(np.float64)))
    return out


def conv(x, w, b):
    B, Ci, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    out = np.zeros((B, w.shape[0], H, W)) + b[None, :, None, None]
    for dy in range(3):
        for dx in range(3):
            out += np.einsum("bchw,oc->bohw", xp[:, :, dy:dy + H, dx:dx + W], w[:, :, dy, dx])
    return out


def forward(params, channels, x):
    acts = [np.asarray(x, dtype=np.float64)]
    layers = unpack(params, channels)
    for l, (w, b) in enumerate(layers):
        z = conv(acts[-1], w, b)
        acts.append(np.maximum(z, 0) if l < len(layers) - 1 else z)
    return acts


def gradients(params, channels, x, target):
    layers = unpack(params, channels)
    acts = forward(params, channels, x)
    out = acts[-1]
    n = out.size
    loss = float(((out - target) ** 2).sum() / n)
    g = 2 * (out - target) / n
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        w, _ = layers[l]
        xin = acts[l]
        B, Ci, H, W = xin.shape
        xp = np.pad(xin, ((0, 0), (0, 0), (1, 1), (1, 1)))
        gw = np.zeros_like(w)
        for dy in range(3):
            for dx in range(3):
                gw[:, :, dy, dx] = np.einsum("bohw,bchw->oc", g, xp[:, :, dy:dy + H, dx:dx + W])
        gb = g.sum(axis=(0, 2, 3))
        grads.append((gw, gb))
        if l > 0:
            gp = np.pad(g, ((0, 0), (0, 0), (1, 1), (1, 1)))
            gi = np.zeros_like(xin)
            for dy in range(3):
                for dx in range(3):
                    gi += np.einsum("bohw,oc->bchw", gp[:, :, 2 - dy:2 - dy + H, 2 - dx:2 - dx + W],
                                    w[:, :, dy, dx])
            g = gi * (xin > 0)
    flat = []
    for gw, gb in reversed(grads):
        flat += [gw.ravel(), gb]
    return loss, np.concatenate(flat)
