"""CPU restatement of the warm-start CNN (test oracle for its CUDA kernels).

3x3 convolutions with zero padding, ReLU after every layer but the last,
weights rounded to FP16 as the device uses them, arithmetic in float64;
loss = mean squared error.  The device runs every convolution on the tensor
cores with TF32 operands (FP16 weights are exact in TF32; activations and
gradients are rounded to TF32 with round-to-nearest, ties away from zero, as
they enter the matrix product), so tf32() rounds the same operands here.
forward() and gradients() follow the layer definitions of
verb-4d_b200/csrc/cnn.cu operation for operation in exact arithmetic (the
device sums in FP32, in another order)."""
import numpy as np


def tf32(a):
    """Round float64 values to float32, then to TF32 (10 explicit mantissa
    bits, round to nearest with ties away from zero: cvt.rna.tf32.f32)."""
    b = np.asarray(a, dtype=np.float32).copy().view(np.uint32)
    b = (b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)
    return b.view(np.float32).astype(np.float64)


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
        z = conv(tf32(acts[-1]), w, b)
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
        xp = np.pad(tf32(xin), ((0, 0), (0, 0), (1, 1), (1, 1)))
        gt = tf32(g)
        gw = np.zeros_like(w)
        for dy in range(3):
            for dx in range(3):
                gw[:, :, dy, dx] = np.einsum("bohw,bchw->oc", gt, xp[:, :, dy:dy + H, dx:dx + W])
        gb = g.sum(axis=(0, 2, 3))
        grads.append((gw, gb))
        if l > 0:
            gp = np.pad(gt, ((0, 0), (0, 0), (1, 1), (1, 1)))
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


# ---- learned preconditioner (sparse approximate inverse on a 5 x 5 stencil)
def precond_apply(A9, Cc, v, nx, ny):
    """M v for one system: A9 [9][n] (slot (dy+1)*3+(dx+1)), Cc [25][n]
    (slot (dy+2)*5+(dx+2)), M v (i) = sum_o (delta(o=0) + C[o](i)) v(i+o)/diag(i+o)
    over the neighbours inside the nx x ny grid."""
    n = nx * ny
    dg = A9[4]
    out = np.zeros(n)
    for i in range(n):
        iy, ix = divmod(i, nx)
        for dy in range(-2, 3):
            for dx in range(-2, 3):
                yy, xx = iy + dy, ix + dx
                if 0 <= yy < ny and 0 <= xx < nx:
                    o = (dy + 2) * 5 + (dx + 2)
                    j = yy * nx + xx
                    out[i] += (Cc[o, i] + (1.0 if o == 12 else 0.0)) * v[j] / dg[j]
    return out


def matvec9(A9, y, nx):
    n = len(y)
    out = np.zeros(n)
    for i in range(n):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                col = i + dy * nx + dx
                if 0 <= col < n:
                    out[i] += A9[(dy + 1) * 3 + (dx + 1), i] * y[col]
    return out


def matvec9_t(A9, e, nx):
    n = len(e)
    out = np.zeros(n)
    for i in range(n):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                r = i - (dy * nx + dx)
                if 0 <= r < n:
                    out[i] += A9[(dy + 1) * 3 + (dx + 1), r] * e[r]
    return out


def precond_loss_grad(A9s, Cs, Zs, nx, ny):
    """Loss mean |D^-1 A M D z - z|^2 (the Jacobi-scaled system) over systems
    and probes, and its gradient with respect to C (the definition of
    verb_precond_loss_grad).  M D z is the stencil of delta + C applied to z."""
    nsys, nprobe, n = Zs.shape
    cnt = nsys * nprobe * n
    loss = 0.0
    g = np.zeros_like(Cs, dtype=np.float64)
    for s in range(nsys):
        dg = A9s[s][4]
        for q in range(nprobe):
            z = Zs[s, q]
            y = precond_apply(A9s[s], Cs[s], z * dg, nx, ny)  # M (D z)
            e = matvec9(A9s[s], y, nx) / dg - z
            loss += float(e @ e) / cnt
            gy = 2.0 / cnt * matvec9_t(A9s[s], e / dg, nx)
            for i in range(n):
                iy, ix = divmod(i, nx)
                for dy in range(-2, 3):
                    for dx in range(-2, 3):
                        yy, xx = iy + dy, ix + dx
                        if 0 <= yy < ny and 0 <= xx < nx:
                            g[s, (dy + 2) * 5 + (dx + 2), i] += gy[i] * z[yy * nx + xx]
    return loss, g
