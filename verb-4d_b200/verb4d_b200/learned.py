"""Host side of the learned warm start: the CNN object of the C ABI
(verb_cnn_*), its input features, triple collection and training.

Features of a local (V,K) system, [4][K][V] FP32 (pitch angle down the
image, energy across): log10 D_VV and log10 D_KK centred on the log-normal
median of the seeded coefficient fields and halved, D_VK / sqrt(D_VV D_KK),
and the state the step starts from, f / max|f|.  Target: (x - f) / max|f|,
the step's relative increment, so that x0 = f + max|f| * out is the Krylov
solve's warm start and a network that outputs zero reproduces the x0 = f
guess.  (The right-hand side b is no guess: the system's interior rows are
scaled by 1/dt, so b is f/dt plus sources there.)  The device computes both
(verb_local_triples / the feature kernel of verb_local_krylov); features() is
their CPU definition.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from . import workload as W

CHANNELS = (4, 32, 32, 32, 1)
D_MEDIAN = 1e-5 * 86400.0


def features(dvv, dkk, dvk, state):
    """[B][V][K] fields -> [B][4][K][V] float32 inputs and the per-system
    scale max|f| (1 where f = 0), in FP32 arithmetic as on the device."""
    f32 = np.float32
    med = np.log10(f32(D_MEDIAN))
    dvv, dkk, dvk = (np.asarray(a, dtype=f32) for a in (dvv, dkk, dvk))
    f = np.asarray(state, dtype=f32)
    scale = np.abs(f).reshape(len(f), -1).max(axis=1)
    scale = np.where(scale > 0, scale, f32(1.0)).astype(f32)
    a = (np.log10(dvv) - med) * f32(0.5)
    b = (np.log10(dkk) - med) * f32(0.5)
    c = dvk / np.sqrt(dvv * dkk)
    r = f / scale[:, None, None]
    out = np.stack([a, b, c, r], axis=1).astype(f32)
    return np.ascontiguousarray(out.transpose(0, 1, 3, 2)), scale


def collect_triples(seeds, steps_per_seed: int, spec=None, sources=True, losses=True,
                    coeff_corr: float = 0.0):
    """Run whole operator-split steps at `spec` (default 24 x 25 x 31 x 31)
    for each seed; the local part of every step is taken by the LU through
    verb_local_triples, which emits one (features, target) pair per (P,R)
    system.  Returns device tensors feat [N][4][K][V] and target [N][1][K][V]."""
    import torch

    from .solver import Solver

    spec = spec or W.CONFIGS["cfg1"]
    nsys = spec.P * spec.R
    n = len(seeds) * steps_per_seed * nsys
    feat = torch.empty((n, 4, spec.K, spec.V), dtype=torch.float32, device="cuda")
    targ = torch.empty((n, 1, spec.K, spec.V), dtype=torch.float32, device="cuda")
    i = 0
    for seed in seeds:
        wl = W.make_workload(spec, seed=seed, sources=sources, losses=losses,
                             coeff_corr=coeff_corr)
        s = Solver(wl)
        s.load()
        fl = wl.flags
        for it in range(1, steps_per_seed + 1):
            s.update_inputs(it)
            s.ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], False)
            s.ctx.local_triples(wl.dt, wl.sub_dt, feat[i:].data_ptr(), targ[i:].data_ptr())
            i += nsys
        s.ctx.sync()
        s.ctx.close()
    return feat, targ


def train(net, feat, targ, epochs: int = 20, batch: int = 256, lr: float = 1e-3, seed: int = 0,
          lr_final: float = 1e-4):
    """Adam on shuffled mini-batches with a geometric learning-rate decay
    from lr to lr_final; returns the mean loss of every epoch."""
    import torch

    n = feat.shape[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    nb = max(1, n // batch)
    decay = (lr_final / lr) ** (1.0 / max(1, epochs * nb - 1))
    rate = lr
    for _ in range(epochs):
        perm = torch.randperm(n, generator=g).to(feat.device)
        tot = 0.0
        for b in range(nb):
            idx = perm[b * batch:(b + 1) * batch]
            xb = feat.index_select(0, idx).contiguous()
            tb = targ.index_select(0, idx).contiguous()
            tot += net.train_step(xb.data_ptr(), tb.data_ptr(), len(idx), rate)
            rate *= decay
        hist.append(tot / nb)
    return hist


PC_CHANNELS = (9, 32, 32, 32, 25)


def precond_inputs(wl, seeds=None):
    """Features [N][9][K][V] and FP32 diagonals [N][9][V*K] of the local
    systems of `wl` (and of the same grid with the coefficients of every
    seed in `seeds`), device tensors."""
    import torch

    from .solver import Solver

    spec = wl.spec
    nsys, n = spec.P * spec.R, spec.V * spec.K
    wls = [wl] + [W.make_workload(spec, seed=sd, sources=True, losses=True) for sd in (seeds or [])]
    feat = torch.empty((len(wls) * nsys, 9, spec.K, spec.V), dtype=torch.float32, device="cuda")
    A9 = torch.empty((len(wls) * nsys, 9, n), dtype=torch.float32, device="cuda")
    for i, w in enumerate(wls):
        s = Solver(w)
        s.load()
        s.ctx.local_precond_inputs(w.dt, w.sub_dt, feat[i * nsys:].data_ptr(), A9[i * nsys:].data_ptr())
        s.ctx.close()
    return feat, A9


def precond_loss_grad(A9, Cc, Z, V, K):
    """mean |D^-1 A M D z - z|^2 (D = diag(A)) over the probes Z
    [B][nprobe][V*K] and its gradient with respect to the coefficients Cc
    [B][25][K][V] (device tensors)."""
    import torch

    g = torch.empty_like(Cc)
    loss = C.c_float()
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    L.check(L.load().verb_precond_loss_grad(vp(A9), vp(Cc), vp(Z), A9.shape[0], V, K, Z.shape[1],
                                            vp(g), C.byref(loss), None), "precond loss")
    return loss.value, g


def train_preconditioner(net, feat, A9, V, K, epochs=30, batch=64, nprobe=4, lr=2e-3,
                         lr_final=2e-4, seed=0):
    """Adam on shuffled system batches with Gaussian probe vectors: the
    network learns coefficients C that make A M close to the identity
    (the loss is mean |D^-1 A M D z - z|^2 over the probes, D = diag(A)).  Returns the mean loss of
    every epoch."""
    import torch

    n = feat.shape[0]
    gen = torch.Generator(device="cuda").manual_seed(seed)
    gcpu = torch.Generator(device="cpu").manual_seed(seed)
    out = torch.empty((batch, 25, K, V), dtype=torch.float32, device="cuda")
    nb = max(1, n // batch)
    decay = (lr_final / lr) ** (1.0 / max(1, epochs * nb - 1))
    rate = lr
    hist = []
    for _ in range(epochs):
        perm = torch.randperm(n, generator=gcpu).to(feat.device)
        tot = 0.0
        for b in range(nb):
            idx = perm[b * batch:(b + 1) * batch]
            xb = feat.index_select(0, idx).contiguous()
            ab = A9.index_select(0, idx).contiguous()
            Z = torch.randn((len(idx), nprobe, V * K), generator=gen, device="cuda")
            net.forward(xb.data_ptr(), out.data_ptr(), len(idx))
            loss, g = precond_loss_grad(ab, out[:len(idx)], Z, V, K)
            net.backward_step(xb.data_ptr(), g.data_ptr(), len(idx), rate)
            tot += loss
            rate *= decay
        hist.append(tot / nb)
    return hist


class CNN:
    def __init__(self, H, W, max_batch, channels=CHANNELS, seed=0, stream=None):
        self.lib = L.load()
        self.channels = tuple(channels)
        self.H, self.W, self.max_batch = H, W, max_batch
        h = C.c_void_p()
        ch = (C.c_int * len(channels))(*channels)
        L.check(self.lib.verb_cnn_create(C.byref(h), len(channels) - 1, ch, H, W, max_batch,
                                         stream), "cnn_create")
        self.h = h
        n = C.c_longlong()
        L.check(self.lib.verb_cnn_param_count(self.h, C.byref(n)), "cnn_params")
        self.nparams = n.value
        self.set_params(self.init_params(seed))

    def init_params(self, seed):
        """He-normal weights, zero biases."""
        rng = np.random.default_rng(seed)
        out = []
        for ci, co in zip(self.channels[:-1], self.channels[1:]):
            out.append(rng.standard_normal(co * ci * 9) * np.sqrt(2.0 / (ci * 9)))
            out.append(np.zeros(co))
        return np.concatenate(out).astype(np.float32)

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        L.check(self.lib.verb_cnn_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))),
                "cnn_set")

    def params(self, with_grad=False):
        p = np.empty(self.nparams, dtype=np.float32)
        g = np.empty(self.nparams, dtype=np.float32) if with_grad else None
        L.check(self.lib.verb_cnn_get_params(
            self.h, p.ctypes.data_as(C.POINTER(C.c_float)),
            g.ctypes.data_as(C.POINTER(C.c_float)) if with_grad else None), "cnn_get")
        return (p, g) if with_grad else p

    def forward(self, x_dev, out_dev, batch):
        L.check(self.lib.verb_cnn_forward(self.h, C.c_void_p(x_dev), C.c_void_p(out_dev), batch),
                "cnn_forward")

    def zero_last_layer(self):
        """Zero the last layer's weights and bias (the network then outputs 0:
        for the preconditioner, exactly the Jacobi one)."""
        p = self.params()
        ci, co = self.channels[-2], self.channels[-1]
        p[self.nparams - co - co * ci * 9:] = 0.0
        self.set_params(p)

    def backward_step(self, x_dev, g_dev, batch, lr):
        L.check(self.lib.verb_cnn_backward_step(self.h, C.c_void_p(x_dev), C.c_void_p(g_dev), batch,
                                                C.c_float(lr)), "cnn_backward")

    def train_step(self, x_dev, t_dev, batch, lr):
        loss = C.c_float()
        L.check(self.lib.verb_cnn_train_step(self.h, C.c_void_p(x_dev), C.c_void_p(t_dev), batch,
                                             C.c_float(lr), C.byref(loss)), "cnn_train")
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.verb_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
