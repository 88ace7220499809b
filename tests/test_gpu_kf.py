"""Batched radial Kalman-filter update on the GPU against the reference
fixtures and the CPU oracle (runKalmanFilterDiffusion1D,
src/DataAssimilationDiffusion.cpp:151-253).  The GPU forms F = B A^-1 from
tridiagonal solves and uses tiled FMA products where the reference calls
dgesv/dgemm, so results agree to rounding; the tolerance is norm-wise."""
import os

import numpy as np
import pytest

from verb4d_b200 import Context
from verb4d_b200 import workload as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
KF_RTOL = 1e-10


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_kf_columns_vs_reference(gpu):
    gold = dict(np.load(os.path.join(GOLD, "slices.npz")))
    for c in range(3):
        g = {k[len(f"kf_{c}_"):]: v for k, v in gold.items() if k.startswith(f"kf_{c}_")}
        n = len(g["x0"])
        ctx = Context(1, n, 1, 1)
        ctx.set_bc_types(dict(Pl=0, Pu=0, Rl=1, Ru=1, Ll=int(g["lbc_t"]), Lu=int(g["ubc_t"]), Vl=1,
                              Vu=1, Kl=1, Ku=1))
        ctx.upload("psd", g["x0"])
        ctx.upload("Rg", g["R"])
        ctx.upload("DLL", g["DLL"])
        ctx.upload("G_radial", g["G"])
        ctx.upload("Ll", np.array([float(g["lbc"])]))
        ctx.upload("Lu", np.array([float(g["ubc"])]))
        obs = g["obs"].reshape(1, n, 1, 1)
        ctx.assimilate_radial(obs, float(g["dt"]), float(g["model_error"]), float(g["obs_error"]))
        ctx.sync()
        assert rel(ctx.download().ravel(), g["x1"]) < KF_RTOL, c
        ctx.assimilate_radial(obs, float(g["dt"]), float(g["model_error"]), float(g["obs_error"]))
        ctx.sync()
        assert rel(ctx.download().ravel(), g["x2"]) < KF_RTOL, c
        ctx.close()


def test_kf_batched_columns_vs_oracle(gpu, oracle_lib):
    spec = W.GridSpec(3, 31, 5, 4)
    wl = W.make_workload(spec, seed=13)
    f = wl.fields
    rng = np.random.default_rng(5)
    obs = np.full(spec.shape, np.nan)
    idx = rng.choice(spec.npts, size=200, replace=False)
    obs.ravel()[idx] = f["psd"].ravel()[idx] * np.exp(0.05 * rng.standard_normal(200))
    obs[:, 0] = np.nan
    obs[:, -1] = np.nan
    ctx = Context(*spec.shape)
    ctx.set_bc_types(wl.bc_types)
    for k in ("psd", "Rg", "DLL", "G_radial", "Ll", "Lu"):
        ctx.upload(k, f[k])
    me, oe = 1e-4, 1e-3
    ctx.assimilate_radial(obs, wl.dt, me, oe, p_index=-1)
    ctx.sync()
    out = ctx.download()
    for p in range(3):
        for v in range(5):
            for k in range(4):
                ln = lambda a: a[p, :, v, k]  # noqa: E731
                st, x1, *_ = oracle_lib.kf_diffusion_1d(
                    ln(f["psd"]), np.zeros((31, 31)), ln(f["Rg"]), ln(f["DLL"]), ln(f["G_radial"]),
                    float(f["Ll"][p, v, k]), float(f["Lu"][p, v, k]), 1, 1, ln(obs), wl.dt, me, oe)
                assert st == 0
                assert rel(out[p, :, v, k], x1) < KF_RTOL, (p, v, k)
    ctx.close()
