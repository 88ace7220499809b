"""The mixed-precision form of the local (V,K) solve against the FP64 form.

The FP64 form is checked bit for bit against the oracle elsewhere; here the
mixed form (the same factorisation stored in FP32, each solve refined in FP64)
is compared with it on the same inputs, one local solve from the same state.
Each refinement step multiplies the error by roughly kappa * eps32; the
seeded 24 x 25 x 31 x 31 systems have condition numbers up to ~1e7, so FP32
factors alone leave errors up to ~0.1 and the worst system needs eight to ten
refinement steps to reach the 1e-8 relative tolerance the mixed form is held
to (norm-wise: max |diff| / max |psd|).  Both forms pick the same pivots (the
factorisation arithmetic is FP64 in both) and the mixed form needs half the
factor memory.

Whole runs are compared one step at a time: convection's limiter is
discontinuous in its inputs, so any perturbation of the PSD (a different
rounding anywhere) grows to ~1e-6 over a dozen steps, for any two paths
that are not bit-identical.
"""
import numpy as np
import pytest

from verb4d_b200 import workload as W

from test_gpu_step import load_ctx

pytestmark = pytest.mark.gpu
MIXED_RTOL = 1e-8


def local_steps(wl, mode, refinements, steps=2):
    c = load_ctx(wl)
    c.set_local_precision(mode, refinements)
    for _ in range(steps):
        c.local(wl.dt, wl.sub_dt)
    c.sync()
    out = (c.download(), c.local_pivots(), c.device_bytes(), c.local_refinement())
    c.close()
    return out


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_mixed_local_solve_converges_to_fp64(gpu):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=3, sources=True, losses=True)
    ref, piv, mem64, corr64 = local_steps(wl, "fp64", 0, steps=1)
    assert corr64 == 0.0
    errs, corrs = [], []
    for nref in (0, 2, 4, 10):
        psd, piv32, mem32, corr = local_steps(wl, "mixed", nref, steps=1)
        errs.append(rel(psd, ref))
        corrs.append(corr)
        assert np.array_equal(piv32, piv)
        assert mem32 < mem64
    # FP32 factors alone leave an error of order kappa * eps32; refinement
    # shrinks it until it reaches the FP64 path's own rounding (kappa * eps64,
    # ~3e-10 here), after which the corrections keep shrinking but the
    # distance to the FP64 path stays
    assert errs[0] > 1e-6
    assert errs[1] < 1e-3 * errs[0]
    assert max(errs[1:]) < MIXED_RTOL
    assert corrs[1] > corrs[3]


def test_mixed_production_band(gpu):
    # the production band (V = 101, kl = 102: 13 x 7 register slots per thread)
    # on short systems: FP32 factors parked and stored in the FP32 L/U arrays
    wl = W.make_workload(W.GridSpec(4, 6, 101, 6), seed=7, sources=True, losses=True)
    ref, piv, mem64, _ = local_steps(wl, "fp64", 0, steps=1)
    psd, piv32, mem32, _ = local_steps(wl, "mixed", 10, steps=1)
    assert np.array_equal(piv32, piv)
    assert mem32 < mem64
    assert rel(psd, ref) < MIXED_RTOL


def test_fp64_refinement(gpu):
    # FP64 factors plus FP64 refinement: the corrections are at the FP64
    # path's rounding level and the result stays within it
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=3, sources=True, losses=True)
    ref = local_steps(wl, "fp64", 0, steps=1)[0]
    psd, _, _, corr = local_steps(wl, "fp64", 2, steps=1)
    assert rel(psd, ref) < MIXED_RTOL
    assert corr < 1e-8


def test_mixed_whole_step_within_tolerance(gpu):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=4)
    res = {}
    for mode in ("fp64", "mixed"):
        c = load_ctx(wl)
        c.set_local_precision(mode, 10)
        c.step(wl.dt, wl.sub_dt)
        c.sync()
        res[mode] = c.download()
        c.close()
    assert rel(res["mixed"], res["fp64"]) < MIXED_RTOL


def test_switching_precision_refactors(gpu):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=5)
    c = load_ctx(wl)
    c.set_local_precision("mixed", 10)
    c.local(wl.dt, wl.sub_dt)
    c.set_local_precision("fp64", 0)
    c.local(wl.dt, wl.sub_dt)
    c.sync()
    two = c.download()
    c.close()
    ref = local_steps(wl, "fp64", 0, steps=1)[0]
    c = load_ctx(wl)
    c.upload("psd", ref)
    c.local(wl.dt, wl.sub_dt)
    c.sync()
    ref2 = c.download()
    c.close()
    # the first step ran mixed, the second on fresh FP64 factors
    assert rel(two, ref2) < MIXED_RTOL
