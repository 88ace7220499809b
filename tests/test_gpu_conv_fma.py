"""The contracted-arithmetic convection (verb_set_convection_arith "fma")
against the oracle.

The same kernel compiled with multiply-add contraction rounds each fused
pair once instead of twice, so a step no longer equals the reference bit for
bit; it is held to the FP64 tolerance of 1e-12 relative (max |diff| over
max |psd|, and pointwise where |psd| is above 1e-6 of its maximum) after
one convection step, on the small grid with sources and loss rates and on
sampled slices of the 101 x 101 x 91 x 48 production grid.  The CFL
sub-step counts are integer work and stay exact.  Runs are compared one
step at a time: the limiter's switches are discontinuous in their inputs,
so any two paths that are not bit-identical drift apart over many steps.
"""
import numpy as np
import pytest

import oracle as O
from verb4d_b200 import workload as W

from test_gpu_step import load_ctx

pytestmark = pytest.mark.gpu
TOL = 1e-12


def close(got, ref):
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= TOL * scale
    big = np.abs(ref) > 1e-6 * scale
    assert np.all(np.abs(got - ref)[big] <= TOL * np.abs(ref)[big])


def test_fma_convection_step_small_grid(gpu, oracle_lib):
    wl = W.make_workload(W.GridSpec(14, 15, 12, 13), seed=31, sources=True, losses=True)
    wl.fields["VP"] = wl.fields["VP"] * 3e-3
    inp = W.oracle_inputs(wl)
    flags = dict(wl.flags, run_convection=1, run_radial=0, run_local=0)
    st = O.OracleStepper(dict(inp, flags=flags), oracle_lib)
    st.step(wl.dt, wl.sub_dt, True)
    c = load_ctx(wl)
    c.set_convection_arith("fma")
    c.step(wl.dt, wl.sub_dt, True, False, False)
    c.sync()
    got = c.download()
    assert np.array_equal(c.convection_substeps(), W.convection_substeps(wl))
    c.close()
    close(got, st.psd)
    assert not np.array_equal(got, st.psd)   # the contracted kernel really ran


def test_fma_convection_production_slices(gpu, oracle_lib):
    wl = W.make_workload(W.CONFIGS["cfg2"], seed=2)
    f = wl.fields
    P, R, V, K = wl.spec.shape
    c = load_ctx(wl)
    c.set_convection_arith("fma")
    c.convection(wl.dt)
    c.sync()
    psd1 = c.download()
    ns = c.convection_substeps()
    c.close()
    assert np.array_equal(ns, W.convection_substeps(wl))
    for iV, iK in [(V - 1, 0), (V // 2, K // 3), (3, K - 1)]:
        sl = lambda a: np.ascontiguousarray(a[:, :, iV, iK])  # noqa: E731
        _, ref, n_ref = oracle_lib.convection_2d(
            sl(f["psd"]), sl(f["Pg"]), sl(f["Rg"]), f["Pl"][:, iV, iK], f["Pu"][:, iV, iK],
            f["Rl"][:, iV, iK], f["Ru"][:, iV, iK], (0, 0, 1, 1), sl(f["VP"]), sl(f["VR"]),
            sl(f["S"]), sl(f["loss_conv"]), sl(f["G_conv"]), wl.dt)
        assert n_ref == ns[iV, iK]
        close(psd1[:, :, iV, iK], ref)


def test_arith_mode_switch(gpu):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=32)
    out = {}
    for mode in ("exact", "fma", "exact"):
        c = load_ctx(wl)
        c.set_convection_arith(mode)
        c.convection(wl.dt)
        c.sync()
        out.setdefault(mode, []).append(c.download())
        c.close()
    assert np.array_equal(out["exact"][0], out["exact"][1])
    close(out["fma"][0], out["exact"][0])
