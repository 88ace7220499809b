"""The streaming convection kernel (verb_set_convection_arith "stream", one
thread per line, all four stages of a QUICKEST pass in register windows)
against the oracle.

Like the contracted kernel it rounds fused multiply-adds once and takes the
limiter's reference value with the rounded reciprocal of |c|, so a step is
held to the FP64 tolerance of 1e-12 relative (max |diff| over max |psd|, and
pointwise where |psd| is above 1e-6 of its maximum) after one convection
step; the CFL sub-step counts are integer work and stay exact.  Covered: the
small grid with sources and loss rates, sampled slices of the 101 x 101 x 91
x 48 production grid, every boundary-type combination of the MLT and L lines
(periodic L runs whole lines, the others split each L line into two
segments), L lines with their own CFL sub-cycles (whole lines, several passes
per sub-step), and the shapes the kernel leaves to the contracted kernel.
"""
import numpy as np
import pytest

import oracle as O
from verb4d_b200 import workload as W

from test_gpu_step import load_ctx

pytestmark = pytest.mark.gpu
TOL = 1e-12
BCS = {"periodic": 0, "value": 1, "deriv": 2}


def close(got, ref):
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= TOL * scale
    big = np.abs(ref) > 1e-6 * scale
    assert np.all(np.abs(got - ref)[big] <= TOL * np.abs(ref)[big])


def conv_step(wl, oracle_lib, mode="stream"):
    inp = W.oracle_inputs(wl)
    flags = dict(wl.flags, run_convection=1, run_radial=0, run_local=0)
    st = O.OracleStepper(dict(inp, flags=flags), oracle_lib)
    st.step(wl.dt, wl.sub_dt, True)
    c = load_ctx(wl)
    c.set_convection_arith(mode)
    c.step(wl.dt, wl.sub_dt, True, False, False)
    c.sync()
    got = c.download()
    ns = c.convection_substeps()
    c.close()
    return got, st.psd, ns


def test_stream_step_small_grid(gpu, oracle_lib):
    wl = W.make_workload(W.GridSpec(14, 15, 12, 13), seed=31, sources=True, losses=True)
    wl.fields["VP"] = wl.fields["VP"] * 3e-3
    got, ref, ns = conv_step(wl, oracle_lib)
    assert np.array_equal(ns, W.convection_substeps(wl))
    close(got, ref)
    assert not np.array_equal(got, ref)   # the contracted kernel really ran


def test_stream_production_slices(gpu, oracle_lib):
    wl = W.make_workload(W.CONFIGS["cfg2"], seed=2)
    f = wl.fields
    P, R, V, K = wl.spec.shape
    c = load_ctx(wl)
    c.set_convection_arith("stream")
    c.convection(wl.dt)
    c.sync()
    psd1 = c.download()
    ns = c.convection_substeps()
    c.close()
    assert np.array_equal(ns, W.convection_substeps(wl))
    for iV, iK in [(V - 1, 0), (V // 2, K // 3), (3, K - 1), (V - 7, K // 2)]:
        sl = lambda a: np.ascontiguousarray(a[:, :, iV, iK])  # noqa: E731
        _, ref, n_ref = oracle_lib.convection_2d(
            sl(f["psd"]), sl(f["Pg"]), sl(f["Rg"]), f["Pl"][:, iV, iK], f["Pu"][:, iV, iK],
            f["Rl"][:, iV, iK], f["Ru"][:, iV, iK], (0, 0, 1, 1), sl(f["VP"]), sl(f["VR"]),
            sl(f["S"]), sl(f["loss_conv"]), sl(f["G_conv"]), wl.dt)
        assert n_ref == ns[iV, iK]
        close(psd1[:, :, iV, iK], ref)


@pytest.mark.parametrize("pbc,rl,ru", [
    ("periodic", "value", "deriv"), ("periodic", "deriv", "value"), ("periodic", "deriv", "deriv"),
    ("periodic", "periodic", "periodic"), ("value", "value", "value"), ("deriv", "value", "deriv"),
])
def test_stream_boundary_types(gpu, oracle_lib, pbc, rl, ru):
    # R = 40 >= 32: non-periodic L lines run as two segments of 20 cells
    wl = W.make_workload(W.GridSpec(14, 40, 5, 4), seed=44, sources=True, losses=True)
    f = wl.fields
    wl.bc_types.update(Pl=BCS[pbc], Pu=BCS[pbc], Rl=BCS[rl], Ru=BCS[ru])
    if pbc != "periodic":
        rng = np.random.default_rng(3)
        f["Pl"] = rng.uniform(0.0, 0.5, f["Pl"].shape)
        f["Pu"] = rng.uniform(0.0, 0.5, f["Pu"].shape)
    if rl == "deriv":
        f["Rl"] = np.full(f["Rl"].shape, 0.05)
    if ru == "deriv":
        f["Ru"] = np.full(f["Ru"].shape, -0.03)
    got, ref, ns = conv_step(wl, oracle_lib)
    assert np.array_equal(ns, W.convection_substeps(wl))
    close(got, ref)


def test_stream_lines_with_own_subcycles(gpu, oracle_lib):
    # L spacing shrinking along MLT: the slice-level Courant limit leaves L
    # lines above Courant 1, which sub-cycle on their own (whole lines)
    wl = W.make_workload(W.GridSpec(14, 40, 5, 4), seed=5, sources=True, losses=True)
    Rg = wl.fields["Rg"].copy()
    nP = Rg.shape[0]
    for iP in range(nP):
        fac = 1.0 / (1.0 + 7.0 * iP / (nP - 1))
        Rg[iP] = Rg[0, 0] + (Rg[0] - Rg[0, 0]) * fac
    wl.fields["Rg"] = Rg
    wl.fields["Lg"] = Rg.copy()
    got, ref, ns = conv_step(wl, oracle_lib)
    assert np.array_equal(ns, W.convection_substeps(wl))
    close(got, ref)


def test_stream_short_mlt_runs_contracted_kernel(gpu):
    # P = 2: no MLT sweep, which the streaming kernel needs; it runs the
    # contracted kernel instead, bit for bit
    wl = W.make_workload(W.GridSpec(2, 15, 6, 5), seed=9, sources=True, losses=True)
    out = {}
    for mode in ("fma", "stream"):
        c = load_ctx(wl)
        c.set_convection_arith(mode)
        c.convection(wl.dt)
        c.sync()
        out[mode] = c.download()
        c.close()
    assert np.array_equal(out["fma"], out["stream"])
