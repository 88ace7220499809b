"""Whole operator-split steps on the GPU (device-resident context, C ABI)
against the CPU oracle.

The GPU path restates every routine operation by operation (no FMA
contraction), so at the small sizes the oracle finishes in seconds the PSD is
compared bit for bit, and the negative-point count, pivots and convection
sub-step counts exactly.  At the production size (101 L x 101 E x 91 alpha x
48 MLT) the same per-slice equality is checked on sampled slices after each
phase, plus size-independent properties of the local solve.
"""
import os

import numpy as np
import pytest

import oracle as O
from verb4d_b200 import Context
from verb4d_b200 import workload as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
# exp(Loss_conv*dt) uses CUDA's exp on the device and the host libm in the
# oracle (one-ulp differences), so steps with convection loss rates agree to
# rounding; everything else is compared bit for bit.
EXP_RTOL = 1e-13


def without_conv_loss(wl):
    wl.fields["loss_conv"] = np.zeros_like(wl.fields["loss_conv"])
    return wl


def load_ctx(wl):
    P, R, V, K = wl.spec.shape
    c = Context(P, R, V, K)
    c.set_bc_types(wl.bc_types)
    fl = wl.flags
    c.set_options(fl["radial_sources"], fl["local_sources"], fl["include_boundary"],
                  fl["positive_psd"])
    for k in ("psd", "Pg", "Rg", "Vg", "Kg", "Lg", "DLL", "DVV", "DKK", "DVK", "VP", "VR", "G_local",
              "G_radial", "G_conv", "S", "loss_local", "loss_radial", "loss_conv"):
        c.upload(k, wl.fields[k])
    for k in ("Pl", "Pu", "Rl", "Ru", "Ll", "Lu", "Vl", "Vu", "Kl", "Ku"):
        c.upload(k, wl.fields[k])
    return c


def test_small_grid_steps_bitexact(gpu, oracle_lib):
    import make_golden as MG

    wl = without_conv_loss(MG.step_workload())
    c = load_ctx(wl)
    st = O.OracleStepper(W.oracle_inputs(wl), oracle_lib)
    for k in range(3):
        n_gpu = c.step(wl.dt, wl.sub_dt, count_negatives=True)
        c.sync()
        n_orc = st.step(wl.dt, wl.sub_dt, k == 0)
        psd = c.download()
        assert np.array_equal(psd, st.psd), f"step {k}: max diff {np.abs(psd - st.psd).max()}"
        assert n_gpu == n_orc
    c.close()


def test_small_grid_steps_vs_reference_fixture(gpu, oracle_lib):
    import make_golden as MG

    wl = MG.step_workload()
    c = load_ctx(wl)
    st = O.OracleStepper(W.oracle_inputs(wl), oracle_lib)
    g = np.load(os.path.join(GOLD, "step.npz"))
    for k in range(2):
        c.step(wl.dt, wl.sub_dt)
        c.sync()
        st.step(wl.dt, wl.sub_dt, k == 0)
        psd = c.download()
        assert np.abs(psd - st.psd).max() / np.abs(st.psd).max() < EXP_RTOL
        ref = g[f"psd{k + 1}"]  # the reference-driven fixture (LU rounding-level tolerance)
        assert np.abs(psd - ref).max() / np.abs(ref).max() < 1e-10
    P, R, V, K = wl.spec.shape
    assert np.array_equal(c.local_pivots().reshape(P * R, V * K), st.ipiv.reshape(P * R, V * K))
    assert np.array_equal(c.local_pivots().reshape(P * R, V * K) + 1, g["ipiv"])
    c.close()


def test_phases_separately(gpu, oracle_lib):
    wl = without_conv_loss(W.make_workload(W.GridSpec(14, 15, 12, 13), seed=21, sources=True,
                                           losses=True))
    wl.fields["VP"] = wl.fields["VP"] * 3e-3
    inp = W.oracle_inputs(wl)
    for phase in ("convection", "radial", "local"):
        c = load_ctx(wl)
        flags = dict(wl.flags, run_convection=int(phase == "convection"),
                     run_radial=int(phase == "radial"), run_local=int(phase == "local"))
        st = O.OracleStepper(dict(inp, flags=flags), oracle_lib)
        c.step(wl.dt, wl.sub_dt, phase == "convection", phase == "radial", phase == "local")
        c.sync()
        st.step(wl.dt, wl.sub_dt, True)
        assert np.array_equal(c.download(), st.psd), phase
        if phase == "convection":
            assert np.array_equal(c.convection_substeps(), W.convection_substeps(wl))
        c.close()


def test_sub_steps_and_options(gpu, oracle_lib):
    # two local sub-steps, sources routed to the radial step, positive_PSD clamp,
    # and include_boundary = false (src/VERB4D_Solver.cpp:1117)
    wl = without_conv_loss(W.make_workload(W.GridSpec(12, 12, 11, 11), seed=4, sources=True,
                                           losses=True))
    wl.fields["VP"] = wl.fields["VP"] * 3e-3
    wl.sub_dt = wl.dt / 2.0
    wl.flags.update(radial_sources=1, local_sources=0, include_boundary=0, positive_psd=1)
    c = load_ctx(wl)
    st = O.OracleStepper(W.oracle_inputs(wl), oracle_lib)
    for k in range(2):
        c.step(wl.dt, wl.sub_dt)
        c.sync()
        st.step(wl.dt, wl.sub_dt, k == 0)
        assert np.array_equal(c.download(), st.psd)
    assert c.download().min() >= 1e-21
    c.close()


def test_cfg1_step_bitexact(gpu, oracle_lib):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=1)
    c = load_ctx(wl)
    st = O.OracleStepper(W.oracle_inputs(wl), oracle_lib)
    n_gpu = c.step(wl.dt, wl.sub_dt, count_negatives=True)
    c.sync()
    n_orc = st.step(wl.dt, wl.sub_dt, True)
    assert np.array_equal(c.download(), st.psd)
    assert n_gpu == n_orc
    assert np.array_equal(c.convection_substeps(), W.convection_substeps(wl))
    c.close()


def test_wide_band_local_step_bitexact(gpu, oracle_lib):
    """V = 111 energies (band kl = 112, the widest the context accepts): wider
    than the register-window factorisation holds, so the shared-memory-window
    kernel factors; one local step on every system, pivots and PSD equal to the
    oracle bit for bit."""
    wl = W.make_workload(W.GridSpec(2, 3, 111, 4), seed=6, sources=True, losses=True)
    f = wl.fields
    P, R, V, K = wl.spec.shape
    c = load_ctx(wl)
    psd0 = c.download()
    c.local(wl.dt, wl.sub_dt)
    c.sync()
    psd1 = c.download()
    piv = c.local_pivots()
    c.close()
    n = V * K
    ldab = 3 * (V + 1) + 1
    for iP in range(P):
        for iR in range(R):
            s2 = lambda a: a[iP, iR]  # noqa: E731
            lu, ip = np.zeros(ldab * n), np.zeros(n, np.int64)
            _, ref = oracle_lib.diffusion_2d(s2(psd0), s2(f["Vg"]), s2(f["Kg"]), f["Vl"][iP, iR],
                                             f["Vu"][iP, iR], f["Kl"][iP, iR], f["Ku"][iP, iR],
                                             (1, 1, 2, 2), s2(f["DVV"]), s2(f["DKK"]), s2(f["DVK"]),
                                             s2(f["DVK"]), s2(f["G_local"]), s2(f["S"]),
                                             s2(f["loss_local"]), wl.dt, wl.sub_dt, lu=lu, ipiv=ip)
            assert np.array_equal(piv[iP, iR], ip), (iP, iR)
            assert np.array_equal(psd1[iP, iR], ref), (iP, iR)


def test_dll_scale_matches_scaled_field(gpu):
    # UpdatableMatrix scale (src/UpdatableMatrix.cpp:698-708): base * scale
    wl = W.make_workload(W.GridSpec(6, 12, 5, 5), seed=8)
    c1, c2 = load_ctx(wl), load_ctx(wl)
    c1.upload("DLL", wl.fields["DLL"])
    c1.set_scale("DLL", 3.7)
    c2.upload("DLL", wl.fields["DLL"] * 3.7)
    for c in (c1, c2):
        c.step(wl.dt, wl.sub_dt, False, True, False)
        c.sync()
    assert np.array_equal(c1.download(), c2.download())
    assert np.array_equal(c1.download("DLL"), c2.download("DLL"))
    c1.close()
    c2.close()


def test_production_size_sampled_slices(gpu, oracle_lib):
    """101 x 101 x 91 x 48: phase by phase, sampled slices must equal the oracle bit for bit."""
    wl = W.make_workload(W.CONFIGS["cfg2"], seed=2)
    f = wl.fields
    P, R, V, K = wl.spec.shape
    c = load_ctx(wl)
    rng = np.random.default_rng(0)
    psd0 = f["psd"]

    c.convection(wl.dt)
    c.sync()
    psd1 = c.download()
    ns = c.convection_substeps()
    assert np.array_equal(ns, W.convection_substeps(wl))
    for iV, iK in [(V - 1, 0), (V // 2, K // 3), (3, K - 1)]:
        sl = lambda a: np.ascontiguousarray(a[:, :, iV, iK])  # noqa: E731
        _, ref, n_ref = oracle_lib.convection_2d(
            sl(psd0), sl(f["Pg"]), sl(f["Rg"]), f["Pl"][:, iV, iK], f["Pu"][:, iV, iK],
            f["Rl"][:, iV, iK], f["Ru"][:, iV, iK], (0, 0, 1, 1), sl(f["VP"]), sl(f["VR"]),
            sl(f["S"]), sl(f["loss_conv"]), sl(f["G_conv"]), wl.dt)
        assert n_ref == ns[iV, iK]
        assert np.array_equal(psd1[:, :, iV, iK], ref), (iV, iK)

    c.radial(wl.dt)
    c.sync()
    psd2 = c.download()
    for _ in range(64):
        iP, iV, iK = rng.integers(0, P), rng.integers(0, V), rng.integers(0, K)
        ln = lambda a: a[iP, :, iV, iK]  # noqa: E731
        _, ref = oracle_lib.diffusion_1d(ln(psd1), ln(f["Lg"]), f["Ll"][iP, iV, iK],
                                         f["Lu"][iP, iV, iK], 1, 1, ln(f["DLL"]), ln(f["G_radial"]),
                                         ln(f["S"]) * 0.0, ln(f["loss_radial"]), wl.dt)
        assert np.array_equal(psd2[iP, :, iV, iK], ref)

    c.local(wl.dt, wl.sub_dt)
    c.sync()
    psd3 = c.download()
    piv = c.local_pivots()
    for iP, iR in [(0, 0), (P // 2, R // 2), (P - 1, R - 2)]:
        s2 = lambda a: a[iP, iR]  # noqa: E731
        n = V * K
        ldab = 3 * (V + 1) + 1
        lu, ip = np.zeros(ldab * n), np.zeros(n, np.int64)
        _, ref = oracle_lib.diffusion_2d(s2(psd2), s2(f["Vg"]), s2(f["Kg"]), f["Vl"][iP, iR],
                                         f["Vu"][iP, iR], f["Kl"][iP, iR], f["Ku"][iP, iR],
                                         (1, 1, 2, 2), s2(f["DVV"]), s2(f["DKK"]), s2(f["DVK"]),
                                         s2(f["DVK"]), s2(f["G_local"]), s2(f["S"]),
                                         s2(f["loss_local"]), wl.dt, wl.sub_dt, lu=lu, ipiv=ip)
        assert np.array_equal(piv[iP, iR], ip), (iP, iR)
        assert np.array_equal(psd3[iP, iR], ref), (iP, iR)
    # a second local step reuses the cached factors: still equal to the oracle
    c.local(wl.dt, wl.sub_dt)
    c.sync()
    psd4 = c.download()
    iP, iR = P // 3, R // 4
    s2 = lambda a: a[iP, iR]  # noqa: E731
    n = V * K
    lu, ip = np.zeros((3 * (V + 1) + 1) * n), np.zeros(n, np.int64)
    args = (s2(f["Vg"]), s2(f["Kg"]), f["Vl"][iP, iR], f["Vu"][iP, iR], f["Kl"][iP, iR],
            f["Ku"][iP, iR], (1, 1, 2, 2), s2(f["DVV"]), s2(f["DKK"]), s2(f["DVK"]), s2(f["DVK"]),
            s2(f["G_local"]), s2(f["S"]), s2(f["loss_local"]), wl.dt, wl.sub_dt)
    _, r1 = oracle_lib.diffusion_2d(s2(psd2), *args, lu=lu, ipiv=ip)
    _, r2 = oracle_lib.diffusion_2d(r1, *args, lu=lu, ipiv=ip, recompute=False)
    assert np.array_equal(psd4[iP, iR], r2)
    assert c.negative_count() == int((psd4 < 0).sum())
    c.close()
