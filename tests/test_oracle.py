"""Pins the CPU oracle (oracle/verb_oracle.c) to the reference.

Against the committed golden fixtures (made by the reference's own routines,
tests/golden/make_golden.py) and, when the reference has been compiled here
(oracle/_ref), against the reference on fresh seeded inputs.  Radial
diffusion, tridag and convection must be bit-identical; the banded LU agrees
to rounding (the reference links OpenBLAS's blocked dgbtrf, the oracle
restates the unblocked algorithm) with identical pivots.
"""
import os

import numpy as np
import pytest

import oracle as O
from verb4d_b200 import workload as W

GOLD = os.path.join(os.path.dirname(__file__), "golden")
LOCAL_RTOL = 1e-12  # norm-wise relative tolerance for one LU-based slice solve
# Whole steps on the stiff synthetic coefficients (log-normal D over a decade,
# kappa(A) ~ 1e5) differ from OpenBLAS's blocked, FMA-using dgbtrf at the
# kappa*eps level; near-zero PSD values (|f| ~ 1e-20 on an O(1) field) can then
# change sign, so negative-point counts agree to a few percent only.
STEP_RTOL = 1e-10
NEG_RTOL = 0.05


def rel(a, b, scale=None):
    """max|a-b| / max|b| (or / scale): the norm-wise relative error."""
    s = np.abs(np.asarray(b)).max() if scale is None else scale
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(s, 1e-300)


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(GOLD, "slices.npz")))


def test_radial_lines_bitexact(oracle_lib, gold):
    for c in range(4):
        g = {k[len(f"d1_{c}_"):]: v for k, v in gold.items() if k.startswith(f"d1_{c}_")}
        st, out = oracle_lib.diffusion_1d(g["psd"], g["x"], float(g["lbc"]), float(g["ubc"]),
                                          int(g["lbc_t"]), int(g["ubc_t"]), g["D"], g["G"], g["S"],
                                          g["loss"], float(g["dt"]))
        assert st == 0
        assert np.array_equal(out, g["out"]), c


def test_tridag_bitexact(oracle_lib, gold):
    u = oracle_lib.tridag(gold["tri_a"], gold["tri_b"], gold["tri_c"], gold["tri_r"])
    assert np.array_equal(u, gold["tri_out"])


def test_local_slices_and_pivots(oracle_lib, gold):
    for c in range(3):
        g = {k[len(f"d2_{c}_"):]: v for k, v in gold.items() if k.startswith(f"d2_{c}_")}
        n = g["psd"].size
        lu = np.zeros_like(g["lu"])
        ip = np.zeros(n, dtype=np.int64)
        st, out = oracle_lib.diffusion_2d(g["psd"], g["x"], g["y"], g["xl"], g["xu"], g["yl"],
                                          g["yu"], tuple(int(t) for t in g["types"]), g["Dxx"],
                                          g["Dyy"], g["Dxy"], g["Dyx"], g["G"], g["S"], g["loss"],
                                          float(g["dt"]), float(g["sub_dt"]), lu=lu, ipiv=ip)
        assert st == 0
        assert np.array_equal(ip + 1, g["ipiv"]), "pivot rows differ from LAPACK dgbtrf"
        assert rel(out, g["out"]) < LOCAL_RTOL
        assert rel(lu, g["lu"]) < 1e-13


def test_convection_bitexact(oracle_lib, gold):
    for c in range(4):
        lb, ub, lt, ut = gold[f"c1_{c}_bc"]
        st, out = oracle_lib.convection_1d(gold[f"c1_{c}_psd"], gold[f"c1_{c}_x"], lb, ub, int(lt),
                                           int(ut), gold[f"c1_{c}_ux"], W.DT_5MIN)
        assert st == 0
        assert np.array_equal(out, gold[f"c1_{c}_out"]), c
    for c in range(3):
        g = {k[len(f"c2_{c}_"):]: v for k, v in gold.items() if k.startswith(f"c2_{c}_")}
        st, out, ns = oracle_lib.convection_2d(g["psd"], g["P"], g["R"], g["pl"], g["pu"], g["rl"],
                                               g["ru"], (0, 0, 1, 1), g["VP"], g["VR"], g["S"],
                                               g["loss"], g["G"], float(g["dt"]))
        assert st == 0 and ns >= 1
        assert np.array_equal(out, g["out"]), c


def test_kalman_filter(oracle_lib, gold):
    for c in range(3):
        g = {k[len(f"kf_{c}_"):]: v for k, v in gold.items() if k.startswith(f"kf_{c}_")}
        args = (g["R"], g["DLL"], g["G"], float(g["lbc"]), float(g["ubc"]), int(g["lbc_t"]),
                int(g["ubc_t"]), g["obs"], float(g["dt"]), float(g["model_error"]),
                float(g["obs_error"]))
        st, x1, pa1, F, Pf = oracle_lib.kf_diffusion_1d(g["x0"], np.zeros_like(g["Pa1"]), *args)
        assert st == 0
        assert rel(F, g["F"]) < 1e-12
        assert rel(Pf, g["Pf"]) < 1e-12
        # Pa = Pf - K H Pf cancels near observed points: measure it on the scale of Pf
        pscale = np.abs(g["Pf"]).max()
        assert rel(pa1, g["Pa1"], pscale) < 1e-12
        assert rel(x1, g["x1"]) < 1e-12
        st, x2, pa2, _, _ = oracle_lib.kf_diffusion_1d(x1, pa1, *args)
        assert rel(x2, g["x2"]) < 1e-12 and rel(pa2, g["Pa2"], pscale) < 1e-12


def test_whole_step_matches_reference_driver(oracle_lib):
    import make_golden as MG

    g = np.load(os.path.join(GOLD, "step.npz"))
    wl = MG.step_workload()
    sums = np.array([wl.fields[k].sum() for k in sorted(wl.fields)])
    assert np.array_equal(sums, g["input_sums"]), "workload generator drifted from the fixture"
    st = O.OracleStepper(W.oracle_inputs(wl), oracle_lib)
    n1 = st.step(wl.dt, wl.sub_dt, True)
    assert abs(n1 - int(g["neg"][0])) <= NEG_RTOL * int(g["neg"][0])
    assert rel(st.psd, g["psd1"]) < STEP_RTOL
    assert np.array_equal(st.ipiv.reshape(g["ipiv"].shape) + 1, g["ipiv"])
    n2 = st.step(wl.dt, wl.sub_dt, False)
    assert abs(n2 - int(g["neg"][1])) <= NEG_RTOL * int(g["neg"][1])
    assert rel(st.psd, g["psd2"]) < STEP_RTOL


@pytest.mark.skipif(not O.have_reference(), reason="reference not compiled here (oracle/_ref)")
def test_oracle_vs_reference_fresh_inputs(oracle_lib):
    ref = O.reference()
    ref_lu = O.reference(lu_caching=True)
    rng = np.random.default_rng(1234)
    wl = W.make_workload(W.GridSpec(16, 21, 13, 14), seed=77, sources=True, losses=True)
    f = wl.fields
    for _ in range(5):
        iP, iV, iK = rng.integers(0, 16), rng.integers(0, 13), rng.integers(0, 14)
        ln = lambda a: a[iP, :, iV, iK]  # noqa: E731
        a = (ln(f["Lg"]), 0.0, float(f["Lu"][iP, iV, iK]), 1, 1, ln(f["DLL"]) * 1e4,
             ln(f["G_radial"]), ln(f["S"]), ln(f["loss_local"]), wl.dt)
        assert np.array_equal(oracle_lib.diffusion_1d(ln(f["psd"]), *a)[1],
                              ref.diffusion_1d(ln(f["psd"]), *a)[1])
        sl = lambda a: np.ascontiguousarray(a[:, :, iV, iK])  # noqa: E731
        ca = (sl(f["Pg"]), sl(f["Rg"]), f["Pl"][:, iV, iK], f["Pu"][:, iV, iK], f["Rl"][:, iV, iK],
              f["Ru"][:, iV, iK], (0, 0, 1, 1), sl(f["VP"]) * 0.1, sl(f["VR"]), sl(f["S"]),
              sl(f["loss_conv"]), sl(f["G_conv"]), wl.dt)
        assert np.array_equal(oracle_lib.convection_2d(sl(f["psd"]), *ca)[1],
                              ref.convection_2d(sl(f["psd"]), *ca)[1])
        iR = rng.integers(0, 21)
        s2 = lambda a: a[iP, iR]  # noqa: E731
        la = (s2(f["Vg"]), s2(f["Kg"]), f["Vl"][iP, iR], f["Vu"][iP, iR], f["Kl"][iP, iR],
              f["Ku"][iP, iR], (1, 1, 2, 2), s2(f["DVV"]), s2(f["DKK"]), s2(f["DVK"]), s2(f["DVK"]),
              s2(f["G_local"]), s2(f["S"]), s2(f["loss_local"]), wl.dt, wl.dt)
        n = 13 * 14
        ldab = 3 * 14 + 1
        lu1, ip1 = np.zeros(ldab * n), np.zeros(n, np.int64)
        lu2, ip2 = np.zeros(ldab * n), np.zeros(n, np.int64)
        o1 = oracle_lib.diffusion_2d(s2(f["psd"]), *la, lu=lu1, ipiv=ip1)[1]
        o2 = ref_lu.diffusion_2d(s2(f["psd"]), *la, lu=lu2, ipiv=ip2)[1]
        assert np.array_equal(ip1 + 1, ip2)
        assert rel(o1, o2) < LOCAL_RTOL


@pytest.mark.skipif(not O.have_reference(), reason="reference not built here")
def test_monot_cubic_matches_reference_interpolator(oracle_lib):
    # the interpolator of the L* remapping (Opm::MonotCubicInterpolator compiled
    # from the reference sources) against the C restatement, including
    # monotone data (derivative adjustment), flat starts and extrapolation
    ref = O.reference(lu_caching=True)
    rng = np.random.default_rng(0)
    for trial in range(300):
        n = int(rng.integers(2, 40))
        x = np.unique(rng.uniform(0, 10, n))
        if len(x) < 2:
            continue
        f = rng.standard_normal(len(x))
        if trial % 3 == 0:
            f = np.sort(f) * (1 if trial % 2 else -1)
        if trial % 7 == 0:
            f[:3] = f[0]
        xq = np.concatenate([rng.uniform(-1, 11, 50), x])
        st, a = oracle_lib.monot_cubic(x, f, xq)
        _, b = ref.monot_cubic(x, f, xq)
        assert st == 0 and np.array_equal(a, b), trial
