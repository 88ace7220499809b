"""The C++ drop-in layer (include/verb4d_dropin.hpp over libverb4d_b200.so)
against the reference's own routines, called through the same harness on the
same Matrix contents: tridag, Diffusion_1D, Convection_1D_ULTIMATE_QUICKEST6
and Convection_2D bit for bit; Diffusion_2D (plain and LU_CACHING builds)
bit for bit against the oracle's restatement of LAPACK's unblocked xGBTF2 /
xGBTRS, and against the reference (OpenBLAS's blocked dgbtrf) to
10 kappa(A) eps64 norm-wise with identical pivots; and the reference's
abort on a singular pivot (src/MatrixSolver.cpp:273-276), which both end with
exit(EXIT_FAILURE)."""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import oracle as O
from verb4d_b200 import workload as W

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(O.DROPIN_SO),
                                 reason="drop-in not built (needs the reference tree)")]
RTOL_LU = 1e-12


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def libs(gpu):
    return O.dropin(), O.reference(), O.reference(lu_caching=True)


@pytest.fixture(scope="module")
def wl():
    return W.make_workload(W.CONFIGS["cfg1"], seed=31, sources=True, losses=True)


def test_tridag_bit_for_bit(libs):
    drop, ref, _ = libs
    rng = np.random.default_rng(1)
    n = 101
    a, c = rng.uniform(-1, 0, n), rng.uniform(-1, 0, n)
    b = 2.5 + rng.uniform(0, 1, n)
    r = rng.standard_normal(n)
    assert np.array_equal(drop.tridag(a, b, c, r), ref.tridag(a, b, c, r))


def test_diffusion_1d_bit_for_bit(libs, wl):
    drop, ref, _ = libs
    f = wl.fields
    for (p, v, k) in ((0, 3, 4), (5, 20, 17), (23, 30, 30)):
        ln = lambda a: a[p, :, v, k]  # noqa: E731
        args = (ln(f["psd"]), ln(f["Lg"]), float(f["Ll"][p, v, k]), float(f["Lu"][p, v, k]), 1, 1,
                ln(f["DLL"]), ln(f["G_radial"]), ln(f["S"]), ln(f["loss_radial"]), wl.dt)
        st_d, got = drop.diffusion_1d(*args)
        st_r, want = ref.diffusion_1d(*args)
        assert st_d == 0 and st_r == 0
        assert np.array_equal(got, want), (p, v, k)


def test_convection_bit_for_bit(libs, wl):
    drop, ref, _ = libs
    f = wl.fields
    for (v, k) in ((30, 12), (8, 3)):
        sl = lambda a: np.ascontiguousarray(a[:, :, v, k])  # noqa: E731
        # exp() of non-zero loss rates may differ in the last bit from the host
        # libm, so the loss rates are zero here
        args = (sl(f["psd"]), sl(f["Pg"]), sl(f["Rg"]), f["Pl"][:, v, k], f["Pu"][:, v, k],
                f["Rl"][:, v, k], f["Ru"][:, v, k], (0, 0, 1, 1), sl(f["VP"]), sl(f["VR"]),
                sl(f["S"]), np.zeros_like(sl(f["psd"])), sl(f["G_conv"]), wl.dt)
        st_d, got, _ = drop.convection_2d(*args)
        st_r, want, _ = ref.convection_2d(*args)
        assert st_d == 0 and st_r == 0
        assert np.array_equal(got, want), (v, k)
        line = (sl(f["psd"])[:, 4], sl(f["Pg"])[:, 4], 0.0, 0.0, 0, 0, sl(f["VP"])[:, 4], wl.dt)
        st_d, got = drop.convection_1d(*line)
        st_r, want = ref.convection_1d(*line)
        assert np.array_equal(got, want), (v, k)


def local_args(wl, p, r):
    f = wl.fields
    s2 = lambda a: np.ascontiguousarray(a[p, r])  # noqa: E731
    bt = wl.bc_types
    return (s2(f["psd"]), s2(f["Vg"]), s2(f["Kg"]), f["Vl"][p, r], f["Vu"][p, r], f["Kl"][p, r],
            f["Ku"][p, r], (bt["Vl"], bt["Vu"], bt["Kl"], bt["Ku"]), s2(f["DVV"]), s2(f["DKK"]),
            s2(f["DVK"]), s2(f["DVK"]), s2(f["G_local"]), s2(f["S"]), s2(f["loss_local"]), wl.dt,
            wl.sub_dt)


def kappa_tol(wl, args):
    """10 kappa(A) eps64 for the system's matrix: the two LU orders (LAPACK's
    unblocked xGBTF2 on the GPU and in the oracle, OpenBLAS's blocked dgbtrf
    in the reference) may differ by that much, and no less on these stiff
    systems (kappa ~ 1e5)."""
    o = O.oracle()
    (psd, x, y, xl, xu, yl, yu, types, Dxx, Dyy, Dxy, Dyx, G, S, loss, dt, sub_dt) = args
    st, diag, _, _ = o.local_matrix(x, y, xl, xu, yl, yu, types, Dxx, Dyy, Dxy, Dyx, G, S, loss, dt)
    nx, ny = np.shape(x)
    n = nx * ny
    A = np.zeros((n, n))
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            off = dy * nx + dx
            d = diag[(dy + 1) * 3 + (dx + 1)]
            for i in range(n):
                if 0 <= i + off < n and d[i] != 0.0:
                    A[i, i + off] = d[i]
    return max(RTOL_LU, 10 * np.linalg.cond(A) * np.finfo(float).eps)


def test_diffusion_2d_plain_and_lu_caching(libs, wl):
    drop, ref, ref_lu = libs
    orc = O.oracle()
    V, K = wl.spec.V, wl.spec.K
    n, ldab = V * K, 3 * (V + 1) + 1
    for (p, r) in ((0, 12), (17, 20)):
        args = local_args(wl, p, r)
        tol = kappa_tol(wl, args)
        _, got = drop.diffusion_2d(*args)
        _, want = ref.diffusion_2d(*args)
        _, exact = orc.diffusion_2d(*args)
        assert np.array_equal(got, exact), (p, r)  # the xGBTF2 restatement, bit for bit
        assert rel(got, want) < tol, (p, r, rel(got, want), tol)
        # LU_CACHING: factor into each side's cache slot, then re-solve from
        # the other side's cache (the slot is LAPACK's band layout)
        lu_d, piv_d = np.zeros(ldab * n), np.zeros(n, dtype=np.int64)
        lu_r, piv_r = np.zeros(ldab * n), np.zeros(n, dtype=np.int64)
        _, got = drop.diffusion_2d(*args, lu=lu_d, ipiv=piv_d, recompute=True)
        _, want = ref_lu.diffusion_2d(*args, lu=lu_r, ipiv=piv_r, recompute=True)
        assert rel(got, want) < tol
        assert np.array_equal(piv_d, piv_r)
        assert rel(lu_d, lu_r) < tol
        _, got2 = drop.diffusion_2d(*args, lu=lu_r, ipiv=piv_r, recompute=False)
        _, want2 = ref_lu.diffusion_2d(*args, lu=lu_d, ipiv=piv_d, recompute=False)
        assert rel(got2, want2) < tol


ABORT = r"""
import sys, numpy as np
sys.path[:0] = {paths!r}
import oracle as O
from verb4d_b200 import workload as W
import test_gpu_dropin as T
wl = W.make_workload(W.CONFIGS["cfg1"], seed=31)
f = wl.fields
for key in ("DVV", "DKK", "DVK"):
    f[key] = np.zeros_like(f[key])
f["loss_local"] = np.zeros_like(f["loss_local"])
f["loss_local"][3, 7, 15, 15] = 1.0 / wl.dt
lib = O.dropin() if sys.argv[1] == "dropin" else O.reference()
args = list(T.local_args(wl, 3, 7))
args[-1] = wl.dt
lib.diffusion_2d(*args)
print("returned")
"""


@pytest.mark.parametrize("which", ["reference", "dropin"])
def test_singular_pivot_aborts_like_the_reference(gpu, which):
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    paths = [here, os.path.join(root, "oracle"), os.path.join(root, "verb-4d_b200")]
    # the reference's Logger writes log.txt into the working directory
    with tempfile.TemporaryDirectory() as cwd:
        r = subprocess.run([sys.executable, "-c", ABORT.format(paths=paths), which],
                           capture_output=True, text=True, timeout=300, cwd=cwd)
    assert r.returncode == 1, (which, r.returncode, r.stdout[-500:], r.stderr[-500:])
    assert "returned" not in r.stdout
