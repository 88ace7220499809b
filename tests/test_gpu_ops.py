"""GPU per-slice operators (through the C ABI) against the reference fixtures
and the CPU oracle.

Radial diffusion, tridag and convection are bit-identical to the reference
(the oracle restates them operation by operation and is pinned bit-exactly in
test_oracle.py).  The banded LU follows the oracle's unblocked xGBTF2/xGBTRS
operation order, so it is bit-identical to the oracle; against LAPACK's
blocked dgbtrf in the reference it agrees to LOCAL_RTOL with identical pivots.
"""
import os

import numpy as np
import pytest

from verb4d_b200 import ops, VerbError
from verb4d_b200 import workload as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
LOCAL_RTOL = 1e-12


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(GOLD, "slices.npz")))


def sub(g, prefix):
    return {k[len(prefix):]: v for k, v in g.items() if k.startswith(prefix)}


def test_tridag_bitexact(gpu, gold):
    u = ops.tridag(gold["tri_a"], gold["tri_b"], gold["tri_c"], gold["tri_r"])
    assert np.array_equal(u, gold["tri_out"])


def test_diffusion_1d_bitexact(gpu, gold):
    for c in range(4):
        g = sub(gold, f"d1_{c}_")
        out = ops.Diffusion_1D(g["psd"], g["x"], len(g["x"]), g["lbc"], g["ubc"], int(g["lbc_t"]),
                               int(g["ubc_t"]), g["D"], g["G"], g["S"], g["loss"], float(g["dt"]))
        assert np.array_equal(out, g["out"]), c


def test_convection_1d_bitexact(gpu, gold):
    for c in range(4):
        lb, ub, lt, ut = gold[f"c1_{c}_bc"]
        x = gold[f"c1_{c}_x"]
        out = ops.Convection_1D(gold[f"c1_{c}_psd"], x, len(x), lb, ub, int(lt), int(ut),
                                gold[f"c1_{c}_ux"], W.DT_5MIN)
        assert np.array_equal(out, gold[f"c1_{c}_out"]), c


# exp(Loss*dt) (src/Convection_2D.cpp:101) comes from CUDA's exp on the device and
# from the host libm in the reference; the two may differ by one ulp, so with
# non-zero loss rates convection agrees to rounding, and bit for bit without.
EXP_RTOL = 1e-13


def test_convection_2d(gpu, gold, oracle_lib):
    for c in range(3):
        g = sub(gold, f"c2_{c}_")
        nP, nR = g["psd"].shape
        args = (g["P"], g["R"], nP, nR, g["pl"], g["pu"], g["rl"], g["ru"], 0, 0, 1, 1, g["VP"],
                g["VR"], g["S"])
        out = ops.Convection_2D(g["psd"], *args, g["loss"], g["G"], float(g["dt"]))
        assert rel(out, g["out"]) < EXP_RTOL, c
        # without loss rates: bit-identical to the oracle (itself bit-identical to the reference)
        zero = np.zeros_like(g["loss"])
        out0 = ops.Convection_2D(g["psd"], *args, zero, g["G"], float(g["dt"]))
        _, ref0, _ = oracle_lib.convection_2d(g["psd"], g["P"], g["R"], g["pl"], g["pu"], g["rl"],
                                              g["ru"], (0, 0, 1, 1), g["VP"], g["VR"], g["S"], zero,
                                              g["G"], float(g["dt"]))
        assert np.array_equal(out0, ref0), c


def test_diffusion_2d_vs_reference_and_oracle(gpu, gold, oracle_lib):
    for c in range(3):
        g = sub(gold, f"d2_{c}_")
        nx, ny = g["psd"].shape
        types = [int(t) for t in g["types"]]
        args = (g["x"], g["y"], nx, ny, g["xl"], g["xu"], g["yl"], g["yu"], *types, g["Dxx"],
                g["Dyy"], g["Dxy"], g["Dyx"], g["G"], g["S"], g["loss"], float(g["dt"]),
                float(g["sub_dt"]))
        lu = np.zeros_like(g["lu"])
        ip = np.zeros(nx * ny, dtype=np.int64)
        out = ops.Diffusion_2D(g["psd"], *args, lu_cache=lu, index_cache=ip, recompute_lu=True)
        # pivots are integers: identical to LAPACK dgbtrf's
        assert np.array_equal(ip, g["ipiv"]), c
        assert rel(out, g["out"]) < LOCAL_RTOL
        assert rel(lu, g["lu"]) < 1e-13
        # bit-identical to the oracle's restatement
        olu = np.zeros_like(lu)
        oip = np.zeros_like(ip)
        _, oout = oracle_lib.diffusion_2d(g["psd"], g["x"], g["y"], g["xl"], g["xu"], g["yl"],
                                          g["yu"], tuple(types), g["Dxx"], g["Dyy"], g["Dxy"],
                                          g["Dyx"], g["G"], g["S"], g["loss"], float(g["dt"]),
                                          float(g["sub_dt"]), lu=olu, ipiv=oip)
        assert np.array_equal(out, oout)
        assert np.array_equal(lu, olu)
        # LU_CACHING reuse: solving again from the cached factors gives the same bits
        out2 = ops.Diffusion_2D(g["psd"], *args, lu_cache=lu, index_cache=ip, recompute_lu=False)
        assert np.array_equal(out2, out)
        # and from LAPACK's own factors, results agree to rounding
        out3 = ops.Diffusion_2D(g["psd"], *args, lu_cache=g["lu"].copy(),
                                index_cache=g["ipiv"].copy(), recompute_lu=False)
        assert rel(out3, g["out"]) < LOCAL_RTOL


def test_error_codes(gpu):
    x = np.linspace(0, 24, 24)
    psd = np.ones(24)
    # more than 1e6 CFL sub-steps is reported as a Courant failure (the
    # reference would sub-cycle practically forever); nothing is iterated
    with pytest.raises(VerbError) as e:
        ops.Convection_1D(psd, x, 24, 0, 0, 0, 0, np.full(24, 1e12), 1.0)
    assert e.value.status == 3
    with pytest.raises(VerbError) as e:  # fewer than 11 points
        ops.Convection_1D(psd[:8], x[:8], 8, 0, 0, 0, 0, np.ones(8), 1.0)
    assert e.value.status == 9
    n = 6
    g2 = np.ones((n, n))
    with pytest.raises(VerbError) as e:  # periodic is not a local-diffusion BC
        ops.Diffusion_2D(g2, g2, g2, n, n, np.ones(n), np.ones(n), np.ones(n), np.ones(n), 0, 1, 1,
                         1, g2, g2, g2 * 0, g2 * 0, g2, g2 * 0, g2 * 0, 0.01, 0.01)
    assert e.value.status == 4
