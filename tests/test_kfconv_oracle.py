"""The CPU restatement of the convection data assimilation (oracle/kfconv.py)
against the reference: the committed fixture (tests/golden/kfconv.npz, made
by tests/golden/make_kfconv_golden.py from the reference compiled here) and,
where oracle/_ref exists, fresh seeded slices through the reference itself.
The model matrices agree bit for bit (same operations, same dgemm order);
states and covariances to 1e-13 norm-wise (dgesv vs numpy's solve)."""
import math
import os

import numpy as np
import pytest

import kfconv as KC
import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "kfconv.npz")
TOL = 1e-13


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def run(inp, use_log, steps=2):
    N = inp["forecast"].size
    x, Pa, model = inp["forecast"], np.zeros((N, N)), None
    xs = []
    for it in range(steps):
        x, Pa, model, _ = KC.kf_convection_2d(
            x, Pa, model, inp["Pg"], inp["Rg"], inp["VP"], inp["VR"], it == 0, inp["loss"], None,
            inp["obs"], float(inp["dt"]), 1e-3, 1e-2, use_log=use_log)
        xs.append(x)
    return xs, Pa, model


def test_restatement_matches_fixture():
    g = np.load(GOLD)
    for c in range(2):
        inp = {k[len(f"c{c}_in_"):]: g[k] for k in g.files if k.startswith(f"c{c}_in_")}
        xs, Pa, model = run(inp, bool(g[f"c{c}_use_log"]))
        assert np.array_equal(model, g[f"c{c}_model"])
        for it in range(2):
            assert rel(xs[it], g[f"c{c}_x{it}"]) < TOL
        assert rel(Pa, g[f"c{c}_Pa"]) < TOL


def test_matrix_power_sequence():
    rng = np.random.default_rng(0)
    A = rng.uniform(0, 1, (7, 7)) / 7
    for p in (1, 2, 3, 5, 8, 36, 37, 559):
        assert rel(KC.matpow(A, p), np.linalg.matrix_power(A, p)) < 1e-12


@pytest.mark.skipif(not O.have_reference(), reason="reference not compiled here (oracle/_ref)")
def test_restatement_matches_reference_fresh():
    import make_kfconv_golden as G

    ref = O.reference()
    for seed, vscale, use_log in [(51, 1.0, False), (52, 25.0, True), (53, 3.0, False)]:
        inp = G.case_inputs(seed, seed % 5, seed % 4, 6 + seed % 7, vscale)
        N = inp["forecast"].size
        x, Pa, model = inp["forecast"], np.zeros((N, N)), None
        for it in range(2):
            args = (inp["Pg"], inp["Rg"], inp["VP"], inp["VR"], it == 0, inp["loss"], None,
                    inp["obs"], float(inp["dt"]), 1e-3, 1e-2)
            st, xr, par, mr, pfr = ref.kf_convection_2d(x, Pa, model, *args, use_log=use_log)
            assert st == 0
            xo, pao, mo, pfo = KC.kf_convection_2d(x, Pa, model, *args, use_log=use_log)
            assert np.array_equal(mo, mr)
            assert rel(xo, xr) < TOL and rel(pao, par) < TOL and rel(pfo, pfr) < TOL
            x, Pa, model = xr, par, mr
