"""Ragged (loss-cone trimmed) local systems on the GPU.

Each (MLT, L) system keeps the pitch angles outside the dipole loss cone
alpha_lc(L) = asin(sqrt(1/(L^5 sqrt(4 - 3/L)))) and is the Diffusion_2D
system of that sub-grid with a ConstantValue 0 boundary at its lower
pitch-angle edge.  Every system is compared bit for bit with the oracle's
Diffusion_2D on the same sub-grid; the mixed-precision form of the ragged
batch is compared with the FP64 one at the 1e-8 tolerance.
"""
import numpy as np
import pytest

from verb4d_b200 import workload as W

from test_gpu_step import load_ctx

pytestmark = pytest.mark.gpu


def trimmed_workload():
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=41, sources=True, losses=True)
    return wl, W.loss_cone_k0(wl)


def test_ragged_local_matches_oracle(gpu, oracle_lib):
    wl, k0 = trimmed_workload()
    f = wl.fields
    P, R, V, K = wl.spec.shape
    c = load_ctx(wl)
    c.set_local_trim(k0)
    c.local(wl.dt, wl.sub_dt)
    c.sync()
    got = c.download()
    c.close()
    t = wl.bc_types
    types = (t["Vl"], t["Vu"], W.BC_VALUE, t["Ku"])
    want = f["psd"].copy()
    solved = 0
    for p in range(P):
        for r in range(R):
            k = int(k0[p, r])
            if K - k < 3:
                continue
            s2 = lambda a: a[p, r, :, k:]  # noqa: E731
            st, out = oracle_lib.diffusion_2d(
                s2(f["psd"]), s2(f["Vg"]), s2(f["Kg"]), f["Vl"][p, r, k:], f["Vu"][p, r, k:],
                np.zeros(V), f["Ku"][p, r], types, s2(f["DVV"]), s2(f["DKK"]), s2(f["DVK"]),
                s2(f["DVK"]), s2(f["G_local"]), s2(f["S"]), s2(f["loss_local"]), wl.dt, wl.sub_dt)
            assert st == 0
            want[p, r, :, k:] = out
            solved += 1
    assert solved > 0.9 * P * (R - 2)
    assert np.array_equal(got, want)


def test_ragged_mixed_within_tolerance(gpu):
    wl, k0 = trimmed_workload()
    res, mem = {}, {}
    for mode, nref in (("fp64", 0), ("mixed", 10)):
        c = load_ctx(wl)
        c.set_local_trim(k0)
        c.set_local_precision(mode, nref)
        c.local(wl.dt, wl.sub_dt)
        c.sync()
        res[mode] = c.download()
        mem[mode] = c.device_bytes()
        c.close()
    assert mem["mixed"] < mem["fp64"]
    d = np.abs(res["mixed"] - res["fp64"]).max() / np.abs(res["fp64"]).max()
    assert d < 1e-8


def test_ragged_every_solve_shape_and_graph(gpu):
    # every local-solve shape of the autotuner gives the same trimmed step,
    # and steps replayed from the captured graph equal eager ones
    wl, k0 = trimmed_workload()
    outs = []
    c = load_ctx(wl)
    nshapes = len(c.solve_variants())
    c.close()
    for v in range(nshapes):
        c = load_ctx(wl)
        c.set_local_trim(k0)
        c.set_local_solve_variant(v)
        c.local(wl.dt, wl.sub_dt)
        c.sync()
        outs.append(c.download())
        c.close()
    for v in range(1, nshapes):
        assert np.array_equal(outs[v], outs[0]), v
    res = []
    for graph in (False, True):
        c = load_ctx(wl)
        c.set_local_trim(k0)
        c.set_step_graph(graph)
        negs = [c.step(wl.dt, wl.sub_dt, 1, 1, 1, count_negatives=True) for _ in range(4)]
        c.sync()
        res.append((c.download(), negs))
        c.close()
    assert np.array_equal(res[0][0], res[1][0]) and res[0][1] == res[1][1]
