"""Pins the restatement of the reference's input-update system
(oracle/updatable.py) to the reference's own UpdatableListMatrix compiled from
source (oracle/_ref, ref_updatable_list): the same .tab file -- components
given as .pltb data files or .lst lists of (time, file), with number or .lst
scale factors and number or .lst from/to limits per axis -- is read by the
reference (src/UpdatableMatrix.cpp:857-898 reading, :308-600 parsing) and
updated at a series of times (:602-846 and :913-961), and the restatement
must give the same field bit for bit, with the same update flags, in both
merge forms (SUM, MEAN).  CPU only."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
import pltb
import updatable as U

pytestmark = pytest.mark.skipif(not os.path.exists(O.REF_SO),
                                reason="reference not built (needs the reference tree)")
SHAPE = (3, 4, 5, 6)
TIMES = [0.0, 0.1, 0.3, 0.5, 0.9, 1.0, 1.7, 2.5, 3.0, 4.0]


def grids():
    g = np.meshgrid(*[np.linspace(0.0, 1.0 + i, n) for i, n in enumerate(SHAPE)], indexing="ij")
    return [np.ascontiguousarray(a) for a in g]


def reference_run(tab, mean, ax):
    lib = O.reference().lib
    n = int(np.prod(SHAPE))
    out = np.zeros((len(TIMES), n))
    upd = np.zeros(len(TIMES), dtype=np.int32)
    t = np.array(TIMES)
    dp = C.POINTER(C.c_double)
    st = lib.ref_updatable_list(str(tab).encode(), C.c_int(int(mean)), *[C.c_int(s) for s in SHAPE],
                                *[a.ctypes.data_as(dp) for a in ax], t.ctypes.data_as(dp),
                                C.c_int(len(TIMES)), out.ctypes.data_as(dp),
                                upd.ctypes.data_as(C.POINTER(C.c_int)))
    assert st == 0
    return out.reshape((len(TIMES),) + SHAPE), upd


def write_lst(path, rows):
    with open(path, "w") as f:
        for t, v in rows:
            f.write(f"{t!r} {v}\n")


@pytest.mark.parametrize("merge", ["sum", "mean"])
def test_restatement_equals_reference_list_matrix(tmp_path, merge):
    ax = grids()
    rng = np.random.default_rng(7)
    arr = {k: rng.uniform(0.5, 2.0, SHAPE) for k in ("a", "b0", "b1", "b2", "c")}
    arr["c"][1, 2, 3, 4] = np.inf  # a non-finite value: MEAN counts finite components only
    for k, v in arr.items():
        pltb.write(tmp_path / f"{k}.pltb", v)
    write_lst(tmp_path / "b.lst", [(0.0, tmp_path / "b0.pltb"), (0.5, tmp_path / "b1.pltb"),
                                   (1.7, tmp_path / "b2.pltb")])
    write_lst(tmp_path / "bscale.lst", [(0.3, 2.0), (0.9, 0.25), (2.5, 3.0)])
    write_lst(tmp_path / "bq1from.lst", [(1.0, 0.4), (4.0, -1.0)])
    write_lst(tmp_path / "cq4to.lst", [(0.5, 3.0)])
    # one component per line: data, scale, then from/to per axis (P, R, V, K)
    lines = [f"{tmp_path}/a.pltb 2.5 - - 0.5 2.5",
             f"{tmp_path}/b.lst {tmp_path}/bscale.lst {tmp_path}/bq1from.lst -",
             f"{tmp_path}/c.pltb - - - - - 0.2 1e99 - {tmp_path}/cq4to.lst"]
    tab = tmp_path / "field.tab"
    tab.write_text("\n".join(lines) + "\n")
    want, upd = reference_run(tab, merge == "mean", ax)

    # the same three components in the restatement
    a = U.Component(arr["a"])
    a.scale = 2.5
    a.lim[1] = [0.5, 2.5]
    b = U.Component(np.zeros(SHAPE))
    b.data_q.extend([(0.0, arr["b0"]), (0.5, arr["b1"]), (1.7, arr["b2"])])
    b.scale_q.extend([(0.3, 2.0), (0.9, 0.25), (2.5, 3.0)])
    b.limit_q[0][0].extend([(1.0, 0.4), (4.0, -1.0)])
    c = U.Component(arr["c"])
    c.lim[2] = [0.2, 1e99]
    c.limit_q[3][1].append((0.5, 3.0))
    f = U.ListField(merge)
    f.comps = [a, b, c]
    for i, t in enumerate(TIMES):
        u, got = f.update(t, ax)
        assert np.array_equal(got, want[i], equal_nan=True), (merge, t)
        assert int(u) == int(upd[i]), (merge, t)
