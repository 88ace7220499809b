"""Updatable input fields on the device against the CPU restatement of the
reference's UpdatableMatrix / UpdatableListMatrix (oracle/updatable.py).

Component lists with scale, limit and replacement-data queues are advanced
through a sequence of times; after every update the device field equals the
restatement bit for bit (the merge is base*scale, zeroing, and a sum from 0
or a division by the finite count: no rounding choices).  A local step after
a D_VV update must use refreshed LU factors: it equals a step of a context
that was given the merged field directly.
"""
import numpy as np
import pytest

import updatable as U
from verb4d_b200 import workload as W

from test_gpu_step import load_ctx

pytestmark = pytest.mark.gpu


def field_axes(wl, name):
    f = wl.fields
    return [f["Pg"], f["Lg"] if name == "DLL" else f["Rg"], f["Vg"], f["Kg"]]


def build(c, name, comps, merge, oracle):
    for base in comps:
        c.add_component(name, base)
        oracle.comps.append(U.Component(base))
    c.set_merge(name, merge)


def test_component_queues_match_restatement(gpu):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=11, losses=True)
    f = wl.fields
    rng = np.random.default_rng(3)
    c = load_ctx(wl)
    orc = {}
    # D_VV: two summed components (e.g. two wave types), one with a scale
    # series and R limits, the other with a replacement file at t = 2
    dvv = f["DVV"]
    orc["DVV"] = U.ListField("sum")
    build(c, "DVV", [0.6 * dvv, 0.4 * dvv], "sum", orc["DVV"])
    for t, sc in [(0.0, 1.0), (1.0, 2.5), (1.5, 0.75), (3.0, 1.25)]:
        c.queue_scale("DVV", 0, t, sc)
        orc["DVV"].comps[0].scale_q.append((t, sc))
    for t, w, v in [(1.0, "from", 2.0), (2.5, "to", 5.5)]:
        c.queue_limit("DVV", 0, 1, w, t, v)
        orc["DVV"].comps[0].limit_q[1][0 if w == "from" else 1].append((t, v))
    repl = dvv * rng.uniform(0.5, 1.5, dvv.shape)
    c.queue_data("DVV", 1, 2.0, repl)
    orc["DVV"].comps[1].data_q.append((2.0, repl))
    # losses: mean of three components, one with non-finite values
    lo = f["loss_local"]
    bad = lo.copy()
    bad[0, 0, :3, :] = np.inf
    orc["loss_local"] = U.ListField("mean")
    build(c, "loss_local", [lo, 2 * lo, bad], "mean", orc["loss_local"])
    # D_LL: limited in L* (axis 1) from t = 0.5
    orc["DLL"] = U.ListField("sum")
    build(c, "DLL", [f["DLL"]], "sum", orc["DLL"])
    c.queue_limit("DLL", 0, 1, "to", 0.5, 5.0)
    orc["DLL"].comps[0].limit_q[1][1].append((0.5, 5.0))

    for t in (0.0, 0.25, 0.5, 1.0, 1.2, 1.5, 2.0, 2.7, 3.0, 4.0):
        rebuilt = set(c.update_fields(t))
        for name, lf in orc.items():
            upd, want = lf.update(t, field_axes(wl, name))
            got = c.download(name)
            assert np.array_equal(got, want, equal_nan=True), (name, t)
            if t > 0.0:
                assert (name in rebuilt) == upd, (name, t)
    c.close()


def test_local_step_uses_updated_coefficients(gpu):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=12)
    f = wl.fields
    c = load_ctx(wl)
    c.local(wl.dt, wl.sub_dt)            # factors of the uploaded D_VV
    c.add_component("DVV", f["DVV"])
    c.queue_scale("DVV", 0, 1.0, 3.0)
    assert "DVV" in c.update_fields(1.0)
    c.local(wl.dt, wl.sub_dt)            # must refactor with 3*D_VV
    c.sync()
    got = c.download()
    c.close()
    ref = load_ctx(wl)
    ref.local(wl.dt, wl.sub_dt)
    ref.upload("DVV", f["DVV"] * 3.0)
    ref.local(wl.dt, wl.sub_dt)
    ref.sync()
    want = ref.download()
    ref.close()
    assert np.array_equal(got, want)
