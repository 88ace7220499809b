"""The autotuner's local-solve shapes (systems per CTA, factor columns in
flight): every shape gives the same solution bit for bit, the tuning run
leaves the PSD untouched, and the chosen shape is the fastest it timed."""
import numpy as np
import pytest

from verb4d_b200 import workload as W

from test_gpu_step import load_ctx

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_shapes_identical_and_tuning_side_effect_free(gpu, form):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=95, sources=True, losses=True)
    c = load_ctx(wl)
    c.set_local_precision(form, 0)
    shapes = c.solve_variants()
    assert len(shapes) >= 2 and shapes[0] == (4, 4, 2, 0)
    before = c.download()
    chosen, times = c.autotune_local_solve(wl.dt, wl.sub_dt)
    assert np.array_equal(c.download(), before)
    assert np.all(times > 0) and times[chosen] == times.min()
    print(form, "local solve shapes (warps/CTA, L cols, U cols, window in registers) -> ms:",
          {str(s): round(float(t), 4) for s, t in zip(shapes, times)}, "chosen", shapes[chosen])
    c.local(wl.dt, wl.sub_dt)
    c.sync()
    tuned = c.download()
    c.close()
    ref = None
    for v in range(len(shapes)):
        c = load_ctx(wl)
        c.set_local_precision(form, 0)
        c.set_local_solve_variant(v)
        c.local(wl.dt, wl.sub_dt)
        c.sync()
        out = c.download()
        c.close()
        if ref is None:
            ref = out
        assert np.array_equal(out, ref), v
    assert np.array_equal(tuned, ref)
