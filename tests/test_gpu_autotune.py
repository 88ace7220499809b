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


def test_every_shape_at_the_production_band(gpu, oracle_lib):
    # V = 101 (kl = 102): the register-window shapes run with 4 / 7 slots per
    # lane, the capped ones with 56 registers; all equal the oracle bit for bit
    wl = W.make_workload(W.GridSpec(2, 3, 101, 5), seed=96, sources=True, losses=True)
    f = wl.fields
    P, R, V, K = wl.spec.shape
    c = load_ctx(wl)
    shapes = c.solve_variants()
    psd0 = c.download()
    c.close()
    n, ldab = V * K, 3 * (V + 1) + 1
    want = np.empty_like(psd0)
    for iP in range(P):
        for iR in range(R):
            s2 = lambda a: a[iP, iR]  # noqa: E731
            lu, ip = np.zeros(ldab * n), np.zeros(n, np.int64)
            _, want[iP, iR] = oracle_lib.diffusion_2d(
                s2(psd0), s2(f["Vg"]), s2(f["Kg"]), f["Vl"][iP, iR], f["Vu"][iP, iR],
                f["Kl"][iP, iR], f["Ku"][iP, iR], (1, 1, 2, 2), s2(f["DVV"]), s2(f["DKK"]),
                s2(f["DVK"]), s2(f["DVK"]), s2(f["G_local"]), s2(f["S"]), s2(f["loss_local"]),
                wl.dt, wl.sub_dt, lu=lu, ipiv=ip)
    for v in range(len(shapes)):
        c = load_ctx(wl)
        c.set_local_solve_variant(v)
        c.local(wl.dt, wl.sub_dt)
        c.sync()
        out = c.download()
        c.close()
        assert np.array_equal(out, want), shapes[v]
