"""Steps replayed from a captured CUDA graph (verb_set_step_graph) against
eager steps: bit-identical PSD and negative-point counts over a run that
crosses hour boundaries (D_LL scale and velocity uploads drop the graph, the
radial factors are rebuilt eagerly, the next step captures again), in the
FP64 form and in the mixed form with refinement (device copies and memsets
inside the captured step)."""
import time

import numpy as np
import pytest

from verb4d_b200 import workload as W
from verb4d_b200.solver import Solver

pytestmark = pytest.mark.gpu


def run(wl, graph, steps, form=("fp64", 0)):
    s = Solver(wl)
    s.load()
    s.ctx.set_local_precision(*form)
    s.ctx.set_step_graph(graph)
    negs = []
    t = []
    for it in range(1, steps + 1):
        t0 = time.perf_counter()
        negs.append(s.step(it, count_negatives=True))
        t.append(time.perf_counter() - t0)
    s.ctx.sync()
    out = s.ctx.download()
    s.ctx.close()
    return out, negs, t


@pytest.mark.parametrize("form", [("fp64", 0), ("mixed", 2)])
def test_graph_steps_identical(gpu, form):
    spec = W.CONFIGS["cfg1"]
    wl = W.make_workload(spec, seed=91, kp=W.kp_series(91, 24), sources=True, losses=True)
    a, na, _ = run(wl, False, 30, form)
    b, nb, _ = run(wl, True, 30, form)
    assert na == nb
    assert np.array_equal(a, b)


def test_graph_step_time(gpu):
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=92)
    _, _, te = run(wl, False, 14)
    _, _, tg = run(wl, True, 14)
    # steady steps (after the factorisation and the capture)
    print("24x25x31x31 step wall time with the negative count read: eager %.3f ms, graph %.3f ms"
          % (1e3 * np.median(te[3:]), 1e3 * np.median(tg[3:])))
