"""A small ensemble on the GPU: members run concurrently (own stream, own
host thread) give bit for bit the same results as when they run in separate
waves, Kalman updates included; the device-memory estimate used for admission
covers what a member actually holds."""
import numpy as np
import pytest

from verb4d_b200 import ensemble as E
from verb4d_b200 import workload as W
from verb4d_b200 import Solver

pytestmark = pytest.mark.gpu

GRIDS = [W.GridSpec(12, 13, 11, 12), W.GridSpec(12, 15, 11, 12), W.GridSpec(13, 13, 12, 11)]


def members():
    return [E.Member(g, seed=100 + i) for i, g in enumerate(GRIDS)]


def test_concurrent_members_match_separate_waves(gpu):
    kw = dict(steps=6, kf_every=3, n_obs=40)
    one = E.Ensemble(members(), budget_bytes=10**12, **kw)
    assert len(one.waves) == 1
    r1 = one.run()
    small = max(E.estimate_bytes(g, "fp64", 0, g.V * g.K) for g in GRIDS)
    sep = E.Ensemble(members(), budget_bytes=small, **kw)
    assert len(sep.waves) == 3
    sep.run()
    by_shape = {m.spec.shape: m for m in sep.members}
    for m in one.members:
        assert np.array_equal(m.psd, by_shape[m.spec.shape].psd)
        assert len(m.latencies_s) == 6
    assert r1["member_steps_per_s"] > 0 and r1["step_latency_p99_ms"] >= r1["step_latency_p50_ms"]


def test_estimate_covers_actual_device_memory(gpu):
    g = W.GridSpec(12, 13, 11, 12)
    wl = W.make_workload(g, seed=7)
    for prec, nref in (("fp64", 0), ("mixed", 3)):
        s = Solver(wl)
        s.load()
        s.ctx.set_local_precision(prec, nref)
        s.step(1)
        obs = np.full(g.shape, np.nan)
        obs[0, 5, 3, 4] = 1.0
        s.ctx.assimilate_radial(obs, wl.dt, 1e-3, 1e-2, p_index=0)
        s.ctx.sync()
        actual = s.ctx.device_bytes()
        s.ctx.close()
        est = E.estimate_bytes(g, prec, nref, g.V * g.K)
        assert actual <= est <= 1.5 * actual, (prec, actual, est)
