"""Admission of ensemble members by HBM budget (host logic, no GPU)."""
import pytest

from verb4d_b200 import ensemble as E
from verb4d_b200 import workload as W


def fake_sizer(spec, precision, refinements, kf_columns):
    b = spec.npts * (100 if precision == "fp64" else 60)
    return b + kf_columns


def test_draws_follow_the_grid_choices():
    ms = E.draw_members(64, seed=1)
    assert len(ms) == 64
    for m in ms:
        assert m.spec.R in (51, 76, 101) and m.spec.V in (61, 101)
        assert m.spec.K in (61, 91) and m.spec.P in (24, 48)
    assert len({m.seed for m in ms}) == 64


def test_waves_respect_the_budget_and_admit_everyone():
    ms = E.draw_members(64, seed=2)
    budget = max(fake_sizer(m.spec, "fp64", 0, 0) for m in ms) * 3
    waves = E.plan_waves(ms, budget, kf=True, sizer=fake_sizer)
    assert sorted(id(m) for w in waves for m in w) == sorted(id(m) for m in ms)
    for w in waves:
        assert sum(m.est_bytes for m in w) <= budget
    assert all(m.precision == "fp64" for m in ms)


def test_large_members_fall_back_to_mixed_or_are_rejected():
    big = E.Member(W.GridSpec(48, 101, 101, 91), seed=1)
    need64 = fake_sizer(big.spec, "fp64", 0, 101 * 91)
    waves = E.plan_waves([big], need64 - 1, kf=True, sizer=fake_sizer)
    assert big.precision == "mixed" and waves == [[big]]
    with pytest.raises(ValueError):
        E.plan_waves([big], 1000, kf=True, sizer=fake_sizer)
