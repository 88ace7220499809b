"""The CPU restatement of the reference's input-update system
(oracle/updatable.py, src/UpdatableMatrix.cpp:602-846, 913-961) on small
hand-checked cases.  The device implementation is compared with it in
test_gpu_updatable.py."""
import numpy as np

import updatable as U


def axes(shape=(2, 3, 4, 5)):
    g = np.meshgrid(*[np.arange(n, dtype=float) for n in shape], indexing="ij")
    return [np.ascontiguousarray(a) for a in g]


def test_scale_queue_keeps_latest_value():
    ax = axes()
    k = U.Component(np.ones(ax[0].shape))
    k.scale_q.extend([(1.0, 2.0), (2.0, 3.0)])
    u, v = k.update(0.5, ax)
    assert not u and np.all(v == 1)
    u, v = k.update(2.5, ax)          # both due: the latest wins
    assert u and np.all(v == 3)
    u, v = k.update(3.0, ax)          # nothing popped: not updated, scale kept
    assert not u and np.all(v == 3)


def test_data_queue_last_due_entry_and_time_rule():
    ax = axes()
    k = U.Component(np.zeros(ax[0].shape))
    k.data_q.extend([(1.0, np.full(ax[0].shape, 5.0)), (2.0, np.full(ax[0].shape, 7.0))])
    u, v = k.update(2.0, ax)
    assert u and np.all(v == 7)
    # entries before the initial last_update_time (-1) are never loaded (:651)
    k2 = U.Component(np.zeros(ax[0].shape))
    k2.data_q.append((-2.0, np.ones(ax[0].shape)))
    u, v = k2.update(0.0, ax)
    assert not u and np.all(v == 0)


def test_limits_zero_outside_range():
    ax = axes()
    k = U.Component(np.ones(ax[0].shape))
    k.limit_q[1][0].append((0.0, 1.0))   # R from 1
    k.limit_q[3][1].append((0.0, 3.0))   # K to 3
    u, v = k.update(0.0, ax)
    assert u
    assert np.all(v[:, 0] == 0) and np.all(v[..., 4] == 0)
    assert np.all(v[:, 1:, :, :4] == 1)


def test_list_sum_and_mean():
    ax = axes()
    f = U.ListField("sum")
    a = np.ones(ax[0].shape)
    b = np.full(ax[0].shape, 2.0)
    b[0, 0, 0, 0] = np.inf
    f.comps = [U.Component(a), U.Component(b)]
    _, v = f.update(0.0, ax)
    assert v[1, 1, 1, 1] == 3 and np.isinf(v[0, 0, 0, 0])
    f.merge = "mean"
    _, v = f.update(0.0, ax)
    assert v[1, 1, 1, 1] == 1.5 and np.isinf(v[0, 0, 0, 0])
