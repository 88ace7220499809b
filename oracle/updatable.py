"""CPU restatement of the reference's input-update system, for tests only.

Restates UpdatableMatrix::update (src/UpdatableMatrix.cpp:602-846), its
MatrixLimit for 4-D fields (:269-300) and UpdatableListMatrix::update
(:913-961) on numpy arrays: a component holds a base array and time-ordered
queues (replacement arrays, scale factors, from/to limits per axis); update(t)
pops every entry due at t and returns the component's current value.  The
replacement queue holds arrays where the reference holds .lst file names.
"""
from __future__ import annotations

from collections import deque

import numpy as np


class Component:
    """One UpdatableMatrix (defaults: src/UpdatableMatrix.h:70-85, :436)."""

    def __init__(self, base):
        self.original = np.array(base, dtype=np.float64)
        self.data_q = deque()
        self.scale_q = deque()
        self.limit_q = [[deque(), deque()] for _ in range(4)]
        self.scale = 1.0
        self.lim = [[-1e99, 1e99] for _ in range(4)]
        self.last_update_time = -1.0

    def update(self, t, axes):
        """src/UpdatableMatrix.cpp:602-846; axes = the four grid arrays."""
        updated = False
        data, update_time = None, None
        while self.data_q and t >= self.data_q[0][0]:                 # :640-644
            update_time, data = self.data_q.popleft()
        if data is not None:
            if t >= update_time and self.last_update_time < update_time:  # :651
                self.original = np.array(data, dtype=np.float64)
                self.last_update_time = t
                updated = True
        cur = self.original.copy()                                     # :672
        while self.scale_q and t >= self.scale_q[0][0]:                # :687-694
            self.scale = self.scale_q.popleft()[1]
            updated = True
        if self.scale != 1:                                           # :697-708
            cur = cur * self.scale
        for a in range(4):                                            # :724-788
            for w in range(2):
                while self.limit_q[a][w] and t >= self.limit_q[a][w][0][0]:
                    self.lim[a][w] = self.limit_q[a][w].popleft()[1]
                    updated = True
        # MatrixLimit, 4-D (:269-300)
        active = any(self.lim[a][0] > axes[a].min() or self.lim[a][1] < axes[a].max()
                     for a in range(4))
        if active:
            out = np.zeros(cur.shape, dtype=bool)
            for a in range(4):
                out |= (axes[a] < self.lim[a][0]) | (axes[a] > self.lim[a][1])
            cur[out] = 0
        return updated, cur


class ListField:
    """UpdatableListMatrix (src/UpdatableMatrix.cpp:913-961), SUM or MEAN."""

    def __init__(self, merge="sum"):
        self.comps = []
        self.merge = merge

    def update(self, t, axes):
        acc = 0.0
        cnt = 0.0
        any_updated = False
        vals = []
        for k in self.comps:
            u, v = k.update(t, axes)
            any_updated = any_updated or u
            vals.append(v)
        acc = np.zeros(vals[0].shape)
        for v in vals:                                                # :934-938 / :945-948
            acc = acc + v
            cnt = cnt + np.isfinite(v)
        if self.merge == "mean":
            with np.errstate(divide="ignore", invalid="ignore"):
                acc = acc / cnt
        return any_updated, acc
