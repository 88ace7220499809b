"""An ensemble of independent VERB-4D runs on one GPU, admitted by HBM budget.

Each member is a whole run (its own grid, seeded inputs and Kp series) held in
its own device context.  Members are admitted in waves: a wave is a set of
members whose device memory, estimated before anything is allocated
(verb_estimate_device_bytes), fits the budget.  The members of a wave run
concurrently, each on its own CUDA stream (the context's) driven by its own
host thread; the next wave starts when every member of the current one has
taken its steps and released its memory.  A member that does not fit the
budget in FP64 is admitted with its local factors stored in FP32 (the mixed
form), or rejected if that does not fit either.

Every `kf_every` steps a member takes a radial Kalman-filter update
(verb_assimilate_radial at MLT index 0, as the reference's assimilation,
src/DataAssimilationDiffusion.cpp:116,139) with `n_obs` synthetic observations
at random (L, E, alpha) points: the member's current PSD there times a
log-normal factor with `obs_noise` spread.

Latency of a member step is the host wall time from the launch of the step to
its completion on the member's stream, so it includes the time the step waits
for the GPU while other members' kernels run.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from . import workload as W
from .solver import Solver

GRID_CHOICES = dict(L=(51, 76, 101), E=(61, 101), alpha=(61, 91), MLT=(24, 48))


@dataclass
class Member:
    spec: W.GridSpec
    seed: int
    precision: str = "fp64"
    refinements: int = 0
    est_bytes: int = 0
    # results
    psd: np.ndarray | None = None
    latencies_s: list = field(default_factory=list)
    negatives: int | None = None


def draw_members(n: int = 64, seed: int = 0) -> list[Member]:
    """n members with grids drawn from {51,76,101} L x {61,101} E x {61,91}
    alpha x {24,48} MLT and seeds derived from one master seed."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        g = {k: int(rng.choice(v)) for k, v in GRID_CHOICES.items()}
        out.append(Member(W.GridSpec(g["MLT"], g["L"], g["E"], g["alpha"]),
                          seed=int(rng.integers(1, 2**31 - 1))))
    return out


def estimate_bytes(spec: W.GridSpec, precision: str = "fp64", refinements: int = 0,
                   kf_columns: int = 0) -> int:
    lib = L.load()
    b = C.c_size_t(0)
    mode = L.VERB_PREC_MIXED if precision == "mixed" else L.VERB_PREC_FP64
    L.check(lib.verb_estimate_device_bytes(spec.P, spec.R, spec.V, spec.K, mode, refinements,
                                           kf_columns, C.byref(b)), "estimate")
    return b.value


def plan_waves(members: list[Member], budget: int, kf: bool = True,
               mixed_refinements: int = 3, sizer=estimate_bytes) -> list[list[Member]]:
    """First-fit-decreasing packing of members into waves within `budget`
    bytes.  Members too large in FP64 fall back to the mixed form; members
    too large even then raise ValueError."""
    for m in members:
        cols = m.spec.V * m.spec.K if kf else 0
        m.precision, m.refinements = "fp64", 0
        m.est_bytes = sizer(m.spec, "fp64", 0, cols)
        if m.est_bytes > budget:
            m.precision, m.refinements = "mixed", mixed_refinements
            m.est_bytes = sizer(m.spec, "mixed", mixed_refinements, cols)
            if m.est_bytes > budget:
                raise ValueError(f"member {m.spec.shape} needs {m.est_bytes} B > budget {budget} B")
    waves: list[list[Member]] = []
    free: list[int] = []
    for m in sorted(members, key=lambda m: -m.est_bytes):
        for w, room in enumerate(free):
            if m.est_bytes <= room:
                waves[w].append(m)
                free[w] -= m.est_bytes
                break
        else:
            waves.append([m])
            free.append(budget - m.est_bytes)
    return waves


class Ensemble:
    def __init__(self, members: list[Member], budget_bytes: int, steps: int, kf_every: int = 12,
                 n_obs: int = 500, obs_noise: float = 0.05, model_error: float = 1e-3,
                 obs_error: float = 1e-2):
        self.members = members
        self.budget = int(budget_bytes)
        self.steps = steps
        self.kf_every = kf_every
        self.n_obs = n_obs
        self.obs_noise = obs_noise
        self.model_error = model_error
        self.obs_error = obs_error
        self.waves = plan_waves(members, self.budget, kf=kf_every > 0)

    def observations(self, m: Member, psd: np.ndarray, it: int) -> np.ndarray:
        spec = m.spec
        rng = np.random.default_rng((m.seed, it))
        obs = np.full(spec.shape, np.nan)
        # random (L, E, alpha) points at MLT index 0, inner and outer L excluded
        # (boundary rows carry no observation operator rows in the reference)
        r = rng.integers(1, spec.R - 1, self.n_obs)
        v = rng.integers(0, spec.V, self.n_obs)
        k = rng.integers(0, spec.K, self.n_obs)
        obs[0, r, v, k] = psd[0, r, v, k] * np.exp(self.obs_noise * rng.standard_normal(self.n_obs))
        return obs

    def run_member(self, m: Member, errors: list):
        try:
            hours = int(np.ceil(self.steps * W.DT_5MIN * 24)) + 2
            wl = W.make_workload(m.spec, seed=m.seed, kp=W.kp_series(m.seed, max(hours, 24)))
            s = Solver(wl)
            s.load()
            s.ctx.set_local_precision(m.precision, m.refinements)
            lat = []
            for it in range(1, self.steps + 1):
                t0 = time.perf_counter()
                s.step(it)
                s.ctx.sync()
                lat.append(time.perf_counter() - t0)
                if self.kf_every and it % self.kf_every == 0:
                    obs = self.observations(m, s.ctx.download(), it)
                    s.ctx.assimilate_radial(obs, wl.dt, self.model_error, self.obs_error, p_index=0)
                    s.ctx.sync()
            m.latencies_s = lat
            m.negatives = s.ctx.negative_count()
            m.psd = s.ctx.download()
            s.ctx.close()
        except Exception as e:  # reported after the wave
            errors.append((m.spec.shape, repr(e)))

    def run(self) -> dict:
        t0 = time.perf_counter()
        errors: list = []
        for wave in self.waves:
            threads = [threading.Thread(target=self.run_member, args=(m, errors)) for m in wave]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
            if errors:
                raise RuntimeError(f"ensemble member failed: {errors[0]}")
        wall = time.perf_counter() - t0
        lat = np.concatenate([np.asarray(m.latencies_s) for m in self.members])
        sim_h = self.steps * W.DT_5MIN * 24.0
        return {"members": len(self.members), "waves": len(self.waves), "steps": self.steps,
                "wall_s": wall, "member_sim_hours_per_s": len(self.members) * sim_h / wall,
                "member_steps_per_s": len(self.members) * self.steps / wall,
                "step_latency_p50_ms": float(np.percentile(lat, 50) * 1e3),
                "step_latency_p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mixed_members": sum(m.precision == "mixed" for m in self.members),
                "budget_gb": self.budget / 1e9,
                "wave_gb": [round(sum(m.est_bytes for m in w) / 1e9, 2) for w in self.waves]}
