"""Generate the convection data-assimilation fixture from the reference.

Runs the UNMODIFIED reference routine runKalmanFilterConvection2D
(src/DataAssimilationConvection.cpp:124-253), compiled from source by
oracle/Makefile into oracle/_ref/libverbref.so, on seeded [P][R] slices of
the workload generator (6 MLT x 11 L) and stores inputs and outputs in
kfconv.npz: two cases (linear and log form; the second with 40x velocities,
so the model matrix is the 9th power of the split step's), each taken
through two assimilations (model matrix built, then reused).

Usage:  python tests/golden/make_kfconv_golden.py   (needs oracle/_ref)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "verb-4d_b200"))

import oracle as O  # noqa: E402
from verb4d_b200 import workload as W  # noqa: E402

SPEC = W.GridSpec(6, 11, 5, 4)
MODEL_ERROR, OBS_ERROR = 1e-3, 1e-2


def case_inputs(seed, iv, ik, nobs, vscale):
    wl = W.make_workload(SPEC, seed=seed, sources=True)
    f = wl.fields
    sl = lambda a: np.ascontiguousarray(a[:, :, iv, ik])  # noqa: E731
    rng = np.random.default_rng(seed)
    psd = sl(f["psd"])
    obs = np.full(psd.shape, np.nan)
    idx = rng.choice(psd.size, nobs, replace=False)
    obs.flat[idx] = psd.flat[idx] * np.exp(0.1 * rng.standard_normal(nobs))
    return dict(forecast=psd, Pg=sl(f["Pg"]), Rg=sl(f["Rg"]), VP=sl(f["VP"]) * vscale,
                VR=sl(f["VR"]) * vscale, loss=sl(f["S"]) / psd, obs=obs, dt=np.float64(wl.dt))


def main():
    ref = O.reference()
    out = {}
    for c, (seed, iv, ik, nobs, vscale, use_log) in enumerate(
            [(41, 1, 2, 9, 1.0, False), (42, 3, 1, 12, 40.0, True)]):
        inp = case_inputs(seed, iv, ik, nobs, vscale)
        for k, v in inp.items():
            out[f"c{c}_in_{k}"] = v
        out[f"c{c}_use_log"] = np.int32(use_log)
        N = inp["forecast"].size
        x, Pa, model = inp["forecast"], np.zeros((N, N)), None
        for it in range(2):
            st, x, Pa, model, _ = ref.kf_convection_2d(
                x, Pa, model, inp["Pg"], inp["Rg"], inp["VP"], inp["VR"], it == 0, inp["loss"],
                None, inp["obs"], float(inp["dt"]), MODEL_ERROR, OBS_ERROR, use_log=use_log)
            assert st == 0
            out[f"c{c}_x{it}"] = x
        out[f"c{c}_Pa"] = Pa
        out[f"c{c}_model"] = model
    np.savez_compressed(os.path.join(HERE, "kfconv.npz"), **out)


if __name__ == "__main__":
    main()
