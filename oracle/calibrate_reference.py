"""Calibration of the sampled reference CPU arm of bench.py -- TEST
INFRASTRUCTURE ONLY (runs the reference's routines compiled from source in
oracle/_ref; nothing here is part of the product path).

bench.py --impl reference, and the cpu_baseline leg of the GPU run, time the
reference's own per-slice routines in the reference's OpenMP phase loops
(oracle/ref_shim.cpp: ref_conv_slices, ref_radial_lines, ref_local_systems)
on bounded samples of one step and extrapolate each phase to a full step.
This script measures that extrapolation against full steps of the same phase
loops on the same host and the same inputs (bench.py's workload: seed 2, its
hourly Kp series):

  cfg1  24 x 25 x 31 x 31:  every convection slice, radial line and local
                            system (LU_CACHING form: all systems factored
                            once, then a timed cached solve)
  cfg2  48 x 101 x 101 x 91: every convection slice and every radial line;
                            the local phase stays sampled (its full LU cache
                            needs 110 GB of host memory)

and prints one JSON line per configuration with the sampled and the measured
seconds per phase and their ratio.

    python oracle/calibrate_reference.py --config cfg1 [--threads N]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [ROOT, HERE, os.path.join(ROOT, "verb-4d_b200")]
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import bench  # noqa: E402
from verb4d_b200 import workload as W  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="cfg1", choices=["cfg1", "cfg2"])
    ap.add_argument("--samples", type=int, default=3)
    args = ap.parse_args()
    spec = W.CONFIGS[args.config]
    wl = W.make_workload(spec, seed=2, kp=W.kp_series(2, 24))
    rs = bench.ReferenceSampler(wl)
    P, R, V, K = spec.shape
    est = {"convection": [], "radial": [], "local": [], "factor_per_step": []}
    for _ in range(args.samples):
        rs.sample_step()
        for k, v in rs.last_phases.items():
            est[k].append(v)
    est = {k: float(np.mean(v)) for k, v in est.items()}
    ip = ctypes.POINTER(ctypes.c_int)
    st = ctypes.byref(rs.state.st)
    vk = np.array([(v, k) for v in range(V - 1, -1, -1) for k in range(K)], dtype=np.int32)
    t0 = time.perf_counter()
    rs.lib.ref_conv_slices(st, ctypes.c_double(wl.dt), vk.ctypes.data_as(ip), ctypes.c_int(V * K),
                           ctypes.c_int(rs.cores))
    full = {"convection": time.perf_counter() - t0}
    pvk = np.array([(p, v, k) for p in range(P) for v in range(V) for k in range(K)],
                   dtype=np.int32)
    t0 = time.perf_counter()
    rs.lib.ref_radial_lines(st, ctypes.c_double(wl.dt), pvk.ctypes.data_as(ip),
                            ctypes.c_int(len(pvk)), ctypes.c_int(rs.cores))
    full["radial"] = time.perf_counter() - t0
    if args.config == "cfg1":
        n, ldab = V * K, 3 * (V + 1) + 1
        pr = np.array([(p, r) for p in range(P) for r in range(R)], dtype=np.int32)
        lu = np.zeros(P * R * ldab * n)
        piv = np.zeros(P * R * n, dtype=np.int64)
        dp, lp = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_long)

        def local(recompute):
            t0 = time.perf_counter()
            rs.lib.ref_local_systems(st, ctypes.c_double(wl.dt), ctypes.c_double(wl.sub_dt),
                                     pr.ctypes.data_as(ip), ctypes.c_int(P * R), lu.ctypes.data_as(dp),
                                     piv.ctypes.data_as(lp), ctypes.c_int(recompute),
                                     ctypes.c_int(rs.cores))
            return time.perf_counter() - t0

        full["factor_per_step"] = local(1) / 288.0
        full["local"] = local(0)
    ratio = {k: round(full[k] / est[k], 3) for k in full}
    tot_est = sum(est.values())
    tot_full = sum(full.get(k, est[k]) for k in est)
    print(json.dumps({"config": args.config, "shape": spec.shape, "threads": rs.cores,
                      "samples": args.samples,
                      "sampled_s_per_step": {k: round(v, 4) for k, v in est.items()},
                      "full_s_per_step": {k: round(v, 4) for k, v in full.items()},
                      "full_over_sampled": ratio,
                      "step_full_over_sampled": round(tot_full / tot_est, 3)}), flush=True)


if __name__ == "__main__":
    main()
