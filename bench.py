"""Benchmark: sim-hours/s of the VERB-4D operator-split step.

Workload (default): the production-size run, 101 L x 101 E x 91 alpha x 48 MLT
(reference layout P=48, R=101, V=101, K=91), dt = 5 min, seeded synthetic
inputs (see verb-4d_b200/verb4d_b200/workload.py) with an hourly Kp series in
[1, 6]: D_LL follows Kp through its scale factor and the drift velocities are
replaced every simulated hour.  One bench step = one time step of the full
operator split (convection, radial diffusion, local diffusion with cached LU
factors, negative-point count).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config cfg2|cfg1]
  python bench.py --impl reference ...   # the reference CPU path, sampled

Ours: W warm-up steps start the run (they include the one-time LU and Thomas
factorisations), then K steps are timed with CUDA events on the context's
stream, bracketed by barrier + synchronize, max over ranks.  Inputs are
resident in HBM (hourly velocity fields pre-staged on the device).  The local
LU factors (110 GB) exceed the 126 MB L2 many times over, so every timed step
streams from HBM.  `e2e` re-runs K steps from a fresh context through the
public API with host buffers: all inputs uploaded from host memory inside the
timed region, hourly velocity uploads, the negative-point count read back
every step and the PSD read back every simulated hour.
N GPUs run N independent replicas (the run does not shard): weak scaling.
"""
from __future__ import annotations

import argparse
import copy
import ctypes
import json
import os
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "verb-4d_b200"))

METRIC = "sim-hours/s at 101x101x91x48"
MEASURED = os.path.join(ROOT, "MEASURED_PEAKS.json")
HBM_FALLBACK = 6650.0


# --------------------------------------------------------------------------- utils
# DRAM bytes per algorithmic byte of the local solve: one ncu capture at
# 48x101x101x8 (the production band, 4848 systems of 808 unknowns) read
# 9,735,437,568 + wrote 66,170,624 bytes for 9,698,947,584 algorithmic bytes
SOLVE_TRAFFIC_PER_ALG_BYTE = (9735437568 + 66170624) / 9698947584


CONV_LABEL = {
    "fma": "fma: multiply-add contraction, within 1e-12 of the reference per step",
    "stream": ("stream: one thread per line, all stages of a pass in registers, multiply-add "
               "contraction, within 1e-12 of the reference per step"),
    "exact": "exact: bit-identical to the reference",
}

def rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value, device=None):
    """The largest of every rank's value (a time: the job ends with its
    slowest replica); the value itself in a single process."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(sim_hours_per_rank, seconds_max, world):
    """Whole-job sim-hours/s of `world` independent replicas that each
    simulate `sim_hours_per_rank`, timed by the slowest one."""
    return world * sim_hours_per_rank / seconds_max


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=10)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = [r.split(",") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "reasons": reasons}


FP64_OPS_PER_FACE = 179
# FP64-pipe share of each convection kernel's active cycles (ncu
# sm__inst_executed_pipe_fp64 over one launch at 48 x 101 x 101 x 8); the
# op-count fraction above counts the reference's operations, the pipe share
# the ones the kernel issues
CONV_FP64_PIPE_NCU = {"fma": 0.336, "stream": 0.402, "exact": 0.471}
CONV_KERNEL = {"fma": "conv_fma::convection_kernel (nine warps per line job set)",
               "stream": "convection_stream_kernel (one thread per line)",
               "exact": "conv_exact::convection_kernel"}


def fp64_peak_tops():
    try:
        with open(MEASURED) as f:
            mhz = float(json.load(f)["sm_max_mhz"])
    except (OSError, KeyError, ValueError):
        mhz = 1965.0
    return round(148 * 64 * mhz * 1e6 / 1e12, 2)


def measured_peaks():
    try:
        with open(MEASURED) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK, "fallback"


# --------------------------------------------------------------------------- ours
def run_ours(args):
    import torch
    import torch.distributed as dist

    from verb4d_b200 import Context, Solver
    from verb4d_b200 import workload as W

    rank, world, local = rank_info()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # a dedicated (non-default) stream: the library launches every kernel on it and
    # the CUDA events below are recorded on it
    stream = torch.cuda.Stream(dev)
    spec = W.CONFIGS[args.config]
    hours = int(np.ceil((args.warmup + args.steps + 1) * W.DT_5MIN * 24)) + 1
    kp = W.kp_series(args.seed + rank, max(hours, 24))
    wl = W.make_workload(spec, seed=args.seed + rank, kp=kp)
    hrs = sorted({min(int(np.floor(it * wl.dt * 24 + 1e-9)), len(kp) - 1)
                  for it in range(1, args.warmup + args.steps + 2)})
    vel_host = {h: W.drift_velocities(spec, float(kp[h])) for h in hrs}

    # ---------------- device-resident run (value)
    vel_dev = {h: (torch.from_numpy(vp).to(dev), torch.from_numpy(vr).to(dev))
               for h, (vp, vr) in vel_host.items()}
    torch.cuda.synchronize(dev)

    def make_solver(form, conv=None, trim=None, refine=None):  # noqa: C901
        sv = Solver(wl, stream=stream.cuda_stream, velocity_provider=None)
        sv.load()
        ref = (args.refine if form == "mixed" else 0) if refine is None else refine
        sv.ctx.set_local_precision(form, ref)
        sv.ctx.set_convection_arith(conv or args.conv)
        if args.trim if trim is None else trim:
            sv.ctx.set_local_trim(W.loss_cone_k0(wl))
        return sv

    solver = make_solver(args.form)
    ctx = solver.ctx
    lib = ctx.lib

    def update_dev(it, sv=None):
        sv = sv or solver
        h = min(int(np.floor(it * wl.dt * 24 + 1e-9)), len(kp) - 1)
        if h != sv.hour:
            sv.hour = h
            sv.ctx.set_scale("DLL", wl.dll_scale(h))
            vp, vr = vel_dev[h]
            lib.verb_upload_field_device(sv.ctx.h, 10, vp.data_ptr())
            lib.verb_upload_field_device(sv.ctx.h, 11, vr.data_ptr())

    fl = wl.flags
    t_w0 = time.perf_counter()
    ctx.set_timing(True)
    psd_step1 = None
    for it in range(1, args.warmup + 1):
        update_dev(it)
        ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], fl["run_local"])
        if it == 1 and args.form == "mixed":
            psd_step1 = ctx.download()  # one step from the initial state (untimed)
    ctx.sync()
    warm = ctx.timing()
    warm_s = time.perf_counter() - t_w0
    tune = None
    if args.autotune and fl["run_local"]:
        # untimed: pick the local-solve shape for this grid on its own systems
        ch, tms = ctx.autotune_local_solve(wl.dt, wl.sub_dt)
        shapes = ctx.solve_variants()
        key = lambda sh: "%dx%dx%d%s" % (sh[0], sh[1], sh[2], "r" if sh[3] else "")  # noqa: E731
        tune = {"local_solve_shapes_ms": {key(sh): round(float(t), 3)
                                          for sh, t in zip(shapes, tms)},
                "chosen": key(shapes[ch]) + " (systems per CTA x L columns x U columns in "
                                            "flight; r: right-hand-side window in registers)"}
    ctx.set_timing(False)
    ctx.set_timing(True)  # zeroes the counters
    if args.graph:
        # steps replayed from the captured graph: no per-phase events in the
        # timed region (the phase split comes from extra steps after it)
        ctx.set_timing(False)
        ctx.set_step_graph(True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for it in range(args.warmup + 1, args.warmup + args.steps + 1):
            update_dev(it)
            ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], fl["run_local"])
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ctx.sync()
    ms = ev0.elapsed_time(ev1)
    tm = ctx.timing()
    tph, nph = tm, args.steps
    psd_timed_end = ctx.download() if args.form == "mixed" else None
    if args.graph:
        # per-phase times from a few more eager steps (outside the timed region)
        ctx.set_step_graph(False)
        nph = 3
        ctx.set_timing(True)
        for it in range(args.warmup + args.steps + 1, args.warmup + args.steps + 1 + nph):
            update_dev(it)
            ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], fl["run_local"])
        ctx.sync()
        tph = ctx.timing()
    neg = ctx.negative_count()
    dev_bytes = ctx.device_bytes()
    conv_substeps = int(ctx.convection_substeps().astype(np.int64).sum())
    form_info = None
    if args.form == "mixed":
        # the same steps in the FP64 form, for the error of the mixed form and
        # the FP64 time on the same box
        psd_mixed = psd_timed_end
        corr = ctx.local_refinement()
        ctx.close()
        del solver, ctx
        sv = make_solver("fp64")
        for it in range(1, args.warmup + 1):
            update_dev(it, sv)
            sv.ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], fl["run_local"])
            if it == 1:
                p64 = sv.ctx.download()
                err1 = float(np.abs(psd_step1 - p64).max() / np.abs(p64).max())
        sv.ctx.sync()
        sv.ctx.set_timing(True)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for it in range(args.warmup + 1, args.warmup + args.steps + 1):
            update_dev(it, sv)
            sv.ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], fl["run_local"])
        e1.record(stream)
        torch.cuda.synchronize(dev)
        tm64 = sv.ctx.timing()
        psd64 = sv.ctx.download()
        sv.ctx.close()
        del sv
        # one step with FP64 factors and 3 FP64 refinement steps: the FP64 path
        # itself is only accurate to ~kappa*eps64 on these stiff systems
        sv = Solver(wl, stream=stream.cuda_stream, velocity_provider=None)
        sv.load()
        sv.ctx.set_local_precision("fp64", 3)
        sv.ctx.set_convection_arith(args.conv)
        if args.trim:
            sv.ctx.set_local_trim(W.loss_cone_k0(wl))
        update_dev(1, sv)
        sv.ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], fl["run_local"])
        p64r = sv.ctx.download()
        sv.ctx.close()
        del sv
        rel = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())  # noqa: E731
        err = float(np.abs(psd_mixed - psd64).max() / np.abs(psd64).max())
        form_info = {"form": "mixed", "refinements": args.refine,
                     "max_rel_err_one_step": err1, "tolerance": 1e-8,
                     "max_rel_err_one_step_vs_fp64_refined": rel(psd_step1, p64r),
                     "fp64_vs_fp64_refined_one_step": rel(p64, p64r),
                     "max_rel_err_after_run": err,
                     "last_relative_correction": corr,
                     "fp64_ms_per_step": round(e0.elapsed_time(e1) / args.steps, 3),
                     "fp64_local_solve_ms_per_step": round(tm64["local_solve_ms"] / args.steps, 3),
                     "err_measured_after_steps": args.warmup + args.steps}
    else:
        ctx.close()
        del solver, ctx
    ms = max_over_ranks(ms, dev)
    sim_h = args.steps * wl.dt * 24.0
    value = replica_throughput(sim_h, ms / 1e3, world)

    # ---------------- the forms side by side (same box, same inputs): the
    # plain FP64 form (the reference's arithmetic), the benchmarked form and
    # the mixed-precision forms; per form the time per step over
    # --form-steps graph-replayed steps and the one-step error against the
    # plain form from the same initial state
    forms = None
    if not args.no_forms:
        forms = measure_forms(args, wl, make_solver, update_dev, stream, dev)
        if world == 1 and args.learned_epochs > 0:
            # the Krylov form with the learned preconditioner is defined at the
            # 24 x 25 x 31 x 31 size (its systems fit one CTA's shared memory)
            torch.cuda.empty_cache()
            forms["learned_krylov_24x25x31x31"] = measure_learned(args.learned_epochs)

    # ---------------- end to end through the public API with host buffers (e2e)
    e2e = None
    if not args.no_e2e:
        torch.cuda.empty_cache()
        del vel_dev
        torch.cuda.empty_cache()

        # the caller's host buffers: page-locked, as a production driver keeps
        # its input and output arrays (filled before the timed region)
        keep = []

        def pinned(a):
            a = np.asarray(a)
            t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            keep.append(t)
            out = t.numpy()
            out[...] = a
            return out

        host_kind = "page-locked"
        try:
            wl_host = copy.copy(wl)
            wl_host.fields = {k: pinned(v) for k, v in wl.fields.items()}
            vel_pinned = {h: (pinned(vp), pinned(vr)) for h, (vp, vr) in vel_host.items()}
        except RuntimeError:
            # the host could not lock that much memory (many ranks on one
            # node): the same run from pageable buffers
            keep.clear()
            host_kind = "pageable (page-locking failed)"
            wl_host = wl
            vel_pinned = vel_host

        def host_provider(h):
            return vel_pinned[h]

        psd_out = pinned(np.zeros(spec.shape)) if keep else np.zeros(spec.shape)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        s2 = Solver(wl_host, stream=stream.cuda_stream, velocity_provider=host_provider)
        s2.load()
        s2.ctx.set_local_precision(args.form, args.refine if args.form == "mixed" else 0)
        s2.ctx.set_convection_arith(args.conv)
        s2.ctx.set_step_graph(bool(args.graph))
        if args.trim:
            s2.ctx.set_local_trim(W.loss_cone_k0(wl))
        h2d = sum(np.asarray(v).nbytes for k, v in wl_host.fields.items() if k != "DLL")
        d2h = 0
        for it in range(1, args.steps + 1):
            h_before = s2.hour
            s2.step(it, count_negatives=True)
            d2h += 8
            if s2.hour != h_before:
                h2d += 2 * psd_out.nbytes
            if it % 12 == 0 or it == args.steps:
                lib.verb_download_psd(s2.ctx.h, psd_out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
                d2h += psd_out.nbytes
        s2.ctx.sync()
        torch.cuda.synchronize(dev)
        e2e_s = time.perf_counter() - t0
        s2.ctx.close()
        e2e_s = max_over_ranks(e2e_s, dev)
        e2e = {"value": replica_throughput(sim_h, e2e_s, world), "unit": "sim-hours/s",
               "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
               "includes": "host upload of every input field, one-time LU/Thomas factorisations, "
                           "hourly velocity uploads, per-step negative count and hourly PSD reads",
               "host_buffers": host_kind}
        del keep, wl_host, vel_pinned

    # ---------------- roofline of the local solve (HBM-bound)
    P, R, V, K = spec.shape
    n = V * K
    kl, kv = V + 1, 2 * (V + 1)
    nsys = P * R
    fbytes = 4 if args.form == "mixed" else 8  # factor storage
    alg_bytes = nsys * (n * (kl + kv + 1) * fbytes + n * 4 + 2 * n * 8)  # band factors + pivots + rhs/x
    solve_ms = tph["local_solve_ms"] / max(tph["local_solve_launches"], 1)
    hbm_peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (solve_ms / 1e3) / 1e9
    conv_ms = tph["convection_ms"] / nph
    # FP64 roofline of convection: the reference's arithmetic per face update
    # (9th-order face 136 ops, limiter 35 incl. comparisons, two cell updates
    # 8) over the faces one outer sub-step sweeps, times the slice sub-steps of
    # the last timed step; peak = FP64 issue rate (64 lanes/SM/clock) at the
    # maximum SM clock
    p_faces = (R - 1) * (P if wl.bc_types["Pl"] == W.BC_PERIODIC else P - 1)
    r_faces = P * (R if wl.bc_types["Rl"] == W.BC_PERIODIC else R - 1)
    conv_ops = FP64_OPS_PER_FACE * (p_faces + r_faces) * conv_substeps
    fp64_peak = fp64_peak_tops()
    conv_tops = conv_ops / (conv_ms / 1e3) / 1e12
    out = {
        "metric": metric_name(spec),
        "value": round(value, 5), "unit": "sim-hours/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.form == "fp64" else "f64 (local LU factors stored f32)",
        "data": "synthetic (seeded)",
        "config": workload_config(args, spec, world),
        "impl": {"local_systems": "loss-cone trimmed (ragged)" if args.trim else "full",
                 "local_precision": args.form,
                 "step_launch": "CUDA graph replay" if args.graph else "eager launches",
                 "convection_arith": CONV_LABEL[args.conv]},
        "phases_ms_per_step": {"convection": round(conv_ms, 3),
                               "radial": round(tph["radial_ms"] / nph, 3),
                               "local_solve": round(tph["local_solve_ms"] / nph, 3),
                               "local_total": round(tph["local_ms"] / nph, 3),
                               "reduce": round(tph["reduce_ms"] / nph, 3),
                               "radial_factor": round(tph["radial_factor_ms"] / nph, 3),
                               "measured_over": ("3 eager steps after the timed region"
                                                 if args.graph else "the timed steps")},
        "one_time": {"local_lu_factor_ms": round(warm["local_factor_ms"], 1),
                     "radial_factor_ms": round(warm["radial_factor_ms"], 3),
                     "warmup_wall_s": round(warm_s, 2)},
        "roofline": {"kernel": "local_solve_kernel (banded LU forward/back substitution)",
                     "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                     "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "algorithmic_bytes_per_launch": int(alg_bytes),
                     "traffic": (args.traffic if args.traffic is not None
                                 else int(alg_bytes * SOLVE_TRAFFIC_PER_ALG_BYTE)),
                     "traffic_source": ("given on the command line" if args.traffic is not None
                                        else "algorithmic bytes x 1.0106, the DRAM/algorithmic "
                                             "ratio of one ncu-captured launch at 48x101x101x8 "
                                             "(the 48x101x101x91 band, kl = 102)")},
        "roofline_fp64": {"kernel": CONV_KERNEL[args.conv] + ", ULTIMATE-QUICKEST sweeps, FP64",
                          "bound": "fp64", "achieved": round(conv_tops, 3), "peak": fp64_peak,
                          "unit": "TOP/s", "frac": round(conv_tops / fp64_peak, 4),
                          "peak_source": "nominal FP64 issue rate, 148 SMs x 64 lanes at "
                                         "MEASURED_PEAKS.json sm_max_mhz",
                          "fp64_ops_per_face": FP64_OPS_PER_FACE,
                          "fp64_pipe_active_ncu": CONV_FP64_PIPE_NCU[args.conv],
                          "fp64_pipe_source": "ncu inst_executed_pipe_fp64 over active cycles, "
                                              "one launch of this kernel at 48x101x101x8",
                          "face_updates_per_step": int((p_faces + r_faces) * conv_substeps)},
        "autotune": tune,
        "clocks": clk.summary(),
        "gpu_launches": int(tm["kernel_launches"]),
        "negative_points_end": int(neg),
        "device_gb": round(dev_bytes / 1e9, 2),
    }
    if e2e:
        out["e2e"] = e2e
    if form_info:
        out["form"] = form_info
    if forms:
        out["forms"] = forms
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        cb = reference_estimate(wl, budget_s=args.cpu_budget)
        out["cpu_baseline"] = {"value": round(cb["value"], 8), "unit": "sim-hours/s",
                               "cores": cb["cores"], "kind": "reference", "sample": cb["sample"]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def metric_name(spec):
    """The metric's label: sim-hours/s at L x E x alpha x MLT."""
    if (spec.R, spec.V, spec.K, spec.P) == (101, 101, 91, 48):
        return METRIC
    return f"sim-hours/s at {spec.R}x{spec.V}x{spec.K}x{spec.P}"


def timed_hours(args, dt):
    """Simulated hours (of the Kp series) that the timed steps
    warmup+1 .. warmup+steps fall in."""
    return sorted({int(np.floor(it * dt * 24 + 1e-9))
                   for it in range(args.warmup + 1, args.warmup + args.steps + 1)})


def workload_config(args, spec, world):
    """The workload both arms run (identical in their JSON lines)."""
    from verb4d_b200 import workload as W

    return {"workload": f"VERB-4D operator-split step {args.config} (P,R,V,K)={spec.shape}, "
                        f"dt=5 min, hourly Kp in [1,6] (seed {args.seed})",
            "P_mlt": spec.P, "R_L": spec.R, "V_energy": spec.V, "K_alpha": spec.K, "dt_min": 5,
            "kp_hours_timed": timed_hours(args, W.DT_5MIN),
            "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (110 GB of LU factors streamed per step)"}


# --------------------------------------------------------------------------- forms
FORMS = {
    # name: (local precision, FP64 refinement steps, convection arithmetic)
    "plain_fp64": ("fp64", 0, "exact"),
    "fp64_fma": ("fp64", 0, "fma"),
    "fp64_stream": ("fp64", 0, "stream"),
    "mixed_stream": ("mixed", 2, "stream"),
    # the accuracy reference: FP64 factors and three FP64 refinement steps
    # (the plain LU itself carries kappa*eps64 ~ 1e-7 on these systems)
    "fp64_refined_exact": ("fp64", 3, "exact"),
}


def measure_forms(args, wl, make_solver, update_dev, stream, dev):
    """Time every form of FORMS for args.form_steps graph-replayed steps after
    3 warm-up steps (the first of which factorises and gives the one-step
    PSD) and the local-solve autotuner, one context at a time (each FP64
    context holds 110 GB of factors); the one-step error of each form is
    measured against the plain FP64 form (the reference's arithmetic) and
    against the refined FP64 form (the most accurate)."""
    import torch

    fl = wl.flags
    out = {}
    psd1 = {}
    for name, (prec, refine, conv) in FORMS.items():
        sv = make_solver(prec, conv=conv, trim=False, refine=refine)
        sv.hour = -1
        for it in range(1, 4):
            update_dev(it, sv)
            sv.ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], fl["run_local"])
            if it == 1:
                psd1[name] = sv.ctx.download()
        sv.ctx.sync()
        sv.ctx.autotune_local_solve(wl.dt, wl.sub_dt)
        sv.ctx.set_step_graph(True)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for it in range(4, 4 + args.form_steps):
            update_dev(it, sv)
            sv.ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], fl["run_local"])
        e1.record(stream)
        torch.cuda.synchronize(dev)
        sv.ctx.sync()
        msf = e0.elapsed_time(e1) / args.form_steps
        sv.ctx.close()
        del sv
        out[name] = {"ms_per_step": round(msf, 3), "local_precision": prec,
                     "refinements": refine, "convection_arith": conv}
    rel = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())  # noqa: E731
    plain = out["plain_fp64"]["ms_per_step"]
    for name, v in out.items():
        v["speedup_vs_plain_fp64"] = round(plain / v["ms_per_step"], 3)
        v["err_one_step_vs_plain_fp64"] = rel(psd1[name], psd1["plain_fp64"])
        v["err_one_step_vs_fp64_refined"] = rel(psd1[name], psd1["fp64_refined_exact"])
    return {"forms": out, "steps_timed": args.form_steps,
            "error": "norm-wise max|psd - psd_ref| / max|psd_ref| after one step from the same "
                     "initial state; the bar is 1e-8",
            "timing": "CUDA events, graph-replayed steps after 3 warm-up steps and the "
                      "local-solve autotuner, one context at a time"}


# --------------------------------------------------------------------------- learned form
def run_learned(args):
    """The learned form at the 24 x 25 x 31 x 31 size: the CNN's training
    step on the tensor cores (256 images of 31 x 31), the learned
    preconditioner trained on the systems of five seeds, and the local step
    of a held-out seed by the LU, by the Krylov form with the Jacobi
    preconditioner and with the learned one (iterations, fallback rate, time,
    agreement with the LU step)."""
    import torch

    from verb4d_b200 import learned
    from verb4d_b200 import workload as W

    torch.cuda.set_device(0)
    spec = W.CONFIGS["cfg1"]
    _, _, V, K = spec.shape
    out = {"metric": "local step ms at 25x31x31x24 (learned form)", "unit": "ms",
           "higher_is_better": False, "n_gpus": 1, "data": "synthetic (seeded)",
           "config": {"workload": "local (V,K) step of the 24 x 25 x 31 x 31 grid, dt=5 min"}}
    # CNN training step on the tensor cores
    B = 256
    net = learned.CNN(K, V, B, seed=1)
    x = torch.randn((B, 4, K, V), device="cuda")
    t = torch.randn((B, 1, K, V), device="cuda")
    for _ in range(3):
        net.train_step(x.data_ptr(), t.data_ptr(), B, 1e-3)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        net.train_step(x.data_ptr(), t.data_ptr(), B, 1e-3)
    e1.record()
    torch.cuda.synchronize()
    out["cnn_train_step_ms"] = round(e0.elapsed_time(e1) / 10, 3)
    net.close()
    if args.learned_epochs <= 0:
        print(json.dumps(out), flush=True)
        return
    out.update(measure_learned(args.learned_epochs))
    out["value"] = out["local_step"]["krylov_learned"]["ms"]
    print(json.dumps(out), flush=True)


def measure_learned(epochs):
    """The learned preconditioner at the 24 x 25 x 31 x 31 size, trained on
    the local systems of five seeds, and the local step of a held-out seed by
    the LU (factorisation included), by the Krylov form with the Jacobi
    preconditioner and with the learned one: time, BiCGSTAB iterations per
    Krylov-solved system, LU-fallback rate and distance from the LU step."""
    import torch

    from verb4d_b200 import Solver, learned
    from verb4d_b200 import workload as W

    spec = W.CONFIGS["cfg1"]
    P, R, V, K = spec.shape
    nsys = P * R
    out = {}
    # the learned preconditioner
    t0 = time.perf_counter()
    base = W.make_workload(spec, seed=1, sources=True, losses=True)
    feat, A9 = learned.precond_inputs(base, seeds=range(2, 7))
    pc = learned.CNN(K, V, max(nsys, 64), channels=learned.PC_CHANNELS, seed=0)
    pc.zero_last_layer()
    hist = learned.train_preconditioner(pc, feat, A9, V, K, epochs=epochs, batch=64)
    out["precond_training"] = {"seconds": round(time.perf_counter() - t0, 1),
                               "systems": int(feat.shape[0]), "epochs": epochs,
                               "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1]}
    wl = W.make_workload(spec, seed=100, sources=True, losses=True)
    fl = wl.flags

    def split():
        s = Solver(wl)
        s.load()
        s.ctx.step(wl.dt, wl.sub_dt, fl["run_convection"], fl["run_radial"], 0)
        return s

    def timed(fn):
        torch.cuda.synchronize()
        a = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, (time.perf_counter() - a) * 1e3

    s = split()
    s.ctx.local(wl.dt, wl.sub_dt)
    s.ctx.sync()
    s.ctx.close()
    s = split()
    _, lu_ms = timed(lambda: (s.ctx.local(wl.dt, wl.sub_dt), s.ctx.sync()))
    ref = s.ctx.download()
    s.ctx.close()
    res = {"lu": {"ms": round(lu_ms, 2), "note": "factorisation included"}}
    for name, net_pc in (("krylov_jacobi", None), ("krylov_learned", pc)):
        calls = []
        for rep in range(3):  # the first call allocates; the best of the others
            s = split()
            s.ctx.set_krylov_preconditioner(net_pc)
            st, ms = timed(lambda: (s.ctx.local_krylov(wl.dt, wl.sub_dt, guess="prev"),
                                    s.ctx.sync())[0])
            got = s.ctx.download()
            s.ctx.close()
            calls.append(round(ms, 2))
        ms = min(calls[1:])
        ns = max(st["systems"] - st["fallbacks"], 1)
        res[name] = {"ms": round(ms, 2), "calls_ms": calls,
                     "iterations_per_krylov_solved_system": round(st["solved_iterations"] / ns, 1),
                     "fallback_rate": round(st["fallbacks"] / st["systems"], 4),
                     "max_rel_err_vs_lu_step": float(np.abs(got - ref).max() / np.abs(ref).max())}
    for name in ("krylov_jacobi", "krylov_learned"):
        res[name]["time_vs_lu"] = round(res[name]["ms"] / lu_ms, 3)
    out["local_step"] = res
    out["timing"] = ("host wall time of one local step (synchronised on both sides) on a "
                     "fresh context, the best of the second and third of three calls")
    pc.close()
    return out


# --------------------------------------------------------------------------- ensemble
def run_ensemble(args):
    """64-member ensemble (grids drawn from {51,76,101} L x {61,101} E x
    {61,91} alpha x {24,48} MLT, own seeded Kp series each), admitted in waves
    by an HBM budget of 90 % of the free device memory; hourly radial Kalman
    updates with 500 synthetic observations (5 % log-normal noise)."""
    import torch

    from verb4d_b200 import ensemble as E

    torch.cuda.set_device(0)
    free, _ = torch.cuda.mem_get_info()
    members = E.draw_members(args.members, seed=args.seed)
    ens = E.Ensemble(members, budget_bytes=int(free * 0.9), steps=args.ens_steps, kf_every=12,
                     n_obs=500, obs_noise=0.05)
    with ClockSampler(0) as clk:
        r = ens.run()
    out = {"metric": f"member sim-hours/s ({args.members}-member ensemble)",
           "value": round(r["member_sim_hours_per_s"], 5), "unit": "sim-hours/s",
           "n_gpus": 1, "steps": args.ens_steps, "higher_is_better": True, "dtype": "f64",
           "data": "synthetic (seeded)",
           "config": {"workload": "ensemble: grids from {51,76,101} L x {61,101} E x {61,91} alpha "
                                  "x {24,48} MLT, dt=5 min, hourly Kp in [1,6], hourly radial KF "
                                  "with 500 observations", "members": args.members},
           "ensemble": r, "clocks": clk.summary(),
           "timing": "host wall time of the whole ensemble (members of a wave run concurrently; "
                     "input generation on the host included)"}
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------------------- reference CPU path
class ReferenceSampler:
    """Times the reference's own routines (oracle/_ref, compiled from source) on
    bounded samples of one step of the workload and extrapolates to full steps.

    The phase loops are the reference's OpenMP loops (src/VERB4D_Solver.cpp
    convection :885-978, radial :1009-1070, local :1101-1216, schedule(dynamic,1)
    over independent slices), compiled in C++ around the unmodified routines
    (oracle/ref_shim.cpp), run over sampled slice lists on all host cores with
    OpenBLAS single-threaded.  Local diffusion is the LU_CACHING form: each
    sampled system is factored once (the factorisation amortised over a
    288-step run), then its cached dgbtrs solve is timed per step."""

    def __init__(self, wl, threads=None, seed=0):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        import oracle as O
        from verb4d_b200 import workload as W

        if not O.have_reference():
            O.build(with_ref=None)
        if not O.have_reference():
            raise RuntimeError("the reference library oracle/_ref is not built")
        self.lib = O.reference(lu_caching=True).lib
        self.wl = wl
        self.cores = threads or len(os.sched_getaffinity(0))
        self.rng = np.random.default_rng(seed)
        self.ns = W.convection_substeps(wl)
        # the 4-D fields in the oracle's state layout (no full-grid LU cache: the
        # sampled systems get their own cache slots below)
        self.state = O.OracleStepper(W.oracle_inputs(wl), O.reference(lu_caching=True),
                                     lu_cache=False)
        P, R, V, K = wl.spec.shape
        n = V * K
        ldab = 3 * (V + 1) + 1
        nsys = self.cores
        self.pr = np.array([(int(self.rng.integers(P)), int(self.rng.integers(R)))
                            for _ in range(nsys)], dtype=np.int32).ravel()
        self.lu = np.zeros(nsys * ldab * n)
        self.ipiv = np.zeros(nsys * n, dtype=np.int64)
        t0 = time.perf_counter()
        self._local(1)
        self.t_factor_step = (time.perf_counter() - t0) * (P * R) / nsys
        self.samples = 0

    def _local(self, recompute):
        wl = self.wl
        self.lib.ref_local_systems(ctypes.byref(self.state.st), ctypes.c_double(wl.dt),
                                   ctypes.c_double(wl.sub_dt),
                                   self.pr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   ctypes.c_int(len(self.pr) // 2),
                                   self.lu.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                   self.ipiv.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                                   ctypes.c_int(recompute), ctypes.c_int(self.cores))

    def set_hour(self, h):
        """Inputs of simulated hour h of the run: the hourly drift velocities
        and the D_LL scale of that hour's Kp (as the timed GPU steps see them)."""
        from verb4d_b200 import workload as W

        wl = self.wl
        h = min(int(h), len(wl.kp) - 1)
        if h == getattr(self, "hour", None):
            return
        self.hour = h
        vp, vr = W.drift_velocities(wl.spec, float(wl.kp[h]))
        self.state.keep["VP"][...] = vp
        self.state.keep["VR"][...] = vr
        self.state.keep["DLL"][...] = wl.fields["DLL_base"] * wl.dll_scale(h)
        w2 = copy.copy(wl)
        w2.fields = dict(wl.fields, VP=vp, VR=vr)
        self.ns = W.convection_substeps(w2)

    def sample_step(self, conv_slices=None):
        """Seconds for one full step on all host cores, from one bounded sample."""
        wl = self.wl
        P, R, V, K = wl.spec.shape
        ip = ctypes.POINTER(ctypes.c_int)
        nconv = min(conv_slices or self.cores, self.cores)
        # convection: a group of slices with (nearly) equal sub-step counts, one
        # per thread, around a point of the sorted counts drawn with
        # probability proportional to the sub-steps (where the step's work
        # is).  Each thread then carries the same work, so the wall time is the
        # per-thread time of ns_max sub-steps with all threads busy, and a full
        # step (dynamic scheduling over all slices, as the reference's loop)
        # is that per-sub-step time times the total sub-steps over the threads.
        flat = self.ns.ravel()
        order = np.argsort(flat, kind="stable")
        cum = np.cumsum(flat[order], dtype=np.float64)
        c = int(np.searchsorted(cum, self.rng.uniform(0.0, cum[-1]), side="right"))
        c = min(c, len(order) - 1)
        lo = max(0, min(c - nconv // 2, len(order) - nconv))
        pick = order[lo:lo + nconv]
        vk = np.array([divmod(int(i), K) for i in pick], dtype=np.int32)
        t0 = time.perf_counter()
        self.lib.ref_conv_slices(ctypes.byref(self.state.st), ctypes.c_double(wl.dt),
                                 vk.ctypes.data_as(ip), ctypes.c_int(nconv), ctypes.c_int(self.cores))
        t_c = time.perf_counter() - t0
        sub = int(flat[pick].sum())
        ns_max = int(flat[pick].max())
        t_conv = t_c / ns_max * float(self.ns.sum()) / self.cores
        # radial: whole runs of K (the fastest index) at random (P, V), in the
        # order the reference's collapse(3) loop visits lines, so that the
        # sampled lines share cache lines as the full loop's do
        nblk = max(1, (256 * self.cores + K - 1) // K)
        blk = [(int(self.rng.integers(P)), int(self.rng.integers(V))) for _ in range(nblk)]
        pvk = np.array([(p, v, k) for p, v in blk for k in range(K)], dtype=np.int32)
        nl = len(pvk)
        t0 = time.perf_counter()
        self.lib.ref_radial_lines(ctypes.byref(self.state.st), ctypes.c_double(wl.dt),
                                  pvk.ctypes.data_as(ip), ctypes.c_int(nl), ctypes.c_int(self.cores))
        t_rad = (time.perf_counter() - t0) * (P * V * K) / nl
        t0 = time.perf_counter()
        self._local(0)
        t_local = (time.perf_counter() - t0) * (P * R) / (len(self.pr) // 2)
        t_fac = self.t_factor_step / 288.0
        self.samples += 1
        self.last_phases = {"convection": t_conv, "radial": t_rad, "local": t_local,
                            "factor_per_step": t_fac}
        self.last = (f"reference routines from source in the reference's OpenMP phase loops "
                     f"(oracle/_ref), {self.cores} threads; per sample: {nconv} convection slices "
                     f"({sub} of {int(self.ns.sum())} slice-substeps), {nl} radial lines, "
                     f"{len(self.pr) // 2} local systems (LU_CACHING cached dgbtrs; factorisation "
                     f"amortised over 288 steps); extrapolated per step: convection {t_conv:.2f}s, "
                     f"radial {t_rad:.3f}s, local {t_local:.2f}s, factor/288 {t_fac:.3f}s")
        return t_conv + t_rad + t_local + t_fac

    def close(self):
        pass


def reference_estimate(wl, budget_s=20.0):
    """One bounded CPU-baseline sample (about `budget_s` seconds of host work)."""
    t0 = time.perf_counter()
    rs = ReferenceSampler(wl)
    steps = []
    while not steps or time.perf_counter() - t0 < 0.6 * budget_s:
        steps.append(rs.sample_step())
        if len(steps) >= 3:
            break
    rs.close()
    t_step = float(np.mean(steps))
    return {"value": wl.dt * 24.0 / t_step, "cores": rs.cores, "t_step_s": t_step,
            "sample": rs.last + f"; {len(steps)} sample(s) averaged"}


def run_reference(args):
    rank, world, local = rank_info()
    if rank != 0:
        return
    from verb4d_b200 import workload as W

    spec = W.CONFIGS[args.config]
    hours = int(np.ceil((args.warmup + args.steps + 1) * W.DT_5MIN * 24)) + 1
    # the Kp series of the GPU arm (rank 0's seed): the same inputs hour by hour
    wl = W.make_workload(spec, seed=args.seed, kp=W.kp_series(args.seed, max(hours, 24)))
    rs = ReferenceSampler(wl)
    # each bench step is one bounded sample of a full step of the same hour
    # as the GPU arm's step; a few convection slices per step keeps the
    # whole --steps/--warmup run within minutes
    nconv = max(1, min(rs.cores, int(8 * rs.cores * 4 / max(args.steps + args.warmup, 1))))
    hour = lambda it: int(np.floor(it * wl.dt * 24 + 1e-9))  # noqa: E731
    for it in range(1, args.warmup + 1):
        rs.set_hour(hour(it))
        rs.sample_step(nconv)
    t_total = 0.0
    for it in range(args.warmup + 1, args.warmup + args.steps + 1):
        rs.set_hour(hour(it))
        t_total += rs.sample_step(nconv)
    rs.close()
    sim_h = args.steps * wl.dt * 24.0
    value = sim_h / t_total
    out = {"metric": metric_name(spec),
           "value": value, "unit": "sim-hours/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(t_total / args.steps * 1e3, 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded)", "impl": "reference",
           "config": workload_config(args, spec, world),
           "impl": {"host_threads": rs.cores},
           "cpu_baseline": {"value": value, "unit": "sim-hours/s", "cores": rs.cores,
                            "kind": "reference", "sample": rs.last},
           "e2e": {"value": value, "unit": "sim-hours/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg2", choices=["cfg2", "cfg1", "cfg2s", "cfg2m"])
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--form", default="fp64", choices=["fp64", "mixed"],
                    help="local solve: FP64 factors, or FP32 factors with FP64 refinement")
    ap.add_argument("--refine", type=int, default=2, help="refinement steps of the mixed form")
    ap.add_argument("--autotune", type=int, default=1, choices=[0, 1],
                    help="time the local-solve shapes before the timed region and use the fastest")
    ap.add_argument("--graph", type=int, default=1, choices=[0, 1],
                    help="replay steady-state steps from a captured CUDA graph (1) or launch "
                         "them eagerly with per-phase events (0)")
    ap.add_argument("--conv", default="stream", choices=["fma", "exact", "stream"],
                    help="convection kernel: fma (contracted), stream (one thread per line, contracted) or exact (bit-identical)")
    ap.add_argument("--trim", action="store_true",
                    help="ragged local systems: pitch angles outside the loss cone only")
    ap.add_argument("--ensemble", action="store_true", help="run the member ensemble instead")
    ap.add_argument("--learned", action="store_true",
                    help="time the learned form (CNN training step, learned preconditioner)")
    ap.add_argument("--learned-epochs", type=int, default=12)
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--ens-steps", type=int, default=12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip timing the plain / mixed forms beside the main run")
    ap.add_argument("--form-steps", type=int, default=5)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--traffic", type=float, default=None,
                    help="dram bytes per local-solve launch from an ncu capture")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.ensemble:
        run_ensemble(args)
    elif args.learned:
        run_learned(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
