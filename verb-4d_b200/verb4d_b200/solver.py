"""Device-resident context and the whole-step driver.

``Context`` is a thin object wrapper over ``verb_ctx`` (include/verb4d_b200.h).
``Solver`` is the host side of the reference's time loop
(src/VERB4D_Solver.cpp:539-1282) for the data path: it uploads a
``Workload``'s fields once, applies the time-varying inputs when they change
(the D_LL scale of the hourly Kp series, hourly velocity fields), and calls
``verb_step`` once per time step.  Everything numerical runs in the CUDA
library; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L
from .workload import Workload, drift_velocities


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    def __init__(self, P: int, R: int, V: int, K: int, stream: int | None = None):
        self.lib = L.load()
        self.shape = (P, R, V, K)
        h = C.c_void_p()
        L.check(self.lib.verb_create(C.byref(h), P, R, V, K, C.c_void_p(stream or 0)),
                "verb_create")
        self.h = h

    # ---------------------------------------------------------------- inputs
    def upload(self, name: str, arr) -> None:
        a = _f64(arr)
        if name in L.FIELD_IDS:
            assert a.size == int(np.prod(self.shape)), name
            L.check(self.lib.verb_upload_field(self.h, L.FIELD_IDS[name], a.ctypes.data_as(L._dp)),
                    f"upload {name}")
        elif name in L.BC_FIELDS:
            L.check(self.lib.verb_upload_bc(self.h, L.BC_FIELDS.index(name),
                                            a.ctypes.data_as(L._dp)), f"upload {name}")
        else:
            raise KeyError(name)

    def set_scale(self, name: str, scale: float) -> None:
        L.check(self.lib.verb_set_field_scale(self.h, L.FIELD_IDS[name], float(scale)), "scale")

    def set_bc_types(self, types: dict) -> None:
        arr = (C.c_int * 10)(*[int(types[k]) for k in L.BC_FIELDS])
        L.check(self.lib.verb_set_bc_types(self.h, arr), "bc types")

    def set_options(self, radial_sources=0, local_sources=1, include_boundary=1, positive_psd=0):
        L.check(self.lib.verb_set_options(self.h, int(radial_sources), int(local_sources),
                                          int(include_boundary), int(positive_psd)), "options")

    def invalidate_lu(self) -> None:
        L.check(self.lib.verb_invalidate_lu(self.h), "invalidate")

    def set_local_precision(self, mode: str = "fp64", refinements: int = 0):
        """'fp64' (LAPACK-equivalent factors) or 'mixed' (the same factors stored
        in FP32); each solve is then refined `refinements` times in FP64."""
        m = {"fp64": L.VERB_PREC_FP64, "mixed": L.VERB_PREC_MIXED}[mode]
        L.check(self.lib.verb_set_local_precision(self.h, m, int(refinements)), "precision")

    def set_local_trim(self, k0=None):
        """Ragged local systems: k0[p, r] is the first pitch-angle index kept
        for system (p, r) (None: full systems)."""
        if k0 is None:
            L.check(self.lib.verb_set_local_trim(self.h, None), "trim")
            return
        a = np.ascontiguousarray(k0, dtype=np.int32).ravel()
        L.check(self.lib.verb_set_local_trim(self.h, a.ctypes.data_as(C.POINTER(C.c_int))), "trim")

    def assimilate_convection(self, obs, dt, model_error, obs_error, use_log=False,
                              correlation_time=float("inf"), growing_q=False,
                              has_vx_updated=False, slice_chunk=0) -> None:
        """Kalman-filter update of every (V,K) slice (convection data
        assimilation); obs is [P][R][V][K] with NaN where unobserved."""
        o = _f64(obs)
        L.check(self.lib.verb_assimilate_convection(
            self.h, o.ctypes.data_as(L._dp), float(dt), float(model_error), float(obs_error),
            int(use_log), float(correlation_time), int(growing_q), int(has_vx_updated),
            int(slice_chunk)), "assimilate_convection")

    def convection_da_state(self, v: int, k: int):
        """(Pa, model matrix) of slice (v, k) after a convection assimilation."""
        N = self.shape[0] * self.shape[1]
        pa = np.empty((N, N))
        mm = np.empty((N, N))
        L.check(self.lib.verb_convection_da_state(self.h, v, k, pa.ctypes.data_as(L._dp),
                                                  mm.ctypes.data_as(L._dp)), "da_state")
        return pa, mm

    def solve_variants(self) -> list:
        """(warps per CTA, L columns in flight, U columns in flight, window in
        registers) of every local-solve shape."""
        n = C.c_int()
        L.check(self.lib.verb_local_solve_variants(C.byref(n)), "variants")
        out = []
        for v in range(n.value):
            w, f, b, r = C.c_int(), C.c_int(), C.c_int(), C.c_int()
            L.check(self.lib.verb_local_solve_variant(v, C.byref(w), C.byref(f), C.byref(b)),
                    "variant")
            L.check(self.lib.verb_local_solve_variant_window(v, C.byref(r)), "variant window")
            out.append((w.value, f.value, b.value, r.value))
        return out

    def set_local_solve_variant(self, v: int = -1):
        L.check(self.lib.verb_set_local_solve_variant(self.h, int(v)), "solve_variant")

    def autotune_local_solve(self, dt: float, sub_dt: float):
        """Time every local-solve shape on this context's systems and keep the
        fastest; returns (chosen index, times in ms)."""
        shapes = self.solve_variants()
        t = np.zeros(len(shapes))
        ch = C.c_int()
        L.check(self.lib.verb_autotune_local_solve(self.h, float(dt), float(sub_dt),
                                                   t.ctypes.data_as(L._dp), C.byref(ch)),
                "autotune")
        return ch.value, t

    def set_step_graph(self, enable: bool = True):
        """Replay steady-state steps from a captured CUDA graph."""
        L.check(self.lib.verb_set_step_graph(self.h, int(enable)), "step_graph")

    def set_convection_arith(self, mode: str = "exact"):
        """"exact": bit-identical to the reference; "fma": multiply-add
        contraction, ~18 % faster, a few ulp per step from "exact";
        "stream": one thread per line, all stages of a pass at once in
        registers, contracted like "fma" (needs P and R >= 11, else runs
        the "fma" kernel)."""
        L.check(self.lib.verb_set_convection_arith(self.h, L.CONV_ARITH[mode]), "conv_arith")

    def local_krylov(self, dt: float, sub_dt: float, guess: str = "prev", cnn=None,
                     smooth: int = 0, omega: float = 2.0 / 3.0, max_outer: int = 10,
                     inner_maxit: int = 100, inner_tol: float = 1e-3,
                     resid_tol: float = 1e-10) -> dict:
        """The local step solved by FP64-refined FP32 BiCGSTAB from the given
        initial guess ("zero", "prev": the state the step starts from, or "cnn"
        with a learned.CNN) after
        `smooth` weighted-Jacobi sweeps, with the LU for systems that stay
        above resid_tol.  Returns the solve stats."""
        st = L.KrylovStats()
        L.check(self.lib.verb_local_krylov(self.h, dt, sub_dt, L.GUESS_IDS[guess],
                                           cnn.h if cnn is not None else None, smooth, omega,
                                           max_outer, inner_maxit, inner_tol, resid_tol,
                                           C.byref(st)),
                "local_krylov")
        return {k: getattr(st, k) for k, _ in L.KrylovStats._fields_}

    def set_krylov_preconditioner(self, net=None) -> None:
        """The learned sparse approximate inverse (a learned.CNN with 9 input
        and 25 output channels) as the preconditioner of local_krylov; None:
        Jacobi."""
        L.check(self.lib.verb_set_krylov_preconditioner(self.h, net.h if net is not None else None),
                "krylov preconditioner")
        self._pc = net  # keep the network alive while the context uses it

    def local_precond_inputs(self, dt: float, sub_dt: float, feat_ptr: int, A9_ptr: int) -> None:
        """The learned preconditioner's features [sys][9][K][V] and the FP32
        diagonals [sys][9][V*K] of every local system (device pointers)."""
        L.check(self.lib.verb_local_precond_inputs(self.h, float(dt), float(sub_dt),
                                                   C.c_void_p(feat_ptr), C.c_void_p(A9_ptr)),
                "precond inputs")

    def local_triples(self, dt: float, sub_dt: float, feat_ptr: int, target_ptr: int) -> None:
        """A local LU step that writes the CNN features and targets of every
        system into the device buffers at feat_ptr ([P*R][4][K][V] float32)
        and target_ptr ([P*R][K][V] float32)."""
        L.check(self.lib.verb_local_triples(self.h, dt, sub_dt, C.c_void_p(feat_ptr),
                                            C.c_void_p(target_ptr)), "local_triples")

    def remap_L(self, new_L):
        """Interpolate the PSD to a new L* grid and make it the L* field."""
        a = np.ascontiguousarray(new_L, dtype=np.float64)
        L.check(self.lib.verb_remap_L(self.h, a.ctypes.data_as(L._dp)), "remap_L")

    # ---- output and restart files (.pltb)
    def write_pltb(self, path: str, name: str = "psd", wait: bool = True):
        """Write a field as a .pltb file; with wait=False the write finishes in
        the background (output_wait() joins it)."""
        L.check(self.lib.verb_write_field_pltb(self.h, L.FIELD_IDS[name], path.encode(),
                                               0 if wait else 1), "write_pltb")

    def output_wait(self):
        L.check(self.lib.verb_output_wait(self.h), "output_wait")

    def read_pltb(self, path: str, name: str = "psd"):
        L.check(self.lib.verb_read_field_pltb(self.h, L.FIELD_IDS[name], path.encode()),
                "read_pltb")

    # ---- updatable fields (UpdatableMatrix / UpdatableListMatrix on the device)
    def add_component(self, name: str, base) -> int:
        """Turn field `name` into a component list (if it is not one yet) and
        add a component with the given base array; returns its index."""
        a = np.ascontiguousarray(base, dtype=np.float64)
        out = C.c_int()
        L.check(self.lib.verb_field_add_component(self.h, L.FIELD_IDS[name],
                                                  a.ctypes.data_as(L._dp), C.byref(out)),
                "add_component")
        return out.value

    def set_merge(self, name: str, merge: str = "sum"):
        L.check(self.lib.verb_field_set_merge(self.h, L.FIELD_IDS[name],
                                              {"sum": 0, "mean": 1}[merge]), "merge")

    def queue_data(self, name: str, comp: int, time: float, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        L.check(self.lib.verb_component_queue_data(self.h, L.FIELD_IDS[name], comp, float(time),
                                                   a.ctypes.data_as(L._dp)), "queue_data")

    def queue_scale(self, name: str, comp: int, time: float, scale: float):
        L.check(self.lib.verb_component_queue_scale(self.h, L.FIELD_IDS[name], comp, float(time),
                                                    float(scale)), "queue_scale")

    def queue_limit(self, name: str, comp: int, axis: int, which: str, time: float, value: float):
        L.check(self.lib.verb_component_queue_limit(self.h, L.FIELD_IDS[name], comp, int(axis),
                                                    {"from": 0, "to": 1}[which], float(time),
                                                    float(value)), "queue_limit")

    def update_fields(self, time: float) -> list:
        """Pop every queued update due at `time`; returns the rebuilt fields."""
        mask = C.c_uint()
        L.check(self.lib.verb_update_fields(self.h, float(time), C.byref(mask)), "update_fields")
        return [n for n, f in L.FIELD_IDS.items() if mask.value >> f & 1]

    def local_refinement(self) -> float:
        """max |d| / max |x| of the last refinement step (0 without refinement)."""
        out = C.c_double()
        L.check(self.lib.verb_local_refinement(self.h, C.byref(out)), "refinement")
        return out.value

    # ----------------------------------------------------------------- phases
    def convection(self, dt: float) -> None:
        L.check(self.lib.verb_convection(self.h, float(dt)), "convection")

    def radial(self, dt: float) -> None:
        L.check(self.lib.verb_radial(self.h, float(dt)), "radial")

    def local(self, dt: float, sub_dt: float) -> None:
        L.check(self.lib.verb_local(self.h, float(dt), float(sub_dt)), "local")

    def step(self, dt: float, sub_dt: float, run_convection=True, run_radial=True, run_local=True,
             count_negatives=False):
        cnt = C.c_longlong(-1)
        ptr = C.byref(cnt) if count_negatives else None
        L.check(self.lib.verb_step(self.h, float(dt), float(sub_dt), int(run_convection),
                                   int(run_radial), int(run_local), ptr), "step")
        return cnt.value if count_negatives else None

    def assimilate_radial(self, obs, dt, model_error, obs_error, p_index=0) -> None:
        o = _f64(obs)
        L.check(self.lib.verb_assimilate_radial(self.h, o.ctypes.data_as(L._dp), float(dt),
                                                float(model_error), float(obs_error),
                                                int(p_index)), "assimilate")

    def negative_count(self) -> int:
        cnt = C.c_longlong(0)
        L.check(self.lib.verb_negative_count(self.h, C.byref(cnt)), "negative count")
        return cnt.value

    def tensor_check(self) -> float:
        v = C.c_double(0)
        L.check(self.lib.verb_tensor_check(self.h, C.byref(v)), "tensor check")
        return v.value

    def maxabs(self, names) -> dict:
        """max |field| of each named field in one pass (the reference's per-step
        log of VP, VR, DLL, DVV, DVK, DKK; NaN values skipped)."""
        ids = (C.c_int * len(names))(*[L.FIELD_IDS[n] for n in names])
        out = np.zeros(len(names))
        L.check(self.lib.verb_field_maxabs(self.h, len(names), ids, out.ctypes.data_as(L._dp)),
                "maxabs")
        return dict(zip(names, out.tolist()))

    def status(self) -> int:
        """The device-side status word after waiting for the stream (0: OK)."""
        return int(self.lib.verb_sync(self.h))

    def sync(self) -> None:
        L.check(self.lib.verb_sync(self.h), "device status")

    # ---------------------------------------------------------------- outputs
    def download(self, name: str = "psd") -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        L.check(self.lib.verb_download_field(self.h, L.FIELD_IDS[name],
                                             out.ctypes.data_as(L._dp)), f"download {name}")
        return out

    def convection_substeps(self) -> np.ndarray:
        out = np.zeros(self.shape[2] * self.shape[3], dtype=np.int32)
        L.check(self.lib.verb_convection_substeps(self.h, out.ctypes.data_as(L._ip)), "substeps")
        return out.reshape(self.shape[2], self.shape[3])

    def local_pivots(self) -> np.ndarray:
        out = np.zeros(int(np.prod(self.shape)), dtype=np.int32)
        L.check(self.lib.verb_local_pivots(self.h, out.ctypes.data_as(L._i32p)), "pivots")
        P, R, V, K = self.shape
        return out.reshape(P, R, V * K)

    def local_factor_lapack(self, p: int, r: int):
        P, R, V, K = self.shape
        n = V * K
        ldab = 3 * (V + 1) + 1
        ab = np.zeros(ldab * n)
        ip = np.zeros(n, dtype=np.int64)
        L.check(self.lib.verb_local_factor_lapack(self.h, p, r, ab.ctypes.data_as(L._dp),
                                                  ip.ctypes.data_as(L._lp)), "factor")
        return ab, ip

    def set_timing(self, on: bool) -> None:
        L.check(self.lib.verb_set_timing(self.h, 1 if on else 0), "timing")

    def timing(self) -> dict:
        t = L.Timing()
        L.check(self.lib.verb_get_timing(self.h, C.byref(t)), "timing")
        return {n: getattr(t, n) for n, _ in L.Timing._fields_}

    def device_bytes(self) -> int:
        b = C.c_size_t(0)
        L.check(self.lib.verb_device_bytes(self.h, C.byref(b)), "bytes")
        return b.value

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.verb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hour_of_step(it: int, dt: float) -> int:
    """Hour index of time step `it` (time = it*dt days, it from 1 as in
    src/VERB4D_Solver.cpp:539-542)."""
    return int(math.floor(it * dt * 24.0 + 1e-9))


class Solver:
    """Runs a Workload on the GPU, one operator-split step per call."""

    def __init__(self, wl: Workload, stream: int | None = None, velocity_provider=None):
        self.wl = wl
        P, R, V, K = wl.spec.shape
        self.ctx = Context(P, R, V, K, stream)
        self.velocity_provider = velocity_provider
        self.hour = None
        self.kp_varies = len(np.unique(wl.kp)) > 1

    def load(self) -> None:
        f = self.wl.fields
        c = self.ctx
        c.set_bc_types(self.wl.bc_types)
        fl = self.wl.flags
        c.set_options(fl["radial_sources"], fl["local_sources"], fl["include_boundary"],
                      fl["positive_psd"])
        for name in L.FIELD_IDS:
            if name == "DLL":
                c.upload("DLL", f["DLL_base"] if "DLL_base" in f else f["DLL"])
            elif name in f:
                c.upload(name, f[name])
        for name in L.BC_FIELDS:
            c.upload(name, f[name])
        if "DLL_base" in f:
            c.set_scale("DLL", self.wl.dll_scale(0))
        self.hour = 0

    def reset_psd(self, psd=None) -> None:
        self.ctx.upload("psd", self.wl.fields["psd"] if psd is None else psd)

    def update_inputs(self, it: int) -> None:
        """UpdatableMatrix::update() for the hourly series (src/UpdatableMatrix.cpp:602-846)."""
        h = min(hour_of_step(it, self.wl.dt), len(self.wl.kp) - 1)
        if h == self.hour or not self.kp_varies:
            self.hour = h
            return
        self.hour = h
        self.ctx.set_scale("DLL", self.wl.dll_scale(h))
        if self.velocity_provider is not None:
            VP, VR = self.velocity_provider(h)
        else:
            VP, VR = drift_velocities(self.wl.spec, float(self.wl.kp[h]))
        self.ctx.upload("VP", VP)
        self.ctx.upload("VR", VR)

    def step(self, it: int, count_negatives=False):
        self.update_inputs(it)
        fl = self.wl.flags
        return self.ctx.step(self.wl.dt, self.wl.sub_dt, fl["run_convection"], fl["run_radial"],
                             fl["run_local"], count_negatives)

    def run(self, steps: int, first: int = 1):
        neg = None
        for it in range(first, first + steps):
            neg = self.step(it, count_negatives=(it == first + steps - 1))
        self.ctx.sync()
        return neg
