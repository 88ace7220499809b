"""ctypes front end for the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads the C restatement (oracle/liboracle.so) and, when built, the reference's
own routines compiled from source (oracle/_ref/libverbref*.so).  Only tests/,
the smoke check and bench.py's CPU-baseline / reference legs use this module;
the product path never imports it.

Both libraries expose the same per-slice calling convention (plain row-major
float64 arrays, boundary-condition codes 0 Periodic / 1 ConstantValue /
2 ConstantDerivative, src/BoundaryConditionType.hpp:53-88), so the same Python
wrappers drive either one.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libverbref.so")
REF_LU_SO = os.path.join(HERE, "_ref", "libverbref_lu.so")
# the C++ drop-in layer (reference signatures over the CUDA library) with the
# same harness entry points under a drop_ prefix
DROPIN_SO = os.path.join(HERE, "_ref", "libverbdropin.so")

BC_PERIODIC, BC_VALUE, BC_DERIV = 0, 1, 2

_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_long)
_ip = C.POINTER(C.c_int)


def build(with_ref: bool | None = None) -> None:
    """Compile the restatement, and the reference libraries when the reference tree exists."""
    # the reference tree: $VERB_REFERENCE, else a checkout named `reference`
    # beside this repository
    ref_dir = os.environ.get("VERB_REFERENCE",
                             os.path.abspath(os.path.join(HERE, "..", "..", "reference")))
    if with_ref is None:
        with_ref = os.path.isdir(os.path.join(ref_dir, "src"))
    target = "ref" if with_ref else "all"
    subprocess.run(["make", "-s", "-C", HERE, target, f"REF={ref_dir}"], check=True)


def _p(a):
    return a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _Renamed:
    """A loaded library whose entry points named prefix_<x> answer to ref_<x>."""

    def __init__(self, lib, prefix: str):
        self._lib = lib
        self._prefix = prefix

    def __getattr__(self, name: str):
        if name.startswith("ref_"):
            name = self._prefix + name[4:]
        return getattr(self._lib, name)


class _Lib:
    def __init__(self, path: str, prefix: str | None = None):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        if prefix:
            self.lib = _Renamed(self.lib, prefix)
        self.path = path

    def has(self, name: str) -> bool:
        return hasattr(self.lib, name)

    # ------------------------------------------------------------------ radial
    def tridag(self, a, b, c, r):
        a, b, c, r = map(_f64, (a, b, c, r))
        u = np.zeros_like(r)
        fn = self.lib.orc_tridag if self.has("orc_tridag") else self.lib.ref_tridag
        fn(_p(a), _p(b), _p(c), _p(r), _p(u), C.c_long(len(r)))
        return u

    def radial_matrix(self, x, lbc, ubc, lbc_t, ubc_t, D, G, S, loss, dt):
        x, D, G, S, loss = map(_f64, (x, D, G, S, loss))
        n = len(x)
        out = [np.zeros(n) for _ in range(5)]
        fn = self.lib.orc_radial_matrix if self.has("orc_radial_matrix") else self.lib.ref_radial_matrix
        st = fn(_p(x), C.c_int(n), C.c_double(lbc), C.c_double(ubc), C.c_int(lbc_t), C.c_int(ubc_t),
                _p(D), _p(G), _p(S), _p(loss), C.c_double(dt), *[_p(o) for o in out])
        return st, out

    def diffusion_1d(self, psd, x, lbc, ubc, lbc_t, ubc_t, D, G, S, loss, dt):
        f = _f64(psd).copy()
        x, D, G, S, loss = map(_f64, (x, D, G, S, loss))
        fn = self.lib.orc_diffusion_1d if self.has("orc_diffusion_1d") else self.lib.ref_diffusion_1d
        st = fn(_p(f), _p(x), C.c_int(len(f)), C.c_double(lbc), C.c_double(ubc), C.c_int(lbc_t),
                C.c_int(ubc_t), _p(D), _p(G), _p(S), _p(loss), C.c_double(dt))
        return st, f

    # ------------------------------------------------------------------ local
    def diffusion_2d(self, psd, x, y, xl, xu, yl, yu, types, Dxx, Dyy, Dxy, Dyx, G, S, loss, dt,
                     sub_dt, lu=None, ipiv=None, recompute=True):
        """psd, x, y, D*, G, S, loss are [nx][ny]; xl/xu have ny entries, yl/yu nx.

        With lu/ipiv given the LU_CACHING form is used (ldab*n doubles, n longs)."""
        f = _f64(psd).copy()
        nx, ny = f.shape
        args = [_f64(a) for a in (x, y, xl, xu, yl, yu)]
        coeffs = [_f64(a) for a in (Dxx, Dyy, Dxy, Dyx, G, S, loss)]
        head = [_p(f), _p(args[0]), _p(args[1]), C.c_int(nx), C.c_int(ny)] + [_p(a) for a in args[2:]]
        head += [C.c_int(t) for t in types] + [_p(a) for a in coeffs]
        head += [C.c_double(dt), C.c_double(sub_dt)]
        if self.has("orc_diffusion_2d"):
            n = nx * ny
            ldab = 3 * (nx + 1) + 1
            own = lu is None
            if own:
                lu = np.zeros(ldab * n)
                ipiv = np.zeros(n, dtype=np.int64)
            st = self.lib.orc_diffusion_2d(*head, _p(lu), ipiv.ctypes.data_as(_lp),
                                           C.c_int(1 if (recompute or own) else 0))
        elif lu is not None:
            st = self.lib.ref_diffusion_2d_lu(*head, _p(lu), ipiv.ctypes.data_as(_lp),
                                              C.c_int(1 if recompute else 0))
        else:
            st = self.lib.ref_diffusion_2d(*head)
        return st, f

    # ------------------------------------------------------------- convection
    def convection_1d(self, psd, x, lbc, ubc, lbc_t, ubc_t, ux, dt):
        f = _f64(psd).copy()
        x, ux = _f64(x), _f64(ux)
        fn = self.lib.orc_convection_1d if self.has("orc_convection_1d") else self.lib.ref_convection_1d
        st = fn(_p(f), _p(x), C.c_int(len(f)), C.c_double(lbc), C.c_double(ubc), C.c_int(lbc_t),
                C.c_int(ubc_t), _p(ux), C.c_double(dt))
        return st, f

    def convection_2d(self, psd, P, R, pl, pu, rl, ru, types, VP, VR, S, loss, G, dt):
        f = _f64(psd).copy()
        nP, nR = f.shape
        arrs = [_f64(a) for a in (P, R, pl, pu, rl, ru)]
        co = [_f64(a) for a in (VP, VR, S, loss, G)]
        head = [_p(f), _p(arrs[0]), _p(arrs[1]), C.c_int(nP), C.c_int(nR)] + [_p(a) for a in arrs[2:]]
        head += [C.c_int(t) for t in types] + [_p(a) for a in co] + [C.c_double(dt)]
        if self.has("orc_convection_2d"):
            ns = C.c_int(0)
            st = self.lib.orc_convection_2d(*head, C.byref(ns))
            return st, f, ns.value
        st = self.lib.ref_convection_2d(*head)
        return st, f, None

    # --------------------------------------------------------------------- KF
    def kf_diffusion_1d(self, forecast, Pa, R, DLL, G, lbc, ubc, lbc_t, ubc_t, obs, dt, model_error,
                        obs_error):
        n = len(forecast)
        f = _f64(forecast).copy()
        pa = _f64(Pa).copy()
        F = np.zeros((n, n))
        Pf = np.zeros((n, n))
        R, DLL, G, obs = map(_f64, (R, DLL, G, obs))
        fn = self.lib.orc_kf_diffusion_1d if self.has("orc_kf_diffusion_1d") else self.lib.ref_kf_diffusion_1d
        st = fn(_p(f), _p(pa), _p(F), _p(Pf), _p(R), _p(DLL), _p(G), C.c_int(n), C.c_double(lbc),
                C.c_double(ubc), C.c_int(lbc_t), C.c_int(ubc_t), _p(obs), C.c_double(dt),
                C.c_double(model_error), C.c_double(obs_error))
        return st, f, pa, F, Pf

    def kf_convection_2d(self, forecast, Pa, model, Pg, Rg, VP, VR, has_vx_updated, loss, sat,
                         obs, dt, model_error, obs_error, use_log=False,
                         correlation_time=float("inf"), growing_q=False):
        """runKalmanFilterConvection2D of the reference build (oracle/_ref) on
        one [P][R] slice; returns (status, forecast, Pa, model, Pf)."""
        f = _f64(forecast).copy()
        nP, nR = f.shape
        N = nP * nR
        pa = _f64(Pa).copy()
        mm = np.zeros((N, N)) if model is None else _f64(model).copy()
        Pf = np.zeros((N, N))
        sat_b = None if sat is None else np.ascontiguousarray(sat, dtype=np.uint8)
        st = self.lib.ref_kf_convection_2d(
            _p(f), _p(pa), _p(mm), C.c_int(model is not None), _p(Pf), _p(_f64(Pg)), _p(_f64(Rg)),
            _p(_f64(VP)), _p(_f64(VR)), C.c_int(int(has_vx_updated)), _p(_f64(loss)),
            sat_b.ctypes.data_as(C.POINTER(C.c_ubyte)) if sat_b is not None else None,
            _p(_f64(obs)), C.c_int(nP), C.c_int(nR), C.c_double(dt), C.c_double(model_error),
            C.c_double(obs_error), C.c_int(int(use_log)), C.c_double(correlation_time),
            C.c_int(int(growing_q)))
        return st, f, pa, mm, Pf

    # ------------------------------------------------------------- band LU
    def monot_cubic(self, x, f, xq):
        """Monotone cubic interpolation: orc_monot_cubic in the oracle,
        ref_monot_cubic (Opm::MonotCubicInterpolator) in the reference build."""
        x, f, xq = _f64(x), _f64(f), _f64(xq)
        out = np.zeros(len(xq))
        fn = self.lib.orc_monot_cubic if self.has("orc_monot_cubic") else self.lib.ref_monot_cubic
        st = fn(_p(x), _p(f), C.c_int(len(x)), _p(xq), _p(out), C.c_int(len(xq)))
        return st, out

    def write_pltb(self, path, arr):
        """Reference writer (Matrix4D::writeToBinaryFile) through oracle/_ref."""
        a = _f64(arr)
        w, x, y, z = a.shape
        return self.lib.ref_write_pltb(_p(a), C.c_int(w), C.c_int(x), C.c_int(y), C.c_int(z),
                                       str(path).encode())

    def read_pltb(self, path, shape):
        out = np.zeros(shape)
        w, x, y, z = shape
        self.lib.ref_read_pltb(_p(out), C.c_int(w), C.c_int(x), C.c_int(y), C.c_int(z),
                               str(path).encode())
        return out

    def gbtrf(self, ab, n, kl, ku):
        ab = _f64(ab).copy()
        ipiv = np.zeros(n, dtype=np.int64)
        self.lib.orc_gbtrf.restype = C.c_long
        info = self.lib.orc_gbtrf(C.c_long(n), C.c_long(kl), C.c_long(ku), _p(ab),
                                  C.c_long(2 * kl + ku + 1), ipiv.ctypes.data_as(_lp))
        return info, ab, ipiv

    def gbtrs(self, ab, ipiv, b, n, kl, ku):
        x = _f64(b).copy()
        ab = _f64(ab)
        ipiv = np.ascontiguousarray(ipiv, dtype=np.int64)
        self.lib.orc_gbtrs(C.c_long(n), C.c_long(kl), C.c_long(ku), _p(ab),
                           C.c_long(2 * kl + ku + 1), ipiv.ctypes.data_as(_lp), _p(x))
        return x

    def local_matrix(self, x, y, xl, xu, yl, yu, types, Dxx, Dyy, Dxy, Dyx, G, S, loss, dt):
        nx, ny = np.shape(x)
        n = nx * ny
        diag = np.zeros(9 * n)
        bd = np.zeros(n)
        cd = np.zeros(n)
        arrs = [_f64(a) for a in (x, y, xl, xu, yl, yu)]
        co = [_f64(a) for a in (Dxx, Dyy, Dxy, Dyx, G, S, loss)]
        st = self.lib.orc_local_matrix(_p(arrs[0]), _p(arrs[1]), C.c_int(nx), C.c_int(ny),
                                       *[_p(a) for a in arrs[2:]], *[C.c_int(t) for t in types],
                                       *[_p(a) for a in co], C.c_double(dt), _p(diag), _p(bd), _p(cd))
        return st, diag.reshape(9, n), bd, cd


class OrcState(C.Structure):
    _fields_ = ([("P", C.c_int), ("R", C.c_int), ("V", C.c_int), ("K", C.c_int), ("psd", _dp)]
                + [(n, _dp) for n in ("Pg", "Rg", "Vg", "Kg", "Lg", "DLL", "DVV", "DKK", "DVK", "VP",
                                      "VR", "G_local", "G_radial", "G_conv", "S", "loss_local",
                                      "loss_radial", "loss_conv", "Pl", "Pu", "Rl", "Ru", "Ll", "Lu",
                                      "Vl", "Vu", "Kl", "Ku")]
                + [(n, C.c_int) for n in ("Pl_t", "Pu_t", "Rl_t", "Ru_t", "Ll_t", "Lu_t", "Vl_t", "Vu_t",
                                          "Kl_t", "Ku_t", "run_convection", "run_radial", "run_local",
                                          "radial_sources", "local_sources", "include_boundary",
                                          "positive_psd")]
                + [("lu", _dp), ("ipiv", _lp)])


class OracleStepper:
    """Whole-step oracle (orc_step) over a dict of 4-D fields; keeps its own LU cache."""

    FIELDS = ("Pg", "Rg", "Vg", "Kg", "Lg", "DLL", "DVV", "DKK", "DVK", "VP", "VR", "G_local",
              "G_radial", "G_conv", "S", "loss_local", "loss_radial", "loss_conv", "Pl", "Pu", "Rl",
              "Ru", "Ll", "Lu", "Vl", "Vu", "Kl", "Ku")

    def __init__(self, inputs: dict, lib: "_Lib | None" = None, lu_cache: bool = True):
        self.lib = lib or oracle()
        self.keep = {k: _f64(inputs[k]) for k in self.FIELDS}
        self.psd = _f64(inputs["psd"]).copy()
        P, R, V, K = self.psd.shape
        st = OrcState()
        st.P, st.R, st.V, st.K = P, R, V, K
        st.psd = _p(self.psd)
        for k in self.FIELDS:
            setattr(st, k, _p(self.keep[k]))
        for k in ("Pl_t", "Pu_t", "Rl_t", "Ru_t", "Ll_t", "Lu_t", "Vl_t", "Vu_t", "Kl_t", "Ku_t"):
            setattr(st, k, int(inputs["bc_types"][k[:-2]]))
        flags = inputs.get("flags", {})
        st.run_convection = int(flags.get("run_convection", 1))
        st.run_radial = int(flags.get("run_radial", 1))
        st.run_local = int(flags.get("run_local", 1))
        st.radial_sources = int(flags.get("radial_sources", 0))
        st.local_sources = int(flags.get("local_sources", 1))
        st.include_boundary = int(flags.get("include_boundary", 1))
        st.positive_psd = int(flags.get("positive_psd", 0))
        n = V * K
        ldab = 3 * (V + 1) + 1
        if lu_cache:
            self.lu = np.zeros(P * R * ldab * n)
            self.ipiv = np.zeros(P * R * n, dtype=np.int64)
            st.lu = _p(self.lu)
            st.ipiv = self.ipiv.ctypes.data_as(_lp)
        self.st = st
        if self.lib.has("orc_step"):
            self.lib.lib.orc_step.restype = C.c_long

    def step(self, dt: float, sub_dt: float, recompute_lu: bool) -> int:
        return int(self.lib.lib.orc_step(C.byref(self.st), C.c_double(dt), C.c_double(sub_dt),
                                         C.c_int(1 if recompute_lu else 0)))


_cache: dict = {}


def oracle() -> _Lib:
    if "o" not in _cache:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        _cache["o"] = _Lib(ORACLE_SO)
    return _cache["o"]


def reference(lu_caching: bool = False) -> _Lib:
    path = REF_LU_SO if lu_caching else REF_SO
    if path not in _cache:
        _cache[path] = _Lib(path)
    return _cache[path]


def dropin() -> _Lib:
    """The C++ drop-in layer built against the reference's headers
    (oracle/_ref/libverbdropin.so): the same per-slice entry points as
    reference(), running on the GPU through libverb4d_b200.so."""
    if DROPIN_SO not in _cache:
        _cache[DROPIN_SO] = _Lib(DROPIN_SO, prefix="drop_")
    return _cache[DROPIN_SO]


def have_reference() -> bool:
    return os.path.exists(REF_SO) and os.path.exists(REF_LU_SO)
