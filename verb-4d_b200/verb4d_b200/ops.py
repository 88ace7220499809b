"""Per-slice operators with the reference's Python operator interface.

The reference exposes its slice routines through the pybind11 module
``verb4d_solver`` (src/python_bindings/Define_python_modules.cpp:17-33):
``Convection_1D``, ``Convection_2D`` and ``Diffusion_2D`` take numpy arrays in
the argument order of the C++ routines and return the updated PSD (the
``const_reference_wrapper`` of src/python_bindings/const_reference_wrapper.h:9-15
returns a copy of the mutated first argument).  The functions below keep those
names, argument orders and return conventions, and add ``Diffusion_1D`` and
``tridag``, which the reference does not bind.  Every call runs on the GPU
through the C ABI; errors that make the reference exit raise ``VerbError``.
"""
from __future__ import annotations

import enum

import numpy as np

from . import _lib as L


class BoundaryConditionType(enum.IntEnum):
    """src/BoundaryConditionType.hpp:53-88."""
    Periodic = 0
    ConstantValue = 1
    ConstantDerivative = 2


Periodic = BoundaryConditionType.Periodic
ConstantValue = BoundaryConditionType.ConstantValue
ConstantDerivative = BoundaryConditionType.ConstantDerivative


def _d(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape)
    return a


def _p(a):
    return a.ctypes.data_as(L._dp)


def tridag(a, b, c, r):
    """Thomas solve of diag(a,b,c) u = r (src/MatrixSolver.cpp:689-720)."""
    a, b, c, r = map(_d, (a, b, c, r))
    u = np.zeros_like(r)
    L.check(L.load().verb_tridag(_p(a), _p(b), _p(c), _p(r), _p(u), len(r)), "tridag")
    return u


def Diffusion_1D(psd, x, x_size, x_LBC, x_UBC, x_LBC_type, x_UBC_type, Dxx, G, Sources, Losses, dt):
    """src/Diffusion_1D.cpp:43-88; returns the updated PSD line."""
    f = _d(psd).copy()
    n = int(x_size)
    args = [_d(a) for a in (x, Dxx, G, Sources, Losses)]
    st = L.load().verb_diffusion_1d(_p(f), _p(args[0]), n, float(x_LBC), float(x_UBC),
                                    int(x_LBC_type), int(x_UBC_type), _p(args[1]), _p(args[2]),
                                    _p(args[3]), _p(args[4]), float(dt))
    L.check(st, "Diffusion_1D")
    return f


def Diffusion_2D(psd, x, y, x_size, y_size, x_LBC, x_UBC, y_LBC, y_UBC, x_LBC_type, x_UBC_type,
                 y_LBC_type, y_UBC_type, Dxx, Dyy, Dxy, Dyx, G, Sources, Losses, dt, sub_dt,
                 lu_cache=None, index_cache=None, recompute_lu=True):
    """src/Diffusion_2D.cpp:19-153 on one [x_size][y_size] slice; returns the PSD.

    ``lu_cache`` (float64, (2kl+ku+1)*n, LAPACK band layout) and
    ``index_cache`` (int64, n, 1-based) are the optional LU_CACHING slot."""
    nx, ny = int(x_size), int(y_size)
    f = _d(psd, (nx, ny)).copy()
    g2 = [_d(a, (nx, ny)) for a in (x, y, Dxx, Dyy, Dxy, Dyx, G, Sources, Losses)]
    b1 = [_d(a) for a in (x_LBC, x_UBC, y_LBC, y_UBC)]
    lu_p = _p(lu_cache) if lu_cache is not None else None
    ip_p = index_cache.ctypes.data_as(L._lp) if index_cache is not None else None
    st = L.load().verb_diffusion_2d(
        _p(f), _p(g2[0]), _p(g2[1]), nx, ny, *[_p(b) for b in b1], int(x_LBC_type),
        int(x_UBC_type), int(y_LBC_type), int(y_UBC_type), *[_p(a) for a in g2[2:]], float(dt),
        float(sub_dt), lu_p, ip_p, 1 if recompute_lu else 0)
    L.check(st, "Diffusion_2D")
    return f


def Convection_1D(PSD, x, x_size, x_LBC, x_UBC, x_LBC_type, x_UBC_type, Ux, dt_total):
    """src/Convection_1D_ULTIMATE_QUICKEST6.cpp:22-482; returns the PSD line."""
    f = _d(PSD).copy()
    x, Ux = _d(x), _d(Ux)
    st = L.load().verb_convection_1d(_p(f), _p(x), int(x_size), float(x_LBC), float(x_UBC),
                                     int(x_LBC_type), int(x_UBC_type), _p(Ux), float(dt_total))
    L.check(st, "Convection_1D")
    return f


def Convection_2D(PSD_PR, P, R, P_size, R_size, P_LBC, P_UBC, R_LBC, R_UBC, P_LBC_type, P_UBC_type,
                  R_LBC_type, R_UBC_type, VP, VR, Sources, Losses, G_conv, dt_total):
    """src/Convection_2D.cpp:36-169 on one [P_size][R_size] slice; returns the PSD."""
    nP, nR = int(P_size), int(R_size)
    f = _d(PSD_PR, (nP, nR)).copy()
    g2 = [_d(a, (nP, nR)) for a in (P, R, VP, VR, Sources, Losses, G_conv)]
    b1 = [_d(a) for a in (P_LBC, P_UBC, R_LBC, R_UBC)]
    st = L.load().verb_convection_2d(
        _p(f), _p(g2[0]), _p(g2[1]), nP, nR, *[_p(b) for b in b1], int(P_LBC_type),
        int(P_UBC_type), int(R_LBC_type), int(R_UBC_type), *[_p(a) for a in g2[2:]],
        float(dt_total))
    L.check(st, "Convection_2D")
    return f
