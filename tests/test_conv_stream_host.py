"""The streaming convection algorithm (conv_stream.cuh), compiled for the host,
against the oracle's Convection_2D (src/Convection_2D.cpp:36-169).

The device kernel and this host build share the line pass itself (register
windows, lags, boundary rewrites, halo slots); tests/conv_stream_host.cpp
drives it over one slice the way convection_stream_kernel does.  Each slice is
held to the FP64 tolerance of the contracted kernels, 1e-12 relative
(norm-wise, and pointwise where |psd| is above 1e-6 of its maximum), with
equal sub-step counts: the small grid with sources and loss rates, every
boundary-type combination of the MLT and L lines, a production-shape slice
(48 x 101, two L segments) with its threads run in order and in reverse, the
same slice with every line whole, and L lines with their own CFL sub-cycles.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from verb4d_b200 import workload as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-12


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    out = tmp_path_factory.mktemp("cstream") / "libconvstreamhost.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared",
                    "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "verb-4d_b200", "csrc"),
                    os.path.join(ROOT, "tests", "conv_stream_host.cpp"), "-o", str(out)],
                   check=True)
    return C.CDLL(str(out))


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def run_host(lib, args, force_whole=0, order=0):
    psd, Pg, Rg, pl, pu, rl, ru, types, VP, VR, S, loss, G, dt = args
    f = np.ascontiguousarray(psd, dtype=np.float64).copy()
    nP, nR = f.shape
    arrs = [np.ascontiguousarray(a, dtype=np.float64)
            for a in (Pg, Rg, pl, pu, rl, ru, VP, VR, S, loss, G)]
    ns = C.c_int(0)
    lib.host_stream_convection_2d(
        _p(f), _p(arrs[0]), _p(arrs[1]), C.c_int(nP), C.c_int(nR), _p(arrs[2]), _p(arrs[3]),
        _p(arrs[4]), _p(arrs[5]), *[C.c_int(t) for t in types], _p(arrs[6]), _p(arrs[7]),
        _p(arrs[8]), _p(arrs[9]), _p(arrs[10]), C.c_double(dt), C.byref(ns), C.c_int(force_whole),
        C.c_int(order))
    return f, ns.value


def slice_args(wl, iV, iK, types):
    f = wl.fields
    sl = lambda a: np.ascontiguousarray(a[:, :, iV, iK])  # noqa: E731
    return (sl(f["psd"]), sl(f["Pg"]), sl(f["Rg"]), f["Pl"][:, iV, iK], f["Pu"][:, iV, iK],
            f["Rl"][:, iV, iK], f["Ru"][:, iV, iK], types, sl(f["VP"]), sl(f["VR"]), sl(f["S"]),
            sl(f["loss_conv"]), sl(f["G_conv"]), wl.dt)


def check(lib, oracle_lib, wl, slices, types=(0, 0, 1, 1), **kw):
    for iV, iK in slices:
        args = slice_args(wl, iV, iK, types)
        _, ref, n_ref = oracle_lib.convection_2d(*args)
        got, ns = run_host(lib, args, **kw)
        assert ns == n_ref
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= TOL * scale
        big = np.abs(ref) > 1e-6 * scale
        assert np.all(np.abs(got - ref)[big] <= TOL * np.abs(ref)[big])


def test_small_grid(host_lib, oracle_lib):
    wl = W.make_workload(W.GridSpec(14, 15, 12, 13), seed=31, sources=True, losses=True)
    wl.fields["VP"] = wl.fields["VP"] * 3e-3
    check(host_lib, oracle_lib, wl, [(11, 0), (5, 6), (0, 12)])


@pytest.mark.parametrize("types", [(0, 0, 1, 1), (0, 0, 2, 2), (0, 0, 1, 2), (0, 0, 2, 1),
                                   (1, 1, 1, 1), (2, 2, 2, 2), (1, 2, 2, 1), (0, 0, 0, 0)])
def test_boundary_types(host_lib, oracle_lib, types):
    wl = W.make_workload(W.GridSpec(14, 40, 5, 4), seed=44, sources=True, losses=True)
    rng = np.random.default_rng(3)
    wl.fields["Pl"] = rng.uniform(0.0, 0.5, wl.fields["Pl"].shape)
    wl.fields["Pu"] = rng.uniform(0.0, 0.5, wl.fields["Pu"].shape)
    if types[2] == 2:
        wl.fields["Rl"] = np.full(wl.fields["Rl"].shape, 0.05)
    if types[3] == 2:
        wl.fields["Ru"] = np.full(wl.fields["Ru"].shape, -0.03)
    check(host_lib, oracle_lib, wl, [(4, 0), (2, 3)], types=types)


def test_production_shape_thread_order(host_lib, oracle_lib):
    wl = W.make_workload(W.GridSpec(48, 101, 6, 5), seed=2)
    for order in (0, 1):
        check(host_lib, oracle_lib, wl, [(2, 3)], order=order)
    check(host_lib, oracle_lib, wl, [(2, 3)], force_whole=1)


def test_lines_with_own_subcycles(host_lib, oracle_lib):
    wl = W.make_workload(W.GridSpec(14, 40, 5, 4), seed=5, sources=True, losses=True)
    Rg = wl.fields["Rg"].copy()
    nP = Rg.shape[0]
    for iP in range(nP):
        fac = 1.0 / (1.0 + 7.0 * iP / (nP - 1))
        Rg[iP] = Rg[0, 0] + (Rg[0] - Rg[0, 0]) * fac
    wl.fields["Rg"] = Rg
    check(host_lib, oracle_lib, wl, [(3, 0), (1, 2)], types=(0, 0, 1, 2))
    check(host_lib, oracle_lib, wl, [(3, 0)], types=(0, 0, 0, 0))
