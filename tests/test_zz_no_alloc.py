"""The no-allocation entry point, verb_convection_2d_noalloc.

It serves callers that cannot allocate device memory (a host application or
plugin that owns every device allocation, or a path where allocating is not
allowed): they pass arrays already on the device and the kernel's scratch
comes from a fixed array the library reserves at load time.  This test calls
it through the C ABI on two different slices in a row (the shared scratch
keeps the previous call's contents) and compares each result with the
allocating entry point verb_convection_2d on the same inputs.  Both run the
same convection kernel, so the tolerance is the one the convection tests use
without loss rates: bit for bit.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from verb4d_b200 import _lib as L
from verb4d_b200 import ops
from verb4d_b200 import workload as W

pytestmark = pytest.mark.gpu


def slice_case(spec, seed, iV, iK, vp_scale):
    wl = W.make_workload(spec, seed=seed, sources=True)
    f = wl.fields
    sl = lambda a: np.ascontiguousarray(a[:, :, iV, iK])  # noqa: E731
    return dict(psd=sl(f["psd"]), P=sl(f["Pg"]), R=sl(f["Rg"]), pl=f["Pl"][:, iV, iK].copy(),
                pu=f["Pu"][:, iV, iK].copy(), rl=f["Rl"][:, iV, iK].copy(),
                ru=f["Ru"][:, iV, iK].copy(), VP=sl(f["VP"]) * vp_scale, VR=sl(f["VR"]),
                S=sl(f["S"]), loss=np.zeros_like(sl(f["psd"])), G=sl(f["G_conv"]), dt=wl.dt)


def run_noalloc(lib, c, torch, stream=None):
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.array(v)).to(dev) for k, v in c.items() if k != "dt"}
    torch.cuda.synchronize()
    nP, nR = c["psd"].shape
    p = lambda k: C.c_void_p(t[k].data_ptr())  # noqa: E731
    handle = C.c_void_p(stream.cuda_stream) if stream is not None else None
    st = lib.verb_convection_2d_noalloc(p("psd"), p("P"), p("R"), nP, nR, p("pl"), p("pu"), p("rl"),
                                        p("ru"), 0, 0, 1, 1, p("VP"), p("VR"), p("S"), p("loss"),
                                        p("G"), c["dt"], handle)
    torch.cuda.synchronize()
    return st, t["psd"].cpu().numpy()


def run_allocating(c):
    nP, nR = c["psd"].shape
    return ops.Convection_2D(c["psd"], c["P"], c["R"], nP, nR, c["pl"], c["pu"], c["rl"], c["ru"],
                             0, 0, 1, 1, c["VP"], c["VR"], c["S"], c["loss"], c["G"], c["dt"])


def test_noalloc_matches_allocating_entry_point_twice(gpu):
    import torch

    lib = L.load()
    cases = [slice_case(W.CONFIGS["cfg2"], 7, 100, 5, 1.0),   # 48 x 101, hundreds of sub-steps
             slice_case(W.CONFIGS["cfg1"], 8, 17, 30, 1.0)]    # 24 x 25 after the larger slice
    for c in cases:
        st, got = run_noalloc(lib, c, torch)
        assert st == L.VERB_OK
        want = run_allocating(c)
        assert np.array_equal(got, want)


def test_noalloc_rejects_oversized_slices(gpu):
    import torch

    lib = L.load()
    c = slice_case(W.GridSpec(100, 100, 1, 1), 9, 0, 0, 1e-3)  # 10000 > 8192 points
    st, got = run_noalloc(lib, c, torch)
    assert st == 11  # VERB_ERR_SIZE
    assert np.array_equal(got, c["psd"])  # nothing was touched


def test_noalloc_on_a_caller_stream(gpu):
    """The caller's own (non-default) stream: the same result bit for bit."""
    import torch

    lib = L.load()
    c = slice_case(W.CONFIGS["cfg1"], 11, 20, 12, 1.0)
    stream = torch.cuda.Stream()
    st, got = run_noalloc(lib, c, torch, stream)
    assert st == L.VERB_OK
    assert np.array_equal(got, run_allocating(c))


def test_noalloc_reports_a_courant_failure(gpu):
    """A duplicated MLT coordinate makes the grid spacing zero, so the
    sub-step count is infinite: the slice is skipped and VERB_ERR_CFL is
    returned (the reference exits, QUICKEST6.cpp:48-52)."""
    import torch

    lib = L.load()
    c = slice_case(W.CONFIGS["cfg1"], 12, 20, 12, 1.0)
    c["P"][1, :] = c["P"][0, :]
    st, got = run_noalloc(lib, c, torch)
    assert st == 3  # VERB_ERR_CFL
    assert np.array_equal(got, c["psd"])
