"""Error paths of the step, each made on the host and reported as a status
code; none of them faults, traps or hangs the GPU.

The reference ends the run with exit(EXIT_FAILURE) or an exception at each of
these points: the diffusion-tensor check (src/VERB4D_Solver.cpp:747-753), a
zero pivot in LAPACK's banded LU (src/MatrixSolver.cpp:273-276) and a NaN
after the Kalman update (src/DataAssimilation.cpp:62-67).  The library
returns VERB_ERR_TENSOR from verb_step, and records VERB_ERR_PIVOT and
VERB_ERR_NAN in the device status word that verb_sync returns.  A NaN
coefficient has no check in the reference (the NaN spreads through the PSD);
here the negative-count pass of every step flags a NaN in the PSD."""
import numpy as np
import pytest

from verb4d_b200 import Context
from verb4d_b200 import _lib as L
from verb4d_b200 import workload as W

pytestmark = pytest.mark.gpu

ERR_PIVOT, ERR_TENSOR, ERR_NAN = 1, 5, 6
SPEC = W.GridSpec(12, 13, 11, 12)


def context_for(wl):
    ctx = Context(*wl.spec.shape)
    ctx.set_bc_types(wl.bc_types)
    fl = wl.flags
    ctx.set_options(fl["radial_sources"], fl["local_sources"], fl["include_boundary"],
                    fl["positive_psd"])
    for k in ("psd", "Pg", "Rg", "Vg", "Kg", "Lg", "DLL", "DVV", "DKK", "DVK", "VP", "VR",
              "G_local", "G_radial", "G_conv", "S", "loss_local", "loss_radial", "loss_conv",
              "Pl", "Pu", "Rl", "Ru", "Ll", "Lu", "Vl", "Vu", "Kl", "Ku"):
        ctx.upload(k, wl.fields[k])
    return ctx


def test_tensor_check_failure_returns_status_and_leaves_psd(gpu):
    wl = W.make_workload(SPEC, seed=21)
    f = wl.fields
    p, r, v, k = 3, 5, 4, 6
    f["DVK"][p, r, v, k] = 1.01 * np.sqrt(f["DVV"][p, r, v, k] * f["DKK"][p, r, v, k])
    ctx = context_for(wl)
    assert ctx.tensor_check() < 0
    st = ctx.lib.verb_step(ctx.h, wl.dt, wl.sub_dt, 1, 1, 1, None)
    assert st == ERR_TENSOR
    assert np.array_equal(ctx.download(), f["psd"])  # nothing ran
    assert ctx.status() == 0
    ctx.close()


def test_exactly_zero_pivot_is_reported(gpu):
    """No local diffusion and a loss rate equal to 1/dt at one interior point:
    that unknown's column of the banded matrix is exactly zero."""
    wl = W.make_workload(SPEC, seed=22)
    f = wl.fields
    for key in ("DVV", "DKK", "DVK"):
        f[key] = np.zeros_like(f[key])
    f["loss_local"] = np.zeros_like(f["loss_local"])
    f["loss_local"][2, 6, 5, 6] = 1.0 / wl.dt
    ctx = context_for(wl)
    assert ctx.lib.verb_step(ctx.h, wl.dt, wl.dt, 0, 0, 1, None) == 0
    assert ctx.status() == ERR_PIVOT
    ctx.close()


def test_nan_coefficient_is_reported(gpu, oracle_lib):
    """The banded LU takes a NaN pivot where LAPACK's idamax does (a NaN first
    entry of the column) and otherwise skips NaN entries, so whether the step
    meets an exactly zero pivot or runs on and fills the PSD with NaN is the
    reference's own outcome (the oracle restates dgbtf2 and reports it)."""
    import oracle as O

    wl = W.make_workload(SPEC, seed=23)
    wl.fields["DVV"][4, 7, 5, 5] = np.nan
    ctx = context_for(wl)
    # the reference's tensor check skips NaN values (std::min), so the step runs
    assert np.isfinite(ctx.tensor_check())
    assert ctx.lib.verb_step(ctx.h, wl.dt, wl.sub_dt, 1, 1, 1, None) == 0
    ref = O.OracleStepper(W.oracle_inputs(wl), oracle_lib).step(wl.dt, wl.sub_dt, True)
    if ref == -ERR_PIVOT:
        assert ctx.status() == ERR_PIVOT
    else:
        assert ctx.status() == ERR_NAN
        assert np.isnan(ctx.download()[4, 7]).any()
    ctx.close()


def test_nan_after_kalman_update_matches_reference(gpu, oracle_lib):
    """A NaN in the forecast of one observed column and of one unobserved
    column: the reference throws for both (DataAssimilation.cpp:62-67, the
    dummy observation row keeps the NaN); the GPU update reports VERB_ERR_NAN."""
    import oracle as O

    try:
        ref = O.reference()
    except FileNotFoundError:
        ref = oracle_lib
    spec = W.GridSpec(1, 25, 2, 2)
    wl = W.make_workload(spec, seed=24)
    f = wl.fields
    obs = np.full(spec.shape, np.nan)
    obs[0, 8, 0, 0] = f["psd"][0, 8, 0, 0] * 1.05
    for (v, k) in ((0, 0), (1, 1)):
        psd = f["psd"].copy()
        psd[0, 12, v, k] = np.nan
        ln = lambda a: a[0, :, v, k]  # noqa: E731
        st, *_ = ref.kf_diffusion_1d(ln(psd), np.zeros((25, 25)), ln(f["Rg"]), ln(f["DLL"]),
                                     ln(f["G_radial"]), float(f["Ll"][0, v, k]),
                                     float(f["Lu"][0, v, k]), 1, 1, ln(obs), wl.dt, 1e-4, 1e-3)
        assert st == 2  # the reference's NaN exception
        ctx = Context(*spec.shape)
        ctx.set_bc_types(wl.bc_types)
        for key in ("Rg", "DLL", "G_radial", "Ll", "Lu"):
            ctx.upload(key, f[key])
        ctx.upload("psd", psd)
        ctx.assimilate_radial(obs, wl.dt, 1e-4, 1e-3, p_index=0)
        assert ctx.status() == ERR_NAN, (v, k)
        ctx.close()


def test_field_maxabs_matches_the_reference_definition(gpu):
    """One fused pass over VP, VR, DLL (scaled), DVV, DVK, DKK; NaN skipped as
    Matrix4D::maxabs skips it."""
    wl = W.make_workload(SPEC, seed=25)
    f = wl.fields
    f["DVK"][1, 2, 3, 4] = np.nan
    ctx = context_for(wl)
    ctx.set_scale("DLL", 3.5)
    names = ["VP", "VR", "DLL", "DVV", "DVK", "DKK"]
    got = ctx.maxabs(names)
    for n in names:
        want = np.nanmax(np.abs(f[n] * (3.5 if n == "DLL" else 1.0)))
        assert got[n] == want, n
    with pytest.raises(L.VerbError):
        ctx.maxabs(["VP"] * 9)
    ctx.close()
