"""Synthetic workload generator: shapes, physical ranges and the checks the
reference applies to its inputs."""
import numpy as np

from verb4d_b200 import workload as W


def test_shapes_and_layout():
    spec = W.GridSpec(8, 9, 7, 6)
    wl = W.make_workload(spec, seed=2)
    f = wl.fields
    for k in ("psd", "Pg", "Rg", "Vg", "Kg", "Lg", "DLL", "DVV", "DKK", "DVK", "VP", "VR"):
        assert f[k].shape == spec.shape and f[k].flags.c_contiguous
    assert f["Rl"].shape == (8, 7, 6) and f["Vl"].shape == (8, 9, 6) and f["Kl"].shape == (8, 9, 7)
    # K fastest: the pitch-angle grid varies along the last axis
    assert np.all(np.diff(f["Kg"][0, 0, 0]) > 0)
    # periodic MLT: endpoint duplicated
    assert f["Pg"][0, 0, 0, 0] == 0.0 and f["Pg"][-1, 0, 0, 0] == 24.0


def test_diffusion_tensor_check_passes():
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=1)
    f = wl.fields
    assert (f["DVV"] * f["DKK"] - f["DVK"] * f["DVK"]).min() >= 0  # src/VERB4D_Solver.cpp:747-753


def test_brautigam_albert_range():
    L = np.array([1.0, 6.6])
    d = W.dll_brautigam_albert(L, 3.0)
    assert 1.5e-8 < d[0] < 1.7e-8 and 2.3 < d[1] < 2.6


def test_seeded_and_deterministic():
    a = W.make_workload(W.GridSpec(6, 7, 5, 5), seed=9).fields["DVV"]
    b = W.make_workload(W.GridSpec(6, 7, 5, 5), seed=9).fields["DVV"]
    c = W.make_workload(W.GridSpec(6, 7, 5, 5), seed=10).fields["DVV"]
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_convection_substeps_cfg1():
    ns = W.convection_substeps(W.make_workload(W.CONFIGS["cfg1"], seed=1))
    # gradient-curvature drift of 10 MeV electrons at L = 6.6 needs hundreds of
    # CFL sub-steps per 5-minute step; the lowest energies need a few
    assert ns.max() > 300 and ns.min() >= 1
    assert np.all(np.diff(ns[:, -1]) >= 0)  # monotone in energy


def test_kp_series():
    k = W.kp_series(3, 24)
    assert k.shape == (24,) and k.min() >= 1 and k.max() <= 6


def test_loss_cone_rows():
    wl = W.make_workload(W.CONFIGS["cfg1"], seed=41)
    k0 = W.loss_cone_k0(wl)
    K = wl.spec.K
    kept = K - k0[0]
    assert kept[0] == 0                       # L = 1: everything in the loss cone
    assert kept[-1] >= K - 1                  # L = 6.6: alpha_lc ~ 0.4 deg
    assert np.all(np.diff(kept) >= 0)
    assert abs(W.loss_cone_deg(2.0) - 8.08) < 0.01


def test_smooth_coefficients_option():
    spec = W.CONFIGS["cfg1"]
    a = W.make_workload(spec, seed=5)
    b = W.make_workload(spec, seed=5, coeff_corr=0.0)
    for k in ("DVV", "DKK", "DVK", "psd"):
        assert np.array_equal(a.fields[k], b.fields[k])
    c = W.make_workload(spec, seed=5, coeff_corr=4.0)
    z = np.log10(c.fields["DVV"] / (1e-5 * 86400.0))
    # unit variance per (MLT, L) slice, and far smoother along alpha than i.i.d. draws
    assert np.allclose(z.std(axis=(2, 3)), 1.0, atol=1e-6)
    rough = np.abs(np.diff(np.log10(a.fields["DVV"]), axis=3)).mean()
    smooth = np.abs(np.diff(z, axis=3)).mean()
    assert smooth < 0.3 * rough
    r = c.fields["DVK"] / np.sqrt(c.fields["DVV"] * c.fields["DKK"])
    assert np.all(np.abs(r) <= 0.99)
