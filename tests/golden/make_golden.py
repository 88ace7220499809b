"""Generate the golden fixtures from the reference's own routines.

Runs the UNMODIFIED reference routines, compiled from source by oracle/Makefile
into oracle/_ref/libverbref*.so, on seeded inputs and stores inputs and
outputs here:

  slices.npz  per-slice cases: Diffusion_1D, tridag, Diffusion_2D (with the
              LAPACK factors and pivots of the LU_CACHING build),
              Convection_1D, Convection_2D, runKalmanFilterDiffusion1D
  step.npz    two whole operator-split steps on a 12x13x11x12 grid, driven in
              the phase order and with the slice extraction of
              src/VERB4D_Solver.cpp:851-1242, each slice solved by the
              reference routine; the inputs come from the seeded workload
              generator (seed and sizes stored with the outputs)

Usage:  python tests/golden/make_golden.py     (needs the reference tree)
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

STEP_SPEC = (12, 13, 11, 12)
STEP_SEED = 5
SLICE_SEED = 11


def step_workload():
    wl = W.make_workload(W.GridSpec(*STEP_SPEC), seed=STEP_SEED, sources=True, losses=True)
    # moderate drifts keep the sub-step counts of this small grid short
    wl.fields["VP"] = wl.fields["VP"] * 1e-2
    return wl


def ref_step(ref, ref_lu, wl, psd, lu, ipiv, recompute):
    """One step with the reference's per-slice routines (src/VERB4D_Solver.cpp:851-1242)."""
    f = wl.fields
    P, R, V, K = wl.spec.shape
    bt = wl.bc_types
    dt = wl.dt
    psd = psd.copy()
    for iV in range(V - 1, -1, -1):
        for iK in range(K):
            sl = lambda a: a[:, :, iV, iK]  # noqa: E731
            _, out, _ = ref.convection_2d(
                sl(psd), sl(f["Pg"]), sl(f["Rg"]), f["Pl"][:, iV, iK], f["Pu"][:, iV, iK],
                f["Rl"][:, iV, iK], f["Ru"][:, iV, iK], (bt["Pl"], bt["Pu"], bt["Rl"], bt["Ru"]),
                sl(f["VP"]), sl(f["VR"]), sl(f["S"]), sl(f["loss_conv"]), sl(f["G_conv"]), dt)
            psd[:, :, iV, iK] = out
    rs = float(wl.flags["radial_sources"])
    for iP in range(P):
        for iV in range(V):
            for iK in range(K):
                ln = lambda a: a[iP, :, iV, iK]  # noqa: E731
                _, out = ref.diffusion_1d(ln(psd), ln(f["Lg"]), f["Ll"][iP, iV, iK],
                                          f["Lu"][iP, iV, iK], bt["Ll"], bt["Lu"], ln(f["DLL"]),
                                          ln(f["G_radial"]), ln(f["S"]) * rs, ln(f["loss_radial"]),
                                          dt)
                psd[iP, :, iV, iK] = out
    ls = float(wl.flags["local_sources"])
    for iP in range(P):
        for iR in range(R):
            sl = lambda a: a[iP, iR]  # noqa: E731
            k = iP * R + iR
            _, out = ref_lu.diffusion_2d(
                sl(psd), sl(f["Vg"]), sl(f["Kg"]), f["Vl"][iP, iR], f["Vu"][iP, iR],
                f["Kl"][iP, iR], f["Ku"][iP, iR], (bt["Vl"], bt["Vu"], bt["Kl"], bt["Ku"]),
                sl(f["DVV"]), sl(f["DKK"]), sl(f["DVK"]), sl(f["DVK"]), sl(f["G_local"]),
                sl(f["S"]) * ls, sl(f["loss_local"]), dt, wl.sub_dt, lu=lu[k], ipiv=ipiv[k],
                recompute=recompute)
            psd[iP, iR] = out
    return psd, int((psd < 0).sum())


def main():
    if not O.have_reference():
        O.build(with_ref=True)
    ref = O.reference()
    ref_lu = O.reference(lu_caching=True)
    rng = np.random.default_rng(SLICE_SEED)
    out = {}

    # ---- radial lines and tridag
    spec = W.GridSpec(12, 25, 11, 12)
    wl = W.make_workload(spec, seed=SLICE_SEED, sources=True, losses=True)
    f = wl.fields
    for c, (lt, ut) in enumerate([(1, 1), (2, 1), (1, 2), (2, 2)]):
        iP, iV, iK = rng.integers(0, 12), rng.integers(0, 11), rng.integers(0, 12)
        ln = lambda a: a[iP, :, iV, iK]  # noqa: E731
        args = dict(x=ln(f["Lg"]), lbc=float(rng.uniform(0, 1e-3)), ubc=float(f["Lu"][iP, iV, iK]),
                    lbc_t=lt, ubc_t=ut, D=ln(f["DLL"]) * 1e3, G=ln(f["G_radial"]), S=ln(f["S"]),
                    loss=ln(f["loss_local"]), dt=wl.dt)
        psd = ln(f["psd"])
        _, res = ref.diffusion_1d(psd, **args)
        for k, v in args.items():
            out[f"d1_{c}_{k}"] = np.asarray(v)
        out[f"d1_{c}_psd"] = psd
        out[f"d1_{c}_out"] = res
    n = 40
    a, c_, r = rng.uniform(-1, 0, n), rng.uniform(-1, 0, n), rng.uniform(-1, 1, n)
    b = 2.5 + rng.uniform(0, 1, n)
    out.update(tri_a=a, tri_b=b, tri_c=c_, tri_r=r, tri_out=ref.tridag(a, b, c_, r))

    # ---- local slices (LU_CACHING build: factors and pivots too)
    spec = W.GridSpec(4, 5, 11, 12)
    wl = W.make_workload(spec, seed=SLICE_SEED + 1, sources=True, losses=True)
    f = wl.fields
    for c, types in enumerate([(1, 1, 2, 2), (1, 1, 1, 1), (2, 1, 2, 1)]):
        iP, iR = int(rng.integers(0, 4)), int(rng.integers(1, 4))
        sl = lambda a: a[iP, iR]  # noqa: E731
        n = 11 * 12
        ldab = 3 * 12 + 1
        lu = np.zeros(ldab * n)
        ip = np.zeros(n, dtype=np.int64)
        args = dict(x=sl(f["Vg"]), y=sl(f["Kg"]), xl=f["Vl"][iP, iR], xu=f["Vu"][iP, iR],
                    yl=f["Kl"][iP, iR] + 0.1 * (types[2] == 1), yu=f["Ku"][iP, iR],
                    Dxx=sl(f["DVV"]), Dyy=sl(f["DKK"]), Dxy=sl(f["DVK"]), Dyx=sl(f["DVK"]),
                    G=sl(f["G_local"]) * (1.0 + 0.1 * rng.uniform(size=(11, 12))), S=sl(f["S"]),
                    loss=sl(f["loss_local"]), dt=wl.dt, sub_dt=wl.dt / 2.5)
        psd = sl(f["psd"])
        _, res = ref_lu.diffusion_2d(psd, types=types, lu=lu, ipiv=ip, recompute=True, **args)
        for k, v in args.items():
            out[f"d2_{c}_{k}"] = np.asarray(v)
        out[f"d2_{c}_types"] = np.asarray(types)
        out[f"d2_{c}_psd"] = psd
        out[f"d2_{c}_out"] = res
        out[f"d2_{c}_lu"] = lu
        out[f"d2_{c}_ipiv"] = ip

    # ---- convection lines and slices
    n = 24
    x = np.linspace(0, 24, n)
    for c, (lt, ut, lb, ub) in enumerate([(0, 0, 0.0, 0.0), (1, 1, 0.3, 0.05), (2, 2, 0.01, -0.02),
                                          (1, 2, 0.2, 0.0)]):
        psd = np.exp(-((x - 9) / 3) ** 2) + 0.05 * rng.uniform(size=n)
        if lt == 0:
            psd[-1] = psd[0]
        ux = rng.uniform(-300, 500, n)
        _, res = ref.convection_1d(psd, x, lb, ub, lt, ut, ux, W.DT_5MIN)
        out.update({f"c1_{c}_psd": psd, f"c1_{c}_x": x, f"c1_{c}_ux": ux,
                    f"c1_{c}_bc": np.array([lb, ub, lt, ut], dtype=np.float64), f"c1_{c}_out": res})
    spec = W.GridSpec(12, 13, 6, 5)
    wl = W.make_workload(spec, seed=SLICE_SEED + 2, sources=True, losses=True)
    f = wl.fields
    for c, (iV, iK) in enumerate([(5, 2), (0, 4), (3, 0)]):
        sl = lambda a: np.ascontiguousarray(a[:, :, iV, iK])  # noqa: E731
        G = sl(f["G_conv"]) * (1.0 + 0.2 * rng.uniform(size=(12, 13)))
        args = dict(P=sl(f["Pg"]), R=sl(f["Rg"]), pl=f["Pl"][:, iV, iK], pu=f["Pu"][:, iV, iK],
                    rl=f["Rl"][:, iV, iK] + 0.01, ru=f["Ru"][:, iV, iK], VP=sl(f["VP"]) * 0.05,
                    VR=sl(f["VR"]), S=sl(f["S"]), loss=sl(f["loss_conv"]), G=G, dt=wl.dt)
        psd = sl(f["psd"])
        _, res, _ = ref.convection_2d(psd, types=(0, 0, 1, 1), **args)
        for k, v in args.items():
            out[f"c2_{c}_{k}"] = np.asarray(v)
        out[f"c2_{c}_psd"] = psd
        out[f"c2_{c}_out"] = res

    # ---- radial Kalman filter columns
    spec = W.GridSpec(2, 25, 3, 3)
    wl = W.make_workload(spec, seed=SLICE_SEED + 3)
    f = wl.fields
    for c, nobs in enumerate([0, 3, 9]):
        ln = lambda a: a[0, :, 1, 2]  # noqa: E731
        obs = np.full(25, np.nan)
        idx = rng.choice(np.arange(1, 24), size=nobs, replace=False)
        obs[idx] = ln(f["psd"])[idx] * np.exp(0.05 * rng.standard_normal(nobs))
        fc = ln(f["psd"]).copy()
        fc[0], fc[-1] = f["Ll"][0, 1, 2], f["Lu"][0, 1, 2]
        pa = np.zeros((25, 25))
        args = dict(R=ln(f["Lg"]), DLL=ln(f["DLL"]) * 100, G=ln(f["G_radial"]),
                    lbc=float(fc[0]), ubc=float(fc[-1]), lbc_t=1, ubc_t=1, obs=obs, dt=wl.dt,
                    model_error=1e-4, obs_error=1e-3)
        st, fo, pao, F, Pf = ref.kf_diffusion_1d(fc, pa, **args)
        # second update starting from the analysis covariance
        st2, fo2, pao2, _, _ = ref.kf_diffusion_1d(fo, pao, **args)
        for k, v in args.items():
            out[f"kf_{c}_{k}"] = np.asarray(v)
        out.update({f"kf_{c}_x0": fc, f"kf_{c}_x1": fo, f"kf_{c}_Pa1": pao, f"kf_{c}_F": F,
                    f"kf_{c}_Pf": Pf, f"kf_{c}_x2": fo2, f"kf_{c}_Pa2": pao2})
    np.savez_compressed(os.path.join(HERE, "slices.npz"), **out)

    # ---- two whole steps
    wl = step_workload()
    P, R, V, K = wl.spec.shape
    n = V * K
    ldab = 3 * (V + 1) + 1
    lu = np.zeros((P * R, ldab * n))
    ipiv = np.zeros((P * R, n), dtype=np.int64)
    psd1, neg1 = ref_step(ref, ref_lu, wl, wl.fields["psd"], lu, ipiv, True)
    psd2, neg2 = ref_step(ref, ref_lu, wl, psd1, lu, ipiv, False)
    fp = np.array([wl.fields[k].sum() for k in sorted(wl.fields)])
    np.savez_compressed(os.path.join(HERE, "step.npz"), spec=np.array(STEP_SPEC), seed=STEP_SEED,
                        psd1=psd1, psd2=psd2, neg=np.array([neg1, neg2]), input_sums=fp,
                        ipiv=ipiv)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
