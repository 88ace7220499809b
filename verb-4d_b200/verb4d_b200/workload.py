"""Seeded synthetic inputs for the VERB-4D operator-split step.

The reference ships no input decks, so workloads are generated here from the
physical models the benchmark configurations name.  All fields are float64
4-D arrays [P][R][V][K] (K fastest, the reference's Matrix4D layout,
src/Matrix.cpp:4211-4220):

* P  = MLT in hours, linspace(0, 24, nP): periodic, endpoint duplicated, as
  the periodic convection assumes PSD[0] == PSD[nP-1]
  (src/Convection_1D_ULTIMATE_QUICKEST6.cpp:97).
* R  = L, linspace(1.0, 6.6, nL); the radial grid L* equals R (static field).
* V  = log10(E / MeV), E = logspace(-2, 1, nE).
* K  = equatorial pitch angle in radians, linspace(0.3, 89.7, nA) degrees.

Coefficients (time unit: day):
* D_LL = 10**(0.506 Kp - 9.325) * L**10 (Brautigam-Albert).
* D_VV, D_KK: i.i.d. log-normal, median 1e-5 /s (0.864 /day), sigma one decade;
  D_VK = u * 0.99 * sqrt(D_VV D_KK), u ~ U[-1, 1] (the reference aborts when
  D_VV D_KK - D_VK**2 < 0, src/VERB4D_Solver.cpp:747-753).
* VP (MLT hours/day) = corotation + Volland-Stern E x B + gradient-curvature
  drift of electrons; VR (L/day) = Volland-Stern E x B radial component.
* PSD0 = exp(-E/0.2 MeV) sin(alpha) exp(-(L-4.5)**2).
* G_radial = L**-2 (radial Jacobian), G_local = G_conv = 1.
* Boundary conditions: zero inner L and fixed outer L (ConstantValue), zero
  pitch-angle gradient at both pitch-angle edges (ConstantDerivative 0),
  ConstantValue from PSD0 at both energy edges, periodic MLT.

The Kp series of the production-size run is hourly, uniform in [1, 6]; D_LL
follows it through a scale factor on a Kp=3 base field (the reference's
UpdatableMatrix scale mechanism, src/UpdatableMatrix.cpp:700-708) and the
velocities through hourly replacement fields.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

BC_PERIODIC, BC_VALUE, BC_DERIV = 0, 1, 2

# physical constants (SI)
_Q = 1.602176634e-19
_B0 = 3.11e-5          # equatorial surface field, T
_RE = 6.371e6          # Earth radius, m
_MC2_MEV = 0.51099895  # electron rest energy, MeV
_MEV = 1.602176634e-13
_OMEGA_E = 7.2921159e-5
_DAY = 86400.0

DT_5MIN = 5.0 / 1440.0


@dataclass
class GridSpec:
    P: int
    R: int
    V: int
    K: int

    @property
    def shape(self):
        return (self.P, self.R, self.V, self.K)

    @property
    def npts(self):
        return self.P * self.R * self.V * self.K


CONFIGS = {
    # 24 MLT x 25 L x 31 E x 31 alpha, Kp = 3, 288 steps of 5 min (CPU-runnable case)
    "cfg1": GridSpec(24, 25, 31, 31),
    # 48 MLT x 101 L x 101 E x 91 alpha, hourly Kp in [1, 6], 288 steps of 5 min
    "cfg2": GridSpec(48, 101, 101, 91),
    # profiling case: the production (MLT, L) slice shape over a coarse (E, alpha)
    # grid that still spans 0.01-10 MeV (small enough for full ncu captures)
    "cfg2s": GridSpec(48, 101, 12, 12),
    # profiling case: the production (MLT, L, E) grid over 8 pitch angles, so
    # that the convection kernel sees the production energy mix and more slices
    # than resident CTAs
    "cfg2m": GridSpec(48, 101, 101, 8),
}


def axes(spec: GridSpec):
    mlt = np.linspace(0.0, 24.0, spec.P)
    L = np.linspace(1.0, 6.6, spec.R)
    logE = np.linspace(-2.0, 1.0, spec.V)
    alpha = np.deg2rad(np.linspace(0.3, 89.7, spec.K))
    return mlt, L, logE, alpha


def dll_brautigam_albert(L, kp):
    return 10.0 ** (0.506 * kp - 9.325) * L ** 10


def volland_stern_a0(kp):
    """Maynard-Chen convection strength, V / RE**2."""
    return 1e3 * 0.045 / (1.0 - 0.159 * kp + 0.0093 * kp * kp) ** 3


def drift_velocities(spec: GridSpec, kp: float):
    """VP (MLT hours/day) and VR (L/day) on the 4-D grid, float64 [P][R][V][K]."""
    mlt, L, logE, alpha = axes(spec)
    phi = 2.0 * np.pi * mlt / 24.0
    a0 = volland_stern_a0(kp)
    k = L[None, :] ** 2 / (_B0 * _RE ** 2)               # [1][R]
    dphi_conv = k * 2.0 * a0 * L[None, :] * np.sin(phi)[:, None]       # rad/s [P][R]
    dL_conv = -k * a0 * L[None, :] ** 2 * np.cos(phi)[:, None]         # 1/s  [P][R]
    W = 10.0 ** logE                                        # MeV
    pv = W * (W + 2 * _MC2_MEV) / (W + _MC2_MEV) * _MEV     # J
    shape = 0.7 + 0.3 * np.sin(alpha)                       # pitch-angle factor
    dphi_gc = (3.0 * L[:, None, None] * pv[None, :, None] * shape[None, None, :]
               / (2.0 * _Q * _B0 * _RE ** 2))               # rad/s [R][V][K]
    to_mlt_per_day = 24.0 / (2.0 * np.pi) * _DAY
    VP = ((_OMEGA_E + dphi_conv)[:, :, None, None] + dphi_gc[None]) * to_mlt_per_day
    VR = np.broadcast_to((dL_conv * _DAY)[:, :, None, None], spec.shape)
    return np.ascontiguousarray(VP), np.ascontiguousarray(VR)


def kp_series(seed: int, hours: int):
    rng = np.random.default_rng(seed + 7919)
    return rng.uniform(1.0, 6.0, size=hours)


@dataclass
class Workload:
    spec: GridSpec
    fields: dict
    bc_types: dict
    flags: dict
    dt: float = DT_5MIN
    sub_dt: float = DT_5MIN
    kp: np.ndarray = field(default_factory=lambda: np.full(24, 3.0))
    dll_base_kp: float = 3.0

    def dll_scale(self, hour: int) -> float:
        kp = self.kp[min(hour, len(self.kp) - 1)]
        return 10.0 ** (0.506 * (kp - self.dll_base_kp))


def _smooth_ek(z: np.ndarray, corr: float) -> np.ndarray:
    """Gaussian-filter a field of unit normals along (E, alpha) with a width of
    `corr` grid points and rescale each (MLT, L) slice back to unit variance."""
    from scipy.ndimage import gaussian_filter

    out = gaussian_filter(z, sigma=(0, 0, corr, corr), mode="nearest")
    sd = out.std(axis=(2, 3), keepdims=True)
    return out / np.where(sd > 0, sd, 1.0)


def make_workload(spec: GridSpec, seed: int = 1, kp: float | np.ndarray = 3.0,
                  sources: bool = False, losses: bool = False,
                  coeff_corr: float = 0.0) -> Workload:
    """Build every input field of one run.  `sources`/`losses` switch on small
    seeded source and loss-rate fields (off in the benchmark configurations).
    The local diffusion coefficients are log-normal with independent values
    at every grid point (coeff_corr = 0), or, with coeff_corr > 0, smooth in
    (E, alpha) with that correlation width in grid points (same draws,
    filtered), as wave-model coefficient tables are."""
    rng = np.random.default_rng(seed)
    mlt, L, logE, alpha = axes(spec)
    shp = spec.shape
    P4 = np.broadcast_to(mlt[:, None, None, None], shp)
    R4 = np.broadcast_to(L[None, :, None, None], shp)
    V4 = np.broadcast_to(logE[None, None, :, None], shp)
    K4 = np.broadcast_to(alpha[None, None, None, :], shp)
    E = 10.0 ** logE
    psd0 = (np.exp(-E / 0.2)[None, None, :, None] * np.sin(alpha)[None, None, None, :]
            * np.exp(-(L - 4.5) ** 2)[None, :, None, None])
    psd0 = np.ascontiguousarray(np.broadcast_to(psd0, shp))

    kps = np.atleast_1d(np.asarray(kp, dtype=np.float64))
    dll_base = np.ascontiguousarray(np.broadcast_to(
        dll_brautigam_albert(L, 3.0)[None, :, None, None], shp))
    med = 1e-5 * _DAY
    zv = rng.standard_normal(shp)
    zk = rng.standard_normal(shp)
    u = rng.uniform(-1.0, 1.0, shp)
    if coeff_corr > 0:
        from scipy.special import erf

        zv, zk = _smooth_ek(zv, coeff_corr), _smooth_ek(zk, coeff_corr)
        # a smooth field uniform on (-1, 1) from a smoothed normal one
        u = erf(_smooth_ek(rng.standard_normal(shp), coeff_corr) / np.sqrt(2.0))
    dvv = med * 10.0 ** zv
    dkk = med * 10.0 ** zk
    dvk = u * 0.99 * np.sqrt(dvv * dkk)
    VP, VR = drift_velocities(spec, float(kps[0]))
    ones = np.ones(shp)
    zeros = np.zeros(shp)
    S = zeros.copy()
    loss = zeros.copy()
    if sources:
        S = 1e-3 * psd0 * rng.uniform(0.0, 1.0, shp)
    if losses:
        # loss rates are negative numbers (applied as exp(Loss dt) in convection)
        loss = -rng.uniform(0.0, 2.0, shp)
    Pl = np.full((spec.R, spec.V, spec.K), -1e99)
    fields = dict(
        psd=psd0, Pg=np.ascontiguousarray(P4), Rg=np.ascontiguousarray(R4),
        Vg=np.ascontiguousarray(V4), Kg=np.ascontiguousarray(K4), Lg=np.ascontiguousarray(R4),
        DLL=dll_base * (10.0 ** (0.506 * (kps[0] - 3.0))), DVV=dvv, DKK=dkk, DVK=dvk,
        VP=VP, VR=VR, G_local=ones, G_radial=np.ascontiguousarray(1.0 / R4 ** 2), G_conv=ones,
        S=S, loss_local=loss.copy() if losses else zeros, loss_radial=zeros.copy(),
        loss_conv=loss.copy() if losses else zeros.copy(),
        Pl=Pl, Pu=Pl.copy(),
        Rl=np.zeros((spec.P, spec.V, spec.K)), Ru=np.ascontiguousarray(psd0[:, -1, :, :]),
        Ll=np.zeros((spec.P, spec.V, spec.K)), Lu=np.ascontiguousarray(psd0[:, -1, :, :]),
        Vl=np.ascontiguousarray(psd0[:, :, 0, :]), Vu=np.ascontiguousarray(psd0[:, :, -1, :]),
        Kl=np.zeros((spec.P, spec.R, spec.V)), Ku=np.zeros((spec.P, spec.R, spec.V)),
        DLL_base=dll_base,
    )
    bc = dict(Pl=BC_PERIODIC, Pu=BC_PERIODIC, Rl=BC_VALUE, Ru=BC_VALUE, Ll=BC_VALUE, Lu=BC_VALUE,
              Vl=BC_VALUE, Vu=BC_VALUE, Kl=BC_DERIV, Ku=BC_DERIV)
    # source/loss routing of src/VERB4D_Solver.cpp:404-426: with local diffusion
    # running on a >=3x3 (V,K) grid, sources and losses go to the local step.
    flags = dict(run_convection=1, run_radial=1, run_local=1, radial_sources=0, local_sources=1,
                 include_boundary=1, positive_psd=0)
    wl = Workload(spec=spec, fields=fields, bc_types=bc, flags=flags,
                  kp=kps if len(kps) > 1 else np.full(24, float(kps[0])), dll_base_kp=3.0)
    return wl


def loss_cone_deg(L):
    """Equatorial bounce loss cone of a dipole, alpha_lc(L) =
    asin(sqrt(1 / (L^5 sqrt(4 - 3/L)))), in degrees."""
    L = np.asarray(L, dtype=np.float64)
    return np.rad2deg(np.arcsin(np.sqrt(1.0 / (L ** 5 * np.sqrt(4.0 - 3.0 / L)))))


def loss_cone_k0(wl: Workload) -> np.ndarray:
    """First pitch-angle index outside the loss cone for every (MLT, L)
    system, [P][R] int32: the trimmed (ragged) local systems keep K indices
    k0..K-1."""
    f = wl.fields
    L = f["Lg"][:, :, 0, 0]
    alpha = np.rad2deg(f["Kg"][:, :, 0, :])  # [P][R][K]
    lc = loss_cone_deg(L)[:, :, None]
    keep = alpha > lc
    k0 = np.where(keep.any(axis=2), keep.argmax(axis=2), alpha.shape[2])
    return k0.astype(np.int32)


def oracle_inputs(wl: Workload) -> dict:
    d = dict(wl.fields)
    d["bc_types"] = wl.bc_types
    d["flags"] = wl.flags
    return d


def convection_substeps(wl: Workload) -> np.ndarray:
    """Slice-level sub-step count of src/Convection_2D.cpp:57-86 for every (V,K)."""
    f = wl.fields
    dt = wl.dt
    vp = np.abs(f["VP"]).max(axis=(0, 1))
    vr = np.abs(f["VR"]).max(axis=(0, 1))
    dP = f["Pg"][1, 0] - f["Pg"][0, 0]
    dR = f["Rg"][0, 1] - f["Rg"][0, 0]
    a = dt * vp / dP / 0.25
    b = dt * vr / dR / 0.25
    na = np.where(a <= 1, 1, np.ceil(a))
    nb = np.where(b <= 1, 1, np.ceil(b))
    return np.maximum(na, nb).astype(np.int64)
