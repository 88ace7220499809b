"""CPU restatement of the reference's convection data assimilation (test
oracle only: tests/ and the GPU smoke check import it; the product path
never does).

One (V,K) slice of nP x nR points is a state of N = nP*nR values ordered
iR + iP*nR.  The functions follow, step by step:

* model_matrix_1step  getModelMatrixConvection2DNoStabilityCheck
                      (src/DataAssimilationHelper.cpp:25-120): first-order
                      upwind transport matrix; rows iR = 0 and nR-1 carry only
                      the correlation factor; MLT rows 0 and nP-1 take their
                      neighbours from the periodic interior (nP-2 and 1)
* split_courant       splitTimeStepCourantCondition (:122-144)
* model_matrix        getModelMatrixConvection2D (:146-171): the one-step
                      matrix of the split step raised to the number of splits
* matpow              operator^ (src/MatrixOperations.cpp:466-620): squarings
                      cached for the set bits, multiplied together, then one
                      more product for odd powers (the same product sequence;
                      dgemm's operand order follows the reference's row-major
                      call, C = B A for dgemm(a=A, b=B))
* observation_space   convertToObservationSpace(Matrix2D)
                      (src/DataAssimilationHelper.cpp:230-269)
* run_kalman_filter   runKalmanFilter (src/DataAssimilation.cpp:18-77)
* kf_convection_2d    runKalmanFilterConvection2D
                      (src/DataAssimilationConvection.cpp:124-253)

Products are numpy matmul (OpenBLAS dgemm); the reference calls dgemm as
well, so the two agree to rounding.  The restatement is pinned against the
reference compiled from source (oracle/_ref, ref_kf_convection_2d).
"""
from __future__ import annotations

import math

import numpy as np


def model_matrix_1step(VP, VR, loss, sat, dt, dP, dR, use_log, corr):
    nP, nR = VP.shape
    N = nP * nR
    M = np.zeros((N, N))
    for iP in range(nP):
        for iR in range(nR):
            row = iR + iP * nR
            if iR == 0 or iR == nR - 1:
                M[row, row] = corr
                continue
            if iP == 0 or iP == nP - 1:
                iPl, iPr = nP - 2, 1
            else:
                iPl, iPr = iP - 1, iP + 1
            vp, vr = VP[iP, iR], VR[iP, iR]
            lc = 0.0 if sat[iP, iR] else loss[iP, iR]
            if use_log:
                mcc = 1. - abs(vp) * dt / dP - abs(vr) * dt / dR
            else:
                mcc = 1. - abs(vp) * dt / dP - abs(vr) * dt / dR + dt * lc
            if mcc < 0:
                raise ValueError("unstable model matrix")
            if vp > 0.:
                mlc, mrc = vp * dt / dP, 0.
            else:
                mlc, mrc = 0., -vp * dt / dP
            if vr > 0.:
                mcl, mcr = vr * dt / dR, 0.
            else:
                mcl, mcr = 0., -vr * dt / dR
            # assignments in the reference's order (later ones win where the
            # periodic neighbours coincide)
            M[row, row] = mcc
            M[row, iR + iPl * nR] = mlc
            M[row, iR + iPr * nR] = mrc
            M[row, iR - 1 + iP * nR] = mcl
            M[row, iR + 1 + iP * nR] = mcr
    return M


def split_courant(cmax, dt, VP, VR, dP, dR):
    c = np.abs(VP * dt / dP) + np.abs(VR * dt / dR)
    cour = np.abs(c).max()
    nt = 1 if cour <= cmax else int(math.ceil(cour / cmax))
    return nt, dt / float(nt)


def _gemm(a, b):
    """dgemm(transb, transa, m, n, k, 1, a, ldb, b, lda, 0, c, ldc) on row-major
    data, as the reference calls it: C = B A."""
    return b @ a


def matpow(A, power):
    if power == 1:
        return A.copy()
    bits = [(power >> i) & 1 for i in range(32)]
    cache_size = sum(bits) - 1 if bits[0] else sum(bits)
    cache = []
    cur = A.copy()
    for i in range(1, 32):
        cur = _gemm(cur, cur)          # A^(2^i)
        if bits[i]:
            cache.append(cur)
            if len(cache) == cache_size:
                break
    if len(cache) == 1:
        answer = cache[0]
    else:
        answer = _gemm(cache[0], cache[1])
        for c in cache[2:]:
            answer = _gemm(answer, c)
    if power % 2 == 1:
        answer = _gemm(answer, A)
    return answer


def model_matrix(VP, VR, loss, sat, dt, dP, dR, use_log, corr_time):
    nt, dtn = split_courant(1.0, dt, VP, VR, dP, dR)
    M1 = model_matrix_1step(VP, VR, loss, sat, dtn, dP, dR, use_log, math.exp(-dtn / corr_time))
    return matpow(M1, nt)


def observation_space(obs):
    flat = obs.reshape(-1)
    idx = np.nonzero(np.isfinite(flat))[0]
    N = flat.size
    if len(idx) == 0:
        return np.zeros(1), np.zeros((1, N))
    H = np.zeros((len(idx), N))
    H[np.arange(len(idx)), idx] = 1.0
    return flat[idx].copy(), H


def run_kalman_filter(x, Pa, M, Q, y, H, R):
    Pf = (M @ Pa) @ M.T + Q
    PfHt = Pf @ H.T
    S = H @ PfHt + R
    K = np.linalg.solve(S.T, PfHt.T).T          # trans_solve: K S = Pf H^T
    x = x + K @ (y - H @ x)
    if np.isnan(x).any():
        raise FloatingPointError("NaN detected in forecast vector after Kalman update.")
    Pa = Pf - (K @ H) @ Pf
    return x, Pa, Pf


def kf_convection_2d(forecast, Pa, model, Pg, Rg, VP, VR, has_vx_updated, loss, sat, obs, dt,
                     model_error, obs_error, use_log=False, correlation_time=math.inf,
                     growing_q=False):
    """One slice: returns (forecast, Pa, model, Pf).  model=None means no
    cached model matrix yet."""
    nP, nR = forecast.shape
    N = nP * nR
    dP = Pg[1, 0] - Pg[0, 0]
    dR = Rg[0, 1] - Rg[0, 0]
    if sat is None:
        sat = np.zeros((nP, nR), dtype=bool)
    if has_vx_updated or model is None:
        model = model_matrix(VP, VR, loss, sat, dt, dP, dR, use_log, correlation_time)
    y, H = observation_space(obs)
    x = forecast.reshape(-1).copy()
    if use_log:
        x = np.log(x)
        y = np.log(y)
    D = np.full(N, model_error)
    cf = math.exp(-dt / correlation_time)
    tmp = np.diag(D)
    bidx = [nR - 1 + iP * nR for iP in range(nP)] + [iP * nR for iP in range(nP)]
    for iP in range(nP):
        tmp[nR - 1 + iP * nR, nR - 1 + iP * nR] = (1. - cf * cf) * model_error
        tmp[iP * nR, iP * nR] = (1. - cf * cf) * model_error
    M1d = matpow(model, int(math.ceil(3. / 24 / dt)))
    Q = (M1d @ tmp) @ M1d.T + np.diag(D) / 10
    if not growing_q:
        for i in bidx:
            Q[i, i] = (1. - cf * cf) * model_error
    Robs = np.diag(np.full(len(y), obs_error)) if use_log else np.diag(y * obs_error)
    Pa = Pa.copy()
    if np.abs(Pa).max() == 0:
        Pa[np.arange(N), np.arange(N)] = 5 * model_error
    x, Pa, Pf = run_kalman_filter(x, Pa, model, Q, y, H, Robs)
    if use_log:
        x = np.power(math.e, x)
    return x.reshape(nP, nR), Pa, model, Pf
