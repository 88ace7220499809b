// extern "C" harness around the UNMODIFIED reference per-slice routines.
//
// Test infrastructure only: compiled together with the reference sources
// (read in place from the reference tree by oracle/Makefile) into
// oracle/_ref/libverbref.so (plain build) and oracle/_ref/libverbref_lu.so
// (built with -DLU_CACHING).  It exists so that the CPU restatement in
// oracle/verb_oracle.c and the golden fixtures can be checked against the
// reference itself, and so bench.py can time the reference CPU path.
//
// Each entry copies plain row-major arrays into the reference's Matrix1D /
// Matrix2D containers, calls the reference routine, and copies the result
// back.  Layouts follow the reference: a local (V,K) slice is [V][K], a
// convection slice is [P][R].
#include <cstring>
#include <tuple>
#include <vector>

#include "BoundaryConditionType.hpp"
#include "Convection_1D_ULTIMATE_QUICKEST6.h"
#include "Convection_2D.h"
#include "DataAssimilation.h"
#include "DataAssimilationConvection.h"
#include "DataAssimilationDiffusion.h"
#include "Diffusion_1D.h"
#include "Diffusion_2D.h"
#include "Matrix.h"
#include "MatrixSolver.h"
#include "MonotCubicInterpolator.hpp"
#include "UpdatableMatrix.h"

namespace {

Matrix1D<double> vec(const double* p, long n)
{
    Matrix1D<double> m(static_cast<size_t>(n));
    std::memcpy(&m[0], p, sizeof(double) * static_cast<size_t>(n));
    return m;
}

Matrix2D<double> mat(const double* p, long n1, long n2)
{
    Matrix2D<double> m(static_cast<size_t>(n1), static_cast<size_t>(n2));
    std::memcpy(m[0], p, sizeof(double) * static_cast<size_t>(n1 * n2));
    return m;
}

BoundaryConditionType bct(int t) { return static_cast<BoundaryConditionType>(t); }

}  // namespace

extern "C" {

// src/MatrixSolver.cpp:689 tridag
int ref_tridag(double* a, double* b, double* c, double* r, double* u, long n)
{
    return tridag(a, b, c, r, u, static_cast<size_t>(n)) ? 0 : 1;
}

// src/Diffusion_1D.cpp:43 Diffusion_1D (psd updated in place)
int ref_diffusion_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                     int ubc_t, const double* D, const double* G, const double* S,
                     const double* loss, double dt)
{
    Matrix1D<double> f = vec(psd, n);
    Diffusion_1D(f, vec(x, n), n, lbc, ubc, bct(lbc_t), bct(ubc_t), vec(D, n), vec(G, n),
                 vec(S, n), vec(loss, n), dt);
    std::memcpy(psd, &f[0], sizeof(double) * n);
    return 0;
}

// src/Diffusion_1D.cpp:91 getCalculationMatrix1DDiffusion: the three diagonals of A,
// diag(B) and C of one radial line.
int ref_radial_matrix(const double* x, int n, double lbc, double ubc, int lbc_t, int ubc_t,
                      const double* D, const double* G, const double* S, const double* loss,
                      double dt, double* a_lo, double* a_d, double* a_up, double* b_d,
                      double* c_d)
{
    auto m = getCalculationMatrix1DDiffusion(vec(x, n), n, lbc, ubc, bct(lbc_t), bct(ubc_t),
                                             vec(D, n), vec(G, n), vec(S, n), vec(loss, n), dt);
    CalculationMatrix& A = std::get<0>(m);
    CalculationMatrix& B = std::get<1>(m);
    CalculationMatrix& C = std::get<2>(m);
    for (int i = 0; i < n; i++) {
        a_lo[i] = A[-1][i];
        a_d[i] = A[0][i];
        a_up[i] = A[1][i];
        b_d[i] = B[0][i];
        c_d[i] = C[0][i];
    }
    return 0;
}

#ifdef LU_CACHING
// src/Diffusion_2D.cpp:20 Diffusion_2D, LU_CACHING form: lu (ldab*n doubles) and
// ipiv (n longs, 1-based LAPACK pivots) are the caller-owned cache slot.
int ref_diffusion_2d_lu(double* psd, const double* x, const double* y, int nx, int ny,
                        const double* xl, const double* xu, const double* yl, const double* yu,
                        int xl_t, int xu_t, int yl_t, int yu_t, const double* Dxx,
                        const double* Dyy, const double* Dxy, const double* Dyx, const double* G,
                        const double* S, const double* loss, double dt, double sub_dt,
                        double* lu, long* ipiv, int recompute)
{
    Matrix2D<double> f = mat(psd, nx, ny);
    Diffusion_2D(f, mat(x, nx, ny), mat(y, nx, ny), nx, ny, vec(xl, ny), vec(xu, ny), vec(yl, nx),
                 vec(yu, nx), bct(xl_t), bct(xu_t), bct(yl_t), bct(yu_t), mat(Dxx, nx, ny),
                 mat(Dyy, nx, ny), mat(Dxy, nx, ny), mat(Dyx, nx, ny), mat(G, nx, ny),
                 mat(S, nx, ny), mat(loss, nx, ny), dt, sub_dt, lu, ipiv, recompute != 0);
    std::memcpy(psd, f[0], sizeof(double) * nx * ny);
    return 0;
}
#else
// src/Diffusion_2D.cpp:32 Diffusion_2D, plain form (factor + solve every call).
int ref_diffusion_2d(double* psd, const double* x, const double* y, int nx, int ny,
                     const double* xl, const double* xu, const double* yl, const double* yu,
                     int xl_t, int xu_t, int yl_t, int yu_t, const double* Dxx, const double* Dyy,
                     const double* Dxy, const double* Dyx, const double* G, const double* S,
                     const double* loss, double dt, double sub_dt)
{
    Matrix2D<double> f = mat(psd, nx, ny);
    Diffusion_2D(f, mat(x, nx, ny), mat(y, nx, ny), nx, ny, vec(xl, ny), vec(xu, ny), vec(yl, nx),
                 vec(yu, nx), bct(xl_t), bct(xu_t), bct(yl_t), bct(yu_t), mat(Dxx, nx, ny),
                 mat(Dyy, nx, ny), mat(Dxy, nx, ny), mat(Dyx, nx, ny), mat(G, nx, ny),
                 mat(S, nx, ny), mat(loss, nx, ny), dt, sub_dt);
    std::memcpy(psd, f[0], sizeof(double) * nx * ny);
    return 0;
}
#endif

// src/Convection_1D_ULTIMATE_QUICKEST6.cpp:22 (psd updated in place)
int ref_convection_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                      int ubc_t, const double* ux, double dt)
{
    Matrix1D<double> f = vec(psd, n);
    Convection_1D_ULTIMATE_QUICKEST6(f, vec(x, n), n, lbc, ubc, bct(lbc_t), bct(ubc_t), vec(ux, n),
                                     dt);
    std::memcpy(psd, &f[0], sizeof(double) * n);
    return 0;
}

// src/Convection_2D.cpp:36 Convection_2D on one [P][R] slice (psd updated in place)
int ref_convection_2d(double* psd, const double* P, const double* R, int nP, int nR,
                      const double* pl, const double* pu, const double* rl, const double* ru,
                      int pl_t, int pu_t, int rl_t, int ru_t, const double* VP, const double* VR,
                      const double* S, const double* loss, const double* G, double dt)
{
    Matrix2D<double> f = mat(psd, nP, nR);
    Convection_2D(f, mat(P, nP, nR), mat(R, nP, nR), nP, nR, vec(pl, nR), vec(pu, nR), vec(rl, nP),
                  vec(ru, nP), bct(pl_t), bct(pu_t), bct(rl_t), bct(ru_t), mat(VP, nP, nR),
                  mat(VR, nP, nR), mat(S, nP, nR), mat(loss, nP, nR), mat(G, nP, nR), dt);
    std::memcpy(psd, f[0], sizeof(double) * nP * nR);
    return 0;
}

// src/DataAssimilationDiffusion.cpp:151 runKalmanFilterDiffusion1D for one radial column.
// forecast[n] and Pa[n*n] are updated in place; F[n*n] receives the model matrix and
// Pf[n*n] the forecast covariance.
int ref_kf_diffusion_1d(double* forecast, double* Pa, double* F, double* Pf, const double* R,
                        const double* DLL, const double* G, int n, double lbc, double ubc,
                        int lbc_t, int ubc_t, const double* obs, double dt, double model_error,
                        double obs_error)
{
    Matrix1D<double> f = vec(forecast, n);
    Matrix2D<double> pa = mat(Pa, n, n);
    Matrix2D<double> model(static_cast<size_t>(n), static_cast<size_t>(n));
    model = 0;
    data_assimilation::Parameters prm{};
    prm.runDataAssimilation = true;
    prm.useLog = false;
    prm.timeStep = dt;
    prm.modelError = model_error;
    prm.observationError = obs_error;
    try {
        auto dbg = data_assimilation::runKalmanFilterDiffusion1D(
            f, pa, model, vec(R, n), vec(DLL, n), vec(G, n), lbc, ubc, bct(lbc_t), bct(ubc_t),
            vec(obs, n), dt, prm);
        std::memcpy(Pf, dbg.a_priori_err_cov[0], sizeof(double) * n * n);
    } catch (...) {
        return 2;  // the reference throws on NaN after the update (DataAssimilation.cpp:62-67)
    }
    std::memcpy(forecast, &f[0], sizeof(double) * n);
    std::memcpy(Pa, pa[0], sizeof(double) * n * n);
    std::memcpy(F, model[0], sizeof(double) * n * n);
    return 0;
}

// src/DataAssimilationConvection.cpp:124 runKalmanFilterConvection2D for one
// (V,K) slice of nP x nR points (N = nP*nR).  forecast[N] ([P][R]) and Pa[N*N]
// are updated in place; model[N*N] is the model-matrix cache (used as given
// when model_valid and !has_vx_updated, else rebuilt and returned); Pf[N*N]
// receives the forecast covariance.  P and R are the [P][R] grids; loss is the
// loss-rate slice; sat (may be NULL) the saturation map as 0/1 bytes.
int ref_kf_convection_2d(double* forecast, double* Pa, double* model, int model_valid, double* Pf,
                         const double* P, const double* R, const double* VP, const double* VR,
                         int has_vx_updated, const double* loss, const unsigned char* sat,
                         const double* obs, int nP, int nR, double dt, double model_error,
                         double obs_error, int use_log, double correlation_time, int growing_q)
{
    const long N = static_cast<long>(nP) * nR;
    Matrix2D<double> f = mat(forecast, nP, nR);
    Matrix2D<double> pa = mat(Pa, N, N);
    Matrix2D<double> mm;
    if (model_valid) mm = mat(model, N, N);
    Matrix2D<bool> satm(static_cast<size_t>(nP), static_cast<size_t>(nR));
    for (long i = 0; i < N; i++) satm[i / nR][i % nR] = sat ? sat[i] != 0 : false;
    data_assimilation::Parameters prm{};
    prm.runDataAssimilation = true;
    prm.useLog = use_log != 0;
    prm.timeStep = dt;
    prm.modelError = model_error;
    prm.observationError = obs_error;
    prm.correlationTime = correlation_time;
    prm.growing_Q_at_boundary = growing_q != 0;
    try {
        auto dbg = data_assimilation::runKalmanFilterConvection2D(
            f, pa, mm, mat(P, nP, nR), mat(R, nP, nR), mat(VP, nP, nR), mat(VR, nP, nR),
            has_vx_updated != 0, mat(loss, nP, nR), satm, mat(obs, nP, nR), dt, prm);
        std::memcpy(Pf, dbg.a_priori_err_cov[0], sizeof(double) * N * N);
    } catch (...) {
        return 2;  // NaN after the update (src/DataAssimilation.cpp:62-67) or an unstable model
    }
    std::memcpy(forecast, f[0], sizeof(double) * N);
    std::memcpy(Pa, pa[0], sizeof(double) * N * N);
    std::memcpy(model, mm[0], sizeof(double) * N * N);
    return 0;
}

// The interpolator behind the L* remapping (Opm::MonotCubicInterpolator,
// src/MonotCubicInterpolator.cpp), built from the points themselves.
int ref_monot_cubic(const double* x, const double* f, int n, const double* xq, double* out, int m)
{
    std::vector<double> xv(x, x + n), fv(f, f + n);
    Opm::MonotCubicInterpolator ip(xv, fv);
    for (int j = 0; j < m; j++) out[j] = ip.evaluate(xq[j]);
    return 0;
}

// PSD output / restart files: Matrix4D::writeToBinaryFile and
// readFromBinaryFile (src/Matrix.cpp:5700-5720, 5780-5808), the .pltb format.
int ref_write_pltb(const double* data, int w, int x, int y, int z, const char* path)
{
    Matrix4D<double> m((size_t)w, (size_t)x, (size_t)y, (size_t)z);
    std::memcpy(&m[0][0][0][0], data, sizeof(double) * (size_t)w * x * y * z);
    m.writeToBinaryFile(path);
    return 0;
}

int ref_read_pltb(double* data, int w, int x, int y, int z, const char* path)
{
    Matrix4D<double> m((size_t)w, (size_t)x, (size_t)y, (size_t)z);
    m.readFromBinaryFile(path);
    std::memcpy(data, &m[0][0][0][0], sizeof(double) * (size_t)w * x * y * z);
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Phase loops for timing the reference CPU path: the OpenMP loops of
// src/VERB4D_Solver.cpp (convection :885-978, radial :1009-1070, local
// :1101-1216) over a caller-chosen list of slices, each slice solved by the
// reference routine.  Slices are copied out of and back into the 4-D arrays
// as the reference's yzSlice / wyzSlice / wxSlice do.  `st` points to the
// oracle's orc_state (oracle/verb_oracle.h), which carries the same fields.
#include <omp.h>

#include "../oracle/verb_oracle.h"

extern "C" {

int ref_conv_slices(orc_state* s, double dt, const int* vk, int nlist, int nthreads)
{
    const int P = s->P, R = s->R, V = s->V, K = s->K;
    auto I4 = [&](int p, int r, int v, int k) { return (((size_t)p * R + r) * V + v) * K + k; };
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int t = 0; t < nlist; t++) {
        const int iV = vk[2 * t], iK = vk[2 * t + 1];
        Matrix2D<double> f(P, R), pg(P, R), rg(P, R), vp(P, R), vr(P, R), sr(P, R), ls(P, R), gg(P, R);
        Matrix1D<double> pl(R), pu(R), rl(P), ru(P);
        for (int iP = 0; iP < P; iP++)
            for (int iR = 0; iR < R; iR++) {
                const size_t g = I4(iP, iR, iV, iK);
                f[iP][iR] = s->psd[g];
                pg[iP][iR] = s->Pg[g];
                rg[iP][iR] = s->Rg[g];
                vp[iP][iR] = s->VP[g];
                vr[iP][iR] = s->VR[g];
                sr[iP][iR] = s->S[g];
                ls[iP][iR] = s->loss_conv[g];
                gg[iP][iR] = s->G_conv[g];
            }
        for (int iR = 0; iR < R; iR++) {
            pl[iR] = s->Pl[((size_t)iR * V + iV) * K + iK];
            pu[iR] = s->Pu[((size_t)iR * V + iV) * K + iK];
        }
        for (int iP = 0; iP < P; iP++) {
            rl[iP] = s->Rl[((size_t)iP * V + iV) * K + iK];
            ru[iP] = s->Ru[((size_t)iP * V + iV) * K + iK];
        }
        Convection_2D(f, pg, rg, P, R, pl, pu, rl, ru, bct(s->Pl_t), bct(s->Pu_t), bct(s->Rl_t),
                      bct(s->Ru_t), vp, vr, sr, ls, gg, dt);
        for (int iP = 0; iP < P; iP++)
            for (int iR = 0; iR < R; iR++) s->psd[I4(iP, iR, iV, iK)] = f[iP][iR];
    }
    return 0;
}

int ref_radial_lines(orc_state* s, double dt, const int* pvk, int nlist, int nthreads)
{
    const int R = s->R, V = s->V, K = s->K;
    const double rs = (double)s->radial_sources;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int t = 0; t < nlist; t++) {
        const int iP = pvk[3 * t], iV = pvk[3 * t + 1], iK = pvk[3 * t + 2];
        Matrix1D<double> f(R), lg(R), dl(R), sr(R), gr(R), ls(R);
        for (int iR = 0; iR < R; iR++) {
            const size_t g = (((size_t)iP * R + iR) * V + iV) * K + iK;
            f[iR] = s->psd[g];
            lg[iR] = s->Lg[g];
            dl[iR] = s->DLL[g];
            sr[iR] = s->S[g];
            gr[iR] = s->G_radial[g];
            ls[iR] = s->loss_radial[g];
        }
        sr *= rs;
        const size_t b = ((size_t)iP * V + iV) * K + iK;
        Diffusion_1D(f, lg, R, s->Ll[b], s->Lu[b], bct(s->Ll_t), bct(s->Lu_t), dl, gr, sr, ls, dt);
        for (int iR = 0; iR < R; iR++) s->psd[(((size_t)iP * R + iR) * V + iV) * K + iK] = f[iR];
    }
    return 0;
}

// src/UpdatableMatrix.cpp:857-961 with :308-600 and :602-846: an
// UpdatableListMatrix<Matrix4D<double>> read from the .tab file `tab` (one
// component per line: a .pltb data file or a .lst list of (time, .pltb file),
// then optionally a scale (a number or a .lst list of (time, value)) and
// from/to limits per axis), merged by SUM (mean = 0) or MEAN, and updated at
// times[0..nt).  out receives the field after every update ([nt][P][R][V][K])
// and updated[t] the update's return value.  q1..q4 are the four grids.
int ref_updatable_list(const char* tab, int mean, int P, int R, int V, int K, const double* q1,
                       const double* q2, const double* q3, const double* q4, const double* times,
                       int nt, double* out, int* updated)
{
    const size_t n = (size_t)P * R * V * K;
    auto grid = [&](const double* q) {
        Matrix4D<double> m((size_t)P, (size_t)R, (size_t)V, (size_t)K);
        std::memcpy(&m[0][0][0][0], q, sizeof(double) * n);
        return m;
    };
    const Matrix4D<double> Q1 = grid(q1), Q2 = grid(q2), Q3 = grid(q3), Q4 = grid(q4);
    using L = UpdatableListMatrix<Matrix4D<double>>;
    L field(mean ? L::MERGE_TYPE::MEAN : L::MERGE_TYPE::SUM);
    field.AllocateMemory((size_t)P, (size_t)R, (size_t)V, (size_t)K);
    field = 0.0;
    if (!field.readFromIniFile(tab, Q1, Q2, Q3, Q4)) return 1;
    for (int t = 0; t < nt; t++) {
        updated[t] = field.update(times[t], Q1, Q2, Q3, Q4) ? 1 : 0;
        std::memcpy(out + (size_t)t * n, &field[0][0][0][0], sizeof(double) * n);
    }
    return 0;
}

#ifdef LU_CACHING
// lu / ipiv: one cache slot per list entry ((2kl+ku+1)*n doubles, n longs).
int ref_local_systems(orc_state* s, double dt, double sub_dt, const int* pr, int nlist,
                      double* lu, long* ipiv, int recompute, int nthreads)
{
    const int R = s->R, V = s->V, K = s->K;
    const size_t n = (size_t)V * K, ldab = 3 * (V + 1) + 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int t = 0; t < nlist; t++) {
        const int iP = pr[2 * t], iR = pr[2 * t + 1];
        const size_t base = ((size_t)iP * R + iR) * n, q = (size_t)iP * R + iR;
        Matrix2D<double> f = mat(s->psd + base, V, K);
        Matrix2D<double> src = mat(s->S + base, V, K) * s->local_sources;
        Diffusion_2D(f, mat(s->Vg + base, V, K), mat(s->Kg + base, V, K), V, K, vec(s->Vl + q * K, K),
                     vec(s->Vu + q * K, K), vec(s->Kl + q * V, V), vec(s->Ku + q * V, V),
                     bct(s->Vl_t), bct(s->Vu_t), bct(s->Kl_t), bct(s->Ku_t), mat(s->DVV + base, V, K),
                     mat(s->DKK + base, V, K), mat(s->DVK + base, V, K), mat(s->DVK + base, V, K),
                     mat(s->G_local + base, V, K), src, mat(s->loss_local + base, V, K), dt, sub_dt,
                     lu + t * ldab * n, ipiv + t * n, recompute != 0);
        std::memcpy(s->psd + base, f[0], sizeof(double) * n);
    }
    return 0;
}
#endif

}  // extern "C"
