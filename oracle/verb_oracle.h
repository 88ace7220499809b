/*
 * CPU restatement of the VERB-4D operator-split Fokker-Planck step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; only tests/, the smoke check and bench.py's CPU-baseline leg load
 * it.  Every routine restates one reference routine (cited by file:line
 * within the reference project) in plain C with the same evaluation order,
 * so that results are bit-identical to the reference wherever the reference
 * does not call LAPACK.  The banded LU is a restatement of LAPACK's published
 * unblocked algorithm (dgbtf2 / dgbtrs / dtbsv); the reference links
 * whatever LAPACK the build finds, so those results agree to rounding only.
 *
 * Boundary-condition type codes follow src/BoundaryConditionType.hpp:53-88:
 * 0 = Periodic, 1 = ConstantValue, 2 = ConstantDerivative.
 */
#ifndef VERB_ORACLE_H
#define VERB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_BC_PERIODIC = 0, ORC_BC_CONSTANT_VALUE = 1, ORC_BC_CONSTANT_DERIVATIVE = 2 };

int orc_tridag(const double* a, const double* b, const double* c, const double* r, double* u,
               long n);

int orc_radial_matrix(const double* x, int n, double lbc, double ubc, int lbc_t, int ubc_t,
                      const double* D, const double* G, const double* S, const double* loss,
                      double dt, double* a_lo, double* a_d, double* a_up, double* b_d,
                      double* c_d);

int orc_diffusion_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                     int ubc_t, const double* D, const double* G, const double* S,
                     const double* loss, double dt);

/* Local 2-D operator: A as 9 diagonals diag[9][nx*ny] in the order of offsets
 * {-nx-1,-nx,-nx+1,-1,0,1,nx-1,nx,nx+1}; B and C as vectors.  Unknown
 * index in = iy*nx + ix (x fastest). Arrays x,y,D*,G,S,loss are [nx][ny]. */
int orc_local_matrix(const double* x, const double* y, int nx, int ny, const double* xl,
                     const double* xu, const double* yl, const double* yu, int xl_t, int xu_t,
                     int yl_t, int yu_t, const double* Dxx, const double* Dyy, const double* Dxy,
                     const double* Dyx, const double* G, const double* S, const double* loss,
                     double dt, double* diag, double* b_d, double* c_d);

void orc_band_pack(const double* diag, int nx, int ny, double* ab);
long orc_gbtrf(long n, long kl, long ku, double* ab, long ldab, long* ipiv);
void orc_gbtrs(long n, long kl, long ku, const double* ab, long ldab, const long* ipiv,
               double* b);

int orc_diffusion_2d(double* psd, const double* x, const double* y, int nx, int ny,
                     const double* xl, const double* xu, const double* yl, const double* yu,
                     int xl_t, int xu_t, int yl_t, int yu_t, const double* Dxx, const double* Dyy,
                     const double* Dxy, const double* Dyx, const double* G, const double* S,
                     const double* loss, double dt, double sub_dt, double* lu, long* ipiv,
                     int recompute);

int orc_convection_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                      int ubc_t, const double* ux, double dt);

int orc_convection_2d(double* psd, const double* P, const double* R, int nP, int nR,
                      const double* pl, const double* pu, const double* rl, const double* ru,
                      int pl_t, int pu_t, int rl_t, int ru_t, const double* VP, const double* VR,
                      const double* S, const double* loss, const double* G, double dt,
                      int* substeps);

int orc_kf_diffusion_1d(double* forecast, double* Pa, double* F, double* Pf, const double* R,
                        const double* DLL, const double* G, int n, double lbc, double ubc,
                        int lbc_t, int ubc_t, const double* obs, double dt, double model_error,
                        double obs_error);

/* Monotone cubic interpolation of (x[i], f[i]), i < n, at xq[j], j < m
 * (Opm::MonotCubicInterpolator, src/MonotCubicInterpolator.cpp:95-104,
 * 160-225, 379-470, 613-700: averaged-secant derivatives, the monotone
 * adjustment when the data are monotone, cubic Hermite evaluation, constant
 * extrapolation).  x must be strictly increasing; returns -1 otherwise. */
int orc_monot_cubic(const double* x, const double* f, int n, const double* xq, double* out, int m);

/* Whole operator-split step over 4-D fields [P][R][V][K] (K fastest), in the
 * order and with the source/loss routing of src/VERB4D_Solver.cpp:851-1242. */
typedef struct {
    int P, R, V, K;
    double *psd;
    const double *Pg, *Rg, *Vg, *Kg, *Lg;
    const double *DLL, *DVV, *DKK, *DVK, *VP, *VR;
    const double *G_local, *G_radial, *G_conv;
    const double *S, *loss_local, *loss_radial, *loss_conv;
    const double *Pl, *Pu;            /* [R][V][K] */
    const double *Rl, *Ru, *Ll, *Lu;  /* [P][V][K] */
    const double *Vl, *Vu;            /* [P][R][K] */
    const double *Kl, *Ku;            /* [P][R][V] */
    int Pl_t, Pu_t, Rl_t, Ru_t, Ll_t, Lu_t, Vl_t, Vu_t, Kl_t, Ku_t;
    int run_convection, run_radial, run_local;
    int radial_sources, local_sources;
    int include_boundary, positive_psd;
    double *lu;                       /* P*R*ldab*V*K doubles, or NULL for no caching */
    long *ipiv;                       /* P*R*V*K */
} orc_state;

long orc_step(orc_state* st, double dt, double sub_dt, int recompute_lu);

#ifdef __cplusplus
}
#endif
#endif
