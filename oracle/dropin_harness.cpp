// extern "C" harness around the C++ drop-in layer (include/verb4d_dropin.hpp,
// verb-4d_b200/dropin/verb4d_dropin.cpp) -- TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles the drop-in and this harness against the
// reference's own Matrix.h, BoundaryConditionType.hpp and Logger.h (read in
// place from the reference tree), links them with the reference's Matrix and
// Logger code and libverb4d_b200.so into oracle/_ref/libverbdropin.so.  The
// entry points mirror those of oracle/ref_shim.cpp (plain row-major arrays in,
// the reference's Matrix containers built from them, the routine called, the
// result copied back), so a test calls the drop-in and the reference routine
// on the same Matrix objects' contents and compares.
#include <cstring>

#include "verb4d_dropin.hpp"

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

int drop_tridag(double* a, double* b, double* c, double* r, double* u, long n)
{
    return tridag(a, b, c, r, u, static_cast<size_t>(n)) ? 0 : 1;
}

int drop_diffusion_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                      int ubc_t, const double* D, const double* G, const double* S,
                      const double* loss, double dt)
{
    Matrix1D<double> f = vec(psd, n);
    Diffusion_1D(f, vec(x, n), n, lbc, ubc, bct(lbc_t), bct(ubc_t), vec(D, n), vec(G, n),
                 vec(S, n), vec(loss, n), dt);
    std::memcpy(psd, &f[0], sizeof(double) * n);
    return 0;
}

int drop_diffusion_2d(double* psd, const double* x, const double* y, int nx, int ny,
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

int drop_diffusion_2d_lu(double* psd, const double* x, const double* y, int nx, int ny,
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

int drop_convection_1d(double* psd, const double* x, int n, double lbc, double ubc, int lbc_t,
                       int ubc_t, const double* ux, double dt)
{
    Matrix1D<double> f = vec(psd, n);
    Convection_1D_ULTIMATE_QUICKEST6(f, vec(x, n), n, lbc, ubc, bct(lbc_t), bct(ubc_t), vec(ux, n),
                                     dt);
    std::memcpy(psd, &f[0], sizeof(double) * n);
    return 0;
}

int drop_convection_2d(double* psd, const double* P, const double* R, int nP, int nR,
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

}  // extern "C"
