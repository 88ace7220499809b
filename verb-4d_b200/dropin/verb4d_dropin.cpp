// The reference's per-slice routines (include/verb4d_dropin.hpp) over the C
// ABI of libverb4d_b200.so.  Each one passes the Matrix containers' contiguous
// storage (row-major, as the reference lays them out: src/Matrix.h:152-179)
// to the matching per-slice entry point and turns a non-OK status into the
// reference's failure path, Logger::error and exit(EXIT_FAILURE).
#include "verb4d_dropin.hpp"

#include <cstdlib>
#include <iostream>

#include "Logger.h"
#include "verb4d_b200.h"

namespace {

// The reference aborts the run at every error site (src/Logger.cpp:45-55).
bool ok_or_exit(int status, const char* routine)
{
    if (status == VERB_OK) return true;
    Logger::error << routine << ": " << verb_status_string(status) << std::endl;
    std::exit(EXIT_FAILURE);
}

int bc(BoundaryConditionType t) { return static_cast<int>(t); }

const double* p1(const Matrix1D<double>& m) { return &m[0]; }
const double* p2(const Matrix2D<double>& m) { return m[0]; }

}  // namespace

bool tridag(double a[], double b[], double c[], double r[], double u[], size_t n)
{
    return ok_or_exit(verb_tridag(a, b, c, r, u, static_cast<long>(n)), "tridag");
}

bool Diffusion_1D(Matrix1D<double>& psd, const Matrix1D<double>& x, int x_size, double x_LBC,
                  double x_UBC, BoundaryConditionType x_LBC_type,
                  BoundaryConditionType x_UBC_type, const Matrix1D<double>& Dxx,
                  const Matrix1D<double>& G, const Matrix1D<double>& Sources,
                  const Matrix1D<double>& Losses, double dt)
{
    return ok_or_exit(verb_diffusion_1d(&psd[0], p1(x), x_size, x_LBC, x_UBC, bc(x_LBC_type),
                                        bc(x_UBC_type), p1(Dxx), p1(G), p1(Sources), p1(Losses),
                                        dt),
                      "Diffusion_1D");
}

bool Diffusion_2D(Matrix2D<double>& psd, const Matrix2D<double>& x, const Matrix2D<double>& y,
                  int x_size, int y_size, const Matrix1D<double>& x_LBC,
                  const Matrix1D<double>& x_UBC, const Matrix1D<double>& y_LBC,
                  const Matrix1D<double>& y_UBC, BoundaryConditionType x_LBC_type,
                  BoundaryConditionType x_UBC_type, BoundaryConditionType y_LBC_type,
                  BoundaryConditionType y_UBC_type, const Matrix2D<double>& Dxx,
                  const Matrix2D<double>& Dyy, const Matrix2D<double>& Dxy,
                  const Matrix2D<double>& Dyx, const Matrix2D<double>& G,
                  const Matrix2D<double>& Sources, const Matrix2D<double>& Losses, double dt,
                  double sub_dt, double* lu_cache, long* index_cache, bool recompute_lu)
{
    return ok_or_exit(
        verb_diffusion_2d(psd[0], p2(x), p2(y), x_size, y_size, p1(x_LBC), p1(x_UBC), p1(y_LBC),
                          p1(y_UBC), bc(x_LBC_type), bc(x_UBC_type), bc(y_LBC_type),
                          bc(y_UBC_type), p2(Dxx), p2(Dyy), p2(Dxy), p2(Dyx), p2(G), p2(Sources),
                          p2(Losses), dt, sub_dt, lu_cache, index_cache, recompute_lu ? 1 : 0),
        "Diffusion_2D");
}

bool Diffusion_2D(Matrix2D<double>& psd, const Matrix2D<double>& x, const Matrix2D<double>& y,
                  int x_size, int y_size, const Matrix1D<double>& x_LBC,
                  const Matrix1D<double>& x_UBC, const Matrix1D<double>& y_LBC,
                  const Matrix1D<double>& y_UBC, BoundaryConditionType x_LBC_type,
                  BoundaryConditionType x_UBC_type, BoundaryConditionType y_LBC_type,
                  BoundaryConditionType y_UBC_type, const Matrix2D<double>& Dxx,
                  const Matrix2D<double>& Dyy, const Matrix2D<double>& Dxy,
                  const Matrix2D<double>& Dyx, const Matrix2D<double>& G,
                  const Matrix2D<double>& Sources, const Matrix2D<double>& Losses, double dt,
                  double sub_dt)
{
    // the plain build: no cache slot, the factorisation runs every call
    return ok_or_exit(
        verb_diffusion_2d(psd[0], p2(x), p2(y), x_size, y_size, p1(x_LBC), p1(x_UBC), p1(y_LBC),
                          p1(y_UBC), bc(x_LBC_type), bc(x_UBC_type), bc(y_LBC_type),
                          bc(y_UBC_type), p2(Dxx), p2(Dyy), p2(Dxy), p2(Dyx), p2(G), p2(Sources),
                          p2(Losses), dt, sub_dt, nullptr, nullptr, 0),
        "Diffusion_2D");
}

bool Convection_2D(Matrix2D<double>& PSD_PR, const Matrix2D<double>& P,
                   const Matrix2D<double>& R, int P_size, int R_size,
                   const Matrix1D<double>& P_LBC, const Matrix1D<double>& P_UBC,
                   const Matrix1D<double>& R_LBC, const Matrix1D<double>& R_UBC,
                   BoundaryConditionType P_LBC_type, BoundaryConditionType P_UBC_type,
                   BoundaryConditionType R_LBC_type, BoundaryConditionType R_UBC_type,
                   const Matrix2D<double>& VP, const Matrix2D<double>& VR,
                   const Matrix2D<double>& Sources, const Matrix2D<double>& Losses,
                   const Matrix2D<double>& G_conv, double dt_total)
{
    return ok_or_exit(
        verb_convection_2d(PSD_PR[0], p2(P), p2(R), P_size, R_size, p1(P_LBC), p1(P_UBC),
                           p1(R_LBC), p1(R_UBC), bc(P_LBC_type), bc(P_UBC_type), bc(R_LBC_type),
                           bc(R_UBC_type), p2(VP), p2(VR), p2(Sources), p2(Losses), p2(G_conv),
                           dt_total),
        "Convection_2D");
}

bool Convection_1D_ULTIMATE_QUICKEST6(Matrix1D<double>& PSD, const Matrix1D<double>& x,
                                      int x_size, double x_LBC, double x_UBC,
                                      BoundaryConditionType x_LBC_type,
                                      BoundaryConditionType x_UBC_type,
                                      const Matrix1D<double>& Ux, double dt_total)
{
    return ok_or_exit(verb_convection_1d(&PSD[0], p1(x), x_size, x_LBC, x_UBC, bc(x_LBC_type),
                                         bc(x_UBC_type), p1(Ux), dt_total),
                      "Convection_1D_ULTIMATE_QUICKEST6");
}
