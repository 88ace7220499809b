/*
 * verb4d_dropin.hpp -- the reference's per-slice C++ routines, with their exact
 * signatures, running on the B200 through libverb4d_b200.so.
 *
 * A maintainer links verb-4d_b200/dropin/verb4d_dropin.cpp and
 * libverb4d_b200.so into the reference driver in place of the reference's
 * Diffusion_1D.cpp, Diffusion_2D.cpp, Convection_2D.cpp,
 * Convection_1D_ULTIMATE_QUICKEST6.cpp and MatrixSolver.cpp's tridag; the
 * driver's OpenMP loops (src/VERB4D_Solver.cpp:851-978, 990-1070, 1081-1216)
 * then run unchanged, one slice per call.  Include it with the reference's
 * src/ directory on the include path (it uses the reference's Matrix1D /
 * Matrix2D containers and BoundaryConditionType).
 *
 * Semantics follow the reference: the routines return true, psd is updated in
 * place, and every error (Courant number > 1, a singular pivot, an unknown
 * boundary type, a line shorter than 11 points) ends the process through
 * Logger::error and exit(EXIT_FAILURE), as the reference does
 * (src/Logger.cpp:45-55, src/MatrixSolver.cpp:273-276,
 * src/Convection_1D_ULTIMATE_QUICKEST6.cpp:48-52).  The batched context of
 * verb4d_b200.h is the fast path; these per-slice calls copy one slice to the
 * device and back and are meant for parity and incremental adoption.
 */
#ifndef VERB4D_DROPIN_HPP
#define VERB4D_DROPIN_HPP

#include <cstddef>

#include "BoundaryConditionType.hpp"
#include "Matrix.h"

/* src/MatrixSolver.h:240 -- Thomas algorithm, u = A^-1 r for the tridiagonal
 * A with sub-diagonal a, diagonal b and super-diagonal c. */
bool tridag(double a[], double b[], double c[], double r[], double u[], size_t n);

/* src/Diffusion_1D.h:69-77 -- one radial line. */
bool Diffusion_1D(Matrix1D<double>& psd, const Matrix1D<double>& x, int x_size, double x_LBC,
                  double x_UBC, BoundaryConditionType x_LBC_type,
                  BoundaryConditionType x_UBC_type, const Matrix1D<double>& Dxx,
                  const Matrix1D<double>& G, const Matrix1D<double>& Sources,
                  const Matrix1D<double>& Losses, double dt);

/* src/Diffusion_2D.h:86-111 -- one local (V,K) system, both builds: the plain
 * form factors every call; the LU_CACHING form reads the caller's cache slot
 * (LAPACK band layout, 1-based pivots) or, with recompute_lu, writes it. */
bool Diffusion_2D(Matrix2D<double>& psd, const Matrix2D<double>& x, const Matrix2D<double>& y,
                  int x_size, int y_size, const Matrix1D<double>& x_LBC,
                  const Matrix1D<double>& x_UBC, const Matrix1D<double>& y_LBC,
                  const Matrix1D<double>& y_UBC, BoundaryConditionType x_LBC_type,
                  BoundaryConditionType x_UBC_type, BoundaryConditionType y_LBC_type,
                  BoundaryConditionType y_UBC_type, const Matrix2D<double>& Dxx,
                  const Matrix2D<double>& Dyy, const Matrix2D<double>& Dxy,
                  const Matrix2D<double>& Dyx, const Matrix2D<double>& G,
                  const Matrix2D<double>& Sources, const Matrix2D<double>& Losses, double dt,
                  double sub_dt, double* lu_cache, long* index_cache, bool recompute_lu);
bool Diffusion_2D(Matrix2D<double>& psd, const Matrix2D<double>& x, const Matrix2D<double>& y,
                  int x_size, int y_size, const Matrix1D<double>& x_LBC,
                  const Matrix1D<double>& x_UBC, const Matrix1D<double>& y_LBC,
                  const Matrix1D<double>& y_UBC, BoundaryConditionType x_LBC_type,
                  BoundaryConditionType x_UBC_type, BoundaryConditionType y_LBC_type,
                  BoundaryConditionType y_UBC_type, const Matrix2D<double>& Dxx,
                  const Matrix2D<double>& Dyy, const Matrix2D<double>& Dxy,
                  const Matrix2D<double>& Dyx, const Matrix2D<double>& G,
                  const Matrix2D<double>& Sources, const Matrix2D<double>& Losses, double dt,
                  double sub_dt);

/* src/Convection_2D.h:98-108 -- one [P][R] slice. */
bool Convection_2D(Matrix2D<double>& PSD_PR, const Matrix2D<double>& P,
                   const Matrix2D<double>& R, int P_size, int R_size,
                   const Matrix1D<double>& P_LBC, const Matrix1D<double>& P_UBC,
                   const Matrix1D<double>& R_LBC, const Matrix1D<double>& R_UBC,
                   BoundaryConditionType P_LBC_type, BoundaryConditionType P_UBC_type,
                   BoundaryConditionType R_LBC_type, BoundaryConditionType R_UBC_type,
                   const Matrix2D<double>& VP, const Matrix2D<double>& VR,
                   const Matrix2D<double>& Sources, const Matrix2D<double>& Losses,
                   const Matrix2D<double>& G_conv, double dt_total);

/* src/Convection_1D_ULTIMATE_QUICKEST6.h:71-79 -- one line. */
bool Convection_1D_ULTIMATE_QUICKEST6(Matrix1D<double>& PSD, const Matrix1D<double>& x,
                                      int x_size, double x_LBC, double x_UBC,
                                      BoundaryConditionType x_LBC_type,
                                      BoundaryConditionType x_UBC_type,
                                      const Matrix1D<double>& Ux, double dt_total);

#endif /* VERB4D_DROPIN_HPP */
