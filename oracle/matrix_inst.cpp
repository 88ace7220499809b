// Compiles the reference's Matrix.cpp (read in place, include path set by
// oracle/Makefile) and adds the one explicit instantiation that file omits:
// Matrix3D<bool>::~Matrix3D, referenced by UpdatableMatrix.  Test
// infrastructure for the oracle build only.
#include "Matrix.cpp"

template Matrix3D<bool>::~Matrix3D();
