// Mixed-precision contractions of the Gram-Schmidt and subspace steps.
#pragma once

#include "common.cuh"

namespace rsdft {

// One CholeskyQR pass with the Gram matrix and the triangular update on the
// tensor cores (split-BF16 or FP32), Cholesky in FP64.  S: nb x nb scratch.
int cholqr_mixed(double* psi, long ld, int nb, int mode, double* S, int* dinfo);

// H = dV/2 (psi^T H psi + (H psi)^T psi) with H psi written to hpsi.
int subspace_matrix_mixed(const double* psi, double* hpsi, long ld, int mb, int spin, int mode, double* H);

// out = psi V (ML x MB by MB x MB).
int rotate_mixed(const double* psi, double* out, long ld, int mb, const double* V, int mode);

}  // namespace rsdft
