// FP64 tensor-core (DMMA) contractions of the plain form: dmma.cu.
#pragma once

namespace rsdft {

// C (m x n, column-major, leading dimension ldc) = alpha A^T B for tall A
// (kdim x m) and B (kdim x n), column-major with leading dimension ld;
// split-K over kdim, partial tiles added in a fixed order.  symmetrize: C =
// alpha/2 (A^T B + B^T A).  A == B, or symmetric_product with symmetrize
// (B = H A for a symmetric operator H, so A^T B is symmetric up to
// rounding), forms only the tiles on and above the diagonal: lower tiles are
// mirrored, diagonal tiles symmetrised.
int dmma_gram(const double* A, const double* B, long ld, long kdim, int m, int n, double alpha, int symmetrize,
              double* C, long ldc, bool symmetric_product = false);

// C = alpha op(A) B + beta C, column-major; op(A) = A (transA false) or A^T,
// m x k; B k x n; C m x n.  C must not overlap A or B.
int dmma_gemm(bool transA, long m, int n, int k, double alpha, const double* A, long lda, const double* B, long ldb,
              double beta, double* C, long ldc);

}  // namespace rsdft
