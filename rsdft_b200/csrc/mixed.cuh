// Mixed-precision contractions of the Gram-Schmidt and subspace steps on the
// tcgen05 tensor cores (split-BF16 operands, FP32 accumulation, FP64 result).
#pragma once

#include "common.cuh"

namespace rsdft {

// C (nb x nb) = alpha A^T B (symmetrize: alpha/2 (A^T B + B^T A)) for tall A,
// B (ML x nb, leading dimension ld).  nterms = 3 (six products) or 2 (three).
// a_split, if given, receives the BF16 split of A (valid until the next
// mixed Gram product), which a rotation of A can reuse.
int gram_mixed(const double* A, const double* B, long ld, int nb, double alpha, int symmetrize, int nterms,
               double* C, const void** a_split = nullptr);

// S = alpha psi^T psi and H = alpha psi^T Hpsi from one split of each
// operand, for a symmetric operator (psi^T Hpsi symmetric): only the tile
// pairs on and above the diagonal are formed, the lower ones mirrored and the
// diagonal tiles symmetrised.  psi_split as a_split above.
int gram_mixed_pair(const double* psi, const double* hpsi, long ld, int nb, double alpha, int nterms, double* S,
                    double* H, const void** psi_split = nullptr);
// the same from FP32 blocks (the split of an FP32 value is exact)
int gram_mixed_pair(const float* psi, const float* hpsi, long ld, int nb, double alpha, int nterms, double* S,
                    double* H, const void** psi_split = nullptr);

// out (ML x nb, leading dimension ld) = psi V with V (nb x nb, leading
// dimension ldv).  psi is read only through its BF16 split, so out may be
// psi itself.  psi_split: the split of psi left by a Gram product, used
// directly (no transposed copy) when ML is a multiple of 32.
int rotate_mixed(const double* psi, double* out, long ld, int nb, const double* V, int ldv, int nterms,
                 const void* psi_split = nullptr);
// the same with an FP32 psi (FP64 out)
int rotate_mixed(const float* psi, double* out, long ld, int nb, const double* V, int ldv, int nterms,
                 const void* psi_split = nullptr);

inline int mode_terms(int mode) { return mode == RSDFT_MODE_MIXED_BF16X3 ? 3 : 2; }

}  // namespace rsdft
