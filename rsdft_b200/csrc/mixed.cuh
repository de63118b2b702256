// Mixed-precision contractions of the Gram-Schmidt and subspace steps on the
// tcgen05 tensor cores (split-BF16 or split-TF32 operands, FP32
// accumulation, FP64 result).
#pragma once

#include "common.cuh"

namespace rsdft {

// C (nb x nb) = alpha A^T B (symmetrize: alpha/2 (A^T B + B^T A)) for tall A,
// B (ML x nb, leading dimension ld), in the operand split of `mode` (3 BF16
// terms: six products; 2 BF16 or 2 TF32 terms: three).  a_split, if given,
// receives the split of A (valid until the next mixed Gram product), which a
// rotation of A can reuse.
int gram_mixed(const double* A, const double* B, long ld, int nb, double alpha, int symmetrize, int mode,
               double* C, const void** a_split = nullptr);

// S = alpha psi^T psi and H = alpha psi^T Hpsi from one split of each
// operand, for a symmetric operator (psi^T Hpsi symmetric): only the tile
// pairs on and above the diagonal are formed, the lower ones mirrored and the
// diagonal tiles symmetrised.  psi_split as a_split above.
int gram_mixed_pair(const double* psi, const double* hpsi, long ld, int nb, double alpha, int mode, double* S,
                    double* H, const void** psi_split = nullptr);
// the same from FP32 blocks (three BF16 terms hold an FP32 value exactly)
int gram_mixed_pair(const float* psi, const float* hpsi, long ld, int nb, double alpha, int mode, double* S,
                    double* H, const void** psi_split = nullptr);

// out (ML x nb, leading dimension ld) = psi V with V (nb x nb, leading
// dimension ldv).  psi is read only through its split, so out may be psi
// itself.  psi_split: the BF16 split of psi left by a Gram product, used
// directly (no transposed copy) when ML is a multiple of 32; TF32 rotations
// always split psi transposed (band index fastest).
int rotate_mixed(const double* psi, double* out, long ld, int nb, const double* V, int ldv, int mode,
                 const void* psi_split = nullptr);
// the same with an FP32 psi (FP64 out)
int rotate_mixed(const float* psi, double* out, long ld, int nb, const double* V, int ldv, int mode,
                 const void* psi_split = nullptr);

// Operand split of a mixed mode: the number of terms and their type.
struct Split {
    int terms;  // 3 or 2
    bool tf32;  // TF32 terms (kind::tf32) instead of BF16 (kind::f16)
};
inline Split mode_split(int mode) {
    return Split{mode == RSDFT_MODE_MIXED_BF16X3 ? 3 : 2, mode == RSDFT_MODE_MIXED_TF32};
}

}  // namespace rsdft
