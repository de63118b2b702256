// Mixed-precision contractions (tensor cores).  Not built yet: every entry
// reports RSDFT_EUNSUP so callers see the gap instead of a silent fallback.
#include "mixed.cuh"

namespace rsdft {

int cholqr_mixed(double*, long, int, int, double*, int*) {
    set_error("mixed-precision Gram-Schmidt is not available in this build");
    return RSDFT_EUNSUP;
}

int subspace_matrix_mixed(const double*, double*, long, int, int, int, double*) {
    set_error("mixed-precision subspace matrix is not available in this build");
    return RSDFT_EUNSUP;
}

int rotate_mixed(const double*, double*, long, int, const double*, int) {
    set_error("mixed-precision rotation is not available in this build");
    return RSDFT_EUNSUP;
}

}  // namespace rsdft
