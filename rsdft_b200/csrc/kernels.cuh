// Internal (C++) entry points shared between the library's translation units.
#pragma once

#include "common.cuh"

namespace rsdft {

// H psi for nb bands of leading dimension ld (device pointers).  Bands with
// band_active[b] == 0 are skipped (output left untouched).
template <typename T>
int hpsi_device(const T* psi, T* hpsi, long ld, int nb, int spin, const int* band_active);

// Deterministic block sum (fixed shuffle tree + fixed warp order).  All
// threads of the block must call it; the result is valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh /* >= NT/32 doubles */) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NT / 32; ++i) r += sh[i];
    }
    __syncthreads();
    return r;
}

// K deterministic block sums with one pair of barriers; results valid in
// thread 0.  sh holds K * NT / 32 doubles.
template <int NT, int K>
__device__ __forceinline__ void block_sum_n(double (&v)[K], double* sh) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], s);
        if (l == 0) sh[k * (NT / 32) + w] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double r = 0.0;
#pragma unroll
            for (int i = 0; i < NT / 32; ++i) r += sh[k * (NT / 32) + i];
            v[k] = r;
        }
    }
    __syncthreads();
}

// Symmetric-positive-definite orthonormalisation (CholeskyQR2 in the dV
// metric) of nb columns, FP64 (DMMA Gram and rotation, the Cholesky factor
// and its inverse by factor.cu) or mixed (tcgen05 tensor cores).
int gram_schmidt_device(double* psi, long ld, int nb, int mode);

// Rayleigh-Ritz (subspace_diag_la) on device data.
int subspace_diag_device(double* psi, long ld, int mb, int spin, double* esp_dev, int mode);

// Gram-Schmidt + Rayleigh-Ritz as one step (device data).  hpsi, when
// given, is H psi already formed (leading dimension ld); else it is formed
// here.
int orth_subspace_diag_device(double* psi, long ld, int mb, int spin, double* esp_dev, int mode,
                              const double* hpsi_in = nullptr);

// One calc_sweep step for spin `spin` on device bands: conjugate_gradient,
// then gram_schmidt + subspace_diag as one Rayleigh-Ritz step; W, R receive
// the Ritz values and CG residuals (device, mb each).
int sweep_device(double* d, long ld, int mb, int spin, double* W, double* R, int ncg, int mloop, int ipc, int mode);

// Mixed forms: the CG sweep on an FP32 copy of unk, left in the workspace
// (*x32_out, leading dimension ld) for orth_subspace_diag_f32.  hx_out (if
// given) receives the sweep's H x32 (in the CG workspace), or null when an
// update was rejected and H x must be formed again.
int cg_device_f32(const double* unk, long ld, int mb, int spin, double* esp, double* res, int ncg, int mloop,
                  int ipc, float** x32_out, const float** hx_out = nullptr);

// The same sweep on a host array: unk_host is uploaded to unk_dev in nchunk
// band blocks on the copy stream, and the CG of each block starts as soon as
// its upload lands (the bands' CG steps are independent), so the upload of
// later blocks overlaps the CG of earlier ones.
int cg_device_f32_staged(const double* unk_host, double* unk_dev, long ld, int mb, int spin, double* esp,
                         double* res, int ncg, int mloop, int ipc, int nchunk, float** x32_out,
                         const float** hx_out);

// Gram-Schmidt + Rayleigh-Ritz of FP32 bands x32 (h32 = H x32 if already
// known, else null); the rotated bands are written to psi (FP64).  Mixed
// forms only.
int orth_subspace_diag_f32(const float* x32, const float* h32, double* psi, long ld, int mb, int spin,
                           double* esp_dev, int mode);

// Eigen-decomposition of the symmetric n x n A (column-major, ld n; the
// `uplo` triangle is read): W ascending, A overwritten by the eigenvectors.
// Cluster-resident tridiagonalisation + bisection / inverse iteration +
// the compact-WY back-transformation of factor.cu; RSDFT_EUNSUP when n is
// outside its range (n < 3, or the rows do not fit the cluster's shared
// memory) or 16-CTA clusters are not available, so the caller takes
// cuSOLVER's syevd.
int syevd_fast(double* A, int n, double* W, cublasFillMode_t uplo);

// C (n x n, ld n) <- Q C for the Q of a lower Householder tridiagonalisation
// (reflectors below the subdiagonal of Q's columns, scalars tau; LAPACK
// dormtr with side 'L', uplo 'L', trans 'N'), factor.cu; the dynamic shared
// memory it needs for n (RSDFT_EUNSUP above the device's limit).
int ormtr_lower_device(const double* Q, const double* tau, int n, double* C);
size_t ormtr_smem_bytes(int n);

// S (n x n, column-major, ld n) = R^T R in place, R in the upper triangle
// (LAPACK dpotrf, uplo 'U'; the strictly lower triangle untouched); dinfo
// (device) receives dpotrf's info.  factor.cu.
int potrf_upper_device(double* S, int n, int* dinfo);

// X = R^-1 for the upper-triangular R (n x n, column-major, ld n; X's lower
// triangle zero), factor.cu; RSDFT_EUNSUP when the staged rows do not fit
// shared memory (n above ~1700).
int trtri_upper_device(const double* R, int n, double* X);

// CG over all bands (device data).  hx_out (FP64 only, if given) receives
// the sweep's H x (in the CG workspace), or null when an update was rejected
// and H x must be formed again.
int cg_device(double* unk, long ld, int mb, int spin, double* esp_dev, double* res_dev, int ncg, int mloop,
              int ipc, int mode, const double** hx_out = nullptr);

}  // namespace rsdft
