// Dense tall-skinny steps of the eigensolver iteration.
//
// Gram-Schmidt (gram_schmidt_t_module.f90:84-316) is a recursive blocked
// classical Gram-Schmidt in the dV metric.  Its output is the unique Q of
// psi = Q R with dV Q^T Q = I and diag(R) > 0.  CholeskyQR2 computes the same
// Q from one Gram matrix, one Cholesky factor and one triangular solve per
// pass (two passes): all the work is in two tall-skinny BLAS-3 calls.
//
// Subspace diagonalisation follows subspace_diag_la (subspace_diag_la_module
// .f90:18-232): Hsub = dV/2 (psi^T H psi + (H psi)^T psi) (dsyr2k), symmetric
// eigen-decomposition (syevd) and the rotation psi V (dgemm).  The mate /
// solv / rotv entries cover the ScaLAPACK route on a 1x1 process grid
// (subspace_mate_sl, subspace_solv_sl, subspace_rotv_sl).
//
// FP64 form: the Gram matrices and rotations on the FP64 tensor pipe
// (dmma.cu), the overlap's Cholesky factor and its inverse by the tile-step
// and staged-column kernels of factor.cu, the eigensolve in eigen.cu
// (cuSOLVER DSYEVD only above its shared-memory limit).  Mixed forms: the contractions go to the split-BF16 /
// split-TF32 tensor-core kernels of mixed.cu; FP64 stays in the Cholesky
// factor, its inverse and the eigensolve.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "dmma.cuh"
#include "mixed.cuh"

namespace rsdft {

__global__ void k_zero_upper(double* a, int n, int lda) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;  // row
    int j = blockIdx.y;                              // column
    if (i < n && i < j) a[(long)j * lda + i] = 0.0;
}

__global__ void k_widen(const float* __restrict__ a, double* __restrict__ b, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

// C = alpha * sum_c P[c] (sym: alpha/2 (G + G^T)), fixed summation order
__global__ void k_reduce_partials(const double* __restrict__ P, int nch, int m, int n, double alpha, int sym,
                                  double* __restrict__ C) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= m) return;
    const long mn = (long)m * n;
    double s = 0.0;
    for (int c = 0; c < nch; ++c) s += P[c * mn + (long)j * m + i];
    if (sym) {
        double t = 0.0;
        for (int c = 0; c < nch; ++c) t += P[c * mn + (long)i * m + j];
        s = 0.5 * (s + t);
    }
    C[(long)j * m + i] = alpha * s;
}

// C (m x n) = alpha A^T B with A, B tall (ML rows, leading dimension ld) on
// the FP64 tensor cores (dmma.cu): split-K over the grid, partial tiles
// reduced in a fixed order.  sym = 1 returns the symmetric part.
// sym_op: B = H A with H symmetric, so only the upper tiles are formed.
static int gemm_tn_splitk(const double* A, const double* B, long ld, int m, int n, double alpha, int sym,
                          double* C, bool sym_op = false) {
    return dmma_gram(A, B, ld, ctx().ml, m, n, alpha, sym, C, m, sym_op);
}

static int check_info(int* dinfo, const char* what) {
    int h = 0;
    RS_CUDA(cudaMemcpyAsync(&h, dinfo, sizeof(int), cudaMemcpyDeviceToHost, ctx().stream));
    RS_CUDA(cudaStreamSynchronize(ctx().stream));
    if (h != 0) {
        set_error("%s: info=%d", what, h);
        return RSDFT_ESOLVER;
    }
    return RSDFT_OK;
}

// S (nb x nb) = R^T R in place: the upper triangle becomes R
// (check = false: the caller reads *dinfo back itself, with its next read)
static int potrf_upper(double* S, int nb, int* dinfo, const char* what, bool check = true) {
    RS_CHECK(potrf_upper_device(S, nb, dinfo));
    return check ? check_info(dinfo, what) : RSDFT_OK;
}

// One read-back of the Cholesky status and of diag(R)'s min and max (the
// spread that picks the one-step Rayleigh-Ritz or the explicit path).
static int read_cholesky(const int* dinfo, const double* mm, double* hmm, const char* what) {
    Context& c = ctx();
    int info = 0;
    RS_CUDA(cudaMemcpyAsync(hmm, mm, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    if (info != 0) {
        set_error("%s: info=%d", what, info);
        return RSDFT_ESOLVER;
    }
    return RSDFT_OK;
}

// X = R^-1 for the upper triangular R (n x n, column-major, leading
// dimension n), X R = I read row by row: one warp per row i of X,
//   X(i, j) = 0 (j < i),  X(i, i) = 1 / R(i, i),
//   X(i, j) = -(sum_{l=i}^{j-1} X(i, l) R(l, j)) / R(j, j)   (j > i),
// each sum split over the lanes (l = i + lane, i + lane + 32, ..., then a
// fixed xor tree), the row kept in shared memory, R's columns read straight
// from global memory (each column is shared by the warps of every row).
// The callers factor R from an overlap whose Cholesky succeeded, so its
// diagonal is positive.
constexpr int TI_W = 4;  // rows (warps) per CTA

__global__ void __launch_bounds__(32 * TI_W) k_trtri_rows(const double* __restrict__ R, int n,
                                                         double* __restrict__ X) {
    extern __shared__ double ti_sm[];
    double* dinv = ti_sm;                // 1 / R(j, j)
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* xr = ti_sm + n + (size_t)w * n;  // this warp's row of X
    for (int j = threadIdx.x; j < n; j += blockDim.x) dinv[j] = 1.0 / R[(long)j * n + j];
    __syncthreads();
    const int i = blockIdx.x * TI_W + w;
    if (i >= n) return;
    for (int j = lane; j < i; j += 32) X[(long)j * n + i] = 0.0;
    if (lane == 0) {
        xr[i] = dinv[i];
        X[(long)i * n + i] = dinv[i];
    }
    __syncwarp();
    for (int j = i + 1; j < n; ++j) {
        const double* rc = R + (long)j * n;
        double s = 0.0;
        for (int l = i + lane; l < j; l += 32) s = fma(xr[l], rc[l], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            const double v = -s * dinv[j];
            xr[j] = v;
            X[(long)j * n + i] = v;
        }
        __syncwarp();
    }
}

// R (upper triangle of S) -> R^-1 in place, the lower triangle zeroed:
// trtri_upper_device (staged columns, eight columns per reduction), or for
// orders whose staged rows exceed shared memory the row-per-warp kernel above
static int trtri_upper(double* S, int nb, int* dinfo, const char* what) {
    (void)dinfo;
    (void)what;
    Context& c = ctx();
    double* X = nullptr;
    RS_CHECK(workspace_t("gs_trtri_x", (size_t)nb * nb, &X));
    const int r = trtri_upper_device(S, nb, X);
    if (r == RSDFT_EUNSUP) {
        const size_t smem = (size_t)(TI_W + 1) * nb * sizeof(double);
        RS_CHECK(set_smem_optin((const void*)k_trtri_rows, (int)smem));
        launch(k_trtri_rows, div_up(nb, TI_W), 32 * TI_W, smem, c.stream, (const double*)S, nb, X);
        RS_LAUNCH();
    } else if (r != RSDFT_OK) {
        return r;
    }
    RS_CUDA(cudaMemcpyAsync(S, X, sizeof(double) * (size_t)nb * nb, cudaMemcpyDeviceToDevice, c.stream));
    return RSDFT_OK;
}

// One CholeskyQR pass in FP64: S = dV psi^T psi = R^T R, out = psi R^-1.
// R^-1 comes from a triangular inverse of the small factor, so the tall
// product is one DGEMM (in and out are different buffers).
static int cholqr_pass(const double* psi, double* out, long ld, int nb, double* S, int* dinfo, int mode) {
    Context& c = ctx();
    const void* split = nullptr;
    if (mode == RSDFT_MODE_FP64)
        RS_CHECK(gemm_tn_splitk(psi, psi, ld, nb, nb, c.dV, 0, S));
    else
        RS_CHECK(gram_mixed(psi, psi, ld, nb, c.dV, 0, mode, S, &split));
    RS_CHECK(potrf_upper(S, nb, dinfo, "gram_schmidt: overlap Cholesky"));
    RS_CHECK(trtri_upper(S, nb, dinfo, "gram_schmidt: triangular inverse"));
    if (mode == RSDFT_MODE_FP64)
        RS_CHECK(dmma_gemm(false, c.ml, nb, nb, 1.0, psi, ld, S, nb, 0.0, out, ld));
    else
        RS_CHECK(rotate_mixed(psi, out, ld, nb, S, nb, mode, split));
    return RSDFT_OK;
}

int gram_schmidt_device(double* psi, long ld, int nb, int mode) {
    double* S = nullptr;
    int* dinfo = nullptr;
    double* tmp = nullptr;
    RS_CHECK(workspace_t("gs_S", (size_t)nb * nb, &S));
    RS_CHECK(workspace_t("gs_info", 4, &dinfo));
    // CholeskyQR2 as ping-pong: psi -> tmp -> psi.  Mixed forms: Gram matrix and
    // the triangular update on the tensor cores, Cholesky and the triangular
    // inverse in FP64.
    RS_CHECK(workspace_t("gs_tmp", (size_t)ld * nb, &tmp));
    RS_CHECK(cholqr_pass(psi, tmp, ld, nb, S, dinfo, mode));
    RS_CHECK(cholqr_pass(tmp, psi, ld, nb, S, dinfo, mode));
    return RSDFT_OK;
}

// symmetric eigensolve in place: A (n x n, lda n) -> eigenvectors, W ascending
static int syevd(double* A, int n, double* W, cublasFillMode_t uplo, const char* what) {
    Context& c = ctx();
    const int r = syevd_fast(A, n, W, uplo);
    if (r != RSDFT_EUNSUP) return r;
    int lwork = 0;
    RS_SOLVER(cusolverDnDsyevd_bufferSize(c.solver, CUSOLVER_EIG_MODE_VECTOR, uplo, n, A, n, W, &lwork));
    double* work = nullptr;
    int* dinfo = nullptr;
    RS_CHECK(workspace_t("syevd_work", (size_t)lwork + 1, &work));
    RS_CHECK(workspace_t("syevd_info", 4, &dinfo));
    RS_SOLVER(cusolverDnDsyevd(c.solver, CUSOLVER_EIG_MODE_VECTOR, uplo, n, A, n, W, work, lwork, dinfo));
    return check_info(dinfo, what);
}

int subspace_diag_device(double* psi, long ld, int mb, int spin, double* esp, int mode) {
    Context& c = ctx();
    double *hpsi = nullptr, *H = nullptr;
    RS_CHECK(workspace_t("sub_hpsi", (size_t)ld * mb, &hpsi));
    RS_CHECK(workspace_t("sub_H", (size_t)mb * mb, &H));
    if (mode == RSDFT_MODE_FP64) {
        RS_CHECK(hpsi_device<double>(psi, hpsi, ld, mb, spin, nullptr));
        // Hsub = dV/2 (psi^T H psi + (H psi)^T psi): the symmetric part of dV psi^T (H psi)
        RS_CHECK(gemm_tn_splitk(psi, hpsi, ld, mb, mb, c.dV, 1, H, true));
        RS_CHECK(syevd(H, mb, esp, CUBLAS_FILL_MODE_UPPER, "subspace_diag: syevd"));
        RS_CHECK(dmma_gemm(false, c.ml, mb, mb, 1.0, psi, ld, H, mb, 0.0, hpsi, ld));
    } else {
        RS_CHECK(hpsi_device<double>(psi, hpsi, ld, mb, spin, nullptr));
        const void* split = nullptr;
        RS_CHECK(gram_mixed(psi, hpsi, ld, mb, c.dV, 1, mode, H, &split));
        RS_CHECK(syevd(H, mb, esp, CUBLAS_FILL_MODE_UPPER, "subspace_diag: syevd"));
        // reads only the BF16 split of psi: written in place
        RS_CHECK(rotate_mixed(psi, psi, ld, mb, H, mb, mode, split));
        return RSDFT_OK;
    }
    RS_CUDA(cudaMemcpy2DAsync(psi, ld * sizeof(double), hpsi, ld * sizeof(double), c.ml * sizeof(double), mb,
                              cudaMemcpyDeviceToDevice, c.stream));
    return RSDFT_OK;
}

// The reduced eigenproblem of the fused Rayleigh-Ritz step: with Rinv = R^-1
// (upper) and H the symmetric Hsub, Hr = R^-T H R^-1 (T = H R^-1, then
// H = R^-T T), Hr = V diag(esp) V^T, T = R^-1 V.  H is overwritten.
static int rr_reduced(const double* Rinv, double* H, double* T, int mb, double* esp, const char* what) {
    RS_CHECK(dmma_gemm(false, mb, mb, mb, 1.0, H, mb, Rinv, mb, 0.0, T, mb));
    RS_CHECK(dmma_gemm(true, mb, mb, mb, 1.0, Rinv, mb, T, mb, 0.0, H, mb));
    RS_CHECK(syevd(H, mb, esp, CUBLAS_FILL_MODE_UPPER, what));
    return dmma_gemm(false, mb, mb, mb, 1.0, Rinv, mb, H, mb, 0.0, T, mb);
}

// min and max of the diagonal of an n x n matrix (one block)
__global__ void k_diag_minmax(const double* __restrict__ a, int n, int lda, double* __restrict__ out) {
    __shared__ double smin[256], smax[256];
    double lo = 1e300, hi = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = fabs(a[(long)i * lda + i]);
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    smin[threadIdx.x] = lo;
    smax[threadIdx.x] = hi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
            smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = smin[0];
        out[1] = smax[0];
    }
}

// Largest (max diag R / min diag R)^2 of the overlap's Cholesky factor for
// which the one-step Rayleigh-Ritz is kept.  The eigenvalue error of the
// R^-T H R^-1 form grows with the overlap's condition, and the Gram matrices'
// own error with the precision form: FP64 1e3, 3-term split-BF16 (24
// significant bits) 1e2, 2-term split-TF32 (22 bits, four times the operand
// error) 25, 2-term split-BF16 (~16 bits) 1e1 (measured: an overlap with diag
// ratio^2 93 and condition 2.4e3 gave 6.5e-4 relative eigenvalue error in the
// 2-term BF16 form, 1.7e-5 in the TF32 form, 2e-6 in the 3-term form).
static double fused_rr_kappa_max(int mode) {
    switch (mode) {
        case RSDFT_MODE_FP64: return 1e3;
        case RSDFT_MODE_MIXED_BF16X2: return 1e1;
        case RSDFT_MODE_MIXED_TF32: return 25.0;
        default: return 1e2;
    }
}

// Gram-Schmidt followed by subspace_diag (the pair calc_sweep calls,
// sweep_module.f90:152-155) as one Rayleigh-Ritz step on the CG output:
//   S = dV psi^T psi = R^T R,  H = dV sym(psi^T H psi),
//   R^-T H R^-1 = V diag(e) V^T,  psi <- psi (R^-1 V).
// psi R^-1 is the Gram-Schmidt basis (the unique positive-R QR factor), so
// the eigenpairs and the rotated bands are those of the pair, with one
// overlap Cholesky, one eigensolve and one tall rotation instead of two
// CholeskyQR passes, the eigensolve and a separate rotation.  When the
// overlap is ill-conditioned (diag(R) spread beyond fused_rr_kappa_max^(1/2); one
// Cholesky pass then loses orthogonality), the explicit CholeskyQR2 +
// subspace_diag path runs instead.
int orth_subspace_diag_device(double* psi, long ld, int mb, int spin, double* esp, int mode,
                              const double* hpsi_in) {
    Context& c = ctx();
    double *hpsi = nullptr, *S = nullptr, *H = nullptr, *T = nullptr, *mm = nullptr;
    int* dinfo = nullptr;
    RS_CHECK(workspace_t("sub_hpsi", (size_t)ld * mb, &hpsi));
    RS_CHECK(workspace_t("gs_S", (size_t)mb * mb, &S));
    RS_CHECK(workspace_t("sub_H", (size_t)mb * mb, &H));
    RS_CHECK(workspace_t("osd_T", (size_t)mb * mb, &T));
    RS_CHECK(workspace_t("osd_minmax", 2, &mm));
    RS_CHECK(workspace_t("gs_info", 4, &dinfo));
    const void* split = nullptr;
    if (!hpsi_in) RS_CHECK(hpsi_device<double>(psi, hpsi, ld, mb, spin, nullptr));
    const double* hp = hpsi_in ? hpsi_in : hpsi;
    if (mode == RSDFT_MODE_FP64) {
        RS_CHECK(gemm_tn_splitk(psi, psi, ld, mb, mb, c.dV, 0, S));
        RS_CHECK(gemm_tn_splitk(psi, hp, ld, mb, mb, c.dV, 1, H, true));
    } else {
        RS_CHECK(gram_mixed_pair(psi, hp, ld, mb, c.dV, mode, S, H, &split));
    }
    RS_CHECK(potrf_upper(S, mb, dinfo, "orth_subspace_diag: overlap Cholesky", false));
    launch(k_diag_minmax, 1, 256, 0, c.stream, S, mb, mb, mm);
    RS_LAUNCH();
    double hmm[2] = {0.0, 0.0};
    RS_CHECK(read_cholesky(dinfo, mm, hmm, "orth_subspace_diag: overlap Cholesky"));
    if (!(hmm[0] > 0.0) || (hmm[1] / hmm[0]) * (hmm[1] / hmm[0]) > fused_rr_kappa_max(mode)) {
        RS_CHECK(gram_schmidt_device(psi, ld, mb, mode));
        return subspace_diag_device(psi, ld, mb, spin, esp, mode);
    }
    RS_CHECK(trtri_upper(S, mb, dinfo, "orth_subspace_diag: triangular inverse"));
    RS_CHECK(rr_reduced(S, H, T, mb, esp, "orth_subspace_diag: syevd"));
    if (mode == RSDFT_MODE_FP64) {
        RS_CHECK(dmma_gemm(false, c.ml, mb, mb, 1.0, psi, ld, T, mb, 0.0, hpsi, ld));
        RS_CUDA(cudaMemcpy2DAsync(psi, ld * sizeof(double), hpsi, ld * sizeof(double), c.ml * sizeof(double), mb,
                                  cudaMemcpyDeviceToDevice, c.stream));
    } else {
        // the tensor-core rotation reads only the BF16 split of psi, so it
        // can write psi itself
        RS_CHECK(rotate_mixed(psi, psi, ld, mb, T, mb, mode, split));
    }
    return RSDFT_OK;
}

// The same step on the FP32 bands of a mixed CG sweep: FP32 H psi, BF16
// split from FP32 (exact), rotated bands written in FP64 to psi.  An
// ill-conditioned overlap converts x32 to psi and takes the explicit path.
int orth_subspace_diag_f32(const float* x32, const float* hx, double* psi, long ld, int mb, int spin, double* esp,
                           int mode) {
    Context& c = ctx();
    float* h32 = nullptr;
    double *S = nullptr, *H = nullptr, *T = nullptr, *mm = nullptr;
    int* dinfo = nullptr;
    RS_CHECK(workspace_t("gs_S", (size_t)mb * mb, &S));
    RS_CHECK(workspace_t("sub_H", (size_t)mb * mb, &H));
    RS_CHECK(workspace_t("osd_T", (size_t)mb * mb, &T));
    RS_CHECK(workspace_t("osd_minmax", 2, &mm));
    RS_CHECK(workspace_t("gs_info", 4, &dinfo));
    if (hx) {
        h32 = const_cast<float*>(hx);
    } else {
        RS_CHECK(workspace_t("sub_h32", (size_t)ld * mb, &h32));
        RS_CHECK(hpsi_device<float>(x32, h32, ld, mb, spin, nullptr));
    }
    const void* split = nullptr;
    RS_CHECK(gram_mixed_pair(x32, h32, ld, mb, c.dV, mode, S, H, &split));
    RS_CHECK(potrf_upper(S, mb, dinfo, "eigensolver_sweep: overlap Cholesky", false));
    launch(k_diag_minmax, 1, 256, 0, c.stream, S, mb, mb, mm);
    RS_LAUNCH();
    double hmm[2] = {0.0, 0.0};
    RS_CHECK(read_cholesky(dinfo, mm, hmm, "eigensolver_sweep: overlap Cholesky"));
    if (!(hmm[0] > 0.0) || (hmm[1] / hmm[0]) * (hmm[1] / hmm[0]) > fused_rr_kappa_max(mode)) {
        launch(k_widen, 4 * c.num_sms, 256, 0, c.stream, x32, psi, ld * (long)mb);
        RS_LAUNCH();
        RS_CHECK(gram_schmidt_device(psi, ld, mb, mode));
        return subspace_diag_device(psi, ld, mb, spin, esp, mode);
    }
    RS_CHECK(trtri_upper(S, mb, dinfo, "eigensolver_sweep: triangular inverse"));
    RS_CHECK(rr_reduced(S, H, T, mb, esp, "eigensolver_sweep: syevd"));
    return rotate_mixed(x32, psi, ld, mb, T, mb, mode, split);
}

}  // namespace rsdft

namespace rsdft {

int sweep_device(double* d, long ld, int mb, int s, double* W, double* R, int ncg, int mloop, int ipc, int mode) {
    if (mode == RSDFT_MODE_FP64) {
        // the CG's H x goes on to the Rayleigh-Ritz step, as in the mixed
        // forms below
        const double* hx = nullptr;
        RS_CHECK(cg_device(d, ld, mb, s, W, R, ncg, mloop, ipc, mode, &hx));
        return orth_subspace_diag_device(d, ld, mb, s, W, mode, hx);
    }
    float* x32 = nullptr;
    const float* hx = nullptr;
    RS_CHECK(cg_device_f32(d, ld, mb, s, W, R, ncg, mloop, ipc, &x32, &hx));
    return orth_subspace_diag_f32(x32, hx, d, ld, mb, s, W, mode);
}

}  // namespace rsdft

using namespace rsdft;

static int check_k_s(int k, int s, const char* who) {
    if (k != 1) {
        set_error("%s: only k=1 (Gamma) is supported", who);
        return RSDFT_EUNSUP;
    }
    if (s < 1 || s > ctx().nspin) {
        set_error("%s: s=%d outside 1..%d", who, s, ctx().nspin);
        return RSDFT_EINVAL;
    }
    return RSDFT_OK;
}

extern "C" {

int rsdft_gpu_gram_schmidt(int n0, int n1, int k, int s, double* unk, long ld, int nblk, int nblk1, int mode) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    (void)nblk;
    (void)nblk1;
    (void)s;
    Context& c = ctx();
    if (k != 1) {
        set_error("gram_schmidt: only k=1 (Gamma) is supported");
        return RSDFT_EUNSUP;
    }
    const int nb = n1 - n0 + 1;
    if (n0 < 1 || nb < 1 || ld < c.ml || !unk || !mode_valid(mode)) {
        set_error("gram_schmidt: bad arguments (n0=%d n1=%d ld=%ld)", n0, n1, ld);
        return RSDFT_EINVAL;
    }
    if (nb > c.ml) {
        set_error("gram_schmidt: %d bands exceed %ld grid points", nb, c.ml);
        return RSDFT_EINVAL;
    }
    double* base = unk + (long)(n0 - 1) * ld;
    double* d;
    bool st;
    RS_CHECK(wf_acquire(base, ld, nb, "gs_unk", &d, &st));
    RS_CHECK(gram_schmidt_device(d, ld, nb, mode));
    RS_CHECK(wf_release(base, d, ld, nb, st));
    return RSDFT_OK;
}

int rsdft_gpu_subspace_mate(int k, int s, const double* unk, long ld, int mb, double* hsub, int ldh) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    RS_CHECK(check_k_s(k, s, "subspace_mate"));
    Context& c = ctx();
    if (ld < c.ml || mb < 1 || ldh < mb || !hsub) {
        set_error("subspace_mate: bad arguments");
        return RSDFT_EINVAL;
    }
    double *d, *hpsi, *H;
    bool st;
    RS_CHECK(wf_acquire(unk, ld, mb, "mate_unk", &d, &st));
    RS_CHECK(workspace_t("sub_hpsi", (size_t)ld * mb, &hpsi));
    RS_CHECK(workspace_t("sub_H", (size_t)mb * mb, &H));
    RS_CHECK(hpsi_device<double>(d, hpsi, ld, mb, s, nullptr));
    RS_CHECK(gemm_tn_splitk(d, hpsi, ld, mb, mb, c.dV, 0, H));
    launch(k_zero_upper, dim3(div_up(mb, 128), mb), 128, 0, c.stream, H, mb, mb);
    RS_LAUNCH();
    RS_CUDA(cudaMemcpy2DAsync(hsub, (size_t)ldh * sizeof(double), H, (size_t)mb * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    return RSDFT_OK;
}

int rsdft_gpu_subspace_solv(int mb, const double* hsub, int ldh, double* esp, double* vsub, int ldv) {
    RS_ENTRY();
    RS_CHECK(require_init());
    Context& c = ctx();
    if (mb < 1 || ldh < mb || ldv < mb || !hsub || !esp || !vsub) {
        set_error("subspace_solv: bad arguments");
        return RSDFT_EINVAL;
    }
    double *H, *W;
    RS_CHECK(workspace_t("solv_H", (size_t)mb * mb, &H));
    RS_CHECK(workspace_t("solv_W", (size_t)mb, &W));
    RS_CUDA(cudaMemcpy2DAsync(H, (size_t)mb * sizeof(double), hsub, (size_t)ldh * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    RS_CHECK(syevd(H, mb, W, CUBLAS_FILL_MODE_LOWER, "subspace_solv: syevd"));
    RS_CUDA(cudaMemcpy2DAsync(vsub, (size_t)ldv * sizeof(double), H, (size_t)mb * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    RS_CUDA(cudaMemcpyAsync(esp, W, sizeof(double) * mb, cudaMemcpyDefault, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    return RSDFT_OK;
}

int rsdft_gpu_subspace_rotv(int k, int s, double* unk, long ld, int mb, const double* vsub, int ldv) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    RS_CHECK(check_k_s(k, s, "subspace_rotv"));
    Context& c = ctx();
    if (ld < c.ml || mb < 1 || ldv < mb || !vsub) {
        set_error("subspace_rotv: bad arguments");
        return RSDFT_EINVAL;
    }
    double *d, *V, *tmp;
    bool st;
    RS_CHECK(wf_acquire(unk, ld, mb, "rotv_unk", &d, &st));
    RS_CHECK(workspace_t("rotv_V", (size_t)mb * mb, &V));
    RS_CHECK(workspace_t("sub_hpsi", (size_t)ld * mb, &tmp));
    RS_CUDA(cudaMemcpy2DAsync(V, (size_t)mb * sizeof(double), vsub, (size_t)ldv * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    RS_CHECK(dmma_gemm(false, c.ml, mb, mb, 1.0, d, ld, V, mb, 0.0, tmp, ld));
    RS_CUDA(cudaMemcpy2DAsync(d, ld * sizeof(double), tmp, ld * sizeof(double), c.ml * sizeof(double), mb,
                              cudaMemcpyDeviceToDevice, c.stream));
    RS_CHECK(wf_release(unk, d, ld, mb, st));
    return RSDFT_OK;
}

int rsdft_gpu_gram(const double* a, const double* b, long ld, long rows, int m, int n, double alpha, int sym,
                   double* cmat, int ldc) {
    RS_ENTRY();
    RS_CHECK(require_init());
    Context& c = ctx();
    if (!a || !b || !cmat || rows < 1 || ld < rows || m < 1 || n < 1 || ldc < m || (sym && m != n)) {
        set_error("gram: bad arguments (rows=%ld ld=%ld m=%d n=%d ldc=%d sym=%d)", rows, ld, m, n, ldc, sym);
        return RSDFT_EINVAL;
    }
    // the span each operand covers: its last column ends at row `rows`
    void *da = nullptr, *db = nullptr;
    RS_CHECK(stage_in(a, sizeof(double) * ((size_t)ld * (m - 1) + rows), "gram_a", &da));
    RS_CHECK(stage_in(b, sizeof(double) * ((size_t)ld * (n - 1) + rows), "gram_b", &db));
    double* C = nullptr;
    RS_CHECK(workspace_t("gram_c", (size_t)m * n, &C));
    RS_CHECK(dmma_gram((const double*)da, (const double*)db, ld, rows, m, n, alpha, sym, C, m));
    RS_CUDA(cudaMemcpy2DAsync(cmat, (size_t)ldc * sizeof(double), C, (size_t)m * sizeof(double),
                              (size_t)m * sizeof(double), n, cudaMemcpyDefault, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    return RSDFT_OK;
}

int rsdft_gpu_overlap_cholesky(int mb, const double* s, int lds, double* rinv, int ldr, double* kappa) {
    RS_ENTRY();
    RS_CHECK(require_init());
    Context& c = ctx();
    if (mb < 1 || lds < mb || ldr < mb || !s || !rinv) {
        set_error("overlap_cholesky: bad arguments");
        return RSDFT_EINVAL;
    }
    double *S = nullptr, *mm = nullptr;
    int* dinfo = nullptr;
    RS_CHECK(workspace_t("slab_S", (size_t)mb * mb, &S));
    RS_CHECK(workspace_t("osd_minmax", 2, &mm));
    RS_CHECK(workspace_t("gs_info", 4, &dinfo));
    RS_CUDA(cudaMemcpy2DAsync(S, (size_t)mb * sizeof(double), s, (size_t)lds * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    RS_CHECK(potrf_upper(S, mb, dinfo, "overlap_cholesky: Cholesky"));
    launch(k_diag_minmax, 1, 256, 0, c.stream, S, mb, mb, mm);
    RS_LAUNCH();
    double hmm[2] = {0.0, 0.0};
    RS_CUDA(cudaMemcpyAsync(hmm, mm, sizeof(hmm), cudaMemcpyDeviceToHost, c.stream));
    RS_CHECK(trtri_upper(S, mb, dinfo, "overlap_cholesky: triangular inverse"));
    RS_CUDA(cudaMemcpy2DAsync(rinv, (size_t)ldr * sizeof(double), S, (size_t)mb * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    if (kappa) *kappa = hmm[0] > 0.0 ? (hmm[1] / hmm[0]) * (hmm[1] / hmm[0]) : INFINITY;
    return RSDFT_OK;
}

int rsdft_gpu_rr_reduced(int mb, const double* rinv, int ldr, const double* hsub, int ldh, double* esp, double* w,
                         int ldw) {
    RS_ENTRY();
    RS_CHECK(require_init());
    Context& c = ctx();
    if (mb < 1 || ldr < mb || ldh < mb || ldw < mb || !rinv || !hsub || !esp || !w) {
        set_error("rr_reduced: bad arguments");
        return RSDFT_EINVAL;
    }
    double *R = nullptr, *H = nullptr, *T = nullptr, *E = nullptr;
    RS_CHECK(workspace_t("slab_S", (size_t)mb * mb, &R));
    RS_CHECK(workspace_t("sub_H", (size_t)mb * mb, &H));
    RS_CHECK(workspace_t("osd_T", (size_t)mb * mb, &T));
    RS_CHECK(workspace_t("slab_esp", (size_t)mb, &E));
    RS_CUDA(cudaMemcpy2DAsync(R, (size_t)mb * sizeof(double), rinv, (size_t)ldr * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    RS_CUDA(cudaMemcpy2DAsync(H, (size_t)mb * sizeof(double), hsub, (size_t)ldh * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    RS_CHECK(rr_reduced(R, H, T, mb, E, "rr_reduced: syevd"));
    RS_CUDA(cudaMemcpy2DAsync(w, (size_t)ldw * sizeof(double), T, (size_t)mb * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    RS_CUDA(cudaMemcpyAsync(esp, E, sizeof(double) * mb, cudaMemcpyDefault, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    return RSDFT_OK;
}

int rsdft_gpu_rotate(double* unk, long ld, long rows, int mb, const double* v, int ldv) {
    RS_ENTRY();
    RS_CHECK(require_init());
    Context& c = ctx();
    if (!unk || !v || rows < 1 || ld < rows || mb < 1 || ldv < mb) {
        set_error("rotate: bad arguments (rows=%ld ld=%ld mb=%d ldv=%d)", rows, ld, mb, ldv);
        return RSDFT_EINVAL;
    }
    void* du = nullptr;
    const size_t span = sizeof(double) * ((size_t)ld * (mb - 1) + rows);
    const int r = resolve(unk, span, &du);
    if (r < 0) return r;
    if (!r) {
        set_error("rotate: unk must be device memory or a registered array");
        return RSDFT_EINVAL;
    }
    double *V = nullptr, *tmp = nullptr;
    RS_CHECK(workspace_t("rotv_V", (size_t)mb * mb, &V));
    RS_CHECK(workspace_t("rot_tmp", (size_t)rows * mb, &tmp));
    RS_CUDA(cudaMemcpy2DAsync(V, (size_t)mb * sizeof(double), v, (size_t)ldv * sizeof(double),
                              (size_t)mb * sizeof(double), mb, cudaMemcpyDefault, c.stream));
    double* d = static_cast<double*>(du);
    RS_CHECK(dmma_gemm(false, rows, mb, mb, 1.0, d, ld, V, mb, 0.0, tmp, rows));
    RS_CUDA(cudaMemcpy2DAsync(d, ld * sizeof(double), tmp, rows * sizeof(double), rows * sizeof(double), mb,
                              cudaMemcpyDeviceToDevice, c.stream));
    return RSDFT_OK;
}

int rsdft_gpu_eigensolver_sweep(int k, int s, double* unk, long ld, int mb, double* esp, double* res, int ncg,
                                int mloop, int ipc, int mode) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    RS_CHECK(check_k_s(k, s, "eigensolver_sweep"));
    Context& c = ctx();
    if (ld != c.ml || mb < 1 || mb > 65535 || !esp || !res || ncg < 0 || mloop < 0 || (ipc != 0 && ipc != 4) ||
        !mode_valid(mode)) {
        set_error("eigensolver_sweep: bad arguments");
        return RSDFT_EINVAL;
    }
    double *d, *W, *R;
    bool st;
    // a host array in the mixed forms is uploaded band block by band block
    // below, overlapped with the CG; every other case copies it in here
    const int nchunk = mb >= 96 ? 8 : 1;
    const bool overlap = mode != RSDFT_MODE_FP64 && nchunk > 1;
    RS_CHECK(wf_acquire(unk, ld, mb, "sweep_unk", &d, &st, !overlap));
    // the copy stream writes the staging buffer: earlier work on it first
    if (st && overlap) RS_CUDA(cudaStreamSynchronize(c.stream));
    RS_CHECK(workspace_t("sweep_W", (size_t)mb, &W));
    RS_CHECK(workspace_t("sweep_R", (size_t)mb, &R));
    if (st && overlap) {
        float* x32 = nullptr;
        const float* hx = nullptr;
        RS_CHECK(cg_device_f32_staged(unk, d, ld, mb, s, W, R, ncg, mloop, ipc, nchunk, &x32, &hx));
        RS_CHECK(orth_subspace_diag_f32(x32, hx, d, ld, mb, s, W, mode));
    } else {
        RS_CHECK(sweep_device(d, ld, mb, s, W, R, ncg, mloop, ipc, mode));
    }
    RS_CHECK(stage_out(esp, W, sizeof(double) * mb));
    RS_CHECK(stage_out(res, R, sizeof(double) * mb));
    RS_CHECK(wf_release(unk, d, ld, mb, st));
    return RSDFT_OK;
}

int rsdft_gpu_orth_subspace_diag(int k, int s, double* unk, long ld, int mb, double* esp, int mode) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    RS_CHECK(check_k_s(k, s, "orth_subspace_diag"));
    Context& c = ctx();
    if (ld < c.ml || mb < 1 || !esp || !mode_valid(mode)) {
        set_error("orth_subspace_diag: bad arguments");
        return RSDFT_EINVAL;
    }
    double *d, *W;
    bool st;
    RS_CHECK(wf_acquire(unk, ld, mb, "sd_unk", &d, &st));
    RS_CHECK(workspace_t("sd_W", (size_t)mb, &W));
    RS_CHECK(orth_subspace_diag_device(d, ld, mb, s, W, mode));
    RS_CHECK(stage_out(esp, W, sizeof(double) * mb));
    RS_CHECK(wf_release(unk, d, ld, mb, st));
    return RSDFT_OK;
}

int rsdft_gpu_subspace_diag(int k, int s, double* unk, long ld, int mb, double* esp, int mode) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    RS_CHECK(check_k_s(k, s, "subspace_diag"));
    Context& c = ctx();
    if (ld < c.ml || mb < 1 || !esp || !mode_valid(mode)) {
        set_error("subspace_diag: bad arguments");
        return RSDFT_EINVAL;
    }
    double *d, *W;
    bool st;
    RS_CHECK(wf_acquire(unk, ld, mb, "sd_unk", &d, &st));
    RS_CHECK(workspace_t("sd_W", (size_t)mb, &W));
    RS_CHECK(subspace_diag_device(d, ld, mb, s, W, mode));
    RS_CHECK(stage_out(esp, W, sizeof(double) * mb));
    RS_CHECK(wf_release(unk, d, ld, mb, st));
    return RSDFT_OK;
}

}  // extern "C"
