// The small dense kernels of the subspace steps that stand in for LAPACK
// calls (the library's own code, no cuSOLVER):
//
//  trtri_upper_device: X = R^-1 for an upper-triangular R (LAPACK dtrtri,
//    uplo 'U', diag 'N').  One warp per row i of X, eight rows per CTA:
//    X(i, j) = 0 (j < i), X(i, i) = 1 / R(i, i),
//    X(i, j) = -(sum_{l=i}^{j-1} X(i, l) R(l, j)) / R(j, j)  (j > i).
//    R's columns are staged in shared memory in chunks (rows from the CTA's
//    first row down to the chunk's last column, by cp.async), the reciprocal
//    diagonal beside them; a warp forms the sums of eight consecutive
//    columns j in one pass over the l below the group (lanes stride l, then
//    eight xor trees), then closes the group's own triangle in order with
//    the values it has just found.  So the serial chain is one reduction
//    per eight columns, and every operand after the staging is in shared
//    memory.
//  potrf_upper_device: S = R^T R with R upper (LAPACK dpotrf, uplo 'U';
//    the strictly lower triangle of S neither read nor written), right-
//    looking over 32 x 32 tiles, one launch per tile step.  Step k runs one
//    CTA per trailing tile (i, j), k < i <= j: it forms the two panel tiles
//    it needs, R(k, i) = X^T S(k, i) with X = R(k, k)^-1 published by the
//    step before (so no CTA waits on another), and subtracts R(k, i)^T
//    R(k, j) from S(i, j).  The CTA of (k+1, k+1) keeps its updated tile,
//    factors it by one warp in dpotf2's order (r = d times 1 / sqrt(d),
//    the row scaled by 1 / r, 1 / sqrt(d) by Newton-Raphson) and inverts
//    the factor for the next step.  The panels go to a side buffer (S's row
//    block k is still being read during step k) and into S at the end.  A
//    pivot that is not positive (or NaN) sets info to its 1-based index as
//    dpotrf does, and the later launches stop.
//  ormtr_lower_device: C <- Q C for Q = H(0) H(1) ... H(n-2) of the lower
//    Householder tridiagonalisation (LAPACK dormtr with side 'L', uplo 'L',
//    trans 'N'; H(i) = I - tau_i v_i v_i^T, v_i(i+1) = 1 and v_i(i+2:n-1)
//    stored below the subdiagonal of column i): the reflectors in blocks of
//    32 as compact WY products H(j0) ... H(j0+31) = I - V T V^T (dlarft's
//    forward, columnwise T, one CTA per block), then each CTA takes eight
//    columns of C (one per warp) and applies the blocks from the last to the
//    first: the block's V staged in shared memory once (cp.async), W = V^T c
//    (a butterfly reduce-transpose over the lanes), W <- T W, c -= V W.
#include "common.cuh"
#include "kernels.cuh"

namespace rsdft {

constexpr unsigned FULL = 0xffffffffu;
constexpr int CF_P = 33;  // shared-memory pitch of the 32-column tiles (doubles)

// 8-byte global -> shared copy, asynchronous (completed by cp_async_wait)
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ------------------------------------------------------------------ trtri
constexpr int TR_W = 8;  // rows of X (one per warp) per CTA
constexpr int TR_G = 8;  // columns per reduction group

__global__ void __launch_bounds__(32 * TR_W) k_trtri(const double* __restrict__ R, int n, int cwmax,
                                                     double* __restrict__ X) {
    extern __shared__ double tr_sm[];
    const int i0 = blockIdx.x * TR_W;
    const int rows = n - i0;           // pitch of a staged column: rows i0 .. n-1 at most
    double* sR = tr_sm;                // cwmax columns, R(i0 + l, c0 + c) at sR[c * rows + l]
    double* sD = sR + (size_t)cwmax * rows;  // 1 / R(j, j) of the chunk
    double* sX = sD + cwmax;           // the CTA's rows of X, n each
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int i = i0 + warp;
    const bool active = i < n;
    double* xr = sX + (size_t)warp * n;
    if (active) {
        for (int l = lane; l < n; l += 32) xr[l] = 0.0;
        for (int j = lane; j < i; j += 32) X[(long)j * n + i] = 0.0;
    }
    for (int c0 = (i0 / cwmax) * cwmax; c0 < n; c0 += cwmax) {
        const int cw = min(cwmax, n - c0);
        const int lr = c0 + cw - i0;  // staged rows i0 .. c0 + cw - 1 (R is upper)
        __syncthreads();
        for (int c = warp; c < cw; c += TR_W)
            for (int l = lane; l < lr; l += 32) cp_async8(sR + (size_t)c * rows + l, R + (long)(c0 + c) * n + i0 + l);
        if (tid < cw) sD[tid] = 1.0 / R[(long)(c0 + tid) * n + c0 + tid];
        cp_async_wait();
        __syncthreads();
        if (!active) continue;
        for (int g0 = 0; g0 < cw; g0 += TR_G) {
            const int jg = c0 + g0;
            if (jg + TR_G <= i) continue;  // the group lies left of the diagonal
            double p[TR_G];
#pragma unroll
            for (int u = 0; u < TR_G; ++u) p[u] = 0.0;
            for (int l = i + lane; l < jg; l += 32) {
                const double xl = xr[l];
                const double* rc = sR + (size_t)g0 * rows + (l - i0);
#pragma unroll
                for (int u = 0; u < TR_G; ++u) p[u] = fma(xl, rc[(size_t)u * rows], p[u]);
            }
#pragma unroll
            for (int u = 0; u < TR_G; ++u)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) p[u] += __shfl_xor_sync(FULL, p[u], o);
            double xv[TR_G];
#pragma unroll
            for (int u = 0; u < TR_G; ++u) {
                const int j = jg + u;
                double x = 0.0;
                if (g0 + u < cw && j >= i) {
                    if (j == i) {
                        x = sD[g0 + u];
                    } else {
                        double s = p[u];
#pragma unroll
                        for (int m = 0; m < u; ++m)
                            if (jg + m >= i) s = fma(xv[m], sR[(size_t)(g0 + u) * rows + (jg + m - i0)], s);
                        x = -s * sD[g0 + u];
                    }
                }
                xv[u] = x;
            }
            if (lane < TR_G && g0 + lane < cw && jg + lane >= i) {
                double x = xv[0];
#pragma unroll
                for (int u = 1; u < TR_G; ++u)
                    if (lane == u) x = xv[u];
                xr[jg + lane] = x;
                X[(long)(jg + lane) * n + i] = x;
            }
            __syncwarp();
        }
    }
}

// ------------------------------------------------------------------ potrf
constexpr int CH_T = 256;  // threads per CTA of the Cholesky kernels

// 1 / sqrt(d) for normal d > 0: Newton-Raphson iteration for the inverse
// square root, y <- y + y (1 - d y^2) / 2 (quadratic convergence), from the
// PTX approximate reciprocal square root; two steps take the seed past
// double precision.
__device__ __forceinline__ double rsqrt_nr(double d) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    y = fma(0.5 * y, fma(-d * y, y, 1.0), y);
    return fma(0.5 * y, fma(-d * y, y, 1.0), y);
}

// Cholesky of the leading kk x kk block of the tile T (row-major, pitch
// CF_P; its upper part read) by one warp, in dpotf2's order: step j,
// R(j, j) = sqrt(A(j, j)) (as d times 1/sqrt(d)), R(j, l) = A(j, l) times
// 1 / R(j, j), then A(i, l) -= R(j, i) R(j, l) for j < i <= l (row by
// row, lane l on column l).  dinv[j] receives 1 / R(j, j).  Returns
// (in every lane) 0, or the 1-based index of the first pivot that is not
// positive (or NaN).
__device__ int chol_tile_warp(double* T, int kk, double* dinv) {
    const int lane = threadIdx.x & 31;
    for (int j = 0; j < kk; ++j) {
        const double d = T[j * CF_P + j];
        if (!(d > 0.0)) return j + 1;  // the same d in every lane
        const double inv = rsqrt_nr(d);
        const double rjl = (lane > j && lane < kk) ? T[j * CF_P + lane] * inv : 0.0;
        __syncwarp();
        if (lane == j) {
            T[j * CF_P + j] = d * inv;
            dinv[j] = inv;
        } else if (lane > j && lane < kk) {
            T[j * CF_P + lane] = rjl;
        }
        __syncwarp();
        // the trailing triangle j < i <= l < kk: row by row, lane l on column
        // l; R(j, i) comes from lane i's register (a shuffle, not a shared
        // load, so no shared-memory access orders the rows' updates)
#pragma unroll 4
        for (int i = j + 1; i < kk; ++i) {
            const double rji = __shfl_sync(FULL, rjl, i);
            if (lane >= i && lane < kk) T[i * CF_P + lane] = fma(-rji, rjl, T[i * CF_P + lane]);
        }
        __syncwarp();
    }
    return 0;
}

// X = R^-1 of the kk x kk upper factor in T (dinv = 1 / diag) by one warp,
// row by row from the last: X(i, i) = dinv[i], X(i, l) = -(sum_{m=i+1}^{l}
// R(i, m) X(m, l)) dinv[i] (l > i), lane l forming X(i, l) with four
// partial sums; written to xs (pitch CF_P) and xg (32 x 32, row-major),
// zero below the diagonal and outside kk.
__device__ void inv_tile_warp(const double* T, int kk, const double* dinv, double* xs, double* __restrict__ xg) {
    const int l = threadIdx.x & 31;
    for (int i = 31; i >= 0; --i) {
        double x = 0.0;
        if (i < kk && l < kk && i <= l) {
            if (i == l) {
                x = dinv[i];
            } else {
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                int m = i + 1;
                for (; m + 3 <= l; m += 4) {
                    s0 = fma(T[i * CF_P + m], xs[m * CF_P + l], s0);
                    s1 = fma(T[i * CF_P + m + 1], xs[(m + 1) * CF_P + l], s1);
                    s2 = fma(T[i * CF_P + m + 2], xs[(m + 2) * CF_P + l], s2);
                    s3 = fma(T[i * CF_P + m + 3], xs[(m + 3) * CF_P + l], s3);
                }
                for (; m <= l; ++m) s0 = fma(T[i * CF_P + m], xs[m * CF_P + l], s0);
                x = -((s0 + s1) + (s2 + s3)) * dinv[i];
            }
        }
        xs[i * CF_P + l] = x;
        __syncwarp();
    }
    for (int r = 0; r < 32; ++r) xg[r * 32 + l] = xs[r * CF_P + l];
}

// the upper part (r <= c, inside n) of tile T into tile (ti, tj) of the
// column-major n x n D
__device__ __forceinline__ void tile_put_upper(const double* T, int n, int ti, int tj, double* __restrict__ D) {
    for (int e = threadIdx.x; e < 1024; e += CH_T) {
        const int r = e & 31, c = e >> 5;
        const int gr = 32 * ti + r, gc = 32 * tj + c;
        if ((ti != tj || r <= c) && gr < n && gc < n) D[(long)gc * n + gr] = T[r * CF_P + c];
    }
}

__device__ __forceinline__ void tile_get(const double* __restrict__ S, int n, int ti, int tj, double* T) {
    for (int e = threadIdx.x; e < 1024; e += CH_T) {
        const int r = e & 31, c = e >> 5;
        const int gr = 32 * ti + r, gc = 32 * tj + c;
        T[r * CF_P + c] = (gr < n && gc < n) ? S[(long)gc * n + gr] : 0.0;
    }
}

// factor the diagonal tile held in sA (global tile index t) and publish it:
// R into Rb, and (want_inv) R^-1 into xg; a bad pivot sets info and fail
__device__ void chol_publish(double* sA, double* sX, double* dinv, int n, int t, bool want_inv,
                             double* __restrict__ Rb, double* __restrict__ xg, int* __restrict__ info,
                             int* __restrict__ fail) {
    __shared__ int bad;
    const int kk = min(32, n - 32 * t);
    if (threadIdx.x < 32) {
        const int b = chol_tile_warp(sA, kk, dinv);
        if (b == 0 && want_inv) inv_tile_warp(sA, kk, dinv, sX, xg);
        if (threadIdx.x == 0) {
            bad = b;
            if (b) {
                *info = 32 * t + b;
                *fail = 1;
            }
        }
    }
    __syncthreads();
    if (!bad) tile_put_upper(sA, n, t, t, Rb);
}

// step -1: the first diagonal tile
__global__ void __launch_bounds__(CH_T) k_chol_first(const double* __restrict__ S, int n, double* __restrict__ Rb,
                                                     double* __restrict__ xg, int* __restrict__ info,
                                                     int* __restrict__ fail) {
    __shared__ double sA[32 * CF_P], sX[32 * CF_P], dinv[32];
    if (threadIdx.x == 0) {
        *info = 0;
        *fail = 0;
    }
    tile_get(S, n, 0, 0, sA);
    __syncthreads();
    chol_publish(sA, sX, dinv, n, 0, n > 32, Rb, xg, info, fail);
}

// step k: one CTA per trailing tile (i, j), k < i <= j, the diagonal tile
// (k+1, k+1) first.  Each CTA forms R(k, i) = X^T S(k, i) and R(k, j) with
// X = R(k, k)^-1 (xin), writes R(k, i) to Rb when i == j, and subtracts
// R(k, i)^T R(k, j) from S(i, j); the CTA of (k+1, k+1) keeps the updated
// tile, factors it and publishes R(k+1, k+1) and its inverse (xout; sX is
// free by then and serves as the inverse's scratch).
__global__ void __launch_bounds__(CH_T) k_chol_step(double* __restrict__ S, int n, int k, double* __restrict__ Rb,
                                                    const double* __restrict__ xin, double* __restrict__ xout,
                                                    int* __restrict__ info, int* __restrict__ fail) {
    __shared__ double sX[32 * CF_P], sA[32 * CF_P], sB[32 * CF_P], sC[32 * CF_P], dinv[32];
    if (*(const volatile int*)fail) return;
    const int nt = (n + 31) / 32;
    int q = blockIdx.x, j = k + 1;
    while (q > j - k - 1) {  // tiles ordered by column j, then row i
        q -= j - k;
        ++j;
    }
    const int i = k + 1 + q;
    const int t = threadIdx.x, r = t & 31, c0 = t >> 5;
    // X, S(k, i), S(k, j) and S(i, j) all in flight at once
    for (int e = t; e < 1024; e += CH_T) sX[(e >> 5) * CF_P + (e & 31)] = xin[e];
    tile_get(S, n, k, i, sA);
    if (j != i) tile_get(S, n, k, j, sB);
    tile_get(S, n, i, j, sC);
    __syncthreads();
    // R(k, i), R(k, j): out(r, c) = sum_{l <= r} X(l, r) A(l, c)
    double oi[4] = {0.0, 0.0, 0.0, 0.0}, oj[4] = {0.0, 0.0, 0.0, 0.0};
    for (int l = 0; l <= r; ++l) {
        const double xl = sX[l * CF_P + r];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            oi[m] = fma(xl, sA[l * CF_P + c0 + 8 * m], oi[m]);
            if (j != i) oj[m] = fma(xl, sB[l * CF_P + c0 + 8 * m], oj[m]);
        }
    }
    __syncthreads();
    double* sRi = sA;
    double* sRj = j != i ? sB : sA;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        sRi[r * CF_P + c0 + 8 * m] = oi[m];
        if (j != i) sRj[r * CF_P + c0 + 8 * m] = oj[m];
    }
    __syncthreads();
    if (i == j) {  // the panel tile R(k, i) (full: row block k lies above the last)
        for (int e = t; e < 1024; e += CH_T) {
            const int rr = e & 31, cc = e >> 5;
            const int gc = 32 * i + cc;
            if (gc < n) Rb[(long)gc * n + 32 * k + rr] = sRi[rr * CF_P + cc];
        }
    }
    double o[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
    for (int l = 0; l < 32; ++l) {
        const double a = sRi[l * CF_P + r];
#pragma unroll
        for (int m = 0; m < 4; ++m) o[m] = fma(a, sRj[l * CF_P + c0 + 8 * m], o[m]);
    }
    if (i == k + 1 && j == k + 1) {
#pragma unroll
        for (int m = 0; m < 4; ++m) sC[r * CF_P + c0 + 8 * m] -= o[m];
        __syncthreads();
        chol_publish(sC, sX, dinv, n, k + 1, k + 2 < nt, Rb, xout, info, fail);
    } else {
        const int gr = 32 * i + r;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int cc = c0 + 8 * m, gc = 32 * j + cc;
            if (gr < n && gc < n && (i != j || r <= cc)) S[(long)gc * n + gr] = sC[r * CF_P + cc] - o[m];
        }
    }
}

// R (the upper triangle of Rb) into S; the strictly lower triangle of S is
// left as it was
__global__ void k_chol_copy(double* __restrict__ S, int n, const double* __restrict__ Rb,
                            const int* __restrict__ fail) {
    if (*fail) return;
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    const int row = (int)(e % n), col = (int)(e / n);
    if (row <= col) S[e] = Rb[e];
}

int potrf_upper_device(double* S, int n, int* dinfo) {
    Context& c = ctx();
    if (n < 1) {
        set_error("potrf: n = %d", n);
        return RSDFT_EINVAL;
    }
    const int nt = (n + 31) / 32;
    double *Rb = nullptr, *xb = nullptr;
    int* fail = nullptr;
    RS_CHECK(workspace_t("chol_R", (size_t)n * n, &Rb));
    RS_CHECK(workspace_t("chol_xinv", 2048, &xb));
    RS_CHECK(workspace_t("chol_fail", 4, &fail));
    launch(k_chol_first, 1, CH_T, 0, c.stream, (const double*)S, n, Rb, xb, dinfo, fail);
    RS_LAUNCH();
    for (int k = 0; k + 1 < nt; ++k) {
        const int m = nt - 1 - k;
        launch(k_chol_step, m * (m + 1) / 2, CH_T, 0, c.stream, S, n, k, Rb, (const double*)(xb + 1024 * (k & 1)),
               xb + 1024 * ((k + 1) & 1), dinfo, fail);
        RS_LAUNCH();
    }
    launch(k_chol_copy, (unsigned)div_up((long)n * n, 256L), 256, 0, c.stream, S, n, (const double*)Rb,
           (const int*)fail);
    RS_LAUNCH();
    return RSDFT_OK;
}

// ------------------------------------------------------------------ ormtr
// T of reflector block b (32 x 32, row-major; zero outside its nr
// reflectors): G = V^T V over the block's rows j0+1 .. n-1, then dlarft's
// recurrence T(j, j) = tau_j, T(i, j) = -tau_j sum_{i <= l < j} T(i, l)
// G(l, j).
__global__ void __launch_bounds__(256) k_larft(const double* __restrict__ Q, int n, const double* __restrict__ tau,
                                               double* __restrict__ T) {
    __shared__ double sV[64 * CF_P], sG[32 * CF_P], sT[32 * CF_P];
    const int b = blockIdx.x, j0 = 32 * b;
    const int nr = min(32, n - 1 - j0), R = n - 1 - j0;
    const int t = threadIdx.x, a = t & 31, c0 = t >> 5;
    double g[4] = {0.0, 0.0, 0.0, 0.0};
    for (int r0 = 0; r0 < R; r0 += 64) {
        __syncthreads();
        for (int e = t; e < 64 * 32; e += 256) {
            const int rr = e & 63, j = e >> 6, row = r0 + rr;
            if (j < nr && row < R && row > j)
                cp_async8(sV + rr * CF_P + j, Q + (long)(j0 + j) * n + j0 + 1 + row);
            else
                sV[rr * CF_P + j] = (j < nr && row == j) ? 1.0 : 0.0;
        }
        cp_async_wait();
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < 64; ++rr) {
            const double va = sV[rr * CF_P + a];
#pragma unroll
            for (int m = 0; m < 4; ++m) g[m] = fma(va, sV[rr * CF_P + c0 + 8 * m], g[m]);
        }
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) sG[a * CF_P + c0 + 8 * m] = g[m];
    for (int e = t; e < 1024; e += 256) sT[(e >> 5) * CF_P + (e & 31)] = 0.0;
    __syncthreads();
    for (int j = 0; j < nr; ++j) {
        const double tj = tau[j0 + j];
        if (t < j) {
            double s = 0.0;
            for (int l = t; l < j; ++l) s = fma(sT[t * CF_P + l], sG[l * CF_P + j], s);
            sT[t * CF_P + j] = -tj * s;
        } else if (t == j) {
            sT[j * CF_P + j] = tj;
        }
        __syncthreads();
    }
    for (int e = t; e < 1024; e += 256) T[(size_t)b * 1024 + e] = sT[(e >> 5) * CF_P + (e & 31)];
}


constexpr int OW = 8;  // columns of C (one per warp) per CTA of k_apply_wy

// dynamic shared memory: the block's V (32 columns, pitch n) and the CTA's
// columns of C (n each)
__global__ void __launch_bounds__(32 * OW) k_apply_wy(const double* __restrict__ Q, int n,
                                                      const double* __restrict__ T, double* __restrict__ C,
                                                      int ldc) {
    extern __shared__ double ow_sm[];
    double* sV = ow_sm;                 // V(rr, j) at sV[j * n + rr]
    double* sT = ow_sm + (size_t)32 * n;  // the block's T (32 x 32, row-major)
    double* sCv = sT + 1024;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int col = blockIdx.x * OW + warp;
    const bool active = col < n;
    double* cv = sCv + (size_t)warp * n;
    if (active)
        for (int r = lane; r < n; r += 32) cv[r] = C[(long)col * ldc + r];
    const int nblk = (n - 1 + 31) / 32;
    for (int b = nblk - 1; b >= 0; --b) {
        const int j0 = 32 * b, nr = min(32, n - 1 - j0), R = n - 1 - j0, row0 = j0 + 1;
        __syncthreads();  // the previous block's V is no longer read
        for (int j = warp; j < 32; j += OW)
            for (int rr = lane; rr < R; rr += 32) {
                double* dst = sV + (size_t)j * n + rr;
                if (j < nr && rr > j)
                    cp_async8(dst, Q + (long)(j0 + j) * n + row0 + rr);
                else
                    *dst = (j < nr && rr == j) ? 1.0 : 0.0;
            }
        for (int e = tid; e < 1024; e += 32 * OW) cp_async8(sT + e, T + (size_t)b * 1024 + e);
        cp_async_wait();
        __syncthreads();
        if (!active) continue;
        double acc[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] = 0.0;
        for (int rr = lane; rr < R; rr += 32) {
            const double cr = cv[row0 + rr];
#pragma unroll
            for (int j = 0; j < 32; ++j) acc[j] = fma(sV[(size_t)j * n + rr], cr, acc[j]);
        }
        // butterfly: after the stage with offset s each lane keeps the half of
        // its sums whose index has the lane's bit s; lane j ends with W(j)
#pragma unroll
        for (int s = 16; s >= 1; s >>= 1) {
            const bool up = (lane & s) != 0;
#pragma unroll
            for (int m = 0; m < s; ++m) {
                const double send = up ? acc[m] : acc[m + s];
                const double keep = up ? acc[m + s] : acc[m];
                acc[m] = keep + __shfl_xor_sync(FULL, send, s);
            }
        }
        const double w = acc[0];
        double wp = 0.0;
        const double* Tb = sT + lane * 32;
#pragma unroll
        for (int l = 0; l < 32; ++l) wp = fma(Tb[(l + lane) & 31], __shfl_sync(FULL, w, (l + lane) & 31), wp);
        double wq[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) wq[j] = __shfl_sync(FULL, wp, j);
        for (int rr = lane; rr < R; rr += 32) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 32; ++j) s = fma(sV[(size_t)j * n + rr], wq[j], s);
            cv[row0 + rr] -= s;
        }
    }
    if (active) {
        __syncwarp();
        for (int r = lane; r < n; r += 32) C[(long)col * ldc + r] = cv[r];
    }
}

size_t ormtr_smem_bytes(int n) { return sizeof(double) * ((size_t)(32 + OW) * n + 1024); }

// the bound device's opt-in shared-memory limit per block
static int smem_limit(Context& c, long* out) {
    if (c.max_smem_optin < 0)
        RS_CUDA(cudaDeviceGetAttribute(&c.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
    *out = c.max_smem_optin;
    return RSDFT_OK;
}

int trtri_upper_device(const double* R, int n, double* X) {
    Context& c = ctx();
    if (n < 1) return RSDFT_OK;
    long lim = 0;
    RS_CHECK(smem_limit(c, &lim));
    int cw = 32;
    auto need = [&](int w) {
        const int rows = n;  // the first CTA stages rows 0 .. n-1
        return sizeof(double) * ((size_t)w * rows + w + (size_t)TR_W * n);
    };
    while (cw > TR_G && (long)need(cw) > lim) cw /= 2;
    if ((long)need(cw) > lim) {
        set_error("trtri: n = %d needs %zu bytes of shared memory", n, need(cw));
        return RSDFT_EUNSUP;
    }
    RS_CHECK(set_smem_optin((const void*)k_trtri, (int)need(cw)));
    launch(k_trtri, div_up(n, TR_W), 32 * TR_W, need(cw), c.stream, R, n, cw, X);
    RS_LAUNCH();
    return RSDFT_OK;
}

int ormtr_lower_device(const double* Q, const double* tau, int n, double* C) {
    Context& c = ctx();
    if (n < 2) return RSDFT_OK;  // Q = I
    const int nblk = (n - 1 + 31) / 32;
    double* T = nullptr;
    RS_CHECK(workspace_t("ormtr_T", (size_t)nblk * 1024, &T));
    launch(k_larft, nblk, 256, 0, c.stream, Q, n, tau, T);
    RS_LAUNCH();
    const size_t smem = ormtr_smem_bytes(n);
    long lim = 0;
    RS_CHECK(smem_limit(c, &lim));
    if ((long)smem > lim) {
        set_error("ormtr: n = %d needs %zu bytes of shared memory", n, smem);
        return RSDFT_EUNSUP;
    }
    RS_CHECK(set_smem_optin((const void*)k_apply_wy, (int)smem));
    launch(k_apply_wy, div_up(n, OW), 32 * OW, smem, c.stream, Q, n, (const double*)T, C, n);
    RS_LAUNCH();
    return RSDFT_OK;
}

}  // namespace rsdft
