// Symmetric eigensolver for the small dense matrices of the subspace steps
// (the Rayleigh-Ritz matrix, n = number of bands, up to ~590): the same
// result as LAPACK dsyevd / cuSOLVER syevd (eigenvalues ascending, an
// orthonormal eigenvector basis), in three steps:
//
//  1. k_sytrd: Householder tridiagonalisation A = Q T Q^T (LAPACK dsytd2,
//     lower form) by ONE thread-block cluster of 16 CTAs with the whole
//     matrix resident in their shared memory: CTA c holds the full rows
//     i = c, c + 16, ... .  Column j: every CTA holds the reflector v, forms
//     p = tau A v on its own rows and its part of p^T v, pulls the rest of p
//     and the look-ahead row j+1 over distributed shared memory, applies the
//     rank-2 update A -= v w^T + w v^T (w = p - tau/2 (p^T v) v) to its own
//     rows and to that row, and forms the next reflector itself.  One
//     cluster barrier per column; nothing leaves the SMs until T and the
//     reflectors are written.
//  2. k_tri_bisect: eigenvalues of T by multisection on Sturm counts (one
//     warp per eigenvalue, 32 trial points per round; LAPACK dstebz's count
//     with its pivmin guard).  k_tri_invit: eigenvectors of T by inverse
//     iteration with partial-pivoting LU of T - lambda I (LAPACK dstein:
//     dgttrf/dgttrs steps, its start-vector scaling, convergence test and two
//     extra iterations, perturbed shifts and modified Gram-Schmidt for
//     eigenvalues closer than 1e-10 |T|_1), one thread per group.  A
//     vector computed on its own is the exact eigenvector of T + F with
//     |F| ~ eps |T|, so two vectors with eigenvalue gap g overlap by
//     ~eps |T| / g; dstein removes that by Gram-Schmidt over chains of gaps
//     below 1e-3 |T|, which turns the compressed spectra of unconverged
//     Rayleigh-Ritz matrices into one serial chain.  Here the chains are
//     cut at 1e-10 |T| (overlaps stay below ~1e-6) and two Newton-Schulz
//     steps Z <- Z (3 I - Z^T Z) / 2 (four DGEMMs) make the basis orthonormal
//     to rounding; they mix vectors i, j by ~eps |T| / |l_i - l_j|, which
//     moves the residuals by ~eps |T| only.
//  3. ormtr_lower_device (factor.cu) applies Q to the eigenvectors of T.
//
// cuSOLVER's one-stage syevd spends ~80 % of its time in sytrd for these
// sizes (3.9 of 5.0 ms at n = 480 on B200), one short kernel per column;
// here each column costs one cluster barrier.
#include <cfloat>

#include "common.cuh"
#include "dmma.cuh"
#include "cluster.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace rsdft {

constexpr int TD_C = 16;          // CTAs in the cluster
constexpr int TD_T = 512;         // threads per CTA
constexpr int TD_W = TD_T / 32;


// Shared-memory layout of k_sytrd (doubles; every array an even count, so
// each starts 16-byte aligned for the bulk copies): own rows R x np, the
// reflectors v_j / v_{j+1}, w, p, the look-ahead row, and the exchange
// buffers: per parity what each CTA sent, px[16][PR], and this CTA's
// outgoing block sb[PR] = [its R pieces of p, its part of p^T v, its rows'
// entries of the look-ahead column, padding]; reduction slots, scalars, and
// the two receive mbarriers.
struct TdLayout {
    int R, np, PR;
    size_t rows, vl, wf, pf, rr, px, sb, red, sc, bar, total;
    __host__ __device__ TdLayout(int n) {
        R = (n + TD_C - 1) / TD_C;
        np = (n + 1) & ~1;
        PR = (2 * R + 2) & ~1;
        rows = 0;
        vl = rows + (size_t)R * np;  // [2][np]
        wf = vl + 2 * (size_t)np;
        pf = wf + np;
        rr = pf + np;
        px = rr + np;                       // [2][TD_C][PR]
        sb = px + 2 * (size_t)TD_C * PR;    // [2][PR]
        red = sb + 2 * (size_t)PR;
        sc = red + TD_W;
        bar = sc + 8;  // 2 x uint64_t
        total = bar + 2;
    }
};

__device__ __forceinline__ uint32_t cl_addr(const void* p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(r)
                 : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(rank));
    return r;
}

// Bulk copy (TMA engine, point to point, no multicast) of `bytes` from this
// CTA's shared memory to the buffer at the same offset as `dst` in CTA
// `rank`, completion counted on that CTA's mbarrier at the offset of `bar`.
// Addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_to_peer(const void* dst, const void* src, uint32_t bytes, const uint64_t* bar,
                                             uint32_t rank) {
    asm volatile(
        "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            cl_addr(dst, rank)),
        "r"((uint32_t)__cvta_generic_to_shared(src)), "r"(bytes), "r"(cl_addr(bar, rank))
        : "memory");
}

// dlarfg on x[0..len): v (v_0 = 1) into vl, sc[0] = tau, sc[1] = beta.  All
// threads of the CTA; fixed reduction order, so every CTA that runs it on
// the same x gets the same bits.
__device__ __forceinline__ void td_reflector(const double* x, int len, double* vl, double* red, double* sc) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double s = 0.0;
    for (int k = 1 + tid; k < len; k += TD_T) s = fma(x[k], x[k], s);
    s = warp_sum_d(s);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
        double sig = 0.0;
        for (int w = 0; w < TD_W; ++w) sig += red[w];
        const double alpha = x[0];
        double t = 0.0, beta = alpha, scal = 0.0;
        if (sig > 0.0) {
            beta = -copysign(sqrt(fma(alpha, alpha, sig)), alpha);
            t = (beta - alpha) * rcp_nr(beta);
            scal = rcp_nr(alpha - beta);
        }
        sc[0] = t;
        sc[1] = beta;
        sc[2] = scal;
        sc[3] = sig > 0.0 ? 1.0 : 0.0;
    }
    __syncthreads();
    const double scal = sc[2];
    const bool nontriv = sc[3] != 0.0;
    for (int k = tid; k < len; k += TD_T) vl[k] = k == 0 ? 1.0 : (nontriv ? x[k] * scal : 0.0);
    __syncthreads();
}

// A (n x n, lda; the `upper` or lower triangle is read) -> d (n), e (n-1),
// tau (n-1) and the reflectors in the strict lower part of Q (n x n, ld n;
// Q(j+1+k, j) = v_k for k >= 1, dsytrd's 'L' storage).
//
// Column j: every CTA holds v_j and has pushed, with bulk copies into every
// CTA of the cluster, its pieces of p_j = tau_j A v_j and of p_j^T v_j and
// its rows' entries of column j+1 as they stand (the look-ahead row, by
// symmetry; gathered from all CTAs, so no SM serves a one-to-all broadcast).
// Each CTA waits on its own mbarrier for those bytes, forms w_j, brings its
// copy of row j+1 up to date and runs dlarfg on it for v_{j+1} (the same bits
// in every CTA), then makes one pass over its own rows that applies
// A -= v_j w_j^T + w_j v_j^T and, on the updated values, forms p_{j+1}; the
// next pushes follow.  The receive barriers carry both the data and the
// ordering: exchange buffers are double-buffered by column parity, and the
// block a CTA must hold before reusing a buffer was sent after that buffer's
// previous use, so no cluster barrier is needed per column.
__global__ void __launch_bounds__(TD_T, 1) k_sytrd(const double* __restrict__ A, int lda, int n, int upper,
                                                  double* __restrict__ Q, double* __restrict__ d,
                                                  double* __restrict__ e, double* __restrict__ tau,
                                                  int* __restrict__ err) {
    extern __shared__ __align__(16) double sm[];
    const TdLayout L(n);
    const int R = L.R, np = L.np, PR = L.PR;
    double* rows = sm + L.rows;
    double* vb = sm + L.vl;  // [2][np]
    double* wf = sm + L.wf;
    double* pf = sm + L.pf;
    double* rr = sm + L.rr;
    double* px = sm + L.px;
    double* sb = sm + L.sb;
    double* red = sm + L.red;
    double* sc = sm + L.sc;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L.bar);
    const int cr = (int)cluster_rank();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    bool ok = true;

    for (int l = 0; l < R; ++l) {
        const int i = l * TD_C + cr;
        if (i >= n) break;
        for (int k = tid; k < n; k += TD_T) {
            const int a = i < k ? i : k, b = i < k ? k : i;  // (min, max)
            rows[(size_t)l * np + k] = upper ? A[a + (size_t)b * lda] : A[b + (size_t)a * lda];
        }
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    cluster_sync();  // rows loaded and receive barriers initialised everywhere

    // push this CTA's block for column jn from sb[buf] into every CTA; arm
    // this CTA's own barrier for the 16 blocks it will receive
    auto send = [&](int buf) {
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            const uint32_t pb = (uint32_t)(PR * sizeof(double));
            mbar_arrive_expect_tx(&bar[buf], TD_C * pb);
            for (int dst = 0; dst < TD_C; ++dst)
                bulk_to_peer(px + ((size_t)buf * TD_C + cr) * PR, sb + (size_t)buf * PR, pb, &bar[buf],
                             (uint32_t)dst);
        }
    };

    // v_0 from row 0 (CTA 0, local row 0)
    for (int k = tid; k < n; k += TD_T) rr[k] = dsmem_ld(rows + k, 0);
    __syncthreads();
    td_reflector(rr + 1, n - 1, vb, red, sc);
    if (cr == 0 && tid == 0) {
        d[0] = rr[0];
        e[0] = sc[1];
        tau[0] = sc[0];
        Q[0] = rr[0];
        Q[1] = sc[1];
    }
    if (cr == 0)
        for (int k = 1 + tid; k < n - 1; k += TD_T) Q[(size_t)(1 + k)] = vb[k];
    double tcur = sc[0];  // tau of the current column
    // p_0 on own rows i > 0
    {
        const double t = tcur;
        const int m = n - 1;
        double kacc = 0.0;
        for (int l = warp; l < R; l += TD_W) {
            const int i = l * TD_C + cr;
            double pv = 0.0;
            if (i >= 1 && i < n) {
                const double* a = rows + (size_t)l * np + 1;
                double s0 = 0.0;
                for (int k = lane; k < m; k += 32) s0 = fma(a[k], vb[k], s0);
                pv = t * warp_sum_d(s0);
                if (lane == 0) kacc = fma(pv, vb[i - 1], kacc);
            }
            if (lane == 0) {
                sb[l] = pv;
                sb[R + 1 + l] = i >= 1 && i < n ? rows[(size_t)l * np + 1] : 0.0;  // A(i, 1)
            }
        }
        if (lane == 0) red[warp] = kacc;
        __syncthreads();
        if (warp == 0) {
            const double s1 = warp_sum_d(lane < TD_W ? red[lane] : 0.0);
            if (lane == 0) sb[R] = s1;
        }
        send(0);
    }

    for (int j = 0; j <= n - 2; ++j) {
        const int m = n - 1 - j;  // length of v_j
        const int par = j & 1, nxt = par ^ 1;
        const double* vj = vb + par * np;
        double* vn = vb + nxt * np;
        const double t = tcur;
        // no cluster barrier: a CTA copies into px[par] of a peer for column
        // j+2 only after it has received that peer's block for column j+1,
        // which the peer sends after its reads of px[par] for column j; and a
        // peer's copies out of sb[par] for column j have all landed once this
        // CTA holds every block for column j+1 (each sender waited for its
        // column-j blocks before sending those)
        if (!mbar_wait(&bar[par], (uint32_t)((j >> 1) & 1))) ok = false;
        {
            // p_j and the look-ahead row j+1 (= column j+1: A(i, j+1) from the
            // owner of row i), both spread over the 16 blocks
            const double* xp = px + (size_t)par * TD_C * PR;
            for (int k = tid; k < m; k += TD_T) {
                const int i = j + 1 + k;
                const double* blk = xp + (size_t)(i % TD_C) * PR;
                pf[k] = blk[i / TD_C];
                rr[k] = blk[R + 1 + i / TD_C];
            }
        }
        // w = p + alpha v (into wf), row j+1 up to date; its columns j+3..
        // give sigma of v_{j+1}
        double sg = 0.0;
        {
            const double* xp = px + (size_t)par * TD_C * PR;
            double kp[TD_C / 2];  // pairwise sum of the 16 partial dots (fixed order)
#pragma unroll
            for (int c = 0; c < TD_C / 2; ++c) kp[c] = xp[(size_t)(2 * c) * PR + R] + xp[(size_t)(2 * c + 1) * PR + R];
#pragma unroll
            for (int h = TD_C / 4; h >= 1; h >>= 1)
#pragma unroll
                for (int c = 0; c < h; ++c) kp[c] = kp[2 * c] + kp[2 * c + 1];
            const double al = -0.5 * t * kp[0];
            const int j1 = j + 1;
            const double p0 = xp[(size_t)(j1 % TD_C) * PR + j1 / TD_C];
            const double vi = vj[0], wi = fma(al, vi, p0);
            for (int k = tid; k < m; k += TD_T) {  // each thread its own k of pf, rr
                const double wk = fma(al, vj[k], pf[k]);
                wf[k] = wk;
                const double r = fma(-wi, vj[k], fma(-vi, wk, rr[k]));
                rr[k] = r;
                if (k >= 2) sg = fma(r, r, sg);
            }
        }
        sg = warp_sum_d(sg);
        if (lane == 0) red[warp] = sg;
        __syncthreads();
        if (j + 1 > n - 2) {
            if (cr == 0 && tid == 0) {
                d[n - 1] = rr[0];
                Q[(size_t)(n - 1) + (size_t)(n - 1) * n] = rr[0];
            }
            break;
        }
        // dlarfg on x = rr[1..m): v_{j+1}; every warp forms the scalars itself
        const int len = m - 1;
        double tn, scal;
        bool nontriv;
        {
            const double sig = warp_sum_d(lane < TD_W ? red[lane] : 0.0);
            const double alpha = rr[1];
            double tt = 0.0, beta = alpha, sl = 0.0;
            if (sig > 0.0) {
                beta = -copysign(sqrt(fma(alpha, alpha, sig)), alpha);
                tt = (beta - alpha) * rcp_nr(beta);
                sl = rcp_nr(alpha - beta);
            }
            tn = tt;
            scal = sl;
            nontriv = sig > 0.0;
            if (cr == 0 && tid == 0) {
                d[j + 1] = rr[0];
                e[j + 1] = beta;
                tau[j + 1] = tt;
                Q[(size_t)(j + 1) + (size_t)(j + 1) * n] = rr[0];
                Q[(size_t)(j + 2) + (size_t)(j + 1) * n] = beta;
            }
        }
        for (int k = tid; k < len; k += TD_T) {
            const double v = k == 0 ? 1.0 : (nontriv ? rr[1 + k] * scal : 0.0);
            vn[k] = v;
            if (cr == 0 && k > 0) Q[(size_t)(j + 2 + k) + (size_t)(j + 1) * n] = v;
        }
        __syncthreads();
        // one pass over own rows i > j: the step-j update, then p_{j+1} on rows
        // i > j+1.  A warp takes its rows two at a time, sharing the loads of
        // v_j, w_j and v_{j+1} between them (vn[-1] is never used: column j+1
        // of the update does not enter p_{j+1})
        double kacc = 0.0;
        double* sbn = sb + (size_t)nxt * PR;
        for (int l0 = warp; l0 < R; l0 += 2 * TD_W) {
            const int l1 = l0 + TD_W;
            const int i0 = l0 * TD_C + cr, i1 = l1 * TD_C + cr;
            const bool h0 = i0 > j && i0 < n, h1 = l1 < R && i1 > j && i1 < n;  // warp-uniform
            const double vi0 = h0 ? vj[i0 - j - 1] : 0.0, wi0 = h0 ? wf[i0 - j - 1] : 0.0;
            const double vi1 = h1 ? vj[i1 - j - 1] : 0.0, wi1 = h1 ? wf[i1 - j - 1] : 0.0;
            double* a0 = rows + (size_t)l0 * np + j + 1;
            double* a1 = rows + (size_t)(h1 ? l1 : l0) * np + j + 1;
            double s0 = 0.0, s1 = 0.0;
            for (int k = lane; k < m; k += 32) {
                const double v = vj[k], w = wf[k], nv = k >= 1 ? vn[k - 1] : 0.0;
                if (h0) {
                    const double x = fma(-wi0, v, fma(-vi0, w, a0[k]));
                    a0[k] = x;
                    s0 = fma(x, nv, s0);
                }
                if (h1) {
                    const double x = fma(-wi1, v, fma(-vi1, w, a1[k]));
                    a1[k] = x;
                    s1 = fma(x, nv, s1);
                }
            }
            const double pv0 = (h0 && i0 >= j + 2) ? tn * warp_sum_d(s0) : 0.0;
            const double pv1 = (h1 && i1 >= j + 2) ? tn * warp_sum_d(s1) : 0.0;
            __syncwarp();  // column j+2 of these rows was updated by other lanes
            if (lane == 0) {
                if (h0 && i0 >= j + 2) kacc = fma(pv0, vn[i0 - j - 2], kacc);
                if (h1 && i1 >= j + 2) kacc = fma(pv1, vn[i1 - j - 2], kacc);
                // A(i, j+2) after this column's update, for the next look-ahead row
                sbn[l0] = pv0;
                sbn[R + 1 + l0] = i0 >= j + 2 && i0 < n ? rows[(size_t)l0 * np + j + 2] : 0.0;
                if (l1 < R) {
                    sbn[l1] = pv1;
                    sbn[R + 1 + l1] = i1 >= j + 2 && i1 < n ? rows[(size_t)l1 * np + j + 2] : 0.0;
                }
            }
        }
        if (lane == 0) red[warp] = kacc;
        __syncthreads();
        if (warp == 0) {
            const double s1 = warp_sum_d(lane < TD_W ? red[lane] : 0.0);
            if (lane == 0) sbn[R] = s1;
        }
        send(nxt);
        tcur = tn;
    }
    if (!ok) {
        // a receive that never completed: give the last column's copies one
        // more bounded wait before leaving, and report
        (void)mbar_wait(&bar[(n - 2) & 1], (uint32_t)(((n - 2) >> 1) & 1));
        atomicExch(err, 4);
    }
    cluster_sync();  // no CTA leaves while another may still read or copy into its shared memory
}

constexpr int BS_WARPS = 2;  // small blocks: the 480-odd warps spread over all SMs
constexpr int BS_PTS = 4;  // trial points per lane (independent Sturm chains)

// w[k] = k-th smallest eigenvalue of T (d, e), one warp per k, 32 x BS_PTS
// trial points per round, each counted with dlaebz's Sturm recurrence
// q_i = d_i - x - e_{i-1}^2 / q_{i-1} (eigenvalues below x = negative q,
// |q| <= pivmin replaced by -pivmin); aux[0] = |T|_1
__global__ void __launch_bounds__(32 * BS_WARPS) k_tri_bisect(const double* __restrict__ d,
                                                             const double* __restrict__ e, int n,
                                                             double* __restrict__ w, double* __restrict__ aux) {
    extern __shared__ double bsh[];
    double* sd = bsh;
    double* se2 = bsh + n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        sd[i] = d[i];
        se2[i] = i < n - 1 ? e[i] * e[i] : 0.0;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double glo = DBL_MAX, ghi = -DBL_MAX, em2 = 0.0, nrm1 = 0.0;
    for (int i = lane; i < n; i += 32) {
        const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
        glo = fmin(glo, sd[i] - r);
        ghi = fmax(ghi, sd[i] + r);
        em2 = fmax(em2, se2[i]);
        nrm1 = fmax(nrm1, fabs(sd[i]) + r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        glo = fmin(glo, __shfl_xor_sync(0xffffffffu, glo, o));
        ghi = fmax(ghi, __shfl_xor_sync(0xffffffffu, ghi, o));
        em2 = fmax(em2, __shfl_xor_sync(0xffffffffu, em2, o));
        nrm1 = fmax(nrm1, __shfl_xor_sync(0xffffffffu, nrm1, o));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) aux[0] = nrm1;
    const int k = blockIdx.x * BS_WARPS + warp;
    if (k >= n) return;
    const double pivmin = DBL_MIN * fmax(1.0, em2);
    const double tnorm = fmax(fabs(glo), fabs(ghi));
    double lo = glo - 2.0 * DBL_EPSILON * tnorm * n - 2.0 * pivmin;
    double hi = ghi + 2.0 * DBL_EPSILON * tnorm * n + 2.0 * pivmin;
    constexpr int NPT = 32 * BS_PTS;
    for (int round = 0; round < 64; ++round) {
        if (hi - lo <= 2.0 * DBL_EPSILON * tnorm + pivmin) break;  // dstebz's absolute tolerance
        const double h = hi - lo;
        double x[BS_PTS], q[BS_PTS];
        int c[BS_PTS];
#pragma unroll
        for (int u = 0; u < BS_PTS; ++u) {
            x[u] = lo + h * ((double)(lane * BS_PTS + u + 1) / (double)(NPT + 1));
            q[u] = sd[0] - x[u];
            if (fabs(q[u]) <= pivmin) q[u] = -pivmin;
            c[u] = q[u] < 0.0 ? 1 : 0;
        }
        for (int i = 1; i < n; ++i) {
            const double di = sd[i], ei = se2[i - 1];
#pragma unroll
            for (int u = 0; u < BS_PTS; ++u) {
                q[u] = di - x[u] - ei * rcp_nr(q[u]);  // |q| > pivmin >= DBL_MIN: normal
                if (fabs(q[u]) <= pivmin) q[u] = -pivmin;
                c[u] += q[u] < 0.0 ? 1 : 0;
            }
        }
        // first trial point (in x order) with more than k eigenvalues below it
        int first = NPT;
#pragma unroll
        for (int u = BS_PTS - 1; u >= 0; --u)
            if (c[u] > k) first = lane * BS_PTS + u;
        const int f = __reduce_min_sync(0xffffffffu, first);
        const double xf = f < NPT ? lo + h * ((double)(f + 1) / (double)(NPT + 1)) : hi;
        const double xb = f > 0 ? lo + h * ((double)f / (double)(NPT + 1)) : lo;
        const double nlo = fmax(lo, xb), nhi = fmin(hi, xf);
        if (nlo == lo && nhi == hi) break;  // the trial points no longer split the interval
        lo = nlo;
        hi = nhi;
    }
    if (lane == 0) w[k] = 0.5 * (lo + hi);
}

// Deterministic start vector entry in [-1, 1) (SplitMix64 of (eigenvalue, row))
__device__ __forceinline__ double start_entry(int j, int i) {
    unsigned long long z = ((unsigned long long)j << 32 | (unsigned)i) + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Eigenvectors of T into Z (columns in the order of w).  One warp per group
// of (nearly) equal eigenvalues, the vectors in registers: lane l holds rows
// l*IV_RPL .. l*IV_RPL + IV_RPL - 1.  Each solve of (T - x I) y = b
// eliminates with partial pivoting row by row (dgttrf's choices), the
// current row handed from lane to lane, keeping U's diagonal reciprocal,
// first and second super-diagonals and the transformed right-hand side in
// the owning lane, then back-substitutes in reverse lane order.
constexpr int IV_RPL = 20;  // rows per lane: n <= 640
constexpr int IV_WARPS = 4;

__global__ void __launch_bounds__(32 * IV_WARPS) k_tri_invit(const double* __restrict__ d,
                                                            const double* __restrict__ e,
                                                            const double* __restrict__ w,
                                                            const double* __restrict__ aux, int n,
                                                            double* __restrict__ Z, int ldz) {
    extern __shared__ double ish[];  // d, e of T for the block's warps
    double* sd = ish;
    double* se = ish + n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        sd[i] = d[i];
        se[i] = i < n - 1 ? e[i] : 0.0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int k = blockIdx.x * IV_WARPS + (threadIdx.x >> 5);
    if (k >= n) return;
    const double onenrm = aux[0];
    const double gtol = 1e-10 * onenrm;  // groups solved with Gram-Schmidt
    if (k > 0 && w[k] - w[k - 1] <= gtol) return;  // inside a group started below
    const double tol = DBL_EPSILON * onenrm;
    const int i0 = lane * IV_RPL;
    double ri[IV_RPL], u1[IV_RPL], u2[IV_RPL], y[IV_RPL];
    double xjm = 0.0;
    for (int j = k; j < n; ++j) {
        if (j > k && w[j] - w[j - 1] > gtol) break;
        const bool grp = j > k || (j + 1 < n && w[j + 1] - w[j] <= gtol);
        double xj = w[j];
        if (j > k) {
            const double pertol = 10.0 * fabs(DBL_EPSILON * xj);
            if (xj - xjm < pertol) xj = xjm + pertol;
        }
        xjm = xj;
#pragma unroll
        for (int r = 0; r < IV_RPL; ++r) y[r] = i0 + r < n ? start_entry(j, i0 + r) : 0.0;
        const int nsolve = grp ? 4 : 2;
        double nrm2 = 0.0;
        for (int its = 0; its < nsolve; ++its) {
            const double bnext = __shfl_down_sync(0xffffffffu, y[0], 1);  // b of the next lane's first row
            // forward elimination; current row (D, C1, R) handed lane to lane
            double D = 0.0, C1 = 0.0, R = 0.0;
            for (int l = 0; l < 32 && l * IV_RPL < n; ++l) {
                if (lane == l) {
                    if (l == 0) {
                        D = sd[0] - xj;
                        C1 = se[0];
                        R = y[0];
                    }
#pragma unroll
                    for (int r = 0; r < IV_RPL; ++r) {
                        const int i = i0 + r;
                        if (i >= n - 1) break;
                        const double sub = se[i];          // T(i+1, i)
                        const double dn = sd[i + 1] - xj;  // T(i+1, i+1)
                        const double up = se[i + 1];       // T(i+1, i+2) (0 past the end)
                        const double bn = r + 1 < IV_RPL ? y[r + 1] : bnext;
                        double ud, v1, v2, rf;
                        if (fabs(D) >= fabs(sub)) {  // pivot on the current row
                            const double f = fabs(D) >= DBL_MIN ? sub * rcp_nr(D) : (D != 0.0 ? sub / D : 0.0);
                            ud = D;
                            v1 = C1;
                            v2 = 0.0;
                            rf = R;
                            D = dn - f * C1;
                            C1 = up;
                            R = bn - f * R;
                        } else {  // interchange: the next row is the pivot
                            const double f = fabs(sub) >= DBL_MIN ? D * rcp_nr(sub) : D / sub;
                            ud = sub;
                            v1 = dn;
                            v2 = up;
                            rf = bn;
                            D = C1 - f * dn;
                            C1 = -f * up;
                            R = R - f * bn;
                        }
                        if (fabs(ud) < tol) ud = copysign(tol, ud);
                        ri[r] = fabs(ud) >= DBL_MIN ? rcp_nr(ud) : 1.0 / ud;
                        u1[r] = v1;
                        u2[r] = v2;
                        y[r] = rf;
                    }
                }
                D = __shfl_sync(0xffffffffu, D, l);
                C1 = __shfl_sync(0xffffffffu, C1, l);
                R = __shfl_sync(0xffffffffu, R, l);
            }
            // last row
            if (fabs(D) < tol) D = copysign(tol, D);
            const int ln = (n - 1) / IV_RPL;  // lane holding the last row
            // back substitution in reverse lane order, carrying y(i+1), y(i+2)
            double y1 = R * rcp_nr(D), y2 = 0.0;  // |D| >= tol
            for (int l = ln; l >= 0; --l) {
                if (lane == l) {
#pragma unroll
                    for (int r = IV_RPL - 1; r >= 0; --r) {
                        const int i = i0 + r;
                        if (i > n - 1) continue;
                        if (i == n - 1) {
                            y[r] = y1;
                            continue;
                        }
                        const double v = (y[r] - u1[r] * y1 - u2[r] * y2) * ri[r];
                        y[r] = v;
                        y2 = y1;
                        y1 = v;
                    }
                }
                y1 = __shfl_sync(0xffffffffu, y1, l);
                y2 = __shfl_sync(0xffffffffu, y2, l);
            }
            // Gram-Schmidt against the group's earlier vectors
            for (int p = k; p < j; ++p) {
                double dot = 0.0;
#pragma unroll
                for (int r = 0; r < IV_RPL; ++r)
                    if (i0 + r < n) dot = fma(Z[i0 + r + (long)p * ldz], y[r], dot);
                dot = warp_sum_d(dot);
#pragma unroll
                for (int r = 0; r < IV_RPL; ++r)
                    if (i0 + r < n) y[r] = fma(-dot, Z[i0 + r + (long)p * ldz], y[r]);
            }
            double ss = 0.0;
#pragma unroll
            for (int r = 0; r < IV_RPL; ++r) ss = fma(y[r], y[r], ss);
            nrm2 = warp_sum_d(ss);
            const double sc1 = 1.0 / sqrt(nrm2);  // the next right-hand side is y / |y|
#pragma unroll
            for (int r = 0; r < IV_RPL; ++r) y[r] *= sc1;
        }
        // the largest component positive (dstein's convention); lowest row on ties
        double big = -1.0;
        int at = n;
#pragma unroll
        for (int r = 0; r < IV_RPL; ++r)
            if (i0 + r < n && fabs(y[r]) > big) {
                big = fabs(y[r]);
                at = i0 + r;
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, big, o);
            const int oa = __shfl_xor_sync(0xffffffffu, at, o);
            if (ob > big || (ob == big && oa < at)) {
                big = ob;
                at = oa;
            }
        }
        double vat = 0.0;
#pragma unroll
        for (int r = 0; r < IV_RPL; ++r)
            if (i0 + r == at) vat = y[r];
        vat = __shfl_sync(0xffffffffu, vat, at / IV_RPL);
        const double sg = vat < 0.0 ? -1.0 : 1.0;
#pragma unroll
        for (int r = 0; r < IV_RPL; ++r)
            if (i0 + r < n) Z[i0 + r + (long)j * ldz] = y[r] * sg;
    }
}

static size_t td_smem_bytes(int n) { return TdLayout(n).total * sizeof(double); }

int syevd_fast(double* A, int n, double* W, cublasFillMode_t uplo) {
    Context& c = ctx();
    if (n < 3 || n > 32 * IV_RPL) return RSDFT_EUNSUP;
    const size_t smem = td_smem_bytes(n);
    if (c.max_smem_optin < 0)
        RS_CUDA(cudaDeviceGetAttribute(&c.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
    if (smem > (size_t)c.max_smem_optin || ormtr_smem_bytes(n) > (size_t)c.max_smem_optin) return RSDFT_EUNSUP;
    if ((int)smem > c.smem_optin[(const void*)k_sytrd]) {
        RS_CUDA(cudaFuncSetAttribute(k_sytrd, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        RS_CHECK(set_smem_optin((const void*)k_sytrd, (int)smem));
        c.sytrd_clusters = -1;
    }
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = TD_C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(TD_C);
    cfg.blockDim = dim3(TD_T);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c.stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (c.sytrd_clusters < 0) {
        if (cudaOccupancyMaxActiveClusters(&c.sytrd_clusters, k_sytrd, &cfg) != cudaSuccess) {
            cudaGetLastError();
            c.sytrd_clusters = 0;
        }
    }
    if (c.sytrd_clusters < 1) return RSDFT_EUNSUP;

    double *Q = nullptr, *dd = nullptr, *ws = nullptr;
    RS_CHECK(workspace_t("eig_Q", (size_t)n * n, &Q));
    RS_CHECK(workspace_t("eig_dd", (size_t)4 * n + 8, &dd));
    RS_CHECK(workspace_t("eig_ws", (size_t)2 * n * n, &ws));
    double* d = dd;
    double* e = dd + n;
    double* tau = dd + 2 * n;
    double* aux = dd + 3 * n;
    ++g_kernel_launches;
    RS_CUDA(cudaLaunchKernelEx(&cfg, k_sytrd, (const double*)A, n, n, uplo == CUBLAS_FILL_MODE_UPPER ? 1 : 0, Q, d,
                               e, tau, c.err_flag));
    RS_LAUNCH();
    launch(k_tri_bisect, div_up(n, BS_WARPS), 32 * BS_WARPS, (size_t)2 * n * sizeof(double), c.stream,
           (const double*)d, (const double*)e, n, W, aux);
    RS_LAUNCH();
    launch(k_tri_invit, div_up(n, IV_WARPS), 32 * IV_WARPS, (size_t)2 * n * sizeof(double), c.stream,
           (const double*)d, (const double*)e, (const double*)W, (const double*)aux, n, A, n);
    RS_LAUNCH();
    // two Newton-Schulz steps on Z (in A), through Z2 (in ws)
    {
        const double one = 1.0, zero = 0.0, half = -0.5, c15 = 1.5;
        double* G = ws;
        double* Z2 = ws + (size_t)n * n;
        double* src = A;
        double* dst = Z2;
        for (int it = 0; it < 2; ++it) {
            RS_CHECK(dmma_gemm(true, n, n, n, one, src, n, src, n, zero, G, n));
            RS_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToDevice, c.stream));
            RS_CHECK(dmma_gemm(false, n, n, n, half, src, n, G, n, c15, dst, n));
            double* t = src;
            src = dst;
            dst = t;
        }
        (void)src;  // two steps: the result is back in A
    }
    return ormtr_lower_device(Q, tau, n, A);
}

}  // namespace rsdft
