// FP64 contractions of the plain form on the FP64 tensor cores of sm_100a
// (mma.sync.m8n8k4 .f64, the DMMA path; tcgen05 has no FP64 kind).
//
// One kernel, k_dmma, computes tiles of C'(m, n) = sum_k A'(m, k) B'(k, n)
// for the two shapes of the eigensolver and every small product of the
// Rayleigh-Ritz step:
//   * Gram matrices psi^T Y (gram_schmidt_t_module.f90:187,
//     subspace_diag_la_module.f90:96, subspace_mate_sl_module.f90:27-366):
//     A' = psi^T, B' = Y, K = the grid; split-K over the grid, each CTA's
//     tile sum written whole, the splits added in a fixed order by
//     k_dmma_reduce (bit-reproducible);
//   * rotations psi V (gram_schmidt_t_module.f90:198, subspace_diag_la_module
//     .f90:200, subspace_rotv_sl_module.f90:92): computed transposed,
//     (psi V)^T = V^T psi^T, so that both tensor-core operands are read from
//     shared memory in the layout the grid dimension arrives in;
//   * the small dense NN / TN products of the Rayleigh-Ritz step and of the
//     eigensolver's Newton-Schulz steps.
// A' is always staged k-contiguous ([m][k] rows of BK + 4 doubles, so the
// eight rows a fragment load touches fall on distinct 32-byte bank groups);
// B' is staged [n][k] when the caller's B is k-contiguous and [k][n] when it
// is n-contiguous (rows of BN + 8 doubles).  Operand tiles arrive through
// 8-byte cp.async copies (any leading dimension), three stages deep.
#include <algorithm>

#include "common.cuh"
#include "dmma.cuh"

namespace rsdft {

namespace {

struct DmmaArgs {
    const double* A;  // A'(m, k) = A[m * lda + k]
    long lda;
    const double* B;  // B'(k, n) = B[k + n * ldb] (KMAJOR) or B[k * ldb + n]
    long ldb;
    double* C;        // C'(m, n) = C[m * ldcm + n * ldcn]
    long ldcm, ldcn;
    int M, N;
    long K;
    long kchunk;      // K values per split (blockIdx.y), a multiple of DM_BK
    double alpha, beta;
    double* partial;  // split-K: raw tile sums [split][tile][BM][BN]; C unused
    int sym;          // only tiles tm <= tn (a symmetric product)
    int ntm, ntiles;
};

constexpr int DM_BK = 16;  // K per stage (four m8n8k4 steps)
constexpr int DM_NS = 3;   // cp.async stages

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    const int n = valid ? 8 : 0;  // 0 source bytes: the 8 destination bytes are zero-filled
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async16(double* dst, const double* src, bool valid) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// D (8x8) += A (8x4, row) B (4x8, col); per lane: a = A[lane/4][lane%4],
// b = B[lane%4][lane/4], d = D[lane/4][2 (lane%4) + {0, 1}]
__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void tile_of(const DmmaArgs& g, int t, int& tm, int& tn) {
    if (!g.sym) {
        tm = t % g.ntm;
        tn = t / g.ntm;
        return;
    }
    tn = 0;  // upper triangle, column by column: (0,0), (0,1), (1,1), (0,2), ...
    while (t > tn) {
        t -= tn + 1;
        ++tn;
    }
    tm = t;
}

template <int BM, int BN, int WM, int WN, bool KMAJOR, bool VEC, int CPS>
__global__ void __launch_bounds__(32 * WM * WN, CPS) k_dmma(DmmaArgs g) {
    constexpr int BK = DM_BK, NS = DM_NS, NT = 32 * WM * WN;
    constexpr int SA = BK + 4;
    constexpr int SB = KMAJOR ? BK + 4 : BN + 8;
    constexpr int AST = BM * SA;
    constexpr int BST = KMAJOR ? BN * SB : BK * SB;
    constexpr int TM = BM / WM / 8, TN = BN / WN / 8;  // 8x8 tiles per warp
    static_assert(TM >= 1 && TN >= 1 && BM % (8 * WM) == 0 && BN % (8 * WN) == 0, "warp tiling");
    extern __shared__ __align__(16) double dsm[];
    double* As = dsm;
    double* Bs = dsm + NS * AST;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm0 = (warp % WM) * (BM / WM), wn0 = (warp / WM) * (BN / WN);
    int tm, tn;
    tile_of(g, blockIdx.x, tm, tn);
    const int m0 = tm * BM, n0 = tn * BN;
    const long k0 = (long)blockIdx.y * g.kchunk;
    const long k1 = min(g.K, k0 + g.kchunk);
    const int nkb = k1 > k0 ? (int)((k1 - k0 + BK - 1) / BK) : 0;

    // operand tiles: 8-byte copies, or 16-byte ones (pairs of doubles along
    // the contiguous dimension) when every row start is 16-byte aligned and
    // the pair is wholly inside or outside the valid range (K, M, N even)
    auto load_stage = [&](int s, int kb) {
        const long kb0 = k0 + (long)kb * BK;
        double* as = As + s * AST;
        constexpr int V = VEC ? 2 : 1;
        for (int e = threadIdx.x; e < BM * BK / V; e += NT) {
            const int r = e / (BK / V), kk = (e % (BK / V)) * V;
            const long k = kb0 + kk;
            const bool ok = m0 + r < g.M && k < k1;
            const double* src = ok ? g.A + (long)(m0 + r) * g.lda + k : g.A;
            if (VEC) cp_async16(as + r * SA + kk, src, ok);
            else cp_async8(as + r * SA + kk, src, ok);
        }
        double* bs = Bs + s * BST;
        if (KMAJOR) {
            for (int e = threadIdx.x; e < BN * BK / V; e += NT) {
                const int r = e / (BK / V), kk = (e % (BK / V)) * V;
                const long k = kb0 + kk;
                const bool ok = n0 + r < g.N && k < k1;
                const double* src = ok ? g.B + k + (long)(n0 + r) * g.ldb : g.B;
                if (VEC) cp_async16(bs + r * SB + kk, src, ok);
                else cp_async8(bs + r * SB + kk, src, ok);
            }
        } else {
            for (int e = threadIdx.x; e < BN * BK / V; e += NT) {
                const int kk = e / (BN / V), c = (e % (BN / V)) * V;
                const long k = kb0 + kk;
                const bool ok = n0 + c < g.N && k < k1;
                const double* src = ok ? g.B + k * g.ldb + (n0 + c) : g.B;
                if (VEC) cp_async16(bs + kk * SB + c, src, ok);
                else cp_async8(bs + kk * SB + c, src, ok);
            }
        }
    };

    double acc[TM][TN][2];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < NS - 1; ++s) {
        if (s < nkb) load_stage(s, s);
        cp_async_commit();
    }
    const int fr = lane >> 2, fc = lane & 3;
    for (int kb = 0; kb < nkb; ++kb) {
        cp_async_wait<NS - 2>();
        __syncthreads();  // stage kb has landed; every warp is done with stage kb - 1
        if (kb + NS - 1 < nkb) load_stage((kb + NS - 1) % NS, kb + NS - 1);
        cp_async_commit();
        const double* as = As + (kb % NS) * AST + (wm0 + fr) * SA + fc;
        const double* bs = Bs + (kb % NS) * BST + (KMAJOR ? (wn0 + fr) * SB + fc : fc * SB + wn0 + fr);
#pragma unroll
        for (int ks = 0; ks < BK; ks += 4) {
            double a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = as[8 * i * SA + ks];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = KMAJOR ? bs[8 * j * SB + ks] : bs[ks * SB + 8 * j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) dmma_884(acc[i][j], a[i], b[j]);
        }
    }
    cp_async_wait<0>();

    if (g.partial) {
        double* P = g.partial + ((size_t)blockIdx.y * g.ntiles + blockIdx.x) * (size_t)(BM * BN);
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) {
                const int r = wm0 + 8 * i + fr, c = wn0 + 8 * j + 2 * fc;
                *reinterpret_cast<double2*>(P + (size_t)r * BN + c) = make_double2(acc[i][j][0], acc[i][j][1]);
            }
        return;
    }
    const bool pair = g.ldcn == 1 && (g.ldcm % 2) == 0 && (reinterpret_cast<uintptr_t>(g.C) % 16) == 0;
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int m = m0 + wm0 + 8 * i + fr, n = n0 + wn0 + 8 * j + 2 * fc;
            if (m >= g.M) continue;
            double* o = g.C + (long)m * g.ldcm + (long)n * g.ldcn;
            if (pair && n + 1 < g.N) {
                double2 v = make_double2(g.alpha * acc[i][j][0], g.alpha * acc[i][j][1]);
                if (g.beta != 0.0) {
                    const double2 old = *reinterpret_cast<const double2*>(o);
                    v.x = fma(g.beta, old.x, v.x);
                    v.y = fma(g.beta, old.y, v.y);
                }
                *reinterpret_cast<double2*>(o) = v;
                continue;
            }
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                if (n + e < g.N) {
                    double* oe = o + (long)e * g.ldcn;
                    const double v = g.alpha * acc[i][j][e];
                    *oe = g.beta == 0.0 ? v : fma(g.beta, *oe, v);
                }
            }
        }
}

// C(i, j) = alpha * sum over splits (fixed order) of the raw tile sums;
// symmetric products read tiles below the diagonal transposed from the upper
// ones; symmetrize returns alpha/2 (G + G^T).
template <int BM, int BN>
__global__ void k_dmma_reduce(const double* __restrict__ P, int nsplit, int ntiles, int ntm, int sym, int m,
                              double alpha, int symmetrize, double* __restrict__ C, long ldc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= m) return;
    auto fetch = [&](int r, int c) {
        int tm = r / BM, tn = c / BN;
        if (sym && tm > tn) {
            const int t = r;
            r = c;
            c = t;
            tm = r / BM;
            tn = c / BN;
        }
        const int t = sym ? tn * (tn + 1) / 2 + tm : tm + tn * ntm;
        const size_t off = (size_t)t * (BM * BN) + (size_t)(r - tm * BM) * BN + (c - tn * BN);
        double s = 0.0;
        for (int z = 0; z < nsplit; ++z) s += P[(size_t)z * ntiles * (BM * BN) + off];
        return s;
    };
    double v = fetch(i, j);
    if (symmetrize) v = 0.5 * (v + fetch(j, i));
    C[(long)j * ldc + i] = alpha * v;
}

template <int BM, int BN, int WM, int WN, bool KMAJOR, int CPS>
int launch_dmma(const DmmaArgs& g, int nsplit, bool vec) {
    constexpr int SA = DM_BK + 4;
    constexpr int SB = KMAJOR ? DM_BK + 4 : BN + 8;
    constexpr size_t smem = (size_t)DM_NS * (BM * SA + (KMAJOR ? BN * SB : DM_BK * SB)) * sizeof(double);
    const void* fn = vec ? (const void*)k_dmma<BM, BN, WM, WN, KMAJOR, true, CPS>
                         : (const void*)k_dmma<BM, BN, WM, WN, KMAJOR, false, CPS>;
    RS_CHECK(set_smem_optin(fn, (int)smem));
    if (vec)
        launch(k_dmma<BM, BN, WM, WN, KMAJOR, true, CPS>, dim3(g.ntiles, nsplit), 32 * WM * WN, smem, ctx().stream, g);
    else
        launch(k_dmma<BM, BN, WM, WN, KMAJOR, false, CPS>, dim3(g.ntiles, nsplit), 32 * WM * WN, smem, ctx().stream,
               g);
    RS_LAUNCH();
    return RSDFT_OK;
}

// 16-byte operand copies are exact when both operands' bases and leading
// dimensions keep every row start 16-byte aligned and the K, M, N limits
// are even (a pair of doubles is then wholly valid or wholly out of range)
bool vec_ok(const DmmaArgs& g) {
    auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) % 16) == 0; };
    return al(g.A) && al(g.B) && g.lda % 2 == 0 && g.ldb % 2 == 0 && g.K % 2 == 0 && g.M % 2 == 0 && g.N % 2 == 0 &&
           g.kchunk % 2 == 0;
}

}  // namespace

// Tall Gram: C (m x n, column-major, ldc) = alpha A^T B for A (K x m), B
// (K x n) column-major with leading dimension ld, K = kdim (the grid).
int dmma_gram(const double* A, const double* B, long ld, long kdim, int m, int n, double alpha, int symmetrize,
              double* C, long ldc, bool symmetric_product) {
    Context& c = ctx();
    constexpr int BM = 128, BN = 128;
    DmmaArgs g{};
    g.A = A;
    g.lda = ld;
    g.B = B;
    g.ldb = ld;
    g.M = m;
    g.N = n;
    g.K = kdim;
    g.ntm = div_up(m, BM);
    const int ntn = div_up(n, BN);
    // upper tiles only for a symmetric product: A^T A, or A^T (H A) of a
    // symmetric operator (its lower tiles equal the upper ones to rounding;
    // the diagonal tiles are symmetrised by the reduction)
    g.sym = (m == n && (A == B || (symmetric_product && symmetrize))) ? 1 : 0;
    g.ntiles = g.sym ? g.ntm * (g.ntm + 1) / 2 : g.ntm * ntn;
    // whole waves of CTAs (one per SM: 123 KB of stages): the largest split
    // count with tiles x splits <= 2 x SMs, K split evenly
    const int sms = c.num_sms > 0 ? c.num_sms : 148;
    const long kblocks = (kdim + DM_BK - 1) / DM_BK;
    int nsplit = (int)std::max<long>(1, std::min<long>(kblocks, (2L * sms) / g.ntiles));
    g.kchunk = ((kblocks + nsplit - 1) / nsplit) * DM_BK;
    nsplit = (int)((kdim + g.kchunk - 1) / g.kchunk);
    double* P = nullptr;
    RS_CHECK(workspace_t("dmma_partials", (size_t)nsplit * g.ntiles * BM * BN, &P));
    g.partial = P;
    RS_CHECK((launch_dmma<BM, BN, 4, 4, true, 1>(g, nsplit, vec_ok(g))));
    launch(k_dmma_reduce<BM, BN>, dim3(div_up(m, 128), n), 128, 0, c.stream, (const double*)P, nsplit, g.ntiles,
           g.ntm, g.sym, m, alpha, symmetrize, C, ldc);
    RS_LAUNCH();
    return RSDFT_OK;
}

// General product C = alpha op(A) B + beta C (column-major; op = A or A^T),
// C m x n, inner dimension k.  Computed as C^T = B^T op(A)^T, so the tensor-
// core A operand is B^T (k-contiguous in memory) and the B operand op(A)^T,
// which is k-contiguous for op = T ([n][k] staging) and row-contiguous for
// op = N ([k][n] staging).
int dmma_gemm(bool transA, long m, int n, int k, double alpha, const double* A, long lda, const double* B, long ldb,
              double beta, double* C, long ldc) {
    DmmaArgs g{};
    g.A = B;  // A'(j, kk) = B[kk + j ldb]
    g.lda = ldb;
    g.B = A;  // B'(kk, i) = op(A)(i, kk)
    g.ldb = lda;
    g.C = C;  // C'(j, i) = C[i + j ldc]
    g.ldcm = ldc;
    g.ldcn = 1;
    g.M = n;
    g.K = k;
    g.alpha = alpha;
    g.beta = beta;
    g.kchunk = ((long)k + DM_BK - 1) / DM_BK * DM_BK;
    if (m > 1L << 30) {
        set_error("dmma_gemm: m = %ld too large", m);
        return RSDFT_EINVAL;
    }
    g.N = (int)m;
    const bool vec = vec_ok(g);
    if (m >= 4096) {
        // tall output (a rotation psi V): 128 bands x 64 grid points per
        // CTA, eight warps of 32 x 32, two CTAs per SM so that one CTA's
        // operand prologue and store epilogue overlap the other's MMAs
        constexpr int BM = 128, BN = 64;
        g.ntm = div_up(n, BM);
        g.ntiles = g.ntm * div_up(m, BN);
        return transA ? launch_dmma<BM, BN, 4, 2, true, 2>(g, 1, vec) : launch_dmma<BM, BN, 4, 2, false, 2>(g, 1, vec);
    }
    // small dense products: 32 x 32 tiles, four warps
    constexpr int BM = 32, BN = 32;
    g.ntm = div_up(n, BM);
    g.ntiles = g.ntm * div_up(m, BN);
    return transA ? launch_dmma<BM, BN, 2, 2, true, 4>(g, 1, vec) : launch_dmma<BM, BN, 2, 2, false, 4>(g, 1, vec);
}

}  // namespace rsdft
