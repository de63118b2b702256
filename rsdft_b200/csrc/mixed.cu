// Mixed-precision contractions on the 5th-generation tensor cores (tcgen05).
//
// Operands are split into BF16 terms, x = x0 + x1 + x2 (x0 = bf16(x),
// x1 = bf16(x - x0), x2 = bf16(x - x0 - x1): 24 significant bits), or into
// two TF32 terms (x0 = tf32(x), x1 = tf32(x - x0): 22 bits), and a product is
// the sum of the term pairs with s + t < NT (NT = 3: six products,
// "split-BF16 x3 terms"; NT = 2: three products), every pair an exact
// BF16 x BF16 (kind::f16) or TF32 x TF32 (kind::tf32) product accumulated in
// FP32 in tensor memory.  A slice row of one K block is 64 bytes in both
// kinds (32 BF16 or 16 TF32 values), so the tiles, stages and descriptors
// are the same; only the MMA kind, the element count per block and the TMA
// element type differ.
//
// k_umma (one CTA = one 128 x BN output tile):
//   warp 0    TMA producer: per K block of 32, the NT slices of the A tile
//             (128 rows) and of the B tile (BN rows), 64-byte swizzle, into a
//             ring of NS shared-memory stages (full/empty mbarriers);
//   warp 1    allocates tensor memory; lane 0 issues the tcgen05.mma chain;
//   warps 2-9 epilogue (two warps per TMEM lane quadrant, half the columns
//             each).
// Two epilogues:
//   DRAIN (Gram matrices A^T B over the grid, K = ML): two TMEM accumulators;
//     every SEG K blocks the epilogue adds the FP32 segment into FP64
//     registers while the MMA fills the other accumulator, so FP32 rounding
//     never spans more than SEG*32 terms.  Each CTA covers a K range
//     (split-K) and writes an FP64 partial tile; k_reduce_tiles adds the
//     partials in a fixed order.
//   DIRECT (rotations psi V, K = MB): D(n, i) = sum_m V(m, n) psi(i, m) is
//     written to out(i, n) in FP64.  Persistent: one CTA per SM walks the
//     output tiles; two TMEM accumulators let the epilogue of one tile run
//     while the MMA chain of the next fills the other.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "mixed.cuh"
#include "vec16.cuh"
#include "tmap.cuh"
#include "umma.cuh"

namespace rsdft {

constexpr int UB_M = 128;      // tile rows (TMEM lanes)
constexpr int UB_K = 32;       // K block in BF16 values (64 bytes: one swizzle row)
constexpr int UB_KB = 64;      // K block in bytes, both element kinds
constexpr int U_EPI_WARPS = 8;
constexpr int U_THREADS = 32 * (2 + U_EPI_WARPS);
constexpr int U_SEG = 4;       // K blocks per FP32 accumulation segment (DRAIN)

__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16& h, __nv_bfloat16& m, __nv_bfloat16& l) {
    h = __float2bfloat16_rn((float)x);
    double r = x - (double)__bfloat162float(h);
    m = __float2bfloat16_rn((float)r);
    r -= (double)__bfloat162float(m);
    l = __float2bfloat16_rn((float)r);
}

// two TF32 terms of x (round to nearest, ties away: cvt.rna.tf32.f32), as
// FP32 bit patterns with the low 13 mantissa bits zero
__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(double x, uint32_t& h, uint32_t& l) {
    h = to_tf32((float)x);
    l = to_tf32((float)(x - (double)__uint_as_float(h)));
}

// TF32 versions of the three split kernels below: two slices of 4-byte
// values in the same layouts
template <typename TI>
__global__ void __launch_bounds__(256) k_split_cols_tf32(const TI* __restrict__ psi, long ld, int nb, long ml,
                                                         uint32_t* __restrict__ out) {
    const long n = ml * nb;
    const int b = blockIdx.y;
    const long k0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (k0 >= ml) return;
    const TI* src = psi + (long)b * ld + k0;
    uint32_t* o = out + (long)b * ml + k0;
    for (long k = 0; k < 4 && k0 + k < ml; ++k) {
        uint32_t h, l;
        split_tf32((double)src[k], h, l);
        o[k] = h;
        o[n + k] = l;
    }
}

template <typename TI>
__global__ void k_split_rows_tf32(const TI* __restrict__ psi, long ld, int nb, long ml, int mbk,
                                  uint32_t* __restrict__ out) {
    __shared__ double tile[32][33];
    const long i0 = (long)blockIdx.x * 32;
    const int m0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const long i = i0 + tx;
        const int m = m0 + r;
        tile[r][tx] = (i < ml && m < nb) ? (double)psi[(long)m * ld + i] : 0.0;
    }
    __syncthreads();
    const long n = ml * mbk;
    for (int r = ty; r < 32; r += 8) {
        const long i = i0 + r;
        const int m = m0 + tx;
        if (i < ml && m < mbk) {
            uint32_t h, l;
            split_tf32(tile[tx][r], h, l);
            const long e = i * mbk + m;
            out[e] = h;
            out[n + e] = l;
        }
    }
}

__global__ void k_split_small_tf32(const double* __restrict__ V, int mb, int ldv, int mbk, uint32_t* __restrict__ out) {
    const long n = (long)mb * mbk;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int col = (int)(e / mbk), m = (int)(e - (long)col * mbk);
        const double x = m < mb ? V[(long)col * ldv + m] : 0.0;
        uint32_t h, l;
        split_tf32(x, h, l);
        out[e] = h;
        out[n + e] = l;
    }
}

// slices[s][b][k] = term s of psi(k, b): same layout as psi (K-major per
// band).  grid (ceil(ml / 2048), nb): 8 consecutive k per thread, read as
// 16-byte pairs and written as one 16-byte group per slice when vec is set
// (ml % 8 == 0, ld even, 16-byte aligned bases).
template <typename TI>
__global__ void __launch_bounds__(256) k_split_cols(const TI* __restrict__ psi, long ld, int nb, long ml,
                                                    __nv_bfloat16* __restrict__ out, int vec) {
    const long n = ml * nb;
    const int b = blockIdx.y;
    const long k0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) * 8;
    if (k0 >= ml) return;
    const TI* src = psi + (long)b * ld + k0;
    __nv_bfloat16* o = out + (long)b * ml + k0;
    if (vec && k0 + 8 <= ml) {
        __nv_bfloat16 h[8], m[8], l[8];
        constexpr int W = 16 / (int)sizeof(TI);  // elements per 16-byte load
#pragma unroll
        for (int q = 0; q < 8 / W; ++q) {
            TI v[W];
            Vec16<TI>::get(*reinterpret_cast<const typename Vec16<TI>::t*>(src + W * q), v);
#pragma unroll
            for (int e = 0; e < W; ++e) split_bf16((double)v[e], h[W * q + e], m[W * q + e], l[W * q + e]);
        }
        *reinterpret_cast<uint4*>(o) = *reinterpret_cast<const uint4*>(h);
        *reinterpret_cast<uint4*>(o + n) = *reinterpret_cast<const uint4*>(m);
        *reinterpret_cast<uint4*>(o + 2 * n) = *reinterpret_cast<const uint4*>(l);
        return;
    }
    for (long k = 0; k < 8 && k0 + k < ml; ++k) {
        __nv_bfloat16 h, m, l;
        split_bf16((double)src[k], h, m, l);
        o[k] = h;
        o[n + k] = m;
        o[2 * n + k] = l;
    }
}

// slices[s][i][m] = term s of psi(i, m), m fastest, padded to mbk (zeros):
// the transpose that makes the band index the K dimension of a rotation
template <typename TI>
__global__ void k_split_rows(const TI* __restrict__ psi, long ld, int nb, long ml, int mbk,
                             __nv_bfloat16* __restrict__ out) {
    __shared__ double tile[32][33];
    const long i0 = (long)blockIdx.x * 32;
    const int m0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const long i = i0 + tx;
        const int m = m0 + r;
        tile[r][tx] = (i < ml && m < nb) ? (double)psi[(long)m * ld + i] : 0.0;
    }
    __syncthreads();
    const long n = ml * mbk;
    for (int r = ty; r < 32; r += 8) {
        const long i = i0 + r;
        const int m = m0 + tx;
        if (i < ml && m < mbk) {
            __nv_bfloat16 h, mm, l;
            split_bf16(tile[tx][r], h, mm, l);
            const long e = i * mbk + m;
            out[e] = h;
            out[n + e] = mm;
            out[2 * n + e] = l;
        }
    }
}

// slices[s][n][m] = term s of V(m, n) (V column-major mb x mb), padded to mbk
__global__ void k_split_small(const double* __restrict__ V, int mb, int ldv, int mbk, __nv_bfloat16* __restrict__ out) {
    const long n = (long)mb * mbk;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int col = (int)(e / mbk), m = (int)(e - (long)col * mbk);
        const double x = m < mb ? V[(long)col * ldv + m] : 0.0;
        __nv_bfloat16 h, mm, l;
        split_bf16(x, h, mm, l);
        out[e] = h;
        out[n + e] = mm;
        out[2 * n + e] = l;
    }
}

struct UmmaMaps {
    CUtensorMap a, b;  // 3-D: {K, rows, slice}
};

struct UmmaArgs {
    int kblocks;       // total K blocks of 32
    int kb_per_split;  // K blocks per CTA (DRAIN)
    int ntm, ntn;      // tiles along M (A rows) and N (B rows)
    int sym;           // DRAIN: only tiles with tm <= tn
    int npairs;
    double* partial;   // DRAIN: [split][pair][BN][128]
    double* out;       // DIRECT: out[(n) * ldo + i]
    long ldo;
    int mrows, nrows;  // valid rows of A and B
    int* err;
};

__device__ __forceinline__ void pair_tiles(const UmmaArgs& g, int pair, int& tm, int& tn) {
    if (!g.sym) {
        tm = pair % g.ntm;
        tn = pair / g.ntm;
        return;
    }
    int r = pair;
    tn = 0;
    while (r >= tn + 1) {
        r -= tn + 1;
        ++tn;
    }
    tm = r;
}

template <int BN, int NT, int NS, bool DRAIN, bool BMN, bool TF = false>
__global__ void __launch_bounds__(U_THREADS, 1) k_umma(const __grid_constant__ UmmaMaps maps, UmmaArgs g) {
    static_assert(!(TF && BMN), "TF32 operands are K-major");
    constexpr int ABYTES = UB_M * UB_KB;  // one A slice tile
    constexpr int BBYTES = BN * UB_KB;
    constexpr int UKE = TF ? UB_KB / 4 : UB_K;  // K values per block
    constexpr int STAGE = NT * (ABYTES + BBYTES);
    // Accumulators, double-buffered between the MMA chain and the epilogue.
    // DRAIN: two per buffer, one for the hi x hi product and one for the
    // smaller cross products (the FP32 accumulation truncates; keeping the
    // dominant term's chain short keeps that bias near 2^-24 x 2 U_SEG
    // instead of x 6 x 2 U_SEG).  DIRECT: one per buffer, so the epilogue of
    // one output tile overlaps the MMA chain of the next.
    constexpr int NACC = DRAIN ? 4 : 2;
    constexpr int TCOLS = NACC * BN;  // 512 for BN = 128 (DRAIN) and BN = 256 (DIRECT)
    static_assert(TCOLS <= 512, "tensor memory holds 512 columns");
    constexpr uint32_t IDESC = TF ? umma_idesc_tf32(UB_M, BN) : umma_idesc_bf16(UB_M, BN, BMN);
    // MN-major B (BMN): the tile is BN / 32 boxes of 32 N values x UB_K K rows
    constexpr uint32_t B_LBO = 32 * UB_K * 2, B_SBO = 8 * 64;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)NS * STAGE);
    uint64_t* empty = full + NS;
    uint64_t* accf = empty + NS;
    uint64_t* acce = accf + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(acce + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // Work units, each ending in one accumulator hand-off: DRAIN, the K
    // segments of U_SEG blocks of this CTA's (tile, split); DIRECT, the output
    // tiles blockIdx.x, blockIdx.x + gridDim.x, ... (tm fastest, so CTAs
    // running together share B tiles in L2), each over all K blocks.
    int tm0 = 0, tn0 = 0, kb0 = 0, kb1 = g.kblocks, nunits;
    if (DRAIN) {
        pair_tiles(g, blockIdx.x, tm0, tn0);
        kb0 = blockIdx.y * g.kb_per_split;
        kb1 = min(kb0 + g.kb_per_split, g.kblocks);
        nunits = (max(kb1 - kb0, 0) + U_SEG - 1) / U_SEG;
    } else {
        const int ntiles = g.ntm * g.ntn;
        nunits = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    }
    auto unit = [&](int u, int& tm, int& tn, int& ka, int& kz) {
        if (DRAIN) {
            tm = tm0;
            tn = tn0;
            ka = kb0 + u * U_SEG;
            kz = min(ka + U_SEG, kb1);
        } else {
            const int t = (int)blockIdx.x + u * (int)gridDim.x;
            tm = t % g.ntm;
            tn = t / g.ntm;
            ka = 0;
            kz = g.kblocks;
        }
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], U_EPI_WARPS);
        }
        mbar_fence_init();
    }
    if (warp == 1) {
        tmem_alloc(tslot, TCOLS);
        tmem_relinquish();
        tc_fence_before();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    bool ok = true;

    if (warp == 0) {
        // ------------------------------------------------------ TMA producer
        if (lane == 0) {
            int it = 0;
            for (int u = 0; u < nunits && ok; ++u) {
                int tm, tn, ka, kz;
                unit(u, tm, tn, ka, kz);
                for (int kb = ka; kb < kz; ++kb, ++it) {
                    const int s = it % NS;
                    if (it >= NS && !mbar_wait(&empty[s], ((it / NS) - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    unsigned char* st = smem + (size_t)s * STAGE;
                    mbar_arrive_expect_tx(&full[s], STAGE);
                    const int k = kb * UKE;
#pragma unroll
                    for (int t = 0; t < NT; ++t) {
                        // the maps are rank 4 ({K, rows, slice, 1}): 4-D loads, w = 0
                        tma_load_4d(st + t * ABYTES, &maps.a, k, tm * UB_M, t, 0, &full[s]);
                        if (BMN)  // map {32, K, N / 32, slice}
                            tma_load_4d(st + NT * ABYTES + t * BBYTES, &maps.b, 0, k, tn * (BN / 32), t, &full[s]);
                        else
                            tma_load_4d(st + NT * ABYTES + t * BBYTES, &maps.b, k, tn * BN, t, 0, &full[s]);
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------- MMA issuer
        if (lane == 0) {
            int it = 0;
            for (int u = 0; u < nunits && ok; ++u) {
                int tm, tn, ka, kz;
                unit(u, tm, tn, ka, kz);
                const int b = u & 1;
                if (u >= 2 && !mbar_wait(&acce[b], ((u >> 1) - 1) & 1)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tbase + (uint32_t)((DRAIN ? 2 * b : b) * BN);
                const uint32_t dx = DRAIN ? d + (uint32_t)BN : d;  // cross products
                bool first = true, firstx = true;
                for (int kb = ka; kb < kz; ++kb, ++it) {
                    const int s = it % NS;
                    if (!mbar_wait(&full[s], (it / NS) & 1)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + (size_t)s * STAGE);
                    const uint32_t sb = sa + NT * ABYTES;
#pragma unroll
                    for (int p = 0; p < (NT == 3 ? 6 : 3); ++p) {
                        const int ta = p == 0 ? 0 : p == 1 ? 0 : p == 2 ? 1 : p == 3 ? 0 : p == 4 ? 1 : 2;
                        const int tb = p == 0 ? 0 : p == 1 ? 1 : p == 2 ? 0 : p == 3 ? 2 : p == 4 ? 1 : 0;
#pragma unroll
                        for (int kk = 0; kk < 2; ++kk) {  // two MMAs of 32 bytes of K
                            const uint64_t ad = umma_desc_sw64(sa + ta * ABYTES + kk * 32);
                            const uint64_t bd =
                                BMN ? umma_desc_mn_sw64(sb + tb * BBYTES + kk * 16 * 64, B_LBO, B_SBO)
                                    : umma_desc_sw64(sb + tb * BBYTES + kk * 32);
                            const uint32_t dd = (DRAIN && p > 0) ? dx : d;
                            const uint32_t accum = (DRAIN && p > 0) ? (firstx ? 0u : 1u) : (first ? 0u : 1u);
                            if (TF)
                                umma_tf32(dd, ad, bd, IDESC, accum);
                            else
                                umma_bf16(dd, ad, bd, IDESC, accum);
                            if (DRAIN && p > 0)
                                firstx = false;
                            else
                                first = false;
                        }
                    }
                    umma_commit(&empty[s]);
                }
                umma_commit(&accf[b]);
            }
        }
    } else {
        // ---------------------------------------------------------- epilogue
        const int q = warp & 3;                 // TMEM lane quadrant of this warp
        const int h = (warp - 2) >> 2;          // column half
        const int row = 32 * q + lane;          // tile row (TMEM lane)
        constexpr int CW = BN / 2;              // columns per warp
        double acc[DRAIN ? CW : 1];
        if (DRAIN) {
#pragma unroll
            for (int c = 0; c < CW; ++c) acc[c] = 0.0;
        }
        for (int u = 0; u < nunits; ++u) {
            int tm, tn, ka, kz;
            unit(u, tm, tn, ka, kz);
            const int b = u & 1;
            if (!mbar_wait(&accf[b], (u >> 1) & 1)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t tq = tbase + ((uint32_t)(32 * q) << 16);
            if (DRAIN) {
#pragma unroll
                for (int c0 = 0; c0 < CW; c0 += 32) {
                    uint32_t r[32];
                    const uint32_t ta = tq + (uint32_t)(2 * b * BN + h * CW + c0);
                    tmem_ld_x32(ta, r);  // hi x hi
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 32; ++j) acc[c0 + j] += (double)__uint_as_float(r[j]);
                    tmem_ld_x32(ta + (uint32_t)BN, r);  // cross products
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 32; ++j) acc[c0 + j] += (double)__uint_as_float(r[j]);
                }
            } else {
                // 32 x 32 blocks (TMEM lane = band, column = grid point) transposed
                // in registers by a shuffle butterfly, so that each store
                // instruction writes 32 consecutive grid points of one band
                const int n0 = tm * UB_M + 32 * q;  // first band of this warp's block
#pragma unroll
                for (int c0 = 0; c0 < CW; c0 += 32) {
                    uint32_t r[32];
                    tmem_ld_x32(tq + (uint32_t)(b * BN + h * CW + c0), r);
                    tmem_ld_wait();
#pragma unroll
                    for (int sft = 16; sft >= 1; sft >>= 1) {
                        const bool upper = (lane & sft) != 0;
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            if (j & sft) continue;
                            const uint32_t send = upper ? r[j] : r[j + sft];
                            const uint32_t recv = __shfl_xor_sync(0xffffffffu, send, sft);
                            if (upper)
                                r[j] = recv;
                            else
                                r[j + sft] = recv;
                        }
                    }
                    // lane: grid point i0 + lane; r[j]: band n0 + j
                    const int i = tn * BN + h * CW + c0 + lane;
                    if (i < g.nrows) {
                        double* o = g.out + (size_t)n0 * g.ldo + i;
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (n0 + j < g.mrows) o[(size_t)j * g.ldo] = (double)__uint_as_float(r[j]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[b]);
        }
        if (DRAIN && ok) {
            double* P = g.partial + ((size_t)blockIdx.y * g.npairs + blockIdx.x) * (size_t)(BN * UB_M);
#pragma unroll
            for (int c = 0; c < CW; ++c) P[(size_t)(h * CW + c) * UB_M + row] = acc[c];
        }
    }
    if (!ok) atomicExch(g.err, 2);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tbase, TCOLS);
    }
}

// C(i, j) = alpha * sum_split P (sym: symmetric part); tiles with tm > tn of a
// symmetric product are read transposed from tile (tn, tm)
__global__ void k_reduce_tiles(const double* __restrict__ P, int nsplit, int npairs, int ntm, int sym, int bn, int m,
                               double alpha, int symmetrize, double* __restrict__ C) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= m) return;
    auto fetch = [&](int r, int c) {  // full product element (r, c)
        int tm = r / UB_M, tn = c / bn, rr = r % UB_M, cc = c % bn;
        if (sym && tm > tn) {
            const int t = r;
            r = c;
            c = t;
            tm = r / UB_M;
            tn = c / bn;
            rr = r % UB_M;
            cc = c % bn;
        }
        const int pair = sym ? tn * (tn + 1) / 2 + tm : tm + tn * ntm;
        double s = 0.0;
        for (int k = 0; k < nsplit; ++k)
            s += P[((size_t)k * npairs + pair) * (size_t)(bn * UB_M) + (size_t)cc * UB_M + rr];
        return s;
    };
    double v = fetch(i, j);
    if (symmetrize) v = 0.5 * (v + fetch(j, i));
    C[(size_t)j * m + i] = alpha * v;
}

// Tensor map over the slices [s][rows][k] of a split (k fastest): 3 BF16 or
// 2 TF32 slices, a 64-byte K block per row, 64-byte swizzle
static int map3(CUtensorMap* mp, const void* base, long k, long rows, int box_rows, bool tf32 = false) {
    const unsigned long long eb = tf32 ? 4 : 2, ns = tf32 ? 2 : 3;
    const unsigned long long dims[4] = {(unsigned long long)k, (unsigned long long)rows, ns, 1ull};
    const unsigned long long strides[3] = {(unsigned long long)k * eb, (unsigned long long)k * rows * eb,
                                           (unsigned long long)k * rows * eb * ns};
    const unsigned int box[4] = {(unsigned)(UB_KB / eb), (unsigned)box_rows, 1u, 1u};
    return encode_tmap_4d(mp, tf32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, base, dims,
                          strides, box, CU_TENSOR_MAP_SWIZZLE_64B);
}

template <int BN, int NT, int NS, bool DRAIN, bool BMN = false, bool TF = false>
static int launch_umma(const UmmaMaps& maps, const UmmaArgs& g, dim3 grid) {
    constexpr int STAGE = NT * (UB_M * UB_KB + BN * UB_KB);
    const size_t smem = (size_t)NS * STAGE + 256;
    RS_CHECK(set_smem_optin((const void*)k_umma<BN, NT, NS, DRAIN, BMN, TF>, (int)smem));
    launch(k_umma<BN, NT, NS, DRAIN, BMN, TF>, grid, U_THREADS, smem, ctx().stream, maps, g);
    RS_LAUNCH();
    return RSDFT_OK;
}

// C (nb x nb) = alpha * A^T B (symmetrize: alpha/2 (A^T B + B^T A)); A, B tall
// (ML x nb, leading dimension ld); B == A computes only the upper tiles.
// Gram matrix from BF16 slices (ML x nb each, 3 slices): C = alpha sa^T sb,
// symmetric tile pairs only when same.
static int gram_from_slices(void* sa, void* sb, bool same, int nb, double alpha, int symmetrize, Split sp,
                            double* C, bool upper_only = false) {
    Context& c = ctx();
    const long ml = c.ml;
    UmmaMaps maps;
    RS_CHECK(map3(&maps.a, sa, ml, nb, UB_M, sp.tf32));
    RS_CHECK(map3(&maps.b, sb, ml, nb, 128, sp.tf32));
    UmmaArgs g{};
    const int uke = sp.tf32 ? UB_KB / 4 : UB_K;
    g.kblocks = (int)((ml + uke - 1) / uke);
    g.ntm = g.ntn = (nb + UB_M - 1) / UB_M;
    // tile pairs tm <= tn only when the product is symmetric: A^T A, or (with
    // upper_only) A^T B for a symmetric operator B = H A, whose lower tiles
    // equal the transposed upper ones
    const bool sym = same || upper_only;
    g.sym = sym ? 1 : 0;
    g.npairs = sym ? g.ntm * (g.ntm + 1) / 2 : g.ntm * g.ntn;
    const int sms = c.num_sms > 0 ? c.num_sms : 148;
    int nsplit = std::max(1, sms / g.npairs);
    nsplit = std::min(nsplit, g.kblocks);
    g.kb_per_split = (g.kblocks + nsplit - 1) / nsplit;
    nsplit = (g.kblocks + g.kb_per_split - 1) / g.kb_per_split;
    RS_CHECK(workspace_t("umma_part", (size_t)nsplit * g.npairs * 128 * UB_M, &g.partial));
    g.err = c.err_flag;
    g.mrows = g.nrows = nb;
    if (sp.tf32)
        RS_CHECK((launch_umma<128, 2, 4, true, false, true>(maps, g, dim3(g.npairs, nsplit))));
    else if (sp.terms == 3)
        RS_CHECK((launch_umma<128, 3, 4, true>(maps, g, dim3(g.npairs, nsplit))));
    else
        RS_CHECK((launch_umma<128, 2, 4, true>(maps, g, dim3(g.npairs, nsplit))));
    launch(k_reduce_tiles, dim3(div_up(nb, 128), nb), 128, 0, c.stream, g.partial, nsplit, g.npairs, g.ntm, g.sym, 128,
           nb, alpha, symmetrize, C);
    RS_LAUNCH();
    return RSDFT_OK;
}

// BF16 (3 slices) or TF32 (2 slices) terms of a tall FP64 / FP32 block into
// the named workspace
template <typename TI>
static int split_cols(const TI* A, long ld, int nb, const char* ws, Split sp, void** out) {
    Context& c = ctx();
    const long ml = c.ml;
    if (ml % 8 != 0) {
        set_error("mixed contractions need ML to be a multiple of 8");
        return RSDFT_EUNSUP;
    }
    if (sp.tf32) {
        uint32_t* o = nullptr;
        RS_CHECK(workspace_t(ws, 2 * (size_t)ml * nb, &o));
        launch(k_split_cols_tf32<TI>, dim3(div_up(ml, 1024), nb), 256, 0, c.stream, A, ld, nb, ml, o);
        RS_LAUNCH();
        *out = o;
        return RSDFT_OK;
    }
    __nv_bfloat16* o = nullptr;
    RS_CHECK(workspace_t(ws, 3 * (size_t)ml * nb, &o));
    const int vec = ((ld * (long)sizeof(TI)) % 16 == 0 && reinterpret_cast<uintptr_t>(A) % 16 == 0) ? 1 : 0;
    launch(k_split_cols<TI>, dim3(div_up(ml, 2048), nb), 256, 0, c.stream, A, ld, nb, ml, o, vec);
    RS_LAUNCH();
    *out = o;
    return RSDFT_OK;
}

int gram_mixed(const double* A, const double* B, long ld, int nb, double alpha, int symmetrize, int mode,
               double* C, const void** a_split) {
    const Split sp = mode_split(mode);
    void *sa = nullptr, *sb = nullptr;
    RS_CHECK(split_cols(A, ld, nb, "umma_sa", sp, &sa));
    const bool same = (A == B);
    if (same)
        sb = sa;
    else
        RS_CHECK(split_cols(B, ld, nb, "umma_sb", sp, &sb));
    if (a_split) *a_split = sa;
    return gram_from_slices(sa, sb, same, nb, alpha, symmetrize, sp, C);
}

template <typename TI>
static int gram_pair(const TI* psi, const TI* hpsi, long ld, int nb, double alpha, int mode, double* S, double* H,
                     const void** psi_split) {
    const Split sp = mode_split(mode);
    void *sa = nullptr, *sb = nullptr;
    RS_CHECK(split_cols(psi, ld, nb, "umma_sa", sp, &sa));
    RS_CHECK(split_cols(hpsi, ld, nb, "umma_sb", sp, &sb));
    if (psi_split) *psi_split = sp.tf32 ? nullptr : sa;  // TF32 rotations split psi transposed
    RS_CHECK(gram_from_slices(sa, sa, true, nb, alpha, 0, sp, S));
    // psi^T (H psi) is symmetric: the upper tile pairs, the diagonal tiles
    // symmetrised (subspace_mate_sl likewise forms one triangle)
    return gram_from_slices(sa, sb, false, nb, alpha, 1, sp, H, true);
}

int gram_mixed_pair(const double* psi, const double* hpsi, long ld, int nb, double alpha, int mode, double* S,
                    double* H, const void** psi_split) {
    return gram_pair<double>(psi, hpsi, ld, nb, alpha, mode, S, H, psi_split);
}

int gram_mixed_pair(const float* psi, const float* hpsi, long ld, int nb, double alpha, int mode, double* S,
                    double* H, const void** psi_split) {
    return gram_pair<float>(psi, hpsi, ld, nb, alpha, mode, S, H, psi_split);
}

// The A operand of a rotation: slices[s][n][m] = term s of V(m, n), K = m
// padded to mbk with zeros.
static int split_v(const double* V, int nb, int ldv, int mbk, Split sp, UmmaMaps* maps) {
    Context& c = ctx();
    if (sp.tf32) {
        uint32_t* sv = nullptr;
        RS_CHECK(workspace_t("umma_sv", 2 * (size_t)nb * mbk, &sv));
        launch(k_split_small_tf32, div_up((long)nb * mbk, 256), 256, 0, c.stream, V, nb, ldv, mbk, sv);
        RS_LAUNCH();
        return map3(&maps->a, sv, mbk, nb, UB_M, true);
    }
    __nv_bfloat16* sv = nullptr;
    RS_CHECK(workspace_t("umma_sv", 3 * (size_t)nb * mbk, &sv));
    launch(k_split_small, div_up((long)nb * mbk, 256), 256, 0, c.stream, V, nb, ldv, mbk, sv);
    RS_LAUNCH();
    return map3(&maps->a, sv, mbk, nb, UB_M);
}

static UmmaArgs rotate_args(long ml, int nb, int mbk, double* out, long ld, bool tf32) {
    UmmaArgs g{};
    const int uke = tf32 ? UB_KB / 4 : UB_K;
    g.kblocks = (mbk + uke - 1) / uke;
    g.ntm = (nb + UB_M - 1) / UB_M;
    g.ntn = (int)((ml + 255) / 256);
    g.out = out;
    g.ldo = ld;
    g.mrows = nb;
    g.nrows = (int)ml;
    g.err = ctx().err_flag;
    return g;
}

template <bool BMN>
static int launch_rotate(const UmmaMaps& maps, const UmmaArgs& g, Split sp) {
    Context& c = ctx();
    const int sms = c.num_sms > 0 ? c.num_sms : 148;
    const dim3 grid((unsigned)std::min(g.ntm * g.ntn, sms));
    if constexpr (!BMN)
        if (sp.tf32) return launch_umma<256, 2, 3, false, false, true>(maps, g, grid);
    if (sp.terms == 3) return launch_umma<256, 3, 3, false, BMN>(maps, g, grid);
    return launch_umma<256, 2, 3, false, BMN>(maps, g, grid);
}

// B operand from the split of psi as the Gram product leaves it (slices
// [s][band][grid], grid fastest), read MN-major: the map views the grid
// index as (32, ML / 32) so that one box is BN / 32 groups of 32 grid values
// x UB_K bands.  Returns RSDFT_EUNSUP when that view is not available.
static int rotate_from_split(const __nv_bfloat16* sp, double* out, long ld, int nb, const double* V, int ldv,
                             Split spl) {
    Context& c = ctx();
    const long ml = c.ml;
    if (ml % 32 != 0) return RSDFT_EUNSUP;
    UmmaMaps maps;
    const unsigned long long dims[4] = {32ull, (unsigned long long)nb, (unsigned long long)(ml / 32), 3ull};
    const unsigned long long strides[3] = {(unsigned long long)ml * 2, 64ull, (unsigned long long)ml * nb * 2};
    const unsigned int box[4] = {32u, (unsigned)UB_K, 256u / 32u, 1u};
    if (encode_tmap_4d_swz64(&maps.b, sp, dims, strides, box) != RSDFT_OK) return RSDFT_EUNSUP;
    const int mbk = (nb + 7) / 8 * 8;
    RS_CHECK(split_v(V, nb, ldv, mbk, spl, &maps));
    return launch_rotate<true>(maps, rotate_args(ml, nb, mbk, out, ld, false), spl);
}

// out (ML x nb, leading dimension ldo) = psi V, V (nb x nb, leading dimension ldv)
template <typename TI>
static int rotate(const TI* psi, double* out, long ld, int nb, const double* V, int ldv, int mode,
                  const void* psi_split) {
    const Split sp = mode_split(mode);
    if (psi_split && !sp.tf32) {
        const int r = rotate_from_split(static_cast<const __nv_bfloat16*>(psi_split), out, ld, nb, V, ldv, sp);
        if (r != RSDFT_EUNSUP) return r;
    }
    // transposed split: slices[s][i][m], K = band index fastest
    Context& c = ctx();
    const long ml = c.ml;
    const int mbk = (nb + 7) / 8 * 8;
    void* st = nullptr;
    const dim3 sg(div_up(ml, 32), div_up(mbk, 32)), sb(32, 8);
    if (sp.tf32) {
        uint32_t* t = nullptr;
        RS_CHECK(workspace_t("umma_st", 2 * (size_t)ml * mbk, &t));
        launch(k_split_rows_tf32<TI>, sg, sb, 0, c.stream, psi, ld, nb, ml, mbk, t);
        st = t;
    } else {
        __nv_bfloat16* t = nullptr;
        RS_CHECK(workspace_t("umma_st", 3 * (size_t)ml * mbk, &t));
        launch(k_split_rows<TI>, sg, sb, 0, c.stream, psi, ld, nb, ml, mbk, t);
        st = t;
    }
    RS_LAUNCH();
    UmmaMaps maps;
    RS_CHECK(split_v(V, nb, ldv, mbk, sp, &maps));
    RS_CHECK(map3(&maps.b, st, mbk, ml, 256, sp.tf32));
    return launch_rotate<false>(maps, rotate_args(ml, nb, mbk, out, ld, sp.tf32), sp);
}

int rotate_mixed(const double* psi, double* out, long ld, int nb, const double* V, int ldv, int mode,
                 const void* psi_split) {
    return rotate<double>(psi, out, ld, nb, V, ldv, mode, psi_split);
}

int rotate_mixed(const float* psi, double* out, long ld, int nb, const double* V, int ldv, int mode,
                 const void* psi_split) {
    return rotate<float>(psi, out, ld, nb, V, ldv, mode, psi_split);
}

}  // namespace rsdft
