// s-step preconditioner of the CG sweep (precond_hprsdft with IPC = 4,
// cgpc_hprsdft_module.f90:126-348, in the Chebyshev-basis form described in
// cgvec.cuh) and the search-direction update folded into it
// (cg_module.f90:232-261).
#include <algorithm>

#include "cgvec.cuh"
#include "kernels.cuh"
#include "tma.cuh"
#include "tmap.cuh"
#include "vec16.cuh"

namespace rsdft {

// Basis vector w_K (K = 0: r0 = g - A g, the reference's first residual).
// STORE: write w_K; dots <w_K, w_j> for j <= K.  !STORE (K = mloop): w_K
// only feeds dots: <w_K, w_j> and <w_j, g> for j < K.
template <typename T, int K, bool STORE>
__global__ void __launch_bounds__(VT) k_ss_basis(const T* __restrict__ g, SSVec<T> sv, long ld, long n, PcArgs pa,
                                                 double* __restrict__ part, const int* __restrict__ active) {
    constexpr int D = K == 0 ? 1 : (STORE ? K + 1 : 2 * K);
    __shared__ double sh[D * (VT / 32)];
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    const T* src = K == 0 ? g + off : sv.w[K > 0 ? K - 1 : 0] + off;
    const T inv_d = (T)(1.0 / pa.d);
    double acc[D];
#pragma unroll
    for (int k = 0; k < D; ++k) acc[k] = 0.0;
    int i1, i2, i3;
    pc_coords(base + threadIdx.x, pa, i1, i2, i3);
#pragma unroll 8
    for (int it = 0; it < VITEMS; ++it) {
        const long i = base + it * VT + threadIdx.x;
        if (i < n) {
            T wk;
            if constexpr (K == 0) {
                wk = src[i] - pc_apply<T>(src, i, i1, i2, i3, pa);
            } else if constexpr (K == 1) {
                wk = pc_offdiag<T>(src, i, i1, i2, i3, pa) * inv_d;
            } else {
                wk = (T)2 * pc_offdiag<T>(src, i, i1, i2, i3, pa) * inv_d - sv.w[K >= 2 ? K - 2 : 0][off + i];
            }
            if constexpr (STORE) sv.w[K < SS_MAXM ? K : 0][off + i] = wk;
            if constexpr (K == 0) {
                acc[0] = fma((double)wk, (double)wk, acc[0]);
            } else {
                double wj[K];
#pragma unroll
                for (int j = 0; j < K; ++j) wj[j] = (double)(j == K - 1 ? src[i] : sv.w[j][off + i]);
#pragma unroll
                for (int j = 0; j < K; ++j) acc[j] = fma((double)wk, wj[j], acc[j]);
                if constexpr (STORE) {
                    acc[K] = fma((double)wk, (double)wk, acc[K]);
                } else {
                    const double gg = (double)g[off + i];
#pragma unroll
                    for (int j = 0; j < K; ++j) acc[K + j] = fma(wj[j], gg, acc[K + j]);
                }
            }
        }
        pc_step(pa, i1, i2, i3);
    }
    block_sum_n<VT, D>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < D; ++k) part[((long)b * gridDim.x + blockIdx.x) * D + k] = acc[k];
    }
}

// fixed-order sum of the per-CTA partials into out[b * ostride + k]
__global__ void k_finish_to(const double* __restrict__ part, int nchunk, int K, int nb, double* __restrict__ out,
                            int ostride, const int* __restrict__ active) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb * K) return;
    int b = i / K, k = i - b * K;
    if (active && !active[b]) return;
    const double* p = part + (long)b * nchunk * K + k;
    double s = 0.0;
    for (int c = 0; c < nchunk; ++c) s += p[(long)c * K];
    out[(long)b * ostride + k] = s;
}

// Per band: the reference's preconditioner recurrences on coefficient
// vectors (early exit when |r0|^2 < 1e-24, cgpc_hprsdft_module.f90:186),
// then rb = dV <Pg|g> = rb + dV sum_j cz_j <w_j|g> and the search-direction
// scalars bk = rb / gkgk, gkgk = rb (cg_module.f90:232-250).
__global__ void s_sstep(CGScal s, const double* __restrict__ ss, double* __restrict__ cz_out, int nb, int m,
                        double d, double dV, int first) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || !s.active[b]) return;
    const double* S = ss + (long)b * SS_STRIDE;
    double G[SS_MAXM + 1][SS_MAXM + 1] = {};
    double gd[SS_MAXM] = {};
    G[0][0] = S[0];
    for (int k = 1; k < m; ++k)
        for (int j = 0; j <= k; ++j) G[k][j] = G[j][k] = S[k * (k + 1) / 2 + j];
    const int o = m * (m + 1) / 2;
    for (int j = 0; j < m; ++j) {
        G[m][j] = G[j][m] = S[o + j];
        gd[j] = S[o + m + j];
    }
    double cz[SS_MAXM + 1] = {};
    double rr = G[0][0];
    if (!(rr < 1e-24)) {
        double r[SS_MAXM + 1] = {}, q[SS_MAXM + 1] = {}, ft[SS_MAXM + 1];
        r[0] = q[0] = 1.0;
        for (int il = 1; il <= m; ++il) {
            // ft = A q in the basis
            for (int i = 0; i <= m; ++i) ft[i] = d * q[i];
            ft[1] += d * q[0];
            for (int j = 1; j < m; ++j) {
                ft[j + 1] += 0.5 * d * q[j];
                ft[j - 1] += 0.5 * d * q[j];
            }
            double pAp = 0.0;
            for (int i = 0; i <= m; ++i)
                for (int j = 0; j <= m; ++j) pAp += q[i] * G[i][j] * ft[j];
            const double a = rr / pAp;
            for (int i = 0; i <= m; ++i) cz[i] += a * q[i];
            if (il == m) break;
            for (int i = 0; i <= m; ++i) r[i] -= a * ft[i];
            double rn = 0.0;
            for (int i = 0; i <= m; ++i)
                for (int j = 0; j <= m; ++j) rn += r[i] * G[i][j] * r[j];
            const double bb = rn / rr;
            rr = rn;
            for (int i = 0; i <= m; ++i) q[i] = r[i] + bb * q[i];
        }
    }
    double gz = 0.0;
    for (int j = 0; j < m; ++j) gz += cz[j] * gd[j];
    const double rb = s.rb[b] + dV * gz;
    s.rb[b] = rb;
    s.bk[b] = first ? 0.0 : rb / s.gkgk[b];
    s.gkgk[b] = rb;
    for (int j = 0; j < SS_MAXM; ++j) cz_out[(long)b * SS_MAXM + j] = j < m ? cz[j] : 0.0;
}

// p = g + sum_j cz_j w_j (+ bk p after the first step)
template <typename T>
__global__ void __launch_bounds__(VT) k_ss_p(const T* __restrict__ g, SSVec<T> sv, T* __restrict__ p,
                                             T* __restrict__ x, long ld, long n, const double* __restrict__ cz,
                                             const double* __restrict__ bk_, int m, int first,
                                             const int* __restrict__ active, const int* __restrict__ pend,
                                             const double* __restrict__ u11_, const double* __restrict__ u21_,
                                             int vec) {
    using G = Grp16<T>;
    constexpr int W = G::W;
    const int b = blockIdx.y;
    const bool act = !active || active[b];
    const bool upd = pend && pend[b];  // the previous step's x update, which needs the old p
    if (!act && !upd) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    T c[SS_MAXM];
#pragma unroll
    for (int j = 0; j < SS_MAXM; ++j) c[j] = (T)cz[(long)b * SS_MAXM + j];
    const T bk = (T)bk_[b];
    const T u11 = upd ? (T)u11_[b] : (T)0, u21 = upd ? (T)u21_[b] : (T)0;
#pragma unroll 2
    for (int it = 0; it < VITEMS / W; ++it) {
        const long i = base + ((long)it * VT + threadIdx.x) * W;
        if (vec && i + W <= n) {
            T pg[W], t[W];
            if (upd || !first) G::load(p + off + i, t);
            if (upd) {
                T xv[W];
                G::load(x + off + i, xv);
#pragma unroll
                for (int q = 0; q < W; ++q) xv[q] = cg_upd2_elem(xv[q], t[q], u11, u21);
                G::store(x + off + i, xv);
            }
            if (!act) continue;
            T pn[W];
#pragma unroll
            for (int q = 0; q < W; ++q) pn[q] = t[q];
            G::load(g + off + i, pg);
#pragma unroll
            for (int j = 0; j < SS_MAXM; ++j) {
                if (j < m) {
                    G::load(sv.w[j] + off + i, t);
#pragma unroll
                    for (int q = 0; q < W; ++q) pg[q] += c[j] * t[q];
                }
            }
            if (!first) {
#pragma unroll
                for (int q = 0; q < W; ++q) pg[q] += bk * pn[q];
            }
            G::store(p + off + i, pg);
        } else {
            for (int q = 0; q < W && i + q < n; ++q) {
                const long k = off + i + q;
                const T po = (upd || !first) ? p[k] : (T)0;
                if (upd) x[k] = cg_upd2_elem(x[k], po, u11, u21);
                if (!act) continue;
                T pg = g[k];
#pragma unroll
                for (int j = 0; j < SS_MAXM; ++j)
                    if (j < m) pg += c[j] * sv.w[j][k];
                p[k] = first ? pg : pg + bk * po;
            }
        }
    }
}

template <typename T>
static int launch_ss_store(int k, dim3 vg, cudaStream_t st, const T* g, SSVec<T> sv, long ld, long n,
                           const PcArgs& pa, double* part, const int* act) {
    switch (k) {
        case 1: launch(k_ss_basis<T, 1, true>, vg, VT, 0, st, g, sv, ld, n, pa, part, act); break;
        case 2: launch(k_ss_basis<T, 2, true>, vg, VT, 0, st, g, sv, ld, n, pa, part, act); break;
        case 3: launch(k_ss_basis<T, 3, true>, vg, VT, 0, st, g, sv, ld, n, pa, part, act); break;
        default: set_error("s-step basis index %d", k); return RSDFT_EUNSUP;
    }
    return RSDFT_OK;
}

template <typename T>
static int launch_ss_fly(int m, dim3 vg, cudaStream_t st, const T* g, SSVec<T> sv, long ld, long n,
                         const PcArgs& pa, double* part, const int* act) {
    switch (m) {
        case 1: launch(k_ss_basis<T, 1, false>, vg, VT, 0, st, g, sv, ld, n, pa, part, act); break;
        case 2: launch(k_ss_basis<T, 2, false>, vg, VT, 0, st, g, sv, ld, n, pa, part, act); break;
        case 3: launch(k_ss_basis<T, 3, false>, vg, VT, 0, st, g, sv, ld, n, pa, part, act); break;
        case 4: launch(k_ss_basis<T, 4, false>, vg, VT, 0, st, g, sv, ld, n, pa, part, act); break;
        default: set_error("s-step mloop %d", m); return RSDFT_EUNSUP;
    }
    return RSDFT_OK;
}

// ------------------------------------------- TMA z-march basis kernel
// One basis step as a z march over the 7-point operator, the hpsi stencil's
// pattern with Md = 1: a CTA owns TY full-width rows of one band; a producer
// warp streams each source plane (TY + 2 rows, periodic y wrap split into
// boxes) into a ring of S shared-memory stages, together with TY-row tiles of
// the operands the step's epilogue needs at the plane that completes there
// (w_0 .. w_{K-2}, and g for the last step).  Consumer threads own VX x 2
// points, push the z contributions into 3 rotating accumulators, and at the
// completed plane form w_K, store it and add the step's dot products; the
// CTA's dot partials are summed in a fixed order at the end.  Every vector
// element is read once from memory.
struct PcMaps {
    CUtensorMap full, edge, mid, wrap;  // source boxes of TY + 2, TY + 1, TY, 1 rows
    CUtensorMap aux[SS_MAXM];           // epilogue operands, TY rows
};

template <int K, bool STORE>
struct PcStep {
    static constexpr int NA = (K >= 2 ? K - 1 : 0) + (STORE ? 0 : 1);  // w_0..w_{K-2}, then g
    static constexpr int D = K == 0 ? 1 : (STORE ? K + 1 : 2 * K);
    // CTAs per SM: the first two steps have no epilogue operands and few
    // dots, so two CTAs (<= 85 registers, half the stage ring each) fit and
    // hide the per-plane latency better
    static constexpr int CTAS = K <= 1 ? 2 : 1;
};

__device__ __forceinline__ int pc_pwrap(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

template <typename T, int K, bool STORE>
__global__ void __launch_bounds__(384, PcStep<K, STORE>::CTAS) k_pc_tma(const __grid_constant__ PcMaps maps,
                                                                      T* __restrict__ wout,
                                                   StencilCoef cf, int n1, int n2, int n3, long ld, int zlen0,
                                                   int nzc, int TY, int RS, int S, int ncw,
                                                   double* __restrict__ part, const int* __restrict__ active,
                                                   int* __restrict__ err) {
    using VT = Vec16<T>;
    using V = typename VT::t;
    constexpr int VX = 16 / (int)sizeof(T);
    constexpr int BY = 2;
    constexpr int NP = VX * BY;
    constexpr int NV = 3;  // x window: x - VX .. x + 2 VX - 1
    constexpr int NA = PcStep<K, STORE>::NA;
    constexpr int D = PcStep<K, STORE>::D;
    extern __shared__ __align__(128) unsigned char smem[];
    const int ROWS = TY + 2;
    const int SE = (ROWS + NA * TY) * RS;
    T* stages = reinterpret_cast<T*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * SE * sizeof(T));
    uint64_t* empty = full + S;
    double* red = reinterpret_cast<double*>(empty + S);  // ncw x D

    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    const int band = blockIdx.y / nzc;
    const int zc = blockIdx.y - band * nzc;
    if (active && !active[band]) return;  // uniform per CTA
    const int y0 = blockIdx.x * TY;
    const int zs = zc * zlen0;
    const int zlen = min(zs + zlen0, n3) - zs;
    const int nk = zlen + 2;  // arrival k <-> source plane zs - 1 + k
    const long plane = (long)n1 * n2;

    if (t == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], ncw);
        }
        mbar_fence_init();
    }
    __syncthreads();

    if (warp == ncw) {
        // ------------------------------------------------------ producer
        bool ok = true;
        if (lane == 0) {
            const uint32_t b_tile = (uint32_t)((size_t)TY * RS * sizeof(T));
            const uint32_t b_src = (uint32_t)((size_t)ROWS * RS * sizeof(T));
            for (int k = 0; k < nk; ++k) {
                const int s = k % S;
                if (k >= S && !mbar_wait(&empty[s], ((k / S) - 1) & 1)) ok = false;
                T* dst = stages + (size_t)s * SE;
                const int zp = pc_pwrap(zs - 1 + k, n3);
                const bool inner = k >= 1 && k < 1 + zlen;
                const bool aux = k >= 2;
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&full[s], (inner ? b_src : b_tile) + (aux ? NA * b_tile : 0u));
                if (!inner) {
                    tma_load_4d(dst + RS, &maps.mid, 0, y0, zp, band, &full[s]);
                } else if (y0 - 1 >= 0 && y0 + TY + 1 <= n2) {
                    tma_load_4d(dst, &maps.full, 0, y0 - 1, zp, band, &full[s]);
                } else if (TY == n2) {
                    tma_load_4d(dst, &maps.wrap, 0, n2 - 1, zp, band, &full[s]);
                    tma_load_4d(dst + RS, &maps.mid, 0, 0, zp, band, &full[s]);
                    tma_load_4d(dst + (1 + TY) * RS, &maps.wrap, 0, 0, zp, band, &full[s]);
                } else if (y0 - 1 < 0) {
                    tma_load_4d(dst, &maps.wrap, 0, n2 - 1, zp, band, &full[s]);
                    tma_load_4d(dst + RS, &maps.edge, 0, 0, zp, band, &full[s]);
                } else {
                    tma_load_4d(dst, &maps.edge, 0, y0 - 1, zp, band, &full[s]);
                    tma_load_4d(dst + (TY + 1) * RS, &maps.wrap, 0, 0, zp, band, &full[s]);
                }
                if (aux) {
#pragma unroll
                    for (int a = 0; a < NA; ++a)
                        tma_load_4d(dst + (ROWS + a * TY) * RS, &maps.aux[a], 0, y0, zs + k - 2, band, &full[s]);
                }
            }
        }
        __syncwarp();
        if (!ok) atomicExch(err, 1);
        return;
    }

    // ---------------------------------------------------------- consumers
    const int nxv = n1 / VX;
    const int ncons = nxv * (TY / BY);
    const bool thr = t < ncons;
    const int px = thr ? t % nxv : 0, py = thr ? t / nxv : 0;
    const int x = VX * px, yl = BY * py;
    const int xw = x - VX;
    T* __restrict__ ob = STORE ? wout + (long)band * ld + (long)n1 * (y0 + yl) + x : nullptr;
    const T c0 = (T)cf.c0, cx = (T)cf.cx[0], cy = (T)cf.cy[0], cz = (T)cf.cz[0];

    T acc[3][NP], cprev[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        acc[0][i] = acc[1][i] = acc[2][i] = (T)0;
        cprev[i] = (T)0;
    }
    double dots[D];
#pragma unroll
    for (int k = 0; k < D; ++k) dots[k] = 0.0;

    bool ok = true;
    int s = 0, u = 0;
    uint32_t ph = 0;
    for (int k = 0; k < nk; ++k) {
        if (!mbar_wait(&full[s], ph)) ok = false;
        const T* st = stages + (size_t)s * SE;
        const bool inner = k >= 1 && k < 1 + zlen;  // uniform
        T c[NP], in[NP];
        if (inner) {
            const T* sp = st + yl * RS + x;
#pragma unroll
            for (int i = 0; i < NP; ++i) in[i] = (T)0;
#pragma unroll
            for (int j = 0; j < BY + 2; ++j) {
                T v[VX];
                VT::get(*reinterpret_cast<const V*>(sp + j * RS), v);
#pragma unroll
                for (int r = 0; r < BY; ++r) {
                    const int m = j - 1 - r;
                    if (m == 0) {
#pragma unroll
                        for (int e = 0; e < VX; ++e) c[r * VX + e] = v[e];
                    } else if (m == 1 || m == -1) {
#pragma unroll
                        for (int e = 0; e < VX; ++e) in[r * VX + e] += cy * v[e];
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < BY; ++r) {
                const T* rp = st + (1 + yl + r) * RS;
                T w[NV * VX];
#pragma unroll
                for (int j = 0; j < NV; ++j) {
                    if (j == 1) {
                        // the centre vector: the row's own, read with the y window
#pragma unroll
                        for (int e = 0; e < VX; ++e) w[VX + e] = c[r * VX + e];
                        continue;
                    }
                    int xx = xw + VX * j;
                    xx += xx < 0 ? n1 : (xx >= n1 ? -n1 : 0);
                    VT::get(*reinterpret_cast<const V*>(rp + xx), w + j * VX);
                }
#pragma unroll
                for (int e = 0; e < VX; ++e) in[r * VX + e] += cx * (w[VX + e - 1] + w[VX + e + 1]);
            }
#pragma unroll
            for (int i = 0; i < NP; ++i) in[i] += c0 * c[i];
        } else {
#pragma unroll
            for (int r = 0; r < BY; ++r)
                VT::get(*reinterpret_cast<const V*>(st + (1 + yl + r) * RS + x), c + r * VX);
        }
        // z pushes: output k + 1 (first touch) and k - 1 (last touch); slot = arrival mod 3
        T o[NP];
#define RS_PC_PUSH(U)                                                  \
    {                                                                  \
        _Pragma("unroll") for (int i = 0; i < NP; ++i) {               \
            acc[(U + 1) % 3][i] = cz * c[i];                           \
            acc[(U + 2) % 3][i] += cz * c[i];                          \
            if (inner) acc[U][i] += in[i];                             \
            o[i] = acc[(U + 2) % 3][i];                                \
        }                                                              \
    }
        if (u == 0)
            RS_PC_PUSH(0)
        else if (u == 1)
            RS_PC_PUSH(1)
        else
            RS_PC_PUSH(2)
#undef RS_PC_PUSH
        if (k >= 2) {
            // plane zs + k - 2 is complete: o = operator part of w_K there
            const long zo = plane * (zs + k - 2);
#pragma unroll
            for (int r = 0; r < BY; ++r) {
                T av[NA > 0 ? NA : 1][VX];
#pragma unroll
                for (int a = 0; a < NA; ++a)
                    VT::get(*reinterpret_cast<const V*>(st + (ROWS + a * TY + yl + r) * RS + x), av[a]);
                T wk[VX];
#pragma unroll
                for (int e = 0; e < VX; ++e) {
                    const int i = r * VX + e;
                    if constexpr (K == 0)
                        wk[e] = -o[i];
                    else if constexpr (K == 1)
                        wk[e] = o[i];
                    else
                        wk[e] = o[i] - av[K >= 2 ? K - 2 : 0][e];
                    const double wd = (double)wk[e];
                    if constexpr (K == 0) {
                        dots[0] = fma(wd, wd, dots[0]);
                    } else {
#pragma unroll
                        for (int j = 0; j < K - 1; ++j) dots[j] = fma(wd, (double)av[j][e], dots[j]);
                        dots[K - 1] = fma(wd, (double)cprev[i], dots[K - 1]);
                        if constexpr (STORE) {
                            dots[K] = fma(wd, wd, dots[K]);
                        } else {
                            const double gg = (double)av[NA - 1][e];
#pragma unroll
                            for (int j = 0; j < K - 1; ++j) dots[K + j] = fma((double)av[j][e], gg, dots[K + j]);
                            dots[2 * K - 1] = fma((double)cprev[i], gg, dots[2 * K - 1]);
                        }
                    }
                }
                if constexpr (STORE) {
                    if (thr) *reinterpret_cast<V*>(ob + zo + (long)r * n1) = VT::make(wk);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < NP; ++i) cprev[i] = c[i];
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with the stage
        if (++s == S) {
            s = 0;
            ph ^= 1u;
        }
        if (++u == 3) u = 0;
    }
    // fixed-order reduction of the dot partials over the consumer warps
#pragma unroll
    for (int k = 0; k < D; ++k) {
        double v = thr ? dots[k] : 0.0;
#pragma unroll
        for (int o2 = 16; o2 > 0; o2 >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o2);
        if (lane == 0) red[warp * D + k] = v;
    }
    asm volatile("bar.sync 1, %0;" ::"r"(ncw * 32) : "memory");
    if (t == 0) {
        const int nchunk = gridDim.x * nzc;
        const int chunk = zc * gridDim.x + blockIdx.x;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            double v = 0.0;
            for (int w = 0; w < ncw; ++w) v += red[w * D + k];
            part[((long)band * nchunk + chunk) * D + k] = v;
        }
    }
    if (!ok) atomicExch(err, 1);
}

// Geometry of k_pc_tma: TY (even, divides n2, n2 == TY or n2 >= TY + 1), row
// pitch RS (n1 rounded up to 128 bytes), ring depth S (2..8), consumer warps.
struct PcGeom {
    int TY = 0, RS = 0, S = 0, ncw = 0, threads = 0;
    size_t smem = 0;
};

template <typename T>
static PcGeom pc_geometry(int n1, int n2, int na, int d, int ctas) {
    PcGeom best;
    constexpr int VX = 16 / (int)sizeof(T);
    const int RS = (int)((((size_t)n1 * sizeof(T) + 127) / 128) * 128 / sizeof(T));
    if (n1 % VX != 0 || n1 < VX || RS > 256 || n2 < 2) return best;
    double best_score = -1.0;
    for (int TY = 2; TY <= std::min(n2, 254); TY += 2) {
        if (n2 % TY != 0 || !(TY == n2 || n2 >= TY + 1)) continue;
        const int ncw = ((n1 / VX) * (TY / 2) + 31) / 32;
        const int threads = 32 * (ncw + 1);
        if (threads > 384) continue;
        const size_t stage = (size_t)(TY + 2 + na * TY) * RS * sizeof(T);
        const size_t fixed = (size_t)ncw * d * sizeof(double);
        const size_t budget = (ctas > 1 ? 110 : 220) * 1024;
        if (budget <= fixed) continue;
        const int S = (int)std::min<size_t>((budget - fixed) / (stage + 16), 8);
        if (S < 2) continue;
        const double used = (double)((n1 / VX) * (TY / 2)) / threads;
        const double score = 100.0 * TY / (TY + 2) + 10.0 * used + 2.0 * std::min(S, 4);
        if (score > best_score) {
            best_score = score;
            best.TY = TY;
            best.RS = RS;
            best.S = S;
            best.ncw = ncw;
            best.threads = threads;
            best.smem = (size_t)S * stage + (size_t)S * 16 + fixed;
        }
    }
    return best;
}

// Launch basis step K through k_pc_tma; *used = false when the shape or the
// pointers do not suit it (the caller then takes the element-wise kernels).
template <typename T, int K, bool STORE>
static int pc_tma_step(const T* src, const T* const* aux, T* wout, const PcArgs& pa, long ld, int mb,
                       const int* active, double* part, int part_cap, int* nchunk, bool* used) {
    Context& c = ctx();
    *used = false;
    constexpr int NA = PcStep<K, STORE>::NA;
    constexpr int D = PcStep<K, STORE>::D;
    const int n1 = pa.n1, n2 = pa.n2, n3 = pa.n3;
    const PcGeom g = pc_geometry<T>(n1, n2, NA, D, PcStep<K, STORE>::CTAS);
    if (g.TY == 0 || (ld * sizeof(T)) % 16 != 0) return RSDFT_OK;
    if (STORE && reinterpret_cast<uintptr_t>(wout) % 16 != 0) return RSDFT_OK;
    const int sms = c.num_sms > 0 ? c.num_sms : 148;
    const long base = (long)(n2 / g.TY) * mb;
    int nzc = (int)std::min<long>(std::max<long>(1, (sms + base - 1) / base), std::max(1, n3 / 4));
    while (((long)mb * nzc > 65535 || (n2 / g.TY) * nzc > part_cap) && nzc > 1) --nzc;
    const int zlen = div_up(n3, nzc);
    nzc = div_up(n3, zlen);
    if ((n2 / g.TY) * nzc > part_cap) return RSDFT_OK;  // partials would not fit
    PcMaps maps;
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const unsigned long long dims[4] = {(unsigned long long)n1, (unsigned long long)n2, (unsigned long long)n3,
                                        (unsigned long long)mb};
    const unsigned long long strides[3] = {(unsigned long long)n1 * sizeof(T),
                                           (unsigned long long)n1 * n2 * sizeof(T),
                                           (unsigned long long)ld * sizeof(T)};
    const unsigned int RS = (unsigned)g.RS, TY = (unsigned)g.TY;
    const unsigned int bf[4] = {RS, TY + 2, 1, 1}, be[4] = {RS, TY + 1, 1, 1}, bm[4] = {RS, TY, 1, 1},
                       bw[4] = {RS, 1, 1, 1};
    if (encode_tmap_4d(&maps.full, dt, src, dims, strides, bf) != RSDFT_OK ||
        encode_tmap_4d(&maps.edge, dt, src, dims, strides, be) != RSDFT_OK ||
        encode_tmap_4d(&maps.mid, dt, src, dims, strides, bm) != RSDFT_OK ||
        encode_tmap_4d(&maps.wrap, dt, src, dims, strides, bw) != RSDFT_OK)
        return RSDFT_OK;
    for (int a = 0; a < NA; ++a)
        if (encode_tmap_4d(&maps.aux[a], dt, aux[a], dims, strides, bm) != RSDFT_OK) return RSDFT_OK;
    RS_CHECK(set_smem_optin((const void*)k_pc_tma<T, K, STORE>, 220 * 1024 + 8 * 16));
    // coefficients of the operator part: (A - I) for w_0, B = offdiag / d for
    // w_1, 2 B for the later steps
    StencilCoef cf{};
    const double sc = K == 0 ? 1.0 : (K == 1 ? 1.0 / pa.d : 2.0 / pa.d);
    cf.c0 = K == 0 ? pa.d - 1.0 : 0.0;
    cf.cx[0] = sc * pa.c1;
    cf.cy[0] = sc * pa.c2;
    cf.cz[0] = sc * pa.c3;
    dim3 grid(n2 / g.TY, (unsigned)(mb * nzc));
    launch(k_pc_tma<T, K, STORE>, grid, g.threads, g.smem, c.stream, maps, wout, cf, n1, n2, n3, ld, zlen, nzc,
           g.TY, g.RS, g.S, g.ncw, part, active, c.err_flag);
    RS_LAUNCH();
    *nchunk = (n2 / g.TY) * nzc;
    *used = true;
    return RSDFT_OK;
}

// basis step K of the s-step form through the TMA kernel (runtime K)
template <typename T>
static int pc_tma_dispatch(int K, bool store, const T* g, const SSVec<T>& sv, const PcArgs& pa, long ld, int mb,
                           const int* active, double* part, int part_cap, int* nchunk, bool* used) {
    const T* src = K == 0 ? g : sv.w[K - 1];
    const T* aux[SS_MAXM] = {};
    int na = 0;
    for (int j = 0; j + 2 <= K; ++j) aux[na++] = sv.w[j];
    if (!store) aux[na++] = g;
    T* wout = store ? sv.w[K] : nullptr;
#define RS_PC_CASE(KK, ST)                                                                              \
    if (K == KK && store == ST)                                                                         \
        return pc_tma_step<T, KK, ST>(src, aux, wout, pa, ld, mb, active, part, part_cap, nchunk, used);
    RS_PC_CASE(0, true)
    RS_PC_CASE(1, true)
    RS_PC_CASE(2, true)
    RS_PC_CASE(3, true)
    RS_PC_CASE(1, false)
    RS_PC_CASE(2, false)
    RS_PC_CASE(3, false)
    RS_PC_CASE(4, false)
#undef RS_PC_CASE
    *used = false;
    return RSDFT_OK;
}

template <typename T>
int sstep_precond(const T* g, const SSVec<T>& sv, T* p, T* x, long ld, int mb, int mloop, int first, const CGScal& s,
                  double* ss, double* cz, double* part, const PcArgs& pa, double dV) {
    const Context& c = ctx();
    cudaStream_t st = c.stream;
    const long n = c.ml;
    const int nchunk = div_up(n, VCHUNK);
    const dim3 vg(nchunk, mb);
    const int sb = div_up(mb, 128);
    auto finish_to = [&](int K, double* out, int nch) {
        launch(k_finish_to, div_up((long)mb * K, 128), 128, 0, st, part, nch, K, mb, out, SS_STRIDE, s.active);
    };
    // basis steps: TMA z march where the shape allows, element-wise otherwise
    for (int k = 0; k <= mloop; ++k) {
        const bool store = k < mloop;
        const int D = k == 0 ? 1 : (store ? k + 1 : 2 * k);
        double* out = ss + (store ? k * (k + 1) / 2 : mloop * (mloop + 1) / 2);
        bool used = false;
        int nch = 0;
        RS_CHECK(pc_tma_dispatch<T>(k, store, g, sv, pa, ld, mb, s.active, part, nchunk, &nch, &used));
        if (!used) {
            if (k == 0)
                launch(k_ss_basis<T, 0, true>, vg, VT, 0, st, g, sv, ld, n, pa, part, s.active);
            else if (store)
                RS_CHECK(launch_ss_store<T>(k, vg, st, g, sv, ld, n, pa, part, s.active));
            else
                RS_CHECK(launch_ss_fly<T>(k, vg, st, g, sv, ld, n, pa, part, s.active));
            nch = nchunk;
        }
        finish_to(D, out, nch);
    }
    launch(s_sstep, sb, 128, 0, st, s, ss, cz, mb, mloop, pa.d, dV, first);
    const int gv = grp16_ok<T>(ld, {g, p, x, sv.w[0], sv.w[1], sv.w[2], sv.w[3]}) ? 1 : 0;
    launch(k_ss_p<T>, vg, VT, 0, st, g, sv, p, x, ld, n, cz, s.bk, mloop, first, s.active,
           (const int*)(first ? nullptr : s.pend), (const double*)s.u11, (const double*)s.u21, gv);
    RS_LAUNCH();
    return RSDFT_OK;
}

template int sstep_precond<double>(const double*, const SSVec<double>&, double*, double*, long, int, int, int,
                                   const CGScal&, double*, double*, double*, const PcArgs&, double);
template int sstep_precond<float>(const float*, const SSVec<float>&, float*, float*, long, int, int, int,
                                  const CGScal&, double*, double*, double*, const PcArgs&, double);

}  // namespace rsdft
