// s-step preconditioner of the CG sweep (precond_hprsdft with IPC = 4,
// cgpc_hprsdft_module.f90:126-348, in the Chebyshev-basis form described in
// cgvec.cuh) and the search-direction update folded into it
// (cg_module.f90:232-261).
#include "cgvec.cuh"
#include "kernels.cuh"

namespace rsdft {

// Basis vector w_K (K = 0: r0 = g - A g, the reference's first residual).
// STORE: write w_K; dots <w_K, w_j> for j <= K.  !STORE (K = mloop): w_K
// only feeds dots: <w_K, w_j> and <w_j, g> for j < K.
template <typename T, int K, bool STORE>
__global__ void __launch_bounds__(VT) k_ss_basis(const T* __restrict__ g, SSVec<T> sv, long ld, long n, PcArgs pa,
                                                 double* __restrict__ part, const int* __restrict__ active) {
    constexpr int D = K == 0 ? 1 : (STORE ? K + 1 : 2 * K);
    __shared__ double sh[VT / 32];
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
#pragma unroll
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
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const double r = block_sum<VT>(acc[k], sh);
        if (threadIdx.x == 0) part[((long)b * gridDim.x + blockIdx.x) * D + k] = r;
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
__global__ void __launch_bounds__(VT) k_ss_p(const T* __restrict__ g, SSVec<T> sv, T* __restrict__ p, long ld,
                                             long n, const double* __restrict__ cz, const double* __restrict__ bk_,
                                             int m, int first, const int* __restrict__ active) {
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    T c[SS_MAXM];
#pragma unroll
    for (int j = 0; j < SS_MAXM; ++j) c[j] = (T)cz[(long)b * SS_MAXM + j];
    const T bk = (T)bk_[b];
#pragma unroll
    for (int it = 0; it < VITEMS; ++it) {
        const long i = base + it * VT + threadIdx.x;
        if (i < n) {
            T pg = g[off + i];
#pragma unroll
            for (int j = 0; j < SS_MAXM; ++j)
                if (j < m) pg += c[j] * sv.w[j][off + i];
            p[off + i] = first ? pg : pg + bk * p[off + i];
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

template <typename T>
int sstep_precond(const T* g, const SSVec<T>& sv, T* p, long ld, int mb, int mloop, int first, const CGScal& s,
                  double* ss, double* cz, double* part, const PcArgs& pa, double dV) {
    const Context& c = ctx();
    cudaStream_t st = c.stream;
    const long n = c.ml;
    const int nchunk = div_up(n, VCHUNK);
    const dim3 vg(nchunk, mb);
    const int sb = div_up(mb, 128);
    auto finish_to = [&](int K, double* out) {
        launch(k_finish_to, div_up((long)mb * K, 128), 128, 0, st, part, nchunk, K, mb, out, SS_STRIDE, s.active);
    };
    launch(k_ss_basis<T, 0, true>, vg, VT, 0, st, g, sv, ld, n, pa, part, s.active);
    finish_to(1, ss);
    for (int k = 1; k < mloop; ++k) {
        RS_CHECK(launch_ss_store<T>(k, vg, st, g, sv, ld, n, pa, part, s.active));
        finish_to(k + 1, ss + k * (k + 1) / 2);
    }
    RS_CHECK(launch_ss_fly<T>(mloop, vg, st, g, sv, ld, n, pa, part, s.active));
    finish_to(2 * mloop, ss + mloop * (mloop + 1) / 2);
    launch(s_sstep, sb, 128, 0, st, s, ss, cz, mb, mloop, pa.d, dV, first);
    launch(k_ss_p<T>, vg, VT, 0, st, g, sv, p, ld, n, cz, s.bk, mloop, first, s.active);
    RS_LAUNCH();
    return RSDFT_OK;
}

template int sstep_precond<double>(const double*, const SSVec<double>&, double*, long, int, int, int, const CGScal&,
                                   double*, double*, double*, const PcArgs&, double);
template int sstep_precond<float>(const float*, const SSVec<float>&, float*, long, int, int, int, const CGScal&,
                                  double*, double*, double*, const PcArgs&, double);

}  // namespace rsdft
