// Preconditioned CG eigensolver sweep (conjugate_gradient_1, cg_module.f90:
// 97-430, with precond_hprsdft, cgpc_hprsdft_module.f90:126-348), all bands
// at once.  The reference runs bands one after another (MB_d = 1) and, with
// SWGS = 0 (cggs_module.f90:24-25), a band's update never reads another
// band, so advancing every band concurrently performs the same arithmetic.
// Every per-band branch of the reference (early exit, 2x2 eigen-pair choice,
// sign fix, 1e8 rejection, preconditioner early exit) is kept per band in
// device arrays; the loop needs no host synchronisation.
//
// Vector kernels share one decomposition (CTA = 2048 points of one band) so
// that dot products leave per-CTA partial sums that k_finish adds in a fixed
// order: results are bit-reproducible run to run.
#include <cmath>

#include "cgvec.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace rsdft {

// ----------------------------------------------------------- reductions
__global__ void k_finish(const double* __restrict__ part, int nchunk, int K, int nb, double scale,
                         double* __restrict__ out, const int* __restrict__ active) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb * K) return;
    int b = i / K, k = i - b * K;
    if (active && !active[b]) return;
    const double* p = part + (long)b * nchunk * K + k;
    double s = 0.0;
    for (int c = 0; c < nchunk; ++c) s += p[(long)c * K];
    out[i] = s * scale;
}

// Dot-product pair tables as types, so every operand index is a compile-time
// constant and the per-element values stay in registers.
struct DotsXY {  // <v0|v1>
    static constexpr int K = 1;
    __host__ __device__ static constexpr int a(int) { return 0; }
    __host__ __device__ static constexpr int b(int) { return 1; }
};
struct DotsCG6 {  // <x|x>, <p|x>, <p|p>, <x|Hx>, <p|Hx>, <p|Hp> for (x, p, Hx, Hp)
    static constexpr int K = 6;
    __host__ __device__ static constexpr int a(int k) { return (k == 0 || k == 3) ? 0 : 1; }
    __host__ __device__ static constexpr int b(int k) { return k < 2 ? 0 : (k == 2 ? 1 : (k == 5 ? 3 : 2)); }
};

// K dot products per band among up to 4 vectors, one read of each vector.
template <typename T, int NV, class P>
__global__ void __launch_bounds__(VT) k_multidot(const T* v0, const T* v1, const T* v2, const T* v3, long ld,
                                                 long n, double* __restrict__ part, const int* __restrict__ active,
                                                 int vec) {
    constexpr int K = P::K;
    using G = Grp16<T>;
    constexpr int W = G::W;
    __shared__ double sh[K * (VT / 32)];
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const T* vs[4] = {v0, v1, v2, v3};
    const long off = (long)b * ld;
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    const long base = (long)blockIdx.x * VCHUNK;
#pragma unroll 4
    for (int j = 0; j < VITEMS / W; ++j) {
        const long i = base + ((long)j * VT + threadIdx.x) * W;
        T vv[NV][W];
        if (vec && i + W <= n) {
#pragma unroll
            for (int q = 0; q < NV; ++q) G::load(vs[q] + off + i, vv[q]);
        } else {
#pragma unroll
            for (int q = 0; q < NV; ++q)
#pragma unroll
                for (int e = 0; e < W; ++e) vv[q][e] = i + e < n ? vs[q][off + i + e] : (T)0;
        }
#pragma unroll
        for (int e = 0; e < W; ++e) {
            double v[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) v[q] = (double)vv[q][e];
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] = fma(v[P::a(k)], v[P::b(k)], acc[k]);
        }
    }
    block_sum_n<VT, K>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) part[((long)b * gridDim.x + blockIdx.x) * K + k] = acc[k];
    }
}

// g = -c1 (hx - E x); partial |g|^2 (cg_module.f90:186-190)
template <typename T>
__global__ void __launch_bounds__(VT) k_cg_g(CGVec<T> v, long ld, long n, const double* __restrict__ E,
                                             double* __restrict__ part, const int* __restrict__ active, int vec) {
    using G = Grp16<T>;
    constexpr int W = G::W;
    __shared__ double sh[VT / 32];
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const T e = (T)E[b];
    double acc = 0.0;
    const long base = (long)blockIdx.x * VCHUNK, off = (long)b * ld;
#pragma unroll 4
    for (int j = 0; j < VITEMS / W; ++j) {
        const long i = base + ((long)j * VT + threadIdx.x) * W;
        if (vec && i + W <= n) {
            T hx[W], x[W], g[W];
            G::load(v.hx + off + i, hx);
            G::load(v.x + off + i, x);
#pragma unroll
            for (int q = 0; q < W; ++q) {
                g[q] = (T)(-2.0) * (hx[q] - e * x[q]);
                acc = fma((double)g[q], (double)g[q], acc);
            }
            G::store(v.g + off + i, g);
        } else {
            for (int q = 0; q < W && i + q < n; ++q) {
                const T g = (T)(-2.0) * (v.hx[off + i + q] - e * v.x[off + i + q]);
                v.g[off + i + q] = g;
                acc = fma((double)g, (double)g, acc);
            }
        }
    }
    double r = block_sum<VT>(acc, sh);
    if (threadIdx.x == 0) part[(long)b * gridDim.x + blockIdx.x] = r;
}

// P0: Pg = g; r = g - A g; q = r; partial |r|^2  (cgpc_hprsdft_module.f90:161-175)
template <typename T>
__global__ void __launch_bounds__(VT) k_pc0(CGVec<T> v, long ld, long n, PcArgs pa, double* __restrict__ part,
                                            const int* __restrict__ active) {
    __shared__ double sh[VT / 32];
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    const T* g = v.g + off;
    double acc = 0.0;
    int i1, i2, i3;
    pc_coords(base + threadIdx.x, pa, i1, i2, i3);
#pragma unroll 8
    for (int it = 0; it < VITEMS; ++it) {
        const long i = base + it * VT + threadIdx.x;
        if (i < n) {
            const T gi = g[i];
            const T f = pc_apply<T>(g, i, i1, i2, i3, pa);
            const T r = gi - f;
            v.Pg[off + i] = gi;
            v.r[off + i] = r;
            v.q[off + i] = r;
            acc = fma((double)r, (double)r, acc);
        }
        pc_step(pa, i1, i2, i3);
    }
    double s = block_sum<VT>(acc, sh);
    if (threadIdx.x == 0) part[(long)b * gridDim.x + blockIdx.x] = s;
}

// P1: ft = A q; partial q.ft  (ft stored in hp, which is free until hpsi(p))
template <typename T>
__global__ void __launch_bounds__(VT) k_pc1(CGVec<T> v, long ld, long n, PcArgs pa, double* __restrict__ part,
                                            const int* __restrict__ active) {
    __shared__ double sh[VT / 32];
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    const T* q = v.q + off;
    double acc = 0.0;
    int i1, i2, i3;
    pc_coords(base + threadIdx.x, pa, i1, i2, i3);
#pragma unroll 8
    for (int it = 0; it < VITEMS; ++it) {
        const long i = base + it * VT + threadIdx.x;
        if (i < n) {
            const T f = pc_apply<T>(q, i, i1, i2, i3, pa);
            v.hp[off + i] = f;
            acc = fma((double)q[i], (double)f, acc);
        }
        pc_step(pa, i1, i2, i3);
    }
    double s = block_sum<VT>(acc, sh);
    if (threadIdx.x == 0) part[(long)b * gridDim.x + blockIdx.x] = s;
}

// P2: Pg += a q; (not last) r -= a ft; partial |r|^2
template <typename T>
__global__ void __launch_bounds__(VT) k_pc2(CGVec<T> v, long ld, long n, const double* __restrict__ pa_,
                                            int last, double* __restrict__ part, const int* __restrict__ active) {
    __shared__ double sh[VT / 32];
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    const T a = (T)pa_[b];
    double acc = 0.0;
#pragma unroll 8
    for (int it = 0; it < VITEMS; ++it) {
        const long i = base + it * VT + threadIdx.x;
        if (i < n) {
            const T qi = v.q[off + i];
            v.Pg[off + i] = v.Pg[off + i] + a * qi;
            if (!last) {
                const T r = v.r[off + i] - a * v.hp[off + i];
                v.r[off + i] = r;
                acc = fma((double)r, (double)r, acc);
            }
        }
    }
    if (!last) {
        double s = block_sum<VT>(acc, sh);
        if (threadIdx.x == 0) part[(long)b * gridDim.x + blockIdx.x] = s;
    }
}

// P3: q = r + b q
template <typename T>
__global__ void __launch_bounds__(VT) k_pc3(CGVec<T> v, long ld, long n, const double* __restrict__ pb_,
                                            const int* __restrict__ active) {
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    const T bb = (T)pb_[b];
#pragma unroll 8
    for (int it = 0; it < VITEMS; ++it) {
        const long i = base + it * VT + threadIdx.x;
        if (i < n) v.q[off + i] = v.r[off + i] + bb * v.q[off + i];
    }
}

// p = Pg + bk p (icg > 1) or p = Pg (cg_module.f90:247-261)
template <typename T>
__global__ void __launch_bounds__(VT) k_cg_p(CGVec<T> v, long ld, long n, const double* __restrict__ bk_,
                                             int first, const int* __restrict__ active) {
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    const T bk = (T)bk_[b];
#pragma unroll 8
    for (int it = 0; it < VITEMS; ++it) {
        const long i = base + it * VT + threadIdx.x;
        if (i < n) v.p[off + i] = first ? v.Pg[off + i] : v.Pg[off + i] + bk * v.p[off + i];
    }
}

// hx = u11 hx + u21 hp; g = -c1 (hx - W (u11 x + u21 p)); partial |g|^2 (:337-347)
template <typename T>
__device__ __forceinline__ T cg_upd1_elem(T& hx, T hp, T x, T p, T u11, T u21, T w) {
    hx = u11 * hx + u21 * hp;
    return (T)(-2.0) * (hx - w * (u11 * x + u21 * p));
}

template <typename T>
__global__ void __launch_bounds__(VT) k_cg_upd1(CGVec<T> v, long ld, long n, CGScal s, double* __restrict__ part,
                                                const int* __restrict__ active, int vec) {
    using G = Grp16<T>;
    constexpr int W = G::W;
    __shared__ double sh[VT / 32];
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    const T u11 = (T)s.u11[b], u21 = (T)s.u21[b], w = (T)s.W[b];
    double acc = 0.0;
#pragma unroll 4
    for (int j = 0; j < VITEMS / W; ++j) {
        const long i = base + ((long)j * VT + threadIdx.x) * W;
        if (vec && i + W <= n) {
            T hx[W], hp[W], x[W], p[W], g[W];
            G::load(v.hx + off + i, hx);
            G::load(v.hp + off + i, hp);
            G::load(v.x + off + i, x);
            G::load(v.p + off + i, p);
#pragma unroll
            for (int q = 0; q < W; ++q) {
                g[q] = cg_upd1_elem(hx[q], hp[q], x[q], p[q], u11, u21, w);
                acc = fma((double)g[q], (double)g[q], acc);
            }
            G::store(v.hx + off + i, hx);
            G::store(v.g + off + i, g);
        } else {
            for (int q = 0; q < W && i + q < n; ++q) {
                const long k = off + i + q;
                T hx = v.hx[k];
                const T g = cg_upd1_elem(hx, v.hp[k], v.x[k], v.p[k], u11, u21, w);
                v.hx[k] = hx;
                v.g[k] = g;
                acc = fma((double)g, (double)g, acc);
            }
        }
    }
    double r = block_sum<VT>(acc, sh);
    if (threadIdx.x == 0) part[(long)b * gridDim.x + blockIdx.x] = r;
}

// x = u11 x + u21 p unless rejected (:366-369)
template <typename T>
__global__ void __launch_bounds__(VT) k_cg_upd2(CGVec<T> v, long ld, long n, CGScal s,
                                                const int* __restrict__ active, int vec) {
    using G = Grp16<T>;
    constexpr int W = G::W;
    const int b = blockIdx.y;
    if (active && !active[b]) return;
    if (s.reject[b]) return;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    const T u11 = (T)s.u11[b], u21 = (T)s.u21[b];
#pragma unroll 4
    for (int j = 0; j < VITEMS / W; ++j) {
        const long i = base + ((long)j * VT + threadIdx.x) * W;
        if (vec && i + W <= n) {
            T x[W], p[W];
            G::load(v.x + off + i, x);
            G::load(v.p + off + i, p);
#pragma unroll
            for (int q = 0; q < W; ++q) x[q] = cg_upd2_elem(x[q], p[q], u11, u21);
            G::store(v.x + off + i, x);
        } else {
            for (int q = 0; q < W && i + q < n; ++q)
                v.x[off + i + q] = cg_upd2_elem(v.x[off + i + q], v.p[off + i + q], u11, u21);
        }
    }
}

// ---------------------------------------------------- per-band scalars
__global__ void s_init(CGScal s, int nb) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    s.E1[b] = 1e10;
    s.gkgk[b] = 0.0;
    s.active[b] = 1;
    s.reject[b] = 0;
    s.pend[b] = 0;
    if (b == 0) *s.rej_any = 0;
    s.res[b] = 0.0;
}

// top of the icg loop (cg_module.f90:205-219): a band stops once its
// Rayleigh quotient moved by less than tol_e in the last line step (the
// reference's 1e-15, cg_module.f90:218, in FP64)
__global__ void s_top(CGScal s, int nb, int last, double tol_e) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || !s.active[b]) return;
    const double rb = s.rb[b];
    s.res[b] = rb / 4.0;
    if (rb < 0.0 || fabs(s.E[b] - s.E1[b]) < tol_e || last) s.active[b] = 0;
}

// The stopping tolerance of a line step.  FP64 bands use the reference's
// 1e-15.  The Rayleigh quotient of an FP32 band (FP64 dots of FP32 vectors
// and an FP32 H x) never settles that far: once converged it keeps moving by
// 3e-12 .. 3e-11 Ha per step (median 2.5e-11, measured on the 216-atom cell
// after 10 to 30 iterations), so the FP32 form stops a band at 1e-10 Ha, the
// same rule one level above its noise floor, four orders of magnitude below
// the 1e-6 Ha eigenvalue tolerance of the mixed forms.
template <typename T>
constexpr double cg_stop_tol() {
    return sizeof(T) == 8 ? 1e-15 : 1e-10;
}

__global__ void s_pc0(CGScal s, int nb) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    s.pc_active[b] = s.active[b] && !(s.rr1[b] < 1e-24);
}

__global__ void s_pc1(CGScal s, int nb) {  // rr0 = rr1; a = rr0/pAp (pAp in dots[b])
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || !s.pc_active[b]) return;
    s.rr0[b] = s.rr1[b];
    s.pa[b] = s.rr0[b] / s.dots[b];
}

__global__ void s_pc2(CGScal s, int nb) {  // b = rr1/rr0
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || !s.pc_active[b]) return;
    s.pb[b] = s.rr1[b] / s.rr0[b];
}

__global__ void s_p(CGScal s, int nb, int first) {  // bk = rb/gkgk; gkgk = rb
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || !s.active[b]) return;
    s.bk[b] = first ? 0.0 : s.rb[b] / s.gkgk[b];
    s.gkgk[b] = s.rb[b];
}

// Smallest-eigenvalue pair of the 2x2 pencil (A, B), B = U^T U, B-normalised.
// Closed form: Cholesky of B, C = U^-T A U^-1, symmetric 2x2 eigen-pairs
// with the cancellation-free root and the better-conditioned eigenvector
// formula, back-transform x = U^-1 z.
__device__ void eig2(double a11, double a12, double a22, double b11, double b12, double b22, double* W,
                     double* X /* 2x2 column-major */, int* info) {
    *info = 0;
    if (!(b11 > 0.0)) { *info = 1; return; }
    const double u11 = sqrt(b11), u12 = b12 / u11, t = b22 - u12 * u12;
    if (!(t > 0.0)) { *info = 2; return; }
    const double u22 = sqrt(t);
    const double c11 = a11 / b11;
    const double r12 = a12 / u11;
    const double c12 = (r12 - c11 * u12) / u22;
    const double c22 = (a22 - 2.0 * u12 * r12 + u12 * u12 * c11) / (u22 * u22);
    const double m = 0.5 * (c11 + c22), d = 0.5 * (c11 - c22);
    const double rt = hypot(d, c12);
    const double det = c11 * c22 - c12 * c12;
    double lo, hi;
    if (m > 0.0) { hi = m + rt; lo = det / hi; }
    else if (m < 0.0) { lo = m - rt; hi = det / lo; }
    else { lo = -rt; hi = rt; }
    double z0, z1;
    if (rt == 0.0) {
        z0 = 1.0; z1 = 0.0;
    } else {
        // eigenvector of lo: (c12, lo - c11) or (lo - c22, c12), the larger one
        const double p0 = c12, p1 = lo - c11, q0 = lo - c22, q1 = c12;
        if (p0 * p0 + p1 * p1 >= q0 * q0 + q1 * q1) { z0 = p0; z1 = p1; } else { z0 = q0; z1 = q1; }
        const double nz = hypot(z0, z1);
        z0 /= nz; z1 /= nz;
    }
    // second pair orthogonal in the reduced space
    const double y0 = -z1, y1 = z0;
    W[0] = lo; W[1] = hi;
    X[1] = z1 / u22; X[0] = (z0 - u12 * X[1]) / u11;
    X[3] = y1 / u22; X[2] = (y0 - u12 * X[3]) / u11;
}

// 2x2 Rayleigh-Ritz, pair choice and sign fix (cg_module.f90:299-333)
__global__ void s_eig(CGScal s, int nb) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || !s.active[b]) return;
    const double* v = s.dots + 6L * b;  // xx, px, pp, xHx, pHx, pHp
    double W[2], X[4];
    int info;
    eig2(v[3], v[4], v[5], v[0], v[1], v[2], W, X, &info);
    if (info != 0) {  // B not positive definite: keep x (no update)
        W[0] = s.E[b]; X[0] = 1.0; X[1] = 0.0;
    } else if (fabs(W[0] - s.E[b]) > 1e-1 && fabs(W[1] - s.E[b]) <= 1e-1) {
        X[0] = X[2]; X[1] = X[3]; W[0] = W[1];
    }
    if (X[0] < 0.0) { X[0] = -X[0]; X[1] = -X[1]; }
    s.E1[b] = s.E[b];
    s.E[b] = W[0];
    s.W[b] = W[0];
    s.u11[b] = X[0];
    s.u21[b] = X[1];
}

__global__ void s_rej(CGScal s, int nb) {  // cg_module.f90:359-365
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    if (!s.active[b]) {
        s.pend[b] = 0;
        return;
    }
    s.reject[b] = 0;
    if (s.rb[b] / s.res[b] > 1e8) {
        s.E[b] = s.E1[b];
        s.reject[b] = 1;
        *s.rej_any = 1;
    }
    s.pend[b] = !s.reject[b];
}

template <typename T>
__global__ void k_convert(const double* __restrict__ a, T* __restrict__ b, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (T)a[i];
}

template <typename T>
__global__ void k_convert_back(const T* __restrict__ a, double* __restrict__ b, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (double)a[i];
}

// sum_i (hx - e x)^2 per band (residual norms after the eigenvalues are known)
__global__ void __launch_bounds__(VT) k_resid(const double* __restrict__ x, const double* __restrict__ hx, long ld,
                                              long n, const double* __restrict__ e, double* __restrict__ part) {
    __shared__ double sh[VT / 32];
    const int b = blockIdx.y;
    const long off = (long)b * ld, base = (long)blockIdx.x * VCHUNK;
    const double eb = e[b];
    double acc = 0.0;
#pragma unroll 8
    for (int it = 0; it < VITEMS; ++it) {
        const long i = base + it * VT + threadIdx.x;
        if (i < n) {
            const double r = hx[off + i] - eb * x[off + i];
            acc = fma(r, r, acc);
        }
    }
    double s = block_sum<VT>(acc, sh);
    if (threadIdx.x == 0) part[(long)b * gridDim.x + blockIdx.x] = s;
}

// e(n) = dV <x_n|H x_n> (esp_calc_module.f90:33-42) and, if res != NULL,
// res(n) = dV |H x_n - e(n) x_n|^2, all FP64 (device pointers)
int esp_device(const double* x, long ld, int nb, int spin, double* e, double* res) {
    Context& c = ctx();
    cudaStream_t st = c.stream;
    const long n = c.ml;
    const int nchunk = div_up(n, VCHUNK);
    double *hx = nullptr, *part = nullptr;
    RS_CHECK(workspace_t("esp_hx", (size_t)ld * nb, &hx));
    RS_CHECK(workspace_t("esp_part", (size_t)nb * nchunk, &part));
    RS_CHECK(hpsi_device<double>(x, hx, ld, nb, spin, nullptr));
    const dim3 vg(nchunk, nb);
    const int gv = grp16_ok<double>(ld, {x, hx}) ? 1 : 0;
    launch(k_multidot<double, 2, DotsXY>, vg, VT, 0, st, x, hx, nullptr, nullptr, ld, n, part, nullptr, gv);
    launch(k_finish, div_up(nb, 128), 128, 0, st, part, nchunk, 1, nb, c.dV, e, nullptr);
    if (res) {
        launch(k_resid, vg, VT, 0, st, x, hx, ld, n, e, part);
        launch(k_finish, div_up(nb, 128), 128, 0, st, part, nchunk, 1, nb, c.dV, res, nullptr);
    }
    RS_LAUNCH();
    return RSDFT_OK;
}

// ------------------------------------------------------------ driver
template <typename T>
static int cg_run(T* x, long ld, int mb, int spin, double* esp, double* res, int ncg, int mloop, int ipc) {
    Context& c = ctx();
    cudaStream_t st = c.stream;
    const long n = c.ml;
    const int nchunk = div_up(n, VCHUNK);
    const size_t vec = (size_t)ld * mb;
    CGVec<T> v{};
    v.x = x;
    T* base = nullptr;
    RS_CHECK(workspace_t("cg_vec", vec * 7, &base));
    v.hx = base;
    v.hp = base + vec;
    v.g = base + 2 * vec;
    v.Pg = base + 3 * vec;
    v.p = base + 4 * vec;
    v.r = base + 5 * vec;
    v.q = base + 6 * vec;
    double* scal = nullptr;
    RS_CHECK(workspace_t("cg_scal", (size_t)mb * (20 + SS_STRIDE + SS_MAXM), &scal));
    CGScal s{};
    s.E = scal; s.E1 = scal + mb; s.rb = scal + 2 * mb; s.gkgk = scal + 3 * mb; s.res = scal + 4 * mb;
    s.u11 = scal + 5 * mb; s.u21 = scal + 6 * mb; s.W = scal + 7 * mb; s.rr0 = scal + 8 * mb;
    s.rr1 = scal + 9 * mb; s.pa = scal + 10 * mb; s.pb = scal + 11 * mb; s.bk = scal + 12 * mb;
    s.dots = scal + 13 * mb;  // 6 per band
    double* ss = scal + 20 * mb;                 // s-step Gram / g-dot slots, SS_STRIDE per band
    double* cz = ss + (size_t)SS_STRIDE * mb;    // s-step coefficients, SS_MAXM per band
    int* flags = nullptr;
    RS_CHECK(workspace_t("cg_flags", (size_t)mb * 4 + 1, &flags));
    s.active = flags; s.pc_active = flags + mb; s.reject = flags + 2 * mb; s.pend = flags + 3 * mb;
    s.rej_any = flags + 4 * mb;
    double* part = nullptr;
    RS_CHECK(workspace_t("cg_part", (size_t)mb * nchunk * 8, &part));

    const dim3 vg(nchunk, mb);
    const int sb = div_up(mb, 128);
    const double dV = c.dV;
    const int gv = grp16_ok<T>(ld, {x, base}) ? 1 : 0;  // 16-byte element groups
    PcArgs pa{c.n1, c.n2, c.n3, VT % c.n1, (VT / c.n1) % c.n2, VT / (c.n1 * c.n2),
              c.pc.c - 0.0, c.pc.c1, c.pc.c2, c.pc.c3};
    auto finish = [&](int K, double scale, double* out, const int* act) {
        launch(k_finish, div_up((long)mb * K, 128), 128, 0, st, part, nchunk, K, mb, scale, out, act);
    };

    launch(s_init, sb, 128, 0, st, s, mb);
    RS_CHECK(hpsi_device<T>(x, v.hx, ld, mb, spin, nullptr));
    {
        launch(k_multidot<T, 2, DotsXY>, vg, VT, 0, st, x, v.hx, nullptr, nullptr, ld, n, part, nullptr, gv);
        finish(1, dV, s.E, nullptr);
    }
    launch(k_cg_g<T>, vg, VT, 0, st, v, ld, n, s.E, part, nullptr, gv);
    finish(1, dV, s.rb, nullptr);
    RS_LAUNCH();

    const bool sstep = ipc == 4 && mloop >= 1 && mloop <= SS_MAXM;
    for (int icg = 1; icg <= ncg + 1; ++icg) {
        const int last = icg == ncg + 1;
        launch(s_top, sb, 128, 0, st, s, mb, last, cg_stop_tol<T>());
        if (last) break;
        if (sstep) {
            // --- preconditioner, rb = <Pg|g> dV and the search direction p
            // in mloop + 2 passes (s-step form; w_j in r, q, Pg, hp, which
            // are free until hpsi(p))
            const SSVec<T> sv{{v.r, v.q, v.Pg, v.hp}};
            RS_CHECK(sstep_precond<T>(v.g, sv, v.p, x, ld, mb, mloop, icg == 1, s, ss, cz, part, pa, dV));
        } else {
            // --- preconditioning (Pgk = gk on entry)
            if (ipc == 4 && mloop > 0) {
                launch(k_pc0<T>, vg, VT, 0, st, v, ld, n, pa, part, s.active);
                finish(1, 1.0, s.rr1, s.active);
                launch(s_pc0, sb, 128, 0, st, s, mb);
                for (int il = 1; il <= mloop; ++il) {
                    launch(k_pc1<T>, vg, VT, 0, st, v, ld, n, pa, part, s.pc_active);
                    finish(1, 1.0, s.dots, s.pc_active);
                    launch(s_pc1, sb, 128, 0, st, s, mb);
                    const int lastl = il == mloop;
                    launch(k_pc2<T>, vg, VT, 0, st, v, ld, n, s.pa, lastl, part, s.pc_active);
                    if (lastl) break;
                    finish(1, 1.0, s.rr1, s.pc_active);
                    launch(s_pc2, sb, 128, 0, st, s, mb);
                    launch(k_pc3<T>, vg, VT, 0, st, v, ld, n, s.pb, s.pc_active);
                }
            } else {
                RS_CUDA(cudaMemcpyAsync(v.Pg, v.g, vec * sizeof(T), cudaMemcpyDeviceToDevice, st));
            }
            RS_LAUNCH();
            // --- rb = <Pg|g> dV; search direction
            {
                launch(k_multidot<T, 2, DotsXY>, vg, VT, 0, st, v.Pg, v.g, nullptr, nullptr, ld, n, part, s.active,
                       gv);
                finish(1, dV, s.rb, s.active);
            }
            launch(s_p, sb, 128, 0, st, s, mb, icg == 1);
            launch(k_cg_p<T>, vg, VT, 0, st, v, ld, n, s.bk, icg == 1, s.active);
            RS_LAUNCH();
        }
        RS_CHECK(hpsi_device<T>(v.p, v.hp, ld, mb, spin, s.active));
        // --- six dots: <x|x>, <p|x>, <p|p>, <x|Hx>, <p|Hx>, <p|Hp>
        {
            launch(k_multidot<T, 4, DotsCG6>, vg, VT, 0, st, x, v.p, v.hx, v.hp, ld, n, part, s.active, gv);
            finish(6, dV, s.dots, s.active);
        }
        launch(s_eig, sb, 128, 0, st, s, mb);
        launch(k_cg_upd1<T>, vg, VT, 0, st, v, ld, n, s, part, s.active, gv);
        finish(1, dV, s.rb, s.active);
        launch(s_rej, sb, 128, 0, st, s, mb);
        // s-step form: the x update waits for the next search-direction pass,
        // which reads the old p anyway
        if (!sstep) launch(k_cg_upd2<T>, vg, VT, 0, st, v, ld, n, s, s.active, gv);
        RS_LAUNCH();
    }
    if (sstep) {  // the last step's update
        launch(k_cg_upd2<T>, vg, VT, 0, st, v, ld, n, s, (const int*)s.pend, gv);
        RS_LAUNCH();
    }
    RS_CUDA(cudaMemcpyAsync(esp, s.E, sizeof(double) * mb, cudaMemcpyDeviceToDevice, st));
    RS_CUDA(cudaMemcpyAsync(res, s.res, sizeof(double) * mb, cudaMemcpyDeviceToDevice, st));
    return RSDFT_OK;
}

int cg_device_f32(const double* unk, long ld, int mb, int spin, double* esp, double* res, int ncg, int mloop,
                  int ipc, float** x32_out, const float** hx_out) {
    Context& c = ctx();
    float* x32 = nullptr;
    const long n = ld * (long)mb;
    RS_CHECK(workspace_t("cg_x32", (size_t)n, &x32));
    launch(k_convert<float>, 4 * c.num_sms, 256, 0, c.stream, unk, x32, n);
    RS_LAUNCH();
    RS_CHECK(cg_run<float>(x32, ld, mb, spin, esp, res, ncg, mloop, ipc));
    *x32_out = x32;
    if (hx_out) {
        // the sweep's H x: the CG keeps hx = H x through its updates, except
        // for a band whose update was rejected (cg_module.f90:359-365)
        *hx_out = nullptr;
        float* hx = nullptr;
        int* flags = nullptr;
        RS_CHECK(workspace_t("cg_vec", (size_t)ld * mb * 7, &hx));
        RS_CHECK(workspace_t("cg_flags", (size_t)mb * 4 + 1, &flags));
        int rej = 1;
        RS_CUDA(cudaMemcpyAsync(&rej, flags + 4 * mb, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
        RS_CUDA(cudaStreamSynchronize(c.stream));
        if (rej == 0) *hx_out = hx;
    }
    return RSDFT_OK;
}

__global__ void k_or_flag(int* __restrict__ dst, const int* __restrict__ src) {
    if (*src) *dst = 1;
}

int cg_device_f32_staged(const double* unk_host, double* unk_dev, long ld, int mb, int spin, double* esp,
                         double* res, int ncg, int mloop, int ipc, int nchunk, float** x32_out,
                         const float** hx_out) {
    Context& c = ctx();
    nchunk = std::max(1, std::min(nchunk, std::min(mb, Context::NEV)));
    const int per = div_up(mb, nchunk);
    float *x32 = nullptr, *hx_all = nullptr;
    int* rej = nullptr;
    RS_CHECK(workspace_t("cg_x32", (size_t)ld * mb, &x32));
    RS_CHECK(workspace_t("sweep_hx", (size_t)ld * mb, &hx_all));
    RS_CHECK(workspace_t("sweep_rej", 1, &rej));
    RS_CUDA(cudaMemsetAsync(rej, 0, sizeof(int), c.stream));
    // every band block's upload on the copy stream, each followed by an event
    for (int k = 0, b0 = 0; b0 < mb; ++k, b0 += per) {
        const int nb = std::min(per, mb - b0);
        RS_CUDA(cudaMemcpyAsync(unk_dev + (size_t)b0 * ld, unk_host + (size_t)b0 * ld,
                                sizeof(double) * (size_t)ld * nb, cudaMemcpyHostToDevice, c.copy_stream));
        RS_CUDA(cudaEventRecord(c.ev[k], c.copy_stream));
    }
    for (int k = 0, b0 = 0; b0 < mb; ++k, b0 += per) {
        const int nb = std::min(per, mb - b0);
        const long n = ld * (long)nb;
        RS_CUDA(cudaStreamWaitEvent(c.stream, c.ev[k], 0));
        float* xb = x32 + (size_t)b0 * ld;
        launch(k_convert<float>, 4 * c.num_sms, 256, 0, c.stream, (const double*)(unk_dev + (size_t)b0 * ld), xb, n);
        RS_LAUNCH();
        RS_CHECK(cg_run<float>(xb, ld, nb, spin, esp + b0, res + b0, ncg, mloop, ipc));
        // this block's H x out of the CG workspace, and its rejection flag
        float* hx = nullptr;
        int* flags = nullptr;
        RS_CHECK(workspace_t("cg_vec", (size_t)ld * nb * 7, &hx));
        RS_CHECK(workspace_t("cg_flags", (size_t)nb * 4 + 1, &flags));
        RS_CUDA(cudaMemcpyAsync(hx_all + (size_t)b0 * ld, hx, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice,
                                c.stream));
        launch(k_or_flag, 1, 1, 0, c.stream, rej, (const int*)(flags + 4 * nb));
        RS_LAUNCH();
    }
    *x32_out = x32;
    int h = 1;
    RS_CUDA(cudaMemcpyAsync(&h, rej, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    *hx_out = h == 0 ? hx_all : nullptr;
    return RSDFT_OK;
}

int cg_device(double* unk, long ld, int mb, int spin, double* esp, double* res, int ncg, int mloop, int ipc,
              int mode, const double** hx_out) {
    if (mode == RSDFT_MODE_FP64) {
        RS_CHECK(cg_run<double>(unk, ld, mb, spin, esp, res, ncg, mloop, ipc));
        if (hx_out) {
            // as in cg_device_f32: the CG's hx is H x unless an update was
            // rejected (cg_module.f90:359-365)
            Context& c = ctx();
            *hx_out = nullptr;
            double* hx = nullptr;
            int* flags = nullptr;
            RS_CHECK(workspace_t("cg_vec", (size_t)ld * mb * 7, &hx));
            RS_CHECK(workspace_t("cg_flags", (size_t)mb * 4 + 1, &flags));
            int rej = 1;
            RS_CUDA(cudaMemcpyAsync(&rej, flags + 4 * mb, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
            RS_CUDA(cudaStreamSynchronize(c.stream));
            if (rej == 0) *hx_out = hx;
        }
        return RSDFT_OK;
    }
    Context& c = ctx();
    float* x32 = nullptr;
    const long n = ld * (long)mb;
    RS_CHECK(workspace_t("cg_x32", (size_t)n, &x32));
    launch(k_convert<float>, 4 * c.num_sms, 256, 0, c.stream, unk, x32, n);
    RS_LAUNCH();
    RS_CHECK(cg_run<float>(x32, ld, mb, spin, esp, res, ncg, mloop, ipc));
    launch(k_convert_back<float>, 4 * c.num_sms, 256, 0, c.stream, x32, unk, n);
    RS_LAUNCH();
    return RSDFT_OK;
}

}  // namespace rsdft

using namespace rsdft;

extern "C" int rsdft_gpu_esp_calc(int k, int s, const double* wf, int n1, int n2, int ns, int ne, double* e) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    if (k != 1) {
        set_error("esp_calc: only k=1 (Gamma) is supported");
        return RSDFT_EUNSUP;
    }
    if (s < 1 || s > c.nspin) {
        set_error("esp_calc: s=%d outside 1..%d", s, c.nspin);
        return RSDFT_EINVAL;
    }
    const long ld = (long)n2 - n1 + 1;
    const int nb = ne - ns + 1;
    if (ld != c.ml || nb < 1 || nb > 65535 || !e) {
        set_error("esp_calc: bad sizes (n2-n1+1=%ld ML=%ld)", ld, c.ml);
        return RSDFT_EINVAL;
    }
    double *d, *de;
    bool sw;
    RS_CHECK(wf_acquire(wf, ld, nb, "esp_wf", &d, &sw));
    RS_CHECK(workspace_t("esp_out", (size_t)nb, &de));
    RS_CHECK(esp_device(d, ld, nb, s, de, nullptr));
    RS_CHECK(stage_out(e, de, sizeof(double) * nb));
    return RSDFT_OK;
}

extern "C" int rsdft_gpu_residual(int k, int s, const double* wf, long ld, int nb, double* e, double* res) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    if (k != 1 || s < 1 || s > c.nspin || ld < c.ml || nb < 1 || nb > 65535 || !e || !res) {
        set_error("residual: bad arguments");
        return RSDFT_EINVAL;
    }
    double *d, *de;
    bool sw;
    RS_CHECK(wf_acquire(wf, ld, nb, "esp_wf", &d, &sw));
    RS_CHECK(workspace_t("esp_out", (size_t)2 * nb, &de));
    RS_CHECK(esp_device(d, ld, nb, s, de, de + nb));
    RS_CHECK(stage_out(e, de, sizeof(double) * nb));
    RS_CHECK(stage_out(res, de + nb, sizeof(double) * nb));
    return RSDFT_OK;
}

extern "C" int rsdft_gpu_conjugate_gradient(int n1, int n2, int mb, int k, int s, double* unk, double* esp,
                                            double* res, int ncg, int mloop, int ipc, int mode) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    if (k != 1) {
        set_error("conjugate_gradient: only k=1 (Gamma) is supported");
        return RSDFT_EUNSUP;
    }
    if (s < 1 || s > c.nspin) {
        set_error("conjugate_gradient: s=%d outside 1..%d", s, c.nspin);
        return RSDFT_EINVAL;
    }
    const long ld = (long)n2 - n1 + 1;
    if (ld != c.ml || mb < 1 || mb > 65535 || ncg < 0 || !esp || !res) {
        set_error("conjugate_gradient: bad sizes (ld=%ld ML=%ld MB=%d Ncg=%d)", ld, c.ml, mb, ncg);
        return RSDFT_EINVAL;
    }
    if (ipc != 0 && ipc != 4) {
        set_error("conjugate_gradient: ipc=%d unsupported (0 or 4)", ipc);
        return RSDFT_EUNSUP;
    }
    if (!mode_valid(mode)) {
        set_error("conjugate_gradient: mode=%d unknown", mode);
        return RSDFT_EINVAL;
    }
    double *du, *desp, *dres;
    bool su;
    RS_CHECK(wf_acquire(unk, ld, mb, "cg_unk", &du, &su));
    RS_CHECK(workspace_t("cg_out", (size_t)2 * mb, &desp));
    dres = desp + mb;
    RS_CHECK(cg_device(du, ld, mb, s, desp, dres, ncg, mloop, ipc, mode));
    RS_CHECK(stage_out(esp, desp, sizeof(double) * mb));
    RS_CHECK(stage_out(res, dres, sizeof(double) * mb));
    RS_CHECK(wf_release(unk, du, ld, mb, su));
    return RSDFT_OK;
}
