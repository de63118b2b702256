// Shared pieces of the CG sweep (cg.cu) and its preconditioner
// (precond.cu): vector-kernel decomposition, per-band scalar arrays, the
// 7-point preconditioner operator and the s-step basis vectors.
#pragma once

#include <cstdint>
#include <initializer_list>

#include "common.cuh"
#include "vec16.cuh"

namespace rsdft {

constexpr int VT = 256;           // threads per vector CTA
constexpr int VITEMS = 32;        // elements per thread
constexpr int VCHUNK = VT * VITEMS;

// 16-byte element groups of the vector kernels: a thread takes W = 16 /
// sizeof(T) consecutive elements per step (one vector access per stream);
// the scalar form serves misaligned shapes and the tail.
template <typename T>
struct Grp16 {
    static constexpr int W = 16 / (int)sizeof(T);
    using V = typename Vec16<T>::t;
    __device__ static __forceinline__ void load(const T* p, T (&v)[W]) {
        Vec16<T>::get(*reinterpret_cast<const V*>(p), v);
    }
    __device__ static __forceinline__ void store(T* p, const T (&v)[W]) {
        *reinterpret_cast<V*>(p) = Vec16<T>::make(v);
    }
};

// Whether 16-byte accesses suit vectors of leading dimension ld at these
// bases (host side).
template <typename T>
inline bool grp16_ok(long ld, std::initializer_list<const void*> ptrs) {
    if ((ld * (long)sizeof(T)) % 16 != 0) return false;
    for (const void* p : ptrs)
        if (p && reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
    return true;
}

struct CGScal {
    double *E, *E1, *rb, *gkgk, *res, *u11, *u21, *W, *rr0, *rr1, *pa, *pb, *bk, *dots;
    int *active, *pc_active, *reject;
    int* pend;     // x = u11 x + u21 p still to be applied (s-step form: by the next p pass)
    int* rej_any;  // set when any band's update was rejected (its hx then no longer equals H x)
};

// x = u11 x + u21 p (cg_module.f90:366-369), shared by the plain update and
// the one folded into the next search-direction pass so both give the same bits
template <typename T>
__device__ __forceinline__ T cg_upd2_elem(T x, T p, T u11, T u21) {
    return fma(u11, x, u21 * p);
}

template <typename T>
struct CGVec {
    T *x, *hx, *hp, *g, *Pg, *p, *r, *q;  // q = preconditioner search direction
};

// 7-point operator of precond_cg_mat2_omp (cgpc_hprsdft_module.f90:
// 290-340, E0 = 0) at point i = i1 + n1 (i2 + n2 i3), periodic.
struct PcArgs {
    int n1, n2, n3;
    int dx, dy, dz;  // VT points = dz planes + dy rows + dx (dx < n1, dy < n2)
    double d, c1, c2, c3;
};

template <typename T>
__device__ __forceinline__ T pc_apply(const T* __restrict__ f, long i, int i1, int i2, int i3, const PcArgs& pa) {
    const int n1 = pa.n1, n2 = pa.n2, n3 = pa.n3;
    const long pl = (long)n1 * n2;
    const long xm = i1 == 0 ? i + n1 - 1 : i - 1, xp = i1 == n1 - 1 ? i - n1 + 1 : i + 1;
    const long ym = i2 == 0 ? i + pl - n1 : i - n1, yp = i2 == n2 - 1 ? i - pl + n1 : i + n1;
    const long zm = i3 == 0 ? i + pl * (n3 - 1) : i - pl, zp = i3 == n3 - 1 ? i - pl * (n3 - 1) : i + pl;
    T v = (T)pa.d * f[i];
    v = v + (T)pa.c1 * (__ldg(f + xp) + __ldg(f + xm)) + (T)pa.c2 * (__ldg(f + yp) + __ldg(f + ym)) +
        (T)pa.c3 * (__ldg(f + zp) + __ldg(f + zm));
    return v;
}

// Grid coordinates of a thread's first point (one 32-bit division per
// thread); pc_step advances them by VT points without dividing.
__device__ __forceinline__ void pc_coords(long i, const PcArgs& pa, int& i1, int& i2, int& i3) {
    const unsigned pl = (unsigned)pa.n1 * (unsigned)pa.n2;
    const unsigned ii = (unsigned)i;
    i3 = (int)(ii / pl);
    const unsigned r = ii - (unsigned)i3 * pl;
    i2 = (int)(r / (unsigned)pa.n1);
    i1 = (int)(r - (unsigned)i2 * (unsigned)pa.n1);
}

__device__ __forceinline__ void pc_step(const PcArgs& pa, int& i1, int& i2, int& i3) {
    i1 += pa.dx;
    i2 += pa.dy;
    i3 += pa.dz;
    if (i1 >= pa.n1) {
        i1 -= pa.n1;
        ++i2;
    }
    if (i2 >= pa.n2) {
        i2 -= pa.n2;
        ++i3;
    }
}

// --------------------------------------- s-step preconditioner (IPC = 4)
// precond_hprsdft (cgpc_hprsdft_module.f90:126-348) runs mloop CG steps on
// A z = g from z = g with the 7-point operator A = d I + offdiag; every
// iterate lies in g + K_mloop(A, r0), r0 = g - A g.  In the Chebyshev basis
//   w_0 = r0,  w_1 = B w_0,  w_{k+1} = 2 B w_k - w_{k-1},   B = (A - d)/d
// (the spectrum of A is [0, 2d], so B maps it onto [-1, 1] and the basis
// stays well conditioned) A acts on coefficients as the tridiagonal
//   A w_0 = d (w_0 + w_1),  A w_k = d w_k + (d/2)(w_{k+1} + w_{k-1}),
// and every dot the recurrences need is a bilinear form in the Gram matrix
// G_ij = <w_i, w_j> (i < mloop, j <= mloop).  So: mloop passes build the
// basis and its Gram entries, the scalar recurrences of the reference run
// per band on coefficient vectors (s_sstep), and one pass forms
//   p = g + sum_j cz_j w_j + bk p
// (Pg itself, the rb = <Pg|g> dot and cg_module.f90:247-261 folded in).
// The result equals the reference's to rounding: the same Krylov
// polynomial, evaluated in another basis.
constexpr int SS_MAXM = 4;   // mloop handled by the s-step form
constexpr int SS_STRIDE = 20;  // Gram / g-dot slots per band

template <typename T>
struct SSVec {
    T* w[SS_MAXM];
};

// off-diagonal part of the 7-point operator at point i
template <typename T>
__device__ __forceinline__ T pc_offdiag(const T* __restrict__ f, long i, int i1, int i2, int i3, const PcArgs& pa) {
    const int n1 = pa.n1, n2 = pa.n2, n3 = pa.n3;
    const long pl = (long)n1 * n2;
    const long xm = i1 == 0 ? i + n1 - 1 : i - 1, xp = i1 == n1 - 1 ? i - n1 + 1 : i + 1;
    const long ym = i2 == 0 ? i + pl - n1 : i - n1, yp = i2 == n2 - 1 ? i - pl + n1 : i + n1;
    const long zm = i3 == 0 ? i + pl * (n3 - 1) : i - pl, zp = i3 == n3 - 1 ? i - pl * (n3 - 1) : i + pl;
    return (T)pa.c1 * (__ldg(f + xp) + __ldg(f + xm)) + (T)pa.c2 * (__ldg(f + yp) + __ldg(f + ym)) +
           (T)pa.c3 * (__ldg(f + zp) + __ldg(f + zm));
}

// Preconditioner + search direction of one CG step in the s-step form:
// p = Pg (first) or Pg + bk p, with rb = dV <Pg|g> and gkgk updated in s.
// ss and cz hold SS_STRIDE and SS_MAXM doubles per band, part the per-CTA
// partial sums (mb x nchunk x 8 doubles).
template <typename T>
int sstep_precond(const T* g, const SSVec<T>& sv, T* p, T* x, long ld, int mb, int mloop, int first, const CGScal& s,
                  double* ss, double* cz, double* part, const PcArgs& pa, double dV);

}  // namespace rsdft
