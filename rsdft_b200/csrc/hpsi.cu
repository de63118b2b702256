// hpsi on sm_100a: H psi = T psi + Vloc psi + V_nl psi for a batch of bands.
//
//  1. k_nl_project: uVunk(lma, b) = iuV dV sum_j uV(j) psi(JJP(j), b)
//     (ps_nloc2_op_module.f90:161-175), one sphere group x 32 bands per CTA.
//  2. k_stencil_tma: the Md-order periodic FD Laplacian (kinetic_sol_module.
//     f90:72-77, 129-149) fused with the Vloc multiply (localpot_module.f90:
//     73): TMA-fed plane ring, z "push" march with register accumulators.
//  3. k_nl_scatter: the nonlocal scatter-add (ps_nloc2_op_module.f90:
//     255-263) turned into a per-point gather over a point-major CSR, so every
//     sum is deterministic.
//  Shapes the TMA kernel does not take (odd row widths, rows wider than 256
//  elements) run k_stencil, a register-queue kernel with per-plane halo
//  loads and the scatter fused in its epilogue.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "tma.cuh"
#include "tmap.cuh"
#include "vec16.cuh"

namespace rsdft {

__device__ __forceinline__ int pwrap(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// ------------------------------------------------------------ projection
// A CTA takes one sphere group (up to 4 projectors sharing a point list) and
// PJ_WARPS x PJ_BW bands (16: two per warp, measured faster than four at
// Si216 480 bands, where more CTAs hide the gather latency better).  The
// group's point indices and projector values are staged in shared memory a
// chunk at a time; each lane strides the points and issues its warp's bands'
// gathers together.  Per (band, projector) the lanes sum points lane,
// lane+32, ... in order, then a fixed xor-shuffle tree.
constexpr int PJ_BW = 2;    // bands per warp
constexpr int PJ_WARPS = 8;
constexpr int PJ_CH = 512;  // sphere points staged per pass (multiple of 32)

template <typename T>
__global__ void __launch_bounds__(256) k_nl_project(const T* __restrict__ psi, long ld, int nb,
                                                    const int* __restrict__ grp_lma0,
                                                    const int* __restrict__ grp_cnt,
                                                    const int* __restrict__ lma_ptr,
                                                    const int* __restrict__ jjp,
                                                    const double* __restrict__ uv,
                                                    const int* __restrict__ iuv, double dV,
                                                    double* __restrict__ uvunk, int nzlma,
                                                    const int* __restrict__ band_active, int* __restrict__ err) {
    __shared__ int s_j[PJ_CH];
    __shared__ double s_u[4][PJ_CH];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = blockIdx.x;
    const int l0 = grp_lma0[g], cnt = grp_cnt[g];
    const int js = lma_ptr[l0], n = lma_ptr[l0 + 1] - js;
    int off[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) off[q] = q < cnt ? lma_ptr[l0 + q] : js;
    const int bw0 = (blockIdx.y * PJ_WARPS + warp) * PJ_BW;
    bool act[PJ_BW];
    const T* p[PJ_BW];
#pragma unroll
    for (int w = 0; w < PJ_BW; ++w) {
        const int b = bw0 + w;
        act[w] = b < nb && (!band_active || band_active[b]);
        p[w] = psi + (long)(act[w] ? b : 0) * ld;
    }
    double acc[PJ_BW][4];
#pragma unroll
    for (int w = 0; w < PJ_BW; ++w)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[w][q] = 0.0;
    for (int c0 = 0; c0 < n; c0 += PJ_CH) {
        const int m = min(PJ_CH, n - c0);
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            s_j[i] = jjp[js + c0 + i];
#pragma unroll
            for (int q = 0; q < 4; ++q) s_u[q][i] = q < cnt ? uv[off[q] + c0 + i] : 0.0;
        }
        __syncthreads();
#pragma unroll 2
        for (int j = lane; j < m; j += 32) {
            const int jj = s_j[j];
            const bool in = RS_DCHECK(jj >= 0 && jj < ld, CK_NL_PROJECT_POINT, jj, err);
            double v[PJ_BW];
#pragma unroll
            for (int w = 0; w < PJ_BW; ++w) v[w] = act[w] && in ? (double)__ldg(p[w] + jj) : 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (q < cnt) {
                    const double u = s_u[q][j];
#pragma unroll
                    for (int w = 0; w < PJ_BW; ++w) acc[w][q] = fma(u, v[w], acc[w][q]);
                }
            }
        }
    }
#pragma unroll
    for (int w = 0; w < PJ_BW; ++w)
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) acc[w][q] += __shfl_xor_sync(0xffffffffu, acc[w][q], s);
    if (lane == 0) {
#pragma unroll
        for (int w = 0; w < PJ_BW; ++w) {
            if (!act[w]) continue;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (q < cnt) uvunk[(long)(bw0 + w) * nzlma + l0 + q] = iuv[l0 + q] * dV * acc[w][q];
        }
    }
}

template <typename T>
static int launch_project(const T* psi, long ld, int nb, double* uvunk, const int* band_active, cudaStream_t st) {
    const Context& c = ctx();
    dim3 grid(c.ngroup, div_up(nb, PJ_WARPS * PJ_BW));
    launch(k_nl_project<T>, grid, 256, 0, st, psi, ld, nb, c.grp_lma0, c.grp_cnt, c.lma_ptr, c.jjp, c.uv, c.iuv,
           c.dV, uvunk, c.nzlma, band_active, c.err_flag);
    RS_LAUNCH();
    return RSDFT_OK;
}

// -------------------------------------------------------------- stencil
template <typename T>
struct StencilArgs {
    const T* psi;
    T* hpsi;
    long ld;
    int n1, n2, n3;
    int zlen, nzc;
    int z0, nzo;  // output planes [z0, z0 + nzo) (0, n3 when nzo = 0)
    const T* vloc;
    const int* pt_ptr;
    const int* pt_lma;
    const T* pt_uv;
    const double* uvunk;
    int nzlma;
    const int* band_active;
    const int* band_map;  // optional: launch band -> data band
    const int* gpt_ptr;   // point-major CSR over sphere groups
    const int* gpt_grp;
    const T* gpt_uv4;
};

template <typename T, int MD, int TX>
__global__ void __launch_bounds__(TX * 16) k_stencil(StencilArgs<T> a, StencilCoef cf) {
    constexpr int TY = 16, SX = TX + 2 * MD, SY = TY + 2 * MD, NT = TX * TY;
    __shared__ T tile[SY * SX];
    const int t = threadIdx.x;
    const int tx = t % TX, ty = t / TX;
    const int nzc = a.nzc;
    int band = blockIdx.z / nzc;
    const int zc = blockIdx.z - band * nzc;
    if (a.band_map) band = a.band_map[band];
    if (a.band_active && !a.band_active[band]) return;  // uniform per CTA
    const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int x = x0 + tx, y = y0 + ty;
    const bool act = (x < n1) && (y < n2);
    const long plane = (long)n1 * n2;
    const T* __restrict__ p = a.psi + (long)band * a.ld;
    T* __restrict__ h = a.hpsi + (long)band * a.ld;
    const int zs = a.z0 + zc * a.zlen;
    const int ze = min(zs + a.zlen, a.z0 + a.nzo);
    const long col = act ? (long)x + (long)n1 * y : 0;

    T cx[MD], cy[MD], cz[MD];
#pragma unroll
    for (int m = 0; m < MD; ++m) {
        cx[m] = (T)cf.cx[m];
        cy[m] = (T)cf.cy[m];
        cz[m] = (T)cf.cz[m];
    }
    const T c0 = (T)cf.c0;

    T q[2 * MD + 1];
#pragma unroll
    for (int k = 0; k < 2 * MD; ++k) q[k] = act ? __ldg(p + col + plane * pwrap(zs - MD + k, n3)) : (T)0;

    for (int z = zs; z < ze; ++z) {
        q[2 * MD] = act ? __ldg(p + col + plane * pwrap(z + MD, n3)) : (T)0;
        __syncthreads();
        if (act) tile[(ty + MD) * SX + tx + MD] = q[MD];
        const T* pz = p + plane * z;
        for (int c = t; c < SY * SX; c += NT) {
            const int sy = c / SX, sx = c - sy * SX;
            const int otx = sx - MD, oty = sy - MD;
            const bool interior = (otx >= 0 && otx < TX && oty >= 0 && oty < TY && x0 + otx < n1 && y0 + oty < n2);
            if (!interior) {
                const int gx = pwrap(x0 + otx, n1), gy = pwrap(y0 + oty, n2);
                tile[c] = __ldg(pz + gx + (long)n1 * gy);
            }
        }
        __syncthreads();
        if (act) {
            const T* row = tile + (ty + MD) * SX + tx + MD;
            T v = c0 * q[MD];
#pragma unroll
            for (int m = 1; m <= MD; ++m) {
                v = v + cx[m - 1] * (row[-m] + row[m]) + cy[m - 1] * (row[-m * SX] + row[m * SX]) +
                    cz[m - 1] * (q[MD - m] + q[MD + m]);
            }
            const long j = col + plane * z;
            v = v + __ldg(a.vloc + j) * q[MD];
            if (a.pt_ptr) {
                const int s = __ldg(a.pt_ptr + j), e = __ldg(a.pt_ptr + j + 1);
                const double* un = a.uvunk + (long)band * a.nzlma;
                for (int k = s; k < e; ++k) v = v + __ldg(a.pt_uv + k) * (T)__ldg(un + __ldg(a.pt_lma + k));
            }
            h[j] = v;
        }
#pragma unroll
        for (int k = 0; k < 2 * MD; ++k) q[k] = q[k + 1];
    }
}

struct TmaMaps {
    CUtensorMap full, edge, mid, wrap;  // psi boxes of height TY + 2 Md, TY + Md, TY, Md
    CUtensorMap vloc;                   // Vloc box of height TY
};

// Stencil coefficients in the kernel's arithmetic type, so every FMA takes
// its coefficient straight from the parameter bank (no per-use conversion).
template <typename T>
struct CoefT {
    T c0;
    T cx[MAXMD], cy[MAXMD], cz[MAXMD];
};

template <typename T>
static CoefT<T> coef_as(const StencilCoef& cf) {
    CoefT<T> o{};
    o.c0 = (T)cf.c0;
    for (int m = 0; m < MAXMD; ++m) {
        o.cx[m] = (T)cf.cx[m];
        o.cy[m] = (T)cf.cy[m];
        o.cz[m] = (T)cf.cz[m];
    }
    return o;
}

// Arithmetic lanes of the TMA stencil: one double, or two floats through the
// packed FP32 instructions of sm_100 (__ffma2_rn and friends: two
// independent IEEE operations per instruction, bitwise the same results as
// the scalar ones, half the issue slots).  A 16-byte shared-memory vector
// holds two packs in both cases.
template <typename T>
struct Pk;
template <>
struct Pk<double> {
    using t = double;
    static constexpr int W = 1;
    __device__ static __forceinline__ t fma(t a, t b, t c) { return __fma_rn(a, b, c); }
    __device__ static __forceinline__ t add(t a, t b) { return __dadd_rn(a, b); }
    __device__ static __forceinline__ t mul(t a, t b) { return __dmul_rn(a, b); }
    __device__ static __forceinline__ t splat(double v) { return v; }
    __device__ static __forceinline__ t of(const double* p) { return p[0]; }
    __device__ static __forceinline__ void get2(const double2& v, t* o) {
        o[0] = v.x;
        o[1] = v.y;
    }
    __device__ static __forceinline__ double2 put2(const t* o) { return make_double2(o[0], o[1]); }
    __device__ static __forceinline__ void unpack2(const t* c, double* o) {
        o[0] = c[0];
        o[1] = c[1];
    }
};
template <>
struct Pk<float> {
    using t = float2;
    static constexpr int W = 2;
    __device__ static __forceinline__ t fma(t a, t b, t c) { return __ffma2_rn(a, b, c); }
    __device__ static __forceinline__ t add(t a, t b) { return __fadd2_rn(a, b); }
    __device__ static __forceinline__ t mul(t a, t b) { return __fmul2_rn(a, b); }
    __device__ static __forceinline__ t splat(float v) { return make_float2(v, v); }
    __device__ static __forceinline__ t of(const float* p) { return make_float2(p[0], p[1]); }
    __device__ static __forceinline__ void get2(const float4& v, t* o) {
        o[0] = make_float2(v.x, v.y);
        o[1] = make_float2(v.z, v.w);
    }
    __device__ static __forceinline__ float4 put2(const t* o) { return make_float4(o[0].x, o[0].y, o[1].x, o[1].y); }
    __device__ static __forceinline__ void unpack2(const t* c, float* o) {
        o[0] = c[0].x;
        o[1] = c[0].y;
        o[2] = c[1].x;
        o[3] = c[1].y;
    }
};

// One arrival's z pushes for accumulator slot U (compile time): outputs
// U + m (first touch at m = Md) and U - m get cz_m c, slot U gets the in-plane
// part when the plane is one of the tile's own, and slot U + Md + 1 (the
// output completed by this arrival) is written when hp is set.  NK packs per
// thread, two per row.
template <typename T, int MD, int NK, int BY, int U>
__device__ __forceinline__ void push_body(typename Pk<T>::t (&acc)[2 * MD + 1][NK], const typename Pk<T>::t* c,
                                          const typename Pk<T>::t* in, bool inner, const CoefT<T>& cf, T* hp,
                                          int n1) {
    using P = Pk<T>;
    constexpr int Q = 2 * MD + 1;
#pragma unroll
    for (int i = 0; i < NK; ++i) {
        acc[(U + MD) % Q][i] = P::mul(P::splat(cf.cz[MD - 1]), c[i]);
#pragma unroll
        for (int m = 1; m < MD; ++m) acc[(U + m) % Q][i] = P::fma(P::splat(cf.cz[m - 1]), c[i], acc[(U + m) % Q][i]);
#pragma unroll
        for (int m = 1; m <= MD; ++m)
            acc[(U + Q - m) % Q][i] = P::fma(P::splat(cf.cz[m - 1]), c[i], acc[(U + Q - m) % Q][i]);
        if (inner) acc[U][i] = P::add(acc[U][i], in[i]);
    }
    if (hp) {
#pragma unroll
        for (int r = 0; r < BY; ++r)
            *reinterpret_cast<typename Vec16<T>::t*>(hp + (long)r * n1) = P::put2(&acc[(U + MD + 1) % Q][2 * r]);
    }
}

// Runtime slot -> compile-time slot: only the short push runs per case, so
// the loop body is not replicated 2 Md + 1 times.
template <typename T, int MD, int NK, int BY>
__device__ __forceinline__ void push_slot(int u, typename Pk<T>::t (&acc)[2 * MD + 1][NK], const typename Pk<T>::t* c,
                                          const typename Pk<T>::t* in, bool inner, const CoefT<T>& cf, T* hp,
                                          int n1) {
    constexpr int Q = 2 * MD + 1;
#define RS_PUSH_CASE(K)                                                                  \
    case K:                                                                              \
        if constexpr (K < Q) push_body<T, MD, NK, BY, K>(acc, c, in, inner, cf, hp, n1); \
        break;
    switch (u) {
        RS_PUSH_CASE(0) RS_PUSH_CASE(1) RS_PUSH_CASE(2) RS_PUSH_CASE(3) RS_PUSH_CASE(4) RS_PUSH_CASE(5)
        RS_PUSH_CASE(6) RS_PUSH_CASE(7) RS_PUSH_CASE(8) RS_PUSH_CASE(9) RS_PUSH_CASE(10) RS_PUSH_CASE(11)
        RS_PUSH_CASE(12) RS_PUSH_CASE(13) RS_PUSH_CASE(14) RS_PUSH_CASE(15) RS_PUSH_CASE(16)
        default: break;
    }
#undef RS_PUSH_CASE
}

// hpsi stencil + Vloc, TMA pipeline with a z "push" march.  A CTA owns TY
// full-width rows of one band and marches along z over planes zs-Md ..
// ze+Md-1.  One producer warp streams each plane (TY + 2 Md rows with the
// periodic y wrap split into boxes, plus the Vloc rows of the tile) into a
// ring of S shared-memory stages.  Each consumer thread owns VX (16 bytes)
// x BY points.  When plane P lands the thread
//  * forms the in-plane part of H psi at P (centre, Md x and y neighbours,
//    the x window read with periodic offsets, Vloc),
//  * adds cz_m psi(P) to the accumulators of the outputs P -+ m (m = 1..Md),
//  * and writes output P - Md, which is then complete.
// The 2 Md + 1 accumulators rotate through registers with compile-time
// indices (a switch on the slot selects the push), so a stage is read only
// while its own plane is current and the ring can stay shallow.
template <typename T, int MD, int BY>
__global__ void __launch_bounds__(384, 1) k_stencil_tma(const __grid_constant__ TmaMaps maps, StencilArgs<T> a,
                                                       const CoefT<T> cf, int TY, int RS, int S, int ncw,
                                                       int* __restrict__ err) {
    using VT = Vec16<T>;
    using V = typename VT::t;
    constexpr int VX = 16 / (int)sizeof(T);
    constexpr int MDX = (MD + VX - 1) / VX * VX;  // x window half-width, whole vectors
    constexpr int NV = 1 + 2 * MDX / VX;           // vectors in the x window
    constexpr int Q = 2 * MD + 1;                  // accumulator ring
    constexpr int NP = VX * BY;                    // points per thread
    extern __shared__ __align__(128) unsigned char smem[];
    const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
    const int ROWS = TY + 2 * MD;
    const int SE = (ROWS + TY) * RS;  // elements per stage: psi rows, then Vloc rows
    T* stages = reinterpret_cast<T*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * SE * sizeof(T));
    uint64_t* empty = full + S;

    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    const int nzc = a.nzc;
    const int band = blockIdx.y / nzc;
    const int zc = blockIdx.y - band * nzc;
    if (a.band_active && !a.band_active[band]) return;  // uniform per CTA
    const int y0 = blockIdx.x * TY;
    const int zs = a.z0 + zc * a.zlen;
    const int zlen = min(zs + a.zlen, a.z0 + a.nzo) - zs;
    const int nk = zlen + 2 * MD;  // arrival k <-> plane zs - Md + k
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
            const uint32_t b_in = (uint32_t)((size_t)(ROWS + TY) * RS * sizeof(T));
            const uint32_t b_out = (uint32_t)((size_t)TY * RS * sizeof(T));
            for (int k = 0; k < nk; ++k) {
                const int s = k % S;
                if (k >= S && !mbar_wait(&empty[s], ((k / S) - 1) & 1)) ok = false;
                T* dst = stages + (size_t)s * SE;
                const int zp = pwrap(zs - MD + k, n3);
                const bool inner = k >= MD && k < MD + zlen;
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&full[s], inner ? b_in : b_out);
                if (!inner) {
                    // halo planes only feed the z accumulators: the TY own rows
                    tma_load_4d(dst + MD * RS, &maps.mid, 0, y0, zp, band, &full[s]);
                    continue;
                }
                if (y0 - MD >= 0 && y0 + TY + MD <= n2) {
                    tma_load_4d(dst, &maps.full, 0, y0 - MD, zp, band, &full[s]);
                } else if (TY == n2) {
                    tma_load_4d(dst, &maps.wrap, 0, n2 - MD, zp, band, &full[s]);
                    tma_load_4d(dst + MD * RS, &maps.mid, 0, 0, zp, band, &full[s]);
                    tma_load_4d(dst + (MD + TY) * RS, &maps.wrap, 0, 0, zp, band, &full[s]);
                } else if (y0 - MD < 0) {
                    tma_load_4d(dst, &maps.wrap, 0, n2 - MD, zp, band, &full[s]);
                    tma_load_4d(dst + MD * RS, &maps.edge, 0, 0, zp, band, &full[s]);
                } else {
                    tma_load_4d(dst, &maps.edge, 0, y0 - MD, zp, band, &full[s]);
                    tma_load_4d(dst + (TY + MD) * RS, &maps.wrap, 0, 0, zp, band, &full[s]);
                }
                tma_load_4d(dst + ROWS * RS, &maps.vloc, 0, y0, zp, 0, &full[s]);
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
    const int xw = x - MDX;  // first x of the periodic window
    T* __restrict__ hb = a.hpsi + (long)band * a.ld + (long)n1 * (y0 + yl) + x;
    using P = Pk<T>;
    using PT = typename P::t;
    constexpr int W = P::W;
    constexpr int NK = NP / W;  // packs per thread, two per row

    PT acc[Q][NK];
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int i = 0; i < NK; ++i) acc[q][i] = P::splat((T)0);

    bool ok = true;
    int s = 0, u = 0;
    uint32_t ph = 0;
    for (int k = 0; k < nk; ++k) {
        if (!mbar_wait(&full[s], ph)) ok = false;
        const T* st = stages + (size_t)s * SE;
        const bool inner = k >= MD && k < MD + zlen;  // uniform
        PT c[NK], in[NK];
        if (inner) {
            const T* sp = st + yl * RS + x;
#pragma unroll
            for (int i = 0; i < NK; ++i) in[i] = P::splat((T)0);
            // y neighbours (the window also holds the thread's own rows)
#pragma unroll
            for (int j = 0; j < BY + 2 * MD; ++j) {
                PT v[2];
                P::get2(*reinterpret_cast<const V*>(sp + j * RS), v);
#pragma unroll
                for (int r = 0; r < BY; ++r) {
                    const int m = j - MD - r;
                    if (m == 0) {
                        c[2 * r] = v[0];
                        c[2 * r + 1] = v[1];
                    } else if (m >= -MD && m <= MD) {
                        const PT cy = P::splat(cf.cy[(m > 0 ? m : -m) - 1]);
#pragma unroll
                        for (int e = 0; e < 2; ++e) in[2 * r + e] = P::fma(cy, v[e], in[2 * r + e]);
                    }
                }
            }
            // x neighbours from the periodic window of each own row (its
            // centre vector is the row's own, already read with the y window)
#pragma unroll
            for (int r = 0; r < BY; ++r) {
                const T* rp = st + (MD + yl + r) * RS;
                T w[NV * VX];
#pragma unroll
                for (int j = 0; j < NV; ++j) {
                    if (j == MDX / VX) {
                        P::unpack2(c + 2 * r, w + j * VX);
                        continue;
                    }
                    int xx = xw + VX * j;
                    xx += xx < 0 ? n1 : (xx >= n1 ? -n1 : 0);
                    VT::get(*reinterpret_cast<const V*>(rp + xx), w + j * VX);
                }
#pragma unroll
                for (int e = 0; e < 2; ++e)
#pragma unroll
                    for (int m = 1; m <= MD; ++m)
                        in[2 * r + e] = P::fma(P::splat(cf.cx[m - 1]),
                                               P::add(P::of(w + MDX + W * e - m), P::of(w + MDX + W * e + m)),
                                               in[2 * r + e]);
            }
            // centre and local potential
#pragma unroll
            for (int r = 0; r < BY; ++r) {
                PT vl[2];
                P::get2(*reinterpret_cast<const V*>(sp + (ROWS + r) * RS), vl);
#pragma unroll
                for (int e = 0; e < 2; ++e)
                    in[2 * r + e] = P::fma(P::add(P::splat(cf.c0), vl[e]), c[2 * r + e], in[2 * r + e]);
            }
        } else {
#pragma unroll
            for (int r = 0; r < BY; ++r) P::get2(*reinterpret_cast<const V*>(st + (MD + yl + r) * RS + x), c + 2 * r);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with the stage
        // z pushes into the accumulator ring (slot = output arrival mod Q)
        // and, from arrival 2 Md on, the write of the completed output k - Md
        T* hp = (k >= 2 * MD && thr) ? hb + plane * (zs + k - 2 * MD) : nullptr;
        push_slot<T, MD, NK, BY>(u, acc, c, in, inner, cf, hp, n1);
        if (++s == S) {
            s = 0;
            ph ^= 1u;
        }
        if (++u == Q) u = 0;
    }
    if (!ok) atomicExch(err, 1);
}

// Nonlocal scatter after the stencil: hpsi(p, b) += sum over the sphere
// groups g covering p of sum_q uV(p, g, q) uVunk(g + q, b)
// (ps_nloc2_op_module.f90:255-263), one thread per covered point and a chunk
// of bands, SC_BU bands in flight at once (2: measured faster than 4 and 8).
// A point's entries are taken in projector order, so every sum has a fixed
// order.
constexpr int SC_BU = 2;

template <typename T>
__global__ void __launch_bounds__(128) k_nl_scatter(T* __restrict__ hpsi, long ld, int nb, int bchunk,
                                                   const int* __restrict__ nl_pts, const int* __restrict__ nl_ptr,
                                                   int npt, const int* __restrict__ gpt_grp,
                                                   const T* __restrict__ gpt_uv4, const double* __restrict__ uvunk,
                                                   int nzlma, const int* __restrict__ band_active,
                                                   int* __restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npt) return;
    const int p = nl_pts[i];
    if (!RS_DCHECK(p >= 0 && p < ld, CK_NL_SCATTER_POINT, p, err)) return;
    const int e0 = nl_ptr[i], e1 = nl_ptr[i + 1];
    const int b0 = blockIdx.y * bchunk, b1 = min(nb, b0 + bchunk);
    for (int b = b0; b < b1; b += SC_BU) {
        bool act[SC_BU];
        T o[SC_BU];
#pragma unroll
        for (int u = 0; u < SC_BU; ++u) {
            const int bb = b + u;
            act[u] = bb < b1 && (!band_active || band_active[bb]);
            o[u] = act[u] ? hpsi[(long)bb * ld + p] : (T)0;
        }
        for (int e = e0; e < e1; ++e) {
            // a group holds 1..4 projectors; missing ones have zero values
            // and must not be read past the end of uVunk
            const int g = __ldg(gpt_grp + e);
            if (!RS_DCHECK(g >= 0 && g < nzlma, CK_NL_SCATTER_GROUP, g, err)) continue;
            T uq[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) uq[q] = __ldg(gpt_uv4 + 4L * e + q);
#pragma unroll
            for (int u = 0; u < SC_BU; ++u) {
                if (!act[u]) continue;
                const double* un = uvunk + (long)(b + u) * nzlma;
                T c = uq[0] * (T)__ldg(un + g);
#pragma unroll
                for (int q = 1; q < 4; ++q)
                    if (g + q < nzlma) c += uq[q] * (T)__ldg(un + g + q);
                o[u] += c;
            }
        }
#pragma unroll
        for (int u = 0; u < SC_BU; ++u)
            if (act[u]) hpsi[(long)(b + u) * ld + p] = o[u];
    }
}

template <typename T, int MD, int TX>
static void launch_stencil_tx(const StencilArgs<T>& a, const StencilCoef& cf, int nb, cudaStream_t st) {
    dim3 grid(div_up(a.n1, TX), div_up(a.n2, 16), nb * a.nzc);
    launch(k_stencil<T, MD, TX>, grid, TX * 16, 0, st, a, cf);
}

template <typename T, int MD>
static void launch_stencil_md(const StencilArgs<T>& a, const StencilCoef& cf, int nb, cudaStream_t st) {
    if (a.n1 % 32 == 0 || a.n1 > 24)
        launch_stencil_tx<T, MD, 32>(a, cf, nb, st);
    else if (a.n1 % 24 == 0)
        launch_stencil_tx<T, MD, 24>(a, cf, nb, st);
    else
        launch_stencil_tx<T, MD, 16>(a, cf, nb, st);
}

// Geometry of k_stencil_tma: tile height TY (multiple of BY, divides n2,
// >= Md, and n2 == TY or n2 >= TY + Md), shared-memory row pitch RS (n1
// rounded up to 128 bytes; the columns past n1 arrive as zeros and are never
// read), ring depth S >= 3, consumer warps ncw, one producer warp, at most
// 384 threads (the register budget of the 2 Md + 1 accumulators).
struct TmaGeom {
    int TY = 0, RS = 0, S = 0, ncw = 0, threads = 0;
    size_t smem = 0;
};

template <typename T, int MD, int BY>
static TmaGeom tma_geometry(int n1, int n2) {
    TmaGeom best;
    constexpr int VX = 16 / (int)sizeof(T);
    constexpr int MDX = (MD + VX - 1) / VX * VX;
    const int RS = (int)((((size_t)n1 * sizeof(T) + 127) / 128) * 128 / sizeof(T));
    if (n1 % VX != 0 || n1 < MDX || RS > 256 || n2 < MD) return best;
    const size_t budget = 220 * 1024;
    double best_score = -1.0;
    for (int TY = BY; TY <= std::min(n2, 256 - 2 * MD); TY += BY) {
        if (n2 % TY != 0 || TY < MD || !(TY == n2 || n2 >= TY + MD)) continue;
        const int ncw = ((n1 / VX) * (TY / BY) + 31) / 32;
        const int threads = 32 * (ncw + 1);
        if (threads > 384) continue;
        const size_t stage = (size_t)(2 * TY + 2 * MD) * RS * sizeof(T);
        const int S = (int)std::min<size_t>(budget / (stage + 16), 8);
        if (S < 3) continue;
        // halo overhead first, then busy threads, then ring depth
        const double used = (double)((n1 / VX) * (TY / BY)) / threads;
        const double score = 100.0 * TY / (TY + 2 * MD) + 10.0 * used + 0.1 * S;
        if (score > best_score) {
            best_score = score;
            best.TY = TY;
            best.RS = RS;
            best.S = S;
            best.ncw = ncw;
            best.threads = threads;
            best.smem = (size_t)S * stage + (size_t)S * 16;
        }
    }
    return best;
}

template <typename T, int MD, int BY>
static int launch_tma(StencilArgs<T> a, const StencilCoef& cf, int nb, cudaStream_t st, bool* used) {
    Context& c = ctx();
    *used = false;
    const TmaGeom g = tma_geometry<T, MD, BY>(a.n1, a.n2);
    if (g.TY == 0) return RSDFT_OK;
    if (reinterpret_cast<uintptr_t>(a.hpsi) % 16 != 0 || (a.ld * sizeof(T)) % 16 != 0) return RSDFT_OK;
    const int sms = c.num_sms > 0 ? c.num_sms : 148;
    const long base = (long)(a.n2 / g.TY) * nb;
    int nzc = (int)std::min<long>(std::max<long>(1, (sms + base - 1) / base), std::max(1, a.nzo / (4 * MD)));
    while ((long)nb * nzc > 65535 && nzc > 1) --nzc;
    a.zlen = div_up(a.nzo, nzc);
    a.nzc = div_up(a.nzo, a.zlen);
    TmaMaps maps;
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const unsigned long long dims[4] = {(unsigned long long)a.n1, (unsigned long long)a.n2,
                                        (unsigned long long)a.n3, (unsigned long long)nb};
    const unsigned long long strides[3] = {(unsigned long long)a.n1 * sizeof(T),
                                           (unsigned long long)a.n1 * a.n2 * sizeof(T),
                                           (unsigned long long)a.ld * sizeof(T)};
    const unsigned long long vdims[4] = {(unsigned long long)a.n1, (unsigned long long)a.n2,
                                         (unsigned long long)a.n3, 1ull};
    const unsigned long long vstrides[3] = {strides[0], strides[1], (unsigned long long)a.n1 * a.n2 * a.n3 * sizeof(T)};
    const unsigned int RS = (unsigned)g.RS, TY = (unsigned)g.TY;
    const unsigned int bf[4] = {RS, TY + 2 * MD, 1, 1}, be[4] = {RS, TY + MD, 1, 1}, bm[4] = {RS, TY, 1, 1},
                       bw[4] = {RS, (unsigned)MD, 1, 1};
    if (encode_tmap_4d(&maps.full, dt, a.psi, dims, strides, bf) != RSDFT_OK ||
        encode_tmap_4d(&maps.edge, dt, a.psi, dims, strides, be) != RSDFT_OK ||
        encode_tmap_4d(&maps.mid, dt, a.psi, dims, strides, bm) != RSDFT_OK ||
        encode_tmap_4d(&maps.wrap, dt, a.psi, dims, strides, bw) != RSDFT_OK ||
        encode_tmap_4d(&maps.vloc, dt, a.vloc, vdims, vstrides, bm) != RSDFT_OK)
        return RSDFT_OK;  // not usable for this shape: the caller takes the general kernel
    RS_CHECK(set_smem_optin((const void*)k_stencil_tma<T, MD, BY>, 220 * 1024 + 8 * 16));
    dim3 grid(a.n2 / g.TY, (unsigned)(nb * a.nzc));
    launch(k_stencil_tma<T, MD, BY>, grid, g.threads, g.smem, st, maps, a, coef_as<T>(cf), g.TY, g.RS, g.S, g.ncw,
           c.err_flag);
    RS_LAUNCH();
    *used = true;
    return RSDFT_OK;
}

template <typename T, int MD>
static int launch_stencil_md2(StencilArgs<T> a, const StencilCoef& cf, int nb, cudaStream_t st) {
    const Context& c = ctx();
    bool used = false;
    // two rows per thread up to Md = 6; one above, where the 2 Md + 1
    // accumulators of two rows no longer fit the register budget
    RS_CHECK((launch_tma<T, MD, (MD <= 6 ? 2 : 1)>(a, cf, nb, st, &used)));
    if (used) {
        if (a.gpt_ptr && c.nl_npt > 0) {
            constexpr int BCH = 32;
            dim3 grid(div_up(c.nl_npt, 128), div_up(nb, BCH));
            launch(k_nl_scatter<T>, grid, 128, 0, st, a.hpsi, a.ld, nb, BCH, (const int*)c.nl_pts,
                   (const int*)c.nl_ptr, c.nl_npt, a.gpt_grp, a.gpt_uv4, a.uvunk, a.nzlma, a.band_active,
                   c.err_flag);
            RS_LAUNCH();
        }
        return RSDFT_OK;
    }
    // general shapes (odd widths, very wide rows): register-queue kernel with
    // per-plane halo loads and the nonlocal scatter fused
    const int tx = (a.n1 % 32 == 0 || a.n1 > 24) ? 32 : (a.n1 % 24 == 0 ? 24 : 16);
    const long base = (long)div_up(a.n1, tx) * div_up(a.n2, 16) * nb;
    const long want = 8L * (c.num_sms > 0 ? c.num_sms : 148);
    int nzc = (int)std::min<long>(std::max<long>(1, (want + base - 1) / base), std::max(1, a.nzo / 8));
    while ((long)nb * nzc > 65535 && nzc > 1) --nzc;
    a.zlen = div_up(a.nzo, nzc);
    a.nzc = div_up(a.nzo, a.zlen);
    launch_stencil_md<T, MD>(a, cf, nb, st);
    RS_LAUNCH();
    return RSDFT_OK;
}

template <typename T>
static int launch_stencil(StencilArgs<T> a, const StencilCoef& cf, int md, int nb, cudaStream_t st) {
    if (a.nzo <= 0) {
        a.z0 = 0;
        a.nzo = a.n3;
    }
    switch (md) {
        case 1: return launch_stencil_md2<T, 1>(a, cf, nb, st);
        case 2: return launch_stencil_md2<T, 2>(a, cf, nb, st);
        case 3: return launch_stencil_md2<T, 3>(a, cf, nb, st);
        case 4: return launch_stencil_md2<T, 4>(a, cf, nb, st);
        case 5: return launch_stencil_md2<T, 5>(a, cf, nb, st);
        case 6: return launch_stencil_md2<T, 6>(a, cf, nb, st);
        case 7: return launch_stencil_md2<T, 7>(a, cf, nb, st);
        case 8: return launch_stencil_md2<T, 8>(a, cf, nb, st);
        default: set_error("Md=%d unsupported", md); return RSDFT_EUNSUP;
    }
}

template <typename T>
int hpsi_device(const T* psi, T* hpsi, long ld, int nb, int spin, const int* band_active) {
    Context& c = ctx();
    if (nb <= 0) return RSDFT_OK;
    if (nb > 65535) {
        set_error("hpsi: nb=%d exceeds 65535", nb);
        return RSDFT_EINVAL;
    }
    if (!c.vloc || c.vloc_ml != c.ml) {
        set_error("hpsi: rsdft_gpu_set_vloc has not been called for the current grid");
        return RSDFT_ENOTINIT;
    }
    const bool nl = c.nl_set && c.nzlma > 0;
    double* uvunk = nullptr;
    if (nl) {
        RS_CHECK(workspace_t("hpsi_uvunk", (size_t)nb * c.nzlma, &uvunk));
        RS_CHECK(launch_project<T>(psi, ld, nb, uvunk, band_active, c.stream));
    }
    StencilArgs<T> a{};
    a.psi = psi;
    a.hpsi = hpsi;
    a.ld = ld;
    a.n1 = c.n1;
    a.n2 = c.n2;
    a.n3 = c.n3;
    a.vloc = (const T*)(sizeof(T) == 8 ? (const void*)(c.vloc + (long)(spin - 1) * c.ml)
                                       : (const void*)(c.vloc32 + (long)(spin - 1) * c.ml));
    a.pt_ptr = nl ? c.pt_ptr : nullptr;
    a.pt_lma = c.pt_lma;
    a.pt_uv = (const T*)(sizeof(T) == 8 ? (const void*)c.pt_uv : (const void*)c.pt_uv32);
    a.uvunk = uvunk;
    a.nzlma = c.nzlma;
    a.band_active = band_active;
    a.band_map = nullptr;
    a.gpt_ptr = nl ? c.gpt_ptr : nullptr;
    a.gpt_grp = c.gpt_grp;
    a.gpt_uv4 = (const T*)(sizeof(T) == 8 ? (const void*)c.gpt_uv4 : (const void*)c.gpt_uv4_32);
    return launch_stencil<T>(a, c.sc, c.md, nb, c.stream);
}

template int hpsi_device<double>(const double*, double*, long, int, int, const int*);
template int hpsi_device<float>(const float*, float*, long, int, int, const int*);

}  // namespace rsdft

using namespace rsdft;

extern "C" int rsdft_gpu_hamiltonian(int k, int s, const double* tpsi, double* htpsi, int n1, int n2, int ib1,
                                     int ib2) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    if (k != 1) {
        set_error("hamiltonian: k=%d, only the Gamma point (k=1) is supported", k);
        return RSDFT_EUNSUP;
    }
    if (s < 1 || s > c.nspin) {
        set_error("hamiltonian: s=%d outside 1..%d", s, c.nspin);
        return RSDFT_EINVAL;
    }
    const long ld = (long)n2 - n1 + 1;
    const int nb = ib2 - ib1 + 1;
    if (ld != c.ml || nb < 1) {
        set_error("hamiltonian: n2-n1+1=%ld must equal ML=%ld and ib2>=ib1", ld, c.ml);
        return RSDFT_EINVAL;
    }
    double *dpsi, *dh;
    bool sp, sh;
    RS_CHECK(wf_acquire(tpsi, ld, nb, "ham_in", &dpsi, &sp));
    RS_CHECK(wf_acquire(htpsi, ld, nb, "ham_out", &dh, &sh, false));
    RS_CHECK(hpsi_device<double>(dpsi, dh, ld, nb, s, nullptr));
    RS_CHECK(wf_release(htpsi, dh, ld, nb, sh));
    return RSDFT_OK;
}

// ----------------------------------------------------- the three operators
// hamiltonian applies op_kinetic, op_localpot and op_nonlocal in turn
// (hamiltonian_module.f90:42-58).  A domain-decomposed caller needs them
// apart: the kinetic + local part on a slab extended by its halo planes, and
// the nonlocal part as projection partial sums over the slab's own points,
// which the ranks add up before the scatter (ps_nloc2_op_module.f90:
// 161-250).  These entries give those pieces on the context's grid and
// projector tables.
namespace rsdft {
namespace {

int check_block(const char* who, int s, long ld, int nb) {
    Context& c = ctx();
    if (s < 1 || s > c.nspin) {
        set_error("%s: s=%d outside 1..%d", who, s, c.nspin);
        return RSDFT_EINVAL;
    }
    if (ld < c.ml || nb < 1 || nb > 65535) {
        set_error("%s: ld=%ld (ML=%ld), nb=%d", who, ld, c.ml, nb);
        return RSDFT_EINVAL;
    }
    return RSDFT_OK;
}

}  // namespace
}  // namespace rsdft

extern "C" int rsdft_gpu_op_local(int s, const double* tpsi, double* htpsi, long ld, int nb, int z0, int nz) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    RS_CHECK(check_block("op_local", s, ld, nb));
    if (z0 < 0 || nz < 1 || z0 + nz > c.n3) {
        set_error("op_local: planes [%d, %d) outside 0..%d", z0, z0 + nz, c.n3);
        return RSDFT_EINVAL;
    }
    if (!c.vloc || c.vloc_ml != c.ml) {
        set_error("op_local: rsdft_gpu_set_vloc has not been called for the current grid");
        return RSDFT_ENOTINIT;
    }
    double *dpsi, *dh;
    bool sp, sh;
    RS_CHECK(wf_acquire(tpsi, ld, nb, "ham_in", &dpsi, &sp));
    RS_CHECK(wf_acquire(htpsi, ld, nb, "ham_out", &dh, &sh, false));
    StencilArgs<double> a{};
    a.psi = dpsi;
    a.hpsi = dh;
    a.ld = ld;
    a.n1 = c.n1;
    a.n2 = c.n2;
    a.n3 = c.n3;
    a.vloc = c.vloc + (long)(s - 1) * c.ml;
    a.nzlma = c.nzlma;
    a.z0 = z0;
    a.nzo = nz;
    RS_CHECK(launch_stencil<double>(a, c.sc, c.md, nb, c.stream));
    RS_CHECK(wf_release(htpsi, dh, ld, nb, sh));
    return RSDFT_OK;
}

extern "C" int rsdft_gpu_op_nonlocal_project(const double* tpsi, long ld, int nb, double* uvunk) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    RS_CHECK(check_block("op_nonlocal_project", 1, ld, nb));
    if (!uvunk) {
        set_error("op_nonlocal_project: NULL uvunk");
        return RSDFT_EINVAL;
    }
    if (!c.nl_set || c.nzlma == 0) return RSDFT_OK;
    double* dpsi;
    bool sp;
    RS_CHECK(wf_acquire(tpsi, ld, nb, "ham_in", &dpsi, &sp));
    double* du = nullptr;
    RS_CHECK(workspace_t("op_uvunk", (size_t)c.nzlma * nb, &du));
    RS_CHECK(launch_project<double>(dpsi, ld, nb, du, nullptr, c.stream));
    RS_CHECK(stage_out(uvunk, du, sizeof(double) * (size_t)c.nzlma * nb));
    return RSDFT_OK;
}

extern "C" int rsdft_gpu_op_nonlocal_add(const double* uvunk, double* htpsi, long ld, int nb) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    RS_CHECK(check_block("op_nonlocal_add", 1, ld, nb));
    if (!uvunk) {
        set_error("op_nonlocal_add: NULL uvunk");
        return RSDFT_EINVAL;
    }
    if (!c.nl_set || c.nzlma == 0 || c.nl_npt == 0) return RSDFT_OK;
    void* du = nullptr;
    RS_CHECK(stage_in(uvunk, sizeof(double) * (size_t)c.nzlma * nb, "op_uvunk_in", &du));
    double* dh;
    bool sh;
    RS_CHECK(wf_acquire(htpsi, ld, nb, "ham_out", &dh, &sh));
    constexpr int BCH = 32;
    dim3 grid(div_up(c.nl_npt, 128), div_up(nb, BCH));
    launch(k_nl_scatter<double>, grid, 128, 0, c.stream, dh, ld, nb, BCH, (const int*)c.nl_pts, (const int*)c.nl_ptr,
           c.nl_npt, (const int*)c.gpt_grp, (const double*)c.gpt_uv4, (const double*)du, c.nzlma, (const int*)nullptr,
           c.err_flag);
    RS_LAUNCH();
    RS_CHECK(wf_release(htpsi, dh, ld, nb, sh));
    return RSDFT_OK;
}

// ------------------------------------------------- allocation-free hamiltonian
// rsdft_gpu_hamiltonian_noalloc: the same H psi, for callers that must not
// allocate device memory during the call.  Its only scratch, the projection
// coefficients uVunk(nzlma, nb), lives in the file-scope array below, which
// every GPU that loads this library holds until the process exits.  In host
// code the array's name is a host-side stand-in, not a device address, so the
// kernel is given the address cudaGetSymbolAddress returns for the bound
// device.  rsdft_gpu_init looks it up (with that device current) and the
// context keeps it, so a finalize / device reset / init sequence looks it up
// again instead of reusing an address from an earlier context.
namespace rsdft {

static __device__ __align__(256) double g_hpsi_noalloc_uvunk[RSDFT_NOALLOC_SCRATCH_VALUES];

int noalloc_bind_scratch() {
    Context& c = ctx();
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_hpsi_noalloc_uvunk);
    if (e != cudaSuccess || !p) {
        set_error("cudaGetSymbolAddress of the static hamiltonian_noalloc scratch failed on device %d: %s", c.device,
                  cudaGetErrorString(e));
        return RSDFT_ECUDA;
    }
    c.noalloc_scratch = static_cast<double*>(p);
    return RSDFT_OK;
}

namespace {

int noalloc_scratch(double** out) {
    int dev = -1;
    RS_CUDA(cudaGetDevice(&dev));
    if (dev != ctx().device) {
        set_error("hamiltonian_noalloc: current device %d is not the device %d given to rsdft_gpu_init", dev,
                  ctx().device);
        return RSDFT_EINVAL;
    }
    if (!ctx().noalloc_scratch) {
        set_error("hamiltonian_noalloc: the static scratch has no device address (rsdft_gpu_init did not bind it)");
        return RSDFT_ENOTINIT;
    }
    *out = ctx().noalloc_scratch;
    return RSDFT_OK;
}

// H psi on device-visible blocks with uVunk in the static scratch.  The
// projection kernel writes every uVunk(lma, b) of the call before the stencil
// reads it, so nothing left from an earlier call is ever read.
int hpsi_static_scratch(const double* psi, double* hpsi, long ld, int nb, int spin) {
    Context& c = ctx();
    if (!c.vloc || c.vloc_ml != c.ml) {
        set_error("hamiltonian_noalloc: rsdft_gpu_set_vloc has not been called for the current grid");
        return RSDFT_ENOTINIT;
    }
    const bool nl = c.nl_set && c.nzlma > 0;
    double* uvunk = nullptr;
    if (nl) {
        RS_CHECK(noalloc_scratch(&uvunk));
        RS_CHECK(launch_project<double>(psi, ld, nb, uvunk, nullptr, c.stream));
    }
    StencilArgs<double> a{};
    a.psi = psi;
    a.hpsi = hpsi;
    a.ld = ld;
    a.n1 = c.n1;
    a.n2 = c.n2;
    a.n3 = c.n3;
    a.vloc = c.vloc + (long)(spin - 1) * c.ml;
    a.pt_ptr = nl ? c.pt_ptr : nullptr;
    a.pt_lma = c.pt_lma;
    a.pt_uv = c.pt_uv;
    a.uvunk = uvunk;
    a.nzlma = c.nzlma;
    a.gpt_ptr = nl ? c.gpt_ptr : nullptr;
    a.gpt_grp = c.gpt_grp;
    a.gpt_uv4 = c.gpt_uv4;
    return launch_stencil<double>(a, c.sc, c.md, nb, c.stream);
}

}  // namespace
}  // namespace rsdft

extern "C" int rsdft_gpu_hamiltonian_noalloc(int k, int s, const double* tpsi, double* htpsi, int n1, int n2,
                                             int ib1, int ib2) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    if (k != 1) {
        set_error("hamiltonian_noalloc: k=%d, only the Gamma point (k=1) is supported", k);
        return RSDFT_EUNSUP;
    }
    if (s < 1 || s > c.nspin) {
        set_error("hamiltonian_noalloc: s=%d outside 1..%d", s, c.nspin);
        return RSDFT_EINVAL;
    }
    const long ld = (long)n2 - n1 + 1;
    const int nb = ib2 - ib1 + 1;
    if (ld != c.ml || nb < 1 || nb > 65535) {
        set_error("hamiltonian_noalloc: n2-n1+1=%ld must equal ML=%ld and 1 <= ib2-ib1+1 <= 65535", ld, c.ml);
        return RSDFT_EINVAL;
    }
    if (c.nl_set && (long)nb * c.nzlma > RSDFT_NOALLOC_SCRATCH_VALUES) {
        set_error("hamiltonian_noalloc: %d bands x %d projectors = %ld scratch values exceed the static maximum "
                  "%ld (%ld MiB); call it on at most %ld bands at a time",
                  nb, c.nzlma, (long)nb * c.nzlma, (long)RSDFT_NOALLOC_SCRATCH_VALUES,
                  (long)RSDFT_NOALLOC_SCRATCH_VALUES * 8 / (1 << 20), (long)RSDFT_NOALLOC_SCRATCH_VALUES / c.nzlma);
        return RSDFT_EINVAL;
    }
    void *dpsi = nullptr, *dh = nullptr;
    const size_t span = sizeof(double) * (size_t)ld * (size_t)nb;
    const int rp = resolve(tpsi, span, &dpsi);
    if (rp < 0) return rp;
    const int rh = resolve(htpsi, span, &dh);
    if (rh < 0) return rh;
    if (!rp || !rh) {
        set_error("hamiltonian_noalloc: tpsi and htpsi must be device memory or lie in a registered wavefunction "
                  "(this entry point stages nothing)");
        return RSDFT_EINVAL;
    }
    return hpsi_static_scratch(static_cast<const double*>(dpsi), static_cast<double*>(dh), ld, nb, s);
}
