// hpsi on sm_100a: H psi = T psi + Vloc psi + V_nl psi for a batch of bands.
//
// Two kernels per call:
//  1. k_nl_project: uVunk(lma, b) = iuV dV sum_j uV(j) psi(JJP(j), b)
//     (ps_nloc2_op_module.f90:161-175).  One warp per band, lanes stride the
//     sphere's point list, the projectors of one sphere (same point list)
//     share each gathered psi value; fixed-order shuffle-tree reduction.
//  2. k_stencil: the Md-order periodic FD Laplacian (kinetic_sol_module.f90:
//     72-77, 129-149) fused with the Vloc multiply (localpot_module.f90:73)
//     and the nonlocal scatter-add (ps_nloc2_op_module.f90:255-263), the
//     scatter turned into a per-point gather over a point-major CSR so the
//     sum is deterministic.  2.5-D blocking: a CTA owns a TX x 16 column tile
//     of one band and marches along z; each thread keeps its column's
//     2*Md+1 z values in a register queue, the x/y neighbours of the current
//     plane come from a shared-memory tile with an Md-wide periodic halo.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"
#include "tma.cuh"
#include "tmap.cuh"

namespace rsdft {

__device__ __forceinline__ int pwrap(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// ------------------------------------------------------------ projection
template <typename T>
__global__ void __launch_bounds__(256) k_nl_project(const T* __restrict__ psi, long ld, int nb,
                                                    const int* __restrict__ grp_lma0,
                                                    const int* __restrict__ grp_cnt,
                                                    const int* __restrict__ lma_ptr,
                                                    const int* __restrict__ jjp,
                                                    const double* __restrict__ uv,
                                                    const int* __restrict__ iuv, double dV,
                                                    double* __restrict__ uvunk, int nzlma,
                                                    const int* __restrict__ band_active) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.y * 8 + warp;
    if (b >= nb) return;
    if (band_active && !band_active[b]) return;
    const int g = blockIdx.x;
    const int l0 = grp_lma0[g], cnt = grp_cnt[g];
    const int js = lma_ptr[l0], n = lma_ptr[l0 + 1] - js;
    const T* p = psi + (long)b * ld;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    int off[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) off[q] = q < cnt ? lma_ptr[l0 + q] : js;
    for (int j = lane; j < n; j += 32) {
        const double v = (double)__ldg(p + jjp[js + j]);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (q < cnt) acc[q] = fma(__ldg(uv + off[q] + j), v, acc[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], s);
    }
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (q < cnt) uvunk[(long)b * nzlma + l0 + q] = iuv[l0 + q] * dV * acc[q];
    }
}

// -------------------------------------------------------------- stencil
template <typename T>
struct StencilArgs {
    const T* psi;
    T* hpsi;
    long ld;
    int n1, n2, n3;
    int zlen, nzc;
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
    const int zs = zc * a.zlen;
    const int ze = min(zs + a.zlen, n3);
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

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
    using t = double2;
};
template <>
struct Vec2<float> {
    using t = float2;
};

// Shared-memory padding (elements) on each side of a row: >= the even
// rounding of Md, and a multiple of 16 bytes so bulk copies land aligned.
template <typename T, int MD>
__host__ __device__ constexpr int ring_pad() {
    return sizeof(T) == 8 ? ((MD + 1) / 2) * 2 : ((MD + 3) / 4) * 4;
}

struct WsMaps {
    CUtensorMap full, edge, mid, wrap;  // box heights ROWS, ROWS - Md, TY, Md
};

// hpsi stencil, warp-specialized TMA pipeline.  A CTA owns TY full-width
// rows (all n1 x) of one band and marches along z.
//  * TMA warp: one 4-D tensor-map TMA per plane tile (TY + 2 Md rows, x from
//    -PAD to n1 + PAD, the out-of-range pad columns arrive as zeros; periodic
//    wrap in y by splitting the box at the boundary) into a ring of S
//    shared-memory stages (full[] barriers); it reuses a stage once every
//    consumer warp has released it (empty[]).
//  * Pad warp: fills the periodic x pads of each landed tile and publishes
//    it (ready[] barriers).
//  * Consumer warps: each thread owns 2 (x) x BY (y) points; x neighbours from
//    a register window of its rows, y neighbours from one 2-wide load per row
//    of the y window, z neighbours from a register queue of 2 Md + 1 planes
//    whose head is read from the stage Md planes ahead.  Epilogue: Vloc,
//    nonlocal scatter (sphere-group CSR, uVunk column in shared memory).
//  No CTA-wide barrier inside the z loop: warps drift, so one warp's memory
//  latency overlaps other warps' arithmetic.
template <typename T, int MD, int BY, int UNR>
__global__ void __launch_bounds__(384, 1) k_stencil_ws(const __grid_constant__ WsMaps maps, StencilArgs<T> a,
                                                      StencilCoef cf, int TY, int S, int ncw, int* __restrict__ err) {
    using T2 = typename Vec2<T>::t;
    constexpr int PAD = ring_pad<T, MD>();
    constexpr int MD2 = ((MD + 1) / 2) * 2;  // even window half-width
    constexpr int NW = 2 * MD2 + 2;           // x window per row (elements)
    extern __shared__ __align__(128) unsigned char smem[];
    const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
    constexpr int RQ = 128 / (int)sizeof(T);      // row stride quantum: rows start on 128-byte boundaries
    const int RS = (n1 + 2 * PAD + RQ - 1) / RQ * RQ;
    const int ROWS = TY + 2 * MD;
    const int SE = ROWS * RS;
    T* stages = reinterpret_cast<T*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * SE * sizeof(T));
    uint64_t* ready = full + S;
    uint64_t* empty = ready + S;
    double* s_un = reinterpret_cast<double*>(empty + S);

    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    const int nzc = a.nzc;
    const int band = blockIdx.y / nzc;
    const int zc = blockIdx.y - band * nzc;
    if (a.band_active && !a.band_active[band]) return;  // uniform per CTA
    const int y0 = blockIdx.x * TY;
    const int zs = zc * a.zlen;
    const int ze = min(zs + a.zlen, n3);
    const int zlen = ze - zs;
    const long plane = (long)n1 * n2;
    const int nload = zlen + MD;  // ring index k <-> plane zs + k

    if (t == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&ready[s], 1);
            mbar_init(&empty[s], ncw);
        }
        mbar_fence_init();
    }
    if (a.gpt_ptr)
        for (int i = t; i < a.nzlma; i += blockDim.x) s_un[i] = a.uvunk[(long)band * a.nzlma + i];
    __syncthreads();

    if (warp == ncw) {
        // ------------------------------------------------- producer: TMA
        const uint32_t bytes = (uint32_t)(SE * sizeof(T));
        bool ok = true;
        for (int k = 0; k < nload; ++k) {
            const int slot = k % S;
            if (k >= S && !mbar_wait(&empty[slot], ((k / S) - 1) & 1)) ok = false;
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) {
                T* dst = stages + (size_t)slot * SE;
                const int zp = pwrap(zs + k, n3);
                mbar_arrive_expect_tx(&full[slot], bytes);
                if (y0 - MD >= 0 && y0 + TY + MD <= n2) {
                    tma_load_4d(dst, &maps.full, -PAD, y0 - MD, zp, band, &full[slot]);
                } else if (TY == n2) {
                    tma_load_4d(dst, &maps.wrap, -PAD, n2 - MD, zp, band, &full[slot]);
                    tma_load_4d(dst + MD * RS, &maps.mid, -PAD, 0, zp, band, &full[slot]);
                    tma_load_4d(dst + (MD + TY) * RS, &maps.wrap, -PAD, 0, zp, band, &full[slot]);
                } else if (y0 - MD < 0) {
                    tma_load_4d(dst, &maps.wrap, -PAD, n2 - MD, zp, band, &full[slot]);
                    tma_load_4d(dst + MD * RS, &maps.edge, -PAD, 0, zp, band, &full[slot]);
                } else {
                    tma_load_4d(dst, &maps.edge, -PAD, y0 - MD, zp, band, &full[slot]);
                    tma_load_4d(dst + (TY + MD) * RS, &maps.wrap, -PAD, 0, zp, band, &full[slot]);
                }
            }
        }
        if (!ok && lane == 0) atomicExch(err, 1);
        return;
    }
    if (warp == ncw + 1) {
        // ------------------------------------------ producer: periodic pads
        // left pad x = -PAD..-1 <- x = n1-PAD..n1-1, right pad x = n1..n1+PAD-1
        // <- x = 0..PAD-1; both are PAD contiguous elements, copied as pairs
        bool ok = true;
        constexpr int H = PAD / 2;  // pairs per pad
        for (int kp = 0; kp < nload; ++kp) {
            const int slot = kp % S;
            if (!mbar_wait(&full[slot], (kp / S) & 1)) ok = false;
            T* st = stages + (size_t)slot * SE;
            for (int c = lane; c < ROWS * 2 * H; c += 32) {
                const int r = c / (2 * H), i = c - r * (2 * H);
                T* row = st + r * RS;
                if (i < H)
                    *reinterpret_cast<T2*>(row + 2 * i) = *reinterpret_cast<const T2*>(row + n1 + 2 * i);
                else
                    *reinterpret_cast<T2*>(row + n1 + PAD + 2 * (i - H)) =
                        *reinterpret_cast<const T2*>(row + PAD + 2 * (i - H));
            }
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&ready[slot]);
        }
        if (!ok && lane == 0) atomicExch(err, 1);
        return;
    }

    // ---------------------------------------------------------- consumers
    const int nxp = n1 >> 1;
    const int ncons = nxp * (TY / BY);
    const bool thr = t < ncons;
    const int px = thr ? t % nxp : 0, py = thr ? t / nxp : 0;
    const int x = 2 * px, yl = BY * py;
    const T* __restrict__ p = a.psi + (long)band * a.ld;
    T* __restrict__ h = a.hpsi + (long)band * a.ld;
    bool rowok[BY];
#pragma unroll
    for (int r = 0; r < BY; ++r) rowok[r] = thr && (y0 + yl + r < n2);

    // z queue: q[k][2r + c] = psi(x + c, y0 + yl + r, z - MD + k); UNR - 1
    // extra slots so the loop can run UNR planes before shifting
    T q[2 * MD + UNR][2 * BY];
#pragma unroll
    for (int k = 0; k < 2 * MD; ++k) {
        const T* pz = p + plane * pwrap(zs - MD + k, n3);
#pragma unroll
        for (int r = 0; r < BY; ++r) {
            T2 v = {0, 0};
            if (rowok[r]) v = __ldg(reinterpret_cast<const T2*>(pz + (long)n1 * (y0 + yl + r) + x));
            q[k][2 * r] = v.x;
            q[k][2 * r + 1] = v.y;
        }
    }
    bool ok = true;
    for (int kz0 = 0; kz0 < zlen; kz0 += UNR) {
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int kz = kz0 + u;
            if (kz >= zlen) break;  // uniform
            const int z = zs + kz;
            const int kh = kz + MD;
            // epilogue operands, issued early so their latency overlaps the stencil
            T2 vl[BY];
            int sp[BY][3];
#pragma unroll
            for (int r = 0; r < BY; ++r) {
                const long j = (long)x + (long)n1 * (y0 + yl + r) + plane * z;
                vl[r].x = 0;
                vl[r].y = 0;
                sp[r][0] = sp[r][1] = sp[r][2] = 0;
                if (rowok[r]) {
                    vl[r] = __ldg(reinterpret_cast<const T2*>(a.vloc + j));
                    if (a.gpt_ptr) {
                        sp[r][0] = __ldg(a.gpt_ptr + j);
                        sp[r][1] = __ldg(a.gpt_ptr + j + 1);
                        sp[r][2] = __ldg(a.gpt_ptr + j + 2);
                    }
                }
            }
            if (!mbar_wait(&ready[kh % S], (kh / S) & 1)) ok = false;
            {
                const T* sh = stages + (size_t)(kh % S) * SE + PAD + x;
#pragma unroll
                for (int r = 0; r < BY; ++r) {
                    const T2 v = *reinterpret_cast<const T2*>(sh + (MD + yl + r) * RS);
                    q[2 * MD + u][2 * r] = v.x;
                    q[2 * MD + u][2 * r + 1] = v.y;
                }
            }
            if (kz < MD && !mbar_wait(&ready[kz % S], (kz / S) & 1)) ok = false;
            const T* st = stages + (size_t)(kz % S) * SE + PAD + x;
            T acc[2 * BY];
#pragma unroll
            for (int i = 0; i < 2 * BY; ++i) acc[i] = (T)cf.c0 * q[MD + u][i];
#pragma unroll
            for (int r = 0; r < BY; ++r) {
                T w[NW];
                const T* rp = st + (MD + yl + r) * RS - MD2;
#pragma unroll
                for (int k = 0; k < NW / 2; ++k) {
                    const T2 v = *reinterpret_cast<const T2*>(rp + 2 * k);
                    w[2 * k] = v.x;
                    w[2 * k + 1] = v.y;
                }
#pragma unroll
                for (int m = 1; m <= MD; ++m) {
                    acc[2 * r] += (T)cf.cx[m - 1] * (w[MD2 - m] + w[MD2 + m]);
                    acc[2 * r + 1] += (T)cf.cx[m - 1] * (w[MD2 + 1 - m] + w[MD2 + 1 + m]);
                }
            }
#pragma unroll
            for (int j = 0; j < BY + 2 * MD; ++j) {
                const T2 v = *reinterpret_cast<const T2*>(st + (yl + j) * RS);
#pragma unroll
                for (int r = 0; r < BY; ++r) {
                    const int m = j - MD - r;
                    if (m != 0 && m >= -MD && m <= MD) {
                        const T c = (T)cf.cy[(m > 0 ? m : -m) - 1];
                        acc[2 * r] += c * v.x;
                        acc[2 * r + 1] += c * v.y;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[kz % S]);  // this warp is done with the stage
#pragma unroll
            for (int m = 1; m <= MD; ++m) {
#pragma unroll
                for (int i = 0; i < 2 * BY; ++i)
                    acc[i] += (T)cf.cz[m - 1] * (q[MD + u - m][i] + q[MD + u + m][i]);
            }
#pragma unroll
            for (int r = 0; r < BY; ++r) {
                if (!rowok[r]) continue;
                const long j = (long)x + (long)n1 * (y0 + yl + r) + plane * z;
                T o0 = acc[2 * r] + vl[r].x * q[MD + u][2 * r];
                T o1 = acc[2 * r + 1] + vl[r].y * q[MD + u][2 * r + 1];
                if (a.gpt_ptr) {
                    for (int e = sp[r][0]; e < sp[r][2]; ++e) {
                        const int g = __ldg(a.gpt_grp + e);
                        const T2 u01 = __ldg(reinterpret_cast<const T2*>(a.gpt_uv4 + 4L * e));
                        const T2 u23 = __ldg(reinterpret_cast<const T2*>(a.gpt_uv4 + 4L * e + 2));
                        const T c = u01.x * (T)s_un[g] + u01.y * (T)s_un[g + 1] + u23.x * (T)s_un[g + 2] +
                                    u23.y * (T)s_un[g + 3];
                        if (e < sp[r][1])
                            o0 += c;
                        else
                            o1 += c;
                    }
                }
                T2 o;
                o.x = o0;
                o.y = o1;
                *reinterpret_cast<T2*>(h + j) = o;
            }
        }
#pragma unroll
        for (int k = 0; k < 2 * MD; ++k)
#pragma unroll
            for (int i = 0; i < 2 * BY; ++i) q[k][i] = q[k + UNR][i];
    }
    if (!ok) atomicExch(err, 1);
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

// Warp-specialized kernel geometry: tile height TY (multiple of BY, divides
// n2, >= Md, and n2 == TY or n2 >= TY + Md), ring depth S >= Md + 3,
// consumer threads (n1/2)(TY/BY) rounded up to warps, plus two producer warps
// (TMA, pads), at most 384 threads.
struct RingGeom {
    int TY = 0, S = 0, threads = 0, ncw = 0;
    size_t smem = 0;
};

template <typename T, int MD, int BY>
static RingGeom ring_geometry(int n1, int n2, int zlen, int nzlma) {
    RingGeom best;
    constexpr int PAD = ring_pad<T, MD>();
    constexpr int RQ = 128 / (int)sizeof(T);
    const int RS = (n1 + 2 * PAD + RQ - 1) / RQ * RQ;
    if (n1 % (16 / (int)sizeof(T)) != 0 || n1 < PAD || RS > 256 || n2 < MD) return best;
    const size_t budget = 220 * 1024 - (size_t)nzlma * 8;
    int best_score = -1;
    for (int TY = BY; TY <= std::min(n2, 96); TY += BY) {
        if (n2 % TY != 0 || TY < MD || !(TY == n2 || n2 >= TY + MD) || TY + 2 * MD > 256) continue;
        const int ncons = (n1 / 2) * (TY / BY);
        const int ncw = (ncons + 31) / 32;
        const int threads = 32 * (ncw + 2);
        if (threads > 384) continue;
        const size_t stage = (size_t)(TY + 2 * MD) * RS * sizeof(T);
        int S = (int)std::min<size_t>(budget / (stage + 24), 16);
        S = std::min(S, std::max(zlen + MD, MD + 3));
        if (S < MD + 3) continue;
        const int score = (int)(1000.0 * TY / (TY + 2 * MD)) * 100 + S;
        if (score > best_score) {
            best_score = score;
            best.TY = TY;
            best.S = S;
            best.threads = threads;
            best.ncw = ncw;
            best.smem = (size_t)S * stage + (size_t)S * 24 + (size_t)nzlma * 8;
        }
    }
    return best;
}

template <typename T, int MD, int BY>
static int launch_ring(StencilArgs<T> a, const StencilCoef& cf, int nb, cudaStream_t st, bool* used) {
    Context& c = ctx();
    *used = false;
    const int sms = c.num_sms > 0 ? c.num_sms : 148;
    RingGeom g0 = ring_geometry<T, MD, BY>(a.n1, a.n2, a.n3, a.nzlma);
    if (g0.TY == 0) return RSDFT_OK;
    const long base = (long)(a.n2 / g0.TY) * nb;
    int nzc = (int)std::min<long>(std::max<long>(1, (2L * sms + base - 1) / base), std::max(1, a.n3 / 8));
    while ((long)nb * nzc > 65535 && nzc > 1) --nzc;
    a.zlen = div_up(a.n3, nzc);
    a.nzc = div_up(a.n3, a.zlen);
    RingGeom g = ring_geometry<T, MD, BY>(a.n1, a.n2, a.zlen, a.nzlma);
    if (g.TY == 0) return RSDFT_OK;
    constexpr int PAD = ring_pad<T, MD>();
    constexpr int RQ = 128 / (int)sizeof(T);
    WsMaps maps;
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const unsigned long long dims[4] = {(unsigned long long)a.n1, (unsigned long long)a.n2,
                                        (unsigned long long)a.n3, (unsigned long long)nb};
    const unsigned long long strides[3] = {(unsigned long long)a.n1 * sizeof(T),
                                           (unsigned long long)a.n1 * a.n2 * sizeof(T),
                                           (unsigned long long)a.ld * sizeof(T)};
    const unsigned int RS = (a.n1 + 2 * PAD + RQ - 1) / RQ * RQ, ROWS = g.TY + 2 * MD;
    const unsigned int bf[4] = {RS, ROWS, 1, 1}, be[4] = {RS, ROWS - MD, 1, 1}, bm[4] = {RS, (unsigned)g.TY, 1, 1},
                       bw[4] = {RS, (unsigned)MD, 1, 1};
    if (encode_tmap_4d(&maps.full, dt, a.psi, dims, strides, bf) != RSDFT_OK ||
        encode_tmap_4d(&maps.edge, dt, a.psi, dims, strides, be) != RSDFT_OK ||
        encode_tmap_4d(&maps.mid, dt, a.psi, dims, strides, bm) != RSDFT_OK ||
        encode_tmap_4d(&maps.wrap, dt, a.psi, dims, strides, bw) != RSDFT_OK)
        return RSDFT_OK;  // not usable for this shape: the caller takes the general kernel
    static bool attr_set = false;
    if (!attr_set) {
        RS_CUDA(cudaFuncSetAttribute(k_stencil_ws<T, MD, BY, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     220 * 1024 + 16 * 24));
        attr_set = true;
    }
    dim3 grid(a.n2 / g.TY, (unsigned)(nb * a.nzc));
    launch(k_stencil_ws<T, MD, BY, 1>, grid, g.threads, g.smem, st, maps, a, cf, g.TY, g.S, g.ncw, c.err_flag);
    RS_LAUNCH();
    *used = true;
    return RSDFT_OK;
}

template <typename T, int MD>
static int launch_stencil_md2(StencilArgs<T> a, const StencilCoef& cf, int nb, cudaStream_t st) {
    bool used = false;
    if ((long)nb * 2 <= 65535) {
        if constexpr (sizeof(T) == 8)
            RS_CHECK((launch_ring<T, MD, 2>(a, cf, nb, st, &used)));
        else
            RS_CHECK((launch_ring<T, MD, 4>(a, cf, nb, st, &used)));
    }
    if (used) return RSDFT_OK;
    // general shapes (odd widths, very wide rows): register-queue kernel with
    // per-plane halo loads
    const Context& c = ctx();
    const int tx = (a.n1 % 32 == 0 || a.n1 > 24) ? 32 : (a.n1 % 24 == 0 ? 24 : 16);
    const long base = (long)div_up(a.n1, tx) * div_up(a.n2, 16) * nb;
    const long want = 8L * (c.num_sms > 0 ? c.num_sms : 148);
    int nzc = (int)std::min<long>(std::max<long>(1, (want + base - 1) / base), std::max(1, a.n3 / 8));
    while ((long)nb * nzc > 65535 && nzc > 1) --nzc;
    a.zlen = div_up(a.n3, nzc);
    a.nzc = div_up(a.n3, a.zlen);
    launch_stencil_md<T, MD>(a, cf, nb, st);
    RS_LAUNCH();
    return RSDFT_OK;
}

template <typename T>
static int launch_stencil(StencilArgs<T> a, const StencilCoef& cf, int md, int nb, cudaStream_t st) {
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
    if (!c.vloc) {
        set_error("hpsi: rsdft_gpu_set_vloc has not been called");
        return RSDFT_ENOTINIT;
    }
    const bool nl = c.nl_set && c.nzlma > 0;
    double* uvunk = nullptr;
    if (nl) {
        RS_CHECK(workspace_t("hpsi_uvunk", (size_t)nb * c.nzlma, &uvunk));
        dim3 grid(c.ngroup, div_up(nb, 8));
        launch(k_nl_project<T>, grid, 256, 0, c.stream, psi, ld, nb, c.grp_lma0, c.grp_cnt, c.lma_ptr, c.jjp, c.uv,
                                                    c.iuv, c.dV, uvunk, c.nzlma, band_active);
        RS_LAUNCH();
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

// ------------------------------------------------- allocation-free hamiltonian
// rsdft_gpu_hamiltonian_noalloc: the same H psi, for callers that must not
// allocate device memory during the call.  Its only scratch, the projection
// coefficients uVunk(nzlma, nb), lives in the file-scope array below, which
// every GPU that loads this library holds until the process exits.  In host
// code the array's name is a host-side stand-in, not a device address, so the
// kernel is given the address cudaGetSymbolAddress returns for the current
// device (looked up on the first call on each device).
namespace rsdft {
namespace {

static __device__ __align__(256) double g_hpsi_noalloc_uvunk[RSDFT_NOALLOC_SCRATCH_VALUES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_addr[kMaxDevices] = {};

int noalloc_scratch(double** out) {
    int dev = -1;
    RS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("hamiltonian_noalloc: device ordinal %d outside 0..%d", dev, kMaxDevices - 1);
        return RSDFT_EUNSUP;
    }
    if (dev != ctx().device) {
        set_error("hamiltonian_noalloc: current device %d is not the device %d given to rsdft_gpu_init", dev,
                  ctx().device);
        return RSDFT_EINVAL;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_hpsi_noalloc_uvunk);
        if (e != cudaSuccess || !p) {
            set_error("hamiltonian_noalloc: cudaGetSymbolAddress of the static scratch failed on device %d: %s", dev,
                      cudaGetErrorString(e));
            return RSDFT_ECUDA;
        }
        g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[dev];
    return RSDFT_OK;
}

// H psi on device-visible blocks with uVunk in the static scratch.  The
// projection kernel writes every uVunk(lma, b) of the call before the stencil
// reads it, so nothing left from an earlier call is ever read.
int hpsi_static_scratch(const double* psi, double* hpsi, long ld, int nb, int spin) {
    Context& c = ctx();
    if (!c.vloc) {
        set_error("hamiltonian_noalloc: rsdft_gpu_set_vloc has not been called");
        return RSDFT_ENOTINIT;
    }
    const bool nl = c.nl_set && c.nzlma > 0;
    double* uvunk = nullptr;
    if (nl) {
        RS_CHECK(noalloc_scratch(&uvunk));
        launch(k_nl_project<double>, dim3(c.ngroup, div_up(nb, 8)), 256, 0, c.stream, psi, ld, nb, c.grp_lma0,
               c.grp_cnt, c.lma_ptr, c.jjp, c.uv, c.iuv, c.dV, uvunk, c.nzlma, (const int*)nullptr);
        RS_LAUNCH();
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
    if (!resolve(tpsi, &dpsi) || !resolve(htpsi, &dh)) {
        set_error("hamiltonian_noalloc: tpsi and htpsi must be device memory or lie in a registered wavefunction "
                  "(this entry point stages nothing)");
        return RSDFT_EINVAL;
    }
    return hpsi_static_scratch(static_cast<const double*>(dpsi), static_cast<double*>(dh), ld, nb, s);
}
