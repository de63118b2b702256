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
#include "common.cuh"
#include "kernels.cuh"

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

template <typename T>
static int launch_stencil(StencilArgs<T> a, const StencilCoef& cf, int md, int nb, cudaStream_t st) {
    const Context& c = ctx();
    // z chunking: enough CTAs to fill the GPU, chunks of at least 8 planes
    const int tx = (a.n1 % 32 == 0 || a.n1 > 24) ? 32 : (a.n1 % 24 == 0 ? 24 : 16);
    const long base = (long)div_up(a.n1, tx) * div_up(a.n2, 16) * nb;
    const long want = 8L * (c.num_sms > 0 ? c.num_sms : 148);
    int nzc = (int)std::min<long>(std::max<long>(1, (want + base - 1) / base), std::max(1, a.n3 / 8));
    while ((long)nb * nzc > 65535 && nzc > 1) --nzc;
    a.zlen = div_up(a.n3, nzc);
    a.nzc = div_up(a.n3, a.zlen);
    switch (md) {
        case 1: launch_stencil_md<T, 1>(a, cf, nb, st); break;
        case 2: launch_stencil_md<T, 2>(a, cf, nb, st); break;
        case 3: launch_stencil_md<T, 3>(a, cf, nb, st); break;
        case 4: launch_stencil_md<T, 4>(a, cf, nb, st); break;
        case 5: launch_stencil_md<T, 5>(a, cf, nb, st); break;
        case 6: launch_stencil_md<T, 6>(a, cf, nb, st); break;
        case 7: launch_stencil_md<T, 7>(a, cf, nb, st); break;
        case 8: launch_stencil_md<T, 8>(a, cf, nb, st); break;
        default: set_error("Md=%d unsupported", md); return RSDFT_EUNSUP;
    }
    RS_LAUNCH();
    return RSDFT_OK;
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
