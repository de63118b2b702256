// Nonlocal force and the adjoint of hpsi.
//
// Force (calc_force_ps_nloc2, ps_nloc2_module.f90:1601-1654, :1760-1773):
//   w0 = iuV (-2 occ_n dV^2) sum_j uV(j) psi_n(JJP(j))
//   wk = sum_j duVdR_k(j) psi_n(JJP(j))
//   F(k, a) += w0 wk   over bands n with occ_n != 0 and projectors lma in a.
// Adjoint of y = H psi for a cotangent chi (the vector-Jacobian product):
//   dL/dV(r)  = sum_n chi_n(r) psi_n(r)                 (op_localpot)
//   dL/dR_ak  = sum_n sum_{lma in a} iuV dV [(chi.dk uV)(uV.psi) + (chi.uV)(dk uV.psi)]
// With chi_n = occ_n dV psi_n the second line is dE/dR = -F.
//
// k_nl_grad gathers psi (and chi) once per sphere for the 4 projector
// contractions of every projector in the sphere group (one warp per band),
// reduces with a fixed shuffle tree and accumulates the band sum of each
// projector in a fixed order (CTA loops over its bands), then k_atom_sum adds
// the projectors of each atom in order: bit-reproducible.
#include "common.cuh"
#include "kernels.cuh"

namespace rsdft {

constexpr int FW = 8;  // warps per CTA

// per projector: out[lma*3 + k] = sum over bands of the contribution
template <bool CHI>
__global__ void __launch_bounds__(FW * 32) k_nl_grad(const double* __restrict__ psi, const double* __restrict__ chi,
                                                     long ld, int nb, const double* __restrict__ occ, double cscale,
                                                     const int* __restrict__ grp_lma0, const int* __restrict__ grp_cnt,
                                                     const int* __restrict__ lma_ptr, const int* __restrict__ jjp,
                                                     const double* __restrict__ uv, const double* __restrict__ duv,
                                                     const int* __restrict__ iuv, double dV,
                                                     double* __restrict__ out, int* __restrict__ err) {
    __shared__ double sh[FW][4][3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = blockIdx.x;
    const int l0 = grp_lma0[g], cnt = grp_cnt[g];
    const int js = lma_ptr[l0], n = lma_ptr[l0 + 1] - js;
    int off[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) off[q] = q < cnt ? lma_ptr[l0 + q] : js;
    double tot[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int k = 0; k < 3; ++k) tot[q][k] = 0.0;
    for (int b = warp; b < nb; b += FW) {
        const double o = occ ? occ[b] : 1.0;
        if (!CHI && o == 0.0) continue;
        const double* p = psi + (long)b * ld;
        const double* x = CHI ? chi + (long)b * ld : nullptr;
        // per projector: t = uV.psi, d_k = duV_k.psi (and the chi versions)
        double t[4], d[4][3], tc[4], dc[4][3];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            t[q] = 0.0;
            tc[q] = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) d[q][k] = dc[q][k] = 0.0;
        }
        for (int j = lane; j < n; j += 32) {
            const int jj = jjp[js + j];
            if (!RS_DCHECK(jj >= 0 && jj < ld, CK_NL_GRAD_POINT, jj, err)) continue;
            const double v = __ldg(p + jj);
            const double xv = CHI ? __ldg(x + jj) : 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (q < cnt) {
                    const long e = off[q] + j;
                    const double u = __ldg(uv + e);
                    const double d0 = __ldg(duv + 3 * e), d1 = __ldg(duv + 3 * e + 1), d2 = __ldg(duv + 3 * e + 2);
                    t[q] = fma(u, v, t[q]);
                    d[q][0] = fma(d0, v, d[q][0]);
                    d[q][1] = fma(d1, v, d[q][1]);
                    d[q][2] = fma(d2, v, d[q][2]);
                    if (CHI) {
                        tc[q] = fma(u, xv, tc[q]);
                        dc[q][0] = fma(d0, xv, dc[q][0]);
                        dc[q][1] = fma(d1, xv, dc[q][1]);
                        dc[q][2] = fma(d2, xv, dc[q][2]);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                t[q] += __shfl_xor_sync(0xffffffffu, t[q], s);
#pragma unroll
                for (int k = 0; k < 3; ++k) d[q][k] += __shfl_xor_sync(0xffffffffu, d[q][k], s);
                if (CHI) {
                    tc[q] += __shfl_xor_sync(0xffffffffu, tc[q], s);
#pragma unroll
                    for (int k = 0; k < 3; ++k) dc[q][k] += __shfl_xor_sync(0xffffffffu, dc[q][k], s);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q < cnt) {
                const double w = iuv[l0 + q] * dV;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    if (CHI)
                        tot[q][k] += w * (dc[q][k] * t[q] + tc[q] * d[q][k]);
                    else
                        tot[q][k] += cscale * o * w * t[q] * d[q][k];
                }
            }
        }
    }
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int k = 0; k < 3; ++k) sh[warp][q][k] = tot[q][k];
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        const int q = threadIdx.x / 3, k = threadIdx.x % 3;
        if (q < cnt) {
            double s = 0.0;
            for (int w = 0; w < FW; ++w) s += sh[w][q][k];
            out[(long)(l0 + q) * 3 + k] = s;
        }
    }
}

__global__ void k_atom_sum(const double* __restrict__ per_lma, const int* __restrict__ atom_ptr,
                           const int* __restrict__ atom_lma, int natom, double* __restrict__ f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= natom * 3) return;
    int a = i / 3, k = i % 3;
    double s = 0.0;
    for (int e = atom_ptr[a]; e < atom_ptr[a + 1]; ++e) s += per_lma[(long)atom_lma[e] * 3 + k];
    f[i] = s;
}

// dL/dV(r) = sum_n chi_n(r) psi_n(r), chi_n = occ_n dV psi_n when chi == NULL
__global__ void k_vloc_adjoint(const double* __restrict__ psi, const double* __restrict__ chi, long ld, int nb,
                               const double* __restrict__ occ, double dV, long n, double* __restrict__ out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    if (chi) {
        for (int b = 0; b < nb; ++b) s = fma(__ldg(chi + (long)b * ld + i), __ldg(psi + (long)b * ld + i), s);
    } else {
        for (int b = 0; b < nb; ++b) {
            const double o = occ[b];
            if (o == 0.0) continue;
            const double v = __ldg(psi + (long)b * ld + i);
            s = fma(o * dV * v, v, s);
        }
    }
    out[i] = s;
}

static int atom_tables(int** aptr, int** alma) {
    Context& c = ctx();
    std::vector<int> cnt(c.natom + 1, 0), lst(c.nzlma);
    for (int l = 0; l < c.nzlma; ++l) cnt[c.h_amap[l] + 1]++;
    for (int a = 0; a < c.natom; ++a) cnt[a + 1] += cnt[a];
    std::vector<int> pos(cnt.begin(), cnt.end() - 1);
    for (int l = 0; l < c.nzlma; ++l) lst[pos[c.h_amap[l]]++] = l;
    RS_CHECK(workspace_t("atom_ptr", cnt.size(), aptr));
    RS_CHECK(workspace_t("atom_lma", lst.size() + 1, alma));
    RS_CUDA(cudaMemcpyAsync(*aptr, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice, c.stream));
    RS_CUDA(cudaMemcpyAsync(*alma, lst.data(), lst.size() * sizeof(int), cudaMemcpyHostToDevice, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    return RSDFT_OK;
}

static int nl_grad(const double* psi, const double* chi, long ld, int nb, const double* occ, double cscale,
                   double* f_dev) {
    Context& c = ctx();
    double* per = nullptr;
    int *aptr, *alma;
    RS_CHECK(workspace_t("force_lma", (size_t)c.nzlma * 3, &per));
    RS_CHECK(atom_tables(&aptr, &alma));
    if (chi)
        launch(k_nl_grad<true>, c.ngroup, FW * 32, 0, c.stream, psi, chi, ld, nb, occ, cscale, c.grp_lma0, c.grp_cnt,
                                                            c.lma_ptr, c.jjp, c.uv, c.duv, c.iuv, c.dV, per, c.err_flag);
    else
        launch(k_nl_grad<false>, c.ngroup, FW * 32, 0, c.stream, psi, chi, ld, nb, occ, cscale, c.grp_lma0, c.grp_cnt,
                                                             c.lma_ptr, c.jjp, c.uv, c.duv, c.iuv, c.dV, per, c.err_flag);
    RS_LAUNCH();
    launch(k_atom_sum, div_up(c.natom * 3, 128), 128, 0, c.stream, per, aptr, alma, c.natom, f_dev);
    RS_LAUNCH();
    return RSDFT_OK;
}

}  // namespace rsdft

using namespace rsdft;

extern "C" {

int rsdft_gpu_force_nloc(int mi, const double* unk, long ld, int mb, const double* occ, double* force2) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    if (!c.nl_set || !c.duv) {
        set_error("force_nloc: nonlocal tables with duvdr are not set");
        return RSDFT_ENOTINIT;
    }
    if (mi != c.natom || ld < c.ml || mb < 1 || !occ || !force2) {
        set_error("force_nloc: bad arguments (MI=%d natom=%d)", mi, c.natom);
        return RSDFT_EINVAL;
    }
    double *d, *docc, *f;
    bool st;
    RS_CHECK(wf_acquire(unk, ld, mb, "force_unk", &d, &st));
    RS_CHECK(stage_in(occ, sizeof(double) * mb, "force_occ", (void**)&docc));
    RS_CHECK(workspace_t("force_out", (size_t)3 * mi, &f));
    if (c.nzlma > 0) {
        // w0 wk with w0 = iuV (-2 occ dV^2) t: cscale * occ * (iuV dV) * t * d
        RS_CHECK(nl_grad(d, nullptr, ld, mb, docc, -2.0 * c.dV, f));
    } else {
        RS_CUDA(cudaMemsetAsync(f, 0, sizeof(double) * 3 * mi, c.stream));
    }
    RS_CHECK(stage_out(force2, f, sizeof(double) * 3 * mi));
    return RSDFT_OK;
}

int rsdft_gpu_hpsi_adjoint(const double* psi, const double* chi, long ld, int nb, const double* occ, double* dl_dv,
                           double* dl_dr) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    if (ld < c.ml || nb < 1 || (!chi && !occ) || (!dl_dv && !dl_dr)) {
        set_error("hpsi_adjoint: bad arguments");
        return RSDFT_EINVAL;
    }
    if (dl_dr && (!c.nl_set || !c.duv)) {
        set_error("hpsi_adjoint: position gradient needs nonlocal tables with duvdr");
        return RSDFT_ENOTINIT;
    }
    double *dp, *dc = nullptr, *docc = nullptr, *gv = nullptr, *gr = nullptr;
    bool sp, sc = false;
    RS_CHECK(wf_acquire(psi, ld, nb, "adj_psi", &dp, &sp));
    if (chi) RS_CHECK(wf_acquire(chi, ld, nb, "adj_chi", &dc, &sc));
    if (occ) RS_CHECK(stage_in(occ, sizeof(double) * nb, "adj_occ", (void**)&docc));
    if (dl_dv) {
        RS_CHECK(workspace_t("adj_dv", (size_t)c.ml, &gv));
        launch(k_vloc_adjoint, div_up(c.ml, 256), 256, 0, c.stream, dp, dc, ld, nb, docc, c.dV, c.ml, gv);
        RS_LAUNCH();
        RS_CHECK(stage_out(dl_dv, gv, sizeof(double) * c.ml));
    }
    if (dl_dr) {
        RS_CHECK(workspace_t("adj_dr", (size_t)3 * c.natom, &gr));
        if (c.nzlma > 0) {
            // chi = occ dV psi: dE/dR = sum 2 occ dV (iuV dV) t d
            RS_CHECK(nl_grad(dp, dc, ld, nb, docc, 2.0 * c.dV, gr));
        } else {
            RS_CUDA(cudaMemsetAsync(gr, 0, sizeof(double) * 3 * c.natom, c.stream));
        }
        RS_CHECK(stage_out(dl_dr, gr, sizeof(double) * 3 * c.natom));
    }
    (void)sp;
    (void)sc;
    return RSDFT_OK;
}

int rsdft_gpu_calc_density(const double* unk, long ld, int mb, const double* occ, double* rho) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    if (ld < c.ml || mb < 1 || !occ || !rho) {
        set_error("calc_density: bad arguments");
        return RSDFT_EINVAL;
    }
    double *dp, *docc = nullptr, *dr = nullptr;
    bool sp;
    RS_CHECK(wf_acquire(unk, ld, mb, "adj_psi", &dp, &sp));
    RS_CHECK(stage_in(occ, sizeof(double) * mb, "adj_occ", (void**)&docc));
    RS_CHECK(workspace_t("adj_dv", (size_t)c.ml, &dr));
    // the V-part adjoint with unit volume element: sum_n occ_n psi_n^2
    launch(k_vloc_adjoint, div_up(c.ml, 256), 256, 0, c.stream, dp, (const double*)nullptr, ld, mb,
           (const double*)docc, 1.0, c.ml, dr);
    RS_LAUNCH();
    RS_CHECK(stage_out(rho, dr, sizeof(double) * c.ml));
    (void)sp;
    return RSDFT_OK;
}

}  // extern "C"
