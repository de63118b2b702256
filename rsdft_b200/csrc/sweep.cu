// calc_sweep's iteration loop on device-resident bands (sweep_module.f90:
// 60-226): per iteration, every spin's conjugate_gradient + gram_schmidt +
// subspace_diag, esp_gather, calc_fermi and conv_check, with the bands, the
// eigenvalues and the occupations never leaving the device.  The host reads
// one scalar per iteration (the eigenvalue change conv_check tests) to decide
// whether to stop, as the reference's loop does after its allreduce.
//
// calc_fermi (fermi_mp_module.f90:95-284) is the Methfessel-Paxton
// occupation of order kinteg with smearing ekbt: bisection for the Fermi
// level on [min esp, max esp + min(100 ekbt, 0.1)] until the electron count
// is matched exactly or the midpoint stops moving, run by one CTA (the
// eigenvalues of one Gamma point are a few thousand values at most).  Sums
// over bands use a fixed reduction tree, so the result is reproducible; its
// order differs from the reference's sequential sum only by rounding.
// esp_gather (esp_gather_module.f90:11-61) gathers band slices held by other
// ranks: with one process holding every band there is nothing to gather.
#include "common.cuh"
#include "kernels.cuh"

namespace rsdft {

namespace {

constexpr int FM_T = 256;

// ff0 (fermi_mp_module.f90:287-306): 0.5 (1 - erf x) plus the Hermite
// series of order n with the coefficients of factor(:) (:147-153)
__device__ double mp_ff0(int n, double x) {
    double ff0 = 0.5 * (1.0 - erf(x));
    if (n <= 0) return ff0;
    double fac = -1.0 / (4.0 * sqrt(acos(-1.0)));  // factor(1)
    double hp0 = 1.0, hp1 = 2.0 * x;
    double ff = fac * hp1;
    for (int i = 2; i <= n; ++i) {
        fac = -fac / (4.0 * i);
        const double hp2 = 2.0 * x * hp1 - 2.0 * (2 * i - 3) * hp0;
        const double hp3 = 2.0 * x * hp2 - 2.0 * (2 * i - 2) * hp1;
        ff += fac * hp3;
        hp0 = hp2;
        hp1 = hp3;
    }
    return ff0 + ff * exp(-x * x);
}

// block min / max / sum over the CTA, result broadcast to every thread
__device__ double block_all_sum(double v, double* sh) {
    const double r = block_sum<FM_T>(v, sh);
    if (threadIdx.x == 0) sh[0] = r;
    __syncthreads();
    const double out = sh[0];
    __syncthreads();
    return out;
}

__device__ double block_all_minmax(double v, double* sh, bool is_max) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const double o = __shfl_xor_sync(0xffffffffu, v, s);
        v = is_max ? fmax(v, o) : fmin(v, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = sh[0];
        for (int i = 1; i < FM_T / 32; ++i) r = is_max ? fmax(r, sh[i]) : fmin(r, sh[i]);
        sh[FM_T / 32] = r;
    }
    __syncthreads();
    const double out = sh[FM_T / 32];
    __syncthreads();
    return out;
}

// Occupations of one bisection over the spins [s0, s1) for a target count
// zne; sets occ (the bare ff values) and returns the last midpoint.  Ends
// when the count is matched exactly or the midpoint stops moving (then
// accepted as is, as the reference's goto 100 does); after 1000 steps *ok =
// 0 if the count is off by more than 1e-10 (the reference's 'EF IS NOT
// CONVERGED' stop).
__device__ double fermi_bisect(const double* esp, double* occ, int mb, int s0, int s1, double zne, double weight,
                               double ekbt, int kinteg, double* sh, int* ok) {
    const int n = (s1 - s0) * mb;
    double lo = 1e300, hi = -1e300;
    for (int i = threadIdx.x; i < n; i += FM_T) {
        lo = fmin(lo, esp[(long)s0 * mb + i]);
        hi = fmax(hi, esp[(long)s0 * mb + i]);
    }
    double ef1 = block_all_minmax(lo, sh, false), ef2 = block_all_minmax(hi, sh, true);
    if (ef1 == ef2) {
        ef1 -= 0.01;
        ef2 += 0.01;
    }
    ef2 += fmin(ekbt * 1e2, 0.1);
    double ef0 = 1e10, ef = 0.5 * (ef1 + ef2), octmp = 0.0;
    for (int id = 1; id <= 1000; ++id) {
        ef = 0.5 * (ef1 + ef2);
        if (ef == ef0) return ef;  // the interval cannot shrink further: accepted without the count check
        double part = 0.0;
        for (int i = threadIdx.x; i < n; i += FM_T) {
            const double ff = mp_ff0(kinteg, (esp[(long)s0 * mb + i] - ef) / ekbt);
            occ[(long)s0 * mb + i] = ff;
            part += ff * weight;
        }
        octmp = block_all_sum(part, sh);
        if (octmp - zne > 0.0)
            ef2 = ef;
        else if (octmp - zne < 0.0)
            ef1 = ef;
        else
            break;
        ef0 = ef;
    }
    if (fabs(octmp - zne) > 1e-10) *ok = 0;
    return ef;
}

// calc_fermi for one Gamma point (MBZ = 1, wbz = 1), all bands (mb1 = 1,
// mb2 = MB): one bisection over all spins (MSP = 1, or iter > nfixed), else
// one per spin with the fixed moment dspn; occ = 2 ff / MSP.  out[0] = ef,
// out[1] = 1 if the electron count was matched.
__global__ void __launch_bounds__(FM_T) k_calc_fermi(const double* __restrict__ esp, double* __restrict__ occ, int mb,
                                                     int msp, double znel, double dspn, int fixed, double ekbt,
                                                     int kinteg, double* __restrict__ out) {
    __shared__ double sh[FM_T / 32 + 1];
    int ok = 1;
    double ef;
    if (!fixed) {
        ef = fermi_bisect(esp, occ, mb, 0, msp, znel, 2.0 / msp, ekbt, kinteg, sh, &ok);
    } else {
        ef = 0.0;
        for (int s = 0; s < msp; ++s)
            ef = fermi_bisect(esp, occ, mb, s, s + 1, 0.5 * znel + (1 - 2 * s) * 0.5 * dspn, 1.0, ekbt, kinteg, sh,
                              &ok);
    }
    for (int i = threadIdx.x; i < msp * mb; i += FM_T) occ[i] = 2.0 * occ[i] / msp;
    if (threadIdx.x == 0) {
        out[0] = ef;
        out[1] = ok;
    }
}

// conv_check_2/3 (sweep_module.f90:255-280): the largest |esp - esp0| over
// bands 1..mb_ref of every spin; mode 3 also writes res = |esp - esp0|, with
// -1 where it is below tol.
__global__ void __launch_bounds__(FM_T) k_conv_check(const double* __restrict__ esp, const double* __restrict__ esp0,
                                                     double* __restrict__ res, int mb, int msp, int mb_ref, int mode,
                                                     double tol, double* __restrict__ out) {
    __shared__ double sh[FM_T / 32 + 1];
    double m = 0.0;
    for (int i = threadIdx.x; i < msp * mb; i += FM_T) {
        const double d = fabs(esp[i] - esp0[i]);
        if (i % mb < mb_ref) m = fmax(m, d);
        if (mode == 3) res[i] = d < tol ? -1.0 : d;
    }
    m = block_all_minmax(m, sh, true);
    if (threadIdx.x == 0) out[2] = m;
}

}  // namespace
}  // namespace rsdft

using namespace rsdft;

extern "C" int rsdft_gpu_calc_sweep(double* unk, long ld, int mb, int nspin, double* esp, double* res, double* occ,
                                    int diter, int iconv_check, double tol_esp, int mb_ref, double nelectron,
                                    int nfixed, double dspn, double ekbt, int kinteg, int ncg, int mloop, int ipc,
                                    int mode, int* iter_out, int* conv_out, double* efermi) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = ctx();
    if (!unk || !esp || !res || !occ || !iter_out || !conv_out || ld != c.ml || mb < 1 || mb > 65535 ||
        nspin < 1 || nspin > c.nspin || nspin > 2 || diter < 0 || mb_ref < 1 || mb_ref > mb || !(ekbt > 0.0) ||
        kinteg < 0 || kinteg > 50 || ncg < 0 || mloop < 0 || (ipc != 0 && ipc != 4) || !mode_valid(mode) ||
        !(nelectron > 0.0)) {
        set_error("calc_sweep: bad arguments");
        return RSDFT_EINVAL;
    }
    if (iconv_check != 2 && iconv_check != 3) {
        set_error("calc_sweep: iconv_check=%d; 1 tests the total energy, which needs the SCF potential (only 2 "
                  "and 3, the eigenvalue tests, are built)",
                  iconv_check);
        return RSDFT_EUNSUP;
    }
    *iter_out = 0;
    *conv_out = 0;
    if (diter == 0) return RSDFT_OK;
    const size_t nval = (size_t)mb * nspin;
    double *d, *E, *E0, *R, *O, *scal;
    bool st;
    RS_CHECK(wf_acquire(unk, ld, mb * nspin, "csweep_unk", &d, &st));
    RS_CHECK(workspace_t("csweep_e", nval * 4 + 4, &E));
    E0 = E + nval;
    R = E0 + nval;
    O = R + nval;
    scal = O + nval;
    // esp on entry is esp0 of the first iteration (the reference keeps the
    // eigenvalues of the previous sweep or of the initial subspace step)
    void* de = nullptr;
    RS_CHECK(stage_in(esp, sizeof(double) * nval, "csweep_esp_in", &de));
    RS_CUDA(cudaMemcpyAsync(E, de, sizeof(double) * nval, cudaMemcpyDeviceToDevice, c.stream));
    bool conv = false;
    int iter = 0;
    double host[3] = {0.0, 0.0, 0.0};
    for (iter = 1; iter <= diter; ++iter) {
        RS_CUDA(cudaMemcpyAsync(E0, E, sizeof(double) * nval, cudaMemcpyDeviceToDevice, c.stream));
        for (int s = 1; s <= nspin; ++s)
            RS_CHECK(sweep_device(d + (size_t)(s - 1) * ld * mb, ld, mb, s, E + (size_t)(s - 1) * mb,
                                  R + (size_t)(s - 1) * mb, ncg, mloop, ipc, mode));
        // esp_gather: one process holds every band
        launch(k_calc_fermi, 1, FM_T, 0, c.stream, (const double*)E, O, mb, nspin, nelectron, dspn,
               (nspin == 2 && iter <= nfixed) ? 1 : 0, ekbt, kinteg, scal);
        RS_LAUNCH();
        launch(k_conv_check, 1, FM_T, 0, c.stream, (const double*)E, (const double*)E0, R, mb, nspin, mb_ref,
               iconv_check, tol_esp, scal);
        RS_LAUNCH();
        RS_CUDA(cudaMemcpyAsync(host, scal, sizeof(host), cudaMemcpyDeviceToHost, c.stream));
        RS_CUDA(cudaStreamSynchronize(c.stream));
        if (host[1] == 0.0) {
            set_error("calc_sweep: Fermi level not converged at iteration %d (electron count not matched)", iter);
            return RSDFT_ESOLVER;
        }
        conv = host[2] < tol_esp;
        if (conv || iter == diter) break;
    }
    RS_CHECK(stage_out(esp, E, sizeof(double) * nval));
    RS_CHECK(stage_out(res, R, sizeof(double) * nval));
    RS_CHECK(stage_out(occ, O, sizeof(double) * nval));
    RS_CHECK(wf_release(unk, d, ld, mb * nspin, st));
    *iter_out = iter;
    *conv_out = conv ? 1 : 0;
    if (efermi) *efermi = host[0];
    return RSDFT_OK;
}
