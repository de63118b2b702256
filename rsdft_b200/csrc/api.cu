// C-ABI set-up entries, device context, workspace and host-pointer registry.
#include <algorithm>
#include <cstdarg>
#include <cstring>
#include <numeric>

#include <cuda.h>

#include "common.cuh"

namespace rsdft {

static Context g_ctx;
long long g_kernel_launches = 0;
static thread_local char g_err[1024] = "";

Context& ctx() { return g_ctx; }

int noalloc_bind_scratch();  // hpsi.cu

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char* get_error() { return g_err; }

int require_init() {
    if (!g_ctx.init) {
        set_error("rsdft_gpu_init has not been called");
        return RSDFT_ENOTINIT;
    }
    return RSDFT_OK;
}

int require_grid() {
    RS_CHECK(require_init());
    if (!g_ctx.grid_set) {
        set_error("rsdft_gpu_set_grid has not been called");
        return RSDFT_ENOTINIT;
    }
    return RSDFT_OK;
}

int set_smem_optin(const void* kernel, int bytes) {
    int& have = g_ctx.smem_optin[kernel];
    if (bytes > have) {
        RS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        have = bytes;
    }
    return RSDFT_OK;
}

char* host_workspace(size_t bytes) {
    if (g_ctx.host_ws.size() < bytes) g_ctx.host_ws.resize(bytes);
    return g_ctx.host_ws.data();
}

int workspace(const char* name, size_t bytes, void** out) {
    Buf& b = g_ctx.ws[name];
    if (b.bytes < bytes) {
        if (b.p) {
            RS_CUDA(cudaStreamSynchronize(g_ctx.stream));
            RS_CUDA(cudaFree(b.p));
            b.p = nullptr;
            b.bytes = 0;
        }
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&b.p, want);
        if (e != cudaSuccess) {
            set_error("workspace '%s': cudaMalloc(%zu) failed: %s", name, want, cudaGetErrorString(e));
            return RSDFT_ENOMEM;
        }
        b.bytes = want;
    }
    *out = b.p;
    return RSDFT_OK;
}

// cuMemGetAddressRange through the driver entry point (no link-time libcuda):
// the allocation that holds a device address, to check a span against it.
using AddressRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);

static AddressRangeFn address_range_fn() {
    static AddressRangeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<AddressRangeFn>(f);
        else
            cudaGetLastError();
    }
    return fn;
}

int resolve(const void* p, size_t bytes, void** dev) {
    if (!p) return 0;
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        at.type = cudaMemoryTypeUnregistered;
    }
    const char* c = static_cast<const char*>(p);
    if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) {
        if (at.type == cudaMemoryTypeDevice && g_ctx.init && at.device != g_ctx.device) {
            set_error("device pointer %p belongs to device %d, the library is bound to device %d", p, at.device,
                      g_ctx.device);
            return RSDFT_EINVAL;
        }
        if (at.type == cudaMemoryTypeDevice && bytes > 0) {
            if (AddressRangeFn fn = address_range_fn()) {
                CUdeviceptr base = 0;
                size_t size = 0;
                if (fn(&base, &size, reinterpret_cast<CUdeviceptr>(p)) == CUDA_SUCCESS) {
                    const size_t off = (size_t)(reinterpret_cast<CUdeviceptr>(p) - base);
                    if (off + bytes > size) {
                        set_error("device array at %p: %zu bytes requested, %zu left in its allocation", p, bytes,
                                  size - off);
                        return RSDFT_EINVAL;
                    }
                }
            }
        }
        *dev = const_cast<void*>(p);
        return 1;
    }
    for (auto& r : g_ctx.regs) {
        if (c >= r.host && c < r.host + r.bytes) {
            if ((size_t)(c - r.host) + bytes > r.bytes) {
                set_error("array at %p: %zu bytes requested, %zu left in its registered wavefunction", p, bytes,
                          (size_t)(r.host + r.bytes - c));
                return RSDFT_EINVAL;
            }
            *dev = r.dev + (c - r.host);
            return 1;
        }
    }
    return 0;
}

int stage_in(const void* p, size_t bytes, const char* wsname, void** dev) {
    const int r = resolve(p, bytes, dev);
    if (r < 0) return r;
    if (r) return RSDFT_OK;
    RS_CHECK(workspace(wsname, bytes, dev));
    RS_CUDA(cudaMemcpyAsync(*dev, p, bytes, cudaMemcpyHostToDevice, g_ctx.stream));
    return RSDFT_OK;
}

int stage_out(void* p, const void* dev, size_t bytes) {
    void* d = nullptr;
    const int r = resolve(p, bytes, &d);
    if (r < 0) return r;
    if (r) {
        if (d != dev) RS_CUDA(cudaMemcpyAsync(d, dev, bytes, cudaMemcpyDeviceToDevice, g_ctx.stream));
        return RSDFT_OK;
    }
    RS_CUDA(cudaMemcpyAsync(p, dev, bytes, cudaMemcpyDeviceToHost, g_ctx.stream));
    RS_CUDA(cudaStreamSynchronize(g_ctx.stream));
    return RSDFT_OK;
}

int wf_acquire(const double* p, long ld, int nb, const char* wsname, double** dev, bool* staged,
               bool copy_in) {
    void* d = nullptr;
    *staged = false;
    if (!p) {
        set_error("NULL wavefunction pointer");
        return RSDFT_EINVAL;
    }
    size_t bytes = sizeof(double) * (size_t)ld * (size_t)nb;
    const int r = resolve(p, bytes, &d);
    if (r < 0) return r;
    if (r) {
        *dev = static_cast<double*>(d);
        return RSDFT_OK;
    }
    RS_CHECK(workspace(wsname, bytes, &d));
    if (copy_in) RS_CUDA(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, g_ctx.stream));
    *dev = static_cast<double*>(d);
    *staged = true;
    return RSDFT_OK;
}

int wf_release(double* p, const double* dev, long ld, int nb, bool staged) {
    if (!staged) return RSDFT_OK;
    size_t bytes = sizeof(double) * (size_t)ld * (size_t)nb;
    RS_CUDA(cudaMemcpyAsync(p, dev, bytes, cudaMemcpyDeviceToHost, g_ctx.stream));
    RS_CUDA(cudaStreamSynchronize(g_ctx.stream));
    return RSDFT_OK;
}

template <typename T>
static int upload(T** dst, const T* src, size_t n) {
    if (*dst) {
        RS_CUDA(cudaFree(*dst));
        *dst = nullptr;
    }
    if (n == 0) return RSDFT_OK;
    if (cudaMalloc(dst, n * sizeof(T)) != cudaSuccess) {
        set_error("cudaMalloc(%zu) failed", n * sizeof(T));
        return RSDFT_ENOMEM;
    }
    RS_CUDA(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyDefault));
    return RSDFT_OK;
}

// copy a caller array (host or device) to host memory
template <typename T>
static int fetch(std::vector<T>& out, const T* src, size_t n) {
    out.resize(n);
    if (n) RS_CUDA(cudaMemcpy(out.data(), src, n * sizeof(T), cudaMemcpyDefault));
    return RSDFT_OK;
}

}  // namespace rsdft

using namespace rsdft;

extern "C" {

int rsdft_gpu_init(int device) {
    RS_ENTRY();
    Context& c = g_ctx;
    if (c.init && c.device == device) return RSDFT_OK;
    if (c.init) rsdft_gpu_finalize();
    int n = 0;
    RS_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) {
        set_error("device %d out of range (%d devices)", device, n);
        return RSDFT_EINVAL;
    }
    RS_CUDA(cudaSetDevice(device));
    RS_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    c.own_stream = true;
    RS_SOLVER(cusolverDnCreate(&c.solver));
    RS_SOLVER(cusolverDnSetStream(c.solver, c.stream));
    RS_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, device));
    RS_CUDA(cudaMalloc(&c.err_flag, 16));
    RS_CUDA(cudaMemset(c.err_flag, 0, 16));
    RS_CUDA(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < Context::NEV; ++i) RS_CUDA(cudaEventCreateWithFlags(&c.ev[i], cudaEventDisableTiming));
    c.device = device;
    // the device address of rsdft_gpu_hamiltonian_noalloc's static scratch,
    // looked up now so that entry never loads a module or allocates
    RS_CHECK(noalloc_bind_scratch());
    c.init = true;
    return RSDFT_OK;
}

int rsdft_gpu_finalize(void) {
    RS_ENTRY();
    Context& c = g_ctx;
    if (!c.init) return RSDFT_OK;
    cudaStreamSynchronize(c.stream);
    if (c.copy_stream) {
        cudaStreamSynchronize(c.copy_stream);
        cudaStreamDestroy(c.copy_stream);
        c.copy_stream = nullptr;
    }
    for (int i = 0; i < Context::NEV; ++i)
        if (c.ev[i]) {
            cudaEventDestroy(c.ev[i]);
            c.ev[i] = nullptr;
        }
    for (auto& kv : c.ws)
        if (kv.second.p) cudaFree(kv.second.p);
    c.ws.clear();
    for (auto& r : c.regs) cudaFree(r.dev);
    c.regs.clear();
    void* ptrs[] = {c.err_flag, c.vloc, c.vloc32, c.lma_ptr, c.jjp, c.uv, c.uv32, c.iuv, c.amap, c.duv,
                    c.grp_lma0, c.grp_cnt, c.pt_ptr, c.pt_lma, c.pt_uv, c.pt_uv32,
                    c.gpt_ptr, c.gpt_grp, c.gpt_uv4, c.gpt_uv4_32, c.nl_pts, c.nl_ptr};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c.solver) cusolverDnDestroy(c.solver);
    if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
    c = Context();
    return RSDFT_OK;
}

const char* rsdft_gpu_last_error(void) { return get_error(); }

long long rsdft_gpu_kernel_launches(void) { return g_kernel_launches; }

long long rsdft_gpu_workspace_bytes(void) {
    long long n = 0;
    for (const auto& kv : g_ctx.ws) n += (long long)kv.second.bytes;
    return n;
}

int rsdft_gpu_set_stream(void* stream) {
    RS_ENTRY();
    RS_CHECK(require_init());
    Context& c = g_ctx;
    if (c.own_stream && c.stream) {
        RS_CUDA(cudaStreamSynchronize(c.stream));
        RS_CUDA(cudaStreamDestroy(c.stream));
        c.own_stream = false;
    }
    if (stream) {
        c.stream = static_cast<cudaStream_t>(stream);
    } else {
        RS_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        c.own_stream = true;
    }
    RS_SOLVER(cusolverDnSetStream(c.solver, c.stream));
    return RSDFT_OK;
}

int rsdft_gpu_synchronize(void) {
    RS_ENTRY();
    RS_CHECK(require_init());
    RS_CUDA(cudaStreamSynchronize(g_ctx.stream));
    int word[4] = {0, 0, 0, 0};
    RS_CUDA(cudaMemcpy(word, g_ctx.err_flag, sizeof(word), cudaMemcpyDeviceToHost));
    if (word[0] || word[1]) RS_CUDA(cudaMemset(g_ctx.err_flag, 0, sizeof(word)));
    if (word[0]) {
        set_error("a kernel's bounded wait for a bulk copy ran out (code %d)", word[0]);
        return RSDFT_ETIMEOUT;
    }
    if (word[1]) {
        set_error("in-kernel index check failed: site %d, index %d (%d failed checks)", word[1], word[2], word[3]);
        return RSDFT_ECHECK;
    }
    return RSDFT_OK;
}

int rsdft_gpu_set_grid(const int* ngrid, int md, double coef_lap0, const double* coef_lap,
                       const double* hgrid, const double* ggg, double dv) {
    RS_ENTRY();
    RS_CHECK(require_init());
    Context& c = g_ctx;
    if (!ngrid || !coef_lap || !hgrid) {
        set_error("set_grid: NULL argument");
        return RSDFT_EINVAL;
    }
    if (md < 1 || md > MAXMD) {
        set_error("set_grid: Md=%d unsupported (1..%d)", md, MAXMD);
        return RSDFT_EUNSUP;
    }
    for (int a = 0; a < 3; ++a)
        if (ngrid[a] < 1) {
            set_error("set_grid: bad Ngrid");
            return RSDFT_EINVAL;
        }
    if (ngrid[0] < 1 || ngrid[1] < 1 || ngrid[2] < 1 || !(dv > 0.0)) {
        set_error("set_grid: bad Ngrid or dV");
        return RSDFT_EINVAL;
    }
    c.n1 = ngrid[0];
    c.n2 = ngrid[1];
    c.n3 = ngrid[2];
    c.ml = (long)c.n1 * c.n2 * c.n3;
    c.md = md;
    c.dV = dv;
    double g[3] = {1.0, 1.0, 1.0};
    if (ggg)
        for (int a = 0; a < 3; ++a) g[a] = ggg[a];
    std::memset(&c.sc, 0, sizeof(c.sc));
    c.sc.c0 = coef_lap0;
    for (int m = 0; m < md; ++m) {
        c.sc.cx[m] = coef_lap[0 * md + m];
        c.sc.cy[m] = coef_lap[1 * md + m];
        c.sc.cz[m] = coef_lap[2 * md + m];
    }
    for (int a = 0; a < 3; ++a) c.hgrid[a] = hgrid[a];
    // precond_cg_mat2_omp, cgpc_hprsdft_module.f90:290-293
    c.pc.c = g[0] / (hgrid[0] * hgrid[0]) + g[1] / (hgrid[1] * hgrid[1]) + g[2] / (hgrid[2] * hgrid[2]);
    c.pc.c1 = -0.5 / (hgrid[0] * hgrid[0]) * g[0];
    c.pc.c2 = -0.5 / (hgrid[1] * hgrid[1]) * g[1];
    c.pc.c3 = -0.5 / (hgrid[2] * hgrid[2]) * g[2];
    // nonlocal tables sized for an earlier grid must not be used with this one
    // (Vloc is checked against the grid at use)
    c.nl_set = false;
    c.grid_set = true;
    return RSDFT_OK;
}

int rsdft_gpu_set_vloc(const double* vloc, long ml, int nspin) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = g_ctx;
    if (!vloc || ml != c.ml || nspin < 1) {
        set_error("set_vloc: ml=%ld (grid %ld), nspin=%d", ml, c.ml, nspin);
        return RSDFT_EINVAL;
    }
    std::vector<double> h;
    RS_CHECK(fetch(h, vloc, (size_t)ml * nspin));
    std::vector<float> h32(h.begin(), h.end());
    RS_CHECK(upload(&c.vloc, h.data(), h.size()));
    RS_CHECK(upload(&c.vloc32, h32.data(), h32.size()));
    c.nspin = nspin;
    c.vloc_ml = ml;
    return RSDFT_OK;
}

int rsdft_gpu_set_nonlocal(int nzlma, const int* lma_ptr, const int* jjp, const double* uv,
                           const int* iuv, const int* amap, int natom, const double* duvdr) {
    RS_ENTRY();
    RS_CHECK(require_grid());
    Context& c = g_ctx;
    if (nzlma < 0 || (nzlma > 0 && (!lma_ptr || !jjp || !uv || !iuv || !amap))) {
        set_error("set_nonlocal: bad arguments");
        return RSDFT_EINVAL;
    }
    std::vector<int> hptr, hjjp, hiuv, hamap;
    std::vector<double> huv, hduv;
    RS_CHECK(fetch(hptr, lma_ptr, (size_t)nzlma + 1));
    long nnz = nzlma > 0 ? hptr[nzlma] : 0;
    if (nzlma > 0 && hptr[0] != 0) {
        set_error("set_nonlocal: lma_ptr[0] must be 0");
        return RSDFT_EINVAL;
    }
    for (int l = 0; l < nzlma; ++l)
        if (hptr[l + 1] < hptr[l]) {
            set_error("set_nonlocal: lma_ptr not monotone at %d", l);
            return RSDFT_EINVAL;
        }
    RS_CHECK(fetch(hjjp, jjp, nnz));
    RS_CHECK(fetch(huv, uv, nnz));
    RS_CHECK(fetch(hiuv, iuv, nzlma));
    RS_CHECK(fetch(hamap, amap, nzlma));
    for (long j = 0; j < nnz; ++j)
        if (hjjp[j] < 0 || hjjp[j] >= c.ml) {
            set_error("set_nonlocal: jjp[%ld]=%d outside the grid", j, hjjp[j]);
            return RSDFT_EINVAL;
        }
    for (int l = 0; l < nzlma; ++l)
        if (hamap[l] < 0 || hamap[l] >= natom) {
            set_error("set_nonlocal: amap[%d]=%d outside 0..%d", l, hamap[l], natom - 1);
            return RSDFT_EINVAL;
        }
    if (duvdr) RS_CHECK(fetch(hduv, duvdr, (size_t)nnz * 3));

    // sphere groups: consecutive projectors with identical point lists
    std::vector<int> g0, gc;
    for (int l = 0; l < nzlma;) {
        int e = l + 1;
        while (e < nzlma && e - l < 4) {
            long n0 = hptr[l + 1] - hptr[l], n1 = hptr[e + 1] - hptr[e];
            if (n0 != n1 || !std::equal(hjjp.begin() + hptr[l], hjjp.begin() + hptr[l + 1], hjjp.begin() + hptr[e]))
                break;
            ++e;
        }
        g0.push_back(l);
        gc.push_back(e - l);
        l = e;
    }
    // point-major CSR of the scatter, entries of one point in projector order
    std::vector<int> cnt(c.ml + 1, 0);
    for (long j = 0; j < nnz; ++j) cnt[hjjp[j] + 1]++;
    std::partial_sum(cnt.begin(), cnt.end(), cnt.begin());
    std::vector<int> pos(cnt.begin(), cnt.end() - 1), plma(nnz);
    std::vector<double> puv(nnz);
    for (int l = 0; l < nzlma; ++l)
        for (int j = hptr[l]; j < hptr[l + 1]; ++j) {
            int q = pos[hjjp[j]]++;
            plma[q] = l;
            puv[q] = huv[j];
        }
    // the same scatter per sphere group: one entry per (point, group) holding
    // the group's (up to 4) projector values at that point
    std::vector<int> gcnt(c.ml + 1, 0);
    for (size_t g = 0; g < g0.size(); ++g)
        for (int j = hptr[g0[g]]; j < hptr[g0[g] + 1]; ++j) gcnt[hjjp[j] + 1]++;
    std::partial_sum(gcnt.begin(), gcnt.end(), gcnt.begin());
    const long ngnnz = gcnt[c.ml];
    std::vector<int> gpos(gcnt.begin(), gcnt.end() - 1), ggrp(ngnnz);
    std::vector<double> guv((size_t)ngnnz * 4, 0.0);
    for (size_t g = 0; g < g0.size(); ++g) {
        const int l0 = g0[g];
        for (int j = hptr[l0]; j < hptr[l0 + 1]; ++j) {
            const int q = gpos[hjjp[j]]++;
            ggrp[q] = l0;
            for (int k = 0; k < gc[g]; ++k) guv[(size_t)q * 4 + k] = huv[hptr[l0 + k] + (j - hptr[l0])];
        }
    }
    // covered points and their entry ranges, for the scatter after the stencil
    std::vector<int> npts, nptr;
    for (long p = 0; p < c.ml; ++p)
        if (gcnt[p + 1] > gcnt[p]) {
            npts.push_back((int)p);
            nptr.push_back(gcnt[p]);
        }
    nptr.push_back(gcnt[c.ml]);
    gcnt.resize(c.ml + 8, gcnt[c.ml]);  // padding for vector reads past the end
    std::vector<float> guv32(guv.begin(), guv.end());
    RS_CHECK(upload(&c.gpt_ptr, gcnt.data(), gcnt.size()));
    RS_CHECK(upload(&c.gpt_grp, ggrp.data(), ggrp.size()));
    RS_CHECK(upload(&c.gpt_uv4, guv.data(), guv.size()));
    RS_CHECK(upload(&c.gpt_uv4_32, guv32.data(), guv32.size()));
    RS_CHECK(upload(&c.nl_pts, npts.data(), npts.size()));
    RS_CHECK(upload(&c.nl_ptr, nptr.data(), nptr.size()));
    c.nl_npt = (int)npts.size();
    std::vector<float> huv32(huv.begin(), huv.end()), puv32(puv.begin(), puv.end());
    RS_CHECK(upload(&c.lma_ptr, hptr.data(), hptr.size()));
    RS_CHECK(upload(&c.jjp, hjjp.data(), hjjp.size()));
    RS_CHECK(upload(&c.uv, huv.data(), huv.size()));
    RS_CHECK(upload(&c.uv32, huv32.data(), huv32.size()));
    RS_CHECK(upload(&c.iuv, hiuv.data(), hiuv.size()));
    RS_CHECK(upload(&c.amap, hamap.data(), hamap.size()));
    RS_CHECK(upload(&c.duv, hduv.data(), hduv.size()));
    RS_CHECK(upload(&c.grp_lma0, g0.data(), g0.size()));
    RS_CHECK(upload(&c.grp_cnt, gc.data(), gc.size()));
    RS_CHECK(upload(&c.pt_ptr, cnt.data(), cnt.size()));
    RS_CHECK(upload(&c.pt_lma, plma.data(), plma.size()));
    RS_CHECK(upload(&c.pt_uv, puv.data(), puv.size()));
    RS_CHECK(upload(&c.pt_uv32, puv32.data(), puv32.size()));
    c.nzlma = nzlma;
    c.natom = natom;
    c.nnz = nnz;
    c.ngroup = (int)g0.size();
    c.h_amap = hamap;
    c.nl_set = true;
    return RSDFT_OK;
}

int rsdft_gpu_register_wf(double* unk, long ml, int mb) {
    RS_ENTRY();
    RS_CHECK(require_init());
    if (!unk || ml <= 0 || mb <= 0) {
        set_error("register_wf: bad arguments");
        return RSDFT_EINVAL;
    }
    Context& c = g_ctx;
    size_t bytes = sizeof(double) * (size_t)ml * mb;
    char* h = reinterpret_cast<char*>(unk);
    for (auto& r : c.regs)
        if (h < r.host + r.bytes && r.host < h + bytes) {
            set_error("register_wf: range overlaps a registered array");
            return RSDFT_EINVAL;
        }
    WfReg r;
    r.host = h;
    r.bytes = bytes;
    if (cudaMalloc(&r.dev, bytes) != cudaSuccess) {
        set_error("register_wf: cudaMalloc(%zu) failed", bytes);
        return RSDFT_ENOMEM;
    }
    RS_CUDA(cudaMemcpyAsync(r.dev, r.host, bytes, cudaMemcpyHostToDevice, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    c.regs.push_back(r);
    return RSDFT_OK;
}

static WfReg* find_reg(double* unk) {
    char* h = reinterpret_cast<char*>(unk);
    for (auto& r : g_ctx.regs)
        if (r.host == h) return &r;
    return nullptr;
}

int rsdft_gpu_unregister_wf(double* unk) {
    RS_ENTRY();
    RS_CHECK(require_init());
    Context& c = g_ctx;
    for (size_t i = 0; i < c.regs.size(); ++i)
        if (c.regs[i].host == reinterpret_cast<char*>(unk)) {
            RS_CUDA(cudaStreamSynchronize(c.stream));
            RS_CUDA(cudaFree(c.regs[i].dev));
            c.regs.erase(c.regs.begin() + i);
            return RSDFT_OK;
        }
    set_error("unregister_wf: pointer not registered");
    return RSDFT_EINVAL;
}

int rsdft_gpu_sync_to_host(double* unk) {
    RS_ENTRY();
    RS_CHECK(require_init());
    WfReg* r = find_reg(unk);
    if (!r) {
        set_error("sync_to_host: pointer not registered");
        return RSDFT_EINVAL;
    }
    RS_CUDA(cudaMemcpyAsync(r->host, r->dev, r->bytes, cudaMemcpyDeviceToHost, g_ctx.stream));
    RS_CUDA(cudaStreamSynchronize(g_ctx.stream));
    return RSDFT_OK;
}

int rsdft_gpu_sync_to_device(double* unk) {
    RS_ENTRY();
    RS_CHECK(require_init());
    WfReg* r = find_reg(unk);
    if (!r) {
        set_error("sync_to_device: pointer not registered");
        return RSDFT_EINVAL;
    }
    RS_CUDA(cudaMemcpyAsync(r->dev, r->host, r->bytes, cudaMemcpyHostToDevice, g_ctx.stream));
    return RSDFT_OK;
}

}  // extern "C"
