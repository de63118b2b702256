// Shared state of the RSDFT B200 library: device context, workspace,
// host-pointer registry and error reporting.  One context per process; the
// library is not thread-safe (one CUDA stream per context).
#pragma once

#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/rsdft_gpu.h"

namespace rsdft {

// A named NVTX range over one C-ABI call (the entry's name), so profiler
// timelines group the kernels by the reference routine they replace (the
// role of the reference's watchb timers, watch_module.f90:89-219).  Without
// a profiler attached the NVTX calls do nothing.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
#define RS_ENTRY() const ::rsdft::NvtxRange rs_entry_range_(__func__)

constexpr int MAXMD = 8;

struct StencilCoef {
    double c0;            // coef_lap0 + const_k2 (Gamma: const_k2 = 0)
    double cx[MAXMD];     // coef_lap(1, m)
    double cy[MAXMD];     // coef_lap(2, m)
    double cz[MAXMD];     // coef_lap(3, m)
};

struct PrecondCoef {
    double c, c1, c2, c3;  // precond_cg_mat2_omp operator
};

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct WfReg {
    char* host = nullptr;
    size_t bytes = 0;
    char* dev = nullptr;
};

struct Context {
    bool init = false;
    int device = -1;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t copy_stream = nullptr;  // host<->device staging that overlaps compute
    static constexpr int NEV = 16;
    cudaEvent_t ev[NEV] = {};
    cusolverDnHandle_t solver = nullptr;
    int num_sms = 0;
    // error word (4 ints): [0] code of a bounded wait that ran out; debug
    // build: [1] site of the first failed index check, [2] its index, [3]
    // the number of failed checks
    int* err_flag = nullptr;

    // grid
    bool grid_set = false;
    int n1 = 0, n2 = 0, n3 = 0, md = 0;
    long ml = 0;
    double dV = 0.0;
    double hgrid[3] = {0, 0, 0};
    StencilCoef sc{};
    PrecondCoef pc{};

    // local potential (ml x nspin)
    int nspin = 0;
    double* vloc = nullptr;
    float* vloc32 = nullptr;
    long vloc_ml = -1;  // grid size Vloc was given for

    // nonlocal tables
    bool nl_set = false;
    int nzlma = 0, natom = 0;
    long nnz = 0;
    int* lma_ptr = nullptr;     // nzlma+1
    int* jjp = nullptr;         // nnz
    double* uv = nullptr;       // nnz
    float* uv32 = nullptr;
    int* iuv = nullptr;         // nzlma
    int* amap = nullptr;        // nzlma
    double* duv = nullptr;      // nnz x 3 (row-major)
    int ngroup = 0;             // sphere groups: consecutive lma sharing one point list
    int* grp_lma0 = nullptr;    // ngroup
    int* grp_cnt = nullptr;     // ngroup
    int* pt_ptr = nullptr;      // ml+1: point-major CSR of the scatter
    int* pt_lma = nullptr;      // nnz
    double* pt_uv = nullptr;    // nnz
    float* pt_uv32 = nullptr;
    int* gpt_ptr = nullptr;     // ml+1: point-major CSR over sphere groups
    int* gpt_grp = nullptr;     // first projector of the group
    double* gpt_uv4 = nullptr;  // 4 projector values of the group at the point
    float* gpt_uv4_32 = nullptr;
    int nl_npt = 0;             // grid points covered by at least one sphere
    int* nl_pts = nullptr;      // nl_npt: those points, ascending
    int* nl_ptr = nullptr;      // nl_npt+1: their first entry in the group CSR
    std::vector<int> h_amap;

    // workspace
    std::map<std::string, Buf> ws;
    std::vector<WfReg> regs;
    std::vector<char> host_ws;               // host scratch of cuSOLVER calls
    std::map<const void*, int> smem_optin;   // dynamic shared memory opted in, per kernel
    int max_smem_optin = -1;                 // device limit (cudaDevAttrMaxSharedMemoryPerBlockOptin)
    int sytrd_clusters = -1;                 // active 16-CTA clusters of the eigensolver kernel
    double* noalloc_scratch = nullptr;       // device address of the static scratch array
};

Context& ctx();

// ---------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
const char* get_error();

#define RS_CUDA(call)                                                                 \
    do {                                                                              \
        cudaError_t _e = (call);                                                      \
        if (_e != cudaSuccess) {                                                      \
            ::rsdft::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,             \
                               cudaGetErrorString(_e));                               \
            return RSDFT_ECUDA;                                                       \
        }                                                                             \
    } while (0)

#define RS_SOLVER(call)                                                               \
    do {                                                                              \
        cusolverStatus_t _s = (call);                                                 \
        if (_s != CUSOLVER_STATUS_SUCCESS) {                                          \
            ::rsdft::set_error("%s:%d %s: cusolver status %d", __FILE__, __LINE__,   \
                               #call, (int)_s);                                       \
            return RSDFT_ESOLVER;                                                     \
        }                                                                             \
    } while (0)

#define RS_CHECK(expr)                                                                \
    do {                                                                              \
        int _r = (expr);                                                              \
        if (_r != RSDFT_OK) return _r;                                                \
    } while (0)

#define RS_LAUNCH()                                                                   \
    do {                                                                              \
        cudaError_t _e = cudaGetLastError();                                          \
        if (_e != cudaSuccess) {                                                      \
            ::rsdft::set_error("%s:%d launch: %s", __FILE__, __LINE__,                \
                               cudaGetErrorString(_e));                               \
            return RSDFT_ECUDA;                                                       \
        }                                                                             \
    } while (0)

// In-kernel index checks of the debug build (-DRSDFT_GPU_CHECK).  A check
// that fails records its site (first failure only), the index and a count in
// the context's error word and yields false, so the caller skips the access;
// rsdft_gpu_synchronize then reports RSDFT_ECHECK.  In the normal build a
// check is the constant true and the compiler removes it.
enum CheckSite : int {
    CK_NL_PROJECT_POINT = 1,  // k_nl_project: grid point of a sphere entry
    CK_NL_SCATTER_POINT = 2,  // k_nl_scatter: grid point of a scatter row
    CK_NL_SCATTER_GROUP = 3,  // k_nl_scatter: projector group of an entry
    CK_NL_GRAD_POINT = 4,     // k_nl_grad: grid point of a sphere entry
    CK_SELFTEST = 99,         // rsdft_gpu_selftest_check
};

#ifdef RSDFT_GPU_CHECK
__device__ __forceinline__ bool dev_check(bool ok, int site, long idx, int* err) {
    if (ok) return true;
    if (atomicCAS(err + 1, 0, site) == 0) atomicExch(err + 2, (int)idx);
    atomicAdd(err + 3, 1);
    return false;
}
#define RS_DCHECK(ok, site, idx, err) ::rsdft::dev_check((ok), (site), (long)(idx), (err))
#else
#define RS_DCHECK(ok, site, idx, err) ((void)(err), true)
#endif

// Number of this library's kernel launches since load (diagnostics).
extern long long g_kernel_launches;

// Launch one of this library's kernels and count it.
template <typename... KArgs, typename... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    ++g_kernel_launches;
    kernel<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
}

int require_init();
int require_grid();

// Opt `kernel` in to `bytes` of dynamic shared memory on the bound device.
// The record lives in the context, so a context on another device sets the
// attribute again; a size no larger than the one set already does nothing.
int set_smem_optin(const void* kernel, int bytes);

// Host scratch owned by the context (grow-only; contents undefined).
char* host_workspace(size_t bytes);

// ------------------------------------------------------------ workspace
// Named device buffer, grown (never shrunk) on demand; contents undefined.
int workspace(const char* name, size_t bytes, void** out);
template <typename T>
inline int workspace_t(const char* name, size_t count, T** out) {
    return workspace(name, count * sizeof(T), reinterpret_cast<void**>(out));
}

// ------------------------------------------------- pointer resolution
// Classify a caller pointer and the `bytes` that follow it: device memory of
// the bound device is used directly; a host pointer inside a registered
// wavefunction range maps onto its device mirror.  Returns 1 if *dev was set
// (device-visible), 0 if p is plain host memory, RSDFT_EINVAL (error set) if
// the span runs past the end of its registration or device allocation, or if
// p is device memory of another device.
int resolve(const void* p, size_t bytes, void** dev);

// Stage a small caller array onto the device (copy if host), and back.
int stage_in(const void* host_or_dev, size_t bytes, const char* wsname, void** dev);
int stage_out(void* host_or_dev, const void* dev, size_t bytes);

// Wavefunction block (ld x nb doubles) as a device pointer; copies host data
// in if the pointer is neither device memory nor registered.  *staged tells
// the caller to copy results back with wf_release.
int wf_acquire(const double* p, long ld, int nb, const char* wsname, double** dev, bool* staged,
               bool copy_in = true);
int wf_release(double* p, const double* dev, long ld, int nb, bool staged);

inline bool mode_valid(int mode) { return mode >= RSDFT_MODE_FP64 && mode <= RSDFT_MODE_MIXED_BF16X2; }

inline int div_up(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace rsdft
