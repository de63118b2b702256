// The library's failure path for device waits, exercised on purpose and
// without a GPU fault: every wait of the library's kernels on an mbarrier
// (a bulk copy landing, a consumer releasing a stage) is bounded, and a wait
// that runs out sets the context's error flag instead of trapping; the next
// rsdft_gpu_synchronize reports RSDFT_ETIMEOUT and clears the flag, and the
// context stays usable.  rsdft_gpu_selftest_timeout launches one CTA whose
// wait can never complete (nothing ever arrives on its mbarrier), bounded by
// an SM clock budget, so a test can check that chain end to end.
// rsdft_gpu_selftest_check does the same for the debug build's index checks.
#include "common.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace rsdft {

__global__ void k_wait_for_nothing(long long cycles, int* __restrict__ err) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        bool done = false;
        const long long t0 = clock64();
        while (!done && clock64() - t0 < cycles) done = mbar_try_wait(&bar, 0);
        if (!done) atomicExch(err, 3);
    }
}

#ifdef RSDFT_GPU_CHECK
// Reads buf[i] only where the debug build's index check passes; i = n is
// out of range, so the check records itself and the read is skipped.
__global__ void k_check_probe(const double* __restrict__ buf, int n, int i, double* __restrict__ out,
                              int* __restrict__ err) {
    double v = 0.0;
    if (RS_DCHECK(i >= 0 && i < n, CK_SELFTEST, i, err)) v = buf[i];
    out[0] = v;
}
#endif

}  // namespace rsdft

using namespace rsdft;

extern "C" int rsdft_gpu_checked_build(void) {
#ifdef RSDFT_GPU_CHECK
    return 1;
#else
    return 0;
#endif
}

extern "C" int rsdft_gpu_selftest_check(void) {
    RS_ENTRY();
    RS_CHECK(require_init());
#ifdef RSDFT_GPU_CHECK
    constexpr int n = 4;
    double* buf = nullptr;
    RS_CHECK(workspace_t("selftest_check", n + 1, &buf));
    RS_CUDA(cudaMemsetAsync(buf, 0, sizeof(double) * (n + 1), ctx().stream));
    // the kernel writes its result one past the n-element buffer it checks
    launch(k_check_probe, 1, 1, 0, ctx().stream, (const double*)buf, n, n, buf + n, ctx().err_flag);
    RS_LAUNCH();
    return RSDFT_OK;
#else
    set_error("selftest_check: this library is not the debug build (RSDFT_GPU_CHECK)");
    return RSDFT_EUNSUP;
#endif
}

extern "C" int rsdft_gpu_selftest_timeout(long long cycles) {
    RS_ENTRY();
    RS_CHECK(require_init());
    if (cycles < 1 || cycles > (1LL << 34)) {
        set_error("selftest_timeout: cycles %lld outside 1 .. 2^34", cycles);
        return RSDFT_EINVAL;
    }
    launch(k_wait_for_nothing, 1, 32, 0, ctx().stream, cycles, ctx().err_flag);
    RS_LAUNCH();
    return RSDFT_OK;
}
