// The library's failure path for device waits, exercised on purpose and
// without a GPU fault: every wait of the library's kernels on an mbarrier
// (a bulk copy landing, a consumer releasing a stage) is bounded, and a wait
// that runs out sets the context's error flag instead of trapping; the next
// rsdft_gpu_synchronize reports RSDFT_ETIMEOUT and clears the flag, and the
// context stays usable.  rsdft_gpu_selftest_timeout launches one CTA whose
// wait can never complete (nothing ever arrives on its mbarrier), bounded by
// an SM clock budget, so a test can check that chain end to end.
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

}  // namespace rsdft

using namespace rsdft;

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
