// Device helpers shared by the cluster kernels (eigen.cu, factor.cu):
// cluster rank and barrier, distributed-shared-memory loads, a warp sum and
// a fast reciprocal for the serial chains of the small dense factorisations.
#pragma once

#include <cstdint>

namespace rsdft {

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// all threads of all CTAs of the cluster; orders the memory writes (shared
// and global) of the cluster's threads before the barrier against their
// reads after it (release / acquire at cluster scope)
__device__ __forceinline__ void cluster_sync() {
    asm volatile(
        "barrier.cluster.arrive.release.aligned;\n"
        "barrier.cluster.wait.acquire.aligned;\n" ::
            : "memory");
}

// load of the double at the same shared-memory offset as p in CTA `rank`
__device__ __forceinline__ double dsmem_ld(const double* p, uint32_t rank) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(r) : "memory");
    return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// 1/q for normal q by Newton-Raphson iteration for the reciprocal
// (r <- r + r (1 - q r), quadratic convergence) from the PTX approximate
// reciprocal: two steps take the ~2^-22 seed past double precision (checked
// against 1/q on 7.6e7 samples spanning exponents +-1000: no difference).
// A dependent IEEE division costs ~310 cycles on B200, this ~60, and the
// serial chains below (Sturm counts, pivots, reflector scalars) are made of
// them.
__device__ __forceinline__ double rcp_nr(double q) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(q));
    r = fma(r, fma(-q, r, 1.0), r);
    return fma(r, fma(-q, r, 1.0), r);
}

}  // namespace rsdft
