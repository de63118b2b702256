// 16-byte vector view of a scalar type: double2 for double, float4 for float.
#pragma once

#include <cuda_runtime.h>

namespace rsdft {

template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
    using t = double2;
    __device__ static __forceinline__ void get(const t& v, double* o) {
        o[0] = v.x;
        o[1] = v.y;
    }
    __device__ static __forceinline__ t make(const double* o) { return make_double2(o[0], o[1]); }
};
template <>
struct Vec16<float> {
    using t = float4;
    __device__ static __forceinline__ void get(const t& v, float* o) {
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    }
    __device__ static __forceinline__ t make(const float* o) { return make_float4(o[0], o[1], o[2], o[3]); }
};

}  // namespace rsdft
