// Host-side encoding of TMA tensor maps through the driver entry point (no
// link-time dependency on libcuda).
#pragma once

#include <cuda.h>

namespace rsdft {

// 4-D tiled map over a column-major array: dims[0] fastest; strides in bytes
// of dims 1..3; box in elements.  Returns RSDFT_OK or an error status.
int encode_tmap_4d(CUtensorMap* map, CUtensorMapDataType dtype, const void* base, const unsigned long long dims[4],
                   const unsigned long long strides_bytes[3], const unsigned int box[4],
                   CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_NONE);

// BF16 map with the 64-byte swizzle (tcgen05 K-major operand tiles)
inline int encode_tmap_4d_swz64(CUtensorMap* map, const void* base, const unsigned long long dims[4],
                                const unsigned long long strides_bytes[3], const unsigned int box[4]) {
    return encode_tmap_4d(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, base, dims, strides_bytes, box,
                          CU_TENSOR_MAP_SWIZZLE_64B);
}

}  // namespace rsdft
