// Tensor memory accelerator (TMA) helpers of the tensor-core passes: tiled box copies
// between a global tensor and shared memory, contiguous bulk copies, and the mbarrier
// transaction accounting they complete on. No copy here uses cluster multicast.
#pragma once

#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>

#include <cstdint>

#include "tc_common.cuh"

namespace tmb {

// Encodes a tiled tensor map of 4-byte elements (no interleave, no swizzle, zero fill
// outside the tensor): dims[0] is the contiguous dimension, strides[i] the byte stride of
// dimension i + 1 (multiples of 16), box[i] the box extent (at most 256, box[0] * 4 a
// multiple of 16). The encoder is the driver's cuTensorMapEncodeTiled, reached through
// cudaGetDriverEntryPointByVersion. Returns TM_OK or an error status with the message set.
int encode_tensor_map_u32(CUtensorMap* map, const void* base, int rank, const uint64_t* dims,
                          const uint64_t* strides, const uint32_t* box);
// Whether the driver offers the encoder.
bool tensor_maps_available();

namespace tma {

// one arrival that also announces `bytes` of asynchronous copies completing on the barrier
__device__ __forceinline__ void arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :
               : "r"(tc::smem_u32(bar)), "r"(bytes)
               : "memory");
}
// box load at (x, y) of a 2D tensor into shared memory, completing on `bar`
__device__ __forceinline__ void load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                        uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];"
      :
      : "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y),
        "r"(tc::smem_u32(bar))
      : "memory");
}
// box load at (x, y, z) of a 3D tensor into shared memory, completing on `bar`
__device__ __forceinline__ void load_3d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                        int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];"
      :
      : "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z),
        "r"(tc::smem_u32(bar))
      : "memory");
}
// box load at (x, y, z, w) of a 4D tensor into shared memory, completing on `bar`
__device__ __forceinline__ void load_4d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                        int z, int w, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];"
      :
      : "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w),
        "r"(tc::smem_u32(bar))
      : "memory");
}
// box store from shared memory to (x, y) of a 2D tensor (bulk async-group completion)
__device__ __forceinline__ void store_2d(const CUtensorMap* map, int x, int y, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
               :
               : "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(src)
               : "memory");
}
// contiguous bulk copy global -> shared (bytes a multiple of 16, both addresses 16-byte
// aligned), completing on `bar`
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :
      : "r"(dst), "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
      : "memory");
}

}  // namespace tma
}  // namespace tmb
