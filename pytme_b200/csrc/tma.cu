// Host side of the TMA helpers: tensor-map encoding through the driver's
// cuTensorMapEncodeTiled, looked up once with cudaGetDriverEntryPointByVersion.
#include "common.cuh"
#include "tma.cuh"

namespace tmb {

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encoder() {
  static const EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault,
                                         &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (EncodeTiledFn) nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

}  // namespace

bool tensor_maps_available() { return encoder() != nullptr; }

int encode_tensor_map_u32(CUtensorMap* map, const void* base, int rank, const uint64_t* dims,
                          const uint64_t* strides, const uint32_t* box) {
  const EncodeTiledFn enc = encoder();
  TM_REQUIRE(enc, "tensor map: the driver has no cuTensorMapEncodeTiled");
  TM_REQUIRE(rank >= 1 && rank <= 5 && reinterpret_cast<uintptr_t>(base) % 16 == 0,
             "tensor map: rank %d or base address not 16-byte aligned", rank);
  cuuint64_t d[5], s[4];
  cuuint32_t b[5], e[5];
  for (int i = 0; i < rank; ++i) {
    TM_REQUIRE(dims[i] >= 1 && dims[i] <= ((uint64_t)1 << 32) && box[i] >= 1 && box[i] <= 256,
               "tensor map: dimension %d (extent %llu, box %u) out of range", i,
               (unsigned long long)dims[i], box[i]);
    d[i] = dims[i];
    b[i] = box[i];
    e[i] = 1;
    if (i + 1 < rank) {
      TM_REQUIRE(strides[i] % 16 == 0 && strides[i] < ((uint64_t)1 << 40),
                 "tensor map: stride %d (%llu bytes) not a multiple of 16", i,
                 (unsigned long long)strides[i]);
      s[i] = strides[i];
    }
  }
  TM_REQUIRE(box[0] * 4 % 16 == 0, "tensor map: inner box of %u words is not 16-byte sized",
             box[0]);
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, (cuuint32_t)rank,
                         const_cast<void*>(base), d, s, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  TM_REQUIRE(r == CUDA_SUCCESS, "tensor map: cuTensorMapEncodeTiled failed (%d)", (int)r);
  return TM_OK;
}

}  // namespace tmb
