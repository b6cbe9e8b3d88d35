#include "host_util.h"

#include <mutex>

namespace dcvc {

int num_sms()
{
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        return 148;
    }
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
            n = 148;
        }
        cache[dev] = n;
    }
    return cache[dev];
}

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn get_encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<EncodeTiledFn>(p);
        }
    });
    return fn;
}

}  // namespace

bool make_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, const void* base, uint64_t inner,
                  uint64_t outer, uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer,
                  int swizzle_bytes)
{
    EncodeTiledFn fn = get_encode_fn();
    if (fn == nullptr) {
        return false;
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (row_bytes & 15) != 0) {
        return false;
    }
    CUtensorMapSwizzle sw;
    switch (swizzle_bytes) {
    case 128: sw = CU_TENSOR_MAP_SWIZZLE_128B; break;
    case 64: sw = CU_TENSOR_MAP_SWIZZLE_64B; break;
    case 32: sw = CU_TENSOR_MAP_SWIZZLE_32B; break;
    case 0: sw = CU_TENSOR_MAP_SWIZZLE_NONE; break;
    default: return false;
    }
    const uint32_t esz = dtype == CU_TENSOR_MAP_DATA_TYPE_UINT8 ? 1u
                         : (dtype == CU_TENSOR_MAP_DATA_TYPE_FLOAT32 || dtype == CU_TENSOR_MAP_DATA_TYPE_INT32) ? 4u
                                                                                                              : 2u;
    if (box_inner * esz > static_cast<uint32_t>(swizzle_bytes == 0 ? 256 : swizzle_bytes)) {
        return false;  // the inner box extent must fit the swizzle span
    }
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {row_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t estride[2] = {1, 1};
    CUresult r = fn(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estride,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace dcvc
