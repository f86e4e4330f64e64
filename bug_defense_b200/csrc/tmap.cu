// Tensor-map encoding for the TMA-fed stencil kernels.
#include <cuda.h>

#include "tma.cuh"

namespace bd {

// cuTensorMapEncodeTiled is a driver-API entry point; it is looked up through the runtime so the
// library does not link libcuda directly (it loads on machines without a driver, for the ABI checks).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
        cudaGetLastError();
    }
    return fn;
}

bool make_tmap_3d_f32(CUtensorMap* out, const void* base, int nx, int ny, int nz, int bz, int by, int bx) {
    if (nz % 4 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
    cuuint64_t strides[2] = {(cuuint64_t)nz * sizeof(float), (cuuint64_t)ny * nz * sizeof(float)};
    cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, (cuuint32_t)bx};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool make_tmap_3d_u8(CUtensorMap* out, const void* base, int nx, int ny, int nz, int pitch, int bz, int by, int bx) {
    if (pitch % 16 != 0 || pitch < nz || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
    cuuint64_t strides[2] = {(cuuint64_t)pitch, (cuuint64_t)ny * pitch};
    cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, (cuuint32_t)bx};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace bd
