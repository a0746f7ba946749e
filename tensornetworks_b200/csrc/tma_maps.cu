// tma_maps.cu -- TMA tensor maps of the BF16 operands of the tcgen05 kernels.
#include <cuda.h>

#include <cstdint>

#include "tma_maps.h"

namespace tnb {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 3-D BF16 operand map {K, rows, batch}, box {64, box_rows, 1}, 128-byte swizzle.
int tc_make_map(CUtensorMap* m, const uint16_t* base, int K, int rows, int batch, long long row_pitch_elems,
                long long batch_pitch_elems, int box_rows) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) {
        set_error("cuTensorMapEncodeTiled unavailable");
        return TN_CUDA_ERROR;
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_pitch_elems * 2) % 16 || (batch_pitch_elems * 2) % 16) {
        set_error("tma map: operand not 16-byte aligned (pitch %lld)", row_pitch_elems);
        return TN_BAD_SHAPE;
    }
    cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)batch};
    cuuint64_t strides[2] = {(cuuint64_t)(row_pitch_elems * 2), (cuuint64_t)(batch_pitch_elems * 2)};
    if (batch == 1) strides[1] = strides[0] * (cuuint64_t)rows;
    cuuint32_t box[3] = {64u, (cuuint32_t)box_rows, 1};  // 64 BF16 = one 128-byte swizzle row
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<uint16_t*>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return TN_CUDA_ERROR;
    }
    return TN_OK;
}

}  // namespace tnb
