// split.cuh -- FP32 values as sums of BF16 pieces, the operand form of the
// split-precision tensor-core contractions.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace tnb {

// v as ns BF16 pieces, each the rounding of what the previous ones left;
// piece q of element e at base[q * pstride + e].
__device__ __forceinline__ void split_bf16(float v, int ns, uint16_t* base, long long pstride, long long e) {
    float r = v;
    for (int q = 0; q < ns; ++q) {
        __nv_bfloat16 h = __float2bfloat16_rn(r);
        base[q * pstride + e] = __bfloat16_as_ushort(h);
        r -= __bfloat162float(h);
    }
}

// Where the producer of a split-precision matvec's input vector writes its
// pieces, so that the matvec needs no splitting launch of its own (out null:
// no pieces).
struct VecSplit {
    uint16_t* out = nullptr;
    int ns = 0;
    long long stride = 0;
};

}  // namespace tnb
