// tma_maps.h -- TMA tensor maps of the BF16 operands of the tcgen05 kernels.
#pragma once
#include <cuda.h>

#include "tn_internal.h"

namespace tnb {

// Tensor maps of up to three BF16 pieces of each operand of a GEMM.
struct TcMaps {
    CUtensorMap a[3], b[3];
};

// 3-D BF16 operand map {K, rows, batch} with box {64, box_rows, 1} and the
// 128-byte swizzle of the K-major UMMA operands.
int tc_make_map(CUtensorMap* m, const uint16_t* base, int K, int rows, int batch, long long row_pitch_elems,
                long long batch_pitch_elems, int box_rows);

}  // namespace tnb
