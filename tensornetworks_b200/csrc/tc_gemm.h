// tc_gemm.h -- BF16x3 tcgen05 batched GEMM (see tc_gemm.cu).
#pragma once
#include <cuda.h>

#include "tn_internal.h"

namespace tnb {

enum { TC_OUT_F32_ROWMAJOR = 0, TC_OUT_F64_COLMAJOR = 1, TC_OUT_F64_COLMAJOR_ACC = 2, TC_OUT_F32_COLMAJOR = 3 };

// C[b](m,n) = alpha * sum_k A[b](m,k) B[b](n,k); A rows are K-contiguous BF16 pieces
// (hi, lo[, lo2]) with row pitch lda and batch pitch a_batch (elements); same for B.
// The A batch coordinate of output batch b is (b / a_bdiv) % a_bmod, the B one
// (b / b_bdiv) % b_bmod, so an operand can repeat across part of the batch.
struct TcGemmArgs {
    int M = 0, N = 0, K = 0, batch = 1;
    int nsplit = 2;  // BF16 pieces per operand: 2 (3 products, ~16-bit) or 3 (6 products, ~24-bit)
    const uint16_t* a[3] = {nullptr, nullptr, nullptr};
    const uint16_t* b[3] = {nullptr, nullptr, nullptr};
    long long lda = 0, a_batch = 0, ldb = 0, b_batch = 0;
    int a_nbatch = 1, b_nbatch = 1;        // batch extents of the operand tensors
    int a_bdiv = 1, a_bmod = 1, b_bdiv = 1, b_bmod = 1;
    int out_mode = 0;
    float* c32 = nullptr;
    double* c64 = nullptr;
    long long ldc = 0, c_batch = 0;
    float alpha = 1.0f;
    const int* skip = nullptr;
    int* err = nullptr;
};

struct TcMaps {
    CUtensorMap a[3], b[3];
};

struct TcGemmPlan {
    TcMaps maps;
    TcGemmArgs args;
    int bn = 128;
};

// 3-D BF16 operand map {K, rows, batch} with box {64, box_rows, 1} and the
// 128-byte swizzle of the K-major UMMA operands.
int tc_make_map(CUtensorMap* m, const uint16_t* base, int K, int rows, int batch, long long row_pitch_elems,
                long long batch_pitch_elems, int box_rows);

int tc_gemm_plan(const TcGemmArgs& a, TcGemmPlan* plan);
int tc_gemm_run(const TcGemmPlan& plan, cudaStream_t st);

}  // namespace tnb
