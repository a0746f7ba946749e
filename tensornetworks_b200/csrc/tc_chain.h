// tc_chain.h -- segmented split-K BF16xN GEMM on tcgen05 with a cluster
// (distributed shared memory) reduction; the two contractions of the fused
// split-precision Heff matvec.  See tc_chain.cu.
#pragma once
#include "tma_maps.h"

namespace tnb {

// One K segment of an output batch: A batch coordinate and B batch coordinate
// (each segment spans the operands' whole K extent).
struct TcSeg {
    int a_batch, b_batch;
};

enum { TCC_OUT_BF16_ROWMAJOR = 0, TCC_OUT_F64_COLMAJOR = 1 };

// C[ob](m, n) = sum_{segments s of ob} sum_k A[s.a_batch](m, k) B[s.b_batch](n, k)
// with both operands K-major BF16 pieces (nsplit of them: products i + j < nsplit).
// The chunks of an output tile are split over `splitk` CTAs of one cluster and
// their FP32 partials summed through distributed shared memory; the sum is
// written as nsplit BF16 pieces (row-major, for the next GEMM's A operand) or
// as FP64 (column-major).
struct TcChainArgs {
    int M = 0, N = 0, K = 0;
    int nbatch = 1;
    int splitk = 1;  // 1, 2, 4 or 8
    int nsplit = 2;
    const uint16_t* a[3] = {nullptr, nullptr, nullptr};
    const uint16_t* b[3] = {nullptr, nullptr, nullptr};
    long long lda = 0, a_batch = 0, ldb = 0, b_batch = 0;
    int a_nbatch = 1, b_nbatch = 1;
    const int* seg_start = nullptr;  // device array, nbatch + 1 entries
    const TcSeg* segs = nullptr;     // device array
    int out_mode = TCC_OUT_F64_COLMAJOR;
    uint16_t* c16 = nullptr;         // BF16 pieces: piece q at c16 + q * c16_piece
    long long c16_piece = 0, ldc16 = 0, c16_batch = 0;
    double* c64 = nullptr;
    long long ldc64 = 0, c64_batch = 0;
    const int* skip = nullptr;
    int* err = nullptr;
};

struct TcChainPlan {
    TcMaps maps;
    TcChainArgs args;
};

// Split-K factor that fills the SMs: the smallest power of two (at most 8 and
// at most the chunks of a tile) with tiles * splitk >= sm_count.
int tc_chain_splitk(int tiles, int chunks, int sm_count);
int tc_chain_plan(const TcChainArgs& a, TcChainPlan* plan);
int tc_chain_run(const TcChainPlan& plan, cudaStream_t st);

}  // namespace tnb
