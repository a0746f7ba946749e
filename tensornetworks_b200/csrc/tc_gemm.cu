// tc_gemm.cu -- split-precision (BF16x3) batched GEMM on the 5th-generation
// tensor cores (tcgen05) for the mixed-precision Heff contractions.
//
//   C[b](m, n) = sum_k A[b](m, k) B[b](n, k)         (both operands K-major)
//   with A = A_hi + A_lo, B = B_hi + B_lo (BF16 pairs) and
//   C ~= A_hi B_hi + A_hi B_lo + A_lo B_hi         (FP32 accumulation in TMEM)
//
// One CTA computes one 128 x BN output tile.  Warp 0 streams the four operand
// tiles of each 64-wide K chunk into a 3-stage shared-memory ring with TMA
// (128-byte swizzle); warp 1 allocates the TMEM accumulator and one elected
// thread issues 3 x 4 tcgen05.mma (K = 16 each) per chunk, releasing a stage
// with tcgen05.commit; warps 2-5 read the accumulator back with tcgen05.ld
// and write the tile (FP32 row-major or FP64 column-major).  Every mbarrier
// wait is bounded: on expiry the kernel records an error code and returns.
#include <cuda.h>

#include <cstdint>

#include "tc_gemm.h"
#include "pdl.cuh"
#include "tc_ptx.cuh"

namespace tnb {

namespace {

using namespace tcp;

template <int BN, int NS>
struct SmemLayout {
    static constexpr int A_BYTES = BM * BK * 2;  // 16 KB per piece
    static constexpr int B_BYTES = BN * BK * 2;
    static constexpr int STAGE_BYTES = NS * A_BYTES + NS * B_BYTES;
    static constexpr int NSTAGE = (3 * STAGE_BYTES + 1024 <= 220 * 1024) ? 3 : 2;
    static constexpr int TOTAL = NSTAGE * STAGE_BYTES + 1024;  // + alignment slack
};

template <int BN, int NS>
__global__ void __launch_bounds__(THREADS, 1)
    tc_gemm_bf16x3_kernel(const __grid_constant__ TcMaps maps, TcGemmArgs p) {
    using SL = SmemLayout<BN, NS>;
    constexpr int STAGES = SL::NSTAGE;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full_bar[3], empty_bar[3], accum_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int s_fail;

    pdl_wait();
    if (p.skip && *p.skip) return;

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN, b = blockIdx.z;
    const int nk = (p.K + BK - 1) / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(&accum_bar, 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"((uint32_t)BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0) {
        if (lane == 0) {
            const int ab = (b / p.a_bdiv) % p.a_bmod;
            const int bb = (b / p.b_bdiv) % p.b_bmod;
            for (int kc = 0; kc < nk; ++kc) {
                const int s = kc % STAGES;
                const uint32_t ph = (kc / STAGES) & 1;
                if (!mbar_wait(&empty_bar[s], ph ^ 1)) { s_fail = 1; break; }
                uint8_t* st = smem + s * SL::STAGE_BYTES;
                mbar_expect_tx(&full_bar[s], SL::STAGE_BYTES);
#pragma unroll
                for (int q = 0; q < NS; ++q) {
                    tma_load_3d(st + q * SL::A_BYTES, &maps.a[q], &full_bar[s], kc * BK, m0, ab);
                    tma_load_3d(st + NS * SL::A_BYTES + q * SL::B_BYTES, &maps.b[q], &full_bar[s], kc * BK, n0, bb);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(BM, BN);
            bool ok = true;
            for (int kc = 0; kc < nk && ok; ++kc) {
                const int s = kc % STAGES;
                const uint32_t ph = (kc / STAGES) & 1;
                if (!mbar_wait(&full_bar[s], ph)) { s_fail = 1; ok = false; break; }
                fence_after();
                const uint32_t st = smem_u32(smem + s * SL::STAGE_BYTES);
                const uint32_t a0 = st, bq0 = st + NS * SL::A_BYTES;
#pragma unroll
                for (int kk = 0; kk < BK / 16; ++kk) {
                    const uint32_t off = kk * 32;  // 16 BF16 = 32 bytes along K inside the swizzle row
                    const uint32_t acc0 = (kc > 0 || kk > 0) ? 1u : 0u;
                    // products (i, j) of A piece i and B piece j with i + j < NS (hi*hi first)
                    mma_bf16(tmem, sdesc_sw128(a0 + off), sdesc_sw128(bq0 + off), idesc, acc0);
#pragma unroll
                    for (int t = 1; t < NS; ++t)
#pragma unroll
                        for (int i = 0; i <= t; ++i) {
                            const int j = t - i;
                            mma_bf16(tmem, sdesc_sw128(a0 + i * SL::A_BYTES + off),
                                     sdesc_sw128(bq0 + j * SL::B_BYTES + off), idesc, 1u);
                        }
                }
                mma_commit(&empty_bar[s]);
            }
            mma_commit(&accum_bar);
        }
    } else {
        // epilogue: warps 2..5 cover TMEM lane quarters (warp % 4)
        const int q = warp & 3;
        const int row = m0 + q * 32 + lane;
        // warp-uniform outcome: tcgen05.ld below is a warp-collective instruction
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&accum_bar, 0) ? 1 : 0) != 0;
        fence_after();
        if (!ok) {
            s_fail = 1;
        } else {
            const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16);
            for (int c0 = 0; c0 < BN; c0 += 16) {
                float v[16];
                tmem_ld16(tbase + (uint32_t)c0, v);
                if (row < p.M) {
                    if (p.out_mode == TC_OUT_F32_COLMAJOR) {
                        float* dst = p.c32 + (long long)b * p.c_batch + row;
#pragma unroll
                        for (int i = 0; i < 16; ++i) {
                            const int col = n0 + c0 + i;
                            if (col < p.N) dst[(long long)col * p.ldc] = v[i] * p.alpha;
                        }
                    } else if (p.out_mode == TC_OUT_F32_ROWMAJOR) {
                        float* dst = p.c32 + (long long)b * p.c_batch + (long long)row * p.ldc + n0 + c0;
                        if (n0 + c0 + 16 <= p.N && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
                            // a thread owns a row: 16-byte stores (a quarter of the transactions)
#pragma unroll
                            for (int i = 0; i < 16; i += 4)
                                *reinterpret_cast<float4*>(dst + i) = make_float4(v[i] * p.alpha, v[i + 1] * p.alpha,
                                                                                  v[i + 2] * p.alpha, v[i + 3] * p.alpha);
                        } else {
#pragma unroll
                            for (int i = 0; i < 16; ++i)
                                if (n0 + c0 + i < p.N) dst[i] = v[i] * p.alpha;
                        }
                    } else {
                        double* dst = p.c64 + (long long)b * p.c_batch + row;
#pragma unroll
                        for (int i = 0; i < 16; ++i) {
                            const int col = n0 + c0 + i;
                            if (col < p.N) {
                                double o = (double)v[i] * p.alpha;
                                if (p.out_mode == TC_OUT_F64_COLMAJOR_ACC) o += dst[(long long)col * p.ldc];
                                dst[(long long)col * p.ldc] = o;
                            }
                        }
                    }
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
    }
    if (threadIdx.x == 0 && s_fail && p.err) atomicExch(p.err, 1);
}

}  // namespace

// ---- tensor maps --------------------------------------------------------------
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
        set_error("tc_gemm: operand not 16-byte aligned (pitch %lld)", row_pitch_elems);
        return TN_BAD_SHAPE;
    }
    cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)batch};
    cuuint64_t strides[2] = {(cuuint64_t)(row_pitch_elems * 2), (cuuint64_t)(batch_pitch_elems * 2)};
    if (batch == 1) strides[1] = strides[0] * (cuuint64_t)rows;
    cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, 1};
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


int tc_gemm_plan(const TcGemmArgs& p, TcGemmPlan* plan) {
    if (p.K % 8 != 0 || p.lda % 8 != 0 || p.ldb % 8 != 0) {
        set_error("tc_gemm: K and operand pitches must be multiples of 8 (K=%d)", p.K);
        return TN_BAD_SHAPE;
    }
    if (p.a_bmod > p.a_nbatch || p.b_bmod > p.b_nbatch) {
        set_error("tc_gemm: batch coordinate exceeds the operand batch extent");
        return TN_BAD_SHAPE;
    }
    if (p.nsplit != 2 && p.nsplit != 3) {
        set_error("tc_gemm: nsplit must be 2 or 3");
        return TN_BAD_ARG;
    }
    plan->args = p;
    const long long tiles128 = (long long)((p.N + 127) / 128) * ((p.M + BM - 1) / BM) * p.batch;
    plan->bn = (p.N <= 64 || tiles128 < 148) ? 64 : 128;
    for (int q = 0; q < p.nsplit; ++q) {
        TN_CHECK(tc_make_map(&plan->maps.a[q], p.a[q], p.K, p.M, p.a_nbatch, p.lda, p.a_batch, BM));
        TN_CHECK(tc_make_map(&plan->maps.b[q], p.b[q], p.K, p.N, p.b_nbatch, p.ldb, p.b_batch, plan->bn));
    }
    return TN_OK;
}

template <int BN, int NS>
static int launch_tc(const TcGemmPlan& pl, cudaStream_t st) {
    const TcGemmArgs& p = pl.args;
    dim3 grid((p.N + BN - 1) / BN, (p.M + BM - 1) / BM, p.batch);
    const int smem = SmemLayout<BN, NS>::TOTAL;
    TN_CUDA_CHECK(cudaFuncSetAttribute(tc_gemm_bf16x3_kernel<BN, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return launch_pdl(tc_gemm_bf16x3_kernel<BN, NS>, grid, dim3(THREADS), (size_t)smem, st, pl.maps, p);
}

int tc_gemm_run(const TcGemmPlan& pl, cudaStream_t st) {
    const TcGemmArgs& p = pl.args;
    if (p.M <= 0 || p.N <= 0 || p.K <= 0 || p.batch <= 0) return TN_OK;
    if (pl.bn == 64) return p.nsplit == 3 ? launch_tc<64, 3>(pl, st) : launch_tc<64, 2>(pl, st);
    return p.nsplit == 3 ? launch_tc<128, 3>(pl, st) : launch_tc<128, 2>(pl, st);
}

}  // namespace tnb
