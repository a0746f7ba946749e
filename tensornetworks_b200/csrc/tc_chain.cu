// tc_chain.cu -- segmented split-K BF16xN GEMM on the 5th-generation tensor
// cores, the building block of the fused split-precision Heff matvec.
//
//   C[ob](m, n) = sum_{s in segments(ob)} sum_k A[s.a](m, k) B[s.b](n, k)
//
// An output batch is a list of K segments (operand batch pairs); all chunks of
// all segments of one 128 x 64 output tile are dealt out to `splitk` CTAs that
// form one thread-block cluster.  Each CTA runs the usual tcgen05 pipeline on
// its chunk range (warp 0: TMA loads into a 128-byte-swizzled ring; warp 1:
// one elected thread issues the BF16 piece products into a TMEM accumulator;
// warps 2-5: tcgen05.ld of the accumulator into shared memory).  The cluster
// then reduces: CTA r sums rows [r*128/splitk, (r+1)*128/splitk) of the tile
// over the partials of all CTAs of the cluster, read through distributed
// shared memory in a fixed order (deterministic), and writes them either as
// BF16 pieces (row-major: the A operand of the next GEMM) or as FP64
// (column-major: the site-tensor layout).  No partial ever goes to HBM.
//
// Every mbarrier wait is bounded; on expiry the CTA records an error code and
// still takes both cluster barriers, so no CTA of a cluster waits for a peer
// that has left.
#include <cuda_bf16.h>

#include "pdl.cuh"
#include "tc_chain.h"
#include "tc_ptx.cuh"

namespace tnb {

namespace {

using namespace tcp;

constexpr int CBN = 64;  // output tile columns

__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(addr), "r"(rank));
    return out;
}

// Not volatile: the loads of one thread are free to overlap; the cluster
// barriers around the reduction order them against the peers' writes.
__device__ __forceinline__ float4 ld_cluster_v4(uint32_t addr) {
    float4 v;
    asm("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
    return v;
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <int NS>
struct ChainSmem {
    static constexpr int A_BYTES = BM * BK * 2;   // 16 KB per piece
    static constexpr int B_BYTES = CBN * BK * 2;  // 8 KB per piece
    static constexpr int STAGE_BYTES = NS * (A_BYTES + B_BYTES);
    static constexpr int NSTAGE = (4 * STAGE_BYTES + 1024 <= 220 * 1024) ? 4 : ((3 * STAGE_BYTES + 1024 <= 220 * 1024) ? 3 : 2);
    static constexpr int SROW = CBN + 4;  // staging row stride (floats): 16-byte rows, float4 traffic conflict-free
    static constexpr int STAGING_BYTES = BM * SROW * 4;
    static constexpr int RING = NSTAGE * STAGE_BYTES;
    static constexpr int TOTAL = (RING > STAGING_BYTES ? RING : STAGING_BYTES) + 1024;
};

template <int NS, int OUT>
__global__ void __launch_bounds__(THREADS, 1)
    tc_chain_kernel(const __grid_constant__ TcMaps maps, TcChainArgs p) {
    using SL = ChainSmem<NS>;
    constexpr int STAGES = SL::NSTAGE;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full_bar[4], empty_bar[4], accum_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int s_fail;

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float* stg = reinterpret_cast<float*>(smem);  // staging of the FP32 tile, reuses the ring
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * CBN;
    const int split = p.splitk > 1 ? (int)cluster_ctarank() : 0;
    const int ob = blockIdx.z / p.splitk;
    const int nkseg = (p.K + BK - 1) / BK;
    const int sbeg = p.seg_start[ob], send = p.seg_start[ob + 1];
    const int nchunk = (send - sbeg) * nkseg;
    const int q0 = (int)((long long)split * nchunk / p.splitk);
    const int q1 = (int)((long long)(split + 1) * nchunk / p.splitk);
    const bool has_work = q1 > q0;

    if (threadIdx.x == 32) {
        // descriptor prefetch overlaps the predecessor's tail
#pragma unroll
        for (int pc = 0; pc < NS; ++pc) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.a[pc])) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.b[pc])) : "memory");
        }
    }
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
                     "r"((uint32_t)CBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base_sh;
    // the prologue above touched nothing the predecessor writes
    pdl_launch_dependents();
    pdl_wait();
    // the flag is read by every CTA of a cluster alike, so a skipped launch leaves no peer waiting
    if (p.skip && *p.skip) {
        if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)CBN));
        return;
    }

    if (warp == 0) {
        if (lane == 0 && has_work) {
            for (int q = q0; q < q1; ++q) {
                const int it = q - q0;
                const int s = it % STAGES;
                const uint32_t ph = (it / STAGES) & 1;
                if (!mbar_wait(&empty_bar[s], ph ^ 1)) { s_fail = 1; break; }
                const TcSeg sg = p.segs[sbeg + q / nkseg];
                const int kc = q % nkseg;
                uint8_t* st = smem + s * SL::STAGE_BYTES;
                mbar_expect_tx(&full_bar[s], SL::STAGE_BYTES);
#pragma unroll
                for (int pc = 0; pc < NS; ++pc) {
                    tma_load_3d(st + pc * SL::A_BYTES, &maps.a[pc], &full_bar[s], kc * BK, m0, sg.a_batch);
                    tma_load_3d(st + NS * SL::A_BYTES + pc * SL::B_BYTES, &maps.b[pc], &full_bar[s], kc * BK, n0,
                                sg.b_batch);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && has_work) {
            constexpr uint32_t idesc = idesc_bf16(BM, CBN);
            for (int q = q0; q < q1; ++q) {
                const int it = q - q0;
                const int s = it % STAGES;
                const uint32_t ph = (it / STAGES) & 1;
                if (!mbar_wait(&full_bar[s], ph)) { s_fail = 1; break; }
                fence_after();
                const uint32_t st = smem_u32(smem + s * SL::STAGE_BYTES);
                const uint32_t a0 = st, b0 = st + NS * SL::A_BYTES;
#pragma unroll
                for (int kk = 0; kk < BK / 16; ++kk) {
                    const uint32_t off = kk * 32;
                    mma_bf16(tmem, sdesc_sw128(a0 + off), sdesc_sw128(b0 + off), idesc, (it > 0 || kk > 0) ? 1u : 0u);
#pragma unroll
                    for (int t = 1; t < NS; ++t)
#pragma unroll
                        for (int i = 0; i <= t; ++i)
                            mma_bf16(tmem, sdesc_sw128(a0 + i * SL::A_BYTES + off),
                                     sdesc_sw128(b0 + (t - i) * SL::B_BYTES + off), idesc, 1u);
                }
                mma_commit(&empty_bar[s]);
            }
            mma_commit(&accum_bar);
        }
    } else {
        // warps 2..5: TMEM lane quarter (warp % 4) = tile rows 32 q .. 32 q + 31
        const int qd = warp & 3;
        const int r = qd * 32 + lane;
        bool ok = true;
        if (has_work) ok = __all_sync(0xffffffffu, mbar_wait(&accum_bar, 0) ? 1 : 0) != 0;
        fence_after();
        if (!ok) s_fail = 1;
        float* srow = stg + r * SL::SROW;
        if (has_work && ok) {
            const uint32_t tbase = tmem + ((uint32_t)(qd * 32) << 16);
#pragma unroll
            for (int c0 = 0; c0 < CBN; c0 += 16) {
                float v[16];
                tmem_ld16(tbase + (uint32_t)c0, v);
#pragma unroll
                for (int i = 0; i < 16; i += 4)
                    *reinterpret_cast<float4*>(srow + c0 + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            }
        } else {
#pragma unroll
            for (int c = 0; c < CBN; c += 4) *reinterpret_cast<float4*>(srow + c) = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)CBN));
    }
    if (p.splitk > 1) cluster_sync_all();

    // cluster reduction of this CTA's rows and the output: work item = one row
    // and four consecutive columns; the partial of every CTA of the cluster is
    // read with one 16-byte load each (all issued before the sum), in rank order.
    const int RB = BM / p.splitk;
    const int rbase = split * RB;
    const uint32_t stg_addr = smem_u32(stg);
    constexpr int CG = CBN / 4;
    const int items = RB * CG;
    for (int e = threadIdx.x; e < items; e += THREADS) {
        int rl, cg;
        if (OUT == TCC_OUT_F64_COLMAJOR) {  // consecutive threads: consecutive rows (coalesced column writes)
            rl = rbase + e % RB;
            cg = e / RB;
        } else {                            // consecutive threads: consecutive column groups of a row
            rl = rbase + e / CG;
            cg = e % CG;
        }
        const uint32_t off = (uint32_t)((rl * SL::SROW + 4 * cg) * 4);
        float4 part[8];
#pragma unroll
        for (int pr = 0; pr < 8; ++pr)
            if (pr < p.splitk)
                part[pr] = p.splitk > 1 ? ld_cluster_v4(mapa_shared(stg_addr + off, pr))
                                        : *reinterpret_cast<const float4*>(stg + rl * SL::SROW + 4 * cg);
        const int row = m0 + rl, col0 = n0 + 4 * cg;
        if (OUT == TCC_OUT_F64_COLMAJOR) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int pr = 0; pr < 8; ++pr)
                if (pr < p.splitk) {
                    acc[0] += (double)part[pr].x;
                    acc[1] += (double)part[pr].y;
                    acc[2] += (double)part[pr].z;
                    acc[3] += (double)part[pr].w;
                }
            if (row < p.M) {
                double* dst = p.c64 + (long long)ob * p.c64_batch + row;
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (col0 + i < p.N) dst[(long long)(col0 + i) * p.ldc64] = acc[i];
            }
        } else {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int pr = 0; pr < 8; ++pr)
                if (pr < p.splitk) {
                    acc[0] += part[pr].x;
                    acc[1] += part[pr].y;
                    acc[2] += part[pr].z;
                    acc[3] += part[pr].w;
                }
            if (row < p.M) {
                uint16_t* dst = p.c16 + (long long)ob * p.c16_batch + (long long)row * p.ldc16 + col0;
                if (col0 + 4 <= p.N) {
                    // four columns per piece in one 8-byte store (row pitch and col0 are multiples of 4)
#pragma unroll
                    for (int pc = 0; pc < NS; ++pc) {
                        uint16_t h[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const __nv_bfloat16 b = __float2bfloat16_rn(acc[i]);
                            h[i] = __bfloat16_as_ushort(b);
                            acc[i] -= __bfloat162float(b);
                        }
                        uint2 w;
                        w.x = (uint32_t)h[0] | ((uint32_t)h[1] << 16);
                        w.y = (uint32_t)h[2] | ((uint32_t)h[3] << 16);
                        *reinterpret_cast<uint2*>(dst + (long long)pc * p.c16_piece) = w;
                    }
                } else {
                    for (int i = 0; i < 4 && col0 + i < p.N; ++i) {
                        float rem = acc[i];
#pragma unroll
                        for (int pc = 0; pc < NS; ++pc) {
                            const __nv_bfloat16 b = __float2bfloat16_rn(rem);
                            dst[(long long)pc * p.c16_piece + i] = __bfloat16_as_ushort(b);
                            rem -= __bfloat162float(b);
                        }
                    }
                }
            }
        }
    }
    // peers may still be reading this CTA's staging tile
    if (p.splitk > 1) cluster_sync_all();
    if (threadIdx.x == 0 && s_fail && p.err) atomicExch(p.err, 1);
}

template <int NS, int OUT>
int launch_chain(const TcChainPlan& pl, cudaStream_t st) {
    const TcChainArgs& p = pl.args;
    const int smem = ChainSmem<NS>::TOTAL;
    auto kern = tc_chain_kernel<NS, OUT>;
    TN_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((p.N + CBN - 1) / CBN, (p.M + BM - 1) / BM, p.nbatch * p.splitk);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    int na = 0;
    attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
    if (p.splitk > 1) {
        attr[na].id = cudaLaunchAttributeClusterDimension;
        attr[na].val.clusterDim.x = 1;
        attr[na].val.clusterDim.y = 1;
        attr[na].val.clusterDim.z = p.splitk;
        ++na;
    }
    cfg.attrs = attr;
    cfg.numAttrs = na;
    TN_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, pl.maps, p));
    count_launch();
    return TN_OK;
}

}  // namespace

int tc_chain_splitk(int tiles, int chunks, int sm_count) {
    int sk = 1;
    while (sk < 8 && sk * 2 <= chunks && (long long)tiles * sk * 2 <= sm_count) sk *= 2;
    return sk;
}

int tc_chain_plan(const TcChainArgs& p, TcChainPlan* plan) {
    if (p.K % 8 != 0 || p.lda % 8 != 0 || p.ldb % 8 != 0) {
        set_error("tc_chain: K and operand pitches must be multiples of 8 (K=%d)", p.K);
        return TN_BAD_SHAPE;
    }
    if (p.nsplit != 2 && p.nsplit != 3) {
        set_error("tc_chain: nsplit must be 2 or 3");
        return TN_BAD_ARG;
    }
    if (p.splitk != 1 && p.splitk != 2 && p.splitk != 4 && p.splitk != 8) {
        set_error("tc_chain: splitk must be 1, 2, 4 or 8");
        return TN_BAD_ARG;
    }
    if (!p.seg_start || !p.segs || p.nbatch < 1) {
        set_error("tc_chain: no segment table");
        return TN_BAD_ARG;
    }
    if (p.out_mode == TCC_OUT_BF16_ROWMAJOR ? !p.c16 : !p.c64) {
        set_error("tc_chain: no output buffer");
        return TN_BAD_ARG;
    }
    plan->args = p;
    for (int q = 0; q < p.nsplit; ++q) {
        TN_CHECK(tc_make_map(&plan->maps.a[q], p.a[q], p.K, p.M, p.a_nbatch, p.lda, p.a_batch, BM));
        TN_CHECK(tc_make_map(&plan->maps.b[q], p.b[q], p.K, p.N, p.b_nbatch, p.ldb, p.b_batch, CBN));
    }
    return TN_OK;
}

int tc_chain_run(const TcChainPlan& pl, cudaStream_t st) {
    const TcChainArgs& p = pl.args;
    if (p.M <= 0 || p.N <= 0 || p.K <= 0 || p.nbatch <= 0) return TN_OK;
    if (p.out_mode == TCC_OUT_BF16_ROWMAJOR)
        return p.nsplit == 3 ? launch_chain<3, TCC_OUT_BF16_ROWMAJOR>(pl, st) : launch_chain<2, TCC_OUT_BF16_ROWMAJOR>(pl, st);
    return p.nsplit == 3 ? launch_chain<3, TCC_OUT_F64_COLMAJOR>(pl, st) : launch_chain<2, TCC_OUT_F64_COLMAJOR>(pl, st);
}

}  // namespace tnb
