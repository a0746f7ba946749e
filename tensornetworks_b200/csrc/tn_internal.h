// tn_internal.h -- shared host/device declarations of libtn_cuda.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/tn_cuda.h"

namespace tnb {

void set_error(const char* fmt, ...);

#define TN_CUDA_CHECK(x)                                                                       \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            ::tnb::set_error("%s:%d %s: %s", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
            return e_ == cudaErrorMemoryAllocation ? TN_OUT_OF_MEMORY : TN_CUDA_ERROR;         \
        }                                                                                      \
    } while (0)

#define TN_CHECK(x)                   \
    do {                              \
        int s_ = (x);                 \
        if (s_ != TN_OK) return s_;   \
    } while (0)

// Makes a handle's device current for the length of one C-ABI call and gives
// the calling thread its own device back on return, so that a context made on
// GPU k is used on GPU k whatever device the caller has selected.
struct DeviceGuard {
    int prev = -1;
    bool restore = false;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int dev) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != dev) {
            err = cudaSetDevice(dev);
            restore = (err == cudaSuccess);
        }
    }
    ~DeviceGuard() {
        if (restore) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};
#define TN_ON_DEVICE(dev)                                                                          \
    ::tnb::DeviceGuard tn_dev_guard_(dev);                                                         \
    do {                                                                                           \
        if (tn_dev_guard_.err != cudaSuccess) {                                                    \
            ::tnb::set_error("cannot make device %d current: %s", (int)(dev),                      \
                             cudaGetErrorString(tn_dev_guard_.err));                               \
            return TN_CUDA_ERROR;                                                                  \
        }                                                                                          \
    } while (0)

// Every launch site calls TN_LAUNCH_CHECK once per kernel launch: it checks the
// launch and counts it (tn_launch_count).
void count_launch();
unsigned long long launch_count();
#define TN_LAUNCH_CHECK()                 \
    do {                                  \
        ::tnb::count_launch();            \
        TN_CUDA_CHECK(cudaGetLastError()); \
    } while (0)

// Incremented by every device (re)allocation of a DevBuf: captured CUDA graphs
// hold raw pointers, so a graph recorded under another generation is stale.
unsigned long long alloc_generation();

// FNV-1a over raw bytes (graph-cache keys).
inline unsigned long long hash_bytes(unsigned long long h, const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ULL;
    return h;
}
template <class T> inline unsigned long long hash_val(unsigned long long h, const T& v) {
    return hash_bytes(h, &v, sizeof(T));
}
constexpr unsigned long long HASH_SEED = 1469598103934665603ULL;

// Growable device buffer (bytes); contents are not preserved on growth.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t nbytes);
    void release();
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
    ~DevBuf() { release(); }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

// Pinned host buffer for small device->host reads.
struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t nbytes);
    ~HostBuf();
};

// ---------------------------------------------------------------------------
// FP64 batched GEMM with general (split-index) addressing.
//   C(i,j) = alpha * sum_k A(i,k) B(k,j) + beta * C(i,j)
// Each index x of an operand maps to  (x % div) * s + (x / div) * sb, so a
// single GEMM can walk a contraction index that is split over two tensor
// indices (e.g. k = (w, j) for environments stored as Dw blocks).
// Two batch levels (b0, b1) with independent strides.
// ---------------------------------------------------------------------------
struct IdxMap {
    long long s = 0, sb = 0;
    int div = 1 << 30;
    __host__ __device__ long long at(int x) const {
        int q = x / div;
        return (long long)(x - q * div) * s + (long long)q * sb;
    }
};
inline IdxMap idx(long long s) { IdxMap m; m.s = s; m.sb = 0; m.div = 1 << 30; return m; }
inline IdxMap idx2(long long s, int div, long long sb) { IdxMap m; m.s = s; m.sb = sb; m.div = div; return m; }

struct GemmOperand {
    const double* ptr = nullptr;
    IdxMap mn;       // row index for A (i), column index for B (j)
    IdxMap k;        // contraction index
    long long sb0 = 0, sb1 = 0;
};
struct GemmOut {
    double* ptr = nullptr;
    IdxMap m, n;
    long long sb0 = 0, sb1 = 0;
};
struct GemmArgs {
    int M = 0, N = 0, K = 0;
    int nb0 = 1, nb1 = 1;
    double alpha = 1.0, beta = 0.0;
    GemmOperand A, B;
    GemmOut C;
    const int* skip = nullptr;  // device flag: when nonzero the launch does nothing
};
int gemm_f64(const GemmArgs& g, cudaStream_t st);

// Sparse MPO term list: out[(m,wout)] += c * in[(win,n)].
struct WTerm {
    int win, n, wout, m;
    double c;
};

// One Lanczos iteration (matvec + dots + update + next) recorded as the body
// of a conditional WHILE node: the device decides when the loop ends.
struct LzGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long kernels_per_iter = 0;
};

// Execution context (one per tn_ctx handle).
struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    // side stream for work that overlaps the main stream's critical path (QR look-ahead)
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_x[3] = {nullptr, nullptr, nullptr};
    // second side stream: the FP64 check of a site's eigenvector, overlapping the gauge move
    cudaStream_t aux2 = nullptr;
    cudaEvent_t ev_y[2] = {nullptr, nullptr};
    // refine sub-phase timing (solver verbose >= 4): device milliseconds in
    // [0] split-operator preparation, [1] restart set-up, [2] Krylov steps,
    // [3] Ritz vector; events pev, created on first use
    bool prof = false;
    cudaEvent_t pev[6] = {};
    double prof_ms[4] = {};
    long long prof_steps = 0, prof_restarts = 0;
    int prof_events();
    // scratch
    DevBuf P, Q;           // contraction intermediates
    DevBuf lz;             // Lanczos basis + work vectors
    DevBuf lzsum;          // summary of a device-driven Lanczos solve
    DevBuf lzstate;        // Lanczos device state
    DevBuf rq;             // Rayleigh-quotient state + partials
    DevBuf dv, dvstate;    // Davidson basis + work vectors, device state
    DevBuf qrw;            // QR workspace
    DevBuf qaccum;         // QR: forward-accumulated Q (transposed)
    DevBuf qrsync;         // QR: progress words of the persistent kernel
    DevBuf derr;           // sticky error word of kernels with bounded waits (zero until one expires)
    DevBuf svdw;           // SVD workspace
    DevBuf wterms;         // MPO term lists
    DevBuf misc;
    DevBuf apiw[3];        // staging copies of the dense-solver entry points
    DevBuf cqr, rr1, rr2;  // RQ / QL factor staging; rank-revealing factorisations' full factors
    HostBuf pinned;
    int sm_count = 148;
    bool use_persistent_qr = true;  // TN_NO_PERSISTENT_QR=1: the two-stream look-ahead QR instead
    bool qr_forward_q = true;       // TN_QR_FORWARD_Q=0: the persistent QR forms the thin Q after the panels
    long long qr_spin_limit = 1LL << 21;  // polls per wait in the persistent QR (TN_QR_SPIN_LIMIT)
    // cache of the last MPO term list uploaded through the C ABI
    std::vector<double> wcache_W;
    int wcache_key[4] = {0, 0, 0, 0};
    int wcache_n = 0;
    // device-looped Lanczos graphs by operator key (TN_NO_GRAPHS=1 disables)
    std::unordered_map<unsigned long long, LzGraph> lzgraphs;
    bool use_graphs = true;
    void clear_graphs();
};

}  // namespace tnb

struct tn_ctx_s {
    tnb::Ctx c;
};
