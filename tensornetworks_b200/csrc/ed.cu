// ed.cu -- exact diagonalisation of the open spin chain on the device: the
// FullState accelerator (FullStateImp<T>, TensorNetworksImp/FullStateImp.C).
//
// The wave function holds all d^L amplitudes, site 1 the most significant base-d
// digit of the index (StateIterator::GetIndex, StateIterator.C:64-71).  The
// Hamiltonian is the sum over the L-1 bonds of the local two-site matrix
// (ContractOverLattice / OperateLocal, FullStateImp.C:91-129):
//     y[i] = sum_b sum_{(ma,mb)} H12(ma mb, na nb) x[i with digits b, b+1 -> ma, mb]
// with (na, nb) the digits of i at the bond.  One thread forms one output
// amplitude: it walks the digits of its index once (one division per site,
// the pair of the current bond kept in registers) and gathers the nonzero
// entries of the local matrix's column (na, nb) -- a pull formulation, so
// every amplitude is written once and nothing is accumulated atomically.
// For d = 2 the digits are bits and the strides shifts.  The field term is
// hz Sz once per site (the MPO's convention, W(4,0) = hz Sz).
//
// FindGroundState runs the library's device Lanczos on this operator (the
// reference drives PRIMME through DoMatVecContraction, FullStateImp.C:207-217);
// PowerIterate restates FullStateImp::PowerIterate / OperateOverLattice
// (:60-89, :155-188).
#include "ed.h"

#include <cmath>
#include <vector>

#include "lanczos.h"

namespace tnb {

namespace {

constexpr int ED_MAXL = 63;
constexpr int ED_MAXDD = 64;  // d^2 for d <= 8

struct EdEntry {
    int r;     // row ma d + mb of the local matrix
    double v;  // its value
};

struct EdParams {
    long long N;
    int L, d, nnz_max;
    double hz, S;
    unsigned pw[ED_MAXL + 1];  // d^(L-1-b): stride of site b (0-based)
    int cnt[ED_MAXDD];         // nonzeros of column c = na d + nb
};

template <bool BITS>
__global__ void ed_matvec_kernel(const double* __restrict__ x, double* __restrict__ y, const EdParams p,
                                 const EdEntry* __restrict__ ent, const int* skip) {
    if (skip && *skip) return;
    const int d = p.d;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < p.N; t += (long long)gridDim.x * blockDim.x) {
        const unsigned i = (unsigned)t;
        unsigned rem = i;
        int dlo;
        if (BITS) { dlo = rem & 1u; rem >>= 1; }
        else { dlo = (int)(rem % (unsigned)d); rem /= (unsigned)d; }
        double acc = 0.0;
        double fz = (double)dlo - p.S;  // field of site L-1
        for (int b = p.L - 2; b >= 0; --b) {
            int dhi;
            if (BITS) { dhi = rem & 1u; rem >>= 1; }
            else { dhi = (int)(rem % (unsigned)d); rem /= (unsigned)d; }
            const unsigned s0 = p.pw[b], s1 = p.pw[b + 1];
            const unsigned base = i - (unsigned)dhi * s0 - (unsigned)dlo * s1;
            const int c = dhi * d + dlo;
            const EdEntry* e = ent + c * p.nnz_max;
            for (int k = 0; k < p.cnt[c]; ++k) {
                const EdEntry en = e[k];
                const int ma = en.r / d, mb = en.r - (en.r / d) * d;
                acc = fma(en.v, __ldg(x + base + (unsigned)ma * s0 + (unsigned)mb * s1), acc);
            }
            fz += (double)dhi - p.S;
            dlo = dhi;
        }
        if (p.hz != 0.0) acc = fma(p.hz * fz, x[i], acc);
        y[i] = acc;
    }
}

// per-block partials of: 0 = x.y, 1 = x.x, 2 = max |x - y|
__global__ void ed_reduce_kernel(const double* __restrict__ x, const double* __restrict__ y, long long n, int mode,
                                 double* __restrict__ partial) {
    __shared__ double sh[32];
    double a = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (mode == 0) a = fma(x[i], y[i], a);
        else if (mode == 1) a = fma(x[i], x[i], a);
        else a = fmax(a, fabs(x[i] - y[i]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double b = __shfl_xor_sync(0xffffffffu, a, o);
        a = mode == 2 ? fmax(a, b) : a + b;
    }
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = mode == 2 ? 0.0 : 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = mode == 2 ? fmax(t, sh[w]) : t + sh[w];
        partial[blockIdx.x] = t;
    }
}

// x[i] = alpha * y[i]   (x may alias y)
__global__ void ed_scale_kernel(double* __restrict__ x, const double* y, long long n, double alpha) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = alpha * y[i];
}

// index of the first amplitude with |a| > 0.01 (FullStateImp::Normalize, :131-149)
__global__ void ed_first_large_kernel(const double* __restrict__ x, long long n, unsigned long long* first) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (fabs(x[i]) > 0.01) {
            atomicMin(first, (unsigned long long)i);
            return;
        }
}

// uniform(-1, 1) from a counter-based hash of (seed, i) (splitmix64 finaliser)
__global__ void ed_random_kernel(double* __restrict__ x, long long n, unsigned long long seed) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        x[i] = 2.0 * ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
    }
}

double spin_sz(int m, double S) { return m - S; }
double spin_sp(int m, int n, double S) {  // <m|S+|n>
    return (m == n + 1) ? std::sqrt(S * (S + 1.0) - spin_sz(m, S) * spin_sz(n, S)) : 0.0;
}
double spin_sm(int m, int n, double S) { return spin_sp(n, m, S); }

}  // namespace

static int ed_grid(long long n, int sm) {
    long long b = (n + 255) / 256;
    const long long cap = (long long)sm * 8;
    return (int)std::max<long long>(1, std::min(b, cap));
}

int FullStateDev::init(Ctx& c, int L_, double S_, unsigned long long seed) {
    ctx = &c;
    L = L_;
    S = S_;
    d = (int)std::lround(2.0 * S + 1.0);
    if (L < 2 || L > ED_MAXL || d < 2 || d * d > ED_MAXDD) {
        set_error("full state: L = %d, d = %d out of range", L, d);
        return TN_BAD_ARG;
    }
    double n = 1.0;
    for (int i = 0; i < L; ++i) n *= d;
    if (n > 2147483647.0) {
        set_error("full state: d^L = %.0f amplitudes exceed 2^31 - 1", n);
        return TN_BAD_SHAPE;
    }
    N = (long long)n;
    TN_CHECK(amp.ensure(sizeof(double) * (size_t)N));
    TN_CHECK(work.ensure(sizeof(double) * ((size_t)N + 4096)));
    ed_random_kernel<<<ed_grid(N, c.sm_count), 256, 0, c.stream>>>(amp.as<double>(), N, seed);  // FillRandom
    TN_LAUNCH_CHECK();
    return TN_OK;
}

int FullStateDev::set_hamiltonian(double Jxy, double Jz, double hz) {
    // local bond matrix H12(ma mb, na nb) of Hamiltonian_1D_NN_Heisenberg::GetH
    // (Hamiltonian_1D_NN_Heisenberg.C:28-33) without its field part; the field
    // goes in once per site
    const int dd = d * d;
    std::vector<std::vector<EdEntry>> cols(dd);
    for (int na = 0; na < d; ++na)
        for (int nb = 0; nb < d; ++nb)
            for (int ma = 0; ma < d; ++ma)
                for (int mb = 0; mb < d; ++mb) {
                    const double v = 0.5 * Jxy * (spin_sp(ma, na, S) * spin_sm(mb, nb, S) +
                                                  spin_sm(ma, na, S) * spin_sp(mb, nb, S)) +
                                     Jz * (ma == na ? spin_sz(ma, S) : 0.0) * (mb == nb ? spin_sz(mb, S) : 0.0);
                    if (v != 0.0) cols[na * d + nb].push_back(EdEntry{ma * d + mb, v});
                }
    nnz_max = 1;
    for (auto& c : cols) nnz_max = std::max(nnz_max, (int)c.size());
    std::vector<EdEntry> flat((size_t)dd * nnz_max, EdEntry{0, 0.0});
    for (int c = 0; c < dd; ++c)
        for (size_t k = 0; k < cols[c].size(); ++k) flat[(size_t)c * nnz_max + k] = cols[c][k];
    TN_CHECK(hl.ensure(sizeof(EdEntry) * flat.size() + sizeof(int) * dd));
    TN_CUDA_CHECK(cudaMemcpyAsync(hl.p, flat.data(), sizeof(EdEntry) * flat.size(), cudaMemcpyHostToDevice, ctx->stream));
    hz_site = hz;
    cnt_.assign(dd, 0);
    for (int c = 0; c < dd; ++c) cnt_[c] = (int)cols[c].size();
    return TN_OK;
}

int FullStateDev::matvec(const double* x, double* y, const int* skip) {
    EdParams p{};
    p.N = N;
    p.L = L;
    p.d = d;
    p.nnz_max = nnz_max;
    p.hz = hz_site;
    p.S = S;
    unsigned s = 1;
    for (int b = L - 1; b >= 0; --b) {
        p.pw[b] = s;
        s *= (unsigned)d;
    }
    for (int c = 0; c < d * d; ++c) p.cnt[c] = cnt_[c];
    const int g = ed_grid(N, ctx->sm_count);
    if (d == 2) ed_matvec_kernel<true><<<g, 256, 0, ctx->stream>>>(x, y, p, hl.as<EdEntry>(), skip);
    else ed_matvec_kernel<false><<<g, 256, 0, ctx->stream>>>(x, y, p, hl.as<EdEntry>(), skip);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

// reduction over two device vectors (mode as ed_reduce_kernel), finished on the host
static int ed_reduce(Ctx& c, const double* x, const double* y, long long n, int mode, double* scratch, double* out) {
    const int g = std::min(ed_grid(n, c.sm_count), 2048);
    ed_reduce_kernel<<<g, 256, 0, c.stream>>>(x, y, n, mode, scratch);
    TN_LAUNCH_CHECK();
    std::vector<double> h(g);
    TN_CUDA_CHECK(cudaMemcpyAsync(h.data(), scratch, sizeof(double) * g, cudaMemcpyDeviceToHost, c.stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    double t = 0.0;
    for (double v : h) t = mode == 2 ? std::max(t, v) : t + v;
    *out = t;
    return TN_OK;
}

// FullStateImp::Normalize: unit norm, then the sign of the first amplitude above 0.01 made positive
static int ed_normalize(Ctx& c, double* x, long long n, double* scratch) {
    double nrm2 = 0.0;
    TN_CHECK(ed_reduce(c, x, x, n, 1, scratch, &nrm2));
    if (!(nrm2 > 0.0)) {
        set_error("full state: zero wave function");
        return TN_NAN_DETECTED;
    }
    const double inv = 1.0 / std::sqrt(nrm2);
    ed_scale_kernel<<<ed_grid(n, c.sm_count), 256, 0, c.stream>>>(x, x, n, inv);
    TN_LAUNCH_CHECK();
    unsigned long long* first = reinterpret_cast<unsigned long long*>(scratch);
    const unsigned long long none = ~0ULL;
    TN_CUDA_CHECK(cudaMemcpyAsync(first, &none, sizeof(none), cudaMemcpyHostToDevice, c.stream));
    ed_first_large_kernel<<<ed_grid(n, c.sm_count), 256, 0, c.stream>>>(x, n, first);
    TN_LAUNCH_CHECK();
    unsigned long long idx = none;
    TN_CUDA_CHECK(cudaMemcpyAsync(&idx, first, sizeof(idx), cudaMemcpyDeviceToHost, c.stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    if (idx != none) {
        double a = 0.0;
        TN_CUDA_CHECK(cudaMemcpy(&a, x + idx, sizeof(double), cudaMemcpyDeviceToHost));
        if (a < 0.0) {
            ed_scale_kernel<<<ed_grid(n, c.sm_count), 256, 0, c.stream>>>(x, x, n, -1.0);
            TN_LAUNCH_CHECK();
        }
    }
    return TN_OK;
}

int FullStateDev::find_ground_state(double epsE, int krylov, int max_restarts, double* E_out, int* matvecs) {
    Ctx& c = *ctx;
    MatvecFn mv = [&](const double* xi, double* yo, const int* skip) { return matvec(xi, yo, skip); };
    LzResult r{};
    TN_CHECK(lanczos_solve(c, N, amp.as<double>(), krylov, max_restarts, epsE, mv, &r));
    TN_CHECK(ed_normalize(c, amp.as<double>(), N, work.as<double>() + N));
    E = r.theta;
    if (E_out) *E_out = E;
    if (matvecs) *matvecs = r.matvecs;
    if (!r.converged) {
        set_error("full state: Lanczos residual %.3e above %.3e after %d restarts", r.resid, epsE, r.restarts);
        return TN_NOT_CONVERGED;
    }
    return TN_OK;
}

int FullStateDev::power_iterate(double epsE, double epsPsi, int max_iter, double* E_out, int* iters) {
    Ctx& c = *ctx;
    double* x = amp.as<double>();
    double* y = work.as<double>();
    double* scratch = y + N;
    TN_CHECK(ed_normalize(c, x, N, scratch));
    double Eprev = 0.0, dE = 0.0, dpsi = 0.0;
    int it = 1;
    for (; it < max_iter; ++it) {
        // OperateOverLattice: new = H old, E = <old|new>, new /= E, dpsi = max |new - old|, old = normalised new
        TN_CHECK(matvec(x, y, nullptr));
        double Ec = 0.0;
        TN_CHECK(ed_reduce(c, x, y, N, 0, scratch, &Ec));
        if (Ec == 0.0) {
            set_error("full state: <psi|H|psi> = 0, power iteration undefined");
            return TN_NAN_DETECTED;
        }
        ed_scale_kernel<<<ed_grid(N, c.sm_count), 256, 0, c.stream>>>(y, y, N, 1.0 / Ec);
        TN_LAUNCH_CHECK();
        TN_CHECK(ed_reduce(c, y, x, N, 2, scratch, &dpsi));
        TN_CUDA_CHECK(cudaMemcpyAsync(x, y, sizeof(double) * (size_t)N, cudaMemcpyDeviceToDevice, c.stream));
        TN_CHECK(ed_normalize(c, x, N, scratch));
        E = Ec;
        dE = std::fabs(E - Eprev);
        Eprev = E;
        if (std::fabs(dpsi) < epsPsi && dE < epsE) break;
    }
    if (E_out) *E_out = E;
    if (iters) *iters = it;
    return TN_OK;
}

}  // namespace tnb
