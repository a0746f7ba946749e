// capi.cu -- the extern "C" boundary declared in include/tn_cuda.h.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <cstdlib>
#include <string>

#include "engine.h"
#include "mixed.h"
#include "itebd.h"
#include "ed.h"

namespace tnb {

static thread_local std::string g_last_error;
static unsigned long long g_launches = 0;

void count_launch() { __atomic_fetch_add(&g_launches, 1ULL, __ATOMIC_RELAXED); }
unsigned long long launch_count() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

static unsigned long long g_alloc_gen = 0;
unsigned long long alloc_generation() { return __atomic_load_n(&g_alloc_gen, __ATOMIC_RELAXED); }

void Ctx::clear_graphs() {
    for (auto& kv : lzgraphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    lzgraphs.clear();
}

int Ctx::prof_events() {
    for (auto& e : pev)
        if (!e) TN_CUDA_CHECK(cudaEventCreate(&e));
    return TN_OK;
}

int DevBuf::ensure(size_t nbytes) {
    if (nbytes <= bytes && p) return TN_OK;
    release();
    if (nbytes == 0) nbytes = 8;
    __atomic_fetch_add(&g_alloc_gen, 1ULL, __ATOMIC_RELAXED);
    cudaError_t e = cudaMalloc(&p, nbytes);
    if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        set_error("cudaMalloc(%zu): %s", nbytes, cudaGetErrorString(e));
        return TN_OUT_OF_MEMORY;
    }
    bytes = nbytes;
    return TN_OK;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

int HostBuf::ensure(size_t nbytes) {
    if (nbytes <= bytes && p) return TN_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMallocHost(&p, nbytes);
    if (e != cudaSuccess) {
        set_error("cudaMallocHost(%zu): %s", nbytes, cudaGetErrorString(e));
        return TN_OUT_OF_MEMORY;
    }
    bytes = nbytes;
    return TN_OK;
}

HostBuf::~HostBuf() {
    if (p) cudaFreeHost(p);
}

}  // namespace tnb

using namespace tnb;

namespace {

// Term list of a host W on the device; the last upload is cached per context so
// repeated calls with the same W (a Krylov loop) add no copy and no sync.
int upload_terms(Ctx& c, const double* W_host, int d, int Dw1, int Dw2, bool lr, const WTermDev** out, int* n) {
    const size_t nw = (size_t)Dw1 * Dw2 * d * d;
    const int key[4] = {d, Dw1, Dw2, lr ? 1 : 0};
    if (c.wcache_n > 0 && std::memcmp(key, c.wcache_key, sizeof(key)) == 0 && c.wcache_W.size() == nw &&
        std::memcmp(c.wcache_W.data(), W_host, nw * sizeof(double)) == 0) {
        *out = c.wterms.as<WTermDev>();
        *n = c.wcache_n;
        return TN_OK;
    }
    auto t = build_terms(W_host, d, Dw1, Dw2, lr);
    TN_CHECK(c.wterms.ensure(sizeof(WTermDev) * t.size()));
    TN_CUDA_CHECK(cudaMemcpyAsync(c.wterms.p, t.data(), sizeof(WTermDev) * t.size(), cudaMemcpyHostToDevice, c.stream));
    // the host vector dies at return: wait for the copy
    TN_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    c.wcache_W.assign(W_host, W_host + nw);
    std::memcpy(c.wcache_key, key, sizeof(key));
    c.wcache_n = (int)t.size();
    *out = c.wterms.as<WTermDev>();
    *n = (int)t.size();
    return TN_OK;
}

bool valid_shape(int d, int Dw1, int Dw2, int D1, int D2) {
    return d >= 1 && Dw1 >= 1 && Dw2 >= 1 && D1 >= 1 && D2 >= 1;
}

}  // namespace

extern "C" {

const char* tn_status_string(int s) {
    switch (s) {
        case TN_OK: return "TN_OK";
        case TN_NOT_CONVERGED: return "TN_NOT_CONVERGED";
        case TN_BAD_SHAPE: return "TN_BAD_SHAPE";
        case TN_NAN_DETECTED: return "TN_NAN_DETECTED";
        case TN_CUDA_ERROR: return "TN_CUDA_ERROR";
        case TN_BAD_ARG: return "TN_BAD_ARG";
        case TN_NO_DEVICE: return "TN_NO_DEVICE";
        case TN_OUT_OF_MEMORY: return "TN_OUT_OF_MEMORY";
    }
    return "TN_UNKNOWN";
}

const char* tn_last_error(void) { return tnb::g_last_error.c_str(); }

int tn_ctx_create(int device, tn_ctx* out) {
    if (!out) return TN_BAD_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) {
        set_error("no CUDA device %d", device);
        return TN_NO_DEVICE;
    }
    cudaDeviceProp prop;
    TN_CUDA_CHECK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        set_error("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
        return TN_NO_DEVICE;
    }
    TN_ON_DEVICE(device);
    tn_ctx c = new tn_ctx_s();
    c->c.device = device;
    c->c.sm_count = prop.multiProcessorCount;
    if (const char* ng = std::getenv("TN_NO_GRAPHS")) c->c.use_graphs = !(ng[0] == '1');
    if (const char* np = std::getenv("TN_NO_PERSISTENT_QR")) c->c.use_persistent_qr = !(np[0] == '1');
    if (const char* fq = std::getenv("TN_QR_FORWARD_Q")) c->c.qr_forward_q = (fq[0] != '0');
    if (const char* sl = std::getenv("TN_QR_SPIN_LIMIT")) c->c.qr_spin_limit = std::max(1LL, std::atoll(sl));
    TN_CUDA_CHECK(cudaStreamCreateWithFlags(&c->c.own_stream, cudaStreamNonBlocking));
    c->c.stream = c->c.own_stream;
    TN_CUDA_CHECK(cudaStreamCreateWithFlags(&c->c.aux, cudaStreamNonBlocking));
    for (auto& e : c->c.ev_x) TN_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    TN_CUDA_CHECK(cudaStreamCreateWithFlags(&c->c.aux2, cudaStreamNonBlocking));
    for (auto& e : c->c.ev_y) TN_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    TN_CUDA_CHECK(cudaEventCreate(&c->c.ev_a));
    TN_CUDA_CHECK(cudaEventCreate(&c->c.ev_b));
    *out = c;
    return TN_OK;
}

int tn_ctx_destroy(tn_ctx c) {
    if (!c) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    cudaStreamSynchronize(c->c.stream);
    c->c.clear_graphs();
    if (c->c.aux) cudaStreamSynchronize(c->c.aux);
    if (c->c.aux2) cudaStreamSynchronize(c->c.aux2);
    for (auto& e : c->c.ev_x)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->c.ev_y)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->c.pev)
        if (e) cudaEventDestroy(e);
    if (c->c.aux) cudaStreamDestroy(c->c.aux);
    if (c->c.aux2) cudaStreamDestroy(c->c.aux2);
    if (c->c.ev_a) cudaEventDestroy(c->c.ev_a);
    if (c->c.ev_b) cudaEventDestroy(c->c.ev_b);
    if (c->c.own_stream) cudaStreamDestroy(c->c.own_stream);
    delete c;
    return TN_OK;
}

int tn_ctx_set_stream(tn_ctx c, void* stream) {
    if (!c) return TN_BAD_ARG;
    c->c.stream = stream ? (cudaStream_t)stream : c->c.own_stream;
    return TN_OK;
}

int tn_ctx_synchronize(tn_ctx c) {
    if (!c) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    TN_CUDA_CHECK(cudaStreamSynchronize(c->c.stream));
    return TN_OK;
}

// ---- Hamiltonian ---------------------------------------------------------------
int tn_hamiltonian_create_heisenberg(tn_ctx c, int L, double S, int form, double Jxy, double Jz, double hz,
                                     tn_hamiltonian* out) {
    if (!c || !out) return TN_BAD_ARG;
    *out = nullptr;
    double twoS = 2.0 * S;
    if (L < 2 || S <= 0 || std::fabs(twoS - std::round(twoS)) > 1e-12) {
        set_error("bad L=%d or S=%g", L, S);
        return TN_BAD_ARG;
    }
    if (form != TN_FORM_REGULAR_LOWER && form != TN_FORM_REGULAR_UPPER) {
        set_error("unsupported MPO form %d", form);
        return TN_BAD_ARG;
    }
    if (std::fabs(Jxy) + std::fabs(Jz) <= 0.0) {  // Hamiltonian_1D_NN_Heisenberg.C:18
        set_error("Jxy and Jz both zero");
        return TN_BAD_ARG;
    }
    TN_ON_DEVICE(c->c.device);
    tn_hamiltonian h = new tn_hamiltonian_s();
    h->h.ctx = &c->c;
    h->h.L = L;
    h->h.S = S;
    h->h.d = (int)std::lround(twoS + 1.0);
    h->h.form = form;
    h->h.Jxy = Jxy;
    h->h.Jz = Jz;
    h->h.hz = hz;
    int s = h->h.build();
    if (s != TN_OK) {
        delete h;
        return s;
    }
    *out = h;
    return TN_OK;
}

int tn_hamiltonian_destroy(tn_hamiltonian h) {
    if (!h) return TN_BAD_ARG;
    TN_ON_DEVICE(h->h.ctx->device);
    delete h;
    return TN_OK;
}

int tn_hamiltonian_site_dims(tn_hamiltonian h, int site, int* Dw1, int* Dw2, int* d) {
    if (!h || site < 1 || site > h->h.L) return TN_BAD_ARG;
    if (Dw1) *Dw1 = h->h.ops[site].Dw1;
    if (Dw2) *Dw2 = h->h.ops[site].Dw2;
    if (d) *d = h->h.d;
    return TN_OK;
}

int tn_hamiltonian_h2_dims(tn_hamiltonian h, int site, int* Dw1, int* Dw2) {
    if (!h || site < 1 || site > h->h.L) return TN_BAD_ARG;
    if (Dw1) *Dw1 = h->h.ops2[site].Dw1;
    if (Dw2) *Dw2 = h->h.ops2[site].Dw2;
    return TN_OK;
}

int tn_hamiltonian_get_w(tn_hamiltonian h, int site, double* W) {
    if (!h || !W || site < 1 || site > h->h.L) return TN_BAD_ARG;
    const auto& w = h->h.ops[site].W;
    std::memcpy(W, w.data(), sizeof(double) * w.size());
    return TN_OK;
}

// ---- MPS --------------------------------------------------------------------------
int tn_mps_create(tn_hamiltonian h, int D, double normEps, double epsSV, tn_mps* out) {
    if (!h || !out || D < 1) return TN_BAD_ARG;
    *out = nullptr;
    TN_ON_DEVICE(h->h.ctx->device);
    tn_mps m = new tn_mps_s();
    m->m.normEps = normEps;
    m->m.epsSV = epsSV;
    int s = m->m.init(&h->h, D);
    if (s != TN_OK) {
        delete m;
        return s;
    }
    *out = m;
    return TN_OK;
}

int tn_mps_destroy(tn_mps m) {
    if (!m) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    cudaStreamSynchronize(m->m.ctx->stream);
    delete m;
    return TN_OK;
}

int tn_mps_initialize_random(tn_mps m, uint64_t seed) {
    if (!m) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    return m->m.initialize_random(seed);
}

int tn_mps_get_site_dims(tn_mps m, int site, int* D1, int* D2) {
    if (!m || site < 1 || site > m->m.L) return TN_BAD_ARG;
    if (D1) *D1 = m->m.D1[site];
    if (D2) *D2 = m->m.D2[site];
    return TN_OK;
}

int tn_mps_get_site(tn_mps m, int site, double* A) {
    if (!m || !A || site < 1 || site > m->m.L) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    auto& s = m->m;
    TN_CUDA_CHECK(cudaStreamSynchronize(s.ctx->stream));
    TN_CUDA_CHECK(cudaMemcpy(A, s.A[site]->p, sizeof(double) * (size_t)s.d * s.D1[site] * s.D2[site],
                             cudaMemcpyDeviceToHost));
    return TN_OK;
}

int tn_mps_set_site(tn_mps m, int site, int D1, int D2, const double* A) {
    if (!m || !A || site < 1 || site > m->m.L || D1 < 1 || D2 < 1) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    auto& s = m->m;
    TN_CHECK(s.ensure_capacity(std::max(D1, D2)));
    TN_CUDA_CHECK(cudaStreamSynchronize(s.ctx->stream));
    TN_CUDA_CHECK(cudaMemcpy(s.A[site]->p, A, sizeof(double) * (size_t)s.d * D1 * D2, cudaMemcpyHostToDevice));
    s.D1[site] = D1;
    s.D2[site] = D2;
    // a new shape changes the adjacent bonds' dimensions (Bond::NewBondDimension)
    if (site > 1 && s.bondK[site - 1] != D1) s.set_bond_dim(site - 1, D1);
    if (site < s.L && s.bondK[site] != D2) s.set_bond_dim(site, D2);
    return TN_OK;
}

int tn_mps_get_bond(tn_mps m, int bond, int* D, double* s_host) {
    if (!m || bond < 1 || bond >= m->m.L) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    TN_CHECK(m->m.ensure_bond_values());
    const auto& s = m->m.bond_s[bond];
    if (D) *D = (int)s.size();
    if (s_host) std::memcpy(s_host, s.data(), sizeof(double) * s.size());
    return TN_OK;
}

int tn_mps_normalize(tn_mps m, int direction) {
    if (!m) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    TN_CHECK(m->m.normalize_all(direction == TN_DLEFT));
    TN_CUDA_CHECK(cudaStreamSynchronize(m->m.ctx->stream));
    return TN_OK;
}

int tn_mps_get_max_d(tn_mps m, int* D) {
    if (!m || !D) return TN_BAD_ARG;
    *D = m->m.max_D();
    return TN_OK;
}

int tn_mps_get_expectation(tn_mps m, tn_hamiltonian h, double* E) {
    if (!m || !h || !E || h->h.L != m->m.L) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    return m->m.expectation(h->h.ops, E);
}

int tn_mps_get_expectation_h2(tn_mps m, tn_hamiltonian h, double* E2) {
    if (!m || !h || !E2 || h->h.L != m->m.L) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    return m->m.expectation(h->h.ops2, E2);
}

int tn_mps_find_itime_ground_state(tn_mps m, tn_hamiltonian h, const tn_itime_line* lines, int nlines,
                                   double* variance, int* iters_out) {
    if (!m || !h || !lines || nlines < 1 || h->h.L != m->m.L) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    for (int i = 0; i < nlines; ++i)
        if (lines[i].max_iter < 1 || lines[i].Dmax < 1 || (lines[i].order != 1 && lines[i].order != 2) ||
            !(lines[i].dt > 0)) {
            set_error("imaginary-time schedule line %d invalid", i);
            return TN_BAD_ARG;
        }
    m->m.H = &h->h;
    return m->m.itime_ground_state(lines, nlines, variance, iters_out);
}

// MPSImp::CalculateOneSiteDMs (MPSImp_ExpectationsAndDMs.C:59-71): L blocks of d x d,
// rho[(ia-1) d^2 + m d + n]; leaves the MPS left-normalised, as the reference.
int tn_mps_one_site_dms(tn_mps m, double* rho_host) {
    if (!m || !rho_host) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    return m->m.one_site_dms(rho_host);
}

// MPSImp::CalculateTwoSiteDMs (MPSImp_ExpectationsAndDMs.C:73-117): for every pair
// ia < ib in order, d^4 values rho[((m d + m2) d + n) d + n2] (m, n on ia; m2, n2 on ib).
int tn_mps_two_site_dms(tn_mps m, double* rho_host) {
    if (!m || !rho_host) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    return m->m.two_site_dms(rho_host);
}

int tn_mps_find_variational_ground_state(tn_mps m, tn_hamiltonian h, const tn_sched_line* lines, int nlines,
                                         const tn_solver_options* opt, tn_sweep_stats* stats, double* variance) {
    if (!m || !h || !lines || nlines < 1 || h->h.L != m->m.L) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    for (int i = 0; i < nlines; ++i)
        if (lines[i].max_sweeps < 1 || lines[i].Dmax < 1) {
            set_error("schedule line %d invalid", i);
            return TN_BAD_ARG;
        }
    if (opt && (opt->precision < TN_PREC_FP64 || opt->precision > TN_PREC_MIXED_HI)) return TN_BAD_ARG;
    m->m.H = &h->h;
    tn_sweep_stats st{};
    TN_CHECK(m->m.find_ground_state(lines, nlines, opt, &st));
    if (stats) *stats = st;
    if (variance) *variance = st.variance;
    return TN_OK;
}

int tn_mps_sweep(tn_mps m, tn_hamiltonian h, int nsweeps, double eps_eigen, const tn_solver_options* opt,
                 tn_sweep_stats* stats) {
    if (!m || !h || nsweeps < 1 || h->h.L != m->m.L) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    m->m.H = &h->h;
    return m->m.sweep_pairs(nsweeps, eps_eigen, opt, stats);
}

int tn_mps_prepare_sweeps(tn_mps m, tn_hamiltonian h) {
    if (!m || !h || h->h.L != m->m.L) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    m->m.H = &h->h;
    return m->m.prepare_sweeps();
}

unsigned long long tn_launch_count(void) { return __atomic_load_n(&tnb::g_launches, __ATOMIC_RELAXED); }

int tn_mps_get_site_energies(tn_mps m, double* E) {
    if (!m || !E) return TN_BAD_ARG;
    for (int ia = 1; ia <= m->m.L; ++ia) E[ia - 1] = m->m.Emin[ia];
    return TN_OK;
}

// ---- solver interfaces -----------------------------------------------------------
}  // extern "C"

struct tn_heff_s {
    tn_ctx ctx = nullptr;
    int precision = TN_PREC_FP64;
    tnb::ContractShape s{};
    tnb::DevBuf terms, P, Q;
    int nterms = 0;
    const double* F = nullptr;
    const double* G = nullptr;
    tnb::MixedSite ms;
};

extern "C" {

int tn_heff_create(tn_ctx c, int precision, int d, int Dw1, int Dw2, int D1, int D2, const double* W_host,
                   const double* F, const double* G, tn_heff* out) {
    if (!c || !W_host || !F || !G || !out) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    *out = nullptr;
    if (!valid_shape(d, Dw1, Dw2, D1, D2)) return TN_BAD_SHAPE;
    if (precision < TN_PREC_FP64 || precision > TN_PREC_MIXED_HI) return TN_BAD_ARG;
    ContractShape s{d, Dw1, Dw2, D1, D2};
    if (precision != TN_PREC_FP64 && !mixed_supported(s)) {
        set_error("split precision needs D1, D2 multiples of 16 (got %d, %d)", D1, D2);
        return TN_BAD_SHAPE;
    }
    tn_heff h = new tn_heff_s();
    h->ctx = c;
    h->precision = precision;
    h->s = s;
    h->F = F;
    h->G = G;
    auto t = build_terms(W_host, d, Dw1, Dw2, true);
    int st = h->terms.ensure(sizeof(WTermDev) * t.size());
    if (st == TN_OK && cudaMemcpy(h->terms.p, t.data(), sizeof(WTermDev) * t.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        st = TN_CUDA_ERROR;
    h->nterms = (int)t.size();
    if (st == TN_OK) {
        if (precision == TN_PREC_FP64) {
            size_t scr = sizeof(double) * contract_scratch_doubles(s);
            st = h->P.ensure(scr);
            if (st == TN_OK) st = h->Q.ensure(scr);
        } else {
            st = mixed_prepare_site(c->c, h->ms, s, W_host, F, G, -1, -1,
                                    precision == TN_PREC_MIXED_HI ? 3 : 2);
        }
    }
    if (st != TN_OK) {
        delete h;
        return st;
    }
    *out = h;
    return TN_OK;
}

long long tn_heff_size(tn_heff h) { return h ? (long long)h->s.d * h->s.D1 * h->s.D2 : -1; }

int tn_heff_apply(tn_heff h, const double* x, double* y) {
    if (!h || !x || !y) return TN_BAD_ARG;
    TN_ON_DEVICE(h->ctx->c.device);
    Ctx& cx = h->ctx->c;
    if (h->precision == TN_PREC_FP64)
        return heff_matvec_f64(h->s, h->terms.as<WTermDev>(), h->nterms, h->F, h->G, x, y, h->P.as<double>(),
                               h->Q.as<double>(), nullptr, cx.stream);
    return heff_matvec_mixed(cx, h->ms, x, y, nullptr);
}

int tn_heff_destroy(tn_heff h) {
    if (!h) return TN_BAD_ARG;
    TN_ON_DEVICE(h->ctx->c.device);
    cudaStreamSynchronize(h->ctx->c.stream);
    int st = TN_OK;
    if (h->precision != TN_PREC_FP64 && h->ms.ready) st = mixed_check_error(h->ms, h->ctx->c.stream);
    delete h;
    return st;
}

int tn_heff_matvec(tn_ctx c, int precision, int d, int Dw1, int Dw2, int D1, int D2, const double* W_host,
                   const double* F, const double* G, const double* x, double* y) {
    if (!c || !W_host || !F || !G || !x || !y) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    if (!valid_shape(d, Dw1, Dw2, D1, D2)) return TN_BAD_SHAPE;
    if (precision != TN_PREC_FP64) {
        tn_heff h = nullptr;
        TN_CHECK(tn_heff_create(c, precision, d, Dw1, Dw2, D1, D2, W_host, F, G, &h));
        int st = tn_heff_apply(h, x, y);
        int st2 = tn_heff_destroy(h);
        return st != TN_OK ? st : st2;
    }
    Ctx& cx = c->c;
    const WTermDev* t;
    int nt;
    TN_CHECK(upload_terms(cx, W_host, d, Dw1, Dw2, true, &t, &nt));
    ContractShape s{d, Dw1, Dw2, D1, D2};
    size_t scr = sizeof(double) * contract_scratch_doubles(s);
    TN_CHECK(cx.P.ensure(scr));
    TN_CHECK(cx.Q.ensure(scr));
    TN_CHECK(heff_matvec_f64(s, t, nt, F, G, x, y, cx.P.as<double>(), cx.Q.as<double>(), nullptr, cx.stream));
    return TN_OK;
}

int tn_heff_diag(tn_ctx c, int d, int Dw1, int Dw2, int D1, int D2, const double* W_host, const double* F,
                 const double* G, double* diag) {
    if (!c || !W_host || !F || !G || !diag) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    if (!valid_shape(d, Dw1, Dw2, D1, D2)) return TN_BAD_SHAPE;
    Ctx& cx = c->c;
    size_t nw = (size_t)Dw1 * Dw2 * d * d;
    TN_CHECK(cx.misc.ensure(sizeof(double) * nw));
    TN_CUDA_CHECK(cudaMemcpyAsync(cx.misc.p, W_host, sizeof(double) * nw, cudaMemcpyHostToDevice, cx.stream));
    ContractShape s{d, Dw1, Dw2, D1, D2};
    TN_CHECK(heff_diag(s, cx.misc.as<double>(), F, G, diag, cx.stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    return TN_OK;
}

int tn_env_left(tn_ctx c, int precision, int d, int Dw1, int Dw2, int D1, int D2, const double* W_host,
                const double* A, const double* F, double* Fout) {
    if (!c || !W_host || !A || !F || !Fout) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    if (!valid_shape(d, Dw1, Dw2, D1, D2)) return TN_BAD_SHAPE;
    if (precision != TN_PREC_FP64) return TN_BAD_ARG;
    Ctx& cx = c->c;
    const WTermDev* t;
    int nt;
    TN_CHECK(upload_terms(cx, W_host, d, Dw1, Dw2, true, &t, &nt));
    ContractShape s{d, Dw1, Dw2, D1, D2};
    size_t scr = sizeof(double) * contract_scratch_doubles(s);
    TN_CHECK(cx.P.ensure(scr));
    TN_CHECK(cx.Q.ensure(scr));
    return env_left_f64(s, t, nt, A, F, Fout, cx.P.as<double>(), cx.Q.as<double>(), cx.stream);
}

int tn_env_right(tn_ctx c, int precision, int d, int Dw1, int Dw2, int D1, int D2, const double* W_host,
                 const double* A, const double* G, double* Gout) {
    if (!c || !W_host || !A || !G || !Gout) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    if (!valid_shape(d, Dw1, Dw2, D1, D2)) return TN_BAD_SHAPE;
    if (precision != TN_PREC_FP64) return TN_BAD_ARG;
    Ctx& cx = c->c;
    const WTermDev* t;
    int nt;
    TN_CHECK(upload_terms(cx, W_host, d, Dw1, Dw2, false, &t, &nt));
    ContractShape s{d, Dw1, Dw2, D1, D2};
    size_t scr = sizeof(double) * contract_scratch_doubles(s);
    TN_CHECK(cx.P.ensure(scr));
    TN_CHECK(cx.Q.ensure(scr));
    return env_right_f64(s, t, nt, A, G, Gout, cx.P.as<double>(), cx.Q.as<double>(), cx.stream);
}

int tn_eigensolve_heff(tn_ctx c, const tn_solver_options* opt, int d, int Dw1, int Dw2, int D1, int D2,
                       const double* W_host, const double* F, const double* G, double* x, double tol,
                       double* theta, double* residual, int* matvecs) {
    if (!c || !W_host || !F || !G || !x) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    if (!valid_shape(d, Dw1, Dw2, D1, D2)) return TN_BAD_SHAPE;
    Ctx& cx = c->c;
    int krylov = (opt && opt->krylov > 0) ? opt->krylov : 20;
    int restarts = (opt && opt->max_restarts > 0) ? opt->max_restarts : 10;
    const WTermDev* t;
    int nt;
    TN_CHECK(upload_terms(cx, W_host, d, Dw1, Dw2, true, &t, &nt));
    ContractShape s{d, Dw1, Dw2, D1, D2};
    size_t scr = sizeof(double) * contract_scratch_doubles(s);
    TN_CHECK(cx.P.ensure(scr));
    TN_CHECK(cx.Q.ensure(scr));
    double* P = cx.P.as<double>();
    double* Q = cx.Q.as<double>();
    MatvecFn mv = [&](const double* xi, double* yo, const int* skip) {
        return heff_matvec_f64(s, t, nt, F, G, xi, yo, P, Q, skip, cx.stream);
    };
    const long long N = (long long)d * D1 * D2;
    if (opt && opt->eigensolver == TN_EIG_DAVIDSON) {
        // diagonal Davidson (the learned correction needs an MPS site context)
        const size_t nw = (size_t)Dw1 * Dw2 * d * d;
        TN_CHECK(cx.misc.ensure(sizeof(double) * (nw + (size_t)N)));
        double* Wd = cx.misc.as<double>();
        double* dg = Wd + nw;
        TN_CUDA_CHECK(cudaMemcpyAsync(Wd, W_host, sizeof(double) * nw, cudaMemcpyHostToDevice, cx.stream));
        TN_CHECK(heff_diag(s, Wd, F, G, dg, cx.stream));
        DvResult r{};
        TN_CHECK(davidson_solve(cx, N, x, std::min(krylov, DV_MAXK), restarts * krylov, tol, mv, dg, nullptr, 0.0,
                                &r));
        if (theta) *theta = r.theta;
        if (residual) *residual = r.resid;
        if (matvecs) *matvecs = r.matvecs;
        return r.converged ? TN_OK : TN_NOT_CONVERGED;
    }
    LzResult r{};
    TN_CHECK(lanczos_solve(cx, N, x, krylov, restarts, tol, mv, &r));
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    if (theta) *theta = r.theta;
    if (residual) *residual = r.resid;
    if (matvecs) *matvecs = r.matvecs;
    return r.converged ? TN_OK : TN_NOT_CONVERGED;
}

int tn_eigensolve_dense(tn_ctx c, int N, const double* A, int lda, int k, double tol, double* w_host, double* U,
                        int ldu) {
    if (!c || !A || !w_host || !U || N < 1 || k < 1 || k > N || lda < N || ldu < N || !(tol >= 0.0)) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    Ctx& cx = c->c;
    if ((size_t)N * 12 + 64 > 200 * 1024) {
        set_error("tn_eigensolve_dense: N = %d exceeds the single-CTA Jacobi limit", N);
        return TN_BAD_SHAPE;
    }
    // A + sigma I is positive definite for sigma above the Gershgorin bound
    // max_i sum_j |A_ij|; its SVD is then its eigen-decomposition, with the
    // eigenvalues s_i - sigma (descending) -- all on the device.
    const size_t n2 = (size_t)N * N;
    DevBuf work;
    TN_CHECK(work.ensure(sizeof(double) * (4 * n2 + (size_t)N + 8)));
    double* W = work.as<double>();
    double* V = W + n2;
    double* Ua = V + n2;
    double* Vt = Ua + n2;
    double* sv = Vt + n2;
    double* scal = sv + N;
    TN_CHECK(dense_shift_spd(N, A, lda, W, scal, cx.stream));
    SvdJob j{W, N, N, V, Ua, N, Vt, N, sv, nullptr};
    TN_CHECK(svd_batched(cx, {j}, true));
    // lowest k pairs, ascending: column N-1-e of Ua and s[N-1-e] - sigma
    TN_CHECK(copy2d(N, k, Ua + (size_t)(N - 1) * N, idx(1), idx(-(long long)N), U, idx(1), idx(ldu), 1.0, cx.stream));
    std::vector<double> hs(N + 1);
    TN_CUDA_CHECK(cudaMemcpyAsync(hs.data(), sv, sizeof(double) * N, cudaMemcpyDeviceToHost, cx.stream));
    TN_CUDA_CHECK(cudaMemcpyAsync(hs.data() + N, scal, sizeof(double), cudaMemcpyDeviceToHost, cx.stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    for (int e = 0; e < k; ++e) w_host[e] = hs[N - 1 - e] - hs[N];
    return TN_OK;
}

static int svd_common(tn_ctx c, int m, int n, const double* A, int lda, double* U, int ldu, double* s, double* Vt,
                      int ldvt, bool vectors) {
    if (!c || !A || !s || m < 1 || n < 1 || lda < m) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    if (vectors && (!U || !Vt || ldu < m || ldvt < std::min(m, n))) return TN_BAD_ARG;
    Ctx& cx = c->c;
    const bool tall = m >= n;
    const int tm = tall ? m : n, tn = tall ? n : m;
    size_t need = (size_t)tm * tn + (size_t)tn * tn + (tall ? 0 : (size_t)tm * tn + (size_t)tn * tn);
    TN_CHECK(cx.svdw.ensure(sizeof(double) * need + sizeof(SvdJob) * 2));
    // svd_batched uploads its job array into cx.svdw: keep the matrices elsewhere
    DevBuf work;
    TN_CHECK(work.ensure(sizeof(double) * need));
    double* Wm = work.as<double>();
    double* V = Wm + (size_t)tm * tn;
    double* Ut = V + (size_t)tn * tn;          // wide case: U of A^T (tm x tn)
    double* Vtt = Ut + (size_t)tm * tn;        // wide case: Vt of A^T (tn x tn)
    if (tall) TN_CHECK(copy2d(m, n, A, idx(1), idx(lda), Wm, idx(1), idx(m), 1.0, cx.stream));
    else TN_CHECK(copy2d(m, n, A, idx(1), idx(lda), Wm, idx(n), idx(1), 1.0, cx.stream));
    SvdJob j{};
    j.W = Wm; j.m = tm; j.n = tn; j.V = V; j.s = s;
    if (vectors) {
        if (tall) { j.U = U; j.ldu = ldu; j.Vt = Vt; j.ldvt = ldvt; }
        else { j.U = Ut; j.ldu = tm; j.Vt = Vtt; j.ldvt = tn; }
    }
    std::vector<SvdJob> jobs{j};
    TN_CHECK(svd_batched(cx, jobs, vectors));
    if (vectors && !tall) {
        // A^T = U' s V'^T  ->  A = V' s U'^T :  U = V' = Vtt^T (m x m), Vt = U'^T (m x n)
        TN_CHECK(copy2d(tn, tn, Vtt, idx(tn), idx(1), U, idx(1), idx(ldu), 1.0, cx.stream));
        TN_CHECK(copy2d(tn, tm, Ut, idx(tm), idx(1), Vt, idx(1), idx(ldvt), 1.0, cx.stream));
    }
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    return TN_OK;
}

int tn_svd(tn_ctx c, int m, int n, const double* A, int lda, double* U, int ldu, double* s, double* Vt, int ldvt) {
    return svd_common(c, m, n, A, lda, U, ldu, s, Vt, ldvt, true);
}

int tn_svd_values(tn_ctx c, int m, int n, const double* A, int lda, double* s) {
    return svd_common(c, m, n, A, lda, nullptr, 0, s, nullptr, 0, false);
}

// SVDSolver<T>::Solve(A, eps, k) (LapackSVDSolver.C:42-90): the k largest
// singular triplets.  eps is checked (< 1) as the reference asserts; the
// decomposition itself is complete before the truncation.
int tn_svd_solve(tn_ctx c, int m, int n, const double* A, int lda, double eps, int k, double* U, int ldu, double* s,
                 double* Vt, int ldvt) {
    const int mn = std::min(m, n);
    if (!c || !A || !U || !s || !Vt || m < 1 || n < 1 || lda < m || k < 1 || k > mn || ldu < m || ldvt < k ||
        !(eps < 1.0))
        return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    Ctx& cx = c->c;
    DevBuf full;
    TN_CHECK(full.ensure(sizeof(double) * ((size_t)m * mn + (size_t)mn * n + mn)));
    double* Uf = full.as<double>();
    double* Vf = Uf + (size_t)m * mn;
    double* sf = Vf + (size_t)mn * n;
    TN_CHECK(svd_common(c, m, n, A, lda, Uf, m, sf, Vf, mn, true));
    TN_CHECK(copy2d(m, k, Uf, idx(1), idx(m), U, idx(1), idx(ldu), 1.0, cx.stream));
    TN_CHECK(copy2d(k, n, Vf, idx(1), idx(mn), Vt, idx(1), idx(ldvt), 1.0, cx.stream));
    TN_CUDA_CHECK(cudaMemcpyAsync(s, sf, sizeof(double) * k, cudaMemcpyDeviceToDevice, cx.stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    return TN_OK;
}

int tn_qr(tn_ctx c, int m, int n, const double* A, int lda, double* Q, int ldq, double* R, int ldr) {
    if (!c || !A || !Q || !R || m < 1 || n < 1 || lda < m) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    const int k = std::min(m, n);
    if (ldq < m || ldr < k) return TN_BAD_ARG;
    Ctx& cx = c->c;
    DevBuf& W = cx.apiw[0];
    TN_CHECK(W.ensure(sizeof(double) * (size_t)m * n));
    TN_CHECK(copy2d(m, n, A, idx(1), idx(lda), W.as<double>(), idx(1), idx(m), 1.0, cx.stream));
    TN_CHECK(qr_dense(cx, m, n, W.as<double>(), Q, ldq, R, ldr));
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    return check_device_error(cx);
}

int tn_lq(tn_ctx c, int m, int n, const double* A, int lda, double* L, int ldl, double* Q, int ldq) {
    if (!c || !A || !Q || !L || m < 1 || n < 1 || lda < m) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    const int k = std::min(m, n);
    if (ldl < m || ldq < k) return TN_BAD_ARG;
    Ctx& cx = c->c;
    DevBuf &W = cx.apiw[0], &Qt = cx.apiw[1], &Rt = cx.apiw[2];
    TN_CHECK(W.ensure(sizeof(double) * (size_t)m * n));
    TN_CHECK(Qt.ensure(sizeof(double) * (size_t)n * k));
    TN_CHECK(Rt.ensure(sizeof(double) * (size_t)k * m));
    // A^T (n x m) = Qt Rt  ->  A = Rt^T Qt^T
    TN_CHECK(copy2d(m, n, A, idx(1), idx(lda), W.as<double>(), idx(n), idx(1), 1.0, cx.stream));
    TN_CHECK(qr_dense(cx, n, m, W.as<double>(), Qt.as<double>(), n, Rt.as<double>(), k));
    TN_CHECK(copy2d(k, m, Rt.as<double>(), idx(1), idx(k), L, idx(ldl), idx(1), 1.0, cx.stream));
    TN_CHECK(copy2d(n, k, Qt.as<double>(), idx(1), idx(n), Q, idx(ldq), idx(1), 1.0, cx.stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    return check_device_error(cx);
}

namespace {

// Row / column abs sums of a column-major k x n matrix (rows: flag 0; columns: 1).
__global__ void abs_sums_kernel(const double* __restrict__ M, int k, int n, int ld, int by_col,
                                double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int cnt = by_col ? n : k;
    if (t >= cnt) return;
    double s = 0.0;
    if (by_col)
        for (int i = 0; i < k; ++i) s += fabs(M[(size_t)t * ld + i]);
    else
        for (int c = 0; c < n; ++c) s += fabs(M[(size_t)c * ld + t]);
    out[t] = s;
}

// dst(r, c) = src(rows[r] or r, cols[c] or c): gather of kept rows / columns.
__global__ void gather2d_kernel(int rows, int cols, const double* __restrict__ src, int lds, const int* ridx,
                                const int* cidx, double* __restrict__ dst, int ldd) {
    const long long total = (long long)rows * cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e % rows), c = (int)(e / rows);
        const int sr = ridx ? ridx[r] : r, sc = cidx ? cidx[c] : c;
        dst[(size_t)c * ldd + r] = src[(size_t)sc * lds + sr];
    }
}

// The reference's ShrinkQR / ShrinkRQ (LapackQRSolver.C:324-365): the pivots of
// the triangular factor T (k x n for rows, m x k for columns) with |T_ii| <= eps
// whose whole row (column) sums to at most eps are dropped, with the matching
// column (row) of the orthonormal factor O.  Outputs are written compacted.
int shrink_factors(Ctx& cx, int k, const double* T, int ldt, int tr, int tc, bool rows, const double* O, int ldo,
                   int orows, int ocols, double eps, double* Tout, int ldto, double* Oout, int ldoo, int* rank) {
    cudaStream_t st = cx.stream;
    DevBuf& sums = cx.apiw[2];
    TN_CHECK(sums.ensure(sizeof(double) * (size_t)k + sizeof(int) * (size_t)k));
    abs_sums_kernel<<<(k + 127) / 128, 128, 0, st>>>(T, tr, tc, ldt, rows ? 0 : 1, sums.as<double>());
    TN_LAUNCH_CHECK();
    std::vector<double> hs(k), diag(k);
    TN_CUDA_CHECK(cudaMemcpyAsync(hs.data(), sums.p, sizeof(double) * k, cudaMemcpyDeviceToHost, st));
    for (int i = 0; i < k; ++i)
        TN_CUDA_CHECK(cudaMemcpyAsync(&diag[i], T + (size_t)i * ldt + i, sizeof(double), cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    std::vector<int> keep;
    for (int i = 0; i < k; ++i)
        if (!(std::fabs(diag[i]) <= eps && hs[i] <= eps)) keep.push_back(i);
    const int r = (int)keep.size();
    *rank = r;
    if (r == 0) return TN_OK;
    int* dk = reinterpret_cast<int*>(sums.as<double>() + k);
    TN_CUDA_CHECK(cudaMemcpyAsync(dk, keep.data(), sizeof(int) * r, cudaMemcpyHostToDevice, st));
    const long long nt = rows ? (long long)r * tc : (long long)tr * r;
    const long long no = rows ? (long long)orows * r : (long long)r * ocols;
    auto grid = [](long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 4096)); };
    if (rows) {  // T's kept rows, O's kept columns
        gather2d_kernel<<<grid(nt), 256, 0, st>>>(r, tc, T, ldt, dk, nullptr, Tout, ldto);
        TN_LAUNCH_CHECK();
        gather2d_kernel<<<grid(no), 256, 0, st>>>(orows, r, O, ldo, nullptr, dk, Oout, ldoo);
    } else {     // T's kept columns, O's kept rows
        gather2d_kernel<<<grid(nt), 256, 0, st>>>(tr, r, T, ldt, nullptr, dk, Tout, ldto);
        TN_LAUNCH_CHECK();
        gather2d_kernel<<<grid(no), 256, 0, st>>>(r, ocols, O, ldo, dk, nullptr, Oout, ldoo);
    }
    TN_LAUNCH_CHECK();
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    return TN_OK;
}

}  // namespace

// QRSolver::SolveThinRQ (LapackQRSolver.C:163-226): A = R Q with R m x k (upper
// for m <= n) and Q k x n with orthonormal rows -- the QR of B = P_n A^T P_m
// (P: index reversal), then R = P_m Rb^T P_k and Q = P_k Qb^T P_n.
int tn_rq(tn_ctx c, int m, int n, const double* A, int lda, double* R, int ldr, double* Q, int ldq) {
    if (!c || !A || !Q || !R || m < 1 || n < 1 || lda < m) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    const int k = std::min(m, n);
    if (ldr < m || ldq < k) return TN_BAD_ARG;
    Ctx& cx = c->c;
    DevBuf &W = cx.apiw[0], &Qb = cx.apiw[1], &Rb = cx.cqr;
    TN_CHECK(W.ensure(sizeof(double) * (size_t)m * n));
    TN_CHECK(Qb.ensure(sizeof(double) * (size_t)n * k));
    TN_CHECK(Rb.ensure(sizeof(double) * (size_t)k * m));
    // W (n x m, ld n): W(i, j) = A(m-1-j, n-1-i)
    TN_CHECK(copy2d(n, m, A + (size_t)(n - 1) * lda + (m - 1), idx(-(long long)lda), idx(-1), W.as<double>(), idx(1),
                    idx(n), 1.0, cx.stream));
    TN_CHECK(qr_dense(cx, n, m, W.as<double>(), Qb.as<double>(), n, Rb.as<double>(), k));
    // R(i, j) = Rb(k-1-j, m-1-i);  Q(i, j) = Qb(n-1-j, k-1-i)
    TN_CHECK(copy2d(m, k, Rb.as<double>() + (size_t)(m - 1) * k + (k - 1), idx(-(long long)k), idx(-1), R, idx(1),
                    idx(ldr), 1.0, cx.stream));
    TN_CHECK(copy2d(k, n, Qb.as<double>() + (size_t)(k - 1) * n + (n - 1), idx(-(long long)n), idx(-1), Q, idx(1),
                    idx(ldq), 1.0, cx.stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    return check_device_error(cx);
}

// QRSolver::SolveThinQL (LapackQRSolver.C:229-274): A = Q L with Q m x k
// (orthonormal columns) and L k x n (lower for n <= m) -- the QR of
// B = P_m A P_n, then Q = P_m Qb P_k and L = P_k Rb P_n.
int tn_ql(tn_ctx c, int m, int n, const double* A, int lda, double* Q, int ldq, double* L, int ldl) {
    if (!c || !A || !Q || !L || m < 1 || n < 1 || lda < m) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    const int k = std::min(m, n);
    if (ldq < m || ldl < k) return TN_BAD_ARG;
    Ctx& cx = c->c;
    DevBuf &W = cx.apiw[0], &Qb = cx.apiw[1], &Rb = cx.cqr;
    TN_CHECK(W.ensure(sizeof(double) * (size_t)m * n));
    TN_CHECK(Qb.ensure(sizeof(double) * (size_t)m * k));
    TN_CHECK(Rb.ensure(sizeof(double) * (size_t)k * n));
    TN_CHECK(copy2d(m, n, A + (size_t)(n - 1) * lda + (m - 1), idx(-1), idx(-(long long)lda), W.as<double>(), idx(1),
                    idx(m), 1.0, cx.stream));
    TN_CHECK(qr_dense(cx, m, n, W.as<double>(), Qb.as<double>(), m, Rb.as<double>(), k));
    TN_CHECK(copy2d(m, k, Qb.as<double>() + (size_t)(k - 1) * m + (m - 1), idx(-1), idx(-(long long)m), Q, idx(1),
                    idx(ldq), 1.0, cx.stream));
    TN_CHECK(copy2d(k, n, Rb.as<double>() + (size_t)(n - 1) * k + (k - 1), idx(-1), idx(-(long long)k), L, idx(1),
                    idx(ldl), 1.0, cx.stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    return check_device_error(cx);
}

// QRSolver::SolveRankRevealingQR / RQ / QL / LQ (LapackQRSolver.C:367-399): the
// thin factorisation, then ShrinkQR / ShrinkRQ with eps.  kind: 0 QR (A = Q R),
// 1 LQ (A = L Q), 2 RQ (A = R Q), 3 QL (A = Q L).  The outputs hold the kept
// factors: QR / QL: F1 = Q m x rank, F2 = R / L rank x n;  LQ / RQ:
// F1 = L / R m x rank, F2 = Q rank x n.  *rank = the number kept.
int tn_qr_rank_revealing(tn_ctx c, int kind, int m, int n, const double* A, int lda, double* F1, int ld1,
                         double* F2, int ld2, double eps, int* rank) {
    if (!c || !A || !F1 || !F2 || !rank || m < 1 || n < 1 || lda < m || kind < 0 || kind > 3 || !(eps >= 0))
        return TN_BAD_ARG;
    const int k = std::min(m, n);
    const bool col_first = (kind == 0 || kind == 3);  // Q first (m x k), triangle second (k x n)
    if (ld1 < m || ld2 < k) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    Ctx& cx = c->c;
    DevBuf &T1 = cx.rr1, &T2 = cx.rr2;
    TN_CHECK(T1.ensure(sizeof(double) * (size_t)m * k));
    TN_CHECK(T2.ensure(sizeof(double) * (size_t)k * n));
    int st = TN_OK;
    if (kind == 0) st = tn_qr(c, m, n, A, lda, T1.as<double>(), m, T2.as<double>(), k);
    else if (kind == 1) st = tn_lq(c, m, n, A, lda, T1.as<double>(), m, T2.as<double>(), k);
    else if (kind == 2) st = tn_rq(c, m, n, A, lda, T1.as<double>(), m, T2.as<double>(), k);
    else st = tn_ql(c, m, n, A, lda, T1.as<double>(), m, T2.as<double>(), k);
    TN_CHECK(st);
    if (col_first)  // triangle T2 (k x n): rows dropped, with Q's columns
        return shrink_factors(cx, k, T2.as<double>(), k, k, n, true, T1.as<double>(), m, m, k, eps, F2, ld2, F1, ld1,
                              rank);
    // triangle T1 (m x k): columns dropped, with Q's rows
    return shrink_factors(cx, k, T1.as<double>(), m, m, k, false, T2.as<double>(), k, k, n, eps, F1, ld1, F2, ld2,
                          rank);
}

// SVCompressorImp<T>::Compress (SVCompressorImp.C:19-73) on a device s vector.
int tn_compress(tn_ctx c, int Dmax, double eps, int k, double* s, int* D_out, double* discarded) {
    if (!c || !s || k < 1 || !D_out) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    Ctx& cx = c->c;
    std::vector<double> h(k);
    TN_CUDA_CHECK(cudaStreamSynchronize(cx.stream));
    TN_CUDA_CHECK(cudaMemcpy(h.data(), s, sizeof(double) * k, cudaMemcpyDeviceToHost));
    int N = k, D = N;
    double integ = 0.0;
    if (eps == 0.0) {
        if (Dmax < 1) return TN_BAD_ARG;
        D = std::min(Dmax, N);
        for (int id = D; id < N; ++id) integ += h[id] * h[id];
    } else {
        for (; D >= 1; --D) {
            double s2 = h[D - 1] * h[D - 1];
            if (integ + s2 >= eps) break;
            integ += s2;
        }
        if (Dmax > 0 && D > Dmax) {
            // capped at Dmax; the discarded weight is still the eps-scan sum (as the reference)
            D = Dmax;
        }
    }
    if (D < N) {
        double before = 0, after = 0;
        for (int i = 0; i < N; ++i) before += h[i] * h[i];
        for (int i = 0; i < D; ++i) after += h[i] * h[i];
        double rescale = after > 0 ? before / after : 1.0;
        for (int i = 0; i < D; ++i) h[i] *= rescale;
        TN_CUDA_CHECK(cudaMemcpy(s, h.data(), sizeof(double) * D, cudaMemcpyHostToDevice));
    }
    *D_out = std::max(D, 0);
    if (discarded) *discarded = integ;
    return TN_OK;
}


struct tn_mlp_s {
    tnb::MlpModel m;
};
struct tn_dataset_s {
    tnb::DvRecorder r;
};

int tn_mlp_create(tn_ctx c, uint64_t seed, tn_mlp* out) {
    if (!c || !out) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    auto* h = new tn_mlp_s();
    const int st = tnb::mlp_init(h->m, c->c, seed);
    if (st != TN_OK) {
        delete h;
        return st;
    }
    *out = h;
    return TN_OK;
}

int tn_mlp_destroy(tn_mlp m) {
    if (!m) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    delete m;
    return TN_OK;
}

int tn_mlp_num_params(void) { return tnb::MLP_NP; }

int tn_mlp_get_params(tn_mlp m, float* host) {
    if (!m || !host) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    return tnb::mlp_get_params(m->m, host);
}

int tn_mlp_set_params(tn_mlp m, const float* host) {
    if (!m || !host) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    return tnb::mlp_set_params(m->m, host);
}

int tn_mlp_forward(tn_mlp m, const float* F, long long n, float* Y) {
    if (!m || !F || !Y || n < 0) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    TN_CHECK(tnb::mlp_forward(m->m, F, n, Y, m->m.ctx->stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(m->m.ctx->stream));
    return TN_OK;
}

int tn_mlp_gradient(tn_mlp m, const float* F, const float* T, long long n, float* grad_host, double* loss) {
    if (!m || !F || !T || !grad_host || n < 1) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    return tnb::mlp_gradient(m->m, F, T, n, grad_host, loss);
}

int tn_mlp_train(tn_mlp m, const float* F, const float* T, long long n, int steps, int batch, double lr,
                 uint64_t seed, double* final_loss) {
    if (!m || !F || !T || n < 1 || steps < 1 || !(lr > 0)) return TN_BAD_ARG;
    TN_ON_DEVICE(m->m.ctx->device);
    if (n > 2000000000LL) return TN_BAD_SHAPE;
    return tnb::mlp_train(m->m, F, T, n, steps, batch, lr, seed, final_loss);
}

int tn_dataset_create(tn_ctx c, long long capacity, tn_dataset* out) {
    if (!c || !out || capacity < 1) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    auto* h = new tn_dataset_s();
    const int st = tnb::recorder_init(h->r, c->c, capacity);
    if (st != TN_OK) {
        delete h;
        return st;
    }
    *out = h;
    return TN_OK;
}

int tn_dataset_destroy(tn_dataset ds) {
    if (!ds) return TN_BAD_ARG;
    TN_ON_DEVICE(ds->r.ctx->device);
    delete ds;
    return TN_OK;
}

long long tn_dataset_size(tn_dataset ds) { return ds ? ds->r.size : -1; }

int tn_dataset_data(tn_dataset ds, const float** F, const float** T) {
    if (!ds || !F || !T) return TN_BAD_ARG;
    *F = ds->r.feats.as<float>();
    *T = ds->r.targets.as<float>();
    return TN_OK;
}

int tn_mps_set_learned_correction(tn_mps psi, tn_mlp m) {
    if (!psi) return TN_BAD_ARG;
    psi->m.mlp = m ? &m->m : nullptr;
    return TN_OK;
}

int tn_mps_set_recorder(tn_mps psi, tn_dataset ds) {
    if (!psi) return TN_BAD_ARG;
    psi->m.recorder = ds ? &ds->r : nullptr;
    return TN_OK;
}


struct tn_itebd_s {
    tnb::ITebdState s;
};

int tn_itebd_create(tn_ctx c, double S, double Jxy, double Jz, double hz, int D, uint64_t seed, tn_itebd* out) {
    if (!c || !out || D < 1 || S <= 0) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    auto* h = new tn_itebd_s();
    const int st = h->s.init(c->c, S, Jxy, Jz, hz, D, seed);
    if (st != TN_OK) {
        delete h;
        return st;
    }
    *out = h;
    return TN_OK;
}

int tn_itebd_destroy(tn_itebd st) {
    if (!st) return TN_BAD_ARG;
    TN_ON_DEVICE(st->s.ctx->device);
    delete st;
    return TN_OK;
}

int tn_itebd_get_site(tn_itebd st, int site, int* Dl, int* Dr, double* host) {
    if (!st || site < 0 || site > 1) return TN_BAD_ARG;
    TN_ON_DEVICE(st->s.ctx->device);
    auto& s = st->s;
    const int l = s.dim(1 - site), r = s.dim(site);
    if (Dl) *Dl = l;
    if (Dr) *Dr = r;
    if (host) {
        TN_CUDA_CHECK(cudaStreamSynchronize(s.ctx->stream));
        TN_CUDA_CHECK(cudaMemcpy(host, s.G[site].p, sizeof(double) * (size_t)s.d * l * r, cudaMemcpyDeviceToHost));
    }
    return TN_OK;
}

int tn_itebd_set_site(tn_itebd st, int site, int Dl, int Dr, const double* host) {
    if (!st || site < 0 || site > 1 || !host) return TN_BAD_ARG;
    TN_ON_DEVICE(st->s.ctx->device);
    auto& s = st->s;
    if (Dl != s.dim(1 - site) || Dr != s.dim(site)) {
        tnb::set_error("tn_itebd_set_site: site %d is %d x %d (set the bond values first)", site, s.dim(1 - site),
                       s.dim(site));
        return TN_BAD_SHAPE;
    }
    TN_CHECK(s.G[site].ensure(sizeof(double) * (size_t)s.d * Dl * Dr));
    TN_CUDA_CHECK(cudaStreamSynchronize(s.ctx->stream));
    TN_CUDA_CHECK(cudaMemcpy(s.G[site].p, host, sizeof(double) * (size_t)s.d * Dl * Dr, cudaMemcpyHostToDevice));
    return TN_OK;
}

int tn_itebd_get_bond(tn_itebd st, int bond, int* D, double* host) {
    if (!st || bond < 0 || bond > 1) return TN_BAD_ARG;
    const auto& v = st->s.lam_h[bond];
    if (D) *D = (int)v.size();
    if (host) std::memcpy(host, v.data(), sizeof(double) * v.size());
    return TN_OK;
}

int tn_itebd_set_bond(tn_itebd st, int bond, int D, const double* host) {
    if (!st || bond < 0 || bond > 1 || D < 1 || !host) return TN_BAD_ARG;
    TN_ON_DEVICE(st->s.ctx->device);
    auto& s = st->s;
    s.lam_h[bond].assign(host, host + D);
    TN_CHECK(s.lam[bond].ensure(sizeof(double) * D));
    TN_CUDA_CHECK(cudaStreamSynchronize(s.ctx->stream));
    TN_CUDA_CHECK(cudaMemcpy(s.lam[bond].p, host, sizeof(double) * D, cudaMemcpyHostToDevice));
    return TN_OK;
}

int tn_itebd_step(tn_itebd st, double dt, int Dmax, int nsteps) {
    if (!st || Dmax < 1 || nsteps < 0) return TN_BAD_ARG;
    TN_ON_DEVICE(st->s.ctx->device);
    for (int k = 0; k < nsteps; ++k) TN_CHECK(st->s.step2(dt, Dmax));
    return TN_OK;
}

// iTEBDStateImp::FindiTimeGroundState(H, iH, H2, line), iTEBDStateImp_iTime.C:44-104:
// per schedule line (one dt each) OrthogonalizeI with eps dt^2/1000 (1e-13 at
// dt = 0) and the current D as compressor, then for D = current .. Dmax in
// steps of deltaD: bond dimensions grown to D (IncreaseBondDimensions), second-
// order Trotter steps until both bond vectors move by at most eps_factor*dt
// (or max_iter steps), OrthogonalizeI again.  steps_out[l] = Trotter steps of line l.
int tn_itebd_find_ground_state(tn_itebd st, const double* dts, int ndt, int max_iter, int Dmax, int deltaD,
                               double eps_factor, int* steps_out) {
    if (!st || !dts || ndt < 1 || max_iter < 1 || Dmax < 1 || deltaD < 1) return TN_BAD_ARG;
    TN_ON_DEVICE(st->s.ctx->device);
    auto& s = st->s;
    constexpr int ORTH_ITER = 100;  // nOrthIter, iTEBDStateImp_iTime.C:57
    for (int l = 0; l < ndt; ++l) {
        const double dt = dts[l];
        const double eps_orth = dt == 0.0 ? 1e-13 : dt * dt / 1000.0;
        int Dcur = std::max(s.dim(0), s.dim(1));
        TN_CHECK(s.orthogonalize_i(Dcur, eps_orth, ORTH_ITER, nullptr, nullptr, nullptr));
        int total = 0;
        for (int D = Dcur; D <= Dmax; D += deltaD) {
            if (D > Dcur) TN_CHECK(s.grow(D));
            for (int n = 1; n <= max_iter; ++n) {
                const std::vector<double> old0 = s.lam_h[0], old1 = s.lam_h[1];
                TN_CHECK(s.step2(dt, D));
                ++total;
                double dl = 0;
                for (int b = 0; b < 2; ++b) {
                    const auto& o = b == 0 ? old0 : old1;
                    const auto& x = s.lam_h[b];
                    if (o.size() != x.size()) {
                        dl = 1.0;
                        continue;
                    }
                    for (size_t i = 0; i < x.size(); ++i) dl = std::max(dl, std::fabs(o[i] - x[i]));
                }
                if (dl <= eps_factor * dt) break;
            }
            TN_CHECK(s.orthogonalize_i(D, eps_orth, ORTH_ITER, nullptr, nullptr, nullptr));
            Dcur = D;
        }
        if (steps_out) steps_out[l] = total;
    }
    return TN_OK;
}

int tn_itebd_orthogonalize(tn_itebd st, int Dmax, double eps, int max_iter, double* delta, int* iters) {
    if (!st || Dmax < 1 || !(eps > 0) || max_iter < 1) return TN_BAD_ARG;
    TN_ON_DEVICE(st->s.ctx->device);
    bool bailed = false;
    TN_CHECK(st->s.orthogonalize_i(Dmax, eps, max_iter, delta, iters, &bailed));
    if (bailed) {
        tnb::set_error("OrthogonalizeI: singular norm matrix, iteration abandoned (state unpacked as it stood)");
        return TN_NOT_CONVERGED;
    }
    return TN_OK;
}

int tn_itebd_energy(tn_itebd st, int max_iters, double tol, double* E) {
    if (!st || !E || max_iters < 1) return TN_BAD_ARG;
    TN_ON_DEVICE(st->s.ctx->device);
    return st->s.energy(E, max_iters, tol);
}


// ---- full state (exact diagonalisation) ------------------------------------------
struct tn_fullstate_s {
    tnb::FullStateDev f;
};

int tn_fullstate_create(tn_hamiltonian h, uint64_t seed, tn_fullstate* out) {
    if (!h || !out) return TN_BAD_ARG;
    TN_ON_DEVICE(h->h.ctx->device);
    *out = nullptr;
    auto* fs = new tn_fullstate_s();
    int st = fs->f.init(*h->h.ctx, h->h.L, h->h.S, seed);
    if (st == TN_OK) st = fs->f.set_hamiltonian(h->h.Jxy, h->h.Jz, h->h.hz);
    if (st == TN_OK && cudaStreamSynchronize(h->h.ctx->stream) != cudaSuccess) st = TN_CUDA_ERROR;
    if (st != TN_OK) {
        delete fs;
        return st;
    }
    *out = fs;
    return TN_OK;
}

int tn_fullstate_destroy(tn_fullstate fs) {
    if (!fs) return TN_BAD_ARG;
    TN_ON_DEVICE(fs->f.ctx->device);
    cudaStreamSynchronize(fs->f.ctx->stream);
    delete fs;
    return TN_OK;
}

long long tn_fullstate_get_size(tn_fullstate fs) { return fs ? fs->f.N : -1; }

static bool same_chain(tn_fullstate fs, tn_hamiltonian h) {
    return h->h.L == fs->f.L && std::fabs(h->h.S - fs->f.S) < 1e-12;
}

int tn_fullstate_find_ground_state(tn_fullstate fs, tn_hamiltonian h, double epsE, double* E, int* matvecs) {
    if (!fs || !h || !(epsE > 0) || !same_chain(fs, h)) return TN_BAD_ARG;
    TN_ON_DEVICE(fs->f.ctx->device);
    TN_CHECK(fs->f.set_hamiltonian(h->h.Jxy, h->h.Jz, h->h.hz));
    return fs->f.find_ground_state(epsE, 40, 200, E, matvecs);
}

int tn_fullstate_power_iterate(tn_fullstate fs, tn_hamiltonian h, double epsE, double epsPsi, int max_iter,
                               double* E, int* iters) {
    if (!fs || !h || max_iter < 1 || !same_chain(fs, h)) return TN_BAD_ARG;
    TN_ON_DEVICE(fs->f.ctx->device);
    TN_CHECK(fs->f.set_hamiltonian(h->h.Jxy, h->h.Jz, h->h.hz));
    return fs->f.power_iterate(epsE, epsPsi, max_iter, E, iters);
}

int tn_fullstate_get_e(tn_fullstate fs, double* E) {
    if (!fs || !E) return TN_BAD_ARG;
    *E = fs->f.E;
    return TN_OK;
}

int tn_fullstate_get_amplitudes(tn_fullstate fs, double* host) {
    if (!fs || !host) return TN_BAD_ARG;
    TN_ON_DEVICE(fs->f.ctx->device);
    TN_CUDA_CHECK(cudaStreamSynchronize(fs->f.ctx->stream));
    TN_CUDA_CHECK(cudaMemcpy(host, fs->f.amp.p, sizeof(double) * (size_t)fs->f.N, cudaMemcpyDeviceToHost));
    return TN_OK;
}

int tn_fullstate_matvec(tn_fullstate fs, tn_hamiltonian h, const double* x, double* y) {
    if (!fs || !h || !x || !y || !same_chain(fs, h)) return TN_BAD_ARG;
    TN_ON_DEVICE(fs->f.ctx->device);
    TN_CHECK(fs->f.set_hamiltonian(h->h.Jxy, h->h.Jz, h->h.hz));
    return fs->f.matvec(x, y, nullptr);
}


}  // extern "C"

namespace {
// y = (1 + i/n) x: a diagonal operator with distinct eigenvalues, so that the
// Krylov space never closes early
__global__ void diag_probe_kernel(const double* __restrict__ x, double* __restrict__ y, long long n, const int* skip) {
    if (skip && *skip) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = (1.0 + (double)i / (double)n) * x[i];
}
}  // namespace

extern "C" {

// Device time per Lanczos step of the library's Krylov kernels (CGS2 dots and
// updates, next vector, tridiagonal decision) on a diagonal operator, the
// steps replayed from the CUDA graph as in a sweep.  A measurement hook with
// no counterpart in the reference.
int tn_lanczos_probe(tn_ctx c, long long N, int m, double* us_per_step, double* bytes_per_step) {
    if (!c || N < 64 || m < 2 || !us_per_step) return TN_BAD_ARG;
    TN_ON_DEVICE(c->c.device);
    Ctx& cx = c->c;
    DevBuf xb;
    TN_CHECK(xb.ensure(sizeof(double) * (size_t)N));
    const int g = (int)std::min<long long>((N + 255) / 256, (long long)cx.sm_count * 8);
    MatvecFn mv = [&](const double* x, double* y, const int* skip) -> int {
        diag_probe_kernel<<<g, 256, 0, cx.stream>>>(x, y, N, skip);
        TN_LAUNCH_CHECK();
        return (int)TN_OK;
    };
    const bool prof0 = cx.prof;
    cx.prof = true;
    unsigned long long key = hash_val(HASH_SEED, 0x70726f6265ULL);
    key = hash_val(key, N);
    key = hash_val(key, m);
    int rc = TN_OK;
    LzResult r{};
    for (int pass = 0; pass < 2 && rc == TN_OK; ++pass) {  // pass 0 records the graph
        cx.prof_ms[2] = 0;
        cx.prof_steps = 0;
        rc = fill(xb.as<double>(), N, 1.0, cx.stream);
        if (rc == TN_OK) rc = lanczos_solve(cx, N, xb.as<double>(), m, 1, 1e-300, mv, &r, 0.0, key);
    }
    const double ms = cx.prof_ms[2];
    const long long steps = cx.prof_steps;
    cx.prof = prof0;
    TN_CHECK(rc);
    if (steps < 1) {
        set_error("tn_lanczos_probe: no Krylov step was timed");
        return TN_CUDA_ERROR;
    }
    *us_per_step = ms * 1e3 / (double)steps;
    if (bytes_per_step) {
        // (j + 4) N doubles per step j of the CGS2 step (basis reads for the two
        // projection passes, the update and the next vector), plus the diagonal
        // operator's read and write
        double b = 0;
        for (long long j = 1; j <= steps; ++j) b += (double)(j + 4) * N * 8.0;
        *bytes_per_step = b / (double)steps + 2.0 * N * 8.0;
    }
    return TN_OK;
}

}  // extern "C"
