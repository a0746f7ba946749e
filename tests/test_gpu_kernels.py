"""GPU parity of the individual kernels against the FP64 CPU oracle.

Every call goes through the C ABI (libtn_cuda.so); device buffers are torch
CUDA tensors.  FP64 kernels are compared at tolerances a few ulps times the
problem norm.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import tensornetworks_b200 as T
    return T


@pytest.fixture(scope="module")
def ctx(T):
    return T.default_context()


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()


def host(t):
    return t.cpu().numpy()


def envs(oracle, d, D1, D2, site, L=6, hz=0.2, seed=3):
    """Physical environments of a random L-site chain around `site`, whose
    tensor is D1 x D2 (D1 = 1 at site 1, D2 = 1 at site L); Heff is symmetric."""
    rng = np.random.default_rng(seed)
    S = (d - 1) / 2
    Ws = {i: oracle.mpo_site(L, S, 2, 1.0, 1.0, hz, i) for i in range(1, L + 1)}
    shapes = {}
    for i in range(1, L + 1):
        if i < site:
            shapes[i] = (1 if i == 1 else D1, D1)
        elif i == site:
            shapes[i] = (D1, D2)
        else:
            shapes[i] = (D2, 1 if i == L else D2)
    A = {i: rng.uniform(-1, 1, size=(d,) + shapes[i]) for i in range(1, L + 1)}
    F = np.ones(1)
    for i in range(1, site):
        F = oracle.env_left(Ws[i], A[i], F)
    G = np.ones(1)
    for i in range(L, site, -1):
        G = oracle.env_right(Ws[i], A[i], G)
    return Ws[site], A[site], F, G


@pytest.mark.parametrize("d,D1,D2,site", [(2, 8, 8, 3), (2, 16, 32, 3), (3, 9, 9, 3), (2, 1, 2, 1),
                                          (2, 64, 64, 3), (2, 48, 40, 4), (2, 8, 1, 6)])
def test_heff_matvec_and_envs(T, ctx, oracle, d, D1, D2, site):
    W, A, F, G = envs(oracle, d, D1, D2, site)
    Dw1, Dw2 = W.shape[:2]
    D1, D2 = A.shape[1:]
    x = oracle.site_flat(A)
    lib = ctx._lib
    Wc = np.ascontiguousarray(W.ravel())
    dF, dG, dx = dev(F), dev(G), dev(x)
    y = dev(np.zeros_like(x))
    T._capi.check(lib.tn_heff_matvec(ctx.handle, 0, d, Dw1, Dw2, D1, D2, Wc.ctypes.data, dF.data_ptr(),
                                     dG.data_ptr(), dx.data_ptr(), y.data_ptr()), "matvec")
    ref = oracle.heff_matvec(W, F, G, x, D1, D2)
    scale = np.abs(ref).max() + 1e-300
    assert np.abs(host(y) - ref).max() <= 1e-12 * scale
    # diag
    dg = dev(np.zeros_like(x))
    T._capi.check(lib.tn_heff_diag(ctx.handle, d, Dw1, Dw2, D1, D2, Wc.ctypes.data, dF.data_ptr(), dG.data_ptr(),
                                   dg.data_ptr()), "diag")
    np.testing.assert_allclose(host(dg), oracle.heff_diag(W, F, G, D1, D2), rtol=1e-12, atol=1e-12 * scale)
    # environments
    outL = dev(np.zeros(Dw2 * D2 * D2))
    T._capi.check(lib.tn_env_left(ctx.handle, 0, d, Dw1, Dw2, D1, D2, Wc.ctypes.data, dx.data_ptr(), dF.data_ptr(),
                                  outL.data_ptr()), "env_left")
    refL = oracle.env_left(W, A, F)
    assert np.abs(host(outL) - refL).max() <= 1e-12 * (np.abs(refL).max() + 1e-300)
    outR = dev(np.zeros(Dw1 * D1 * D1))
    T._capi.check(lib.tn_env_right(ctx.handle, 0, d, Dw1, Dw2, D1, D2, Wc.ctypes.data, dx.data_ptr(), dG.data_ptr(),
                                   outR.data_ptr()), "env_right")
    refR = oracle.env_right(W, A, G)
    assert np.abs(host(outR) - refR).max() <= 1e-12 * (np.abs(refR).max() + 1e-300)


@pytest.mark.parametrize("d,D1,D2,site", [(2, 8, 8, 3), (2, 32, 32, 3), (3, 9, 9, 3), (2, 2, 4, 2)])
def test_lanczos_heff(T, ctx, oracle, d, D1, D2, site):
    W, A, F, G = envs(oracle, d, D1, D2, site)
    Dw1, Dw2 = W.shape[:2]
    D1, D2 = A.shape[1:]
    H = oracle.heff_dense(W, F, G, D1, D2)
    H = 0.5 * (H + H.T)
    w = np.linalg.eigvalsh(H)
    x0 = oracle.site_flat(A)
    dx = dev(x0)
    th, res, nmv = C.c_double(), C.c_double(), C.c_int()
    opt = T.SolverOptions(krylov=20, max_restarts=30).to_c()
    Wc = np.ascontiguousarray(W.ravel())
    dF, dG = dev(F), dev(G)   # keep the device buffers alive across the call
    st = ctx._lib.tn_eigensolve_heff(ctx.handle, C.byref(opt), d, Dw1, Dw2, D1, D2, Wc.ctypes.data,
                                     dF.data_ptr(), dG.data_ptr(), dx.data_ptr(), 1e-10, C.byref(th),
                                     C.byref(res), C.byref(nmv))
    assert st == 0, T._capi.last_error()
    assert abs(th.value - w[0]) < 1e-9 * max(1, abs(w[0]))
    x = host(dx)
    assert abs(np.linalg.norm(x) - 1) < 1e-12
    assert np.linalg.norm(H @ x - th.value * x) < 1e-8 * max(1, abs(w[0]))
    # same algorithm as the oracle: same Ritz value
    tho, _, _, _ = oracle.lanczos_heff(W, F, G, x0, D1, D2, krylov=20, max_restarts=30, tol=1e-10)
    assert abs(th.value - tho) < 1e-10 * max(1, abs(tho))


def test_lanczos_bulk_sizes(T, oracle):
    """The device Lanczos gives the oracle's Ritz value on bulk sites whose
    vectors fill a fraction of the grid, about one element per thread and
    several per thread (N = 8192, 180 000, 307 200)."""
    c = T.Context(0)
    for (d, D, site) in [(2, 64, 3), (2, 300, 3), (3, 320, 3)]:
        W, A, F, G = envs(oracle, d, D, D, site)
        Dw1, Dw2 = W.shape[:2]
        D1, D2 = A.shape[1:]
        x0 = oracle.site_flat(A)
        dx = dev(x0)
        th, res, nmv = C.c_double(), C.c_double(), C.c_int()
        opt = T.SolverOptions(krylov=20, max_restarts=30).to_c()
        Wc = np.ascontiguousarray(W.ravel())
        dF, dG = dev(F), dev(G)
        st = c._lib.tn_eigensolve_heff(c.handle, C.byref(opt), d, Dw1, Dw2, D1, D2, Wc.ctypes.data, dF.data_ptr(),
                                       dG.data_ptr(), dx.data_ptr(), 1e-10, C.byref(th), C.byref(res), C.byref(nmv))
        assert st == 0, T._capi.last_error()
        tho, _, _, _ = oracle.lanczos_heff(W, F, G, x0, D1, D2, krylov=20, max_restarts=30, tol=1e-10)
        assert abs(th.value - tho) < 1e-10 * max(1, abs(tho))
        x = host(dx)
        assert abs(np.linalg.norm(x) - 1) < 1e-12


@pytest.mark.parametrize("m,n", [(7, 5), (5, 7), (64, 32), (32, 64), (512, 256), (130, 130), (1, 5), (9, 1),
                                 (700, 700), (1024, 300), (600, 40), (2000, 64)])
def test_qr_lq(T, ctx, oracle, m, n):
    rng = np.random.default_rng(m * 1000 + n)
    A = rng.uniform(-1, 1, size=(m, n))
    Q, R = T.CudaQRSolver(ctx).SolveThinQR(A)
    k = min(m, n)
    assert np.abs(Q.T @ Q - np.eye(k)).max() < 1e-13
    assert np.allclose(np.triu(R), R)
    assert np.abs(Q @ R - A).max() < 1e-12
    Qo, Ro = oracle.qr(A)
    np.testing.assert_allclose(R, Ro, atol=1e-11)    # same reflector convention -> same factors
    Lm, Q2 = T.CudaQRSolver(ctx).SolveThinLQ(A)
    assert np.abs(Q2 @ Q2.T - np.eye(k)).max() < 1e-13
    assert np.abs(Lm @ Q2 - A).max() < 1e-12
    assert np.allclose(np.tril(Lm), Lm)


@pytest.mark.parametrize("m,n", [(512, 256), (300, 200), (256, 96)])
def test_qr_rank_deficient_panels(T, ctx, oracle, m, n):
    """Several panels (with a ragged last one) on a matrix whose columns repeat."""
    rng = np.random.default_rng(m + n)
    A = rng.uniform(-1, 1, size=(m, n))
    A[:, 1::3] = A[:, 0::3][:, :A[:, 1::3].shape[1]] * 0.5
    k = min(m, n)
    # exact dependence: past a zero pivot R is set by rounding, so check the invariants
    Q, R = T.CudaQRSolver(ctx).SolveThinQR(A)
    assert np.abs(Q.T @ Q - np.eye(k)).max() < 1e-13
    assert np.abs(Q @ R - A).max() < 1e-12
    assert np.allclose(np.triu(R), R)
    assert np.abs(np.diag(R)[1::3]).max() < 1e-12
    # near dependence: the factors are determined, so they match the oracle's
    A[:, 1::3] += 1e-3 * rng.uniform(-1, 1, size=A[:, 1::3].shape)
    Q, R = T.CudaQRSolver(ctx).SolveThinQR(A)
    Qo, Ro = oracle.qr(A)
    np.testing.assert_allclose(R, Ro, atol=1e-10)
    assert np.abs(Q @ R - A).max() < 1e-12


def test_qr_tall_path(T, oracle):
    """The 16-column-panel QR for 512 < m <= 1536 (the S = 1, D = 512 gauge
    shape 1536 x 512 among them): orthonormal Q, Q R = A and the oracle's R,
    ragged last panels and wide matrices included; the LQ of the transposed
    shape goes the same way."""
    c = T.Context(0)
    rng = np.random.default_rng(41)
    shapes = [(1536, 512), (1100, 300), (1300, 1400), (1536, 23), (768, 256), (1024, 512), (600, 700), (513, 40)]
    for m, n in shapes:
        A = rng.uniform(-1, 1, size=(m, n))
        Q, R = T.CudaQRSolver(c).SolveThinQR(A)
        k = min(m, n)
        assert np.abs(Q.T @ Q - np.eye(k)).max() < 1e-13, (m, n)
        assert np.abs(Q @ R - A).max() < 1e-12, (m, n)
        np.testing.assert_allclose(R, oracle.qr(A)[1], atol=1e-11)
    A = rng.uniform(-1, 1, size=(512, 1536))
    Lm, Q2 = T.CudaQRSolver(c).SolveThinLQ(A)
    assert np.abs(Q2 @ Q2.T - np.eye(512)).max() < 1e-13
    assert np.abs(Lm @ Q2 - A).max() < 1e-12


@pytest.mark.parametrize("cond", [1.0, 1e4, 1e8, 1e14])
def test_qr_graded_conditioning(T, ctx, oracle, cond):
    """The gauge shape 512 x 256 with singular values graded over `cond` (the
    spread of a site tensor's Schmidt values): orthonormal Q, Q R = A, and R
    equal to the oracle's up to the rounding that the conditioning amplifies."""
    rng = np.random.default_rng(int(np.log10(cond)) + 5)
    m, n = 512, 256
    U, _ = np.linalg.qr(rng.standard_normal((m, n)))
    V, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = (U * np.logspace(0, -np.log10(cond), n)) @ V.T
    Q, R = T.CudaQRSolver(ctx).SolveThinQR(A)
    assert np.abs(Q.T @ Q - np.eye(n)).max() < 1e-13
    assert np.abs(Q @ R - A).max() < 1e-13
    np.testing.assert_allclose(R, oracle.qr(A)[1], atol=1e-14 * max(1.0, cond ** 0.5), rtol=0)


@pytest.mark.parametrize("env", [{}, {"TN_QR_FORWARD_Q": "0"}, {"TN_NO_PERSISTENT_QR": "1"}])
def test_qr_paths_gauge_shapes(T, oracle, monkeypatch, env):
    """The persistent QR -- Q^T accumulated beside the panels (default) or the
    thin Q formed after them -- and the two-stream look-ahead QR, at the gauge
    shapes of a bulk
    D = 256 site: same R as the oracle, orthonormal Q, and zero-padded columns
    (a grown bond) completed to an orthonormal basis."""
    for k_, v_ in env.items():
        monkeypatch.setenv(k_, v_)
    c = T.Context(0)
    rng = np.random.default_rng(77)
    for m, n in [(512, 256), (512, 512), (256, 512), (480, 200)]:
        A = rng.uniform(-1, 1, size=(m, n))
        Q, R = T.CudaQRSolver(c).SolveThinQR(A)
        k = min(m, n)
        assert np.abs(Q.T @ Q - np.eye(k)).max() < 1e-13
        assert np.abs(Q @ R - A).max() < 1e-12
        np.testing.assert_allclose(R, oracle.qr(A)[1], atol=1e-11)
        Ap = A.copy()
        Ap[:, n // 2 + 3:] = 0.0
        Q, R = T.CudaQRSolver(c).SolveThinQR(Ap)
        assert np.abs(Q.T @ Q - np.eye(k)).max() < 1e-13
        assert np.abs(Q @ R - Ap).max() < 1e-12


@pytest.mark.parametrize("m,n", [(7, 5), (5, 7), (64, 32), (32, 64), (256, 512), (512, 256), (130, 130)])
def test_rq_ql(T, ctx, m, n):
    """SolveThinRQ / SolveThinQL (LapackQRSolver.C:163-274): A = R Q with R upper
    (m <= n) and orthonormal rows of Q; A = Q L with L lower (n <= m) and
    orthonormal columns of Q."""
    rng = np.random.default_rng(3 * m + n)
    A = rng.uniform(-1, 1, size=(m, n))
    k = min(m, n)
    s = T.CudaQRSolver(ctx)
    R, Q = s.SolveThinRQ(A)
    assert np.abs(Q @ Q.T - np.eye(k)).max() < 1e-13
    assert np.abs(R @ Q - A).max() < 1e-12
    if m <= n:
        assert np.allclose(np.triu(R), R)
    Q2, L = s.SolveThinQL(A)
    assert np.abs(Q2.T @ Q2 - np.eye(k)).max() < 1e-13
    assert np.abs(Q2 @ L - A).max() < 1e-12
    if n <= m:
        assert np.allclose(np.tril(L), L)


@pytest.mark.parametrize("kind", ["QR", "LQ", "RQ", "QL"])
def test_rank_revealing(T, ctx, kind):
    """SolveRankRevealingQR / LQ / RQ / QL (LapackQRSolver.C:324-399): four
    columns (rows for the row forms) that depend on the others, placed where
    the factorisation meets them last, leave four zero rows (columns) of the
    triangular factor; those are removed with the matching part of Q and the
    kept factors still give A."""
    rng = np.random.default_rng(11)
    m, n = (40, 24) if kind in ("QR", "QL") else (24, 40)
    A = rng.uniform(-1, 1, size=(m, n))
    M = rng.uniform(-1, 1, size=(4, 4))
    if kind == "QR":
        A[:, -4:] = A[:, :4] @ M
    elif kind == "QL":
        A[:, :4] = A[:, -4:] @ M
    elif kind == "LQ":
        A[-4:, :] = M @ A[:4, :]
    else:
        A[:4, :] = M @ A[-4:, :]
    s = T.CudaQRSolver(ctx)
    F1, F2 = getattr(s, "SolveRankRevealing" + kind)(A, 1e-10)
    k = min(m, n)
    if kind in ("QR", "QL"):
        Q, Tr = F1, F2
        assert Q.shape[1] == Tr.shape[0] == k - 4
        assert np.abs(Q.T @ Q - np.eye(Q.shape[1])).max() < 1e-13
        assert np.abs(Q @ Tr - A).max() < 1e-12
    else:
        Tr, Q = F1, F2
        assert Tr.shape[1] == Q.shape[0] == k - 4
        assert np.abs(Q @ Q.T - np.eye(Q.shape[0])).max() < 1e-13
        assert np.abs(Tr @ Q - A).max() < 1e-12
    # a full-rank matrix keeps everything
    B = rng.uniform(-1, 1, size=(m, n))
    G1, G2 = getattr(s, "SolveRankRevealing" + kind)(B, 1e-10)
    assert (G1.shape[1] if kind in ("QR", "QL") else G2.shape[0]) == k


def test_qr_zero_columns_complete(T, ctx):
    rng = np.random.default_rng(1)
    A = np.zeros((40, 16))
    A[:, :5] = rng.uniform(-1, 1, size=(40, 5))
    Q, R = T.CudaQRSolver(ctx).SolveThinQR(A)
    assert np.abs(Q.T @ Q - np.eye(16)).max() < 1e-13
    assert np.abs(Q @ R - A).max() < 1e-13


@pytest.mark.parametrize("m,n", [(7, 5), (5, 7), (64, 32), (32, 64), (200, 120), (1, 4), (6, 1)])
def test_svd(T, ctx, oracle, m, n):
    rng = np.random.default_rng(m * 7 + n)
    A = rng.uniform(-1, 1, size=(m, n))
    U, s, Vt = T.CudaSVDSolver(ctx).SolveAll(A)
    k = min(m, n)
    tol = 2 * np.sqrt(m * n) * 1e-13
    np.testing.assert_allclose(s, oracle.svd_values(A), atol=tol * s[0])
    np.testing.assert_allclose(s, np.linalg.svd(A, compute_uv=False), atol=tol * s[0])
    assert np.abs(U.T @ U - np.eye(k)).max() < tol
    assert np.abs(Vt @ Vt.T - np.eye(k)).max() < tol
    assert np.abs(U @ np.diag(s) @ Vt - A).max() < tol


def test_svd_rank_deficient(T, ctx):
    rng = np.random.default_rng(5)
    A = np.zeros((24, 12))
    A[:, :3] = rng.uniform(-1, 1, size=(24, 3))
    U, s, Vt = T.CudaSVDSolver(ctx).SolveAll(A)
    assert np.all(s[3:] < 1e-13)
    assert np.abs(U.T @ U - np.eye(12)).max() < 1e-12
    assert np.abs(U @ np.diag(s) @ Vt - A).max() < 1e-12


def test_dense_eigensolver(T, ctx):
    rng = np.random.default_rng(2)
    B = rng.uniform(-1, 1, size=(60, 60))
    A = B + B.T
    U, w = T.CudaEigenSolver(ctx).Solve(A, 1e-12, 2)
    ev = np.linalg.eigvalsh(A)
    np.testing.assert_allclose(w, ev[:2], atol=1e-12 * np.abs(ev).max())
    assert np.linalg.norm(A @ U - U * w) < 1e-10 * np.abs(ev).max()


def test_dense_eigensolver_structured(T, ctx, oracle):
    """LapackEigenSolver::Solve contract (LapackEigenSolver.C:62-109: zheevx,
    RANGE='I', the lowest k pairs ascending) on matrices whose ground state is
    orthogonal to the all-ones vector: the two-site Heisenberg term (singlet
    ground state, ExactDiagTests.C:79-85), the full L = 8 spin-1/2 chain
    Hamiltonian, and a matrix with a prescribed spectrum and eigenvectors."""
    h = oracle.local_h12(0.5, 1.0, 1.0, 0.0)
    U, w = T.CudaEigenSolver(ctx).Solve(h, 1e-13, 4)
    np.testing.assert_allclose(w, [-0.75, 0.25, 0.25, 0.25], atol=1e-14)
    singlet = np.array([0, 1, -1, 0]) / np.sqrt(2)
    assert abs(abs(U[:, 0] @ singlet) - 1) < 1e-13
    # L = 8 chain, 256 x 256: sum of bond terms
    L, dd = 8, 2
    H = np.zeros((dd ** L, dd ** L))
    for b in range(L - 1):
        H += np.kron(np.kron(np.eye(dd ** b), h), np.eye(dd ** (L - b - 2)))
    U, w = T.CudaEigenSolver(ctx).Solve(H, 1e-13, 3)
    ev, evec = np.linalg.eigh(H)
    np.testing.assert_allclose(w, ev[:3], atol=1e-12)
    assert abs(abs(U[:, 0] @ evec[:, 0]) - 1) < 1e-10
    assert abs(U[:, 0].sum()) < 1e-10          # the singlet ground state is orthogonal to the ones vector
    # prescribed spectrum, eigenvectors from a random orthogonal matrix with the lowest one orthogonal to ones
    rng = np.random.default_rng(5)
    n = 40
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    Q[:, 0] = np.r_[1.0, -1.0, np.zeros(n - 2)] / np.sqrt(2)
    Q, _ = np.linalg.qr(Q)
    lam = np.sort(rng.uniform(-3, 3, n))
    A = (Q * lam) @ Q.T
    U, w = T.CudaEigenSolver(ctx).Solve(A, 1e-13, 5)
    np.testing.assert_allclose(w, lam[:5], atol=1e-12)
    assert np.linalg.norm(A @ U - U * w) < 1e-11
    assert np.abs(U.T @ U - np.eye(5)).max() < 1e-12


def test_svd_solve_truncates(T, ctx):
    """SVDSolver::Solve(A, eps, k) (LapackSVDSolver.C:42-90): the k largest triplets."""
    rng = np.random.default_rng(8)
    A = rng.uniform(-1, 1, size=(30, 20))
    U, s, Vt = T.CudaSVDSolver(ctx).Solve(A, 1e-12, 7)
    u0, s0, vt0 = np.linalg.svd(A, full_matrices=False)
    assert U.shape == (30, 7) and s.shape == (7,) and Vt.shape == (7, 20)
    np.testing.assert_allclose(s, s0[:7], rtol=1e-12)
    np.testing.assert_allclose(np.abs(U.T @ u0[:, :7]), np.eye(7), atol=1e-10)
    np.testing.assert_allclose(np.abs(Vt @ vt0[:7].T), np.eye(7), atol=1e-10)


def test_compressor(T, ctx, oracle):
    rng = np.random.default_rng(4)
    A = rng.uniform(-1, 1, size=(12, 10))
    U, s, Vt = oracle.svd(A)
    for Dmax, eps in [(4, 0.0), (0, np.sum(s[7:] ** 2) * 1.0001), (5, 1e-3)]:
        U2, s2, Vt2, err = T.SVCompressor(Dmax, eps, ctx).Compress(U, s, Vt)
        Uo, so, Vto, erro = oracle.compress(U, s, Vt, Dmax, eps)
        np.testing.assert_allclose(s2, so, rtol=1e-14)
        np.testing.assert_allclose(err, erro, rtol=1e-14)
        assert U2.shape == Uo.shape and Vt2.shape == Vto.shape
