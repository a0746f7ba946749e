"""Oracle building blocks checked against scipy's LAPACK (the routines the
reference calls: zgesvd/dgesvd, dgeqrf/dorgqr, zheevx/dsyevx) and against the
reference's literal contraction loops.

Tolerances follow LinearAlgebraTests.H:206-217,421-483,677-745
(2*sqrt(N*M)*1e-13 style bounds).
"""
import numpy as np
import pytest
import scipy.linalg as sla


def _rand(seed, *shape):
    return np.random.default_rng(seed).uniform(-1, 1, size=shape)


@pytest.mark.parametrize("m,n", [(7, 5), (5, 7), (32, 16), (16, 48), (1, 6), (6, 1), (64, 64)])
def test_svd_vs_lapack(oracle, m, n):
    A = _rand(m * 100 + n, m, n)
    U, s, Vt = oracle.svd(A)
    k = min(m, n)
    s_ref = sla.svd(A, compute_uv=False, lapack_driver="gesvd")
    tol = 2 * np.sqrt(m * n) * 1e-13
    np.testing.assert_allclose(s, s_ref, atol=tol * s_ref[0])
    assert np.abs(U.T @ U - np.eye(k)).max() < tol
    assert np.abs(Vt @ Vt.T - np.eye(k)).max() < tol
    assert np.abs(U @ np.diag(s) @ Vt - A).max() < tol


def test_svd_rank_deficient_completion(oracle):
    """Zero singular values (the zero-padded bonds of IncreaseBondDimensions)
    must still give orthonormal U and Vt, as zgesvd does."""
    A = np.zeros((12, 6))
    A[:, :2] = _rand(3, 12, 2)
    U, s, Vt = oracle.svd(A)
    assert np.all(s[2:] < 1e-14)
    assert np.abs(U.T @ U - np.eye(6)).max() < 1e-13
    assert np.abs(Vt @ Vt.T - np.eye(6)).max() < 1e-13
    assert np.abs(U @ np.diag(s) @ Vt - A).max() < 1e-13


@pytest.mark.parametrize("m,n", [(9, 4), (4, 9), (40, 40), (30, 12), (1, 1)])
def test_qr_lq(oracle, m, n):
    A = _rand(m + 7 * n, m, n)
    Q, R = oracle.qr(A)
    k = min(m, n)
    assert np.abs(Q.T @ Q - np.eye(k)).max() < 1e-13
    assert np.allclose(np.triu(R), R)
    assert np.abs(Q @ R - A).max() < 1e-13
    Rs = sla.qr(A, mode="r")[0][:k]
    np.testing.assert_allclose(np.abs(np.diag(R)), np.abs(np.diag(Rs)), atol=1e-12)
    Lm, Q2 = oracle.lq(A)
    assert np.abs(Q2 @ Q2.T - np.eye(k)).max() < 1e-13
    assert np.allclose(np.tril(Lm), Lm)
    assert np.abs(Lm @ Q2 - A).max() < 1e-13


def test_qr_zero_column_completion(oracle):
    A = _rand(5, 10, 4)
    A[:, 2] = 0
    Q, R = oracle.qr(A)
    assert np.abs(Q.T @ Q - np.eye(4)).max() < 1e-13
    assert np.abs(Q @ R - A).max() < 1e-13


def test_eigh_and_tridiag(oracle):
    B = _rand(9, 20, 20)
    A = B + B.T
    w, V = oracle.eigh(A)
    np.testing.assert_allclose(w, np.linalg.eigvalsh(A), atol=1e-12)
    a = _rand(1, 15)
    b = _rand(2, 14)
    th, Y = oracle.tridiag_lowest(a, b, 2)
    T = np.diag(a) + np.diag(b, 1) + np.diag(b, -1)
    ev = np.linalg.eigvalsh(T)
    np.testing.assert_allclose(th, ev[:2], atol=1e-13)
    assert np.abs(T @ Y - Y * th).max() < 1e-12


def _random_env_setup(oracle, d=2, D1=6, D2=5, seed=4):
    rng = np.random.default_rng(seed)
    W = oracle.mpo_site(10, (d - 1) / 2, 2, 1.0, 1.0, 0.3, 5)
    Dw1, Dw2 = W.shape[:2]
    A = rng.uniform(-1, 1, size=(d, D1, D2))
    F = rng.uniform(-1, 1, size=Dw1 * D1 * D1)
    G = rng.uniform(-1, 1, size=Dw2 * D2 * D2)
    return W, A, F, G


@pytest.mark.parametrize("d", [2, 3])
def test_env_staged_equals_literal(oracle, d):
    W, A, F, G = _random_env_setup(oracle, d=d)
    np.testing.assert_allclose(oracle.env_left(W, A, F), oracle.env_left(W, A, F, literal=True), atol=1e-12)
    np.testing.assert_allclose(oracle.env_right(W, A, G), oracle.env_right(W, A, G, literal=True), atol=1e-12)


@pytest.mark.parametrize("d", [2, 3])
def test_matvec_equals_dense_heff(oracle, d):
    W, A, F, G = _random_env_setup(oracle, d=d)
    D1, D2 = A.shape[1:]
    H = oracle.heff_dense(W, F, G, D1, D2)
    x = oracle.site_flat(A)
    np.testing.assert_allclose(oracle.heff_matvec(W, F, G, x, D1, D2), H @ x, atol=1e-11)
    np.testing.assert_allclose(oracle.heff_diag(W, F, G, D1, D2), np.diag(H), atol=1e-12)


def physical_envs(oracle, d=2, D=4, L=4, site=2, seed=8, hz=0.2):
    """Environments of a random 4-site chain around `site`: Heff is symmetric."""
    rng = np.random.default_rng(seed)
    S = (d - 1) / 2
    Ws = {i: oracle.mpo_site(L, S, 2, 1.0, 1.0, hz, i) for i in range(1, L + 1)}
    dims = {1: (1, D), L: (D, 1)}
    A = {i: rng.uniform(-1, 1, size=(d,) + dims.get(i, (D, D))) for i in range(1, L + 1)}
    F = np.ones(1)
    for i in range(1, site):
        F = oracle.env_left(Ws[i], A[i], F)
    G = np.ones(1)
    for i in range(L, site, -1):
        G = oracle.env_right(Ws[i], A[i], G)
    return Ws[site], A[site], F, G


def test_lanczos_lowest(oracle):
    W, A, F, G = physical_envs(oracle)
    D1, D2 = A.shape[1:]
    H = oracle.heff_dense(W, F, G, D1, D2)
    assert np.abs(H - H.T).max() < 1e-12
    th, x, res, nmv = oracle.lanczos_heff(W, F, G, np.ones(H.shape[0]), D1, D2, krylov=20, max_restarts=50,
                                          tol=1e-10)
    assert abs(th - np.linalg.eigvalsh(H)[0]) < 1e-9
    assert np.linalg.norm(H @ x - th * x) < 1e-8


def test_compressor_semantics(oracle):
    """SVCompressorImp::Compress (SVCompressorImp.C:19-73): eps==0 -> Dmax;
    else the smallest D with discarded sum s^2 < eps, capped at Dmax; s
    rescaled by the ratio of squares."""
    A = _rand(11, 12, 10)
    U, s, Vt = oracle.svd(A)
    U2, s2, Vt2, err = oracle.compress(U, s, Vt, 4, 0.0)
    assert s2.size == 4 and U2.shape == (12, 4) and Vt2.shape == (4, 10)
    np.testing.assert_allclose(err, np.sum(s[4:] ** 2))
    np.testing.assert_allclose(s2, s[:4] * np.sum(s ** 2) / np.sum(s[:4] ** 2))
    np.testing.assert_allclose(Vt2, Vt[:4])
    eps = np.sum(s[7:] ** 2) * 1.0001
    U3, s3, Vt3, err3 = oracle.compress(U, s, Vt, 0, eps)
    assert s3.size == 7
    np.testing.assert_allclose(err3, np.sum(s[7:] ** 2))
