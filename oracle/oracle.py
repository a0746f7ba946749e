"""ctypes binding of the FP64 CPU oracle (oracle/_build/libtn_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker.  The product package
(tensornetworks_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtn_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class SchedLine(C.Structure):
    _fields_ = [("max_sweeps", C.c_int), ("Dmax", C.c_int), ("deltaD", C.c_int),
                ("eps_energy", C.c_double), ("eps_lambda", C.c_double), ("eps_eigen", C.c_double)]


class Options(C.Structure):
    _fields_ = [("eig_mode", C.c_int), ("gauge", C.c_int), ("krylov", C.c_int),
                ("max_restarts", C.c_int), ("nthreads", C.c_int), ("verbose", C.c_int)]


class Result(C.Structure):
    _fields_ = [("energy", C.c_double), ("energy2", C.c_double), ("variance", C.c_double),
                ("total_sweeps", C.c_int), ("matvecs", C.c_longlong), ("final_D", C.c_int),
                ("last_dE", C.c_double), ("last_dlambda", C.c_double)]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, no GPU needed)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        i, d, ip, ull, ll = C.c_int, C.c_double, C.POINTER(C.c_int), C.c_ulonglong, C.c_longlong
        L.orc_uniform.argtypes = [ull, ll, ll, _dp]
        L.orc_mpo_site.argtypes = [i, d, i, d, d, d, i, _dp]
        L.orc_local_h12.argtypes = [d, d, d, d, _dp]
        for f in ("orc_env_left", "orc_env_right", "orc_env_left_literal", "orc_env_right_literal"):
            getattr(L, f).argtypes = [i, i, i, i, i, _dp, _dp, _dp, _dp]
        L.orc_heff_matvec.argtypes = [i, i, i, i, i, _dp, _dp, _dp, _dp, _dp]
        L.orc_heff_dense.argtypes = [i, i, i, i, i, _dp, _dp, _dp, _dp]
        L.orc_heff_diag.argtypes = [i, i, i, i, i, _dp, _dp, _dp, _dp]
        L.orc_svd.argtypes = [i, i, _dp, _dp, _dp, _dp]
        L.orc_svd_values.argtypes = [i, i, _dp, _dp]
        L.orc_qr.argtypes = [i, i, _dp, _dp, _dp]
        L.orc_lq.argtypes = [i, i, _dp, _dp, _dp]
        L.orc_eigh.argtypes = [i, _dp, _dp, _dp]
        L.orc_tridiag_lowest.argtypes = [i, _dp, _dp, i, _dp, _dp]
        L.orc_lanczos_heff.argtypes = [i, i, i, i, i, _dp, _dp, _dp, _dp, i, i, d,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_compress.argtypes = [i, d, i, i, i, _dp, _dp, _dp, ip]
        L.orc_compress.restype = C.c_double
        L.orc_find_ground_state.argtypes = [i, d, i, d, d, d, i, ull, C.POINTER(SchedLine), i,
                                            C.POINTER(Options), C.POINTER(Result), C.c_void_p]
        L.orc_sweep_sample.argtypes = [i, d, i, d, d, d, C.c_void_p, C.c_void_p, _dp, i, i, i, i, d, i,
                                       C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
        L.orc_ed_ground.argtypes = [i, d, d, d, d, i, d, C.POINTER(C.c_double)]
        L.orc_itebd.argtypes = [d, d, d, d, i, _dp, C.POINTER(C.c_int), i, ull, d, C.POINTER(C.c_double)]
        _lib = L
    return _lib


# ---- numpy-friendly helpers (Fortran-ordered arrays <-> column-major) -------

def _f(a):
    """Column-major buffer of a 2-D array as a flat C-contiguous float64 array."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).T).ravel()


def _unf(buf, r, c):
    return np.asarray(buf, dtype=np.float64).reshape(c, r).T.copy()


def uniform(seed: int, count: int, offset: int = 0) -> np.ndarray:
    out = np.empty(count)
    lib().orc_uniform(seed, offset, count, out)
    return out


def mpo_site(L, S, form, Jxy, Jz, hz, site):
    """W of one site as an array (Dw1, Dw2, d, d)."""
    d = int(round(2 * S + 1))
    Dw1 = 1 if site == 1 else 5
    Dw2 = 1 if site == L else 5
    W = np.empty(Dw1 * Dw2 * d * d)
    assert lib().orc_mpo_site(L, S, form, Jxy, Jz, hz, site, W) == 0
    return W.reshape(Dw1, Dw2, d, d)


def local_h12(S, Jxy, Jz, hz):
    d = int(round(2 * S + 1))
    H = np.empty(d ** 4)
    lib().orc_local_h12(S, Jxy, Jz, hz, H)
    return _unf(H, d * d, d * d)


def env_left(W, A, F, literal=False):
    """W (Dw1,Dw2,d,d); A flat site tensor with dims (d,D1,D2); F (Dw1*D1*D1)."""
    Dw1, Dw2, d, _ = W.shape
    D1, D2 = A.shape[1], A.shape[2]
    out = np.empty(Dw2 * D2 * D2)
    f = lib().orc_env_left_literal if literal else lib().orc_env_left
    f(d, Dw1, Dw2, D1, D2, np.ascontiguousarray(W.ravel()), site_flat(A), np.ascontiguousarray(F), out)
    return out


def env_right(W, A, G, literal=False):
    Dw1, Dw2, d, _ = W.shape
    D1, D2 = A.shape[1], A.shape[2]
    out = np.empty(Dw1 * D1 * D1)
    f = lib().orc_env_right_literal if literal else lib().orc_env_right
    f(d, Dw1, Dw2, D1, D2, np.ascontiguousarray(W.ravel()), site_flat(A), np.ascontiguousarray(G), out)
    return out


def site_flat(A):
    """Site tensor A[n, i1, i2] -> the shared flat layout n*D1*D2 + i2*D1 + i1."""
    return np.ascontiguousarray(np.transpose(A, (0, 2, 1))).ravel()


def site_unflat(x, d, D1, D2):
    return np.transpose(np.asarray(x).reshape(d, D2, D1), (0, 2, 1)).copy()


def heff_matvec(W, F, G, x, D1, D2):
    Dw1, Dw2, d, _ = W.shape
    y = np.empty(d * D1 * D2)
    lib().orc_heff_matvec(d, Dw1, Dw2, D1, D2, np.ascontiguousarray(W.ravel()), np.ascontiguousarray(F),
                          np.ascontiguousarray(G), np.ascontiguousarray(x), y)
    return y


def heff_dense(W, F, G, D1, D2):
    Dw1, Dw2, d, _ = W.shape
    N = d * D1 * D2
    H = np.empty(N * N)
    lib().orc_heff_dense(d, Dw1, Dw2, D1, D2, np.ascontiguousarray(W.ravel()), np.ascontiguousarray(F),
                         np.ascontiguousarray(G), H)
    return _unf(H, N, N)


def heff_diag(W, F, G, D1, D2):
    Dw1, Dw2, d, _ = W.shape
    out = np.empty(d * D1 * D2)
    lib().orc_heff_diag(d, Dw1, Dw2, D1, D2, np.ascontiguousarray(W.ravel()), np.ascontiguousarray(F),
                        np.ascontiguousarray(G), out)
    return out


def svd(A):
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    k = min(m, n)
    U = np.empty(m * k); s = np.empty(k); Vt = np.empty(k * n)
    lib().orc_svd(m, n, _f(A), U, s, Vt)
    return _unf(U, m, k), s, _unf(Vt, k, n)


def svd_values(A):
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    s = np.empty(min(m, n))
    lib().orc_svd_values(m, n, _f(A), s)
    return s


def qr(A):
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    k = min(m, n)
    Q = np.empty(m * k); R = np.empty(k * n)
    lib().orc_qr(m, n, _f(A), Q, R)
    return _unf(Q, m, k), _unf(R, k, n)


def lq(A):
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    k = min(m, n)
    Lm = np.empty(m * k); Q = np.empty(k * n)
    lib().orc_lq(m, n, _f(A), Lm, Q)
    return _unf(Lm, m, k), _unf(Q, k, n)


def eigh(A):
    A = np.asarray(A, dtype=np.float64)
    N = A.shape[0]
    w = np.empty(N); V = np.empty(N * N)
    lib().orc_eigh(N, _f(A), w, V)
    return w, _unf(V, N, N)


def tridiag_lowest(alpha, beta, k):
    alpha = np.ascontiguousarray(alpha, dtype=np.float64)
    beta = np.ascontiguousarray(beta, dtype=np.float64)
    n = alpha.size
    th = np.empty(k); Y = np.empty(k * n)
    assert lib().orc_tridiag_lowest(n, alpha, beta if beta.size else np.zeros(1), k, th, Y) == 0
    return th, Y.reshape(k, n).T.copy()


def lanczos_heff(W, F, G, x0, D1, D2, krylov=20, max_restarts=10, tol=1e-10):
    Dw1, Dw2, d, _ = W.shape
    x = np.ascontiguousarray(x0, dtype=np.float64).copy()
    th = C.c_double(); res = C.c_double()
    nmv = lib().orc_lanczos_heff(d, Dw1, Dw2, D1, D2, np.ascontiguousarray(W.ravel()), np.ascontiguousarray(F),
                                 np.ascontiguousarray(G), x, krylov, max_restarts, tol, C.byref(th), C.byref(res))
    return th.value, x, res.value, nmv


def compress(U, s, Vt, Dmax, eps):
    U = np.asarray(U, dtype=np.float64); s = np.asarray(s, dtype=np.float64).copy()
    Vt = np.asarray(Vt, dtype=np.float64)
    m, k = U.shape
    n = Vt.shape[1]
    Ub = _f(U); Vb = _f(Vt)
    kout = C.c_int()
    err = lib().orc_compress(Dmax, eps, m, n, k, Ub, s, Vb, C.byref(kout))
    D = kout.value
    return _unf(Ub[: m * D], m, D), s[:D], _unf(Vb[: D * n], D, n), err


def find_ground_state(L, S, Dstart, lines, *, form=2, Jxy=1.0, Jz=1.0, hz=0.0, seed=1234,
                      eig_mode=0, gauge=0, krylov=20, max_restarts=10, nthreads=0, verbose=0,
                      want_site_energies=False):
    """lines: list of (max_sweeps, Dmax, deltaD, eps_energy, eps_lambda, eps_eigen)."""
    arr = (SchedLine * len(lines))(*[SchedLine(*ln) for ln in lines])
    opt = Options(eig_mode, gauge, krylov, max_restarts, nthreads, verbose)
    res = Result()
    se = np.zeros(L) if want_site_energies else None
    rc = lib().orc_find_ground_state(L, S, form, Jxy, Jz, hz, Dstart, seed, arr, len(lines), C.byref(opt),
                                     C.byref(res), se.ctypes.data if se is not None else None)
    if rc != 0:
        raise RuntimeError(f"orc_find_ground_state failed rc={rc}")
    out = {f: getattr(res, f) for f, _ in Result._fields_}
    if se is not None:
        out["site_energies"] = se
    return out


def sweep_sample(L, S, sites, first, nsites, *, form=2, Jxy=1.0, Jz=1.0, hz=0.0, krylov=20, max_restarts=10,
                 tol=1e-10, nthreads=0):
    """Time nsites DLeft site updates of the oracle on the given MPS (list of A[n,i1,i2])."""
    D1s = np.array([a.shape[1] for a in sites], dtype=np.int32)
    D2s = np.array([a.shape[2] for a in sites], dtype=np.int32)
    flat = np.concatenate([site_flat(a) for a in sites])
    sec = C.c_double(); nmv = C.c_longlong()
    rc = lib().orc_sweep_sample(L, S, form, Jxy, Jz, hz, D1s.ctypes.data, D2s.ctypes.data, flat, first, nsites,
                                krylov, max_restarts, tol, nthreads, C.byref(sec), C.byref(nmv))
    if rc != 0:
        raise RuntimeError("orc_sweep_sample failed")
    return sec.value, nmv.value


def ed_ground(L, S, Jxy=1.0, Jz=1.0, hz=0.0, field_mode=0, tol=1e-12):
    E = C.c_double()
    rc = lib().orc_ed_ground(L, S, Jxy, Jz, hz, field_mode, tol, C.byref(E))
    if rc != 0:
        raise RuntimeError("ED too large")
    return E.value
