"""Split-precision (BF16 pieces on tcgen05) Heff matvec and sweep against the FP64 oracle.

Tolerances (normwise relative error of Heff x, random environments):
  MIXED    (2 BF16 pieces, 3 products):  <= 2e-4
  MIXED_HI (3 BF16 pieces, 6 products):  <= 2e-5 (FP32 accumulation and FP32
                                         stage-2 intermediates set this floor)
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {1: 2e-4, 2: 2e-5}


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


@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("d,D1,D2,Dw1,Dw2", [(2, 16, 16, 5, 5), (2, 32, 64, 5, 5), (2, 128, 128, 5, 5),
                                              (2, 256, 256, 5, 5), (3, 48, 32, 5, 5), (2, 64, 64, 5, 1),
                                              (2, 144, 96, 5, 5)])
def test_mixed_matvec_vs_oracle(T, ctx, oracle, precision, d, D1, D2, Dw1, Dw2):
    rng = np.random.default_rng(D1 * 7 + D2 + precision)
    W = oracle.mpo_site(10, (d - 1) / 2, 2, 1.0, 1.0, 0.3, 5 if Dw2 == 5 else 10)
    assert W.shape[:2] == (Dw1, Dw2)
    F = rng.uniform(-1, 1, size=Dw1 * D1 * D1)
    G = rng.uniform(-1, 1, size=Dw2 * D2 * D2)
    x = rng.uniform(-1, 1, size=d * D1 * D2)
    ref = oracle.heff_matvec(W, F, G, x, D1, D2)
    dF, dG, dx = dev(F), dev(G), dev(x)
    y = dev(np.zeros_like(x))
    Wc = np.ascontiguousarray(W.ravel())
    T._capi.check(ctx._lib.tn_heff_matvec(ctx.handle, precision, d, Dw1, Dw2, D1, D2, Wc.ctypes.data,
                                          dF.data_ptr(), dG.data_ptr(), dx.data_ptr(), y.data_ptr()), "mixed matvec")
    out = y.cpu().numpy()
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err <= TOL[precision], err


def test_operator_handle_repeated_apply(T, ctx, oracle):
    """tn_heff_create once, apply many times (the device SparseEigenSolverClient)."""
    d, D1, D2 = 2, 64, 64
    rng = np.random.default_rng(11)
    W = oracle.mpo_site(10, 0.5, 2, 1.0, 1.0, 0.0, 5)
    F = rng.uniform(-1, 1, size=5 * D1 * D1)
    G = rng.uniform(-1, 1, size=5 * D2 * D2)
    dF, dG = dev(F), dev(G)
    Wc = np.ascontiguousarray(W.ravel())
    h = C.c_void_p()
    T._capi.check(ctx._lib.tn_heff_create(ctx.handle, 1, d, 5, 5, D1, D2, Wc.ctypes.data, dF.data_ptr(),
                                          dG.data_ptr(), C.byref(h)), "create")
    assert ctx._lib.tn_heff_size(h) == d * D1 * D2
    for k in range(4):
        x = rng.uniform(-1, 1, size=d * D1 * D2)
        dx = dev(x)
        y = dev(np.zeros_like(x))
        T._capi.check(ctx._lib.tn_heff_apply(h, dx.data_ptr(), y.data_ptr()), "apply")
        ref = oracle.heff_matvec(W, F, G, x, D1, D2)
        assert np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref) <= TOL[1]
    T._capi.check(ctx._lib.tn_heff_destroy(h), "destroy")


def run(T, L, D, precision, sweeps=3, seed=5, **kw):
    f = T.Factory.GetFactory()
    H = f.Make1D_NN_HeisenbergHamiltonian(L, 0.5, T.RegularLower, 1.0, 1.0, 0.0)
    psi = H.CreateMPS(D, 1e-12, 1e-12)
    psi.InitializeWith(T.Random, seed=seed)
    isched = T.IterationSchedule()
    eps = T.Epsilons(1e-12)
    eps.itsEigenSolverEpsilon = 1e-10
    isched.Insert(T.IterationScheduleLine(sweeps, D, 1, eps))
    var = psi.FindVariationalGroundState(H, isched, T.SolverOptions(precision=precision, **kw))
    return psi.GetExpectation(H), var, psi.last_stats


@pytest.mark.parametrize("precision,tol", [(1, 1e-6), (2, 1e-9)])
def test_mixed_sweep_energy_vs_fp64(T, precision, tol):
    """Same seed and schedule: the split-precision sweep reaches the FP64 sweep's
    energy per site (the site energies come from an FP64 Rayleigh quotient)."""
    L, D = 32, 32
    E64, var64, st64 = run(T, L, D, 0, sweeps=4)
    Em, varm, stm = run(T, L, D, precision, sweeps=4)
    print("FP64", E64 / L, var64, st64["matvecs"], "mixed", Em / L, varm, stm["matvecs"], stm["matvecs_fp64"])
    assert abs(Em - E64) / L <= tol
    assert stm["matvecs_fp64"] < stm["matvecs"]


@pytest.mark.parametrize("split", ["1,1", "2,1", "1,2", "1,4", "2,8", "1,8"])
def test_mixed_matvec_every_splitk(T, ctx, oracle, split, monkeypatch):
    """Every split-K pair of the two tcgen05 GEMMs (the cluster reduction over
    1..8 CTAs) gives the same operator: D1 = D2 = 128 against the FP64 oracle."""
    import ctypes as C
    monkeypatch.setenv("TN_CHAIN_SPLITK", split)
    rng = np.random.default_rng(21)
    d, D1, D2 = 2, 128, 128
    W = oracle.mpo_site(10, 0.5, 2, 1.0, 1.0, 0.2, 5)
    F = rng.uniform(-1, 1, size=5 * D1 * D1)
    G = rng.uniform(-1, 1, size=5 * D2 * D2)
    dF, dG = dev(F), dev(G)
    Wc = np.ascontiguousarray(W.ravel())
    for prec, tol in ((1, TOL[1]), (2, TOL[2])):
        h = C.c_void_p()
        T._capi.check(ctx._lib.tn_heff_create(ctx.handle, prec, d, 5, 5, D1, D2, Wc.ctypes.data, dF.data_ptr(),
                                              dG.data_ptr(), C.byref(h)), "create")
        x = rng.uniform(-1, 1, size=d * D1 * D2)
        dx, y = dev(x), dev(np.zeros(d * D1 * D2))
        T._capi.check(ctx._lib.tn_heff_apply(h, dx.data_ptr(), y.data_ptr()), "apply")
        ref = oracle.heff_matvec(W, F, G, x, D1, D2)
        assert np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref) <= tol
        T._capi.check(ctx._lib.tn_heff_destroy(h), "destroy")
