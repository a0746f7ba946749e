"""Device Davidson (diagonal and learned correction) and the learned
correction's hand-written kernels, against the CPU oracles.

Tolerances: Davidson eigenvalues 1e-9 relative (as Lanczos); MLP gradients
(FP32 accumulation over <= 1000 pairs) 1e-4 of the largest component against
the FP64 numpy oracle; BF16 inference 2e-2 relative against the oracle run with
BF16-rounded weights."""
import ctypes as C

import numpy as np
import pytest

from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import tensornetworks_b200 as T
    return T


@pytest.fixture(scope="module")
def ctx(T):
    return T.default_context()


def dev(x, dtype=np.float64):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=dtype)).cuda()


def physical_envs(oracle, d, D1, D2, site, L=6, hz=0.2, seed=3):
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


@pytest.mark.parametrize("d,D1,D2,site", [(2, 8, 8, 3), (2, 32, 32, 3), (3, 9, 9, 3)])
def test_davidson_heff(T, ctx, oracle, d, D1, D2, site):
    W, A, F, G = physical_envs(oracle, d, D1, D2, site)
    Dw1, Dw2 = W.shape[:2]
    D1, D2 = A.shape[1:]
    H = oracle.heff_dense(W, F, G, D1, D2)
    H = 0.5 * (H + H.T)
    w = np.linalg.eigvalsh(H)
    x0 = oracle.site_flat(A)
    dx, dF, dG = dev(x0), dev(F), dev(G)
    th, res, nmv = C.c_double(), C.c_double(), C.c_int()
    opt = T.SolverOptions(eigensolver=T.DAVIDSON, krylov=16, max_restarts=20).to_c()
    Wc = np.ascontiguousarray(W.ravel())
    st = ctx._lib.tn_eigensolve_heff(ctx.handle, C.byref(opt), d, Dw1, Dw2, D1, D2, Wc.ctypes.data, dF.data_ptr(),
                                     dG.data_ptr(), dx.data_ptr(), 1e-10, C.byref(th), C.byref(res), C.byref(nmv))
    assert st == 0, T._capi.last_error()
    assert abs(th.value - w[0]) < 1e-9 * max(1, abs(w[0]))
    x = dx.cpu().numpy()
    assert abs(np.linalg.norm(x) - 1) < 1e-12
    assert np.linalg.norm(H @ x - th.value * x) < 1e-8 * max(1, abs(w[0]))


def run_sweeps(T, L, D, opts, sweeps=3, seed=5, model=None, recorder=None):
    f = T.Factory.GetFactory()
    H = f.Make1D_NN_HeisenbergHamiltonian(L, 0.5, T.RegularLower, 1.0, 1.0, 0.0)
    psi = H.CreateMPS(D, 1e-12, 1e-12)
    psi.InitializeWith(T.Random, seed=seed)
    if model is not None:
        psi.SetLearnedCorrection(model)
    if recorder is not None:
        psi.SetRecorder(recorder)
    psi.PrepareSweeps(H)
    mv, learned, st = 0, 0, None
    for _ in range(sweeps):
        st = psi.Sweep(H, 1, 1e-10, opts)
        mv += st["matvecs"]
        learned += st["learned_steps"]
    return psi.GetExpectation(H), mv, learned, st


def test_davidson_sweep_matches_lanczos(T):
    L, D = 12, 16
    E_lz, mv_lz, _, _ = run_sweeps(T, L, D, T.SolverOptions(krylov=20))
    E_dv, mv_dv, _, _ = run_sweeps(T, L, D, T.SolverOptions(eigensolver=T.DAVIDSON, krylov=16))
    print("lanczos", E_lz, mv_lz, "davidson", E_dv, mv_dv)
    assert abs(E_lz - E_dv) / L < 1e-10


def test_davidson_mixed_sweep(T):
    """Davidson on the split-precision operator, FP64 Rayleigh quotient at the end."""
    L, D = 24, 32
    E_lz, _, _, _ = run_sweeps(T, L, D, T.SolverOptions(krylov=20), sweeps=4)
    E_dm, mv, _, st = run_sweeps(T, L, D, T.SolverOptions(eigensolver=T.DAVIDSON, krylov=16, precision=T.MIXED_HI),
                                 sweeps=4)
    print("lanczos fp64", E_lz, "davidson mixed_hi", E_dm, mv, st["matvecs_fp64"])
    assert abs(E_lz - E_dm) / L < 1e-9


def test_mlp_gradient_vs_oracle(T, ctx):
    rng = np.random.default_rng(11)
    m = T.LearnedCorrection(seed=3)
    p = m.get_params().astype(np.float64)
    p[M.B1:M.W2] = rng.normal(size=M.H) * 0.1   # non-zero biases exercise every term
    p[M.B2:M.W3] = rng.normal(size=M.H) * 0.1
    p[M.B3] = 0.2
    m.set_params(p.astype(np.float32))
    p32 = m.get_params().astype(np.float64)
    for n in (1, 130, 1000):
        F = rng.normal(size=(n, 4)).astype(np.float32)
        Tt = rng.normal(size=n).astype(np.float32)
        g, loss = m.gradient(dev(F, np.float32), dev(Tt, np.float32))
        lref, gref = M.loss_and_grad(p32, F.astype(np.float64), Tt.astype(np.float64))
        assert abs(loss - lref) <= 1e-5 * max(1.0, lref)
        assert np.abs(g - gref).max() <= 1e-4 * np.abs(gref).max(), np.abs(g - gref).max()


def test_mlp_forward_bf16_vs_oracle(T, ctx):
    rng = np.random.default_rng(12)
    m = T.LearnedCorrection(seed=4)
    p = m.get_params()
    F = rng.normal(size=(777, 4)).astype(np.float32)
    y = m.forward(dev(F, np.float32)).cpu().numpy()
    yref, _ = M.forward(M.bf16_round(p).astype(np.float64), F.astype(np.float64))
    assert np.abs(y - yref).max() <= 2e-2 * max(1.0, np.abs(yref).max())


def test_mlp_training_reduces_loss(T, ctx):
    """Adam on the device fits a smooth per-element map (the diagonal
    correction itself, y = -f1 / f0 on |f0| > 0.5)."""
    rng = np.random.default_rng(13)
    n = 20000
    F = rng.normal(size=(n, 4)).astype(np.float32)
    F[:, 0] = np.sign(F[:, 0]) * (0.5 + np.abs(F[:, 0]))
    Tt = (-F[:, 1] / F[:, 0]).astype(np.float32)
    m = T.LearnedCorrection(seed=5)
    dF, dT = dev(F, np.float32), dev(Tt, np.float32)
    _, l0 = m.gradient(dF, dT)
    m.train(dF, dT, steps=600, batch=2048, lr=3e-3, seed=1)
    _, l2 = m.gradient(dF, dT)
    print("loss", l0, l2)
    assert l2 < 0.1 * l0


def test_learned_correction_gain(T, ctx):
    """Record exact corrections from FP64 diagonal-Davidson sweeps, train the
    MLP on the device, then sweep a different chain with it.  Diagonal Davidson
    is the judge: same energy per site; the printed matvec counts show what the
    learned correction gains (or loses) against diagonal Davidson."""
    L, D = 16, 32
    ds = T.TrainingSet(2_000_000)
    run_sweeps(T, L, D, T.SolverOptions(eigensolver=T.DAVIDSON, krylov=16), sweeps=2, seed=21, recorder=ds)
    assert len(ds) > 10000
    F, Tt = ds.device_arrays()
    assert F.shape[1] == 4 and bool(F.isfinite().all()) and bool(Tt.isfinite().all())
    m = T.LearnedCorrection(seed=9)
    _, l0 = m.gradient(F, Tt)
    m.train(F, Tt, steps=1500, batch=4096, lr=2e-3, seed=3)
    _, l2 = m.gradient(F, Tt)
    assert l2 < l0
    L2 = 20
    E_dg, mv_dg, _, _ = run_sweeps(T, L2, D, T.SolverOptions(eigensolver=T.DAVIDSON, krylov=16), seed=33)
    E_ml, mv_ml, nlearned, st = run_sweeps(T, L2, D, T.SolverOptions(eigensolver=T.DAVIDSON, krylov=16,
                                                                      use_learned=1), seed=33, model=m)
    print(f"training loss {l0:.4g} -> {l2:.4g} on {len(ds)} pairs; matvecs diagonal {mv_dg}, learned {mv_ml} "
          f"(gain x{mv_dg / max(mv_ml, 1):.3f}), learned corrections {nlearned}, stalls->diagonal {st['fallbacks']}")
    assert nlearned > 0
    assert abs(E_ml - E_dg) / L2 < 1e-9
