"""One- and two-site reduced density matrices on the device
(MPSImp::CalculateOneSiteDMs / CalculateTwoSiteDMs,
MPSImp_ExpectationsAndDMs.C:59-117) through the C ABI.

Checks, after a converged L = 9, D = 4 search (the reference's
ExpectationsTests.C:101-129 set-up, both MPO forms):
  - every trace is 1 to 1e-14 (the reference's TestOneSiteDMs_*);
  - both against the reduced density matrices of the full wave function
    built on the host from the same site tensors (1e-13);
  - sum over bonds of tr(rho_{i,i+1} h12) equals <H> (1e-12);
  - the state is left-normalised afterwards, as the reference leaves it."""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import tensornetworks_b200 as T
    return T


def converged(T, L, S, D, form):
    f = T.Factory.GetFactory()
    H = f.Make1D_NN_HeisenbergHamiltonian(L, S, form, 1.0, 1.0, 0.0)
    psi = H.CreateMPS(D, 1e-12, 1e-12)
    psi.InitializeWith(T.Random, seed=5)
    sched = T.IterationSchedule()
    eps = T.Epsilons(1e-12)
    eps.itsDelatEnergy1Epsilon = 1e-10
    sched.Insert(T.IterationScheduleLine(100, D, 1, eps))
    psi.FindVariationalGroundState(H, sched, T.SolverOptions())
    return H, psi


def full_state(psi, L):
    """psi[n1, ..., nL] from the site tensors A[n](i1, i2) (site 1 the slowest index)."""
    v = psi.GetSite(1)  # (d, 1, D2)
    state = v[:, 0, :]  # (d, D2)
    for ia in range(2, L + 1):
        A = psi.GetSite(ia)  # (d, D1, D2)
        state = np.einsum("xi,nij->xnj", state, A).reshape(-1, A.shape[2])
    return state[:, 0]


@pytest.mark.parametrize("form", [1, 2])
def test_dms_vs_full_state(T, oracle, form):
    L, S, D = 9, 0.5, 4
    H, psi = converged(T, L, S, D, form)
    d = 2
    E = psi.GetExpectation(H)
    v = full_state(psi, L)
    v = v / np.linalg.norm(v)
    t = v.reshape([d] * L)
    ro1 = psi.CalculateOneSiteDMs()
    for ia in range(1, L + 1):
        assert abs(np.trace(ro1[ia - 1]) - 1.0) < 1e-14
        ax = [k for k in range(L) if k != ia - 1]
        ref = np.tensordot(t, t, axes=(ax, ax))  # rho[m, n]
        np.testing.assert_allclose(ro1[ia - 1], ref, atol=1e-13)
    # CalculateOneSiteDMs left the state left-normalised: sites 1..L-1 are isometries
    for ia in range(1, L):
        A = psi.GetSite(ia)
        M = np.concatenate([A[n] for n in range(d)], axis=0)
        np.testing.assert_allclose(M.T @ M, np.eye(M.shape[1]), atol=1e-12)
    ro2 = psi.CalculateTwoSiteDMs()
    assert len(ro2) == L * (L - 1) // 2
    h12 = oracle.local_h12(S, 1.0, 1.0, 0.0)  # rows (ma d + mb), columns (na d + nb)
    Ebonds = 0.0
    for (ia, ib), r in ro2.items():
        ax = [k for k in range(L) if k not in (ia - 1, ib - 1)]
        ref = np.tensordot(t, t, axes=(ax, ax))  # [m, m2, n, n2]
        np.testing.assert_allclose(r, ref, atol=1e-13)
        assert abs(np.einsum("abab->", r) - 1.0) < 1e-13
        if ib == ia + 1:
            Ebonds += np.einsum("pq,pq->", h12.T, r.reshape(d * d, d * d))
    assert abs(Ebonds - E) < 1e-12
