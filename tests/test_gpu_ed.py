"""Exact diagonalisation on the device (FullState, FullStateImp.C) against the
reference's ED golden energies and the CPU oracle, through the C ABI.

Goldens (total energy, open S = 1/2 Heisenberg chain, J = Jz = 1):
  L = 10 -> -4.258035207282882   (ExactDiagTests.C:269)
  L = 12 -> -5.1420906328405342  (ExactDiagTests.C:283)
  L = 14 -> -6.0267246618621693  (ExactDiagTests.C:293)
  L = 16 -> -6.9117371455751222  (ExactDiagTests.C:300)
Tolerance: 1e-10 absolute (the Lanczos residual target is 1e-11)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import tensornetworks_b200 as T
    return T


def ham(T, L, S, hz=0.0):
    return T.Factory.GetFactory().Make1D_NN_HeisenbergHamiltonian(L, S, T.RegularLower, 1.0, 1.0, hz)


@pytest.mark.parametrize("L,Eexp", [(10, -4.258035207282882), (12, -5.1420906328405342),
                                    (14, -6.0267246618621693), (16, -6.9117371455751222)])
def test_ed_golden(T, L, Eexp):
    H = ham(T, L, 0.5)
    psi = H.CreateFullState(seed=7)
    assert psi.GetSize() == 2 ** L
    E = psi.FindGroundState(H, 1e-11)
    assert abs(E - Eexp) < 1e-10
    assert abs(psi.GetE() - E) == 0.0


@pytest.mark.parametrize("L,S,hz", [(8, 1.0, 0.0), (9, 1.0, 0.2), (6, 1.5, 0.0), (11, 0.5, 0.3)])
def test_ed_matches_oracle(T, oracle, L, S, hz):
    """Spins 1/2, 1, 3/2 and a field (MPO convention, oracle field_mode 0)."""
    H = ham(T, L, S, hz)
    E = H.CreateFullState(seed=3).FindGroundState(H, 1e-11)
    Eref = oracle.ed_ground(L, S, 1.0, 1.0, hz, field_mode=0)
    assert abs(E - Eref) < 1e-9


def test_ed_matvec_and_ground_vector(T):
    """DoMatVecContraction against a dense H built on the host from the bond
    terms (site 1 the most significant digit), and the ground vector: unit
    norm, H psi = E psi, first amplitude above 0.01 positive."""
    import torch
    L, S = 8, 0.5
    H = ham(T, L, S)
    psi = H.CreateFullState(seed=5)
    h = np.array([[0.25, 0, 0, 0], [0, -0.25, 0.5, 0], [0, 0.5, -0.25, 0], [0, 0, 0, 0.25]])
    Hd = np.zeros((2 ** L, 2 ** L))
    for b in range(L - 1):
        Hd += np.kron(np.kron(np.eye(2 ** b), h), np.eye(2 ** (L - b - 2)))
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, 2 ** L)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    psi.DoMatVecContraction(xd, yd)
    torch.cuda.synchronize()
    np.testing.assert_allclose(yd.cpu().numpy(), Hd @ x, atol=1e-13)
    E = psi.FindGroundState(H, 1e-12)
    a = psi.GetAmplitudes()
    assert abs(np.linalg.norm(a) - 1) < 1e-12
    assert np.linalg.norm(Hd @ a - E * a) < 1e-9
    assert a[np.argmax(np.abs(a) > 0.01)] > 0
    assert abs(E - np.linalg.eigvalsh(Hd)[0]) < 1e-11


def test_ed_power_iterate(T):
    """FullState::PowerIterate (FullStateImp.C:155-188) reaches the Lanczos
    energy on a small chain (|E0| dominates the spectrum)."""
    L = 6
    H = ham(T, L, 0.5)
    psi = H.CreateFullState(seed=9)
    E = psi.PowerIterate(H, 1e-12, 1e-9, 20000)
    E0 = H.CreateFullState(seed=1).FindGroundState(H, 1e-12)
    assert abs(E - E0) < 1e-8


def test_ed_large_chain(T):
    """L = 22 (4.2M amplitudes): a size the CPU oracle no longer reaches in
    seconds; the energy lies between the variational DMRG bound and the
    Bethe-ansatz per-bond limit."""
    L = 22
    H = ham(T, L, 0.5)
    E = H.CreateFullState(seed=2).FindGroundState(H, 1e-10)
    assert (L - 1) * (0.25 - np.log(2)) - 1.0 < E < -9.3
