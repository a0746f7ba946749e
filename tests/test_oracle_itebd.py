"""CPU checks of the iTEBD oracle against the reference's own bounds
(TensorNetworksUnittests/iTEBDTests.C:737-759): the D = 8 imaginary-time
ground state lies between the exact 1/4 - ln 2 and -0.442846 per bond."""
import numpy as np

from oracle import itebd_oracle as I
from oracle import oracle as O

EXACT = 0.25 - np.log(2.0)


def test_gate_is_exp_of_h():
    G = I.gate(0.5, 1.0, 1.0, 0.0, 0.3)
    h = O.local_h12(0.5, 1.0, 1.0, 0.0)
    w, U = np.linalg.eigh(h)
    np.testing.assert_allclose(G, U @ np.diag(np.exp(-0.3 * w)) @ U.T, atol=1e-14)
    np.testing.assert_allclose(I.gate(0.5, 1.0, 1.0, 0.0, 0.0), np.eye(4), atol=1e-14)


def test_compress_rule():
    s = np.array([0.9, 0.4, 1e-4, 1e-5])
    assert I.compress(s, 0, 1e-7)[0] == 2       # discarded 1e-8 + 1e-10 < 1e-7
    assert I.compress(s, 0, 1e-9)[0] == 3       # 1e-10 < 1e-9 <= 1e-8 + 1e-10
    assert I.compress(s, 2, 1e-16)[0] == 2      # Dmax caps
    assert I.compress(s, 3, 0.0)[0] == 3


def test_d8_ground_state_within_reference_bounds():
    h = O.local_h12(0.5, 1.0, 1.0, 0.0)
    E, st, steps = I.find_ground_state(0.5, 8, [0.5, 0.2, 0.1, 0.01, 0.001], 1000)
    Ex = I.expectation(st, h)
    assert EXACT < Ex < -0.442846, Ex
    assert all(x.size == 8 for x in st.l)


def orthonormality_error(st):
    """GetOrthonormalityErrors (iTEBDStateImp_OrthoNorm.C:69-98) at centre 1:
    the norm matrices of gamma = GA lA GB with lambdaB, scaled to unit mean
    diagonal, against the identity (Frobenius)."""
    d = st.d
    gam = np.stack([(st.G[0][na] * st.l[0][None, :]) @ st.G[1][nb] for nb in range(d) for na in range(d)])
    Vr, Vl = I.norm_matrices(gam, st.l[1])
    D = Vr.shape[0]
    err = 0.0
    for V in (Vr, Vl):
        V = V / (np.trace(V) / D)
        err = max(err, np.linalg.norm(V - np.eye(D)))
    return err


def test_orthogonalize_restores_canonical_form():
    """OrthogonalizeI (iTEBDStateImp_OrthoNorm.C:110-128,511-637) on a state
    made non-canonical by truncated gates: afterwards both norm matrices are
    the identity, and the state (its energy) is unchanged up to the iteration
    tolerance."""
    h = O.local_h12(0.5, 1.0, 1.0, 0.0)
    st = I.State(0.5, 12, seed=3)
    gates = [I.gate(0.5, 1, 1, 0, 0.05), I.gate(0.5, 1, 1, 0, 0.1), I.gate(0.5, 1, 1, 0, 0.05)]
    for _ in range(40):
        st.step(gates, 12)
    e0 = I.expectation(st, h)
    before = orthonormality_error(st)
    I.orthogonalize_i(st, 12, 1e-12, 100)
    after = orthonormality_error(st)
    assert before > 1e-6, before
    assert after < 1e-9, after
    assert abs(I.expectation(st, h) - e0) < 1e-8


def test_d32_reference_schedule_bound():
    """iTEBDTests.C:930-955 FindiTimeGSD32S12: Dstart 8, Dmax 32, deltaD 8,
    maxIter 1000, dt 0.5 -> 0.2 -> 0.1 -> 0.01 -> 0.001 -> 0 with dlambda
    epsilon 5e-5 dt (MakeSchedule, :720-733), OrthogonalizeI around every D
    stage; the reference asserts 1/4 - ln 2 < E < -0.443137."""
    E, st, steps = I.find_ground_state_lines(0.5, 8, 32, 8, [0.5, 0.2, 0.1, 0.01, 0.001, 0.0], 1000, seed=12)
    assert EXACT < E < -0.443137, E
    assert st.l[0].size == 32 and st.l[1].size == 32
