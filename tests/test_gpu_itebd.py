"""iTEBD gates path on the device against the CPU oracle (same initial
Gammas and bond values, same gate sequence) and against the reference's
bounds (TensorNetworksUnittests/iTEBDTests.C:737-759).

Tolerances: bond values after a few Trotter steps 1e-10 (FP64 throughout;
the SVD and the contraction order differ); energies 1e-9."""
import numpy as np
import pytest

from oracle import itebd_oracle as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu
EXACT = 0.25 - np.log(2.0)


@pytest.fixture(scope="module")
def T():
    import tensornetworks_b200 as T
    return T


def load(T, st_or, D):
    s = T.iTEBDState(st_or.S, D, seed=1)
    for b in range(2):
        s.SetBond(b, st_or.l[b])
    for site in range(2):
        s.SetSite(site, st_or.G[site])
    return s


@pytest.mark.parametrize("S,D,dt,nsteps", [(0.5, 4, 0.1, 3), (0.5, 8, 0.05, 5), (1.0, 6, 0.1, 3)])
def test_trotter_steps_match_oracle(T, S, D, dt, nsteps):
    ref = I.State(S, D, seed=7)
    dev = load(T, ref, D)
    gates = [I.gate(S, 1, 1, 0, dt / 2), I.gate(S, 1, 1, 0, dt), I.gate(S, 1, 1, 0, dt / 2)]
    for _ in range(nsteps):
        ref.step(gates, D)
        dev.Step(dt, D, 1)
        for b in range(2):
            lb = dev.GetBond(b)
            assert lb.size == ref.l[b].size
            np.testing.assert_allclose(lb, ref.l[b], atol=1e-10)
    h = O.local_h12(S, 1, 1, 0)
    e_ref = I.expectation(ref, h)
    assert abs(dev.GetExpectation() - e_ref) < 1e-9
    # Gammas agree up to the sign of each singular vector
    for site in range(2):
        g, gr = dev.GetSite(site), ref.G[site]
        assert g.shape == gr.shape
        np.testing.assert_allclose(np.abs(g), np.abs(gr), rtol=1e-7, atol=1e-8)


def test_ground_state_d8_within_reference_bounds(T):
    """The D = 8 bound of iTEBDTests.C:737-759 (E < -0.442846, above the
    exact 1/4 - ln 2) with the reference's line driver: D grown from 2 to 8
    by 1 in the first line, OrthogonalizeI around every D stage, dt 0.5 ->
    0.2 -> 0.1 -> 0.01 -> 0.001 -> 0.  The device starts from the oracle's
    initial state and ends at the oracle's energy."""
    dts = [0.5, 0.2, 0.1, 0.01, 0.001, 0.0]
    ref = I.State(0.5, 2, seed=11)
    dev = load(T, ref, 2)
    steps = dev.FindiTimeGroundState(dts, 1000, 8, 5e-5, deltaD=1)
    E = dev.GetExpectation()
    Eref, st, _ = I.find_ground_state_lines(0.5, 2, 8, 1, dts, 1000, seed=11)
    print("iTEBD D=8", E, Eref, steps)
    assert EXACT < E < -0.442846
    assert abs(E - Eref) < 1e-8
    assert dev.GetBond(0).size == 8 and dev.GetBond(1).size == 8


def test_orthogonalize_matches_oracle(T):
    """OrthogonalizeI (iTEBDStateImp_OrthoNorm.C:110-128,511-637) on the
    device and in the oracle from the same non-canonical state: same bond
    values (1e-9) and the same Gammas up to singular-vector signs."""
    S, D = 0.5, 12
    ref = I.State(S, D, seed=3)
    gates = [I.gate(S, 1, 1, 0, 0.05), I.gate(S, 1, 1, 0, 0.1), I.gate(S, 1, 1, 0, 0.05)]
    for _ in range(40):
        ref.step(gates, D)
    dev = load(T, ref, D)
    I.orthogonalize_i(ref, D, 1e-12, 100)
    delta, iters = dev.OrthogonalizeI(D, 1e-12, 100)
    assert delta < 1e-12 and iters < 100
    for b in range(2):
        np.testing.assert_allclose(dev.GetBond(b), ref.l[b], atol=1e-9)
    for site in range(2):
        np.testing.assert_allclose(np.abs(dev.GetSite(site)), np.abs(ref.G[site]), rtol=1e-6, atol=1e-8)
    h = O.local_h12(S, 1, 1, 0)
    assert abs(dev.GetExpectation() - I.expectation(ref, h)) < 1e-9


def test_ground_state_d32_reference_bound(T):
    """iTEBDTests.C:930-955 FindiTimeGSD32S12 as the reference runs it: Dstart
    8 grown to Dmax 32 by 8, maxIter 1000, dt 0.5 -> 0.2 -> 0.1 -> 0.01 ->
    0.001 -> 0 (MakeSchedule, :720-733), with its bound 1/4 - ln 2 < E < -0.443137."""
    st = T.iTEBDState(0.5, 8, seed=12)
    steps = st.FindiTimeGroundState([0.5, 0.2, 0.1, 0.01, 0.001, 0.0], 1000, 32, 5e-5, deltaD=8)
    E = st.GetExpectation()
    print("iTEBD D=32", E, steps)
    assert EXACT < E < -0.443137
    assert st.GetBond(0).size == 32 and st.GetBond(1).size == 32
