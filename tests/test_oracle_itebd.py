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
