"""Pins the FP64 CPU oracle against the reference's own golden values.

Every expected number below is quoted from the reference's tests, with the
file:line it comes from.  The oracle is the checker of the CUDA path, so these
tests must pass before any GPU parity claim means anything.
"""
import numpy as np
import pytest

E12 = 1e-12


# PyTensorNetworks/test_Unittest1.py:4-45 -- Dstart=2, grow by 1 to Dfinal,
# Epsilons() defaults (1e-12), maxIter=100; |E1-Eexpected| <= 1e-11.
@pytest.mark.parametrize("L,S,Dfinal,Eexp,E2exp", [
    (2, 0.5, 2, -0.750000000000000, 1e-13),
    (2, 1.0, 3, -2.000000000000000, 1e-13),
    (2, 1.5, 4, -3.750000000000000, 1e-13),
    (2, 2.0, 5, -6.000000000000000, 1e-13),
    (2, 2.5, 6, -8.750000000000000, 1e-13),
    (3, 0.5, 2, -0.500000000000000, 1e-13),
    (3, 1.0, 3, -1.500000000000000, 1e-13),
    (3, 1.5, 4, -3.000000000000000, 1e-13),
    (3, 2.0, 5, -5.000000000000000, 2e-13),
    (3, 2.5, 6, -7.500000000000000, 1e-12),
    (4, 0.5, 4, -0.538675134594813, 1e-13),
    (4, 1.0, 9, -1.548583770354863, 1e-13),
    (5, 0.5, 4, -0.481971563329499, 1e-13),
    (6, 0.5, 8, -0.498715426777585, 1e-13),
    (7, 0.5, 8, -0.472706613447776, 1e-13),
    (8, 0.5, 8, -0.482132838467071, 2e-05),
    (10, 0.5, 8, -0.473113399629092, 5e-05),
    (16, 0.5, 8, -0.460770570536169, 5e-04),
])
def test_variational_golden_pytn(oracle, L, S, Dfinal, Eexp, E2exp):
    r = oracle.find_ground_state(L, S, 2, [(100, Dfinal, 1, E12, E12, E12)], eig_mode=0, gauge=0)
    E1 = r["energy"] / (L - 1)
    assert abs(E1 - Eexp) <= 1e-11
    assert r["variance"] < E2exp


# TensorNetworksUnittests/VariationalGroundStateTests.C
@pytest.mark.parametrize("L,S,D,epsE,Eexp,tol,form", [
    (9, 0.5, 2, 1e-9, -0.45317425, 1e-7, 2),            # :137-154 TestSweep_Lower_L9S1D2
    (9, 0.5, 2, 1e-9, -0.45317425, 1e-7, 1),            # :155-176 TestSweep_Upper_L9S1D2
    (9, 0.5, 4, 1e-10, -0.46664265599414939, 1e-7, 2),  # :220-237 TestSweep_Lower_L9S1D4
    (9, 0.5, 4, 1e-10, -0.46664265599414939, 1e-7, 1),  # :238-255 TestSweep_Upper_L9S1D4
    (9, 0.5, 8, 1e-9, -0.46703753, 1e-7, 2),            # :200-218 TestSweep_Lower_L9S1D8
    (9, 2.5, 2, 1e-9, -7.025661, 1e-7, 2),              # :278-294 TestSweep_Lower_L9S5D2
])
def test_variational_golden_gtest(oracle, L, S, D, epsE, Eexp, tol, form):
    r = oracle.find_ground_state(L, S, D, [(100, D, 1, epsE, E12, E12)], form=form, eig_mode=0, gauge=0)
    assert abs(r["energy"] / (L - 1) - Eexp) <= tol
    assert r["total_sweeps"] < 100


def test_variational_growD_L9_D8(oracle):
    # VariationalGroundStateTests.C:180-198: Dstart 2 -> 8, eps_E = 1, dlambda 1e-9.
    r = oracle.find_ground_state(9, 0.5, 2, [(100, 8, 1, 1.0, 1e-9, E12)], eig_mode=1, gauge=1)
    assert abs(r["energy"] / 8 - (-0.46703753899)) <= 1e-10


def test_variational_L2_h2_exact(oracle):
    # VariationalGroundStateTests.C:86-109: L=2 -> E = -0.75, <H^2> = <H>^2 to 1e-14.
    r = oracle.find_ground_state(2, 0.5, 2, [(100, 2, 1, 1e-9, E12, E12)], eig_mode=0, gauge=0)
    assert abs(r["energy"] - (-0.75)) < 1e-7
    assert abs(r["energy2"] - r["energy"] ** 2) < 1e-14


@pytest.mark.parametrize("eig_mode,gauge", [(1, 0), (1, 1), (0, 1)])
def test_modes_agree_L10(oracle, eig_mode, gauge):
    """Lanczos eigensolver and QR gauge reach the same golden as the reference path."""
    r = oracle.find_ground_state(10, 0.5, 2, [(100, 8, 1, E12, E12, E12)], eig_mode=eig_mode, gauge=gauge)
    assert abs(r["energy"] / 9 - (-0.473113399629092)) <= 1e-11


# TensorNetworksUnittests/ExactDiagTests.C:265-284 and test_Unittest1.py:47-70.
@pytest.mark.parametrize("L,S,Eexp,per_bond", [
    (2, 0.5, -0.75, False),
    (2, 2.5, -8.75, False),
    (10, 0.5, -4.258035207282882, False),
    (12, 0.5, -5.1420906328405342, False),
    (8, 0.5, -0.482133228383984, True),
    (12, 0.5, -0.467462784803685, True),
])
def test_exact_diag_golden(oracle, L, S, Eexp, per_bond):
    E = oracle.ed_ground(L, S)
    if per_bond:
        E /= (L - 1)
    assert abs(E - Eexp) <= 2e-11


def test_h12_matrices(oracle):
    # ExactDiagTests.C:79-85 (S=1/2) and the S=1 spectrum of :110-115.
    H = oracle.local_h12(0.5, 1.0, 1.0, 0.0)
    exp = np.array([[0.25, 0, 0, 0], [0, -0.25, 0.5, 0], [0, 0.5, -0.25, 0], [0, 0, 0, 0.25]])
    np.testing.assert_array_equal(H, exp)
    w = np.linalg.eigvalsh(oracle.local_h12(1.0, 1.0, 1.0, 0.0))
    np.testing.assert_allclose(w, [-2, -1, -1, -1, 1, 1, 1, 1, 1], atol=1e-14)
    w = np.linalg.eigvalsh(oracle.local_h12(2.5, 1.0, 1.0, 0.0))
    assert abs(w[0] + 8.75) < 1e-13 and abs(w[-1] - 6.25) < 1e-13


def test_variational_is_above_exact(oracle):
    """Config 1 (L=10, D=8): the variational energy lies above ED by the golden gap."""
    r = oracle.find_ground_state(10, 0.5, 2, [(100, 8, 1, E12, E12, E12)], eig_mode=1, gauge=1)
    Eed = oracle.ed_ground(10, 0.5)
    gap = r["energy"] - Eed
    assert gap > 0
    assert abs(gap - 9 * (-0.473113399629092 + 0.473115023031432)) < 1e-10
