"""Imaginary-time ground states of the finite MPS on the device, following the
reference's ImaginaryTimeTests (TensorNetworksUnittests/ImaginaryTimeTests.C:295-431,
516-546): S=1/2 Heisenberg chains, first and second order Trotter schedules."""
import pytest

import tensornetworks_b200 as tn

pytestmark = pytest.mark.gpu

E_L9 = -0.46664265599414939  # ImaginaryTimeTests.C:430 (L=9, D=4), energy per bond


def _setup(L, D, seed):
    H = tn.Factory().Make1D_NN_HeisenbergHamiltonian(L, 0.5, tn.RegularLower, 1.0, 1.0, 0.0)
    psi = H.CreateMPS(D)
    psi.InitializeWith(tn.Random, seed=seed)
    return H, psi


def _eps(**kw):
    e = tn.Epsilons(1e-12)
    for k, v in kw.items():
        setattr(e, k, v)
    return e


def test_itime_second_order_L2():
    """ImaginaryTimeTests.C:333-366: L=2 D=2, dt 0.5 / 0.1 / 0.05 second order."""
    L, D = 2, 2
    H, psi = _setup(L, D, 11)
    psi.Normalize(tn.DRight)
    s = tn.IterationSchedule()
    s.Insert(tn.IterationScheduleLine(50, D, 1, 0, 0.5, tn.SecondOrder,
                                      _eps(itsDelatNormEpsilon=1e-5, itsMPSCompressEpsilon=0.0,
                                           itsDeltaLambdaEpsilon=1e-5, itsDelatEnergy1Epsilon=1e-5)))
    s.Insert(tn.IterationScheduleLine(500, D, 1, 3, 0.1, tn.SecondOrder,
                                      _eps(itsDelatNormEpsilon=1e-5, itsMPSCompressEpsilon=0.0,
                                           itsDeltaLambdaEpsilon=1e-8, itsDelatEnergy1Epsilon=1e-8)))
    s.Insert(tn.IterationScheduleLine(500, D, 1, 3, 0.05, tn.SecondOrder,
                                      _eps(itsDelatNormEpsilon=1e-5, itsMPSCompressEpsilon=0.0,
                                           itsDeltaLambdaEpsilon=1e-10, itsDelatEnergy1Epsilon=1e-10)))
    var = psi.FindiTimeGroundState(H, s)
    E1 = psi.GetExpectation(H)
    assert abs(E1 / (L - 1) + 0.75) < 1e-9
    E2 = psi.GetExpectationH2(H)
    assert abs(E2 - E1 * E1) < 1e-9
    assert abs(var) < 1e-9


def test_itime_first_order_L2():
    """ImaginaryTimeTests.C:295-331: L=2 D=4, first order down to dt = 0.01."""
    L, D = 2, 4
    H, psi = _setup(L, D, 12)
    psi.Normalize(tn.DLeft)
    psi.Normalize(tn.DRight)
    s = tn.IterationSchedule()
    for nmax, nopt, dt, e in [(50, 0, 0.5, 1e-3), (500, 0, 0.2, 1e-5), (500, 1, 0.1, 1e-6), (500, 2, 0.05, 1e-7),
                              (500, 3, 0.02, 1e-8), (500, 4, 0.01, 1e-9)]:
        s.Insert(tn.IterationScheduleLine(nmax, D, 1, nopt, dt, tn.FirstOrder,
                                          _eps(itsDelatNormEpsilon=1e-5, itsMPSCompressEpsilon=0.0,
                                               itsDeltaLambdaEpsilon=e, itsDelatEnergy1Epsilon=e)))
    psi.FindiTimeGroundState(H, s)
    E1 = psi.GetExpectation(H)
    assert abs(E1 / (L - 1) + 0.75) < 1e-6
    assert abs(psi.GetExpectationH2(H) - E1 * E1) < 1e-6


def test_itime_first_order_L9():
    """ImaginaryTimeTests.C:402-431: L=9 D=4, first order dt 0.5 .. 0.005, five
    optimisation sweeps per step; energy per bond within 2e-6 of the D=4 value."""
    L, D, nmax, nopt = 9, 4, 1000, 5
    H, psi = _setup(L, D, 13)
    psi.Normalize(tn.DLeft)
    psi.Normalize(tn.DRight)
    s = tn.IterationSchedule()
    s.Insert(tn.IterationScheduleLine(nmax, D, 1, nopt, 0.5, tn.FirstOrder,
                                      _eps(itsDelatNormEpsilon=1e-5, itsMPSCompressEpsilon=0.0,
                                           itsDeltaLambdaEpsilon=1e-5, itsDelatEnergy1Epsilon=1e-5)))
    for dt in (0.2, 0.1, 0.05, 0.02, 0.01, 0.005):
        s.Insert(tn.IterationScheduleLine(nmax, D, 1, nopt, dt, tn.FirstOrder,
                                          _eps(itsDelatNormEpsilon=1e-10, itsMPSCompressEpsilon=0.0,
                                               itsDeltaLambdaEpsilon=1e-6, itsDelatEnergy1Epsilon=1e-6)))
    psi.FindiTimeGroundState(H, s)
    E = psi.GetExpectation(H)
    assert abs(E / (L - 1) - E_L9) < 2e-6
    assert all(n >= 1 for n in psi.last_itime_iterations)


def test_itime_second_order_L9():
    """ImaginaryTimeTests.C:516-546: L=9 D=4, second order dt 2.0 .. 0.01; energy
    per bond within 1e-7 of the D=4 value."""
    L, D, nmax, nopt = 9, 4, 100, 5
    H, psi = _setup(L, D, 14)
    psi.Normalize(tn.DRight)
    s = tn.IterationSchedule()
    for dt, e in [(2.0, 1e-5), (0.5, 1e-5), (0.2, 1e-6), (0.1, 1e-6), (0.05, 1e-6), (0.02, 1e-6), (0.01, 1e-6)]:
        s.Insert(tn.IterationScheduleLine(nmax, D, 1, nopt, dt, tn.SecondOrder,
                                          _eps(itsDelatNormEpsilon=1e-5, itsMPSCompressEpsilon=0.0,
                                               itsDeltaLambdaEpsilon=e, itsDelatEnergy1Epsilon=e)))
    psi.FindiTimeGroundState(H, s)
    E = psi.GetExpectation(H)
    assert abs(E / (L - 1) - E_L9) < 1e-7


def test_itime_bad_order_is_an_error():
    H, psi = _setup(4, 2, 15)
    s = tn.IterationSchedule()
    s.Insert(tn.IterationScheduleLine(5, 2, 1, 1, 0.1, 4, _eps()))
    with pytest.raises(RuntimeError):
        psi.FindiTimeGroundState(H, s)
