"""Split-precision sweeps against the FP64 oracle (not only against the FP64
GPU path), through the reference-shaped API and the C ABI.

Same seed, fixed bond dimension, Lanczos eigensolver and QR gauge on both
sides, so the two runs follow the same trajectory up to the eigensolver
tolerance; the energies are compared after a fixed number of sweeps.

Tolerances (energy per site, |E_gpu - E_oracle| / L):
  TN_PREC_MIXED_HI (six BF16 products, FP32-level operator): 1e-9
  TN_PREC_MIXED    (three BF16 products, ~2^-16 operator):   1e-6
The mixed path's site energies and the final energy come from FP64 Rayleigh
quotients, so these bounds measure how far the split-precision Krylov
subspace steers the sweep, not the accuracy of the reported numbers.
"""
import pytest

pytestmark = pytest.mark.gpu

TOL = {1: 1e-6, 2: 1e-9}


@pytest.fixture(scope="module")
def T():
    import tensornetworks_b200 as T
    return T


def run_gpu(T, L, S, D, sweeps, precision, seed, hz=0.0):
    f = T.Factory.GetFactory()
    H = f.Make1D_NN_HeisenbergHamiltonian(L, S, T.RegularLower, 1.0, 1.0, hz)
    psi = H.CreateMPS(D, 1e-12, 1e-12)
    psi.InitializeWith(T.Random, seed=seed)
    isched = T.IterationSchedule()
    eps = T.Epsilons(1e-12)
    eps.itsEigenSolverEpsilon = 1e-10
    isched.Insert(T.IterationScheduleLine(sweeps, D, 1, eps))
    var = psi.FindVariationalGroundState(H, isched, T.SolverOptions(precision=precision))
    return psi.GetExpectation(H), var, psi.last_stats


@pytest.mark.parametrize("precision", [2, 1])
def test_mixed_sweep_D128_vs_oracle(T, oracle, precision):
    """L = 20, S = 1/2, D = 128 (sites 7..14 at the full 128 x 2 x 128): two
    sweep pairs on the split-precision tensor-core path against the oracle."""
    L, S, D, sw, seed = 20, 0.5, 128, 2, 77
    E, var, st = run_gpu(T, L, S, D, sw, precision, seed)
    r = oracle.find_ground_state(L, S, D, [(sw, D, 1, 1e-12, 1e-12, 1e-10)], seed=seed, eig_mode=1, gauge=1)
    print("D128", precision, E / L, r["energy"] / L, (E - r["energy"]) / L, st["matvecs"], st["matvecs_fp64"])
    assert abs(E - r["energy"]) / L <= TOL[precision]
    assert st["total_sweeps"] == r["total_sweeps"]
    assert st["matvecs_fp64"] < st["matvecs"]  # the split-precision operator did the Krylov work


def test_mixed_sweep_spin1_vs_oracle(T, oracle):
    """Spin 1 (d = 3), config 3's model at a size the oracle runs in seconds:
    L = 16, D = 32 (bulk sites 4..12 on the split-precision path), 16 sweeps
    on both sides.  The open spin-1 chain has a near-fourfold ground state
    (free spin-1/2 edge states split only by ~exp(-L/6)); a field hz = 0.1
    polarises the edge spins and makes the ground state unique.  Early in the
    optimisation the energy is first-order sensitive to where each site solve
    stops (the state is far from stationary), so the comparison is made after
    16 sweeps, where the trajectories have settled into the same optimum."""
    L, S, D, sw, seed, hz = 16, 1.0, 32, 16, 77, 0.1
    E, var, st = run_gpu(T, L, S, D, sw, 2, seed, hz=hz)
    r = oracle.find_ground_state(L, S, D, [(sw, D, 1, 1e-12, 1e-12, 1e-10)], hz=hz, seed=seed, eig_mode=1, gauge=1)
    print("d3", E / L, r["energy"] / L, (E - r["energy"]) / L, st["matvecs"], st["matvecs_fp64"])
    assert abs(E - r["energy"]) / L <= TOL[2]
    assert st["total_sweeps"] == r["total_sweeps"]
    assert st["matvecs_fp64"] < st["matvecs"]
