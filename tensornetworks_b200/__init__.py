"""tensornetworks_b200 -- B200-native (sm_100a) variational ground-state sweep
for open 1-D spin chains, with the API surface of JanReimers/TensorNetworks'
Factory -> Hamiltonian -> MPS::FindVariationalGroundState path."""
from ._capi import LIB_PATH, TNError, load  # noqa: F401
from .api import (  # noqa: F401
    DAVIDSON, FP64, LANCZOS, MIXED, MIXED_HI, Context, CudaEigenSolver, CudaQRSolver, CudaSVDSolver, DLeft, DRight,
    Epsilons, Factory, Hamiltonian, IterationSchedule, IterationScheduleLine, LearnedCorrection, MPS, Random,
    FirstOrder, FullState, RegularLower, SecondOrder, RegularUpper, SolverOptions, SVCompressor, TrainingSet, default_context, iTEBDState)
