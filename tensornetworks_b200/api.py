"""Reference-shaped Python API over the C ABI.

Mirrors the public surface of JanReimers/TensorNetworks used by the
variational ground-state path (TensorNetworks/Factory.H, Hamiltonian.H,
MPS.H, IterationSchedule.H, Epsilons.H, SVCompressor.H and the solver
interfaces of NumericalMethods/), with the same names and argument meaning, so
that a script written against PyTensorNetworks reads the same here:

    f = Factory.GetFactory()
    H = f.Make1D_NN_HeisenbergHamiltonian(L, S, Jxy, Jz, hz)
    psi = H.CreateMPS(D, 1e-12, 1e-12)
    psi.InitializeWith(Random)
    isched = IterationSchedule(); isched.Insert(IterationScheduleLine(100, Dfinal, Epsilons()))
    E2 = psi.FindVariationalGroundState(H, isched)
    E1 = psi.GetExpectation(H) / (L - 1)

All arithmetic runs in libtn_cuda.so on the GPU.  Device memory for the solver
classes is handled with torch CUDA tensors (plumbing only).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _capi as capi
from ._capi import check

# Enums (TensorNetworks/Enums.H)
DLeft, DRight = capi.TN_DLEFT, capi.TN_DRIGHT
Product, Random, Neel, Constant = 0, 1, 2, 3
RegularUpper, RegularLower = capi.TN_FORM_REGULAR_UPPER, capi.TN_FORM_REGULAR_LOWER
FP64, MIXED, MIXED_HI = capi.TN_PREC_FP64, capi.TN_PREC_MIXED, capi.TN_PREC_MIXED_HI
LANCZOS, DAVIDSON = capi.TN_EIG_LANCZOS, capi.TN_EIG_DAVIDSON


# ---------------------------------------------------------------------------
# Context
# ---------------------------------------------------------------------------
class Context:
    """One CUDA device + stream (tn_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = capi.load()
        h = C.c_void_p()
        check(self._lib.tn_ctx_create(device, C.byref(h)), "tn_ctx_create")
        self.handle = h
        self.device = device

    def synchronize(self):
        check(self._lib.tn_ctx_synchronize(self.handle), "tn_ctx_synchronize")

    def close(self):
        if getattr(self, "handle", None):
            self._lib.tn_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


# ---------------------------------------------------------------------------
# Schedule (TensorNetworks/Epsilons.H, IterationSchedule.H)
# ---------------------------------------------------------------------------
@dataclass
class Epsilons:
    """Epsilons (Epsilons.H:11-26); every field defaults to default_eps (Epsilons.C:9-19)."""
    default_eps: float = 1e-12
    itsDelatEnergy1Epsilon: float = None
    itsDelatEnergy2Epsilon: float = None
    itsDelatNormEpsilon: float = None
    itsEigenSolverEpsilon: float = None
    itsNormalizationEpsilon: float = None
    itsMPSCompressEpsilon: float = None
    itsMPOCompressEpsilon: float = None
    itsSparseMatrixEpsilon: float = None
    itsDeltaLambdaEpsilon: float = None

    def __post_init__(self):
        for f in self.__dataclass_fields__:
            if f != "default_eps" and getattr(self, f) is None:
                setattr(self, f, self.default_eps)


FirstOrder, SecondOrder = 1, 2  # TrotterOrder (Enums.H:13)


class IterationScheduleLine:
    """IterationScheduleLine (IterationSchedule.H:13-35, IterationSchedule.C:9-100):
    variational forms (maxiter, Dmax, [DeltaD,] eps) and imaginary-time forms
    (maxiter, Dmax, [DeltaD,] dt, order, eps) and
    (maxiter, Dmax, DeltaD, maxOptIter, dt, order, eps)."""

    def __init__(self, maxiter: int, Dmax: int, *args):
        DeltaD, nopt, dt, order = 1, 1, 0.0, FirstOrder
        if len(args) == 1:
            eps = args[0]
        elif len(args) == 2:
            DeltaD, eps = args
        elif len(args) == 3:
            dt, order, eps = args
        elif len(args) == 4:
            DeltaD, dt, order, eps = args
        elif len(args) == 5:
            DeltaD, nopt, dt, order, eps = args
        else:
            raise TypeError("IterationScheduleLine(maxiter, Dmax, [DeltaD, [maxOptIter,]] [dt, order,] eps)")
        if maxiter <= 0 or Dmax <= 0 or DeltaD <= 0:
            raise ValueError("maxiter, Dmax and DeltaD must be positive")
        self.itsMaxGSSweepIterations = int(maxiter)
        self.itsDmax = int(Dmax)
        self.itsDeltaD = int(DeltaD)
        self.itsMaxOptimizeIterations = int(nopt)
        self.itsdt = float(dt)
        self.itsTrotterOrder = int(order)
        self.itsEps = eps

    def to_itime(self) -> capi.ITimeLine:
        e = self.itsEps
        return capi.ITimeLine(self.itsMaxGSSweepIterations, self.itsDmax, self.itsMaxOptimizeIterations,
                              self.itsTrotterOrder, self.itsdt, e.itsDelatEnergy1Epsilon, e.itsDeltaLambdaEpsilon,
                              e.itsDelatNormEpsilon, e.itsMPSCompressEpsilon)

    def to_c(self) -> capi.SchedLine:
        e = self.itsEps
        return capi.SchedLine(self.itsMaxGSSweepIterations, self.itsDmax, self.itsDeltaD,
                              e.itsDelatEnergy1Epsilon, e.itsDeltaLambdaEpsilon, e.itsEigenSolverEpsilon)


class IterationSchedule:
    def __init__(self):
        self.lines: List[IterationScheduleLine] = []

    def Insert(self, line: IterationScheduleLine):
        self.lines.append(line)

    def __len__(self):
        return len(self.lines)


@dataclass
class SolverOptions:
    precision: int = FP64
    eigensolver: int = LANCZOS
    krylov: int = 20
    max_restarts: int = 10
    use_learned: int = 0
    verbose: int = 0
    mixed_tol: float = 0.0
    refine_tol: float = 0.0
    fp64_tol_rel: float = 0.0
    phase_timing: int = 0

    def to_c(self):
        return capi.SolverOptions(self.precision, self.eigensolver, self.krylov, self.max_restarts,
                                  self.use_learned, self.verbose, self.mixed_tol, self.refine_tol,
                                  self.fp64_tol_rel, self.phase_timing)


# ---------------------------------------------------------------------------
# Factory / Hamiltonian / MPS
# ---------------------------------------------------------------------------
class Factory:
    """Factory (TensorNetworks/Factory.H:9-33) for the Heisenberg/XXZ chain."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()

    @staticmethod
    def GetFactory(ctx: Optional[Context] = None) -> "Factory":
        return Factory(ctx)

    def Make1D_NN_HeisenbergHamiltonian(self, L: int, S: float, *args) -> "Hamiltonian":
        """(L, S, MPOForm, Jxy, Jz, hz) as Factory.H:16, or (L, S, Jxy, Jz, hz) as the Python bindings."""
        if len(args) == 4:
            form, Jxy, Jz, hz = args
        elif len(args) == 3:
            form, (Jxy, Jz, hz) = RegularLower, args
        else:
            raise TypeError("Make1D_NN_HeisenbergHamiltonian(L, S, [form,] Jxy, Jz, hz)")
        return Hamiltonian(self.ctx, L, S, form, Jxy, Jz, hz)

    def MakeMPSCompressor(self, Dmax: int, epsSV: float) -> "SVCompressor":
        return SVCompressor(Dmax, epsSV, self.ctx)


class Hamiltonian:
    """HamiltonianImp: the MPO of L sites (Hamiltonian.H:15-41)."""

    def __init__(self, ctx: Context, L, S, form, Jxy, Jz, hz):
        self.ctx = ctx
        self._lib = ctx._lib
        self.L, self.S, self.form = int(L), float(S), int(form)
        self.Jxy, self.Jz, self.hz = float(Jxy), float(Jz), float(hz)
        h = C.c_void_p()
        check(self._lib.tn_hamiltonian_create_heisenberg(ctx.handle, self.L, self.S, self.form, self.Jxy,
                                                         self.Jz, self.hz, C.byref(h)),
              "tn_hamiltonian_create_heisenberg")
        self.handle = h

    def GetL(self):
        return self.L

    def Getd(self):
        return int(round(2 * self.S + 1))

    def GetS(self):
        return self.S

    def GetW(self, site: int) -> np.ndarray:
        """SiteOperator::GetW of a site (1-based) as an array (Dw1, Dw2, d, d)."""
        a, b, d = C.c_int(), C.c_int(), C.c_int()
        check(self._lib.tn_hamiltonian_site_dims(self.handle, site, C.byref(a), C.byref(b), C.byref(d)),
              "tn_hamiltonian_site_dims")
        W = np.empty((a.value, b.value, d.value, d.value))
        check(self._lib.tn_hamiltonian_get_w(self.handle, site, W.ctypes.data), "tn_hamiltonian_get_w")
        return W

    def CreateMPS(self, D: int, normEps: float = 1e-12, epsSV: float = 1e-12) -> "MPS":
        return MPS(self, D, normEps, epsSV)

    def CreateFullState(self, seed: int = 1234) -> "FullState":
        """Hamiltonian::CreateFullState (Hamiltonian.H:28): the d^L wave function on the GPU."""
        return FullState(self, seed)

    def __del__(self):  # pragma: no cover
        try:
            if getattr(self, "handle", None):
                self._lib.tn_hamiltonian_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class MPS:
    """Finite MPS resident on the GPU (TensorNetworks/MPS.H:14-75)."""

    def __init__(self, H: Hamiltonian, D: int, normEps: float, epsSV: float):
        self.H = H
        self._lib = H._lib
        self.L, self.d = H.L, H.Getd()
        h = C.c_void_p()
        check(self._lib.tn_mps_create(H.handle, int(D), normEps, epsSV, C.byref(h)), "tn_mps_create")
        self.handle = h
        self.last_stats: Optional[dict] = None

    def InitializeWith(self, state: int = Random, seed: int = 1234):
        if state != Random:
            raise NotImplementedError("only the Random initial state is provided")
        check(self._lib.tn_mps_initialize_random(self.handle, int(seed)), "tn_mps_initialize_random")

    def Normalize(self, direction: int):
        check(self._lib.tn_mps_normalize(self.handle, int(direction)), "tn_mps_normalize")

    def GetMaxD(self) -> int:
        D = C.c_int()
        check(self._lib.tn_mps_get_max_d(self.handle, C.byref(D)), "tn_mps_get_max_d")
        return D.value

    def GetSite(self, site: int) -> np.ndarray:
        """Site tensor as an array A[n, i1, i2]."""
        D1, D2 = C.c_int(), C.c_int()
        check(self._lib.tn_mps_get_site_dims(self.handle, site, C.byref(D1), C.byref(D2)), "dims")
        buf = np.empty(self.d * D1.value * D2.value)
        check(self._lib.tn_mps_get_site(self.handle, site, buf.ctypes.data), "tn_mps_get_site")
        return np.transpose(buf.reshape(self.d, D2.value, D1.value), (0, 2, 1)).copy()

    def SetSite(self, site: int, A: np.ndarray):
        d, D1, D2 = A.shape
        buf = np.ascontiguousarray(np.transpose(A, (0, 2, 1)), dtype=np.float64).ravel()
        check(self._lib.tn_mps_set_site(self.handle, site, D1, D2, buf.ctypes.data), "tn_mps_set_site")

    def GetBondSVs(self, bond: int) -> np.ndarray:
        D = C.c_int()
        check(self._lib.tn_mps_get_bond(self.handle, bond, C.byref(D), None), "tn_mps_get_bond")
        s = np.empty(D.value)
        check(self._lib.tn_mps_get_bond(self.handle, bond, C.byref(D), s.ctypes.data), "tn_mps_get_bond")
        return s

    def GetExpectation(self, H: Hamiltonian) -> float:
        E = C.c_double()
        check(self._lib.tn_mps_get_expectation(self.handle, H.handle, C.byref(E)), "tn_mps_get_expectation")
        return E.value

    def GetExpectationH2(self, H: Hamiltonian) -> float:
        E = C.c_double()
        check(self._lib.tn_mps_get_expectation_h2(self.handle, H.handle, C.byref(E)), "h2")
        return E.value

    def GetSiteEnergies(self) -> np.ndarray:
        E = np.empty(self.L)
        check(self._lib.tn_mps_get_site_energies(self.handle, E.ctypes.data), "site energies")
        return E

    def FindVariationalGroundState(self, H: Hamiltonian, schedule: IterationSchedule,
                                   options: Optional[SolverOptions] = None) -> float:
        """Returns <H^2>-<H>^2 (MPSImp_Variational.C:16-25); stats in self.last_stats."""
        lines = (capi.SchedLine * len(schedule.lines))(*[ln.to_c() for ln in schedule.lines])
        opt = (options or SolverOptions()).to_c()
        st = capi.SweepStats()
        var = C.c_double()
        check(self._lib.tn_mps_find_variational_ground_state(self.handle, H.handle, lines, len(schedule.lines),
                                                              C.byref(opt), C.byref(st), C.byref(var)),
              "tn_mps_find_variational_ground_state")
        self.last_stats = st.as_dict()
        return var.value

    def PrepareSweeps(self, H: Hamiltonian):
        """Normalize(DRight) + LoadHeffCaches (MPSImp_Variational.C:18-19)."""
        check(self._lib.tn_mps_prepare_sweeps(self.handle, H.handle), "tn_mps_prepare_sweeps")

    def Sweep(self, H: Hamiltonian, nsweeps: int = 1, eps_eigen: float = 1e-10,
              options: Optional[SolverOptions] = None) -> dict:
        """nsweeps pairs of Sweep(DLeft)+Sweep(DRight) at the current D; returns the stats."""
        opt = (options or SolverOptions()).to_c()
        st = capi.SweepStats()
        check(self._lib.tn_mps_sweep(self.handle, H.handle, int(nsweeps), float(eps_eigen), C.byref(opt),
                                     C.byref(st)), "tn_mps_sweep")
        self.last_stats = st.as_dict()
        return self.last_stats

    def FindiTimeGroundState(self, H: Hamiltonian, schedule: IterationSchedule) -> float:
        """MPS::FindiTimeGroundState (MPSImp_iTime.C:18-88): returns <H^2> - <H>^2;
        the iterations of each line are kept in last_itime_iterations."""
        lines = (capi.ITimeLine * len(schedule))(*[ln.to_itime() for ln in schedule.lines])
        var = C.c_double()
        iters = (C.c_int * len(schedule))()
        check(self._lib.tn_mps_find_itime_ground_state(self.handle, H.handle, lines, len(schedule), C.byref(var),
                                                       iters), "tn_mps_find_itime_ground_state")
        self.last_itime_iterations = list(iters)
        return var.value

    def CalculateOneSiteDMs(self) -> np.ndarray:
        """MPS::CalculateOneSiteDMs: (L, d, d), rho[ia-1][m, n] (the state ends left-normalised)."""
        d = self.H.Getd()
        out = np.empty(self.L * d * d)
        check(self._lib.tn_mps_one_site_dms(self.handle, out.ctypes.data), "tn_mps_one_site_dms")
        return out.reshape(self.L, d, d)

    def CalculateTwoSiteDMs(self) -> dict:
        """MPS::CalculateTwoSiteDMs: {(ia, ib): rho (d, d, d, d)} for 1 <= ia < ib <= L,
        indexed rho[m, m2, n, n2] as the reference's Matrix4 (m, n on ia; m2, n2 on ib)."""
        d, L = self.H.Getd(), self.L
        npairs = L * (L - 1) // 2
        out = np.empty(npairs * d ** 4)
        check(self._lib.tn_mps_two_site_dms(self.handle, out.ctypes.data), "tn_mps_two_site_dms")
        out = out.reshape(npairs, d, d, d, d)
        res, k = {}, 0
        for ia in range(1, L):
            for ib in range(ia + 1, L + 1):
                res[(ia, ib)] = out[k]
                k += 1
        return res

    def SetLearnedCorrection(self, model: Optional["LearnedCorrection"]):
        """Attach (None: detach) the learned Davidson correction used when the
        options select eigensolver=DAVIDSON with use_learned=1."""
        self._mlp = model  # keep it alive while attached
        check(self._lib.tn_mps_set_learned_correction(self.handle, model.handle if model is not None else None),
              "tn_mps_set_learned_correction")

    def SetRecorder(self, ds: Optional["TrainingSet"]):
        """Record (feature, exact-correction) pairs in FP64 diagonal-Davidson sweeps."""
        self._rec = ds
        check(self._lib.tn_mps_set_recorder(self.handle, ds.handle if ds is not None else None),
              "tn_mps_set_recorder")

    def __del__(self):  # pragma: no cover
        try:
            if getattr(self, "handle", None):
                self._lib.tn_mps_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


# ---------------------------------------------------------------------------
# FullState (TensorNetworks/FullState.H): exact diagonalisation on the GPU
# ---------------------------------------------------------------------------
class FullState:
    """FullState: all d^L amplitudes of the chain on the device (FullStateImp.C)."""

    def __init__(self, H: Hamiltonian, seed: int = 1234):
        self.H = H
        self._lib = H._lib
        h = C.c_void_p()
        check(self._lib.tn_fullstate_create(H.handle, int(seed), C.byref(h)), "tn_fullstate_create")
        self.handle = h

    def GetSize(self) -> int:
        return int(self._lib.tn_fullstate_get_size(self.handle))

    def GetE(self) -> float:
        E = C.c_double()
        check(self._lib.tn_fullstate_get_e(self.handle, C.byref(E)), "tn_fullstate_get_e")
        return E.value

    def FindGroundState(self, H: Hamiltonian, epsE: float = 1e-10) -> float:
        """Lanczos ground state; returns the energy (the reference returns it via GetE)."""
        E, mv = C.c_double(), C.c_int()
        check(self._lib.tn_fullstate_find_ground_state(self.handle, H.handle, float(epsE), C.byref(E), C.byref(mv)),
              "tn_fullstate_find_ground_state")
        self.last_matvecs = mv.value
        return E.value

    def PowerIterate(self, H: Hamiltonian, epsE: float, epsPsi: float, maxIter: int = 1000) -> float:
        E, it = C.c_double(), C.c_int()
        check(self._lib.tn_fullstate_power_iterate(self.handle, H.handle, float(epsE), float(epsPsi), int(maxIter),
                                                   C.byref(E), C.byref(it)), "tn_fullstate_power_iterate")
        self.last_iterations = it.value
        return E.value

    def GetAmplitudes(self) -> np.ndarray:
        out = np.empty(self.GetSize())
        check(self._lib.tn_fullstate_get_amplitudes(self.handle, out.ctypes.data), "tn_fullstate_get_amplitudes")
        return out

    def DoMatVecContraction(self, x_dev, y_dev):
        """SparseEigenSolverClient face: y = H x on device buffers (torch tensors)."""
        check(self._lib.tn_fullstate_matvec(self.handle, self.H.handle, x_dev.data_ptr(), y_dev.data_ptr()),
              "tn_fullstate_matvec")

    def __del__(self):  # pragma: no cover
        try:
            if getattr(self, "handle", None):
                self._lib.tn_fullstate_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


# ---------------------------------------------------------------------------
# iTEBD (TensorNetworks/iTEBDState.H): infinite chain, two-site unit cell
# ---------------------------------------------------------------------------
class iTEBDState:
    """iTEBDState on the GPU: Gammas and bond values of a two-site unit cell
    (Vidal form); FindiTimeGroundState with second-order Trotter gates."""

    def __init__(self, S: float, D: int, Jxy: float = 1.0, Jz: float = 1.0, hz: float = 0.0, seed: int = 1234,
                 ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self._lib = self.ctx._lib
        self.d = int(round(2 * S + 1))
        h = C.c_void_p()
        check(self._lib.tn_itebd_create(self.ctx.handle, float(S), float(Jxy), float(Jz), float(hz), int(D),
                                        int(seed), C.byref(h)), "tn_itebd_create")
        self.handle = h

    def GetSite(self, site: int) -> np.ndarray:
        """Gamma of site 0 or 1 as (d, Dl, Dr)."""
        Dl, Dr = C.c_int(), C.c_int()
        check(self._lib.tn_itebd_get_site(self.handle, site, C.byref(Dl), C.byref(Dr), None), "tn_itebd_get_site")
        buf = np.empty(self.d * Dl.value * Dr.value)
        check(self._lib.tn_itebd_get_site(self.handle, site, C.byref(Dl), C.byref(Dr), buf.ctypes.data),
              "tn_itebd_get_site")
        return np.transpose(buf.reshape(self.d, Dr.value, Dl.value), (0, 2, 1)).copy()

    def SetSite(self, site: int, G: np.ndarray):
        d, Dl, Dr = G.shape
        buf = np.ascontiguousarray(np.transpose(G, (0, 2, 1)), dtype=np.float64).ravel()
        check(self._lib.tn_itebd_set_site(self.handle, site, Dl, Dr, buf.ctypes.data), "tn_itebd_set_site")

    def GetBond(self, bond: int) -> np.ndarray:
        D = C.c_int()
        check(self._lib.tn_itebd_get_bond(self.handle, bond, C.byref(D), None), "tn_itebd_get_bond")
        out = np.empty(D.value)
        check(self._lib.tn_itebd_get_bond(self.handle, bond, C.byref(D), out.ctypes.data), "tn_itebd_get_bond")
        return out

    def SetBond(self, bond: int, s: np.ndarray):
        s = np.ascontiguousarray(s, dtype=np.float64)
        check(self._lib.tn_itebd_set_bond(self.handle, bond, s.size, s.ctypes.data), "tn_itebd_set_bond")

    def Step(self, dt: float, Dmax: int, nsteps: int = 1):
        check(self._lib.tn_itebd_step(self.handle, float(dt), int(Dmax), int(nsteps)), "tn_itebd_step")

    def FindiTimeGroundState(self, dts, max_iter: int, Dmax: int, eps_factor: float = 5e-5,
                             deltaD: int = 1) -> List[int]:
        """One schedule line per dt (IterationScheduleLine itsdt, itsDmax,
        itsDeltaD; dlambda epsilon eps_factor*dt as iTEBDTests.C MakeSchedule):
        OrthogonalizeI, bond dimension grown to Dmax by deltaD with steps until
        the bond values move by at most eps_factor*dt (or max_iter steps) at
        each D, OrthogonalizeI again.  Returns the Trotter steps per line."""
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        steps = np.zeros(dts.size, dtype=np.int32)
        check(self._lib.tn_itebd_find_ground_state(self.handle, dts.ctypes.data, dts.size, int(max_iter), int(Dmax),
                                                   int(deltaD), float(eps_factor), steps.ctypes.data),
              "tn_itebd_find_ground_state")
        return steps.tolist()

    def OrthogonalizeI(self, Dmax: int, eps: float, max_iter: int = 100):
        """iTEBDStateImp::OrthogonalizeI: returns (last bond-value change, iterations)."""
        delta, iters = C.c_double(), C.c_int()
        check(self._lib.tn_itebd_orthogonalize(self.handle, int(Dmax), float(eps), int(max_iter), C.byref(delta),
                                               C.byref(iters)), "tn_itebd_orthogonalize")
        return delta.value, iters.value

    def GetExpectation(self, max_iters: int = 20000, tol: float = 1e-13) -> float:
        """Energy per bond of the infinite chain."""
        E = C.c_double()
        check(self._lib.tn_itebd_energy(self.handle, int(max_iters), float(tol), C.byref(E)), "tn_itebd_energy")
        return E.value

    def __del__(self):  # pragma: no cover
        try:
            if getattr(self, "handle", None):
                self._lib.tn_itebd_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Learned Davidson correction (no reference counterpart)
# ---------------------------------------------------------------------------
class _DevArray:
    """__cuda_array_interface__ view of library-owned device memory (float32)."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (ptr, False),
                                         "version": 3, "strides": None}


class TrainingSet:
    """Device buffer of (features[4], target) pairs filled by FP64 diagonal-Davidson sweeps."""

    def __init__(self, capacity: int, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self._lib = self.ctx._lib
        h = C.c_void_p()
        check(self._lib.tn_dataset_create(self.ctx.handle, int(capacity), C.byref(h)), "tn_dataset_create")
        self.handle = h

    def __len__(self):
        return int(self._lib.tn_dataset_size(self.handle))

    def device_arrays(self):
        """(features, targets) as torch CUDA tensors viewing the library's buffers."""
        torch = _torch()
        fp, tp = C.c_void_p(), C.c_void_p()
        check(self._lib.tn_dataset_data(self.handle, C.byref(fp), C.byref(tp)), "tn_dataset_data")
        n = len(self)
        F = torch.as_tensor(_DevArray(fp.value or 0, (n, 4)), device="cuda")
        T = torch.as_tensor(_DevArray(tp.value or 0, (n,)), device="cuda")
        return F, T

    def __del__(self):  # pragma: no cover
        try:
            if getattr(self, "handle", None):
                self._lib.tn_dataset_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class LearnedCorrection:
    """Per-element MLP (4 -> 64 -> 64 -> 1, tanh) for the Davidson correction;
    BF16 weights for inference, FP32 master copy trained with Adam on the GPU."""

    def __init__(self, seed: int = 1, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self._lib = self.ctx._lib
        h = C.c_void_p()
        check(self._lib.tn_mlp_create(self.ctx.handle, int(seed), C.byref(h)), "tn_mlp_create")
        self.handle = h
        self.n_params = int(self._lib.tn_mlp_num_params())

    def get_params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        check(self._lib.tn_mlp_get_params(self.handle, out.ctypes.data), "tn_mlp_get_params")
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        check(self._lib.tn_mlp_set_params(self.handle, p.ctypes.data), "tn_mlp_set_params")

    def forward(self, F):
        """F: (n, 4) float32 CUDA tensor -> (n,) outputs (BF16 weights)."""
        torch = _torch()
        F = F.contiguous()
        Y = torch.empty(F.shape[0], dtype=torch.float32, device=F.device)
        check(self._lib.tn_mlp_forward(self.handle, F.data_ptr(), int(F.shape[0]), Y.data_ptr()), "tn_mlp_forward")
        return Y

    def gradient(self, F, T):
        """Gradient of mean((MLP(F) - T)^2) w.r.t. the FP32 parameters, and the loss."""
        F, T = F.contiguous(), T.contiguous()
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_double()
        check(self._lib.tn_mlp_gradient(self.handle, F.data_ptr(), T.data_ptr(), int(F.shape[0]), g.ctypes.data,
                                        C.byref(loss)), "tn_mlp_gradient")
        return g, loss.value

    def train(self, F, T, steps: int = 2000, batch: int = 4096, lr: float = 2e-3, seed: int = 7) -> float:
        F, T = F.contiguous(), T.contiguous()
        loss = C.c_double()
        check(self._lib.tn_mlp_train(self.handle, F.data_ptr(), T.data_ptr(), int(F.shape[0]), int(steps),
                                     int(batch), float(lr), int(seed), C.byref(loss)), "tn_mlp_train")
        return loss.value

    def __del__(self):  # pragma: no cover
        try:
            if getattr(self, "handle", None):
                self._lib.tn_mlp_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Solver interfaces (NumericalMethods/*.H) on the GPU
# ---------------------------------------------------------------------------
def _torch():
    import torch
    return torch


def _dev(a: np.ndarray):
    """Column-major device copy of a 2-D host array (torch tensor, returned with its shape)."""
    torch = _torch()
    a = np.asarray(a, dtype=np.float64)
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def _host(t, rows, cols):
    return t.cpu().numpy().reshape(cols, rows).T.copy()


class CudaSVDSolver:
    """SVDSolver<double> (SVDSolver.H:11-23): one-sided Jacobi on the GPU."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()

    def SolveAll(self, A, eps: float = 1e-13):
        torch = _torch()
        m, n = np.shape(A)
        k = min(m, n)
        dA = _dev(A)
        U = torch.empty(m * k, dtype=torch.float64, device="cuda")
        s = torch.empty(k, dtype=torch.float64, device="cuda")
        Vt = torch.empty(k * n, dtype=torch.float64, device="cuda")
        check(self.ctx._lib.tn_svd(self.ctx.handle, m, n, dA.data_ptr(), m, U.data_ptr(), m, s.data_ptr(),
                                   Vt.data_ptr(), k), "tn_svd")
        return _host(U, m, k), s.cpu().numpy(), _host(Vt, k, n)

    def Solve(self, A, eps: float, NumSingularValues: int):
        """The NumSingularValues largest triplets (tn_svd_solve)."""
        torch = _torch()
        m, n = np.shape(A)
        k = int(NumSingularValues)
        dA = _dev(A)
        U = torch.empty(m * k, dtype=torch.float64, device="cuda")
        s = torch.empty(k, dtype=torch.float64, device="cuda")
        Vt = torch.empty(k * n, dtype=torch.float64, device="cuda")
        check(self.ctx._lib.tn_svd_solve(self.ctx.handle, m, n, dA.data_ptr(), m, float(eps), k, U.data_ptr(), m,
                                         s.data_ptr(), Vt.data_ptr(), k), "tn_svd_solve")
        return _host(U, m, k), s.cpu().numpy(), _host(Vt, k, n)


class CudaQRSolver:
    """QRSolver<double> (QRSolver.H:10-56): Householder on the GPU."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()

    def SolveThinQR(self, A):
        torch = _torch()
        m, n = np.shape(A)
        k = min(m, n)
        dA = _dev(A)
        Q = torch.empty(m * k, dtype=torch.float64, device="cuda")
        R = torch.empty(k * n, dtype=torch.float64, device="cuda")
        check(self.ctx._lib.tn_qr(self.ctx.handle, m, n, dA.data_ptr(), m, Q.data_ptr(), m, R.data_ptr(), k),
              "tn_qr")
        return _host(Q, m, k), _host(R, k, n)

    def SolveThinLQ(self, A):
        torch = _torch()
        m, n = np.shape(A)
        k = min(m, n)
        dA = _dev(A)
        Lm = torch.empty(m * k, dtype=torch.float64, device="cuda")
        Q = torch.empty(k * n, dtype=torch.float64, device="cuda")
        check(self.ctx._lib.tn_lq(self.ctx.handle, m, n, dA.data_ptr(), m, Lm.data_ptr(), m, Q.data_ptr(), k),
              "tn_lq")
        return _host(Lm, m, k), _host(Q, k, n)

    def SolveThinRQ(self, A):
        """A = R Q (LapackQRSolver.C:163-226): R m x k, Q k x n."""
        torch = _torch()
        m, n = np.shape(A)
        k = min(m, n)
        dA = _dev(A)
        R = torch.empty(m * k, dtype=torch.float64, device="cuda")
        Q = torch.empty(k * n, dtype=torch.float64, device="cuda")
        check(self.ctx._lib.tn_rq(self.ctx.handle, m, n, dA.data_ptr(), m, R.data_ptr(), m, Q.data_ptr(), k),
              "tn_rq")
        return _host(R, m, k), _host(Q, k, n)

    def SolveThinQL(self, A):
        """A = Q L (LapackQRSolver.C:229-274): Q m x k, L k x n."""
        torch = _torch()
        m, n = np.shape(A)
        k = min(m, n)
        dA = _dev(A)
        Q = torch.empty(m * k, dtype=torch.float64, device="cuda")
        Lm = torch.empty(k * n, dtype=torch.float64, device="cuda")
        check(self.ctx._lib.tn_ql(self.ctx.handle, m, n, dA.data_ptr(), m, Q.data_ptr(), m, Lm.data_ptr(), k),
              "tn_ql")
        return _host(Q, m, k), _host(Lm, k, n)

    def _rank_revealing(self, kind, A, eps):
        torch = _torch()
        m, n = np.shape(A)
        k = min(m, n)
        dA = _dev(A)
        F1 = torch.empty(m * k, dtype=torch.float64, device="cuda")
        F2 = torch.empty(k * n, dtype=torch.float64, device="cuda")
        r = C.c_int(0)
        check(self.ctx._lib.tn_qr_rank_revealing(self.ctx.handle, kind, m, n, dA.data_ptr(), m, F1.data_ptr(), m,
                                                 F2.data_ptr(), k, float(eps), C.byref(r)), "tn_qr_rank_revealing")
        rank = r.value
        f1 = F1[: m * rank].cpu().numpy().reshape((rank, m)).T
        f2 = F2.cpu().numpy()[: k * n].reshape((n, k)).T[:rank, :]
        return f1, f2

    def SolveRankRevealingQR(self, A, eps: float):
        """(Q, R) with the zero rows of R and matching columns of Q removed (LapackQRSolver.C:367-373)."""
        return self._rank_revealing(0, A, eps)

    def SolveRankRevealingLQ(self, A, eps: float):
        """(L, Q) with the zero columns of L and matching rows of Q removed (LapackQRSolver.C:393-399)."""
        return self._rank_revealing(1, A, eps)

    def SolveRankRevealingRQ(self, A, eps: float):
        """(R, Q) with the zero columns of R and matching rows of Q removed (LapackQRSolver.C:374-380)."""
        return self._rank_revealing(2, A, eps)

    def SolveRankRevealingQL(self, A, eps: float):
        """(Q, L) with the zero rows of L and matching columns of Q removed (LapackQRSolver.C:384-390)."""
        return self._rank_revealing(3, A, eps)


class CudaEigenSolver:
    """EigenSolver<double>::Solve (EigenSolver.H:31): lowest eigenpairs of a dense symmetric matrix."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()

    def Reset(self):
        pass

    def Solve(self, A, eps: float, NumEigenValues: int):
        torch = _torch()
        N = np.shape(A)[0]
        k = int(NumEigenValues)
        dA = _dev(A)
        U = torch.empty(N * k, dtype=torch.float64, device="cuda")
        w = np.empty(k)
        check(self.ctx._lib.tn_eigensolve_dense(self.ctx.handle, N, dA.data_ptr(), N, k, max(eps, 1e-13),
                                                w.ctypes.data, U.data_ptr(), N), "tn_eigensolve_dense")
        return _host(U, N, k), w


class SVCompressor:
    """SVCompressor<double> (SVCompressor.H:10-24, SVCompressorImp.C:19-73)."""

    def __init__(self, Dmax: int, eps: float, ctx: Optional[Context] = None):
        self.Dmax, self.eps = int(Dmax), float(eps)
        self.ctx = ctx or default_context()

    def GetDmax(self):
        return self.Dmax

    def Donly(self):
        return self.eps == 0.0

    def Compress(self, U, s, Vt):
        """Returns (U, s, Vt, discarded sum s^2) truncated as the reference does."""
        torch = _torch()
        ds = torch.from_numpy(np.ascontiguousarray(s, dtype=np.float64)).cuda()
        D = C.c_int()
        disc = C.c_double()
        check(self.ctx._lib.tn_compress(self.ctx.handle, self.Dmax, self.eps, ds.numel(), ds.data_ptr(),
                                        C.byref(D), C.byref(disc)), "tn_compress")
        D = D.value
        s2 = ds.cpu().numpy()[:D]
        return np.asarray(U)[:, :D], s2, np.asarray(Vt)[:D, :], disc.value
