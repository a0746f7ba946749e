"""ctypes binding of libtn_cuda.so (the C ABI of include/tn_cuda.h).

The library is built in-tree (tensornetworks_b200/lib/libtn_cuda.so) by
``python -m tensornetworks_b200.build`` or ``__graft_entry__.build()``.  There
is no CPU fallback: if the library is missing or no sm_100 device is visible,
every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtn_cuda.so")

TN_OK, TN_NOT_CONVERGED, TN_BAD_SHAPE, TN_NAN_DETECTED = 0, 1, 2, 3
TN_CUDA_ERROR, TN_BAD_ARG, TN_NO_DEVICE, TN_OUT_OF_MEMORY = 4, 5, 6, 7
TN_FORM_REGULAR_UPPER, TN_FORM_REGULAR_LOWER = 1, 2
TN_PREC_MIXED_HI = 2
TN_DLEFT, TN_DRIGHT = 0, 1
TN_PREC_FP64, TN_PREC_MIXED = 0, 1
TN_EIG_LANCZOS, TN_EIG_DAVIDSON = 0, 1


class TNError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        msg = f"{where} failed: {status_string(status)}"
        err = last_error()
        if err:
            msg += f" ({err})"
        super().__init__(msg)


class SchedLine(C.Structure):
    _fields_ = [("max_sweeps", C.c_int), ("Dmax", C.c_int), ("deltaD", C.c_int),
                ("eps_energy", C.c_double), ("eps_lambda", C.c_double), ("eps_eigen", C.c_double)]


class ITimeLine(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("Dmax", C.c_int), ("max_opt_iter", C.c_int), ("order", C.c_int),
                ("dt", C.c_double), ("eps_energy", C.c_double), ("eps_lambda", C.c_double),
                ("eps_norm", C.c_double), ("eps_mps_compress", C.c_double)]


class SolverOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("eigensolver", C.c_int), ("krylov", C.c_int),
                ("max_restarts", C.c_int), ("use_learned", C.c_int), ("verbose", C.c_int),
                ("mixed_tol", C.c_double), ("refine_tol", C.c_double), ("fp64_tol_rel", C.c_double),
                ("phase_timing", C.c_int)]


class SweepStats(C.Structure):
    _fields_ = [("energy", C.c_double), ("energy2", C.c_double), ("variance", C.c_double),
                ("total_sweeps", C.c_int), ("final_D", C.c_int), ("matvecs", C.c_longlong),
                ("matvecs_fp64", C.c_longlong), ("heff_flop", C.c_double), ("heff_ms", C.c_double),
                ("sweep_ms", C.c_double), ("last_dE", C.c_double), ("last_dlambda", C.c_double),
                ("not_converged", C.c_int), ("fallbacks", C.c_int), ("learned_steps", C.c_longlong),
                ("refine_ms", C.c_double), ("gauge_ms", C.c_double), ("env_ms", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None

# name -> (restype, argtypes); every function declared in include/tn_cuda.h
_V, _I, _D, _ULL = C.c_void_p, C.c_int, C.c_double, C.c_uint64
_PI, _PD, _PV = C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_void_p)
SIGNATURES = {
    "tn_status_string": (C.c_char_p, [_I]),
    "tn_last_error": (C.c_char_p, []),
    "tn_ctx_create": (_I, [_I, _PV]),
    "tn_ctx_destroy": (_I, [_V]),
    "tn_ctx_set_stream": (_I, [_V, _V]),
    "tn_ctx_synchronize": (_I, [_V]),
    "tn_hamiltonian_create_heisenberg": (_I, [_V, _I, _D, _I, _D, _D, _D, _PV]),
    "tn_hamiltonian_destroy": (_I, [_V]),
    "tn_hamiltonian_site_dims": (_I, [_V, _I, _PI, _PI, _PI]),
    "tn_hamiltonian_h2_dims": (_I, [_V, _I, _PI, _PI]),
    "tn_hamiltonian_get_w": (_I, [_V, _I, _V]),
    "tn_mps_create": (_I, [_V, _I, _D, _D, _PV]),
    "tn_mps_destroy": (_I, [_V]),
    "tn_mps_initialize_random": (_I, [_V, _ULL]),
    "tn_mps_get_site_dims": (_I, [_V, _I, _PI, _PI]),
    "tn_mps_get_site": (_I, [_V, _I, _V]),
    "tn_mps_set_site": (_I, [_V, _I, _I, _I, _V]),
    "tn_mps_get_bond": (_I, [_V, _I, _PI, _V]),
    "tn_mps_normalize": (_I, [_V, _I]),
    "tn_mps_get_max_d": (_I, [_V, _PI]),
    "tn_mps_get_expectation": (_I, [_V, _V, _PD]),
    "tn_mps_get_expectation_h2": (_I, [_V, _V, _PD]),
    "tn_mps_find_variational_ground_state": (_I, [_V, _V, C.POINTER(SchedLine), _I,
                                                  C.POINTER(SolverOptions), C.POINTER(SweepStats), _PD]),
    "tn_mps_get_site_energies": (_I, [_V, _V]),
    "tn_mps_sweep": (_I, [_V, _V, _I, _D, C.POINTER(SolverOptions), C.POINTER(SweepStats)]),
    "tn_mps_prepare_sweeps": (_I, [_V, _V]),
    "tn_launch_count": (C.c_ulonglong, []),
    "tn_heff_matvec": (_I, [_V, _I, _I, _I, _I, _I, _I, _V, _V, _V, _V, _V]),
    "tn_heff_matvec_static": (_I, [_V, _I, _I, _I, _I, _I, _V, _V, _V, _V, _V]),
    "tn_itebd_create": (_I, [_V, _D, _D, _D, _D, _I, _ULL, _PV]),
    "tn_itebd_destroy": (_I, [_V]),
    "tn_itebd_get_site": (_I, [_V, _I, _PI, _PI, _V]),
    "tn_itebd_set_site": (_I, [_V, _I, _I, _I, _V]),
    "tn_itebd_get_bond": (_I, [_V, _I, _PI, _V]),
    "tn_itebd_set_bond": (_I, [_V, _I, _I, _V]),
    "tn_itebd_step": (_I, [_V, _D, _I, _I]),
    "tn_itebd_find_ground_state": (_I, [_V, _V, _I, _I, _I, _I, _D, _V]),
    "tn_itebd_orthogonalize": (_I, [_V, _I, _D, _I, _PD, _PI]),
    "tn_mps_find_itime_ground_state": (_I, [_V, _V, _V, _I, _PD, _V]),
    "tn_mps_one_site_dms": (_I, [_V, _V]),
    "tn_mps_two_site_dms": (_I, [_V, _V]),
    "tn_lanczos_probe": (_I, [_V, C.c_longlong, _I, _PD, _PD]),
    "tn_fullstate_create": (_I, [_V, _ULL, _PV]),
    "tn_fullstate_destroy": (_I, [_V]),
    "tn_fullstate_get_size": (C.c_longlong, [_V]),
    "tn_fullstate_find_ground_state": (_I, [_V, _V, _D, _PD, _PI]),
    "tn_fullstate_power_iterate": (_I, [_V, _V, _D, _D, _I, _PD, _PI]),
    "tn_fullstate_get_e": (_I, [_V, _PD]),
    "tn_fullstate_get_amplitudes": (_I, [_V, _V]),
    "tn_fullstate_matvec": (_I, [_V, _V, _V, _V]),
    "tn_itebd_energy": (_I, [_V, _I, _D, _PD]),
    "tn_mlp_create": (_I, [_V, _ULL, _PV]),
    "tn_mlp_destroy": (_I, [_V]),
    "tn_mlp_num_params": (_I, []),
    "tn_mlp_get_params": (_I, [_V, _V]),
    "tn_mlp_set_params": (_I, [_V, _V]),
    "tn_mlp_forward": (_I, [_V, _V, C.c_longlong, _V]),
    "tn_mlp_gradient": (_I, [_V, _V, _V, C.c_longlong, _V, _PD]),
    "tn_mlp_train": (_I, [_V, _V, _V, C.c_longlong, _I, _I, _D, _ULL, _PD]),
    "tn_dataset_create": (_I, [_V, C.c_longlong, _PV]),
    "tn_dataset_destroy": (_I, [_V]),
    "tn_dataset_size": (C.c_longlong, [_V]),
    "tn_dataset_data": (_I, [_V, _PV, _PV]),
    "tn_mps_set_learned_correction": (_I, [_V, _V]),
    "tn_mps_set_recorder": (_I, [_V, _V]),
    "tn_heff_diag": (_I, [_V, _I, _I, _I, _I, _I, _V, _V, _V, _V]),
    "tn_heff_create": (_I, [_V, _I, _I, _I, _I, _I, _I, _V, _V, _V, _PV]),
    "tn_heff_size": (C.c_longlong, [_V]),
    "tn_heff_apply": (_I, [_V, _V, _V]),
    "tn_heff_destroy": (_I, [_V]),
    "tn_env_left": (_I, [_V, _I, _I, _I, _I, _I, _I, _V, _V, _V, _V]),
    "tn_env_right": (_I, [_V, _I, _I, _I, _I, _I, _I, _V, _V, _V, _V]),
    "tn_eigensolve_heff": (_I, [_V, C.POINTER(SolverOptions), _I, _I, _I, _I, _I, _V, _V, _V, _V, _D,
                                _PD, _PD, _PI]),
    "tn_eigensolve_dense": (_I, [_V, _I, _V, _I, _I, _D, _V, _V, _I]),
    "tn_svd": (_I, [_V, _I, _I, _V, _I, _V, _I, _V, _V, _I]),
    "tn_svd_solve": (_I, [_V, _I, _I, _V, _I, _D, _I, _V, _I, _V, _V, _I]),
    "tn_svd_values": (_I, [_V, _I, _I, _V, _I, _V]),
    "tn_qr": (_I, [_V, _I, _I, _V, _I, _V, _I, _V, _I]),
    "tn_rq": (_I, [_V, _I, _I, _V, _I, _V, _I, _V, _I]),
    "tn_ql": (_I, [_V, _I, _I, _V, _I, _V, _I, _V, _I]),
    "tn_qr_rank_revealing": (_I, [_V, _I, _I, _I, _V, _I, _V, _I, _V, _I, _D, _PI]),
    "tn_lq": (_I, [_V, _I, _I, _V, _I, _V, _I, _V, _I]),
    "tn_compress": (_I, [_V, _I, _D, _I, _V, _PI, _PD]),
}


def load():
    """Load libtn_cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m tensornetworks_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(s: int) -> str:
    return load().tn_status_string(s).decode()


def last_error() -> str:
    try:
        return load().tn_last_error().decode()
    except Exception:  # pragma: no cover
        return ""


def check(status: int, where: str, allow=(TN_OK,)):
    if status not in allow:
        raise TNError(status, where)
    return status
