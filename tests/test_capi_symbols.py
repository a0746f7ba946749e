"""CPU checks of the C-ABI library: it loads without a GPU and exports every
entry point that include/tn_cuda.h declares (with a Python signature)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "tn_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tn_[a-z0-9_]+)\s*\(", src)))


def test_header_parses():
    syms = declared_symbols()
    assert "tn_mps_find_variational_ground_state" in syms
    assert len(syms) >= 30


def test_library_exports_every_declared_symbol():
    import tensornetworks_b200._capi as capi
    lib = capi.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s
        assert s in capi.SIGNATURES, f"{s} has no ctypes signature"


def test_status_strings():
    import tensornetworks_b200._capi as capi
    assert capi.status_string(0) == "TN_OK"
    assert capi.status_string(2) == "TN_BAD_SHAPE"


def test_no_device_is_reported():
    """Without a GPU the context constructor fails loudly (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import tensornetworks_b200 as T
    with pytest.raises(T.TNError):
        T.Context(0)


def test_schedule_objects():
    import tensornetworks_b200 as T
    eps = T.Epsilons()
    assert eps.itsEigenSolverEpsilon == 1e-12
    line = T.IterationScheduleLine(2, 32, 16, eps)
    c = line.to_c()
    assert (c.max_sweeps, c.Dmax, c.deltaD) == (2, 32, 16)
    with pytest.raises(ValueError):
        T.IterationScheduleLine(0, 8, eps)


# entry points whose null-argument call is not an error
NOT_STATUS = {"tn_last_error", "tn_status_string", "tn_launch_count", "tn_mlp_num_params", "tn_heff_size",
              "tn_dataset_size"}

CHILD = r"""
import ctypes as C, json, sys
sys.path.insert(0, {root!r})
import tensornetworks_b200._capi as capi
lib = capi.load()
for name in sorted(capi.SIGNATURES):
    restype, argtypes = capi.SIGNATURES[name]
    args = [0 if a in (C.c_int, C.c_long, C.c_longlong, C.c_uint, C.c_ulonglong, C.c_size_t)
            else 0.0 if a in (C.c_double, C.c_float) else None for a in argtypes]
    print("CALL", name, flush=True)
    r = getattr(lib, name)(*args)
    print("RET", name, json.dumps(r.decode() if isinstance(r, bytes) else r), flush=True)
"""


def test_null_arguments_are_rejected_without_a_device():
    """Every entry point called with null handles, null pointers and zero sizes
    returns an error status (or the documented sentinel) instead of crashing or
    touching a device: the argument checks come first.  One child process makes
    all the calls, so a crash names the entry point that caused it."""
    import subprocess
    import sys
    out = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], capture_output=True, text=True,
                         timeout=300)
    lines = out.stdout.splitlines()
    called = [ln.split()[1] for ln in lines if ln.startswith("CALL ")]
    assert out.returncode == 0, f"crashed in {called[-1] if called else '?'}: {out.stderr[-500:]}"
    rets = {ln.split()[1]: ln.split(" ", 2)[2] for ln in lines if ln.startswith("RET ")}
    import tensornetworks_b200._capi as capi
    assert set(rets) == set(capi.SIGNATURES)
    for name, r in rets.items():
        if name in NOT_STATUS:
            continue
        assert r != "0", f"{name} accepted null arguments"
    assert rets["tn_heff_size"] == "-1" and rets["tn_dataset_size"] == "-1"
