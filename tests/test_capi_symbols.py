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
