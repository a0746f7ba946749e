"""The persistent QR's waits between CTAs are bounded: when a wait runs out the
kernel raises an error word instead of hanging, every other wait gives up, and
the host call reports the failure; the context stays usable.  The limit is
forced down to one poll (TN_QR_SPIN_LIMIT, read when a context is created) in a
child process, so that the first wait that is not already satisfied expires.
No GPU fault is involved."""
import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

@pytest.fixture(scope="module")
def T():
    import tensornetworks_b200 as T
    return T


CHILD = textwrap.dedent("""
    import sys
    import numpy as np
    sys.path.insert(0, {root!r})
    import tensornetworks_b200 as T
    from tensornetworks_b200 import _capi
    lib = _capi.load()
    import ctypes as C
    import torch
    ctx = T.Context(0)
    m, n = 512, 256
    A = torch.rand(m * n, dtype=torch.float64, device="cuda")
    Q = torch.empty(m * n, dtype=torch.float64, device="cuda")
    R = torch.empty(n * n, dtype=torch.float64, device="cuda")
    rc = lib.tn_qr(ctx.handle, m, n, A.data_ptr(), m, Q.data_ptr(), m, R.data_ptr(), n)
    print("RC", rc)
    print("MSG", _capi.last_error())
""")


@pytest.mark.gpu
def test_expired_wait_reports_error_and_context_survives(T):
    env = dict(os.environ, TN_QR_SPIN_LIMIT="1")
    out = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    rc = int(out.stdout.split("RC")[1].split()[0])
    assert rc == 4, out.stdout  # TN_CUDA_ERROR
    assert "bounded wait" in out.stdout
    # a context with the normal limit still factors correctly
    import numpy as np
    rng = np.random.default_rng(5)
    A = rng.uniform(-1, 1, size=(512, 256))
    Qm, Rm = T.CudaQRSolver(T.Context(0)).SolveThinQR(A)
    assert np.abs(Qm @ Rm - A).max() < 1e-12
